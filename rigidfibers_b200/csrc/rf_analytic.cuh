// Closed-form inner integral of the slender-body kernel along a straight fiber.
#pragma once
#include "rf_common.cuh"

namespace rf {

// Closed-form inner integral over fiber j (fortran/compute_inner_integral_
// analytically.incl:1-338, src/kernels/compute_inner_integral_analytically.cu)
// for one outer point: R0 = x_i + s t_i - x_j, R(s) = R0 - s t_j.
// I1(n), I3(n), I5(n) (1-based) = int_{-1}^{1} s^{n-1} |R(s)|^{-1,-3,-5} ds,
// forward recursion when |R0|^2 < 10, backward from n = 27 otherwise, the
// degenerate closed forms when |R0 x t_j|^2 < 1e-7; then for every Legendre
// degree f = 0..M the seven weighted moments L01..L25 and the six entries
// of G_f = int P_f(s) K(R(s)) ds.  All in FP64: the REAL*4 evaluation of
// these formulas loses ~1e-3 to cancellation.
template <int M>
__device__ void analytic_G(const double R0[3], const double tj[3], double e2, float (&G)[6][M + 1]) {
  constexpr int NI = M + 4;   // 1-based up to M+3
  double I1[NI], I3[NI], I5[NI];
#pragma unroll
  for (int n = 0; n < NI; ++n) I1[n] = I3[n] = I5[n] = 0.0;
  const double b = -2.0 * (R0[0] * tj[0] + R0[1] * tj[1] + R0[2] * tj[2]);
  const double l = R0[0] * R0[0] + R0[1] * R0[1] + R0[2] * R0[2];
  const double invL = 1.0 / l;
  const double m = l - 0.25 * b * b;
  const double uu = sqrt(1.0 + b + l), ul = sqrt(1.0 - b + l);
  const bool degen = m < 1e-7;
  const double au = 2.0 + b, al = -2.0 + b;
  I1[1] = log(fabs(au + 2.0 * uu)) - log(fabs(al + 2.0 * ul));
  I1[2] = uu - ul + (-b / 2.0) * I1[1];
  I3[1] = degen ? (-2.0 / (au * au)) - (-2.0 / (al * al)) : (au / (2.0 * m * uu)) - (al / (2.0 * m * ul));
  I3[2] = (-1.0 / uu) - (-1.0 / ul) - b / 2.0 * I3[1];
  I5[1] = degen ? (-4.0 / (au * au * au * au)) - (-4.0 / (al * al * al * al))
                : (au / (6.0 * m * uu * uu * uu)) - (al / (6.0 * m * ul * ul * ul)) + (2.0 / (3.0 * m)) * I3[1];
  I5[2] = degen ? (-8.0 / (3.0 * au * au * au)) - (-8.0 / (3.0 * al * al * al)) - (b / 2.0) * I5[1]
                : (-(b + 2.0 * l) / (6.0 * m * uu * uu * uu)) - (-(-b + 2.0 * l) / (6.0 * m * ul * ul * ul)) -
                      (b / (3.0 * m)) * I3[1];
  if (l < 10.0) {
    double psu = 1.0, psl = -1.0;
#pragma unroll
    for (int n = 2; n <= M + 2; ++n) {
      I1[n + 1] = (psu * uu) / n - (psl * ul) / n + ((1.0 - 2.0 * n) * b) / (2.0 * n) * I1[n] -
                  ((double)(n - 1) * l) / n * I1[n - 1];
      I3[n + 1] = I1[n - 1] - b * I3[n] - l * I3[n - 1];
      I5[n + 1] = I3[n - 1] - b * I5[n] - l * I5[n - 1];
      psl = -psl;   // s_lower^(n) with s_lower = -1; s_upper^n = 1
    }
  } else {
    double i1n2 = 0, i1n1 = 0, i3n2 = 0, i3n1 = 0, i5n2 = 0, i5n1 = 0;
    for (int n = 27; n >= 2; --n) {
      const double np2 = n + 2.0, np1 = n + 1.0;
      const double sln = ((n + 1) & 1) ? -1.0 : 1.0;   // (-1)^(n+1)
      const double i1n0 = np2 / (np1 * l) * ((uu / np2) - ((sln * ul) / np2) +
                                              ((1.0 - 2.0 * np2) / (2.0 * np2)) * b * i1n1 - i1n2);
      const double i3n0 = invL * (i1n0 - b * i3n1 - i3n2);
      const double i5n0 = invL * (i3n0 - b * i5n1 - i5n2);
      if (n < M + 3) {
#pragma unroll
        for (int q = 3; q < NI; ++q)
          if (q == n + 1) { I1[q] = i1n0; I3[q] = i3n0; I5[q] = i5n0; }
      }
      i1n2 = i1n1; i1n1 = i1n0;
      i3n2 = i3n1; i3n1 = i3n0;
      i5n2 = i5n1; i5n1 = i5n0;
    }
  }
  // P_f monomial coefficients: P_f = s * sum_p cf[p] s^(f-2p)
#pragma unroll
  for (int f = 0; f <= M; ++f) {
    double sc = 1.0, c0 = 1.0, c1 = 0.0, c2 = 0.0, c3 = 0.0, c4 = 0.0;
    int nc = 1;
    switch (f) {
      case 2: sc = 0.5; c0 = 3; c1 = -1; nc = 2; break;
      case 3: sc = 0.5; c0 = 5; c1 = -3; nc = 2; break;
      case 4: sc = 0.125; c0 = 35; c1 = -30; c2 = 3; nc = 3; break;
      case 5: sc = 0.125; c0 = 63; c1 = -70; c2 = 15; nc = 3; break;
      case 6: sc = 0.0625; c0 = 231; c1 = -315; c2 = 105; c3 = -5; nc = 4; break;
      case 7: sc = 0.0625; c0 = 429; c1 = -693; c2 = 315; c3 = -35; nc = 4; break;
      case 8: sc = 0.0078125; c0 = 6435; c1 = -12012; c2 = 6930; c3 = -1260; c4 = 35; nc = 5; break;
      default: break;
    }
    const double cf[5] = {c0, c1, c2, c3, c4};
    // X(f+1+shift) combined: moment of s^shift P_f
    auto comb = [&](const double* X, int shift) -> double {
      if (nc == 1) return X[f + 1 + shift];
      double acc = cf[0] * X[f + 1 + shift];
#pragma unroll
      for (int q = 1; q < 5; ++q)
        if (q < nc) acc += cf[q] * X[f + 1 + shift - 2 * q];
      return sc * acc;
    };
    const double L01 = comb(I1, 0), L03 = comb(I3, 0), L05 = comb(I5, 0);
    const double L13 = comb(I3, 1), L15 = comb(I5, 1), L23 = comb(I3, 2), L25 = comb(I5, 2);
    const int ia[6] = {0, 1, 2, 0, 0, 1};
    const int ib[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      const int a = ia[c], bb = ib[c];
      const double diag = (a == bb) ? 1.0 : 0.0;
      const double rr = R0[a] * R0[bb], tr = tj[a] * R0[bb] + R0[a] * tj[bb], tt = tj[a] * tj[bb];
      G[c][f] = (float)(diag * L01 + L03 * rr - L13 * tr + L23 * tt +
                        e2 * (diag * L03 - 3.0 * L05 * rr + 3.0 * L15 * tr - 3.0 * L25 * tt));
    }
  }
}



}  // namespace rf
