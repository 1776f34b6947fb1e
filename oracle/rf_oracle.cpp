// CPU oracle for the rigid-fiber time step -- TEST INFRASTRUCTURE ONLY.
//
// This file restates, in C++, the reference's Fortran/OpenMP path, which is
// the path that produced the reference's golden vectors
// (tests/reference/100_{numeric,analytic}_{gmres,direct}/*.ref).  It is used
// by the tests, by __graft_entry__.smoke() and by bench.py's cpu_baseline /
// reference arm as the checker and the CPU baseline, never as the product:
// the product path (rigidfibers_b200/) never links, loads or calls it.
//
// Everything is templated on the working precision:
//   float  -> the reference's own REAL*4 arithmetic (parity with the golden files)
//   double -> the FP64 accuracy oracle of the same discretisation
//
// Reference files followed (paths relative to the reference project):
//   fortran/fibers.f95:141-149          constants c, d, e, cc, D1 and F/2
//   fortran/fibers.f95:353-476          quadrature, Legendre tables, lambda, eigen
//   fortran/assemble_matrix.incl:1-161  assembly of A and b
//   fortran/compute_inner_integral_numerically.incl:1-40
//   fortran/compute_inner_integral_analytically.incl:1-338
//   fortran/solve_system.incl:1-175     direct (sgesv) or GMRES driver
//   fortran/sgmres.f:125-190,886-889,1240-1400  GMRES semantics (restart m,
//        x0 = 0, Arnoldi estimate then true residual ||b-Ax||/||b|| <= tol);
//        the GMRES below is written from the published method (Saad & Schultz
//        1986, modified Gram-Schmidt + Givens rotations), not from sgmres.f.
//   lib/viennacl/linalg/bicgstab.hpp:80-166  BiCGSTAB semantics (restart every
//        200 iterations, relative residual), restated from van der Vorst 1992.
//   fortran/update_velocities.incl:1-89
//   fortran/update_fibers_firststep.incl:1-10, fortran/update_fibers.incl:1-17
//
// Layouts follow the Fortran program: positions / orientations / velocities
// are 3N arrays (fiber-major xyz); A is column-major R x R with R = 3*M*N,
// row index i*3M + 3*k_i + d_r, column index j*3M + 3*k_j + d_c; b is R.
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace rfo {

static const int kPointsPerInterval = 3;
static const int kMaxTerms = 8;

struct Tables {
  int M, Q;
  std::vector<double> points, weights;   // Q
  std::vector<double> legendre;          // Q x M, legendre[q*M + k] = P_{k+1}(s_q)
  std::vector<double> lambda, eigen;     // M
};

// fortran/fibers.f95:442-476 (closed forms of P_0..P_8).
static double legendre_poly(double x, int n) {
  switch (n) {
    case 0: return 1.0;
    case 1: return x;
    case 2: return 0.5 * (3.0 * x * x - 1.0);
    case 3: return 0.5 * (5.0 * x * x * x - 3.0 * x);
    case 4: return 0.125 * (35.0 * std::pow(x, 4) - 30.0 * x * x + 3.0);
    case 5: return 0.125 * (63.0 * std::pow(x, 5) - 70.0 * std::pow(x, 3) + 15.0 * x);
    case 6: return 0.0625 * (231.0 * std::pow(x, 6) - 315.0 * std::pow(x, 4) + 105.0 * x * x - 5.0);
    case 7: return 0.0625 * (429.0 * std::pow(x, 7) - 693.0 * std::pow(x, 5) + 315.0 * std::pow(x, 3) - 35.0 * x);
    case 8: return (1.0 / 128.0) * (6435.0 * std::pow(x, 8) - 12012.0 * std::pow(x, 6) + 6930.0 * std::pow(x, 4) - 1260.0 * x * x + 35.0);
  }
  return 0.0;
}

// fortran/fibers.f95:353-440: 3-point Gauss-Legendre on each of `intervals`
// equal sub-intervals of [-1,1]; P_{k+1} at the points; lambda_k and the
// eigenvalue ratio E_k, all in double.
static Tables make_tables(int M, int intervals, double eps) {
  Tables t;
  t.M = M;
  t.Q = intervals * kPointsPerInterval;
  const double p[3] = {-std::sqrt(15.0) / 5.0, 0.0, std::sqrt(15.0) / 5.0};
  const double w[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
  const double h = 2.0 / intervals;
  double lower = -1.0;
  for (int iv = 0; iv < intervals; ++iv) {
    for (int k = 0; k < 3; ++k) {
      t.points.push_back((2.0 * lower + h + p[k] * h) / 2.0);
      t.weights.push_back(w[k] / intervals);
    }
    lower += h;
  }
  t.legendre.resize((size_t)t.Q * M);
  for (int k = 0; k < M; ++k)
    for (int q = 0; q < t.Q; ++q) t.legendre[(size_t)q * M + k] = legendre_poly(t.points[q], k + 1);
  const double c = std::log(eps * eps * std::exp(1.0));
  const double d = -c, e = 2.0, cc = 1.0;
  t.lambda.resize(M);
  t.eigen.resize(M);
  t.lambda[0] = 2.0;
  t.eigen[0] = ((d - e - cc * t.lambda[0]) / 2.0) / (d - cc * t.lambda[0]);
  for (int k = 1; k < M; ++k) {
    t.lambda[k] = t.lambda[k - 1] + 2.0 / (k + 1);
    t.eigen[k] = ((d - e - cc * t.lambda[k]) / 2.0) / (d - cc * t.lambda[k]);
  }
  return t;
}

template <typename T>
struct Model {
  int N, M, Q, R;
  T eps;          // slenderness
  T c, d, e, cc, D1;
  T fhalf[3];     // external force / 2 (fortran/fibers.f95:149)
  std::vector<T> pts, wts, leg, lambda, eigen;

  Model(int N_, int M_, int intervals, double eps_) : N(N_), M(M_) {
    Tables t = make_tables(M_, intervals, eps_);
    Q = t.Q;
    R = 3 * M * N;
    eps = (T)eps_;
    // fortran/fibers.f95:141-145 -- evaluated in the working precision.
    c = std::log(eps * eps * std::exp((T)1.0));
    d = -c;
    e = (T)2.0;
    cc = (T)1.0;
    D1 = (T)0.75 / (d - (T)2.0 * cc);
    fhalf[0] = 0; fhalf[1] = 0; fhalf[2] = (T)-0.5;
    pts.assign(t.points.begin(), t.points.end());
    wts.assign(t.weights.begin(), t.weights.end());
    leg.assign(t.legendre.begin(), t.legendre.end());
    lambda.assign(t.lambda.begin(), t.lambda.end());
    eigen.assign(t.eigen.begin(), t.eigen.end());
  }

  T P(int q, int k) const { return leg[(size_t)q * M + k]; }  // P_{k+1}(s_q)

  // fortran/compute_inner_integral_numerically.incl:1-40
  void inner_numerical(const T* xi, const T* ti, const T* xj, const T* tj, int kj,
                       T* G /*Q x 6*/, T* GF /*Q x 3*/) const {
    const T e2 = (T)2.0 * eps * eps;
    for (int qi = 0; qi < Q; ++qi) {
      T g[6] = {0, 0, 0, 0, 0, 0}, gf[3] = {0, 0, 0};
      T pi[3];
      for (int a = 0; a < 3; ++a) pi[a] = xi[a] + pts[qi] * ti[a];
      for (int qj = 0; qj < Q; ++qj) {
        T r[3], r2[3];
        for (int a = 0; a < 3; ++a) {
          r[a] = pi[a] - (xj[a] + pts[qj] * tj[a]);
          r2[a] = r[a] * r[a];
        }
        const T inv = (T)1.0 / std::sqrt(r2[0] + r2[1] + r2[2]);
        const T inv3 = inv * inv * inv;
        const T inv5 = inv3 * inv * inv;
        T K[6];
        K[0] = inv + inv3 * r2[0] + e2 * (inv3 - (T)3.0 * inv5 * r2[0]);
        K[1] = inv + inv3 * r2[1] + e2 * (inv3 - (T)3.0 * inv5 * r2[1]);
        K[2] = inv + inv3 * r2[2] + e2 * (inv3 - (T)3.0 * inv5 * r2[2]);
        K[3] = inv3 * r[0] * r[1] + e2 * (T)(-3.0) * inv5 * r[0] * r[1];
        K[4] = inv3 * r[0] * r[2] + e2 * (T)(-3.0) * inv5 * r[0] * r[2];
        K[5] = inv3 * r[1] * r[2] + e2 * (T)(-3.0) * inv5 * r[1] * r[2];
        const T w = wts[qj];
        const T lp = P(qj, kj);
        for (int a = 0; a < 6; ++a) g[a] += w * K[a] * lp;
        gf[0] += w * (K[0] * fhalf[0] + K[3] * fhalf[1] + K[4] * fhalf[2]);
        gf[1] += w * (K[3] * fhalf[0] + K[1] * fhalf[1] + K[5] * fhalf[2]);
        gf[2] += w * (K[4] * fhalf[0] + K[5] * fhalf[1] + K[2] * fhalf[2]);
      }
      for (int a = 0; a < 6; ++a) G[qi * 6 + a] = g[a];
      for (int a = 0; a < 3; ++a) GF[qi * 3 + a] = gf[a];
    }
  }

  // G entries from the Legendre-weighted moments (the seven L values) of
  // fortran/compute_inner_integral_analytically.incl:207-260.
  void g_from_moments(const T* R0, const T* tj, T L01, T L03, T L05, T L13, T L15, T L23, T L25,
                      T* out) const {
    const T e2 = (T)2.0 * eps * eps;
    const int ia[6] = {0, 1, 2, 0, 0, 1};
    const int ib[6] = {0, 1, 2, 1, 2, 2};
    for (int c6 = 0; c6 < 6; ++c6) {
      const int a = ia[c6], b = ib[c6];
      const T diag = (a == b) ? (T)1 : (T)0;
      out[c6] = diag * L01 + L03 * (R0[a] * R0[b]) - L13 * (tj[a] * R0[b] + R0[a] * tj[b]) +
                L23 * (tj[a] * tj[b]) +
                e2 * (diag * L03 - (T)3.0 * L05 * (R0[a] * R0[b]) +
                      (T)3.0 * L15 * (tj[a] * R0[b] + R0[a] * tj[b]) - (T)3.0 * L25 * (tj[a] * tj[b]));
    }
  }

  // fortran/compute_inner_integral_analytically.incl:1-338.  I1(n), I3(n),
  // I5(n) (1-based, n = 1..M+3) are the moments int_{-1}^{1} s^{n-1} / |R|^{1,3,5}
  // ds along fiber j, R(s) = R0 - s t_j.  Forward recursion when |R0|^2 < 10,
  // backward recursion from n = 27 otherwise.
  void inner_analytical(const T* xi, const T* ti, const T* xj, const T* tj, int kj,
                        T* G, T* GF) const {
    const int f = kj + 1;
    const int nI = M + 4;  // 1-based, up to M+3
    T I1[kMaxTerms + 4], I3[kMaxTerms + 4], I5[kMaxTerms + 4];
    for (int qi = 0; qi < Q; ++qi) {
      for (int n = 0; n < nI; ++n) I1[n] = I3[n] = I5[n] = 0;
      T R0[3];
      for (int a = 0; a < 3; ++a) R0[a] = xi[a] + pts[qi] * ti[a] - xj[a];
      const T b = (T)-2.0 * (R0[0] * tj[0] + R0[1] * tj[1] + R0[2] * tj[2]);
      const T l = R0[0] * R0[0] + R0[1] * R0[1] + R0[2] * R0[2];
      const T invL = (T)1.0 / l;
      const T llimit = (T)10.0;
      const T m = l - (T)0.25 * b * b;
      const T su = 1, sl = -1;
      const T uu = std::sqrt(su * su + b * su + l);
      const T ul = std::sqrt(sl * sl + b * sl + l);
      const bool degen = m < (T)1e-7;
      const T au = (T)2.0 * su + b, al = (T)2.0 * sl + b;
      I1[1] = std::log(std::fabs(au + (T)2.0 * uu)) - std::log(std::fabs(al + (T)2.0 * ul));
      I1[2] = uu - ul + (-b / (T)2.0) * I1[1];
      I3[1] = degen ? ((T)-2.0 / (au * au)) - ((T)-2.0 / (al * al))
                    : (au / ((T)2.0 * m * uu)) - (al / ((T)2.0 * m * ul));
      I3[2] = ((T)-1.0 / uu) - ((T)-1.0 / ul) - b / (T)2.0 * I3[1];
      I5[1] = degen ? ((T)-4.0 / (au * au * au * au)) - ((T)-4.0 / (al * al * al * al))
                    : (au / ((T)6.0 * m * uu * uu * uu)) - (al / ((T)6.0 * m * ul * ul * ul)) +
                          ((T)2.0 / ((T)3.0 * m)) * I3[1];
      I5[2] = degen ? ((T)-8.0 / ((T)3.0 * au * au * au)) - ((T)-8.0 / ((T)3.0 * al * al * al)) -
                          (b / (T)2.0) * I5[1]
                    : (-(b * su + (T)2.0 * l) / ((T)6.0 * m * uu * uu * uu)) -
                          (-(b * sl + (T)2.0 * l) / ((T)6.0 * m * ul * ul * ul)) -
                          (b / ((T)3.0 * m)) * I3[1];
      if (l < llimit) {
        T psu = su, psl = sl;
        for (int n = 2; n <= f + 2; ++n) {
          I1[n + 1] = (psu * uu) / (T)n - (psl * ul) / (T)n +
                      (((T)1.0 - (T)2.0 * (T)n) * b) / ((T)2.0 * (T)n) * I1[n] -
                      ((T)(n - 1) * l) / (T)n * I1[n - 1];
          I3[n + 1] = I1[n - 1] - b * I3[n] - l * I3[n - 1];
          I5[n + 1] = I3[n - 1] - b * I5[n] - l * I5[n - 1];
          psu *= su;
          psl *= sl;
        }
      } else {
        T i1n2 = 0, i1n1 = 0, i1n0 = 0, i3n2 = 0, i3n1 = 0, i3n0 = 0, i5n2 = 0, i5n1 = 0, i5n0 = 0;
        for (int n = 27; n >= 2; --n) {
          const T np2 = (T)n + (T)2.0, np1 = (T)n + (T)1.0;
          const T sun = (T)1.0;                              // s_upper^(n+1), s_upper = 1
          const T sln = ((n + 1) % 2 == 0) ? (T)1.0 : (T)-1.0;  // s_lower^(n+1), s_lower = -1
          i1n0 = np2 / (np1 * l) *
                 (((sun * uu) / np2) - ((sln * ul) / np2) +
                  (((T)1.0 - (T)2.0 * np2) / ((T)2.0 * np2)) * b * i1n1 - i1n2);
          i3n0 = invL * (i1n0 - b * i3n1 - i3n2);
          i5n0 = invL * (i3n0 - b * i5n1 - i5n2);
          if (n < M + 3) {
            I1[n + 1] = i1n0;
            I3[n + 1] = i3n0;
            I5[n + 1] = i5n0;
          }
          i1n2 = i1n1; i1n1 = i1n0;
          i3n2 = i3n1; i3n1 = i3n0;
          i5n2 = i5n1; i5n1 = i5n0;
        }
      }
      // Legendre recombination: L_ab = int P_f(s) s^a / |R|^b ds.
      T L01, L03, L05, L13, L15, L23, L25;
      legendre_moments(f, I1, I3, I5, L01, L03, L05, L13, L15, L23, L25);
      g_from_moments(R0, tj, L01, L03, L05, L13, L15, L23, L25, &G[qi * 6]);
      if (kj == 0) {
        T g[6];
        g_from_moments(R0, tj, I1[1], I3[1], I5[1], I3[2], I5[2], I3[3], I5[3], g);
        GF[qi * 3 + 0] = g[0] * fhalf[0] + g[3] * fhalf[1] + g[4] * fhalf[2];
        GF[qi * 3 + 1] = g[3] * fhalf[0] + g[1] * fhalf[1] + g[5] * fhalf[2];
        GF[qi * 3 + 2] = g[4] * fhalf[0] + g[5] * fhalf[1] + g[2] * fhalf[2];
      } else {
        GF[qi * 3 + 0] = GF[qi * 3 + 1] = GF[qi * 3 + 2] = 0;
      }
    }
  }

  // Coefficients of P_f in the monomial basis applied to the moment arrays
  // (fortran/compute_inner_integral_analytically.incl:135-205).  With
  // X(n) = moment of s^(n-1):  L0x = sum_p c_p X(p+1), L1x = sum_p c_p X(p+2),
  // L2x = sum_p c_p X(p+3), where P_f(s) = sum_p c_p s^p.
  static void legendre_moments(int f, const T* I1, const T* I3, const T* I5, T& L01, T& L03, T& L05,
                               T& L13, T& L15, T& L23, T& L25) {
    // monomial coefficients (scale, c_f, c_{f-2}, c_{f-4}, ...) of P_f
    T s = 1;
    T cf[5] = {0, 0, 0, 0, 0};
    int nc = 1;
    switch (f) {
      case 0: case 1: s = 1; cf[0] = 1; nc = 1; break;
      case 2: s = (T)0.5; cf[0] = 3; cf[1] = -1; nc = 2; break;
      case 3: s = (T)0.5; cf[0] = 5; cf[1] = -3; nc = 2; break;
      case 4: s = (T)0.125; cf[0] = 35; cf[1] = -30; cf[2] = 3; nc = 3; break;
      case 5: s = (T)0.125; cf[0] = 63; cf[1] = -70; cf[2] = 15; nc = 3; break;
      case 6: s = (T)0.0625; cf[0] = 231; cf[1] = -315; cf[2] = 105; cf[3] = -5; nc = 4; break;
      case 7: s = (T)0.0625; cf[0] = 429; cf[1] = -693; cf[2] = 315; cf[3] = -35; nc = 4; break;
      case 8: s = (T)0.0078125; cf[0] = 6435; cf[1] = -12012; cf[2] = 6930; cf[3] = -1260; cf[4] = 35; nc = 5; break;
    }
    auto comb = [&](const T* X, int shift) {
      if (nc == 1) return X[f + 1 + shift];
      T acc = cf[0] * X[f + 1 + shift];
      for (int p = 1; p < nc; ++p) acc = acc + cf[p] * X[f + 1 + shift - 2 * p];
      return s * acc;
    };
    L01 = comb(I1, 0);
    L03 = comb(I3, 0);
    L05 = comb(I5, 0);
    L13 = comb(I3, 1);
    L15 = comb(I5, 1);
    L23 = comb(I3, 2);
    L25 = comb(I5, 2);
  }

  // fortran/assemble_matrix.incl:1-161.  A is column-major R x R, zeroed here.
  void assemble(const T* pos, const T* ori, bool analytical, T* A, T* bvec) const {
    const size_t RR = (size_t)R;
    std::fill(A, A + RR * RR, (T)0);
    std::fill(bvec, bvec + RR, (T)0);
    const int M3 = 3 * M;
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < N; ++i) {
      std::vector<T> G((size_t)Q * 6), GF((size_t)Q * 3);
      const T* xi = pos + 3 * i;
      const T* ti = ori + 3 * i;
      for (int j = 0; j < N; ++j) {
        if (i == j) {
          for (int k = 0; k < M; ++k)
            for (int a = 0; a < 3; ++a) {
              const size_t r = (size_t)i * M3 + 3 * k + a;
              A[r + r * RR] = (T)1.0;
            }
          continue;
        }
        const T* xj = pos + 3 * j;
        const T* tj = ori + 3 * j;
        for (int kj = 0; kj < M; ++kj) {
          if (analytical) inner_analytical(xi, ti, xj, tj, kj, G.data(), GF.data());
          else inner_numerical(xi, ti, xj, tj, kj, G.data(), GF.data());
          for (int ki = 0; ki < M; ++ki) {
            T Tm[6] = {0, 0, 0, 0, 0, 0}, TF[3] = {0, 0, 0};
            for (int qi = 0; qi < Q; ++qi) {
              const T w = wts[qi];
              const T lp = P(qi, ki);
              for (int a = 0; a < 6; ++a) Tm[a] += w * G[qi * 6 + a] * lp;
              if (kj == 0)
                for (int a = 0; a < 3; ++a) TF[a] += w * GF[qi * 3 + a] * lp;
            }
            T Qv[3];
            Qv[0] = Tm[0] * ti[0] + Tm[3] * ti[1] + Tm[4] * ti[2];
            Qv[1] = Tm[3] * ti[0] + Tm[1] * ti[1] + Tm[5] * ti[2];
            Qv[2] = Tm[4] * ti[0] + Tm[5] * ti[1] + Tm[2] * ti[2];
            const size_t r0 = (size_t)i * M3 + 3 * ki;
            const size_t c0 = (size_t)j * M3 + 3 * kj;
            // full symmetric 3x3 of T (order 11,22,33,12,13,23)
            const T Tf[3][3] = {{Tm[0], Tm[3], Tm[4]}, {Tm[3], Tm[1], Tm[5]}, {Tm[4], Tm[5], Tm[2]}};
            if (ki == 0) {
              for (int a = 0; a < 3; ++a)
                for (int bb = 0; bb < 3; ++bb) A[(r0 + a) + (c0 + bb) * RR] = D1 * ti[a] * Qv[bb];
              if (kj == 0) {
                const T QF = TF[0] * ti[0] + TF[1] * ti[1] + TF[2] * ti[2];
                for (int a = 0; a < 3; ++a) bvec[r0 + a] -= D1 * ti[a] * QF;
              }
            } else {
              const T gamma = (T)0.5 * ((T)2.0 * (T)(ki + 1) + (T)1.0) / (d + e - cc * lambda[ki]);
              const T Ek = eigen[ki];
              for (int a = 0; a < 3; ++a)
                for (int bb = 0; bb < 3; ++bb)
                  A[(r0 + a) + (c0 + bb) * RR] = gamma * (Tf[a][bb] - Ek * ti[a] * Qv[bb]);
              if (kj == 0) {
                const T QF = TF[0] * ti[0] + TF[1] * ti[1] + TF[2] * ti[2];
                for (int a = 0; a < 3; ++a) bvec[r0 + a] -= gamma * (TF[a] - Ek * ti[a] * QF);
              }
            }
          }
        }
      }
    }
  }

  // Row-block assembly used by the bounded CPU baseline sample: rows of
  // fibers [i0, i1) only, into a column-major (rows x R) slab.  Same
  // arithmetic as assemble().
  void assemble_rows(const T* pos, const T* ori, bool analytical, int i0, int i1, T* slab, T* bpart) const {
    const int M3 = 3 * M;
    const size_t rows = (size_t)(i1 - i0) * M3;
    std::fill(slab, slab + rows * (size_t)R, (T)0);
    std::fill(bpart, bpart + rows, (T)0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = i0; i < i1; ++i) {
      std::vector<T> G((size_t)Q * 6), GF((size_t)Q * 3);
      const T* xi = pos + 3 * i;
      const T* ti = ori + 3 * i;
      for (int j = 0; j < N; ++j) {
        if (i == j) {
          for (int k = 0; k < M; ++k)
            for (int a = 0; a < 3; ++a) {
              const size_t rl = (size_t)(i - i0) * M3 + 3 * k + a;
              slab[rl + ((size_t)i * M3 + 3 * k + a) * rows] = (T)1.0;
            }
          continue;
        }
        const T* xj = pos + 3 * j;
        const T* tj = ori + 3 * j;
        for (int kj = 0; kj < M; ++kj) {
          if (analytical) inner_analytical(xi, ti, xj, tj, kj, G.data(), GF.data());
          else inner_numerical(xi, ti, xj, tj, kj, G.data(), GF.data());
          for (int ki = 0; ki < M; ++ki) {
            T Tm[6] = {0, 0, 0, 0, 0, 0}, TF[3] = {0, 0, 0};
            for (int qi = 0; qi < Q; ++qi) {
              const T w = wts[qi];
              const T lp = P(qi, ki);
              for (int a = 0; a < 6; ++a) Tm[a] += w * G[qi * 6 + a] * lp;
              if (kj == 0)
                for (int a = 0; a < 3; ++a) TF[a] += w * GF[qi * 3 + a] * lp;
            }
            T Qv[3];
            Qv[0] = Tm[0] * ti[0] + Tm[3] * ti[1] + Tm[4] * ti[2];
            Qv[1] = Tm[3] * ti[0] + Tm[1] * ti[1] + Tm[5] * ti[2];
            Qv[2] = Tm[4] * ti[0] + Tm[5] * ti[1] + Tm[2] * ti[2];
            const size_t r0 = (size_t)(i - i0) * M3 + 3 * ki;
            const size_t c0 = (size_t)j * M3 + 3 * kj;
            const T Tf[3][3] = {{Tm[0], Tm[3], Tm[4]}, {Tm[3], Tm[1], Tm[5]}, {Tm[4], Tm[5], Tm[2]}};
            const T gamma = ki == 0 ? D1 : (T)0.5 * ((T)2.0 * (T)(ki + 1) + (T)1.0) / (d + e - cc * lambda[ki]);
            for (int a = 0; a < 3; ++a)
              for (int bb = 0; bb < 3; ++bb)
                slab[(r0 + a) + (c0 + bb) * rows] =
                    ki == 0 ? D1 * ti[a] * Qv[bb] : gamma * (Tf[a][bb] - eigen[ki] * ti[a] * Qv[bb]);
            if (kj == 0) {
              const T QF = TF[0] * ti[0] + TF[1] * ti[1] + TF[2] * ti[2];
              for (int a = 0; a < 3; ++a)
                bpart[r0 + a] -= ki == 0 ? D1 * ti[a] * QF : gamma * (TF[a] - eigen[ki] * ti[a] * QF);
            }
          }
        }
      }
    }
  }

  // fortran/update_velocities.incl:1-89 (always numerical integration).
  // `coeff` holds the solved force coefficients (the solution x).
  void update_velocities(const T* pos, const T* ori, const T* coeff, int i0, int i1, T* tvel, T* rvel, bool analytical = false) const {
    const int M3 = 3 * M;
    const T e2 = (T)2.0 * eps * eps;
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = i0; i < i1; ++i) {
      std::vector<T> GF((size_t)Q * 3);
      const T* xi = pos + 3 * i;
      const T* ti = ori + 3 * i;
      T of[3];
      const T tdotf = ti[0] * ((T)2.0 * fhalf[0]) + ti[1] * ((T)2.0 * fhalf[1]) + ti[2] * ((T)2.0 * fhalf[2]);
      for (int a = 0; a < 3; ++a) of[a] = tdotf * ti[a];
      T U[3], W[3] = {0, 0, 0};
      for (int a = 0; a < 3; ++a) U[a] = (d + (T)2.0) * (T)2.0 * fhalf[a] + (d - (T)2.0) * of[a];
      std::vector<T> Gk((size_t)Q * 6), GFk((size_t)Q * 3);
      for (int j = 0; j < N; ++j) {
        if (i == j) continue;
        const T* xj = pos + 3 * j;
        const T* tj = ori + 3 * j;
        if (analytical) {
          // Exact inner integral of K(R) f_j(s) over fiber j, with
          // f_j = F/2 + sum_k a_{j,k} P_{k+1}: the analytic G for every k and
          // the analytic GF (F/2 term).
          for (int q = 0; q < Q * 3; ++q) GF[q] = 0;
          for (int kj = 0; kj < M; ++kj) {
            inner_analytical(xi, ti, xj, tj, kj, Gk.data(), GFk.data());
            const size_t row = (size_t)j * M3 + 3 * kj;
            const T a0 = coeff[row], a1 = coeff[row + 1], a2 = coeff[row + 2];
            for (int qi = 0; qi < Q; ++qi) {
              const T* g = &Gk[qi * 6];
              if (kj == 0)
                for (int a = 0; a < 3; ++a) GF[qi * 3 + a] += GFk[qi * 3 + a];
              GF[qi * 3 + 0] += g[0] * a0 + g[3] * a1 + g[4] * a2;
              GF[qi * 3 + 1] += g[3] * a0 + g[1] * a1 + g[5] * a2;
              GF[qi * 3 + 2] += g[4] * a0 + g[5] * a1 + g[2] * a2;
            }
          }
        } else
        for (int qi = 0; qi < Q; ++qi) {
          T gf[3] = {0, 0, 0};
          T pi[3];
          for (int a = 0; a < 3; ++a) pi[a] = xi[a] + pts[qi] * ti[a];
          for (int qj = 0; qj < Q; ++qj) {
            T r[3], r2[3];
            for (int a = 0; a < 3; ++a) {
              r[a] = pi[a] - (xj[a] + pts[qj] * tj[a]);
              r2[a] = r[a] * r[a];
            }
            const T inv = (T)1.0 / std::sqrt(r2[0] + r2[1] + r2[2]);
            const T inv3 = inv * inv * inv;
            const T inv5 = inv3 * inv * inv;
            T K[6];
            K[0] = inv + inv3 * r2[0] + e2 * (inv3 - (T)3.0 * inv5 * r2[0]);
            K[1] = inv + inv3 * r2[1] + e2 * (inv3 - (T)3.0 * inv5 * r2[1]);
            K[2] = inv + inv3 * r2[2] + e2 * (inv3 - (T)3.0 * inv5 * r2[2]);
            K[3] = inv3 * r[0] * r[1] + e2 * (T)(-3.0) * inv5 * r[0] * r[1];
            K[4] = inv3 * r[0] * r[2] + e2 * (T)(-3.0) * inv5 * r[0] * r[2];
            K[5] = inv3 * r[1] * r[2] + e2 * (T)(-3.0) * inv5 * r[1] * r[2];
            T fj[3] = {fhalf[0], fhalf[1], fhalf[2]};
            for (int k = 0; k < M; ++k) {
              const T lp = P(qj, k);
              const size_t row = (size_t)j * M3 + 3 * k;
              for (int a = 0; a < 3; ++a) fj[a] += coeff[row + a] * lp;
            }
            const T w = wts[qj];
            gf[0] += w * (K[0] * fj[0] + K[3] * fj[1] + K[4] * fj[2]);
            gf[1] += w * (K[3] * fj[0] + K[1] * fj[1] + K[5] * fj[2]);
            gf[2] += w * (K[4] * fj[0] + K[5] * fj[1] + K[2] * fj[2]);
          }
          for (int a = 0; a < 3; ++a) GF[qi * 3 + a] = gf[a];
        }
        T A0[3] = {0, 0, 0}, A1[3] = {0, 0, 0};
        for (int qi = 0; qi < Q; ++qi) {
          const T w = wts[qi];
          const T lp = P(qi, 0);
          for (int a = 0; a < 3; ++a) {
            A0[a] += w * GF[qi * 3 + a];
            A1[a] += w * GF[qi * 3 + a] * lp;
          }
        }
        for (int a = 0; a < 3; ++a) U[a] += A0[a];
        const T tA1 = A1[0] * ti[0] + A1[1] * ti[1] + A1[2] * ti[2];
        for (int a = 0; a < 3; ++a) W[a] += A1[a] - ti[a] * tA1;
      }
      for (int a = 0; a < 3; ++a) {
        tvel[3 * i + a] = U[a] * ((T)0.5 / d);
        rvel[3 * i + a] = W[a] * ((T)1.5 / d);
      }
    }
  }
};

// y = A x, column-major A (rows x cols), OpenMP over row chunks.
template <typename T>
static void gemv_colmajor(int rows, int cols, const T* A, const T* x, T* y) {
#pragma omp parallel
  {
#ifdef _OPENMP
    const int nt = omp_get_num_threads(), tid = omp_get_thread_num();
#else
    const int nt = 1, tid = 0;
#endif
    const int chunk = (rows + nt - 1) / nt;
    const int r0 = tid * chunk, r1 = std::min(rows, r0 + chunk);
    if (r0 < r1) {
      std::vector<T> acc(r1 - r0, (T)0);
      for (int c = 0; c < cols; ++c) {
        const T xc = x[c];
        const T* col = A + (size_t)c * rows;
        for (int r = r0; r < r1; ++r) acc[r - r0] += col[r] * xc;
      }
      for (int r = r0; r < r1; ++r) y[r] = acc[r - r0];
    }
  }
}

template <typename T>
static double dot(int n, const T* a, const T* b) {
  double s = 0;
#pragma omp parallel for reduction(+ : s)
  for (int i = 0; i < n; ++i) s += (double)a[i] * (double)b[i];
  return s;
}

// Restarted GMRES(m), x0 = 0, modified Gram-Schmidt Arnoldi, Givens
// rotations; stops when the Arnoldi residual estimate drops below tol*||b||
// and the true residual ||b - A x|| confirms it (fortran/sgmres.f semantics,
// icntl(8) = 1).  Returns total inner iterations, or -1 without convergence.
template <typename T>
static int gmres(int n, const T* A, const T* b, T* x, int restart, int maxit, double tol, double* relres) {
  const int m = restart;
  std::vector<T> V((size_t)(m + 1) * n), w(n), r(n);
  std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
  std::fill(x, x + n, (T)0);
  const double bnorm = std::sqrt(dot(n, b, b));
  if (bnorm == 0) { *relres = 0; return 0; }
  int it = 0;
  // r = b - A x (x = 0)
  for (int i = 0; i < n; ++i) r[i] = b[i];
  double beta = bnorm;
  while (true) {
    for (int i = 0; i < n; ++i) V[i] = (T)(r[i] / beta);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int jdone = 0;
    bool est_conv = false;
    for (int j = 0; j < m && it < maxit; ++j) {
      gemv_colmajor(n, n, A, &V[(size_t)j * n], w.data());
      for (int i = 0; i <= j; ++i) {
        const double h = dot(n, w.data(), &V[(size_t)i * n]);
        H[(size_t)i * m + j] = h;
        const T hf = (T)h;
        for (int k = 0; k < n; ++k) w[k] -= hf * V[(size_t)i * n + k];
      }
      const double hn = std::sqrt(dot(n, w.data(), w.data()));
      H[(size_t)(j + 1) * m + j] = hn;
      for (int k = 0; k < n; ++k) V[(size_t)(j + 1) * n + k] = hn > 0 ? (T)(w[k] / hn) : (T)0;
      for (int i = 0; i < j; ++i) {
        const double a = H[(size_t)i * m + j], bb = H[(size_t)(i + 1) * m + j];
        H[(size_t)i * m + j] = cs[i] * a + sn[i] * bb;
        H[(size_t)(i + 1) * m + j] = -sn[i] * a + cs[i] * bb;
      }
      const double a = H[(size_t)j * m + j], bb = H[(size_t)(j + 1) * m + j];
      const double rr = std::hypot(a, bb);
      cs[j] = rr > 0 ? a / rr : 1.0;
      sn[j] = rr > 0 ? bb / rr : 0.0;
      H[(size_t)j * m + j] = rr;
      H[(size_t)(j + 1) * m + j] = 0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      ++it;
      jdone = j + 1;
      if (std::fabs(g[j + 1]) / bnorm <= tol) { est_conv = true; break; }
    }
    for (int i = jdone - 1; i >= 0; --i) {
      double s = g[i];
      for (int k = i + 1; k < jdone; ++k) s -= H[(size_t)i * m + k] * y[k];
      y[i] = s / H[(size_t)i * m + i];
    }
    for (int i = 0; i < jdone; ++i) {
      const T yi = (T)y[i];
      for (int k = 0; k < n; ++k) x[k] += yi * V[(size_t)i * n + k];
    }
    gemv_colmajor(n, n, A, x, w.data());
    for (int k = 0; k < n; ++k) r[k] = b[k] - w[k];
    beta = std::sqrt(dot(n, r.data(), r.data()));
    *relres = beta / bnorm;
    if (*relres <= tol) return it;
    (void)est_conv;
    if (it >= maxit) return -1;
  }
}

// BiCGSTAB (van der Vorst 1992) with the semantics of the reference's
// ViennaCL 1.5.1 solver (lib/viennacl/linalg/bicgstab.hpp:80-166): x0 = 0,
// convergence when ||r||/||b|| < tol on the recursive residual after a full
// iteration, restart from the true residual when rho or omega vanish or more
// than `restart_every` iterations passed since the last restart.
template <typename T>
static int bicgstab(int n, const T* A, const T* b, T* x, int maxit, double tol, int restart_every, double* relres) {
  std::vector<T> r(n), r0(n), p(n), v(n), s(n), t(n);
  std::fill(x, x + n, (T)0);
  const double bnorm = std::sqrt(dot(n, b, b));
  if (bnorm == 0) { *relres = 0; return 0; }
  bool restart = true;
  int last_restart = 0;
  double rho = 0;
  for (int i = 0; i < maxit; ++i) {
    if (restart) {
      gemv_colmajor(n, n, A, x, t.data());
      for (int k = 0; k < n; ++k) { r[k] = b[k] - t[k]; p[k] = r[k]; r0[k] = r[k]; }
      rho = dot(n, r.data(), r.data());
      restart = false;
      last_restart = i;
    }
    gemv_colmajor(n, n, A, p.data(), v.data());
    const double alpha = rho / dot(n, v.data(), r0.data());
    for (int k = 0; k < n; ++k) s[k] = r[k] - (T)alpha * v[k];
    gemv_colmajor(n, n, A, s.data(), t.data());
    const double tt = dot(n, t.data(), t.data());
    const double omega = tt > 0 ? dot(n, t.data(), s.data()) / tt : 0.0;
    for (int k = 0; k < n; ++k) {
      x[k] = x[k] + (T)alpha * p[k] + (T)omega * s[k];
      r[k] = s[k] - (T)omega * t[k];
    }
    const double rho_new = dot(n, r.data(), r0.data());
    const double rn = std::sqrt(dot(n, r.data(), r.data()));
    *relres = rn / bnorm;
    if (rn / bnorm < tol) return i + 1;
    const double beta = (rho_new / rho) * (alpha / omega);
    rho = rho_new;
    if (rho == 0 || omega == 0 || i - last_restart > restart_every) restart = true;
    for (int k = 0; k < n; ++k) p[k] = r[k] + (T)beta * (p[k] - (T)omega * v[k]);
  }
  return -1;
}

// LU with partial pivoting and solve (the arithmetic of LAPACK xGESV:
// right-looking elimination, row interchanges).  A is overwritten.
template <typename T>
static int lu_solve(int n, T* A, T* b) {
  std::vector<int> piv(n);
  for (int k = 0; k < n; ++k) {
    int p = k;
    T best = std::fabs(A[k + (size_t)k * n]);
    for (int i = k + 1; i < n; ++i) {
      const T v = std::fabs(A[i + (size_t)k * n]);
      if (v > best) { best = v; p = i; }
    }
    if (best == (T)0) return k + 1;
    piv[k] = p;
    if (p != k) {
      for (int c = 0; c < n; ++c) std::swap(A[k + (size_t)c * n], A[p + (size_t)c * n]);
      std::swap(b[k], b[p]);
    }
    const T inv = (T)1 / A[k + (size_t)k * n];
    for (int i = k + 1; i < n; ++i) A[i + (size_t)k * n] *= inv;
#pragma omp parallel for schedule(static)
    for (int c = k + 1; c < n; ++c) {
      const T akc = A[k + (size_t)c * n];
      if (akc != (T)0) {
        T* col = A + (size_t)c * n;
        const T* lk = A + (size_t)k * n;
        for (int i = k + 1; i < n; ++i) col[i] -= lk[i] * akc;
      }
    }
  }
  for (int i = 0; i < n; ++i) {  // forward (unit lower)
    T s = b[i];
    for (int k = 0; k < i; ++k) s -= A[i + (size_t)k * n] * b[k];
    b[i] = s;
  }
  for (int i = n - 1; i >= 0; --i) {  // backward
    T s = b[i];
    for (int k = i + 1; k < n; ++k) s -= A[i + (size_t)k * n] * b[k];
    b[i] = s / A[i + (size_t)i * n];
  }
  return 0;
}

// fortran/update_fibers_firststep.incl:1-10 (first == 1) and
// fortran/update_fibers.incl:1-17 (second order), then renormalise t.
template <typename T>
static void update_fibers(int N, int first, T dt, const T* prev_pos, const T* cur_pos, const T* prev_ori,
                          const T* cur_ori, const T* prev_tv, const T* cur_tv, const T* prev_rv, const T* cur_rv,
                          T* next_pos, T* next_ori) {
  for (int i = 0; i < N; ++i) {
    T o[3];
    for (int a = 0; a < 3; ++a) {
      const int k = 3 * i + a;
      if (first) {
        next_pos[k] = cur_pos[k] + dt * cur_tv[k];
        o[a] = cur_ori[k] + dt * cur_rv[k];
      } else {
        next_pos[k] = ((T)4.0 / (T)3.0) * cur_pos[k] - ((T)1.0 / (T)3.0) * prev_pos[k] +
                      ((T)2.0 / (T)3.0) * dt * ((T)2.0 * cur_tv[k] - prev_tv[k]);
        o[a] = ((T)4.0 / (T)3.0) * cur_ori[k] - ((T)1.0 / (T)3.0) * prev_ori[k] +
               ((T)2.0 / (T)3.0) * dt * ((T)2.0 * cur_rv[k] - prev_rv[k]);
      }
    }
    const T nrm = std::sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
    for (int a = 0; a < 3; ++a) next_ori[3 * i + a] = o[a] / nrm;
  }
}

}  // namespace rfo

// ---------------------------------------------------------------------------
// C ABI for the tests (ctypes).  Suffix _f32 = REAL*4 parity oracle, _f64 =
// FP64 accuracy oracle.
// ---------------------------------------------------------------------------
#define RFO_DEFINE(SUF, T)                                                                              \
  extern "C" int rfo_tables_##SUF(int M, int intervals, double eps, T* points, T* weights, T* legendre, \
                                  T* lambda, T* eigen) {                                                \
    rfo::Model<T> m(1, M, intervals, eps);                                                              \
    for (int q = 0; q < m.Q; ++q) { points[q] = m.pts[q]; weights[q] = m.wts[q]; }                      \
    for (size_t k = 0; k < m.leg.size(); ++k) legendre[k] = m.leg[k];                                   \
    for (int k = 0; k < M; ++k) { lambda[k] = m.lambda[k]; eigen[k] = m.eigen[k]; }                     \
    return 0;                                                                                           \
  }                                                                                                     \
  extern "C" int rfo_assemble_##SUF(int N, int M, int intervals, double eps, int analytical,            \
                                    const T* pos, const T* ori, T* A, T* b) {                           \
    rfo::Model<T> m(N, M, intervals, eps);                                                              \
    m.assemble(pos, ori, analytical != 0, A, b);                                                        \
    return 0;                                                                                           \
  }                                                                                                     \
  extern "C" int rfo_assemble_rows_##SUF(int N, int M, int intervals, double eps, int analytical,       \
                                         const T* pos, const T* ori, int i0, int i1, T* slab, T* b) {   \
    rfo::Model<T> m(N, M, intervals, eps);                                                              \
    m.assemble_rows(pos, ori, analytical != 0, i0, i1, slab, b);                                        \
    return 0;                                                                                           \
  }                                                                                                     \
  extern "C" int rfo_update_velocities_##SUF(int N, int M, int intervals, double eps, const T* pos,     \
                                             const T* ori, const T* coeff, int i0, int i1, T* tvel,     \
                                             T* rvel, int analytical) {                                 \
    rfo::Model<T> m(N, M, intervals, eps);                                                              \
    m.update_velocities(pos, ori, coeff, i0, i1, tvel, rvel, analytical != 0);                                           \
    return 0;                                                                                           \
  }                                                                                                     \
  extern "C" int rfo_gmres_##SUF(int n, const T* A, const T* b, T* x, int restart, int maxit,           \
                                 double tol, double* relres) {                                          \
    return rfo::gmres<T>(n, A, b, x, restart, maxit, tol, relres);                                      \
  }                                                                                                     \
  extern "C" int rfo_bicgstab_##SUF(int n, const T* A, const T* b, T* x, int maxit, double tol,         \
                                    int restart_every, double* relres) {                                \
    return rfo::bicgstab<T>(n, A, b, x, maxit, tol, restart_every, relres);                             \
  }                                                                                                     \
  extern "C" int rfo_lu_solve_##SUF(int n, T* A, T* b) { return rfo::lu_solve<T>(n, A, b); }           \
  extern "C" int rfo_gemv_##SUF(int rows, int cols, const T* A, const T* x, T* y) {                     \
    rfo::gemv_colmajor<T>(rows, cols, A, x, y);                                                         \
    return 0;                                                                                           \
  }                                                                                                     \
  extern "C" int rfo_update_fibers_##SUF(int N, int first, double dt, const T* pp, const T* cp,         \
                                         const T* po, const T* co, const T* ptv, const T* ctv,          \
                                         const T* prv, const T* crv, T* np, T* no) {                    \
    rfo::update_fibers<T>(N, first, (T)dt, pp, cp, po, co, ptv, ctv, prv, crv, np, no);                 \
    return 0;                                                                                           \
  }

RFO_DEFINE(f32, float)
RFO_DEFINE(f64, double)

extern "C" int rfo_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
