// Assembly of the rigid-fiber linear system (numerical inner integrals).
//
// Reference: fortran/assemble_matrix.incl:1-161 with
// fortran/compute_inner_integral_numerically.incl:1-40, and the CUDA kernels
// src/kernels/assemble_system_2D.cu:8-367 + compute_inner_integral_numerically.cu.
//
// What is computed is the reference's: for every ordered pair (i, j), i != j,
//   T^{ij}_{ki,kj} = sum_qi sum_qj W[ki][qi] K(R_ij(qi,qj)) W[kj][qj]      (3x3 sym)
// with W[k][q] = w_q P_k(s_q), then the 15x15 block A_(i,j) = C_i T^{ij} and
// b_i -= C_i T^{ij}_{.,P0} F/2, where C_i is D1 t t^T (force index 0) or
// gamma_k (I - E_k t t^T).  How it is computed is not the reference's:
//  * K is even in R, so T^{ji}_{kj,ki} = T^{ij}_{ki,kj}: one CTA tile of
//    unordered fiber pairs evaluates K once per (qi, qj) and serves both
//    blocks (i,j) and (j,i)  -- half the kernel evaluations;
//  * the reference re-evaluates K once per k_j (M times); here once;
//  * the sum over fiber j's points splits each separation at its projection
//    onto fiber j's axis (r = d + u t_j, d perpendicular to t_j), so the six
//    components of K contract to four scalar moments (see phase 1);
//  * the quadrature is mirror-symmetric (s_{Q-1-q} = -s_q, w equal, P_k of
//    parity k), so both contractions fold q with Q-1-q into an even and an
//    odd part and use half the multiply-adds;
//  * the force terms F_i[k] = sum_j T^{ij}_{k,P0} F/2 are reduced
//    deterministically (per-tile partial rows, then a fixed-order sum)
//    instead of with float atomics; b_i = -C_i F_i.
//
// Two outputs share the pair-tile core:
//  * dense:      A column-major with leading dimension lda >= R (padded to 32
//                so every column starts on a 128-byte boundary), A[r + c*lda];
//  * structured: the blocks T^{ij}_{k,kj}, k,kj = P_0..P_M, once per
//                unordered pair, in FP32 (all (M+1)^2 blocks) and in 16 bits
//                (the M^2 blocks of the operator), laid out per 16x16 fiber
//                storage tile as [tile][sub-tile][j][value][i] so that one
//                CTA's writes for one j are contiguous and the matvec reads
//                whole 32-byte sectors (see rf_struct.cu).
#include "rf_common.cuh"
#include "rf_kernels.cuh"
#include "rf_analytic.cuh"

namespace rf {

// Decode a linear index over the upper triangle (I <= J) of T x T tiles.
__device__ __forceinline__ void tile_pair(int64_t L, int& I, int& J) {
  int64_t j = (int64_t)((sqrt(8.0 * (double)L + 1.0) - 1.0) * 0.5);
  while ((j + 1) * (j + 2) / 2 <= L) ++j;
  while (j * (j + 1) / 2 > L) --j;
  J = (int)j;
  I = (int)(L - j * (j + 1) / 2);
}

// kAsmApply: nothing stored; the pair blocks are applied to a vector (the
// matrix-free product) or, without a vector, only the force terms are formed
enum AsmMode { kAsmDense = 0, kAsmStructF16 = 1, kAsmStructBF16 = 2, kAsmApply = 3 };
enum AsmInteg { kNumerical = 0, kAnalytical = 1 };

template <int M, int Q>
struct AsmShape {
  static constexpr int TI = 192 / Q;     // fibers per tile side
  static constexpr int U = TI * Q;       // (fiber, quadrature point) units = threads used
  static constexpr int K1 = M + 1;       // P_0..P_M
  static constexpr int NC = 6 * K1;      // G columns per unit
  static constexpr int H = Q / 2;        // folded quadrature points
  static constexpr int NT = 192;         // threads per CTA
  // dynamic shared memory: G as NC columns of U units (unit u = qi * TI + il),
  // then the T blocks (6 floats each).  The column stride is TI (mod 32)
  // words: phase 2 has lanes (col, tl), TI consecutive tl per column and
  // 32 / TI columns per warp, and reads 32 distinct banks.
  static constexpr int GS = (U + 31) / 32 * 32 + TI;
  // the T blocks start on a 16-byte boundary (they are copied out as float4);
  // NC * GS is odd for odd M + 1
  static constexpr int GOFF = (NC * GS + 3) / 4 * 4;
  static constexpr size_t kGBytes = sizeof(float) * GOFF;
  // T pair stride padded so that 8 consecutive pairs start on distinct banks
  // that are multiples of 4 (stride = 4 * odd mod 32)
  static constexpr int TP = (K1 * K1 * 6 + 7) / 8 * 8 + 4;
  static constexpr size_t kTBytes = sizeof(float) * TI * TP;
  static constexpr size_t kSmem = kGBytes + 2 * kTBytes;   // T double-buffered across j
  static_assert(GOFF % 4 == 0 && TP % 4 == 0, "T buffers must be 16-byte aligned");
  // structured storage
  static constexpr int SUB = kStoreTile / TI;      // assembly tiles per storage-tile side
  static constexpr int NQ32 = K1 * K1 * 6;         // FP32 values per pair
  static constexpr int NQ16 = M * M * 6 / 2;       // 16-bit pairs per pair (M*M*6 is even)
  static_assert(kStoreTile % TI == 0, "assembly tile must divide the storage tile");
};

struct AsmOut {
  // dense
  float* A;
  int64_t lda;
  // structured
  float* S32;
  uint32_t* S16;
  // both: partial force terms ffpart[X][i][k][3]
  float* ffpart;
  // analytical: the FP64 fiber state (the closed-form integral is ~7x more
  // sensitive to the rounding of its inputs than the quadrature)
  const double4* pos64;
  const double4* ori64;
  // kAsmApply: z partial rows of T x (null x: force terms only) into
  // zpart[(assemble tiles + 1) x R]; skip: a device word that, when set,
  // makes the launch return at once (a converged Krylov solve)
  const float* x;
  float* zpart;
  const int* skip;
};

// Tile pair L of a suspension of N fibers: numerical, unordered pairs (I <= J)
// whose one evaluation of K serves both blocks; analytical, ordered pairs.
template <int Q, int INTEG>
__device__ __forceinline__ void asm_tile_of(int N, unsigned L, int& I, int& J) {
  constexpr int TI = 192 / Q;
  if (INTEG == kNumerical) {
    tile_pair(L, I, J);
  } else {
    const int T = (N + TI - 1) / TI;
    I = (int)(L / T);
    J = (int)(L % T);
  }
}

// Phase 1 of a pair tile, numerical: G[c][k] = sum_q K_c(p - s_q t_j) W[k][q]
// for one point p of fiber i (relative to fiber j's centre) against the Q
// points of fiber j, written to gcol[(6 k + c) GS].
//
// The separation r = p - s_q t_j is split at p's projection onto fiber j's
// axis: r = d + u_q t_j with d = p - s* t_j perpendicular to t_j and
// u_q = s* - s_q, so |r|^2 = |d|^2 + u_q^2 and
//   K(r) = a I + b r r^T = a I + b [d d^T + u (d t^T + t d^T) + u^2 t t^T]
// (a = 1/|r| + 2eps^2/|r|^3, b = 1/|r|^3 - 6eps^2/|r|^5).  The sum over q then
// needs four scalar moments per k instead of six tensor components,
//   A_k = sum W a,  B0_k = sum W b,  B1_k = sum W b u,  B2_k = sum W b u^2,
// and every term of the recombination is bounded by |r|^2 (|d|, |u| <= |r|),
// so nothing cancels.  s* is refined once (d . t_j, already ~1e-7 |p|, is
// folded back) so that d is perpendicular to t_j to rounding.  Points q and
// Q-1-q are evaluated together and their values folded into even and odd
// parts (W[k][Q-1-q] = (-1)^k W[k][q]).
//
// P2 = true evaluates the two mirror points in the two lanes of packed FP32
// instructions (add/mul/fma .f32x2) and accumulates the moments in lane pairs
// (A, B0), (B1, B2) against the duplicated weights W2; every rounding is the
// same as in the scalar form (all steps are explicit _rn operations, none can
// be contracted), so both give bit-identical G.
template <int K1, int Q, int GS, bool P2>
__device__ __forceinline__ void stokeslet_moments_G(const Tables& tab, const float p[3], const float4 tj, float e2,
                                                    float e2x3, float* __restrict__ gcol) {
  constexpr int H = Q / 2;
  float ss = fmaf(p[0], tj.x, fmaf(p[1], tj.y, p[2] * tj.z));
  float dx = fmaf(-ss, tj.x, p[0]), dy = fmaf(-ss, tj.y, p[1]), dz = fmaf(-ss, tj.z, p[2]);
  const float dl = fmaf(dx, tj.x, fmaf(dy, tj.y, dz * tj.z));
  ss += dl;
  dx = fmaf(-dl, tj.x, dx);
  dy = fmaf(-dl, tj.y, dy);
  dz = fmaf(-dl, tj.z, dz);
  const float dd = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  float2 m01[K1], m23[K1];   // (A_k, B0_k), (B1_k, B2_k)
#pragma unroll
  for (int k = 0; k < K1; ++k) m01[k] = m23[k] = make_float2(0.f, 0.f);
#pragma unroll
  for (int q = 0; q < H; ++q) {
    float2 fa, fb, fc, fd;   // lane x: point q, lane y: point Q-1-q
    if constexpr (P2) {
      const float2 u = __fadd2_rn(make_float2(ss, ss), make_float2(-tab.pts[q], -tab.pts[Q - 1 - q]));
      const float2 r2 = __ffma2_rn(u, u, make_float2(dd, dd));
      const float2 inv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
      const float2 inv2 = __fmul2_rn(inv, inv);
      const float2 inv3 = __fmul2_rn(inv2, inv);
      const float2 inv5 = __fmul2_rn(inv3, inv2);
      fa = __ffma2_rn(make_float2(e2, e2), inv3, inv);
      fb = __ffma2_rn(make_float2(e2x3, e2x3), inv5, inv3);
      fc = __fmul2_rn(fb, u);
      fd = __fmul2_rn(fc, u);
    } else {
      float r[4][2];
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        const float u = __fadd_rn(ss, -tab.pts[side == 0 ? q : Q - 1 - q]);
        const float r2 = __fmaf_rn(u, u, dd);
        const float inv = rsqrtf(r2);
        const float inv2 = __fmul_rn(inv, inv);
        const float inv3 = __fmul_rn(inv2, inv);
        const float inv5 = __fmul_rn(inv3, inv2);
        r[0][side] = __fmaf_rn(e2, inv3, inv);
        r[1][side] = __fmaf_rn(e2x3, inv5, inv3);
        r[2][side] = __fmul_rn(r[1][side], u);
        r[3][side] = __fmul_rn(r[2][side], u);
      }
      fa = make_float2(r[0][0], r[0][1]);
      fb = make_float2(r[1][0], r[1][1]);
      fc = make_float2(r[2][0], r[2][1]);
      fd = make_float2(r[3][0], r[3][1]);
    }
    const float2 e01 = make_float2(__fadd_rn(fa.x, fa.y), __fadd_rn(fb.x, fb.y));
    const float2 o01 = make_float2(__fsub_rn(fa.x, fa.y), __fsub_rn(fb.x, fb.y));
    const float2 e23 = make_float2(__fadd_rn(fc.x, fc.y), __fadd_rn(fd.x, fd.y));
    const float2 o23 = make_float2(__fsub_rn(fc.x, fc.y), __fsub_rn(fd.x, fd.y));
#pragma unroll
    for (int k = 0; k < K1; ++k) {
      if constexpr (P2) {
        m01[k] = __ffma2_rn((k & 1) ? o01 : e01, tab.W2[k][q], m01[k]);
        m23[k] = __ffma2_rn((k & 1) ? o23 : e23, tab.W2[k][q], m23[k]);
      } else {
        const float w = tab.W[k][q];
        m01[k].x = __fmaf_rn((k & 1) ? o01.x : e01.x, w, m01[k].x);
        m01[k].y = __fmaf_rn((k & 1) ? o01.y : e01.y, w, m01[k].y);
        m23[k].x = __fmaf_rn((k & 1) ? o23.x : e23.x, w, m23[k].x);
        m23[k].y = __fmaf_rn((k & 1) ? o23.y : e23.y, w, m23[k].y);
      }
    }
  }
  // components in the order (11, 22, 33, 12, 13, 23)
  const float Dd[6] = {dx * dx, dy * dy, dz * dz, dx * dy, dx * dz, dy * dz};
  const float Sd[6] = {2.f * dx * tj.x, 2.f * dy * tj.y, 2.f * dz * tj.z, fmaf(dx, tj.y, dy * tj.x),
                       fmaf(dx, tj.z, dz * tj.x), fmaf(dy, tj.z, dz * tj.y)};
  const float Tt[6] = {tj.x * tj.x, tj.y * tj.y, tj.z * tj.z, tj.x * tj.y, tj.x * tj.z, tj.y * tj.z};
#pragma unroll
  for (int c = 0; c < 6; ++c)
#pragma unroll
    for (int k = 0; k < K1; ++k)
      gcol[(k * 6 + c) * GS] =
          fmaf(m01[k].y, Dd[c], fmaf(m23[k].x, Sd[c], fmaf(m23[k].y, Tt[c], c < 3 ? m01[k].x : 0.f)));
}

// One CTA's tile pair (I, J) of one suspension (the body of k_assemble_pairs and
// of the packed assembly, which maps its blocks onto many suspensions' tiles).
template <int M, int Q, int MODE, int INTEG, bool P2>
__device__ __forceinline__ void assemble_pair_tile(const Tables& tab, int N, const float4* __restrict__ pos,
                                                   const float4* __restrict__ ori, const AsmOut& out, int I, int J) {
  using S = AsmShape<M, Q>;
  constexpr int TI = S::TI, K1 = S::K1, NC = S::NC, H = S::H;
  constexpr int M3 = 3 * M;
  constexpr int FF = K1 * 3;   // force-term floats per fiber
  static_assert(Q % 2 == 0, "mirror folding needs an even number of quadrature points");

  __shared__ float4 sTi[TI], sTj[TI];    // orientations
  __shared__ float sD[TI][TI][3];        // x_i - x_j, formed in FP64 and rounded once (numerical)
  extern __shared__ __align__(16) float smem_dyn[];
  float (*sG)[S::GS] = reinterpret_cast<float (*)[S::GS]>(smem_dyn);                          // [NC][GS]
  float* const sTbase = smem_dyn + S::GOFF;                                                  // 2 x [TI][TP]
  __shared__ float sCoef[kMaxTerms], sEig[kMaxTerms];
  __shared__ float sfJ[TI][FF];
  __shared__ short sMapS[S::NQ32];   // stored value q (s32_block order) -> offset of its T entry within a pair

  // numerical: unordered tile pairs (I <= J), both blocks of a pair from one
  // evaluation of K; analytical: ordered tile pairs, direct blocks only
  constexpr bool SYM = INTEG == kNumerical;
  static_assert(SYM || MODE == kAsmDense, "structured storage needs the symmetric numerical blocks");
  const bool diag = (I == J);
  const int tid = threadIdx.x;
  const int i0 = I * TI, j0 = J * TI;

  if (tid < M) { sCoef[tid] = tab.gamma[tid]; sEig[tid] = tab.eigen[tid]; }
  if (tid < TI) {
    const int i = min(i0 + tid, N - 1), j = min(j0 + tid, N - 1);
    sTi[tid] = ori[i];
    sTj[tid] = ori[j];
  }
  if (SYM && tid < TI * TI) {
    const int a = tid / TI, c = tid % TI;
    const double4 xi = out.pos64[min(i0 + a, N - 1)], xj = out.pos64[min(j0 + c, N - 1)];
    sD[a][c][0] = (float)(xi.x - xj.x);
    sD[a][c][1] = (float)(xi.y - xj.y);
    sD[a][c][2] = (float)(xi.z - xj.z);
  }
  for (int k = tid; k < TI * FF; k += S::NT) (&sfJ[0][0])[k] = 0.f;
  constexpr bool STRUCT = MODE == kAsmStructF16 || MODE == kAsmStructBF16;
  constexpr bool APPLY = MODE == kAsmApply;
  // kAsmApply with a vector applies the blocks; without one it forms the force terms
  const bool do_apply = APPLY && out.x != nullptr;
  const bool do_force = !do_apply;
  constexpr int XW = APPLY ? TI * M3 : 1;
  __shared__ float sXi[XW], sXj[XW], sZj[XW];   // x rows of the I and J tiles, z_j of this tile's j
  if constexpr (APPLY) {
    if (do_apply) {
      for (int k = tid; k < TI * M3; k += S::NT) {
        const int f = k / M3, c = k % M3;
        sXi[k] = i0 + f < N ? out.x[(int64_t)(i0 + f) * M3 + c] : 0.f;
        sXj[k] = j0 + f < N ? out.x[(int64_t)(j0 + f) * M3 + c] : 0.f;
      }
    }
  }
  if constexpr (STRUCT) {
    for (int q = tid; q < S::NQ32; q += S::NT) {
      const int c = q % 6, blk = q / 6;
      int row = 0, col = 0;
      if (blk < M * M) {
        row = blk / M + 1;
        col = blk % M + 1;
      } else if (blk < M * M + K1) {
        col = blk - M * M;
      } else {
        row = blk - M * M - M;
      }
      sMapS[q] = (short)((row * K1 + col) * 6 + c);
    }
  }

  // own unit: u = qi * TI + il (a warp holds 32 / TI points of TI fibers)
  const int il = tid % TI, qi = tid / TI;
  const int i = i0 + il;
  const bool unit_ok = (tid < S::U) && (i < N);
  // numerical: the separation of quadrature points is formed as
  // (x_i - x_j) + s_qi t_i - s_qj t_j with the centre difference taken in
  // FP64 and rounded once, so its error scales with the fibers' distance
  // rather than with their distance from the origin (FP32 points x + s t far
  // from the origin lose ~1e-6 absolutely, which for nearly touching fibers
  // is ~1e-4 of the kernel)
  const float e2 = tab.e2;
  const float e2x3 = -3.f * e2;
  const float fz = tab.fz_half;

  // force-term accumulator of task (tl, k) = (tid / K1, tid % K1): F_i[k]
  float facc[3] = {0.f, 0.f, 0.f};
  // kAsmApply: z_i of task (tl, kI) = (tid / M, tid % M) over the tile's j
  float zacc[3] = {0.f, 0.f, 0.f};
  __syncthreads();

  const int jcount = min(TI, N - j0);
  for (int jl = 0; jl < jcount; ++jl) {
    // T is double-buffered: phase 2 of step jl+1 may run while phase 3 of
    // step jl still reads, so one barrier per step suffices after phase 2
    float* const sTflat = sTbase + (jl & 1) * (TI * S::TP);
    auto sT = [&](int tl, int k, int kj) -> float* { return sTflat + tl * S::TP + (k * K1 + kj) * 6; };
    // structured storage keeps T as [value q][i] (the storage record's own
    // order, so phase 3 is a straight copy); dense keeps [i][value]
    constexpr bool QT = STRUCT;
    auto tv = [&](int tl, int q) -> float& { return QT ? sTflat[q * TI + tl] : sTflat[tl * S::TP + q]; };
    const bool pair_ok = unit_ok && (!diag || (SYM ? il < jl : il != jl));
    // ---- phase 1: G[c][k] = sum_qj K_c(qi,qj) W[k][qj] (numerical, mirror-
    // folded over qj) or the closed-form integral (analytical)
    // G goes straight to shared memory, column k * 6 + c of unit tid
    float* const gcol = &sG[0][0] + tid;
    if (!SYM && tid < S::U) {
      float g[6][K1];
#pragma unroll
      for (int c = 0; c < 6; ++c)
#pragma unroll
        for (int k = 0; k < K1; ++k) g[c][k] = 0.f;
      if (pair_ok) {
        const double4 xi4 = out.pos64[i], ti4 = out.ori64[i];
        const double4 xj4 = out.pos64[j0 + jl], tj4 = out.ori64[j0 + jl];
        const double s = (double)tab.pts[qi];
        const double R0[3] = {xi4.x + s * ti4.x - xj4.x, xi4.y + s * ti4.y - xj4.y, xi4.z + s * ti4.z - xj4.z};
        const double tj[3] = {tj4.x, tj4.y, tj4.z};
        analytic_G<M>(R0, tj, 2.0 * (double)tab.eps * (double)tab.eps, g);
      }
#pragma unroll
      for (int c = 0; c < 6; ++c)
#pragma unroll
        for (int k = 0; k < K1; ++k) gcol[(k * 6 + c) * S::GS] = g[c][k];
    }
    if (SYM && pair_ok) {
      const float4 ti = sTi[il];
      const float si = tab.pts[qi];
      const float p[3] = {fmaf(si, ti.x, sD[il][jl][0]), fmaf(si, ti.y, sD[il][jl][1]),
                          fmaf(si, ti.z, sD[il][jl][2])};
      stokeslet_moments_G<K1, Q, S::GS, P2>(tab, p, sTj[jl], e2, e2x3, gcol);
    } else if (SYM && tid < S::U) {
#pragma unroll
      for (int c = 0; c < NC; ++c) gcol[c * S::GS] = 0.f;
    }
    __syncthreads();

    // ---- phase 2: T[ki][kj][c] = sum_qi W[ki][qi] G[qi][c][kj], folded over qi
    // lanes (col, tl), tl fastest; column col = kj * 6 + c.  P2: a lane takes
    // columns col and col + NC/2 in the two lanes of packed FP32 instructions
    // (lo - hi as fma(hi, -1, lo): the same rounding as the scalar subtraction)
    if constexpr (P2 && NC % 2 == 0) {
      constexpr int NC2 = NC / 2;
      for (int task = tid; task < TI * NC2; task += S::NT) {
        const int col = task / TI, tl = task % TI;
        const float* ga = &sG[col][tl];
        const float* gb = &sG[col + NC2][tl];
        float2 acc[K1];
#pragma unroll
        for (int k = 0; k < K1; ++k) acc[k] = make_float2(0.f, 0.f);
#pragma unroll
        for (int q = 0; q < H; ++q) {
          const float2 lo = make_float2(ga[q * TI], gb[q * TI]);
          const float2 hi = make_float2(ga[(Q - 1 - q) * TI], gb[(Q - 1 - q) * TI]);
          const float2 ev = __fadd2_rn(lo, hi), od = __ffma2_rn(hi, make_float2(-1.f, -1.f), lo);
#pragma unroll
          for (int k = 0; k < K1; ++k) acc[k] = __ffma2_rn((k & 1) ? od : ev, tab.W2[k][q], acc[k]);
        }
        const int kja = col / 6, ca = col % 6, kjb = (col + NC2) / 6, cb = (col + NC2) % 6;
#pragma unroll
        for (int k = 0; k < K1; ++k) {
          tv(tl, (k * K1 + kja) * 6 + ca) = acc[k].x;
          tv(tl, (k * K1 + kjb) * 6 + cb) = acc[k].y;
        }
      }
    } else {
      for (int task = tid; task < TI * NC; task += S::NT) {
        const int col = task / TI, tl = task % TI;
        const int kj = col / 6, c = col % 6;
        const float* gp = &sG[col][tl];
        float acc[K1];
#pragma unroll
        for (int k = 0; k < K1; ++k) acc[k] = 0.f;
#pragma unroll
        for (int q = 0; q < H; ++q) {
          const float lo = gp[q * TI], hi = gp[(Q - 1 - q) * TI];
          const float ev = __fadd_rn(lo, hi), od = __fsub_rn(lo, hi);
#pragma unroll
          for (int k = 0; k < K1; ++k) acc[k] = __fmaf_rn((k & 1) ? od : ev, tab.W[k][q], acc[k]);
        }
#pragma unroll
        for (int k = 0; k < K1; ++k) tv(tl, (k * K1 + kj) * 6 + c) = acc[k];
      }
    }
    __syncthreads();

    const int j = j0 + jl;
    if constexpr (MODE == kAsmDense) {
      // ---- phase 3a: block (i, j) -- rows of fiber i, columns of fiber j
      for (int task = tid; task < TI * M * M; task += S::NT) {
        const int kJp = task / (TI * M), rem = task % (TI * M);
        const int tl = rem / M, kIp = rem % M;
        const int ii = i0 + tl;
        if (ii >= N || (SYM && diag && tl > jl)) continue;
        float* dst = out.A + (int64_t)(i0 * M3 + 3 * rem) + (int64_t)(j * M3 + 3 * kJp) * out.lda;
        if (diag && tl == jl) {
#pragma unroll
          for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int a = 0; a < 3; ++a) dst[a + b * out.lda] = (kIp == kJp && a == b) ? 1.f : 0.f;
          continue;
        }
        const float* T6 = sT(tl, kIp + 1, kJp + 1);
        const float4 ti = sTi[tl];
        const float t3[3] = {ti.x, ti.y, ti.z};
        float Qv[3];
#pragma unroll
        for (int b = 0; b < 3; ++b)
          Qv[b] = sym_get(T6, b, 0) * t3[0] + sym_get(T6, b, 1) * t3[1] + sym_get(T6, b, 2) * t3[2];
        const float coef = sCoef[kIp], E = sEig[kIp];
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
          for (int a = 0; a < 3; ++a)
            dst[a + b * out.lda] = kIp == 0 ? coef * t3[a] * Qv[b] : coef * (sym_get(T6, a, b) - E * t3[a] * Qv[b]);
      }
      // ---- phase 3b: block (j, i) -- rows of fiber j, columns of fiber i
      if (SYM) {
        const float4 tj = sTj[jl];
        const float t3[3] = {tj.x, tj.y, tj.z};
        for (int task = tid; task < TI * M * M; task += S::NT) {
          const int tl = task / (M * M), rem = task % (M * M);
          const int kIp = rem / M, kJp = rem % M;
          const int ii = i0 + tl;
          if (ii >= N || (diag && tl >= jl)) continue;
          float* dst = out.A + (int64_t)(j * M3 + 3 * kJp) + (int64_t)(ii * M3 + 3 * kIp) * out.lda;
          const float* T6 = sT(tl, kIp + 1, kJp + 1);
          float Qv[3];
#pragma unroll
          for (int b = 0; b < 3; ++b)
            Qv[b] = sym_get(T6, b, 0) * t3[0] + sym_get(T6, b, 1) * t3[1] + sym_get(T6, b, 2) * t3[2];
          const float coef = sCoef[kJp], E = sEig[kJp];
#pragma unroll
          for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int a = 0; a < 3; ++a)
              dst[a + b * out.lda] = kJp == 0 ? coef * t3[a] * Qv[b] : coef * (sym_get(T6, a, b) - E * t3[a] * Qv[b]);
        }
      }
    } else if constexpr (APPLY) {
      // ---- phase 3 (matrix-free product): z_i[kI] += sum_kJ T(kI+1, kJ+1) x_j[kJ]
      // for the i side and z_j[kJ] += sum_kI T(kI+1, kJ+1) x_i[kI] for the j side
      // (each 3x3 block symmetric; blocks of pairs that do not exist are zero)
      if (do_apply) {
        if (tid < TI * M) {
          const int tl = tid / M, kI = tid % M;
#pragma unroll
          for (int kJ = 0; kJ < M; ++kJ) {
            const float* T6 = sT(tl, kI + 1, kJ + 1);
            const float* xv = &sXj[jl * M3 + 3 * kJ];
#pragma unroll
            for (int a = 0; a < 3; ++a)
              zacc[a] = fmaf(sym_get(T6, a, 0), xv[0], fmaf(sym_get(T6, a, 1), xv[1], fmaf(sym_get(T6, a, 2), xv[2], zacc[a])));
          }
        }
        // j side: lanes (kJ, tl) of whole warps from thread 64, TI-lane sums
        constexpr int JW = (M * TI + 31) / 32 * 32;
        static_assert(64 + JW <= S::NT && 32 % TI == 0, "j-side lanes of the matrix-free product");
        if (tid >= 64 && tid < 64 + JW) {
          const int u = tid - 64, kJ = u / TI, tl = u % TI;
          float zs[3] = {0.f, 0.f, 0.f};
          if (kJ < M) {
#pragma unroll
            for (int kI = 0; kI < M; ++kI) {
              const float* T6 = sT(tl, kI + 1, kJ + 1);
              const float* xv = &sXi[tl * M3 + 3 * kI];
#pragma unroll
              for (int a = 0; a < 3; ++a)
                zs[a] = fmaf(sym_get(T6, a, 0), xv[0], fmaf(sym_get(T6, a, 1), xv[1], fmaf(sym_get(T6, a, 2), xv[2], zs[a])));
            }
          }
#pragma unroll
          for (int o = TI / 2; o > 0; o >>= 1)
#pragma unroll
            for (int a = 0; a < 3; ++a) zs[a] += __shfl_xor_sync(0xffffffffu, zs[a], o);
          if (tl == 0 && kJ < M)
#pragma unroll
            for (int a = 0; a < 3; ++a) sZj[jl * M3 + 3 * kJ + a] = zs[a];
        }
      }
    } else {
      // ---- phase 3: the pair blocks into structured storage; one j, all i of
      // the tile: [jl][q][tl] is a contiguous run of NQ32*TI floats
      const int I16 = I / S::SUB, J16 = J / S::SUB;
      const int sub = (I % S::SUB) * S::SUB + (J % S::SUB);
      const int64_t L16 = (int64_t)J16 * (J16 + 1) / 2 + I16;
      const int64_t rec = (L16 * S::SUB * S::SUB + sub) * TI + jl;
      // T is [q][tl] with q in (row, col) order; stored in s32_block order.
      // Pairs that do not exist (i >= N, i >= j on a diagonal tile) came out
      // of phases 1-2 as exact zeros.  No FP32 copy in the recompute modes
      // (out.S32 null: the residual and the velocities form the blocks again)
      if (out.S32 != nullptr) {
        float* d32 = out.S32 + rec * (int64_t)(S::NQ32 * TI);
        for (int v = tid; v < S::NQ32 * TI / 4; v += S::NT) {
          const int q = v / (TI / 4), g4 = (v % (TI / 4)) * 4;
          reinterpret_cast<float4*>(d32)[v] = *reinterpret_cast<const float4*>(&sTflat[sMapS[q] * TI + g4]);
        }
      }
      // 16-bit records [tl][NW]: pair tl's words are contiguous; a warp stores
      // 64-byte runs of 8 records
      constexpr int NW = s16_record_words(M);
      uint32_t* d16 = out.S16 + rec * (int64_t)(NW * TI);
      for (int v = tid; v < TI * NW / 4; v += S::NT) {
        const int tl = v % TI, w4 = v / TI;
        uint32_t w[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int q2 = 4 * w4 + u;
          const float lo = q2 < S::NQ16 ? sTflat[sMapS[2 * q2] * TI + tl] : 0.f;
          const float hi = q2 < S::NQ16 ? sTflat[sMapS[2 * q2 + 1] * TI + tl] : 0.f;
          if constexpr (MODE == kAsmStructF16) {
            __half2 hv = __floats2half2_rn(lo, hi);
            w[u] = *reinterpret_cast<uint32_t*>(&hv);
          } else {
            __nv_bfloat162 hv = __floats2bfloat162_rn(lo, hi);
            w[u] = *reinterpret_cast<uint32_t*>(&hv);
          }
        }
        *reinterpret_cast<uint4*>(&d16[tl * NW + 4 * w4]) = make_uint4(w[0], w[1], w[2], w[3]);
      }
    }
    // ---- phase 3c: force terms F_i[k] += T^{ij}[k][P0] F/2 and
    //      F_j[kj] += T^{ij}[P0][kj] F/2 (F/2 = (0, 0, fz): column z of the block)
    if (do_force && tid < TI * K1) {
      const int tl = tid / K1, k = tid % K1;
      if (i0 + tl < N && (!diag || (SYM ? tl < jl : tl != jl))) {
        const int q0 = (k * K1 + 0) * 6;
        facc[0] = fmaf(tv(tl, q0 + 4), fz, facc[0]);
        facc[1] = fmaf(tv(tl, q0 + 5), fz, facc[1]);
        facc[2] = fmaf(tv(tl, q0 + 2), fz, facc[2]);
      }
    }
    if (SYM && do_force && tid < K1) {
      const int kj = tid;
      float s[3] = {0.f, 0.f, 0.f};
      for (int tl = 0; tl < TI; ++tl) {
        if (i0 + tl >= N || (diag && tl >= jl)) continue;
        const int q0 = (0 * K1 + kj) * 6;
        s[0] = fmaf(tv(tl, q0 + 4), fz, s[0]);
        s[1] = fmaf(tv(tl, q0 + 5), fz, s[1]);
        s[2] = fmaf(tv(tl, q0 + 2), fz, s[2]);
      }
#pragma unroll
      for (int a = 0; a < 3; ++a) sfJ[jl][3 * kj + a] += s[a];
    }
  }
  __syncthreads();

  if constexpr (APPLY) {
    if (do_apply) {
      // partial rows of z: the i side of tile (I, J) to slot J, the j side to
      // slot I (a diagonal tile's j side to slot T8): every slot of every
      // fiber is written exactly once per product
      const int64_t R = (int64_t)M3 * N;
      const int T8 = (N + TI - 1) / TI;
      if (tid < TI * M) {
        const int tl = tid / M, kI = tid % M;
        if (i0 + tl < N) {
          float* dst = out.zpart + (int64_t)J * R + (int64_t)(i0 + tl) * M3 + 3 * kI;
#pragma unroll
          for (int a = 0; a < 3; ++a) dst[a] = zacc[a];
        }
      }
      float* zj = out.zpart + (int64_t)(diag ? T8 : I) * R + (int64_t)j0 * M3;
      for (int k = tid; k < TI * M3; k += S::NT)
        if (j0 + k / M3 < N) zj[k] = sZj[k];
      return;
    }
  }
  // ---- partial force terms: ffpart[X][fiber of Y][k][3] written exactly once
  float* ffpart = out.ffpart;
  if (tid < TI * K1) {
    const int tl = tid / K1, k = tid % K1;
    if (i0 + tl < N) {
      float v[3] = {facc[0], facc[1], facc[2]};
      if (SYM && diag) {
#pragma unroll
        for (int a = 0; a < 3; ++a) v[a] += sfJ[tl][3 * k + a];
      }
      float* dst = ffpart + ((int64_t)J * N + i0 + tl) * FF + 3 * k;
#pragma unroll
      for (int a = 0; a < 3; ++a) dst[a] = v[a];
    }
  }
  if (SYM && !diag) {
    for (int k = tid; k < TI * FF; k += S::NT) {
      const int jl = k / FF;
      if (j0 + jl < N) ffpart[((int64_t)I * N + j0) * FF + k] = (&sfJ[0][0])[k];
    }
  }
}

template <int M, int Q, int MODE, int INTEG, bool P2>
__global__ void __launch_bounds__(192, INTEG == kNumerical ? 4 : 2)
k_assemble_pairs(const Tables tab, int N, const float4* __restrict__ pos, const float4* __restrict__ ori,
                 AsmOut out) {
  if (MODE == kAsmApply && out.skip != nullptr && *out.skip) return;
  int I, J;
  asm_tile_of<Q, INTEG>(N, blockIdx.x, I, J);
  assemble_pair_tile<M, Q, MODE, INTEG, P2>(tab, N, pos, ori, out, I, J);
}

// F[i][k] = sum_X ffpart[X][i][k] (fixed order); b[i][k'] = -C_i(k') F[i][k'+1]
// for unit u = (i, k) of N (M + 1).
__device__ __forceinline__ void force_term_unit(const Tables& tab, int N, const float4* __restrict__ ori,
                                                const float* __restrict__ ffpart, int nparts, float* __restrict__ F,
                                                float* __restrict__ b, int64_t u) {
  const int M = tab.M, K1 = M + 1, FFn = 3 * K1;
  {
    const int i = (int)(u / K1), k = (int)(u % K1);
    float s[3] = {0.f, 0.f, 0.f};
    for (int p = 0; p < nparts; ++p) {
      const float* src = ffpart + ((int64_t)p * N + i) * FFn + 3 * k;
      s[0] += src[0]; s[1] += src[1]; s[2] += src[2];
    }
    float* f = F + (int64_t)i * FFn + 3 * k;
    f[0] = s[0]; f[1] = s[1]; f[2] = s[2];
    if (k >= 1) {
      const int kp = k - 1;
      const float4 t = ori[i];
      const float t3[3] = {t.x, t.y, t.z};
      const float QF = s[0] * t3[0] + s[1] * t3[1] + s[2] * t3[2];
      const float coef = tab.gamma[kp], E = tab.eigen[kp];
      float* dst = b + (int64_t)i * 3 * M + 3 * kp;
#pragma unroll
      for (int a = 0; a < 3; ++a) dst[a] = kp == 0 ? -coef * t3[a] * QF : -coef * (s[a] - E * t3[a] * QF);
    }
  }
}

__global__ void k_force_terms(const Tables tab, int N, const float4* __restrict__ ori,
                              const float* __restrict__ ffpart, int nparts, float* __restrict__ F,
                              float* __restrict__ b) {
  const int64_t n = (int64_t)N * (tab.M + 1);
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x)
    force_term_unit(tab, N, ori, ffpart, nparts, F, b, u);
}

// ---- packed step: every member of a group (one Tables) in one launch ------
// Block b belongs to the member whose tile pairs it falls in; the member's
// blocks run exactly the single-suspension kernel's tile code, so a member's
// system is bit for bit the one k_assemble_pairs forms.
template <int MODE>
__global__ void __launch_bounds__(192, 4)
k_pack_assemble(const Tables tab, const PackStepMember* __restrict__ mem, int n) {
  const int L = (int)blockIdx.x;
  const PackStepMember& p = mem[pack_member_of(n, L, [&](int m) { return mem[m].asm_start; })];
  AsmOut out{};
  out.S32 = p.S32;
  out.S16 = p.S16;
  out.ffpart = p.ffpart;
  out.pos64 = p.pos64;
  int I, J;
  asm_tile_of<24, kNumerical>(p.N, (unsigned)(L - p.asm_start), I, J);
  assemble_pair_tile<5, 24, MODE, kNumerical, false>(tab, p.N, p.pos32, p.ori32, out, I, J);
}

// one block per member: its force terms and right-hand side
__global__ void __launch_bounds__(256) k_pack_force_terms(const Tables tab, const PackStepMember* __restrict__ mem) {
  const PackStepMember& p = mem[blockIdx.x];
  const int N = p.N;
  const int64_t n = (int64_t)N * (tab.M + 1);
  const int nparts = (N + AsmShape<5, 24>::TI - 1) / AsmShape<5, 24>::TI;
  for (int64_t u = threadIdx.x; u < n; u += blockDim.x) force_term_unit(tab, N, p.ori32, p.ffpart, nparts, p.F, p.b, u);
}

int launch_pack_assemble(const Tables& tab, const PackStepMember* members, int n, int64_t blocks, bool bf16,
                         cudaStream_t st) {
  if (tab.M != 5 || tab.Q != 24 || n < 1 || blocks < 1) return RF_E_UNSUPPORTED;
  constexpr size_t smem = AsmShape<5, 24>::kSmem;
  if (bf16) {
    static const cudaError_t attr = cudaFuncSetAttribute(k_pack_assemble<kAsmStructBF16>,
                                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    RF_CUDA_TRY(attr);
    k_pack_assemble<kAsmStructBF16><<<(unsigned)blocks, 192, smem, st>>>(tab, members, n);
  } else {
    static const cudaError_t attr = cudaFuncSetAttribute(k_pack_assemble<kAsmStructF16>,
                                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    RF_CUDA_TRY(attr);
    k_pack_assemble<kAsmStructF16><<<(unsigned)blocks, 192, smem, st>>>(tab, members, n);
  }
  RF_LAUNCH_CHECK();
  k_pack_force_terms<<<(unsigned)n, 256, 0, st>>>(tab, members);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

// out[r] = sum over parts p of part[p][r], fixed order.
__global__ void k_reduce_rows(const float* __restrict__ part, int nparts, int64_t R, float* __restrict__ out) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < R; r += (int64_t)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int p = 0; p < nparts; ++p) s += part[(int64_t)p * R + r];
    out[r] = s;
  }
}

int launch_reduce_rows(const float* part, int nparts, int64_t R, float* out, cudaStream_t st) {
  const int threads = 256;
  const int blocks = (int)std::min<int64_t>(ceil_div(R, threads), 148 * 8);
  k_reduce_rows<<<blocks, threads, 0, st>>>(part, nparts, R, out);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

int assemble_tiles(int M, int Q, int N) { return (int)ceil_div(N, 192 / Q); }

int64_t struct_store_tiles(int N) {
  const int64_t T16 = ceil_div(N, kStoreTile);
  return T16 * (T16 + 1) / 2;
}

int64_t struct_floats32(int M, int N) {
  return struct_store_tiles(N) * (int64_t)kStoreTile * kStoreTile * (M + 1) * (M + 1) * 6;
}

int64_t struct_words16(int M, int N) {
  return struct_store_tiles(N) * (int64_t)kStoreTile * kStoreTile * s16_record_words(M);
}

template <int M, int Q, int MODE, int INTEG, bool P2>
static int launch_pairs(const Tables& tab, int N, const float4* pos, const float4* ori, const AsmOut& out,
                        cudaStream_t st) {
  using S = AsmShape<M, Q>;
  const int64_t T = ceil_div(N, S::TI);
  const int64_t ntp = INTEG == kNumerical ? T * (T + 1) / 2 : T * T;
  // once per process (thread-safe static initialisation; handles of a serving
  // loop launch from several threads)
  static const cudaError_t attr = cudaFuncSetAttribute(k_assemble_pairs<M, Q, MODE, INTEG, P2>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::kSmem);
  RF_CUDA_TRY(attr);
  k_assemble_pairs<M, Q, MODE, INTEG, P2><<<(unsigned)ntp, 192, S::kSmem, st>>>(tab, N, pos, ori, out);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

template <int M, int Q, int MODE, int INTEG>
static int launch_assemble_mq(const Tables& tab, int N, const float4* pos, const float4* ori, const AsmOut& out,
                              float* F, float* b, int variant, cudaStream_t st) {
  using S = AsmShape<M, Q>;
  const int64_t T = ceil_div(N, S::TI);
  if (INTEG == kNumerical && variant == 1) {
    RF_TRY_RF((launch_pairs<M, Q, MODE, INTEG, INTEG == kNumerical>(tab, N, pos, ori, out, st)));
  } else {
    RF_TRY_RF((launch_pairs<M, Q, MODE, INTEG, false>(tab, N, pos, ori, out, st)));
  }
  if (MODE == kAsmApply && out.x != nullptr) return RF_OK;   // the product: no force terms
  const int64_t n = (int64_t)N * (M + 1);
  k_force_terms<<<(unsigned)std::min<int64_t>(ceil_div(n, 256), 148 * 8), 256, 0, st>>>(tab, N, ori, out.ffpart,
                                                                                         (int)T, F, b);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

template <int MODE, int INTEG>
static int dispatch_assemble(const Tables& tab, int N, const float4* pos, const float4* ori, const AsmOut& out,
                             float* F, float* b, int variant, cudaStream_t st) {
  if (variant < 0 || variant >= kAsmVariants) {
    set_last_error_str("assemble: unknown kernel variant");
    return RF_E_INPUT;
  }
#define RF_ASM_CASE(MM, QQ) \
  if (tab.M == MM && tab.Q == QQ)  \
    return launch_assemble_mq<MM, QQ, MODE, INTEG>(tab, N, pos, ori, out, F, b, variant, st);
  RF_FOR_EACH_MQ(RF_ASM_CASE)
#undef RF_ASM_CASE
  set_last_error_str("assemble: (M, Q) combination not instantiated");
  return RF_E_UNSUPPORTED;
}

int launch_assemble_numerical(const Tables& tab, int N, const float4* pos, const float4* ori, const double4* pos64,
                              float* A, int64_t lda, float* ffpart, float* F, float* b, cudaStream_t st,
                              int variant) {
  AsmOut out{};
  out.pos64 = pos64;
  out.A = A;
  out.lda = lda;
  out.ffpart = ffpart;
  return dispatch_assemble<kAsmDense, kNumerical>(tab, N, pos, ori, out, F, b, variant, st);
}

int launch_assemble_analytical(const Tables& tab, int N, const float4* pos, const float4* ori,
                               const double4* pos64, const double4* ori64, float* A, int64_t lda, float* ffpart,
                               float* F, float* b, cudaStream_t st) {
  AsmOut out{};
  out.pos64 = pos64;
  out.ori64 = ori64;
  out.A = A;
  out.lda = lda;
  out.ffpart = ffpart;
  return dispatch_assemble<kAsmDense, kAnalytical>(tab, N, pos, ori, out, F, b, 0, st);
}

int launch_assemble_apply(const Tables& tab, int N, const float4* pos, const float4* ori, const double4* pos64,
                          const float* x, float* zpart, const int* skip, float* ffpart, float* F, float* b,
                          cudaStream_t st, int variant) {
  AsmOut out{};
  out.pos64 = pos64;
  out.x = x;
  out.zpart = zpart;
  out.skip = skip;
  out.ffpart = ffpart;
  return dispatch_assemble<kAsmApply, kNumerical>(tab, N, pos, ori, out, F, b, variant, st);
}

int launch_assemble_structured(const Tables& tab, int N, const float4* pos, const float4* ori, const double4* pos64,
                               float* S32, uint32_t* S16, bool bf16, float* ffpart, float* F, float* b,
                               cudaStream_t st, int variant) {
  AsmOut out{};
  out.pos64 = pos64;
  out.S32 = S32;
  out.S16 = S16;
  out.ffpart = ffpart;
  if (bf16) return dispatch_assemble<kAsmStructBF16, kNumerical>(tab, N, pos, ori, out, F, b, variant, st);
  return dispatch_assemble<kAsmStructF16, kNumerical>(tab, N, pos, ori, out, F, b, variant, st);
}

}  // namespace rf
