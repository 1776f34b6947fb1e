// Direct solver: blocked right-looking LU with partial pivoting, triangular
// solves and FP64-residual iterative refinement.
//
// Replaces the reference's direct path: MAGMA magma_sgesv_gpu on the GPU
// (src/simulation.cu:403-418, --magma) and LAPACK sgesv on the CPU
// (fortran/solve_system.incl:117-119).  Both factor A = P L U in FP32 with
// partial pivoting (row of the largest |a_ij| in the column, first one on
// ties, as LAPACK's isamax) and solve L U x = P b.  Written here from the
// textbook blocked algorithm (Golub & Van Loan, alg. 3.4.2):
//   for each panel of nb columns:
//     factor the panel (rows k..R) with partial pivoting    k_lu_panel (cooperative)
//     apply the panel's row swaps to the other columns      k_lu_laswp
//     U12 = L11^{-1} A12                                    k_lu_trsm
//     A22 -= L21 U12                                        k_lu_gemm
// The factorization overwrites a copy of A; the original stays for the
// refinement residual r = b - A x, accumulated in FP64, and x is corrected
// with the factors until ||r|| / ||b|| meets the tolerance.
#include <cooperative_groups.h>

#include <algorithm>
#include <climits>
#include <cmath>

#include "rf_common.cuh"
#include "rf_kernels.cuh"
#include "rf_lu.cuh"

namespace cg = cooperative_groups;

namespace rf {

// ---------------------------------------------------------------------------
// panel: columns [k, k+nb) over rows [k, R).  Per column j: (pivot search
// fused with the previous column's update) -> grid sync -> swap (block 0) ->
// grid sync -> scale + rank-1 update of the remaining panel columns with the
// next column's partial max -> grid sync ...
// ---------------------------------------------------------------------------
struct PanelArgs {
  float* A;
  int64_t lda;
  int64_t R;
  int64_t k;
  int nb;
  int* ipiv;
  float* pmax;   // per-block partial max |a|
  int* pidx;     // per-block partial argmax
  int* info;     // first zero pivot (1-based), 0 if none
};

__device__ __forceinline__ void better(float& bv, int& bi, float v, int i) {
  // larger |value| wins; equal values: the smaller row index (first occurrence)
  if (v > bv || (v == bv && i < bi)) { bv = v; bi = i; }
}

__device__ void block_argmax(float v, int i, float* pmax, int* pidx) {
  __shared__ float sv[32];
  __shared__ int si[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float ov = __shfl_down_sync(0xffffffffu, v, o);
    const int oi = __shfl_down_sync(0xffffffffu, i, o);
    better(v, i, ov, oi);
  }
  if (lane == 0) { sv[wid] = v; si[wid] = i; }
  __syncthreads();
  if (threadIdx.x == 0) {
    float bv = sv[0];
    int bi = si[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) better(bv, bi, sv[w], si[w]);
    pmax[blockIdx.x] = bv;
    pidx[blockIdx.x] = bi;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(256) k_lu_panel(PanelArgs a) {
  cg::grid_group grid = cg::this_grid();
  __shared__ int s_piv;
  __shared__ float s_pabs;
  const int64_t R = a.R, lda = a.lda, k = a.k;
  const int nb = a.nb;
  float* A = a.A;
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t nth = (int64_t)gridDim.x * blockDim.x;
  // partial max of the first panel column
  {
    float bv = -1.f;
    int bi = INT_MAX;
    for (int64_t r = k + tid; r < R; r += nth) better(bv, bi, fabsf(A[r + k * lda]), (int)r);
    block_argmax(bv, bi, a.pmax, a.pidx);
  }
  for (int jj = 0; jj < nb; ++jj) {
    const int64_t j = k + jj;
    grid.sync();
    // every block reduces the partials the same way
    if (threadIdx.x == 0) {
      float bv = -1.f;
      int bi = INT_MAX;
      for (int b = 0; b < (int)gridDim.x; ++b) better(bv, bi, a.pmax[b], a.pidx[b]);
      s_piv = bi;
      s_pabs = bv;
    }
    __syncthreads();
    const int64_t p = s_piv;
    // swap rows j and p inside the panel (block 0), record the pivot
    if (blockIdx.x == 0) {
      for (int c = threadIdx.x; c < nb; c += blockDim.x) {
        const int64_t col = (k + c) * lda;
        const float t = A[j + col];
        A[j + col] = A[p + col];
        A[p + col] = t;
      }
      if (threadIdx.x == 0) {
        a.ipiv[j] = (int)p;
        // the largest |a_ij| of the column is the pivot's magnitude
        if (!(s_pabs > 0.f) && *a.info == 0) *a.info = (int)(j + 1);
      }
    }
    grid.sync();
    // scale column j below the diagonal, update the remaining panel columns,
    // partial max of the next column
    const float piv = A[j + j * lda];
    const float inv = piv != 0.f ? 1.f / piv : 0.f;
    float bv = -1.f;
    int bi = INT_MAX;
    for (int64_t r = j + 1 + tid; r < R; r += nth) {
      const float l = A[r + j * lda] * inv;
      A[r + j * lda] = l;
      for (int c = jj + 1; c < nb; ++c) {
        const int64_t col = (k + c) * lda;
        A[r + col] = fmaf(-l, A[j + col], A[r + col]);
      }
      if (jj + 1 < nb) better(bv, bi, fabsf(A[r + (j + 1) * lda]), (int)r);
    }
    if (jj + 1 < nb) block_argmax(bv, bi, a.pmax, a.pidx);
  }
}

// ---------------------------------------------------------------------------
// The same panel factorisation with the panel held in shared memory: block b
// owns rows [k + b*rows_per, ...) of the panel's nb columns (column-major in
// shared memory) for the whole kernel, so the panel is read and written once,
// and one grid sync per column suffices: before it, every block publishes its
// candidate pivot (largest |a| of the column among its rows, smallest row on
// ties) together with that row's values, and the owner of the diagonal row
// publishes it; after it, every block reduces the candidates in the same way,
// the owners of the two rows exchange them, and each block scales and updates
// its rows and publishes the next column's candidate.  The candidate buffers
// alternate by column parity.  Per element the arithmetic is that of
// k_lu_panel (a * (1 / pivot), then fmaf(-l, u, a) per column), so both give
// the same factors.
// ---------------------------------------------------------------------------
struct PanelSmArgs {
  float* A;
  int64_t lda, R, k;
  int nb, rows_per;
  int* ipiv;
  float* pmax;   // [2][gridDim.x]
  int* pidx;     // [2][gridDim.x]
  float* prow;   // [2][gridDim.x][64]
  float* jrow;   // [2][64]
  int* info;
};

constexpr int kPanelSmemBytes = 192 * 1024;

__global__ void __launch_bounds__(256) k_lu_panel_smem(PanelSmArgs a) {
  cg::grid_group grid = cg::this_grid();
  extern __shared__ float sp[];   // [nb][rows_per]
  __shared__ float s_prow[64];
  __shared__ int s_p, s_loc;
  __shared__ float s_pabs;
  const int nb = a.nb, rp = a.rows_per, nblk = (int)gridDim.x;
  const int64_t k = a.k, R = a.R, lda = a.lda;
  const int64_t r0 = k + (int64_t)blockIdx.x * rp;
  const int nloc = (int)max((int64_t)0, min((int64_t)rp, R - r0));
  float* A = a.A;
  for (int c = 0; c < nb; ++c)
    for (int r = threadIdx.x; r < nloc; r += blockDim.x) sp[c * rp + r] = A[r0 + r + (k + c) * lda];
  __syncthreads();
  // candidate of column jj (rows >= k + jj) into buffer buf, and the diagonal row
  auto publish = [&](int jj, int buf) {
    float bv = -1.f;
    int bi = INT_MAX;
    for (int r = threadIdx.x; r < nloc; r += blockDim.x)
      if (r0 + r >= k + jj) better(bv, bi, fabsf(sp[jj * rp + r]), (int)(r0 + r));
    block_argmax(bv, bi, a.pmax + buf * nblk, a.pidx + buf * nblk);   // writes [blockIdx.x], syncs
    if (threadIdx.x == 0) s_loc = a.pidx[buf * nblk + blockIdx.x];
    __syncthreads();
    const int loc = s_loc;
    if (loc != INT_MAX && threadIdx.x < nb)
      a.prow[((int64_t)buf * nblk + blockIdx.x) * 64 + threadIdx.x] = sp[threadIdx.x * rp + (loc - r0)];
    const int64_t j = k + jj;
    if (j >= r0 && j < r0 + nloc && threadIdx.x < nb) a.jrow[buf * 64 + threadIdx.x] = sp[threadIdx.x * rp + (j - r0)];
  };
  publish(0, 0);
  for (int jj = 0; jj < nb; ++jj) {
    const int buf = jj & 1;
    const int64_t j = k + jj;
    grid.sync();
    if (threadIdx.x < 32) {
      float bv = -1.f;
      int bi = INT_MAX;
      for (int b = threadIdx.x; b < nblk; b += 32) better(bv, bi, a.pmax[buf * nblk + b], a.pidx[buf * nblk + b]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_down_sync(0xffffffffu, bv, o);
        const int oi = __shfl_down_sync(0xffffffffu, bi, o);
        better(bv, bi, ov, oi);
      }
      if (threadIdx.x == 0) { s_p = bi; s_pabs = bv; }
    }
    __syncthreads();
    const int64_t p = s_p == INT_MAX ? j : (int64_t)s_p;   // an all-zero column keeps its row
    const int bw = (int)((p - k) / rp);
    if (threadIdx.x < nb) s_prow[threadIdx.x] = a.prow[((int64_t)buf * nblk + bw) * 64 + threadIdx.x];
    __syncthreads();
    if (p != j && threadIdx.x < nb) {
      if (j >= r0 && j < r0 + nloc) sp[threadIdx.x * rp + (j - r0)] = s_prow[threadIdx.x];
      if (p >= r0 && p < r0 + nloc) sp[threadIdx.x * rp + (p - r0)] = a.jrow[buf * 64 + threadIdx.x];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      a.ipiv[j] = (int)p;
      if (!(s_pabs > 0.f) && *a.info == 0) *a.info = (int)(j + 1);
    }
    __syncthreads();
    const float piv = s_prow[jj];
    const float inv = piv != 0.f ? 1.f / piv : 0.f;
    for (int r = threadIdx.x; r < nloc; r += blockDim.x) {
      if (r0 + r <= j) continue;
      const float l = sp[jj * rp + r] * inv;
      sp[jj * rp + r] = l;
      for (int c = jj + 1; c < nb; ++c) sp[c * rp + r] = fmaf(-l, s_prow[c], sp[c * rp + r]);
    }
    __syncthreads();
    if (jj + 1 < nb) publish(jj + 1, buf ^ 1);
  }
  __syncthreads();
  for (int c = 0; c < nb; ++c)
    for (int r = threadIdx.x; r < nloc; r += blockDim.x) A[r0 + r + (k + c) * lda] = sp[c * rp + r];
}

// Row swaps of the panel [k, k+nb) on the columns outside it.
__global__ void k_lu_laswp(float* __restrict__ A, int64_t lda, int64_t R, int64_t k, int nb,
                           const int* __restrict__ ipiv) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= R || (c >= k && c < k + nb)) return;
  float* col = A + c * lda;
  for (int jj = 0; jj < nb; ++jj) {
    const int64_t j = k + jj, p = ipiv[j];
    if (p != j) {
      const float t = col[j];
      col[j] = col[p];
      col[p] = t;
    }
  }
}

// U12 = L11^{-1} A12 for columns [k+nb, R): one thread per column, L11
// (unit lower, nb x nb) in shared memory.
template <int NB>
__global__ void __launch_bounds__(256) k_lu_trsm(float* __restrict__ A, int64_t lda, int64_t R, int64_t k) {
  __shared__ float L[NB][NB + 1];
  for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
    const int r = e % NB, c = e / NB;
    L[r][c] = A[(k + r) + (k + c) * lda];
  }
  __syncthreads();
  const int64_t c = k + NB + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= R) return;
  float x[NB];
  float* col = A + c * lda + k;
#pragma unroll
  for (int r = 0; r < NB; ++r) x[r] = col[r];
#pragma unroll
  for (int r = 0; r < NB; ++r) {
#pragma unroll
    for (int q = r + 1; q < NB; ++q) x[q] = fmaf(-L[q][r], x[r], x[q]);
  }
#pragma unroll
  for (int r = 0; r < NB; ++r) col[r] = x[r];
}

// C -= A_panel * B_panel on the trailing block: C = A[k+nb.., k+nb..],
// A_panel = A[k+nb.., k..k+nb) (L21), B_panel = A[k..k+nb, k+nb..) (U12).
// Trailing update A22 -= L21 U12 on the tensor cores (mma.sync m16n8k8, TF32
// inputs, FP32 accumulation).  SPLIT = false: one TF32 product (the operands
// keep 10 mantissa bits; the FP64 refinement wins the accuracy back).  SPLIT =
// true: a = a_hi + a_lo (both TF32) and a b ~ a_hi b_hi + a_hi b_lo + a_lo
// b_hi, three products with FP32-level accuracy, for matrices whose
// conditioning makes the refinement of TF32 factors stall.
// 128x128 output tile per CTA, 8 warps of 64x32; K = NB in chunks of 32 staged
// through shared memory with float4 loads (L21 columns and U12 columns are both
// contiguous in the column-major matrix).  Padded strides put the fragment
// loads on distinct banks: a (row g, k t) at 8t + g, b (k t, col g) at 4g + t.
// The output is updated straight from the accumulator fragments: each column's
// 8 consecutive rows fill a 32-byte sector.
__device__ __forceinline__ uint32_t tf32_bits(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

template <int NB, bool SPLIT>
__global__ void __launch_bounds__(256, 1) k_lu_gemm(float* __restrict__ A, int64_t lda, int64_t R, int64_t k,
                                                    bool vec4) {
  constexpr int TM = 128, TN = 128, TK = NB;
  constexpr int LA = TM + 8, LB = TK + 4;
  extern __shared__ __align__(16) float gsm[];
  float* sa = gsm;              // [k][m], -L21
  float* sb = gsm + TK * LA;    // [n][k], U12
  const int64_t m0 = k + NB + (int64_t)blockIdx.x * TM;
  const int64_t n0 = k + NB + (int64_t)blockIdx.y * TN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int wm = (warp & 1) * 64, wn = (warp >> 1) * 32;
  // the output tile goes into the accumulators first (its loads overlap the
  // staging below) and the product is subtracted by staging -L21
  float acc[4][4][4];
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) {
      const int64_t r0 = m0 + wm + mi * 16 + g, c0 = n0 + wn + ni * 8 + 2 * t;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int64_t r = r0 + (e >> 1) * 8, c = c0 + (e & 1);
        acc[mi][ni][e] = (r < R && c < R) ? A[r + c * lda] : 0.f;
      }
    }
  // -L21: TK columns of TM rows
  for (int e = threadIdx.x; e < TK * TM / 4; e += blockDim.x) {
    const int c = e / (TM / 4), r4 = (e % (TM / 4)) * 4;
    const int64_t gr = m0 + r4;
    const float* src = A + gr + (k + c) * lda;
    float4 v;
    if (vec4 && gr + 3 < R) {
      v = *reinterpret_cast<const float4*>(src);
    } else {
      v.x = gr < R ? src[0] : 0.f;
      v.y = gr + 1 < R ? src[1] : 0.f;
      v.z = gr + 2 < R ? src[2] : 0.f;
      v.w = gr + 3 < R ? src[3] : 0.f;
    }
    *reinterpret_cast<float4*>(&sa[c * LA + r4]) = make_float4(-v.x, -v.y, -v.z, -v.w);
  }
  // U12: TN columns of TK rows (rows k.., always inside the matrix)
  for (int e = threadIdx.x; e < TN * TK / 4; e += blockDim.x) {
    const int n = e / (TK / 4), r4 = (e % (TK / 4)) * 4;
    const int64_t gc = n0 + n;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (gc < R) {
      const float* src = A + (k + r4) + gc * lda;
      if (vec4) v = *reinterpret_cast<const float4*>(src);
      else v = make_float4(src[0], src[1], src[2], src[3]);
    }
    *reinterpret_cast<float4*>(&sb[n * LB + r4]) = v;
  }
  __syncthreads();
#pragma unroll
  for (int ks = 0; ks < TK; ks += 8) {
    uint32_t ah[4][4], al[4][4], bh[4][2], bl[4][2];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
      const int mr = wm + mi * 16 + g;
      const float v[4] = {sa[(ks + t) * LA + mr], sa[(ks + t) * LA + mr + 8], sa[(ks + t + 4) * LA + mr],
                          sa[(ks + t + 4) * LA + mr + 8]};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        ah[mi][e] = tf32_bits(v[e]);
        if constexpr (SPLIT) al[mi][e] = tf32_bits(v[e] - __uint_as_float(ah[mi][e]));
      }
    }
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) {
      const int nc = wn + ni * 8 + g;
      const float v[2] = {sb[nc * LB + ks + t], sb[nc * LB + ks + t + 4]};
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        bh[ni][e] = tf32_bits(v[e]);
        if constexpr (SPLIT) bl[ni][e] = tf32_bits(v[e] - __uint_as_float(bh[ni][e]));
      }
    }
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
        if constexpr (SPLIT) {
          mma_tf32(acc[mi][ni], al[mi], bh[ni]);
          mma_tf32(acc[mi][ni], ah[mi], bl[ni]);
        }
        mma_tf32(acc[mi][ni], ah[mi], bh[ni]);
      }
  }
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) {
      const int64_t r0 = m0 + wm + mi * 16 + g, c0 = n0 + wn + ni * 8 + 2 * t;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int64_t r = r0 + (e >> 1) * 8, c = c0 + (e & 1);
        if (r < R && c < R) A[r + c * lda] = acc[mi][ni][e];
      }
    }
}

// ---------------------------------------------------------------------------
// The TF32 trailing update with the 5th-generation tensor cores: tcgen05.mma
// (kind::tf32, M = 128, N = 128, K = 8 per instruction) reading both operands
// from shared memory through matrix descriptors and accumulating in tensor
// memory.  One 128x128 output tile per CTA of 4 warps:
//  * all threads stage -L21 (128 x 64) and U12 (64 x 128) into the canonical
//    non-swizzled K-major layout (core matrices of 8 rows x 4 k = 16 bytes per
//    row: [k-chunk][row-group][8 rows][4 k]), rounding to TF32 on the way:
//    U12 with 16-byte loads (k is contiguous), L21 with 4-byte loads that are
//    coalesced over its m-contiguous columns (TF32 operands in the MN-major
//    form left the accumulator untouched on this part, so both are K-major);
//  * one thread issues the 8 MMAs (K = 64) into a 128-column accumulator and
//    commits them to an mbarrier, which all threads wait on (bounded);
//  * the epilogue reads the accumulator rows (thread = row = TMEM lane) 16
//    columns at a time and adds them to C (-L21 U12), coalesced per column.
// 64 KB of shared memory per CTA keeps at most 3 CTAs (384 TMEM columns) on an
// SM, so the allocation never waits.  A timed-out wait records -1 in *info.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t lu_smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// mbarrier wait (phase parity) bounded in time: non-blocking test_wait polled
// for at most limit_ns of %globaltimer (one second by default); false on timeout
__device__ __forceinline__ bool lu_mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns = 1000000000ull) {
  uint64_t t0;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(lu_smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (t - t0 > limit_ns) return false;
  }
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  // start address, leading / stride byte offsets (16-byte units), version 1,
  // base offset 0, no swizzle
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

template <int NB>
__global__ void __launch_bounds__(128, 3) k_lu_gemm_tc(float* __restrict__ A, int64_t lda, int64_t R, int64_t k,
                                                       bool vec4, int* __restrict__ info, uint64_t wait_ns) {
  constexpr int TM = 128, TN = 128;
  static_assert(NB == 64, "the staging below is written for a 64-column panel");
  constexpr uint32_t kABytes = TM * NB * 4;   // B follows A in shared memory
  constexpr uint32_t kAKChunk = (TM / 8) * 128;   // bytes per k-chunk of 4 (A)
  constexpr uint32_t kBKChunk = (TN / 8) * 128;   // bytes per k-chunk of 4 (B)
  constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TN >> 3) << 17) |
                              ((uint32_t)(TM >> 4) << 24);   // F32 accum, TF32 A and B, both K-major
  extern __shared__ __align__(1024) unsigned char tsm[];
  float* sA = reinterpret_cast<float*>(tsm);
  float* sB = reinterpret_cast<float*>(tsm + kABytes);
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int64_t m0 = k + NB + (int64_t)blockIdx.x * TM;
  const int64_t n0 = k + NB + (int64_t)blockIdx.y * TN;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(lu_smem_u32(&s_tmem)),
                 "r"(TN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(lu_smem_u32(&bar)), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // -L21: 4 consecutive k of row m (4-byte loads, coalesced over m across the
  // warp) -> A[kc][mg][mr][0..3]
  for (int e = tid; e < TM * NB / 4; e += blockDim.x) {
    const int m = e % TM, kc = e / TM;
    const int64_t gr = m0 + m;
    float v[4] = {0.f, 0.f, 0.f, 0.f};
    if (gr < R) {
#pragma unroll
      for (int i = 0; i < 4; ++i) v[i] = A[gr + (k + 4 * kc + i) * lda];
    }
    const float4 t = make_float4(__uint_as_float(tf32_bits(-v[0])), __uint_as_float(tf32_bits(-v[1])),
                                 __uint_as_float(tf32_bits(-v[2])), __uint_as_float(tf32_bits(-v[3])));
    *reinterpret_cast<float4*>(&sA[((kc * (TM / 8) + (m >> 3)) * 8 + (m & 7)) * 4]) = t;
  }
  // U12: float4 of 4 consecutive k of column n -> B[kc][ng][nr][0..3]
  for (int e = tid; e < TN * NB / 4; e += blockDim.x) {
    const int n = e / (NB / 4), r4 = (e % (NB / 4)) * 4;
    const int64_t gc = n0 + n;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (gc < R) {
      const float* src = A + (k + r4) + gc * lda;
      if (vec4) v = *reinterpret_cast<const float4*>(src);
      else v = make_float4(src[0], src[1], src[2], src[3]);
    }
    const float4 t = make_float4(__uint_as_float(tf32_bits(v.x)), __uint_as_float(tf32_bits(v.y)),
                                 __uint_as_float(tf32_bits(v.z)), __uint_as_float(tf32_bits(v.w)));
    *reinterpret_cast<float4*>(&sB[(((r4 >> 2) * (TN / 8) + (n >> 3)) * 8 + (n & 7)) * 4]) = t;
  }
  // generic-proxy stores -> tensor-core (async proxy) reads
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  if (tid == 0) {
    const uint32_t a0 = lu_smem_u32(sA), b0 = lu_smem_u32(sB);
#pragma unroll
    for (int g = 0; g < NB / 8; ++g) {
      const uint64_t da = umma_desc(a0 + 2 * g * kAKChunk, kAKChunk, 128);
      const uint64_t db = umma_desc(b0 + 2 * g * kBKChunk, kBKChunk, 128);
      const uint32_t acc = g > 0 ? 1u : 0u;
      asm volatile(
          "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
          "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
          "l"(da), "l"(db), "r"(kIdesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     lu_smem_u32(&bar))
                 : "memory");
  }
  bool ok = lu_mbar_wait(&bar, 0, wait_ns);
  const bool all_ok = __syncthreads_and(ok) != 0;
  if (!all_ok) {
    if (tid == 0) {
      atomicCAS(info, 0, -1);
      (void)lu_mbar_wait(&bar, 0);   // let the issued MMAs drain (bounded) before freeing
    }
    __syncthreads();
  } else {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int row = tid;                      // TMEM lane = accumulator row
    const int64_t gr = m0 + row;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
    for (int cc = 0; cc < TN; cc += 16) {
      float cv[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int64_t gc = n0 + cc + j;
        cv[j] = (gr < R && gc < R) ? A[gr + gc * lda] : 0.f;
      }
      uint32_t d[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
          "%15}, [%16];"
          : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
            "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15])
          : "r"(lane_addr + (uint32_t)cc));
      // the registers are valid only after wait::ld: tie them to it so that no
      // use is scheduled before
      asm volatile("tcgen05.wait::ld.sync.aligned;"
                   : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3]), "+r"(d[4]), "+r"(d[5]), "+r"(d[6]), "+r"(d[7]),
                     "+r"(d[8]), "+r"(d[9]), "+r"(d[10]), "+r"(d[11]), "+r"(d[12]), "+r"(d[13]), "+r"(d[14]),
                     "+r"(d[15])
                   :
                   : "memory");
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int64_t gc = n0 + cc + j;
        if (gr < R && gc < R) A[gr + gc * lda] = cv[j] + __uint_as_float(d[j]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TN));
  }
}

template <int NB>
constexpr size_t lu_gemm_smem() { return sizeof(float) * ((size_t)NB * (128 + 8) + (size_t)128 * (NB + 4)); }

// ---------------------------------------------------------------------------
// solve L U x = P r for one right-hand side (in place in x):
// row swaps, then blocked forward / backward substitution: a diagonal block
// solved by one CTA, then the rows below / above updated in parallel.
// ---------------------------------------------------------------------------
// out[i] = in[perm[i]]
__global__ void k_permute(const float* __restrict__ in, const int* __restrict__ perm, int64_t R,
                          float* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in[perm[i]];
}

constexpr int kSB = 128;   // substitution block

// Diagonal block [j0, j0+n): the block in shared memory, one column of the
// substitution per step, all threads update the entries below (or above).
template <bool LOWER>
__global__ void __launch_bounds__(kSB) k_trsv_diag(const float* __restrict__ A, int64_t lda, int64_t R, int64_t j0,
                                                   float* __restrict__ x) {
  extern __shared__ float trsv_sm[];
  float (*Ls)[kSB + 1] = reinterpret_cast<float (*)[kSB + 1]>(trsv_sm);
  __shared__ float xs[kSB];
  const int n = (int)std::min<int64_t>(kSB, R - j0);
  const int t = threadIdx.x;
  for (int c = 0; c < n; ++c)
    if (t < n) Ls[t][c] = A[(j0 + t) + (j0 + c) * lda];
  if (t < n) xs[t] = x[j0 + t];
  __syncthreads();
  if (LOWER) {
    for (int r = 0; r < n; ++r) {
      if (t > r && t < n) xs[t] = fmaf(-Ls[t][r], xs[r], xs[t]);
      __syncthreads();
    }
  } else {
    for (int r = n - 1; r >= 0; --r) {
      if (t == r) xs[r] = xs[r] / Ls[r][r];
      __syncthreads();
      if (t < r) xs[t] = fmaf(-Ls[t][r], xs[r], xs[t]);
      __syncthreads();
    }
  }
  if (t < n) x[j0 + t] = xs[t];
}

// rows [r0, r1): x[r] -= sum_{q in block} A[r, j0+q] x[j0+q]
__global__ void k_trsv_update(const float* __restrict__ A, int64_t lda, int64_t j0, int nbk, int64_t r0, int64_t r1,
                              float* __restrict__ x) {
  __shared__ float xs[kSB];
  if (threadIdx.x < nbk) xs[threadIdx.x] = x[j0 + threadIdx.x];
  __syncthreads();
  const int64_t r = r0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= r1) return;
  float s = 0.f;
  for (int q = 0; q < nbk; ++q) s = fmaf(A[r + (j0 + q) * lda], xs[q], s);
  x[r] -= s;
}

// x = (LU)^{-1} P rhs; rhs and x distinct
static int lu_solve(const float* LU, int64_t lda, int64_t R, const int* perm, const float* rhs, float* x,
                    cudaStream_t st) {
  constexpr size_t kDiagSmem = sizeof(float) * kSB * (kSB + 1);
  static const cudaError_t attr[2] = {
      cudaFuncSetAttribute(k_trsv_diag<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDiagSmem),
      cudaFuncSetAttribute(k_trsv_diag<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDiagSmem)};
  RF_CUDA_TRY(attr[0]);
  RF_CUDA_TRY(attr[1]);
  k_permute<<<(unsigned)std::min<int64_t>(ceil_div(R, 256), 4096), 256, 0, st>>>(rhs, perm, R, x);
  RF_LAUNCH_CHECK();
  for (int64_t j0 = 0; j0 < R; j0 += kSB) {
    const int nbk = (int)std::min<int64_t>(kSB, R - j0);
    k_trsv_diag<true><<<1, kSB, kDiagSmem, st>>>(LU, lda, R, j0, x);
    const int64_t r0 = j0 + nbk;
    if (r0 < R) k_trsv_update<<<(unsigned)ceil_div(R - r0, 256), 256, 0, st>>>(LU, lda, j0, nbk, r0, R, x);
  }
  const int64_t last = (R - 1) / kSB * kSB;
  for (int64_t j0 = last; j0 >= 0; j0 -= kSB) {
    const int nbk = (int)std::min<int64_t>(kSB, R - j0);
    k_trsv_diag<false><<<1, kSB, kDiagSmem, st>>>(LU, lda, R, j0, x);
    if (j0 > 0) k_trsv_update<<<(unsigned)ceil_div(j0, 256), 256, 0, st>>>(LU, lda, j0, nbk, 0, j0, x);
  }
  RF_LAUNCH_CHECK();
  return RF_OK;
}

// r = b - A x (A FP32 column-major, x FP64, accumulation FP64): the columns
// are split over blockIdx.y (nsplit chunks of cps columns), each split writes
// FP64 partial rows, and k_residual_sum adds them in fixed order.
__global__ void __launch_bounds__(256) k_residual64_part(const float* __restrict__ A, int64_t lda, int64_t R,
                                                         const double* __restrict__ x, int64_t cps,
                                                         double* __restrict__ part) {
  const int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (row >= R) return;
  const int64_t c0 = (int64_t)blockIdx.y * cps, c1 = std::min<int64_t>(R, c0 + cps);
  double s0 = 0.0, s1 = 0.0;
  int64_t c = c0;
  for (; c + 1 < c1; c += 2) {
    s0 = fma((double)__ldcs(A + row + c * lda), x[c], s0);
    s1 = fma((double)__ldcs(A + row + (c + 1) * lda), x[c + 1], s1);
  }
  if (c < c1) s0 = fma((double)__ldcs(A + row + c * lda), x[c], s0);
  part[(int64_t)blockIdx.y * R + row] = s0 + s1;
}

__global__ void k_residual_sum(const double* __restrict__ part, int nsplit, int64_t R, const float* __restrict__ b,
                               double* __restrict__ r) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R; i += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int p = 0; p < nsplit; ++p) s += part[(int64_t)p * R + i];
    r[i] = (double)b[i] - s;
  }
}

static int launch_residual64(const LuSetup& s, const float* A, const float* b, cudaStream_t st) {
  const int64_t R = s.R;
  const int row_blocks = (int)ceil_div(R, 256);
  int nsplit = std::max(1, std::min(kLuResidualSplits, (int)ceil_div(148 * 8, row_blocks)));
  nsplit = (int)std::min<int64_t>(nsplit, R);
  const int64_t cps = ceil_div(R, nsplit);
  nsplit = (int)ceil_div(R, cps);
  k_residual64_part<<<dim3((unsigned)row_blocks, (unsigned)nsplit), 256, 0, st>>>(A, s.lda, R, s.x64, cps, s.rpart);
  RF_LAUNCH_CHECK();
  k_residual_sum<<<(unsigned)std::min<int64_t>(ceil_div(R, 256), 1024), 256, 0, st>>>(s.rpart, nsplit, R, b, s.r64);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

__global__ void k_norm2_pair(const double* __restrict__ r, const float* __restrict__ b, int64_t R,
                             double* __restrict__ out) {
  __shared__ double s1[256], s2[256];
  double a = 0.0, c = 0.0;
  for (int64_t i = threadIdx.x; i < R; i += blockDim.x) {
    a = fma(r[i], r[i], a);
    c = fma((double)b[i], (double)b[i], c);
  }
  s1[threadIdx.x] = a;
  s2[threadIdx.x] = c;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      s1[threadIdx.x] += s1[threadIdx.x + o];
      s2[threadIdx.x] += s2[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = s1[0];
    out[1] = s2[0];
  }
}

__global__ void k_to_float(const double* __restrict__ in, float* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

__global__ void k_axpy64(double* __restrict__ x, const float* __restrict__ d, int64_t n, int init) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = (init ? 0.0 : x[i]) + (double)d[i];
}

// Factor a copy of A (panels, swaps, triangular block rows, trailing updates)
// and compose the row permutation.
static int lu_factor(const LuSetup& s, const float* A, bool split, cudaStream_t st, int* launches_out,
                     bool* pivoted, bool* tc_factors, float* max_l) {
  *tc_factors = false;
  const int64_t R = s.R, lda = s.ldlu ? s.ldlu : s.lda;
  constexpr int NB = 64;
  *pivoted = false;
  RF_CUDA_TRY(cudaMemcpy2DAsync(s.LU, lda * sizeof(float), A, s.lda * sizeof(float), R * sizeof(float), R,
                                cudaMemcpyDeviceToDevice, st));
  if (!split && s.use_tc && s.LT && (lda % 4) == 0) {
    // the tensor-core factorization without row exchanges; its factors are
    // kept when they are those of partial pivoting (every |l_ij| <= 1)
    bool clean = false;
    const int rc = lu_factor_tc(s, st, &clean, launches_out, max_l);
    if (rc == RF_E_TIMEOUT) return rc;
    if (rc == RF_OK && clean) {
      *tc_factors = true;
      return RF_OK;
    }
    cudaGetLastError();
    RF_CUDA_TRY(cudaMemcpy2DAsync(s.LU, lda * sizeof(float), A, s.lda * sizeof(float), R * sizeof(float), R,
                                  cudaMemcpyDeviceToDevice, st));
  }
  *pivoted = true;
  RF_CUDA_TRY(cudaMemsetAsync(s.info, 0, sizeof(int), st));
  int launches = 0;
  // float4 staging needs every column start 16-byte aligned (k and the chunk
  // offsets are multiples of 4)
  const bool vec4 = (lda % 4 == 0) && (reinterpret_cast<uintptr_t>(s.LU) % 16 == 0);
  static const cudaError_t smem_attr =
      cudaFuncSetAttribute(k_lu_panel_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, kPanelSmemBytes);
  static const cudaError_t gemm_attr[2] = {
      cudaFuncSetAttribute(k_lu_gemm<NB, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lu_gemm_smem<NB>()),
      cudaFuncSetAttribute(k_lu_gemm<NB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lu_gemm_smem<NB>())};
  RF_CUDA_TRY(gemm_attr[split ? 1 : 0]);
  constexpr int kTcSmem = 2 * 128 * NB * 4;
  static const cudaError_t tc_attr =
      cudaFuncSetAttribute(k_lu_gemm_tc<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
  const int64_t lim = device_wait_limit();
  const uint64_t wait_ns = lim < 0 ? 1000000000ull : (uint64_t)lim;
  int dev = 0, num_sms = 148;
  RF_CUDA_TRY(cudaGetDevice(&dev));
  RF_CUDA_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
  for (int64_t k = 0; k < R; k += NB) {
    const int nb = (int)std::min<int64_t>(NB, R - k);
    // shared-memory panel: one block per SM at most (its rows of the panel
    // fit in kPanelSmemBytes); the global-memory panel otherwise
    const int want = s.panel_blocks > 0 ? s.panel_blocks : num_sms;
    const int sm_blocks = (int)std::max<int64_t>(
        1, std::min<int64_t>(std::min<int64_t>((int64_t)s.coop_blocks, (int64_t)want), ceil_div(R - k, 32)));
    const int rows_per = (int)ceil_div(R - k, sm_blocks);
    const size_t psmem = (size_t)rows_per * nb * sizeof(float);
    if (smem_attr == cudaSuccess && psmem <= (size_t)kPanelSmemBytes) {
      const int nblk = (int)ceil_div(R - k, rows_per);
      PanelSmArgs pa{s.LU, lda, R, k, nb, rows_per, s.ipiv, s.pmax, s.pidx, s.prow, s.jrow, s.info};
      void* args[] = {&pa};
      RF_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_lu_panel_smem, dim3(nblk), dim3(256), args, psmem, st));
    } else {
      PanelArgs pa{s.LU, lda, R, k, nb, s.ipiv, s.pmax, s.pidx, s.info};
      const int nblk = (int)std::max<int64_t>(1, std::min<int64_t>(s.coop_blocks, ceil_div(R - k, 256)));
      void* args[] = {&pa};
      RF_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_lu_panel, dim3(nblk), dim3(256), args, 0, st));
    }
    k_lu_laswp<<<(unsigned)ceil_div(R, 256), 256, 0, st>>>(s.LU, lda, R, k, nb, s.ipiv);
    launches += 2;
    if (k + nb < R) {
      if (nb != NB) {
        set_last_error_str("lu: internal panel width");
        return RF_E_INPUT;
      }
      k_lu_trsm<NB><<<(unsigned)ceil_div(R - k - NB, 256), 256, 0, st>>>(s.LU, lda, R, k);
      dim3 g((unsigned)ceil_div(R - k - NB, 128), (unsigned)ceil_div(R - k - NB, 128));
      if (split) {
        k_lu_gemm<NB, true><<<g, 256, lu_gemm_smem<NB>(), st>>>(s.LU, lda, R, k, vec4);
      } else if (tc_attr == cudaSuccess) {
        k_lu_gemm_tc<NB><<<g, 128, kTcSmem, st>>>(s.LU, lda, R, k, vec4, s.info, wait_ns);
      } else {
        k_lu_gemm<NB, false><<<g, 256, lu_gemm_smem<NB>(), st>>>(s.LU, lda, R, k, vec4);
      }
      launches += 2;
    }
    RF_LAUNCH_CHECK();
  }
  int info = 0;
  RF_CUDA_TRY(cudaMemcpyAsync(&info, s.info, sizeof(int), cudaMemcpyDeviceToHost, st));
  RF_CUDA_TRY(cudaMemcpyAsync(s.host_ipiv, s.ipiv, R * sizeof(int), cudaMemcpyDeviceToHost, st));
  RF_CUDA_TRY(cudaStreamSynchronize(st));
  *launches_out += launches;
  if (info < 0) {
    set_last_error_str("lu: a bounded device-side wait timed out");
    return RF_E_TIMEOUT;
  }
  if (info != 0) {
    set_last_error_str("lu: zero pivot");
    return RF_E_SINGULAR;
  }
  // the sequence of row swaps as one permutation (applied by a gather)
  for (int64_t i = 0; i < R; ++i) s.host_perm[i] = (int)i;
  for (int64_t j = 0; j < R; ++j) {
    const int p = s.host_ipiv[j];
    if (p != j) std::swap(s.host_perm[j], s.host_perm[p]);
  }
  RF_CUDA_TRY(cudaMemcpyAsync(s.perm, s.host_perm, R * sizeof(int), cudaMemcpyHostToDevice, st));
  return RF_OK;
}

int lu_time_panel(const LuSetup& s, const float* A, int blocks, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1,
                  float* ms) {
  const int64_t R = s.R, lda = s.ldlu ? s.ldlu : s.lda, k = 0;
  const int nb = (int)std::min<int64_t>(64, R);
  static const cudaError_t smem_attr =
      cudaFuncSetAttribute(k_lu_panel_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, kPanelSmemBytes);
  RF_CUDA_TRY(smem_attr);
  const int nblk0 = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)std::min(blocks, s.coop_blocks),
                                                                ceil_div(R - k, 32)));
  const int rows_per = (int)ceil_div(R - k, nblk0);
  const size_t psmem = (size_t)rows_per * nb * sizeof(float);
  if (psmem > (size_t)kPanelSmemBytes) return RF_E_UNSUPPORTED;
  const int nblk = (int)ceil_div(R - k, rows_per);
  RF_CUDA_TRY(cudaMemcpy2DAsync(s.LU, lda * sizeof(float), A, s.lda * sizeof(float), R * sizeof(float), R,
                                cudaMemcpyDeviceToDevice, st));
  RF_CUDA_TRY(cudaMemsetAsync(s.info, 0, sizeof(int), st));
  PanelSmArgs pa{s.LU, lda, R, k, nb, rows_per, s.ipiv, s.pmax, s.pidx, s.prow, s.jrow, s.info};
  void* args[] = {&pa};
  RF_CUDA_TRY(cudaEventRecord(e0, st));
  RF_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_lu_panel_smem, dim3(nblk), dim3(256), args, psmem, st));
  RF_CUDA_TRY(cudaEventRecord(e1, st));
  RF_CUDA_TRY(cudaEventSynchronize(e1));
  RF_CUDA_TRY(cudaEventElapsedTime(ms, e0, e1));
  return RF_OK;
}

// The TF32 factors first; FP64-residual refinement until ||b - A x|| / ||b||
// <= tol.  If the refinement stalls (the residual falls by less than half in a
// step, after the first two), the matrix is factored again with the split
// 3xTF32 update and refined from the start.
int lu_factor_solve(const LuSetup& s, const float* A, const float* b, float* x, cudaStream_t st, LuResult* res) {
  const int64_t R = s.R, ldlu = s.ldlu ? s.ldlu : s.lda;
  bool pivoted = false;
  float max_l = 0.f;
  const unsigned eb = (unsigned)std::min<int64_t>(ceil_div(R, 256), 4096);
  int launches = 0, steps = 0;
  double rel = 0.0;
  int factorizations = 0;
  for (int pass = 0; pass < 2; ++pass) {
    const bool split = pass == 1;
    bool tcf = false;
    RF_TRY_RF(lu_factor(s, A, split, st, &launches, &pivoted, &tcf, &max_l));
    auto solve = [&](const float* rhs, float* out) -> int {
      launches += tcf ? 2 : 1 + 4 * (int)ceil_div(R, kSB);
      return tcf ? lu_solve_tc(s, rhs, out, st) : lu_solve(s.LU, ldlu, R, s.perm, rhs, out, st);
    };
    ++factorizations;
    // x0 = (LU)^{-1} P b, then refine: r = b - A x (FP64), d = (LU)^{-1} P r
    RF_TRY_RF(solve(b, s.d));
    k_axpy64<<<eb, 256, 0, st>>>(s.x64, s.d, R, 1);
    double h[2] = {0, 0};
    steps = 0;
    double prev = 0.0;
    bool stalled = false;
    for (;;) {
      RF_TRY_RF(launch_residual64(s, A, b, st));
      k_norm2_pair<<<1, 256, 0, st>>>(s.r64, b, R, s.norms);
      RF_LAUNCH_CHECK();
      RF_CUDA_TRY(cudaMemcpyAsync(h, s.norms, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
      RF_CUDA_TRY(cudaStreamSynchronize(st));
      rel = h[1] > 0 ? std::sqrt(h[0] / h[1]) : 0.0;
      // factors without row exchanges that do not refine (non-finite, stalled
      // or out of steps) are replaced by partially pivoted ones
      if (!std::isfinite(rel)) {
        if (tcf) { stalled = true; break; }
        return RF_E_NAN;
      }
      if (rel <= s.tol) break;
      if (steps >= s.max_refine) {
        stalled = tcf;
        break;
      }
      if (!split && steps >= 2 && rel > 0.5 * prev) { stalled = true; break; }
      prev = rel;
      // the FP32 residual goes through the output vector, which is overwritten at the end
      k_to_float<<<eb, 256, 0, st>>>(s.r64, x, R);
      RF_TRY_RF(solve(x, s.d));
      k_axpy64<<<eb, 256, 0, st>>>(s.x64, s.d, R, 0);
      ++steps;
    }
    if (!stalled) break;
  }
  k_to_float<<<eb, 256, 0, st>>>(s.x64, x, R);
  RF_LAUNCH_CHECK();
  res->refinement_steps = steps;
  res->relative_residual = rel;
  res->launches = launches;
  res->factorizations = factorizations;
  res->pivoted = pivoted;
  res->max_multiplier = max_l;
  return rel <= s.tol ? RF_OK : RF_E_NOCONV;
}

}  // namespace rf
