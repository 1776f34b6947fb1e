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
// 128x128 output tiles, 256 threads with 8x8 register tiles, K = NB staged
// through shared memory in chunks of 16.
template <int NB>
__global__ void __launch_bounds__(256) k_lu_gemm(float* __restrict__ A, int64_t lda, int64_t R, int64_t k) {
  constexpr int TM = 128, TN = 128, TK = 16;
  __shared__ float sa[TK][TM + 4];
  __shared__ float sb[TK][TN + 4];
  const int64_t m0 = k + NB + (int64_t)blockIdx.x * TM;
  const int64_t n0 = k + NB + (int64_t)blockIdx.y * TN;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int jx = 0; jx < 8; ++jx) acc[i][jx] = 0.f;
  for (int kk = 0; kk < NB; kk += TK) {
    // L21 tile: rows m0.., cols k+kk..  (column-major: consecutive rows contiguous)
    for (int e = threadIdx.x; e < TK * TM; e += blockDim.x) {
      const int r = e % TM, c = e / TM;
      const int64_t gr = m0 + r;
      sa[c][r] = gr < R ? A[gr + (k + kk + c) * lda] : 0.f;
    }
    // U12 tile: rows k+kk.., cols n0..
    for (int e = threadIdx.x; e < TK * TN; e += blockDim.x) {
      const int r = e % TK, c = e / TK;
      const int64_t gc = n0 + c;
      sb[r][c] = gc < R ? A[(k + kk + r) + gc * lda] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < TK; ++q) {
      float av[8], bv[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) av[i] = sa[q][ty * 8 + i];
#pragma unroll
      for (int jx = 0; jx < 8; ++jx) bv[jx] = sb[q][tx * 8 + jx];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int jx = 0; jx < 8; ++jx) acc[i][jx] = fmaf(av[i], bv[jx], acc[i][jx]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int jx = 0; jx < 8; ++jx) {
    const int64_t gc = n0 + tx * 8 + jx;
    if (gc >= R) continue;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int64_t gr = m0 + ty * 8 + i;
      if (gr < R) A[gr + gc * lda] -= acc[i][jx];
    }
  }
}

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

constexpr int kSB = 64;   // substitution block

// Diagonal block [j0, j0+n): the block in shared memory, one column of the
// substitution per step, all threads update the entries below (or above).
template <bool LOWER>
__global__ void __launch_bounds__(kSB) k_trsv_diag(const float* __restrict__ A, int64_t lda, int64_t R, int64_t j0,
                                                   float* __restrict__ x) {
  __shared__ float Ls[kSB][kSB + 1];
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
  k_permute<<<(unsigned)std::min<int64_t>(ceil_div(R, 256), 4096), 256, 0, st>>>(rhs, perm, R, x);
  RF_LAUNCH_CHECK();
  for (int64_t j0 = 0; j0 < R; j0 += kSB) {
    const int nbk = (int)std::min<int64_t>(kSB, R - j0);
    k_trsv_diag<true><<<1, kSB, 0, st>>>(LU, lda, R, j0, x);
    const int64_t r0 = j0 + nbk;
    if (r0 < R) k_trsv_update<<<(unsigned)ceil_div(R - r0, 256), 256, 0, st>>>(LU, lda, j0, nbk, r0, R, x);
  }
  const int64_t last = (R - 1) / kSB * kSB;
  for (int64_t j0 = last; j0 >= 0; j0 -= kSB) {
    const int nbk = (int)std::min<int64_t>(kSB, R - j0);
    k_trsv_diag<false><<<1, kSB, 0, st>>>(LU, lda, R, j0, x);
    if (j0 > 0) k_trsv_update<<<(unsigned)ceil_div(j0, 256), 256, 0, st>>>(LU, lda, j0, nbk, 0, j0, x);
  }
  RF_LAUNCH_CHECK();
  return RF_OK;
}

// r = b - A x (A FP32 column-major, x FP64, accumulation FP64); ||r||^2 and
// ||b||^2 partial sums into part[blk*2 + {0,1}].
__global__ void __launch_bounds__(256) k_residual64(const float* __restrict__ A, int64_t lda, int64_t R,
                                                    const double* __restrict__ x, const float* __restrict__ b,
                                                    double* __restrict__ r) {
  const int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (row >= R) return;
  double s = 0.0;
  for (int64_t c = 0; c < R; ++c) s = fma((double)A[row + c * lda], x[c], s);
  r[row] = (double)b[row] - s;
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

int lu_factor_solve(const LuSetup& s, const float* A, const float* b, float* x, cudaStream_t st, LuResult* res) {
  const int64_t R = s.R, lda = s.lda;
  constexpr int NB = 64;
  RF_CUDA_TRY(cudaMemcpy2DAsync(s.LU, lda * sizeof(float), A, lda * sizeof(float), R * sizeof(float), R,
                                cudaMemcpyDeviceToDevice, st));
  RF_CUDA_TRY(cudaMemsetAsync(s.info, 0, sizeof(int), st));
  int launches = 0;
  for (int64_t k = 0; k < R; k += NB) {
    const int nb = (int)std::min<int64_t>(NB, R - k);
    PanelArgs pa{s.LU, lda, R, k, nb, s.ipiv, s.pmax, s.pidx, s.info};
    const int nblk = (int)std::max<int64_t>(1, std::min<int64_t>(s.coop_blocks, ceil_div(R - k, 256)));
    void* args[] = {&pa};
    RF_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_lu_panel, dim3(nblk), dim3(256), args, 0, st));
    k_lu_laswp<<<(unsigned)ceil_div(R, 256), 256, 0, st>>>(s.LU, lda, R, k, nb, s.ipiv);
    launches += 2;
    if (k + nb < R) {
      if (nb != NB) {
        set_last_error_str("lu: internal panel width");
        return RF_E_INPUT;
      }
      k_lu_trsm<NB><<<(unsigned)ceil_div(R - k - NB, 256), 256, 0, st>>>(s.LU, lda, R, k);
      dim3 g((unsigned)ceil_div(R - k - NB, 128), (unsigned)ceil_div(R - k - NB, 128));
      k_lu_gemm<NB><<<g, 256, 0, st>>>(s.LU, lda, R, k);
      launches += 2;
    }
    RF_LAUNCH_CHECK();
  }
  int info = 0;
  RF_CUDA_TRY(cudaMemcpyAsync(&info, s.info, sizeof(int), cudaMemcpyDeviceToHost, st));
  RF_CUDA_TRY(cudaMemcpyAsync(s.host_ipiv, s.ipiv, R * sizeof(int), cudaMemcpyDeviceToHost, st));
  RF_CUDA_TRY(cudaStreamSynchronize(st));
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
  // x0 = (LU)^{-1} P b, then refine: r = b - A x (FP64), d = (LU)^{-1} P r
  RF_TRY_RF(lu_solve(s.LU, lda, R, s.perm, b, s.d, st));
  const unsigned eb = (unsigned)std::min<int64_t>(ceil_div(R, 256), 4096);
  k_axpy64<<<eb, 256, 0, st>>>(s.x64, s.d, R, 1);
  double h[2] = {0, 0};
  int steps = 0;
  double rel = 0.0;
  for (;;) {
    k_residual64<<<(unsigned)ceil_div(R, 256), 256, 0, st>>>(A, lda, R, s.x64, b, s.r64);
    k_norm2_pair<<<1, 256, 0, st>>>(s.r64, b, R, s.norms);
    RF_LAUNCH_CHECK();
    RF_CUDA_TRY(cudaMemcpyAsync(h, s.norms, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    RF_CUDA_TRY(cudaStreamSynchronize(st));
    rel = h[1] > 0 ? std::sqrt(h[0] / h[1]) : 0.0;
    if (!std::isfinite(rel)) return RF_E_NAN;
    if (rel <= s.tol || steps >= s.max_refine) break;
    // the FP32 residual goes through the output vector, which is overwritten at the end
    k_to_float<<<eb, 256, 0, st>>>(s.r64, x, R);
    RF_TRY_RF(lu_solve(s.LU, lda, R, s.perm, x, s.d, st));
    k_axpy64<<<eb, 256, 0, st>>>(s.x64, s.d, R, 0);
    ++steps;
  }
  k_to_float<<<eb, 256, 0, st>>>(s.x64, x, R);
  RF_LAUNCH_CHECK();
  res->refinement_steps = steps;
  res->relative_residual = rel;
  res->launches = launches;
  return rel <= s.tol ? RF_OK : RF_E_NOCONV;
}

}  // namespace rf
