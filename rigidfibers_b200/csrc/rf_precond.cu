// Near-field preconditioner of the stored mixed-precision modes (no reference
// counterpart: the reference's GMRES runs unpreconditioned).  For every fiber i
// and its k nearest neighbours by centre distance, the (k+1) x 15 rows of the
// system A = I + C T restricted to those fibers form a small dense block B_i
// (identity diagonal blocks, the stored FP32 pair blocks off the diagonal);
// the preconditioner keeps the 15 rows of B_i^-1 that belong to fiber i and
// applies them to the neighbourhood's entries of a vector (restricted additive
// Schwarz).  The solve uses it on the right, in flexible GMRES form: the
// matvec computes z_j = P v_j, stores z_j, and applies A to it; the solution
// update reads the stored z_j, so every convergence test still sees the true
// residual of A.  All sums run in a fixed order: results are reproducible.
//
// Storage read here: the FP32 record of the unordered pair (p, q), p < q, in
// assembly tiles of 8 fibers (I = p / 8 <= J = q / 8) grouped into storage
// tiles of 16: record ((L16 * 4 + sub) * 8 + q % 8) of NQ32 x 8 floats, value
// ((kI * M + kJ) * 6 + c) of pair p % 8 at [value][p % 8]; kI is p's force
// term, kJ q's, c the symmetric component (11, 22, 33, 12, 13, 23).
#include <algorithm>

#include "rf_common.cuh"
#include "rf_kernels.cuh"

namespace rf {
namespace {

constexpr int kNfM = 5;                       // force terms (the mixed modes' M)
constexpr int kNfM3 = 3 * kNfM;               // rows per fiber
constexpr int kNfNQ32 = (kNfM + 1) * (kNfM + 1) * 6;
constexpr int kNfStride = 16;                 // floats per column of a fiber's stored rows

// k nearest fibers of fiber i (centre distance, ties by index): nb[i][0] = i,
// nb[i][1..k]; slots past N - 1 neighbours hold -1.  One thread per fiber,
// the centres streamed through shared memory.
__global__ void __launch_bounds__(128) k_nf_neighbours(const float4* __restrict__ pos, int N, int k,
                                                       int* __restrict__ nb) {
  constexpr int kChunk = 1024;
  __shared__ float4 sp[kChunk];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float bd[kNfMaxNeighbours];
  int bi[kNfMaxNeighbours];
#pragma unroll
  for (int s = 0; s < kNfMaxNeighbours; ++s) {
    bd[s] = 3.0e38f;
    bi[s] = -1;
  }
  const float4 pi = pos[min(i, N - 1)];
  for (int c0 = 0; c0 < N; c0 += kChunk) {
    const int cn = min(kChunk, N - c0);
    __syncthreads();
    for (int u = threadIdx.x; u < cn; u += blockDim.x) sp[u] = pos[c0 + u];
    __syncthreads();
    if (i < N) {
      for (int u = 0; u < cn; ++u) {
        const int j = c0 + u;
        if (j == i) continue;
        const float dx = sp[u].x - pi.x, dy = sp[u].y - pi.y, dz = sp[u].z - pi.z;
        const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        // insertion into the sorted list (the last slot in use is k - 1)
        if (d2 < bd[k - 1] || (d2 == bd[k - 1] && j < bi[k - 1])) {
          int s = k - 1;
#pragma unroll
          for (int t = kNfMaxNeighbours - 1; t > 0; --t) {
            if (t <= s && (bd[t - 1] > d2 || (bd[t - 1] == d2 && bi[t - 1] > j))) {
              bd[t] = bd[t - 1];
              bi[t] = bi[t - 1];
              s = t - 1;
            }
          }
          bd[s] = d2;
          bi[s] = j;
        }
      }
    }
  }
  if (i < N) {
    nb[(int64_t)i * (k + 1)] = i;
    for (int s = 0; s < k; ++s) nb[(int64_t)i * (k + 1) + 1 + s] = bi[s];
  }
}

// S (the symmetric 3x3 component c) of T^{pq}[kp][kq] for fibers p != q with
// kp p's force term: the record of the unordered pair, transposed when p > q
__device__ __forceinline__ float nf_block(const float* __restrict__ S32, int p, int q, int kp, int kq, int c) {
  const int a = min(p, q), b = max(p, q);
  const int ka = p < q ? kp : kq, kb = p < q ? kq : kp;
  const int I = a / 8, J = b / 8;
  const int64_t I16 = I / 2, J16 = J / 2;
  const int sub = (I % 2) * 2 + (J % 2);
  const int64_t L16 = J16 * (J16 + 1) / 2 + I16;
  const int64_t rec = (L16 * 4 + sub) * 8 + (b % 8);
  return S32[(rec * kNfNQ32 + (ka * kNfM + kb) * 6 + c) * 8 + (a % 8)];
}

__device__ __forceinline__ int sym_index(int d, int e) {
  // (11, 22, 33, 12, 13, 23)
  if (d == e) return d;
  const int lo = min(d, e), hi = max(d, e);
  return lo == 0 ? (hi == 1 ? 3 : 4) : 5;
}

// One CTA per fiber i: Gauss-Jordan elimination without row exchanges on
// [B_i^T | E] (E: the first 15 columns of the identity), so that the right
// part ends as the transpose of fiber i's rows of B_i^-1; those rows go to
// W[i] as [column c][row r] (kNfStride floats per column).  A pivot below
// 1e-6 in magnitude or a non-finite entry leaves fiber i unpreconditioned
// (its rows of the identity).
__global__ void __launch_bounds__(256) k_nf_setup(const Tables tab, int N, int k, const float4* __restrict__ ori,
                                                  const float* __restrict__ S32, const int* __restrict__ nb,
                                                  float* __restrict__ W) {
  extern __shared__ float nsm[];
  const int i = blockIdx.x;
  const int kk = min(k, N - 1);
  const int n = (kk + 1) * kNfM3;            // rows of B_i
  const int ld = n + kNfM3;                  // [B^T | E] row length
  float* aug = nsm;                          // n x ld
  float* fcol = nsm + (size_t)n * ld;        // n: the pivot column
  __shared__ int snb[kNfMaxNeighbours + 1];
  __shared__ float4 st[kNfMaxNeighbours + 1];
  __shared__ int bad;
  if (threadIdx.x <= kk) {
    snb[threadIdx.x] = nb[(int64_t)i * (k + 1) + threadIdx.x];
    st[threadIdx.x] = ori[snb[threadIdx.x]];
  }
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  // aug[r][c] = B(c, r) for c < n; B(row of fiber a, term ka, comp d;
  // column of fiber b, term kb, comp e) = delta when a == b, else
  // [C_{a,ka} S^{ab}_{ka,kb}]_{d,e}, C_k(S) = k == 0 ? g t (t^T S) : g (S - E t (t^T S))
  for (int u = threadIdx.x; u < n * n; u += blockDim.x) {
    const int r = u / n, c = u % n;          // aug row r (a column of B), aug column c (a row of B)
    const int la = c / kNfM3, lb = r / kNfM3;
    const int ka = (c % kNfM3) / 3, d = c % 3, kb = (r % kNfM3) / 3, e = r % 3;
    float v;
    if (la == lb) {
      v = (ka == kb && d == e) ? 1.f : 0.f;
    } else {
      const int a = snb[la], b = snb[lb];
      const float4 t = st[la];
      const float t3[3] = {t.x, t.y, t.z};
      // (t^T S)_e and S_de of the symmetric block
      float tS = 0.f;
#pragma unroll
      for (int f = 0; f < 3; ++f) tS = fmaf(t3[f], nf_block(S32, a, b, ka, kb, sym_index(f, e)), tS);
      const float Sde = nf_block(S32, a, b, ka, kb, sym_index(d, e));
      const float g = tab.gamma[ka];
      v = ka == 0 ? g * t3[d] * tS : g * (Sde - tab.eigen[ka] * t3[d] * tS);
    }
    aug[(size_t)r * ld + c] = v;
  }
  for (int u = threadIdx.x; u < n * kNfM3; u += blockDim.x) {
    const int r = u / kNfM3, c = u % kNfM3;
    aug[(size_t)r * ld + n + c] = r == c ? 1.f : 0.f;
  }
  __syncthreads();
  for (int piv = 0; piv < n; ++piv) {
    const float p = aug[(size_t)piv * ld + piv];
    if (threadIdx.x == 0 && (!(fabsf(p) >= 1e-6f) || !isfinite(p))) bad = 1;
    __syncthreads();
    if (bad) break;
    const float inv = 1.f / p;
    for (int c = threadIdx.x; c < ld; c += blockDim.x) aug[(size_t)piv * ld + c] *= inv;
    for (int r = threadIdx.x; r < n; r += blockDim.x) fcol[r] = aug[(size_t)r * ld + piv];
    __syncthreads();
    for (int u = threadIdx.x; u < n * ld; u += blockDim.x) {
      const int r = u / ld, c = u % ld;
      if (r != piv) aug[u] = fmaf(-fcol[r], aug[(size_t)piv * ld + c], aug[u]);
    }
    __syncthreads();
  }
  // W[i][c][r] = (B^-1)[r][c] = X[c][r], X the right part of aug
  float* wi = W + (size_t)i * (kNfMaxNeighbours + 1) * kNfM3 * kNfStride;
  for (int u = threadIdx.x; u < n * kNfStride; u += blockDim.x) {
    const int c = u / kNfStride, r = u % kNfStride;
    float v = 0.f;
    if (r < kNfM3) v = bad ? (c == r ? 1.f : 0.f) : aug[(size_t)c * ld + n + r];
    wi[u] = v;
  }
}

// z_i = W_i v[neighbourhood of i]; lane r < 15 of one warp per fiber forms row r
__global__ void __launch_bounds__(256) k_nf_apply(int N, int k, const int* __restrict__ nb,
                                                  const float* __restrict__ W, const float* __restrict__ v,
                                                  float* __restrict__ z, const int* __restrict__ skip) {
  if (skip != nullptr && *skip) return;
  const int lane = threadIdx.x & 31;
  const int i = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  if (i >= N) return;
  const int kk = min(k, N - 1);
  const float* wi = W + (size_t)i * (kNfMaxNeighbours + 1) * kNfM3 * kNfStride;
  float acc = 0.f;
  for (int l = 0; l <= kk; ++l) {
    const int f = nb[(int64_t)i * (k + 1) + l];
    const float* vf = v + (int64_t)f * kNfM3;
    const float* wl = wi + (size_t)l * kNfM3 * kNfStride;
#pragma unroll
    for (int c = 0; c < kNfM3; ++c) acc = fmaf(wl[c * kNfStride + (lane & 15)], vf[c], acc);
  }
  if (lane < kNfM3) z[(int64_t)i * kNfM3 + lane] = acc;
}

}  // namespace

int64_t nf_w_floats(int N) { return (int64_t)N * (kNfMaxNeighbours + 1) * kNfM3 * kNfStride; }

int launch_nf_setup(const Tables& tab, int N, int k, const float4* pos, const float4* ori, const float* S32, int* nb,
                    float* W, cudaStream_t st) {
  if (tab.M != kNfM || k < 1 || k > kNfMaxNeighbours || N < 1) return RF_E_UNSUPPORTED;
  k_nf_neighbours<<<(unsigned)ceil_div(N, 128), 128, 0, st>>>(pos, N, k, nb);
  RF_LAUNCH_CHECK();
  const int kk = std::min(k, N - 1);
  const int n = (kk + 1) * kNfM3;
  const size_t smem = sizeof(float) * ((size_t)n * (n + kNfM3) + n);
  RF_CUDA_TRY(cudaFuncSetAttribute(k_nf_setup, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_nf_setup<<<(unsigned)N, 256, smem, st>>>(tab, N, k, ori, S32, nb, W);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

int launch_nf_apply(int N, int k, const int* nb, const float* W, const float* v, float* z, const int* skip,
                    cudaStream_t st) {
  k_nf_apply<<<(unsigned)ceil_div((int64_t)N * 32, 256), 256, 0, st>>>(N, k, nb, W, v, z, skip);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

}  // namespace rf
