// Dense matvec and Krylov solvers (GMRES, BiCGSTAB) on the device.
//
// Reference semantics: the reference solves with ViennaCL 1.5.1 on the GPU
// (src/simulation.cu:421-442 -> lib/viennacl/linalg/gmres.hpp:169-353,
// bicgstab.hpp:80-166) and CERFACS sgmres on the CPU (fortran/solve_system.incl,
// sgmres.f): restarted GMRES(m) from x0 = 0, convergence on the relative
// residual ||b - A x|| / ||b|| <= tol, confirmed on the true residual at each
// restart; BiCGSTAB restarted every 200 iterations.  Written here from the
// published methods (Saad & Schultz 1986; van der Vorst 1992):
//  * Arnoldi with classical Gram-Schmidt applied twice (CGS2), FP64 dot
//    products, Hessenberg and Givens rotations in FP64 on the device;
//  * one cooperative kernel per Arnoldi step (grid-wide syncs between the
//    dot / update phases) after the matvec, so an iteration is 2-3 launches
//    and the host reads one status word per restart cycle;
//  * converged cycles are skipped on the device (a control word every
//    kernel reads first), so the host never waits per iteration.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "rf_common.cuh"
#include "rf_krylov.cuh"

namespace cg = cooperative_groups;

namespace rf {

// ---------------------------------------------------------------------------
// Dense column-major FP32 matvec, split over column chunks:
//   ypart[s][r] = sum_{c in chunk s} A[r + c*lda] x[c]
// Each thread owns 4 consecutive rows (one 16-byte load per column), 8
// columns in flight; x is read through the read-only path (warp-uniform).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_gemv_cm_f32(const float* __restrict__ A, int64_t lda, int64_t R, const float* __restrict__ x, int64_t cps,
              float* __restrict__ ypart, const int* __restrict__ skip) {
  if (skip != nullptr && *skip) return;
  const int64_t r0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (r0 >= R) return;
  const int64_t c0 = (int64_t)blockIdx.y * cps;
  const int64_t c1 = min(R, c0 + cps);
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  const float* p = A + r0 + c0 * lda;
  int64_t c = c0;
  for (; c + 8 <= c1; c += 8) {
    float4 a[8];
    float xv[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) a[u] = __ldcs(reinterpret_cast<const float4*>(p + u * lda));
#pragma unroll
    for (int u = 0; u < 8; ++u) xv[u] = __ldg(x + c + u);
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      acc.x = fmaf(a[u].x, xv[u], acc.x);
      acc.y = fmaf(a[u].y, xv[u], acc.y);
      acc.z = fmaf(a[u].z, xv[u], acc.z);
      acc.w = fmaf(a[u].w, xv[u], acc.w);
    }
    p += 8 * lda;
  }
  for (; c < c1; ++c) {
    const float4 a = __ldcs(reinterpret_cast<const float4*>(p));
    const float xv = __ldg(x + c);
    acc.x = fmaf(a.x, xv, acc.x);
    acc.y = fmaf(a.y, xv, acc.y);
    acc.z = fmaf(a.z, xv, acc.z);
    acc.w = fmaf(a.w, xv, acc.w);
    p += lda;
  }
  float* out = ypart + (int64_t)blockIdx.y * R + r0;
  if (r0 + 3 < R) {
    out[0] = acc.x; out[1] = acc.y; out[2] = acc.z; out[3] = acc.w;
  } else {
    const float v[4] = {acc.x, acc.y, acc.z, acc.w};
    for (int k = 0; k < 4 && r0 + k < R; ++k) out[k] = v[k];
  }
}

DenseGemvPlan plan_dense_gemv(int64_t R, int num_sms, int ctas_per_sm) {
  DenseGemvPlan p;
  p.row_blocks = (int)ceil_div(R, 1024);
  // about ctas_per_sm CTAs of 256 threads per SM in flight
  int splits = (int)ceil_div((int64_t)num_sms * ctas_per_sm, p.row_blocks);
  splits = std::max(1, std::min<int>(splits, (int)ceil_div(R, 64)));
  p.cps = ceil_div(R, splits);
  p.splits = (int)ceil_div(R, p.cps);
  return p;
}

// Any leading dimension / alignment: one row per thread, scalar loads.
__global__ void __launch_bounds__(256)
k_gemv_cm_f32_scalar(const float* __restrict__ A, int64_t lda, int64_t R, const float* __restrict__ x, int64_t cps,
                     float* __restrict__ ypart, const int* __restrict__ skip) {
  if (skip != nullptr && *skip) return;
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  const int64_t c0 = (int64_t)blockIdx.y * cps;
  const int64_t c1 = min(R, c0 + cps);
  float acc = 0.f;
  for (int64_t c = c0; c < c1; ++c) acc = fmaf(__ldcs(A + r + c * lda), __ldg(x + c), acc);
  ypart[(int64_t)blockIdx.y * R + r] = acc;
}

int launch_dense_gemv(const DenseGemvPlan& p, const float* A, int64_t lda, int64_t R, const float* x, float* ypart,
                      const int* skip, cudaStream_t st) {
  if ((lda % 4) != 0 || (reinterpret_cast<uintptr_t>(A) % 16) != 0) {
    dim3 grid((unsigned)ceil_div(R, 256), (unsigned)p.splits);
    k_gemv_cm_f32_scalar<<<grid, 256, 0, st>>>(A, lda, R, x, p.cps, ypart, skip);
    RF_LAUNCH_CHECK();
    return RF_OK;
  }
  dim3 grid((unsigned)p.row_blocks, (unsigned)p.splits);
  k_gemv_cm_f32<<<grid, 256, 0, st>>>(A, lda, R, x, p.cps, ypart, skip);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

// ---------------------------------------------------------------------------
// Block / grid reductions (FP64)
// ---------------------------------------------------------------------------
template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], double* __restrict__ dst /* NV */) {
  __shared__ double red[32][NV];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double s = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    v[k] = s;
  }
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) red[wid][k] = v[k];
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    const int nw = blockDim.x >> 5;
    for (int w = 0; w < nw; ++w) s += red[w][threadIdx.x];
    dst[threadIdx.x] = s;
  }
  __syncthreads();
}

// Sum of part[b*stride + k] over blocks b, fixed order; every block computes
// the same value (used after a grid sync).
__device__ __forceinline__ double sum_parts(const double* __restrict__ part, int nblk, int stride, int k) {
  double s = 0.0;
  for (int b = 0; b < nblk; ++b) s += part[(int64_t)b * stride + k];
  return s;
}

// Dots of w with V[i0 .. i0+NV) (FP64), for the rows this thread owns.
template <int NV>
__device__ __forceinline__ void partial_dots(const float* __restrict__ w, const float* __restrict__ V, int64_t ldv,
                                             int i0, int nv, int64_t R, double (&acc)[NV]) {
#pragma unroll
  for (int k = 0; k < NV; ++k) acc[k] = 0.0;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < R; r += (int64_t)gridDim.x * blockDim.x) {
    const double wr = f2d(w[r]);
#pragma unroll
    for (int k = 0; k < NV; ++k)
      if (k < nv) acc[k] = fma(wr, f2d(V[(int64_t)(i0 + k) * ldv + r]), acc[k]);
  }
}

constexpr int kDotGroup = 8;

// All dots w . V[0..nv) into part[blk*stride + i].
__device__ void grid_partial_dots(const float* __restrict__ w, const float* __restrict__ V, int64_t ldv, int nv,
                                  int64_t R, double* __restrict__ part, int stride) {
  for (int i0 = 0; i0 < nv; i0 += kDotGroup) {
    double acc[kDotGroup];
    partial_dots<kDotGroup>(w, V, ldv, i0, min(kDotGroup, nv - i0), R, acc);
    __shared__ double tmp[kDotGroup];
    block_reduce_store<kDotGroup>(acc, tmp);
    if (threadIdx.x < kDotGroup && i0 + (int)threadIdx.x < nv)
      part[(int64_t)blockIdx.x * stride + i0 + threadIdx.x] = tmp[threadIdx.x];
    __syncthreads();
  }
}

__device__ void grid_partial_norm(const float* __restrict__ w, int64_t R, double* __restrict__ part, int stride,
                                  int slot) {
  double acc[1] = {0.0};
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < R; r += (int64_t)gridDim.x * blockDim.x) {
    const double v = f2d(w[r]);
    acc[0] = fma(v, v, acc[0]);
  }
  __shared__ double tmp[1];
  block_reduce_store<1>(acc, tmp);
  if (threadIdx.x == 0) part[(int64_t)blockIdx.x * stride + slot] = tmp[0];
  __syncthreads();
}

// ---------------------------------------------------------------------------
// GMRES kernels
// ---------------------------------------------------------------------------
struct GmresArgs {
  const float* ypart;  // matvec result, nsplit partial rows
  int nsplit;
  const float* b;
  void* x;             // float or double (x_double)
  int x_double;
  float* V;            // (m+1) x ldv
  const float* Z;      // basis of the solution update (V, or the preconditioned z_j)
  int64_t ldv;
  int64_t R;
  int m;
  double* part;        // 3 partial buffers, each nblk x stride
  int stride;
  double* H;           // (m+1) x m, column j at H[j*(m+1)]
  double* cs;
  double* sn;
  double* g;           // m+1
  GmresCtl* ctl;
};

__device__ __forceinline__ float sum_splits(const float* __restrict__ ypart, int nsplit, int64_t R, int64_t r) {
  float s = ypart[r];
  for (int k = 1; k < nsplit; ++k) s += ypart[(int64_t)k * R + r];
  return s;
}

// Norm of b -> ctl->bnorm; resets the cycle state.
__global__ void k_gmres_init(GmresArgs a) {
  cg::grid_group grid = cg::this_grid();
  grid_partial_norm(a.b, a.R, a.part, a.stride, 0);
  grid.sync();
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const double bn = sqrt(sum_parts(a.part, gridDim.x, a.stride, 0));
    a.ctl->bnorm = bn;
    a.ctl->total_iters = 0;
    a.ctl->converged = (bn == 0.0) ? 1 : 0;
    a.ctl->cycle_done = a.ctl->converged;
    a.ctl->beta = bn;
    a.ctl->restarts = 0;
    a.ctl->nan = isfinite(bn) ? 0 : 1;
  }
}

// r = b - A x, beta = ||r||; convergence test on the true residual;
// V[0] = r / beta, g = (beta, 0, ...).  mode 0: x = 0 (r = b); 1: r = b - sum
// of the matvec partials of A x; 2: V[0] already holds r (written by a
// residual operator, e.g. FP64-accumulated).
__global__ void k_gmres_residual(GmresArgs a, int mode) {
  cg::grid_group grid = cg::this_grid();
  if (a.ctl->converged || a.ctl->nan) return;
  float* V0 = a.V;
  if (mode != 2)
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.R; r += (int64_t)gridDim.x * blockDim.x)
      V0[r] = mode == 0 ? a.b[r] : a.b[r] - sum_splits(a.ypart, a.nsplit, a.R, r);
  grid_partial_norm(V0, a.R, a.part, a.stride, 0);
  grid.sync();
  const double beta = sqrt(sum_parts(a.part, gridDim.x, a.stride, 0));
  const double bn = a.ctl->bnorm;
  const bool conv = beta <= a.ctl->tol * bn;
  const bool bad = !isfinite(beta);
  if (!conv && !bad) {
    const float inv = (float)(1.0 / beta);
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.R; r += (int64_t)gridDim.x * blockDim.x)
      V0[r] *= inv;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (mode != 0) a.ctl->heads += 1;
    a.ctl->beta = beta;
    a.ctl->converged = conv ? 1 : 0;
    a.ctl->nan = bad ? 1 : 0;
    a.ctl->cycle_done = (conv || bad || a.ctl->total_iters >= a.ctl->maxit) ? 1 : 0;
    a.ctl->jconv = 0;
    a.g[0] = beta;
    for (int k = 1; k <= a.m; ++k) a.g[k] = 0.0;
  }
}

// One Arnoldi step j: w = A v_j (from ypart) -> CGS2 against V[0..j] -> v_{j+1};
// Hessenberg column, Givens rotation, residual estimate |g_{j+1}|.
__global__ void k_gmres_arnoldi(GmresArgs a, int j) {
  cg::grid_group grid = cg::this_grid();
  if (a.ctl->cycle_done) return;
  const int nv = j + 1;
  float* w = a.V + (int64_t)(j + 1) * a.ldv;
  double* p0 = a.part;
  double* p1 = a.part + (int64_t)gridDim.x * a.stride;
  double* p2 = a.part + 2 * (int64_t)gridDim.x * a.stride;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.R; r += (int64_t)gridDim.x * blockDim.x)
    w[r] = sum_splits(a.ypart, a.nsplit, a.R, r);
  grid_partial_dots(w, a.V, a.ldv, nv, a.R, p0, a.stride);
  grid.sync();
  __shared__ double h[kMaxRestart + 1], h2[kMaxRestart + 1];
  for (int k = threadIdx.x; k < nv; k += blockDim.x) h[k] = sum_parts(p0, gridDim.x, a.stride, k);
  __syncthreads();
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.R; r += (int64_t)gridDim.x * blockDim.x) {
    double s = f2d(w[r]);
    for (int k = 0; k < nv; ++k) s -= h[k] * f2d(a.V[(int64_t)k * a.ldv + r]);
    w[r] = (float)s;
  }
  grid_partial_dots(w, a.V, a.ldv, nv, a.R, p1, a.stride);
  grid.sync();
  for (int k = threadIdx.x; k < nv; k += blockDim.x) h2[k] = sum_parts(p1, gridDim.x, a.stride, k);
  __syncthreads();
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.R; r += (int64_t)gridDim.x * blockDim.x) {
    double s = f2d(w[r]);
    for (int k = 0; k < nv; ++k) s -= h2[k] * f2d(a.V[(int64_t)k * a.ldv + r]);
    w[r] = (float)s;
  }
  grid_partial_norm(w, a.R, p2, a.stride, 0);
  grid.sync();
  const double nrm = sqrt(sum_parts(p2, gridDim.x, a.stride, 0));
  if (nrm > 0.0 && isfinite(nrm)) {
    const float inv = (float)(1.0 / nrm);
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.R; r += (int64_t)gridDim.x * blockDim.x)
      w[r] *= inv;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int ldh = a.m + 1;
    double* Hc = a.H + (int64_t)j * ldh;
    for (int k = 0; k < nv; ++k) Hc[k] = h[k] + h2[k];
    Hc[j + 1] = nrm;
    for (int k = 0; k < j; ++k) {
      const double x0 = Hc[k], x1 = Hc[k + 1];
      Hc[k] = a.cs[k] * x0 + a.sn[k] * x1;
      Hc[k + 1] = -a.sn[k] * x0 + a.cs[k] * x1;
    }
    const double x0 = Hc[j], x1 = Hc[j + 1];
    const double rr = hypot(x0, x1);
    const double c = rr > 0.0 ? x0 / rr : 1.0, s = rr > 0.0 ? x1 / rr : 0.0;
    a.cs[j] = c;
    a.sn[j] = s;
    Hc[j] = rr;
    Hc[j + 1] = 0.0;
    a.g[j + 1] = -s * a.g[j];
    a.g[j] = c * a.g[j];
    GmresCtl* ctl = a.ctl;
    ctl->total_iters += 1;
    ctl->jconv = j + 1;
    const double est = fabs(a.g[j + 1]);
    ctl->estimate = est;
    const bool bad = !isfinite(est);
    if (bad) ctl->nan = 1;
    if (bad || est <= ctl->tol * ctl->bnorm || j + 1 >= a.m || ctl->total_iters >= ctl->maxit || nrm == 0.0)
      ctl->cycle_done = 1;
  }
}

// x += V y, H y = g (upper triangular, size jconv).
__global__ void k_gmres_update(GmresArgs a) {
  if (a.ctl->converged || a.ctl->nan) return;
  const int jc = a.ctl->jconv;
  if (jc == 0) return;
  __shared__ double y[kMaxRestart];
  if (threadIdx.x == 0) {
    const int ldh = a.m + 1;
    for (int i = jc - 1; i >= 0; --i) {
      double s = a.g[i];
      for (int k = i + 1; k < jc; ++k) s -= a.H[(int64_t)k * ldh + i] * y[k];
      y[i] = s / a.H[(int64_t)i * ldh + i];
    }
  }
  __syncthreads();
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.R; r += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < jc; ++k) s += y[k] * f2d(a.Z[(int64_t)k * a.ldv + r]);
    if (a.x_double) {
      double* x = static_cast<double*>(a.x);
      x[r] += s;
    } else {
      float* x = static_cast<float*>(a.x);
      x[r] = (float)(f2d(x[r]) + s);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) a.ctl->restarts += 1;
}

template <typename T>
__global__ void k_fill_zero(T* __restrict__ p, int64_t n) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
    p[r] = (T)0;
}

static int coop_launch(const void* fn, int nblk, int threads, void** args, cudaStream_t st) {
  RF_CUDA_TRY(cudaLaunchCooperativeKernel(fn, dim3(nblk), dim3(threads), args, 0, st));
  return RF_OK;
}

static thread_local int t_coop_cap = 0;

void set_coop_block_cap(int cap) { t_coop_cap = cap; }

int coop_blocks_per_sm_capped(int num_sms) { return t_coop_cap > 0 ? std::min(num_sms, t_coop_cap) : num_sms; }

void GmresGraphCache::release() {
  for (int v = 0; v < kGmresGraphVariants; ++v) {
    if (exec[v]) cudaGraphExecDestroy(exec[v]);
    exec[v] = nullptr;
    state[v] = 0;
  }
}

int krylov_coop_blocks(int64_t R, int num_sms) {
  // 256-thread blocks; at most 2 per SM (always co-resident), fewer for small systems
  int want = (int)ceil_div(R, 256 * 4);
  int n = std::max(1, std::min(want, 2 * num_sms));
  // Handles that share the device with other handles' cooperative grids keep
  // the sum of all grids within one block per SM, so every grid can become
  // fully resident once the non-cooperative kernels beside it drain.
  if (t_coop_cap > 0) n = std::min(n, t_coop_cap);
  return n;
}

int gmres_solve(const GmresSetup& s, const MatvecFn& matvec, const float* b, float* x, cudaStream_t st,
                GmresResult* res) {
  return gmres_solve_ex(s, matvec, ResidualFn(), b, x, false, st, res);
}

int gmres_solve_ex(const GmresSetup& s, const MatvecFn& matvec, const ResidualFn& residual, const float* b, void* x,
                   bool x_double, cudaStream_t st, GmresResult* res) {
  const int m = s.m;
  if (m < 1 || m > kMaxRestart) {
    set_last_error_str("gmres: restart length out of range");
    return RF_E_INPUT;
  }
  GmresArgs a;
  a.ypart = s.ypart;
  a.nsplit = s.nsplit;
  a.b = b;
  a.x = x;
  a.x_double = x_double ? 1 : 0;
  a.V = s.V;
  a.Z = s.Z ? s.Z : s.V;
  a.ldv = s.ldv;
  a.R = s.R;
  a.m = m;
  a.part = s.part;
  a.stride = kMaxRestart + 2;
  a.H = s.H;
  a.cs = s.cs;
  a.sn = s.sn;
  a.g = s.g;
  a.ctl = s.ctl;
  const int nblk = s.coop_blocks;
  GmresCtl init{};
  init.tol = s.tol;
  init.maxit = s.maxit;
  RF_CUDA_TRY(cudaMemcpyAsync(s.ctl, &init, sizeof(GmresCtl), cudaMemcpyHostToDevice, st));
  if (x_double)
    k_fill_zero<double><<<std::min<int64_t>(ceil_div(s.R, 256), 1024), 256, 0, st>>>(static_cast<double*>(x), s.R);
  else
    k_fill_zero<float><<<std::min<int64_t>(ceil_div(s.R, 256), 1024), 256, 0, st>>>(static_cast<float*>(x), s.R);
  RF_LAUNCH_CHECK();
  {
    void* args[] = {&a};
    int rc = coop_launch((const void*)k_gmres_init, nblk, 256, args, st);
    if (rc) return rc;
  }
  res->launches = 2;
  GmresCtl h{};
  int cycles_run = 0;
  // Pieces of the restart cycles, each launched directly or replayed from a
  // CUDA graph: variant 0 the first cycle whole (residual kernel, m x (matvec
  // + Arnoldi step), update); variant 1 the head of a later cycle (residual of
  // x, residual kernel); variant 2 + c the c-th chunk of kGmresChunk (matvec +
  // Arnoldi step) of a later cycle.  The host reads the control block after a
  // head and after every chunk, so a cycle whose residual has converged, or
  // whose Arnoldi steps have, launches nothing more.
  auto chunk_end = [&](int c) { return std::min(m, (c + 1) * kGmresChunk); };
  auto own_kernels = [&](int v) { return v == 0 ? 2 + m : v == 1 ? 1 : chunk_end(v - 2) - (v - 2) * kGmresChunk; };
  auto enqueue = [&](int v) -> int {
    int mode = 0;
    if (v == 1) {
      const int rc = residual ? residual(x, s.V, &s.ctl->converged, st)
                              : matvec(static_cast<const float*>(x), &s.ctl->converged, st);
      if (rc) return rc;
      mode = residual ? 2 : 1;
    }
    if (v <= 1) {
      void* args[] = {&a, &mode};
      const int rc = coop_launch((const void*)k_gmres_residual, nblk, 256, args, st);
      if (rc) return rc;
    }
    if (v == 1) return RF_OK;
    const int j0 = v == 0 ? 0 : (v - 2) * kGmresChunk, j1 = v == 0 ? m : chunk_end(v - 2);
    for (int j = j0; j < j1; ++j) {
      int rc = matvec(s.V + (int64_t)j * s.ldv, &s.ctl->cycle_done, st);
      if (rc) return rc;
      void* args[] = {&a, &j};
      rc = coop_launch((const void*)k_gmres_arnoldi, nblk, 256, args, st);
      if (rc) return rc;
    }
    if (v == 0) {
      k_gmres_update<<<nblk, 256, 0, st>>>(a);
      RF_LAUNCH_CHECK();
    }
    return RF_OK;
  };
  auto run = [&](int v) -> int {
    GmresGraphCache* gc = s.graphs;
    bool from_graph = false;
    if (gc && gc->state[v] == 2) {
      // capture this piece once (the capture does not run it; the replay below
      // does).  A variant is captured on its second use, so the kernels' one-time
      // set-up (function attributes) has run outside any capture.
      cudaGraph_t graph = nullptr;
      int rc = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess ? RF_OK : RF_E_CUDA;
      if (rc == RF_OK) {
        rc = enqueue(v);
        const cudaError_t ec = cudaStreamEndCapture(st, &graph);
        if (rc == RF_OK && ec == cudaSuccess && graph &&
            cudaGraphInstantiate(&gc->exec[v], graph, 0) == cudaSuccess) {
          size_t n = 0;
          cudaGraphGetNodes(graph, nullptr, &n);
          std::vector<cudaGraphNode_t> nodes(n);
          if (n) cudaGraphGetNodes(graph, nodes.data(), &n);
          int kn = 0;
          for (auto nd : nodes) {
            cudaGraphNodeType ty;
            if (cudaGraphNodeGetType(nd, &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) ++kn;
          }
          gc->kernels[v] = kn;
          gc->state[v] = 1;
        } else {
          gc->exec[v] = nullptr;
          gc->state[v] = -1;
        }
        if (graph) cudaGraphDestroy(graph);
      } else {
        gc->state[v] = -1;
      }
      cudaGetLastError();   // a refused capture leaves no sticky error; clear the non-sticky one
      if (gc->state[v] == 1) {
        // the callbacks counted their kernels while capturing; count ours as a direct launch does
        res->launches += own_kernels(v);
        RF_CUDA_TRY(cudaGraphLaunch(gc->exec[v], st));
        from_graph = true;
      }
    } else if (gc && gc->state[v] == 1) {
      RF_CUDA_TRY(cudaGraphLaunch(gc->exec[v], st));
      res->launches += gc->kernels[v];
      from_graph = true;
    }
    if (from_graph) {
      ++res->graph_replays;
    } else {
      const int rc = enqueue(v);
      if (rc) return rc;
      res->launches += own_kernels(v);
      if (gc && gc->state[v] == 0) gc->state[v] = 2;
    }
    return RF_OK;
  };
  auto read_ctl = [&]() -> int {
    RF_CUDA_TRY(cudaMemcpyAsync(s.host_ctl, s.ctl, sizeof(GmresCtl), cudaMemcpyDeviceToHost, st));
    RF_CUDA_TRY(host_wait(st, s.wait_ev));
    h = *s.host_ctl;
    return RF_OK;
  };
  for (int cycle = 0;; ++cycle) {
    ++cycles_run;
    if (cycle == 0) {
      if (int rc = run(0)) return rc;
      if (int rc = read_ctl()) return rc;
      if (h.converged || h.nan || h.timeout) break;
      continue;
    }
    if (int rc = run(1)) return rc;
    if (int rc = read_ctl()) return rc;
    // converged, failed, or out of iterations (the residual kernel then ends the cycle)
    if (h.converged || h.nan || h.timeout || h.cycle_done) break;
    for (int c = 0; c * kGmresChunk < m; ++c) {
      if (int rc = run(2 + c)) return rc;
      if (int rc = read_ctl()) return rc;
      if (h.cycle_done || h.nan || h.timeout) break;
    }
    if (h.nan || h.timeout) break;
    k_gmres_update<<<nblk, 256, 0, st>>>(a);
    RF_LAUNCH_CHECK();
    res->launches += 1;
    if (cycle > s.maxit + 2) break;
  }
  res->residual_calls = residual ? cycles_run - 1 : 0;
  res->iterations = h.total_iters;
  res->restarts = h.restarts;
  // a restart cycle opens with a matvec of x, or with the caller's residual (not a matvec)
  res->matvecs = h.total_iters + (residual ? 0 : cycles_run - 1);
  res->relative_residual = h.bnorm > 0 ? h.beta / h.bnorm : 0.0;
  if (h.timeout) {
    set_last_error_str("a bounded device-side wait timed out");
    return RF_E_TIMEOUT;
  }
  if (h.nan) return RF_E_NAN;
  if (!h.converged) return RF_E_NOCONV;
  return RF_OK;
}

// ---------------------------------------------------------------------------
// GMRES as a graph with a device-side restart loop
// ---------------------------------------------------------------------------
__global__ void k_gmres_ctl_init(GmresCtl* ctl, double tol, int maxit) {
  GmresCtl c{};
  c.tol = tol;
  c.maxit = maxit;
  *ctl = c;
}

// another restart cycle is needed: not converged, no failure, iterations left
__global__ void k_gmres_loop_cond(cudaGraphConditionalHandle cond, GmresCtl* ctl) {
  const bool more = !ctl->converged && !ctl->nan && !ctl->timeout && ctl->total_iters < ctl->maxit &&
                    ctl->restarts <= ctl->maxit + 2;
  ctl->halt = (ctl->nan || ctl->timeout) ? 1 : 0;
  cudaGraphSetConditional(cond, more ? 1u : 0u);
}

static GmresArgs gmres_args(const GmresSetup& s, const float* b, void* x, bool x_double) {
  GmresArgs a;
  a.ypart = s.ypart;
  a.nsplit = s.nsplit;
  a.b = b;
  a.x = x;
  a.x_double = x_double ? 1 : 0;
  a.V = s.V;
  a.Z = s.Z ? s.Z : s.V;
  a.ldv = s.ldv;
  a.R = s.R;
  a.m = s.m;
  a.part = s.part;
  a.stride = kMaxRestart + 2;
  a.H = s.H;
  a.cs = s.cs;
  a.sn = s.sn;
  a.g = s.g;
  a.ctl = s.ctl;
  return a;
}

// m x (matvec + Arnoldi step) of the cycle whose first basis vector is in V[0]
static int enqueue_arnoldi_steps(const GmresSetup& s, GmresArgs& a, const MatvecFn& matvec, cudaStream_t st,
                                 int* kernels) {
  for (int j = 0; j < s.m; ++j) {
    int rc = matvec(s.V + (int64_t)j * s.ldv, &s.ctl->cycle_done, st);
    if (rc) return rc;
    void* args[] = {&a, &j};
    rc = coop_launch((const void*)k_gmres_arnoldi, s.coop_blocks, 256, args, st);
    if (rc) return rc;
    *kernels += 1;
  }
  k_gmres_update<<<s.coop_blocks, 256, 0, st>>>(a);
  RF_LAUNCH_CHECK();
  *kernels += 1;
  return RF_OK;
}

int gmres_enqueue_first(const GmresSetup& s, const MatvecFn& matvec, const ResidualFn& residual, const float* b,
                        void* x, bool x_double, cudaGraphConditionalHandle cond, cudaStream_t st, int* kernels) {
  if (s.m < 1 || s.m > kMaxRestart) {
    set_last_error_str("gmres: restart length out of range");
    return RF_E_INPUT;
  }
  GmresArgs a = gmres_args(s, b, x, x_double);
  k_gmres_ctl_init<<<1, 1, 0, st>>>(s.ctl, s.tol, s.maxit);
  if (x_double)
    k_fill_zero<double><<<std::min<int64_t>(ceil_div(s.R, 256), 1024), 256, 0, st>>>(static_cast<double*>(x), s.R);
  else
    k_fill_zero<float><<<std::min<int64_t>(ceil_div(s.R, 256), 1024), 256, 0, st>>>(static_cast<float*>(x), s.R);
  RF_LAUNCH_CHECK();
  *kernels += 2;
  void* args0[] = {&a};
  if (int rc = coop_launch((const void*)k_gmres_init, s.coop_blocks, 256, args0, st)) return rc;
  int mode = 0;
  void* args1[] = {&a, &mode};
  if (int rc = coop_launch((const void*)k_gmres_residual, s.coop_blocks, 256, args1, st)) return rc;
  *kernels += 2;
  if (int rc = enqueue_arnoldi_steps(s, a, matvec, st, kernels)) return rc;
  k_gmres_loop_cond<<<1, 1, 0, st>>>(cond, s.ctl);
  RF_LAUNCH_CHECK();
  *kernels += 1;
  (void)residual;
  return RF_OK;
}

int gmres_enqueue_cycle(const GmresSetup& s, const MatvecFn& matvec, const ResidualFn& residual, const float* b,
                        void* x, bool x_double, cudaGraphConditionalHandle cond, cudaStream_t st, int* kernels) {
  GmresArgs a = gmres_args(s, b, x, x_double);
  const int rc0 = residual ? residual(x, s.V, &s.ctl->converged, st)
                           : matvec(static_cast<const float*>(x), &s.ctl->converged, st);
  if (rc0) return rc0;
  int mode = residual ? 2 : 1;
  void* args1[] = {&a, &mode};
  if (int rc = coop_launch((const void*)k_gmres_residual, s.coop_blocks, 256, args1, st)) return rc;
  *kernels += 1;
  if (int rc = enqueue_arnoldi_steps(s, a, matvec, st, kernels)) return rc;
  k_gmres_loop_cond<<<1, 1, 0, st>>>(cond, s.ctl);
  RF_LAUNCH_CHECK();
  *kernels += 1;
  return RF_OK;
}

int gmres_result_from_ctl(const GmresCtl& h, bool has_residual, GmresResult* res) {
  res->iterations = h.total_iters;
  res->restarts = h.restarts;
  res->residual_calls = has_residual ? h.heads : 0;
  res->matvecs = h.total_iters + (has_residual ? 0 : h.heads);
  res->relative_residual = h.bnorm > 0 ? h.beta / h.bnorm : 0.0;
  if (h.timeout) {
    set_last_error_str("a bounded device-side wait timed out");
    return RF_E_TIMEOUT;
  }
  if (h.nan) return RF_E_NAN;
  if (!h.converged) return RF_E_NOCONV;
  return RF_OK;
}

// ---------------------------------------------------------------------------
// BiCGSTAB (van der Vorst 1992) with the semantics of the reference's
// ViennaCL 1.5.1 solver (lib/viennacl/linalg/bicgstab.hpp:80-166): x0 = 0,
// two matvecs per iteration, convergence when ||r||/||b|| < tol on the
// recursive residual, restart from the true residual when rho or omega
// vanish or every `restart_every` iterations.  FP64 dots and scalars.
// ---------------------------------------------------------------------------
struct BicgArgs {
  const float* ypart;
  int nsplit;
  const float* b;
  float* x;
  float* r;
  float* r0;
  float* p;
  float* v;
  float* sv;
  float* t;
  int64_t R;
  double* part;
  int stride;
  BicgCtl* ctl;
};

// a.b and c.d partial dots of this block into part[blk*stride + slot], slot+1
__device__ void grid_partial_dot2(const float* __restrict__ a, const float* __restrict__ b,
                                  const float* __restrict__ c, const float* __restrict__ d, int64_t R,
                                  double* __restrict__ part, int stride, int slot) {
  double acc[2] = {0.0, 0.0};
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < R; r += (int64_t)gridDim.x * blockDim.x) {
    acc[0] = fma(f2d(a[r]), f2d(b[r]), acc[0]);
    acc[1] = fma(f2d(c[r]), f2d(d[r]), acc[1]);
  }
  __shared__ double tmp[2];
  block_reduce_store<2>(acc, tmp);
  if (threadIdx.x < 2) part[(int64_t)blockIdx.x * stride + slot + threadIdx.x] = tmp[threadIdx.x];
  __syncthreads();
}

__device__ __forceinline__ bool bicg_stopped(const BicgCtl* c) {
  return c->converged || c->nan || c->need_restart || c->iters >= c->maxit;
}

// ||b||, x = 0, r = r0 = p = b, rho = ||b||^2
__global__ void k_bicg_init(BicgArgs a) {
  cg::grid_group grid = cg::this_grid();
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.R; r += (int64_t)gridDim.x * blockDim.x) {
    const float bv = a.b[r];
    a.x[r] = 0.f;
    a.r[r] = bv;
    a.r0[r] = bv;
    a.p[r] = bv;
  }
  grid_partial_norm(a.b, a.R, a.part, a.stride, 0);
  grid.sync();
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const double bb = sum_parts(a.part, gridDim.x, a.stride, 0);
    BicgCtl* c = a.ctl;
    c->bnorm = sqrt(bb);
    c->rho = bb;
    c->rnorm = sqrt(bb);
    c->iters = 0;
    c->last_restart = 0;
    c->converged = bb == 0.0 ? 1 : 0;
    c->nan = isfinite(bb) ? 0 : 1;
    c->need_restart = 0;
    c->restarts = 0;
  }
}

// after the matvec of x: r = b - A x, r0 = p = r, rho = ||r||^2
__global__ void k_bicg_restart(BicgArgs a) {
  cg::grid_group grid = cg::this_grid();
  if (a.ctl->converged || a.ctl->nan || !a.ctl->need_restart) return;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.R; r += (int64_t)gridDim.x * blockDim.x) {
    const float rv = a.b[r] - sum_splits(a.ypart, a.nsplit, a.R, r);
    a.r[r] = rv;
    a.r0[r] = rv;
    a.p[r] = rv;
  }
  grid_partial_norm(a.r, a.R, a.part, a.stride, 0);
  grid.sync();
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const double rr = sum_parts(a.part, gridDim.x, a.stride, 0);
    a.ctl->rho = rr;
    a.ctl->need_restart = 0;
    a.ctl->last_restart = a.ctl->iters;
    a.ctl->restarts += 1;
    if (!isfinite(rr)) a.ctl->nan = 1;
  }
}

// after v = A p: alpha = rho / (v . r0), s = r - alpha v
__global__ void k_bicg_step1(BicgArgs a) {
  cg::grid_group grid = cg::this_grid();
  if (bicg_stopped(a.ctl)) return;
  const double rho = a.ctl->rho;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.R; r += (int64_t)gridDim.x * blockDim.x)
    a.v[r] = sum_splits(a.ypart, a.nsplit, a.R, r);
  grid_partial_dot2(a.v, a.r0, a.v, a.v, a.R, a.part, a.stride, 0);
  grid.sync();
  const double vr0 = sum_parts(a.part, gridDim.x, a.stride, 0);
  const double alpha = rho / vr0;
  const float af = (float)alpha;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.R; r += (int64_t)gridDim.x * blockDim.x)
    a.sv[r] = a.r[r] - af * a.v[r];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.ctl->alpha = alpha;
    if (!isfinite(alpha)) a.ctl->nan = 1;
  }
}

// after t = A s: omega = (t.s)/(t.t), x += alpha p + omega s, r = s - omega t,
// rho' = r.r0, ||r||; convergence; beta; p = r + beta (p - omega v)
__global__ void k_bicg_step2(BicgArgs a) {
  cg::grid_group grid = cg::this_grid();
  if (bicg_stopped(a.ctl)) return;
  // every block reads the control block before the first grid sync; block 0
  // updates it only after the last one
  BicgCtl* c = a.ctl;
  const double rho = c->rho, alpha = c->alpha, bnorm = c->bnorm, tol = c->tol;
  const int it = c->iters + 1, last_restart = c->last_restart, restart_every = c->restart_every;
  double* p0 = a.part;
  double* p1 = a.part + (int64_t)gridDim.x * a.stride;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.R; r += (int64_t)gridDim.x * blockDim.x)
    a.t[r] = sum_splits(a.ypart, a.nsplit, a.R, r);
  grid_partial_dot2(a.t, a.sv, a.t, a.t, a.R, p0, a.stride, 0);
  grid.sync();
  const double ts = sum_parts(p0, gridDim.x, a.stride, 0);
  const double tt = sum_parts(p0, gridDim.x, a.stride, 1);
  const double omega = tt > 0.0 ? ts / tt : 0.0;
  const float af = (float)alpha, of = (float)omega;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.R; r += (int64_t)gridDim.x * blockDim.x) {
    a.x[r] = a.x[r] + af * a.p[r] + of * a.sv[r];
    a.r[r] = a.sv[r] - of * a.t[r];
  }
  grid_partial_dot2(a.r, a.r0, a.r, a.r, a.R, p1, a.stride, 0);
  grid.sync();
  const double rho_new = sum_parts(p1, gridDim.x, a.stride, 0);
  const double rnorm = sqrt(sum_parts(p1, gridDim.x, a.stride, 1));
  const bool conv = rnorm / bnorm < tol;
  const double beta = (rho_new / rho) * (alpha / omega);
  const bool restart = !conv && (rho_new == 0.0 || omega == 0.0 || (it - 1) - last_restart > restart_every);
  if (!conv && !restart) {
    const float bf = (float)beta;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.R; r += (int64_t)gridDim.x * blockDim.x)
      a.p[r] = a.r[r] + bf * (a.p[r] - of * a.v[r]);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    c->iters = it;
    c->rnorm = rnorm;
    c->rho = rho_new;
    if (conv) c->converged = 1;
    if (restart) c->need_restart = 1;
    if (!isfinite(rnorm)) c->nan = 1;
  }
}

__global__ void k_bicg_stopword(BicgCtl* c) {
  c->stop_word = (c->converged || c->nan || c->need_restart || c->iters >= c->maxit) ? 1 : 0;
}

int bicgstab_solve(const BicgSetup& s, const MatvecFn& matvec, const float* b, float* x, cudaStream_t st,
                   BicgResult* res) {
  BicgArgs a;
  a.ypart = s.ypart;
  a.nsplit = s.nsplit;
  a.b = b;
  a.x = x;
  a.r = s.work;
  a.r0 = s.work + s.ldv;
  a.p = s.work + 2 * s.ldv;
  a.v = s.work + 3 * s.ldv;
  a.sv = s.work + 4 * s.ldv;
  a.t = s.work + 5 * s.ldv;
  a.R = s.R;
  a.part = s.part;
  a.stride = kMaxRestart + 2;
  a.ctl = s.ctl;
  const int nblk = s.coop_blocks;
  BicgCtl init{};
  init.tol = s.tol;
  init.maxit = s.maxit;
  init.restart_every = s.restart_every;
  RF_CUDA_TRY(cudaMemcpyAsync(s.ctl, &init, sizeof(BicgCtl), cudaMemcpyHostToDevice, st));
  {
    void* args[] = {&a};
    int rc = coop_launch((const void*)k_bicg_init, nblk, 256, args, st);
    if (rc) return rc;
  }
  res->launches = 1;
  res->matvecs = 0;
  BicgCtl h{};
  const int chunk = 10;   // iterations between host checks
  for (int guard = 0; guard < s.maxit + 4 * (s.maxit / std::max(1, s.restart_every) + 2); ++guard) {
    for (int k = 0; k < chunk; ++k) {
      int rc = matvec(a.p, (const int*)&s.ctl->stop_word, st);
      if (rc) return rc;
      void* args[] = {&a};
      rc = coop_launch((const void*)k_bicg_step1, nblk, 256, args, st);
      if (rc) return rc;
      rc = matvec(a.sv, (const int*)&s.ctl->stop_word, st);
      if (rc) return rc;
      rc = coop_launch((const void*)k_bicg_step2, nblk, 256, args, st);
      if (rc) return rc;
      // the matvec kernels read one word: fold the stop conditions into it
      k_bicg_stopword<<<1, 1, 0, st>>>(s.ctl);
      RF_LAUNCH_CHECK();
      res->launches += 5;
    }
    RF_CUDA_TRY(cudaMemcpyAsync(s.host_ctl, s.ctl, sizeof(BicgCtl), cudaMemcpyDeviceToHost, st));
    RF_CUDA_TRY(cudaStreamSynchronize(st));
    h = *s.host_ctl;
    if (h.converged || h.nan || h.iters >= s.maxit) break;
    if (h.need_restart) {
      int rc = matvec(x, nullptr, st);
      if (rc) return rc;
      void* args[] = {&a};
      rc = coop_launch((const void*)k_bicg_restart, nblk, 256, args, st);
      if (rc) return rc;
      k_bicg_stopword<<<1, 1, 0, st>>>(s.ctl);
      RF_LAUNCH_CHECK();
      res->launches += 2;
      ++res->matvecs;
    }
  }
  res->iterations = h.iters;
  res->restarts = h.restarts;
  res->matvecs += 2 * h.iters;
  res->relative_residual = h.bnorm > 0 ? h.rnorm / h.bnorm : 0.0;
  if (h.nan) return RF_E_NAN;
  if (!h.converged) return RF_E_NOCONV;
  return RF_OK;
}

// ---------------------------------------------------------------------------
// BiCGSTAB with iterative refinement (mixed precision): the outer loop keeps
// x in FP64 and recomputes r = b - A x with the caller's residual (FP64
// accumulation over the FP32 operator); the inner BiCGSTAB above solves
// A d = r on the caller's matvec (the 16-bit operator, FP32 sums) until its
// recursive residual falls below inner_tol relative to ||r||, and d is added
// to x in FP64.  The correction equation has x0 = 0, as the reference's
// solver has for the full system.
// ---------------------------------------------------------------------------
// ||v||^2 in FP64, one block, fixed order
__global__ void __launch_bounds__(1024) k_norm2_f32(const float* __restrict__ v, int64_t R, double* __restrict__ out) {
  double acc[1] = {0.0};
  for (int64_t i = threadIdx.x; i < R; i += blockDim.x) {
    const double t = (double)v[i];
    acc[0] = fma(t, t, acc[0]);
  }
  __shared__ double tmp[1];
  block_reduce_store<1>(acc, tmp);
  if (threadIdx.x == 0) *out = tmp[0];
}

__global__ void k_add_correction(double* __restrict__ x, const float* __restrict__ d, int64_t R) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < R; i += (int64_t)gridDim.x * blockDim.x)
    x[i] += (double)d[i];
}

int bicgstab_ir_solve(const BicgSetup& s, const MatvecFn& matvec, const ResidualFn& residual, const float* b,
                      const BicgIr& ir, cudaStream_t st, BicgResult* res) {
  const int64_t R = s.R;
  const unsigned eb = (unsigned)std::min<int64_t>(ceil_div(R, 256), 1024);
  k_fill_zero<double><<<eb, 256, 0, st>>>(ir.x64, R);
  k_norm2_f32<<<1, 1024, 0, st>>>(b, R, ir.norm_dev);
  RF_LAUNCH_CHECK();
  RF_CUDA_TRY(cudaMemcpyAsync(ir.norm_host, ir.norm_dev, sizeof(double), cudaMemcpyDeviceToHost, st));
  RF_CUDA_TRY(cudaStreamSynchronize(st));
  const double bnorm = std::sqrt(*ir.norm_host);
  *res = BicgResult();
  res->launches = 2;
  double rel = 0.0;
  int outer = 0, inner_left = s.maxit;
  for (;;) {
    // r = b - A x (FP64 sums); the first pass has x = 0, so r = b
    if (int rc = residual(ir.x64, ir.r, nullptr, st)) return rc;
    k_norm2_f32<<<1, 1024, 0, st>>>(ir.r, R, ir.norm_dev);
    RF_LAUNCH_CHECK();
    RF_CUDA_TRY(cudaMemcpyAsync(ir.norm_host, ir.norm_dev, sizeof(double), cudaMemcpyDeviceToHost, st));
    RF_CUDA_TRY(cudaStreamSynchronize(st));
    res->launches += 1;   // the norm (the residual's kernels are the caller's to count)
    const double rnorm = std::sqrt(*ir.norm_host);
    rel = bnorm > 0.0 ? rnorm / bnorm : 0.0;
    if (!std::isfinite(rel)) {
      res->relative_residual = rel;
      return RF_E_NAN;
    }
    if (rel <= ir.tol || outer >= ir.max_outer || inner_left <= 0) break;
    BicgSetup in = s;
    in.tol = ir.inner_tol;
    in.maxit = inner_left;
    BicgResult br;
    const int rc = bicgstab_solve(in, matvec, ir.r, ir.d, st, &br);
    if (rc != RF_OK && rc != RF_E_NOCONV) return rc;
    res->iterations += br.iterations;
    res->restarts += br.restarts;
    res->matvecs += br.matvecs;
    res->launches += br.launches + 1;
    inner_left -= std::max(1, br.iterations);
    k_add_correction<<<eb, 256, 0, st>>>(ir.x64, ir.d, R);
    RF_LAUNCH_CHECK();
    ++outer;
  }
  res->refinements = outer;
  res->relative_residual = rel;
  return rel <= ir.tol ? RF_OK : RF_E_NOCONV;
}

}  // namespace rf
