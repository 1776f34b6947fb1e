// Velocity update (numerical inner integrals) and the fiber time integrator.
//
// Reference: fortran/update_velocities.incl:1-89 (and the CUDA kernels
// src/kernels/reset_velocities.cu:6-39, update_velocities_2D.cu:6-166):
//   U_i = (0.5/d) [ (d+2) F + (d-2)(t_i.F) t_i + sum_{j!=i} sum_qi w_qi GF_ij(qi) ]
//   W_i = (1.5/d) (I - t_i t_i^T) sum_{j!=i} sum_qi w_qi P_1(s_qi) GF_ij(qi)
//   GF_ij(qi) = sum_qj w_qj K(R_ij(qi,qj)) f_j(qj),  f_j = F/2 + sum_k a_{j,k} P_{k+1}
// fortran/update_fibers_firststep.incl:1-10 and update_fibers.incl:1-17 for
// the time step, here accumulated in FP64 on FP64 state.
// Reductions are deterministic: per-(j-chunk, fiber) partial sums, then a
// fixed-order sum; no atomics.
#include "rf_common.cuh"
#include "rf_kernels.cuh"
#include "rf_analytic.cuh"

namespace rf {

int velocity_chunks(int N);

// fw[j*Q + q] = w_q f_j(s_q) = W[0][q] F/2 + sum_k a_{j,k} W[k+1][q]
__global__ void k_source_density(const Tables tab, int N, const float* __restrict__ x, float4* __restrict__ fw) {
  const int Q = tab.Q, M = tab.M;
  const int64_t n = (int64_t)N * Q;
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x) {
    const int j = (int)(u / Q), q = (int)(u % Q);
    float f0 = 0.f, f1 = 0.f, f2 = tab.W[0][q] * tab.fz_half;
    const float* a = x + (int64_t)j * 3 * M;
    for (int k = 0; k < M; ++k) {
      const float w = tab.W[k + 1][q];
      f0 = fmaf(a[3 * k + 0], w, f0);
      f1 = fmaf(a[3 * k + 1], w, f1);
      f2 = fmaf(a[3 * k + 2], w, f2);
    }
    fw[u] = make_float4(f0, f1, f2, 0.f);
  }
}

// One CTA = TI fibers i x one chunk of source fibers j.  Thread u < TI*Q owns
// (fiber il, quadrature point qi) and accumulates sum_j GF_ij(qi).
template <int Q>
__global__ void __launch_bounds__(192, 4)
k_velocity_numerical(const Tables tab, int N, const double4* __restrict__ pos64, const float4* __restrict__ ori,
                     const float4* __restrict__ fw, int jchunk, float* __restrict__ vpart) {
  constexpr int TI = 192 / Q;
  constexpr int U = TI * Q;
  // quadrature-point separations (x_i - x_j) + s_qi t_i - s_qj t_j with the
  // centre difference in FP64, rounded once (as in the assembly): the error
  // scales with the fibers' distance, not with their distance from the origin
  __shared__ float4 sP[TI][Q], sF[TI][Q];    // s_q t_j, w_q f_j(s_q)
  __shared__ double sXi[TI][3], sXj[TI][3];
  __shared__ float sGs[3][U];
  const int tid = threadIdx.x;
  const int il = tid / Q, qi = tid % Q;
  const int i0 = blockIdx.x * TI;
  const int i = i0 + il;
  const bool unit_ok = tid < U && i < N;
  float tix = 0.f, tiy = 0.f, tiz = 0.f;
  if (unit_ok) {
    const float4 t = ori[i];
    const float s = tab.pts[qi];
    tix = s * t.x; tiy = s * t.y; tiz = s * t.z;
  }
  if (tid < TI) {
    const double4 x = pos64[min(i0 + tid, N - 1)];
    sXi[tid][0] = x.x; sXi[tid][1] = x.y; sXi[tid][2] = x.z;
  }
  const float e2 = tab.e2, e2x3 = -3.f * tab.e2;
  float g0 = 0.f, g1 = 0.f, g2 = 0.f;
  const int jbeg = blockIdx.y * jchunk, jend = min(N, jbeg + jchunk);
  for (int js = jbeg; js < jend; js += TI) {
    __syncthreads();
    if (tid < U) {
      const int jl = tid / Q, q = tid % Q;
      const int j = min(js + jl, N - 1);
      const float4 t = ori[j];
      const float s = tab.pts[q];
      sP[jl][q] = make_float4(s * t.x, s * t.y, s * t.z, 0.f);
      sF[jl][q] = fw[(int64_t)j * Q + q];
      if (q == 0) {
        const double4 x = pos64[j];
        sXj[jl][0] = x.x; sXj[jl][1] = x.y; sXj[jl][2] = x.z;
      }
    }
    __syncthreads();
    const int jn = min(TI, jend - js);
    if (unit_ok) {
      for (int jl = 0; jl < jn; ++jl) {
        if (js + jl == i) continue;
        const float pix = (float)(sXi[il][0] - sXj[jl][0]) + tix;
        const float piy = (float)(sXi[il][1] - sXj[jl][1]) + tiy;
        const float piz = (float)(sXi[il][2] - sXj[jl][2]) + tiz;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          const float4 pj = sP[jl][q];
          const float4 f = sF[jl][q];
          const float rx = pix - pj.x, ry = piy - pj.y, rz = piz - pj.z;
          const float r2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
          const float inv = rsqrtf(r2);
          const float inv2 = inv * inv;
          const float inv3 = inv2 * inv;
          const float inv5 = inv3 * inv2;
          const float a = fmaf(e2, inv3, inv);
          const float bb = fmaf(e2x3, inv5, inv3);
          // K f = a f + bb R (R.f)
          const float rf = fmaf(rx, f.x, fmaf(ry, f.y, rz * f.z)) * bb;
          g0 = fmaf(a, f.x, fmaf(rf, rx, g0));
          g1 = fmaf(a, f.y, fmaf(rf, ry, g1));
          g2 = fmaf(a, f.z, fmaf(rf, rz, g2));
        }
      }
    }
  }
  if (tid < U) { sGs[0][tid] = g0; sGs[1][tid] = g1; sGs[2][tid] = g2; }
  __syncthreads();
  // per fiber: sum_qi w_qi gs(qi) and sum_qi w_qi P_1(s_qi) gs(qi)
  if (tid < TI * 6) {
    const int fl = tid / 6, comp = tid % 6;
    const int a = comp % 3;
    const bool rot = comp >= 3;
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q) s = fmaf(rot ? tab.W[1][q] : tab.W[0][q], sGs[a][fl * Q + q], s);
    if (i0 + fl < N) vpart[((int64_t)blockIdx.y * N + i0 + fl) * 6 + comp] = s;
  }
}

// Self term, fixed-order sum over chunks, projection and scaling.
__global__ void k_velocity_finalize(const Tables tab, int N, const float4* __restrict__ ori,
                                    const float* __restrict__ vpart, int nchunks, float4* __restrict__ tvel,
                                    float4* __restrict__ rvel) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float4 t = ori[i];
  const float d = tab.d;
  const float Fz = 2.f * tab.fz_half;            // F = (0, 0, -1)
  const float tF = t.z * Fz;
  float U[3] = {(d - 2.f) * tF * t.x, (d - 2.f) * tF * t.y, (d + 2.f) * Fz + (d - 2.f) * tF * t.z};
  float W[3] = {0.f, 0.f, 0.f};
  for (int c = 0; c < nchunks; ++c) {
    const float* p = vpart + ((int64_t)c * N + i) * 6;
    U[0] += p[0]; U[1] += p[1]; U[2] += p[2];
    W[0] += p[3]; W[1] += p[4]; W[2] += p[5];
  }
  const float tW = t.x * W[0] + t.y * W[1] + t.z * W[2];
  const float su = 0.5f / d, sr = 1.5f / d;
  tvel[i] = make_float4(U[0] * su, U[1] * su, U[2] * su, 0.f);
  rvel[i] = make_float4((W[0] - t.x * tW) * sr, (W[1] - t.y * tW) * sr, (W[2] - t.z * tW) * sr, 0.f);
}

// Analytical variant: the inner integral over fiber j in closed form (FP64),
// GF_ij(qi) = G_0(qi) F/2 + sum_k G_{k+1}(qi) a_{j,k}; the outer quadrature
// over fiber i as in the numerical kernel.  This is how the reference's
// 100_analytic_* golden files were produced (its committed
// fortran/update_velocities.incl integrates numerically in both modes).
template <int M, int Q>
__global__ void __launch_bounds__(192, 2)
k_velocity_analytical(const Tables tab, int N, const double4* __restrict__ pos, const double4* __restrict__ ori,
                      const float* __restrict__ coeff, int jchunk, float* __restrict__ vpart) {
  constexpr int TI = 192 / Q;
  constexpr int U = TI * Q;
  constexpr int M3 = 3 * M;
  __shared__ float sGs[3][U];
  const int tid = threadIdx.x;
  const int il = tid / Q, qi = tid % Q;
  const int i0 = blockIdx.x * TI;
  const int i = i0 + il;
  const bool unit_ok = tid < U && i < N;
  const double e2 = 2.0 * (double)tab.eps * (double)tab.eps;
  const float fz = tab.fz_half;
  float g0 = 0.f, g1 = 0.f, g2 = 0.f;
  const int jbeg = blockIdx.y * jchunk, jend = min(N, jbeg + jchunk);
  if (unit_ok) {
    const double4 xi4 = pos[i], ti4 = ori[i];
    const double s = (double)tab.pts[qi];
    for (int j = jbeg; j < jend; ++j) {
      if (j == i) continue;
      const double4 xj4 = pos[j], tj4 = ori[j];
      const double R0[3] = {xi4.x + s * ti4.x - xj4.x, xi4.y + s * ti4.y - xj4.y, xi4.z + s * ti4.z - xj4.z};
      const double tj[3] = {tj4.x, tj4.y, tj4.z};
      float G[6][M + 1];
      analytic_G<M>(R0, tj, e2, G);
      // F/2 = (0, 0, fz): column z of G_0
      float f0 = G[4][0] * fz, f1 = G[5][0] * fz, f2 = G[2][0] * fz;
      const float* a = coeff + (int64_t)j * M3;
#pragma unroll
      for (int k = 0; k < M; ++k) {
        const float a0 = a[3 * k], a1 = a[3 * k + 1], a2 = a[3 * k + 2];
        f0 += G[0][k + 1] * a0 + G[3][k + 1] * a1 + G[4][k + 1] * a2;
        f1 += G[3][k + 1] * a0 + G[1][k + 1] * a1 + G[5][k + 1] * a2;
        f2 += G[4][k + 1] * a0 + G[5][k + 1] * a1 + G[2][k + 1] * a2;
      }
      g0 += f0; g1 += f1; g2 += f2;
    }
  }
  if (tid < U) { sGs[0][tid] = g0; sGs[1][tid] = g1; sGs[2][tid] = g2; }
  __syncthreads();
  if (tid < TI * 6) {
    const int fl = tid / 6, comp = tid % 6;
    const int a = comp % 3;
    const bool rot = comp >= 3;
    float acc = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q) acc = fmaf(rot ? tab.W[1][q] : tab.W[0][q], sGs[a][fl * Q + q], acc);
    if (i0 + fl < N) vpart[((int64_t)blockIdx.y * N + i0 + fl) * 6 + comp] = acc;
  }
}

int launch_velocity_analytical(const Tables& tab, int N, const float4* ori, const double4* pos64,
                               const double4* ori64, const float* x, float* vpart, float4* tvel, float4* rvel,
                               cudaStream_t st) {
  const int chunks = velocity_chunks(N);
  const int jchunk = (int)ceil_div(N, chunks);
  const int TI = 192 / tab.Q;
  dim3 grid((unsigned)ceil_div(N, TI), (unsigned)chunks);
  bool done = false;
#define RF_VA_CASE(MM, QQ)                                                                   \
  if (!done && tab.M == MM && tab.Q == QQ) {                                                 \
    k_velocity_analytical<MM, QQ><<<grid, 192, 0, st>>>(tab, N, pos64, ori64, x, jchunk, vpart); \
    done = true;                                                                             \
  }
  RF_FOR_EACH_MQ(RF_VA_CASE)
#undef RF_VA_CASE
  if (!done) {
    set_last_error_str("velocity: (M, Q) combination not instantiated");
    return RF_E_UNSUPPORTED;
  }
  RF_LAUNCH_CHECK();
  k_velocity_finalize<<<(unsigned)ceil_div(N, 128), 128, 0, st>>>(tab, N, ori, vpart, chunks, tvel, rvel);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

int velocity_chunks(int N) {
  // enough CTAs to fill 148 SMs several times over for any N
  const int tiles = (int)ceil_div(N, 8);
  int chunks = (int)ceil_div(148 * 8, tiles);
  chunks = std::max(1, std::min(chunks, (int)ceil_div(N, 8)));
  return chunks;
}

// flag = 1 if any component of a or b (N float4, xyz used) is not finite
__global__ void k_check_finite(const float4* __restrict__ a, const float4* __restrict__ b, int N,
                               int* __restrict__ flag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const float4 u = a[i], w = b[i];
    const bool ok = isfinite(u.x) && isfinite(u.y) && isfinite(u.z) && isfinite(w.x) && isfinite(w.y) && isfinite(w.z);
    if (!ok) *flag = 1;   // every writer stores the same value
  }
}

int launch_check_finite(const float4* a, const float4* b, int N, int* flag, cudaStream_t st) {
  RF_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(int), st));
  k_check_finite<<<(unsigned)std::min<int64_t>(ceil_div(N, 256), 592), 256, 0, st>>>(a, b, N, flag);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

int launch_velocity_numerical(const Tables& tab, int N, const double4* pos64, const float4* ori, const float* x,
                              float4* fw, float* vpart, float4* tvel, float4* rvel, cudaStream_t st) {
  const int Q = tab.Q;
  k_source_density<<<(unsigned)std::min<int64_t>(ceil_div((int64_t)N * Q, 256), 148 * 16), 256, 0, st>>>(tab, N, x, fw);
  RF_LAUNCH_CHECK();
  const int chunks = velocity_chunks(N);
  const int jchunk = (int)ceil_div(N, chunks);
  const int TI = 192 / Q;
  dim3 grid((unsigned)ceil_div(N, TI), (unsigned)chunks);
  switch (Q) {
    case 12: k_velocity_numerical<12><<<grid, 192, 0, st>>>(tab, N, pos64, ori, fw, jchunk, vpart); break;
    case 24: k_velocity_numerical<24><<<grid, 192, 0, st>>>(tab, N, pos64, ori, fw, jchunk, vpart); break;
    case 48: k_velocity_numerical<48><<<grid, 192, 0, st>>>(tab, N, pos64, ori, fw, jchunk, vpart); break;
    default: set_last_error_str("velocity: quadrature size not instantiated"); return RF_E_UNSUPPORTED;
  }
  RF_LAUNCH_CHECK();
  k_velocity_finalize<<<(unsigned)ceil_div(N, 128), 128, 0, st>>>(tab, N, ori, vpart, chunks, tvel, rvel);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

// first != 0: x1 = x0 + dt U0, t1 = normalize(t0 + dt W0)
// otherwise: x^{n+1} = 4/3 x^n - 1/3 x^{n-1} + 2/3 dt (2 U^n - U^{n-1}), same for t, normalised.
// The state rotates in place (the reference swaps buffers, src/simulation.cu:
// 307-311): each fiber's previous state becomes its current one, the current
// one the new state, and the previous velocities the current ones, so the
// buffers a step reads and writes never change (one CUDA graph serves every
// step).
__global__ void k_update_fibers(int N, int first, double dt, double4* __restrict__ prev_pos,
                                double4* __restrict__ cur_pos, double4* __restrict__ prev_ori,
                                double4* __restrict__ cur_ori, float4* __restrict__ prev_tv,
                                const float4* __restrict__ cur_tv, float4* __restrict__ prev_rv,
                                const float4* __restrict__ cur_rv, float4* __restrict__ pos32,
                                float4* __restrict__ ori32, const int* __restrict__ halt) {
  if (halt != nullptr && *halt) return;   // the solve failed: the state stays as it is
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  update_fiber(i, first, dt, prev_pos, cur_pos, prev_ori, cur_ori, prev_tv, cur_tv[i], prev_rv, cur_rv[i], pos32,
               ori32);
}

int launch_update_fibers(int N, int first, double dt, double4* pp, double4* cp, double4* po, double4* co,
                         float4* ptv, const float4* ctv, float4* prv, const float4* crv, float4* pos32, float4* ori32,
                         const int* halt, cudaStream_t st) {
  k_update_fibers<<<(unsigned)ceil_div(N, 128), 128, 0, st>>>(N, first, dt, pp, cp, po, co, ptv, ctv, prv, crv, pos32,
                                                              ori32, halt);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

}  // namespace rf
