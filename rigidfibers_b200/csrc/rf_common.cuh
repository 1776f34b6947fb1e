// Shared definitions of the rigid-fiber CUDA library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <cstdio>

#include "../../include/rigidfibers.h"

namespace rf {

constexpr int kMaxTerms = 8;      // Legendre terms supported (closed forms to P_8)
constexpr int kMaxQuad = 48;      // quadrature points per fiber (16 intervals x 3)

// Per-launch tables, passed by value so every kernel sees them through the
// constant parameter bank (no module-global state: handles with different
// slenderness / M / Q can run side by side).
//   W[k][q] = w_q * P_k(s_q) for k = 0..M (P_0 = 1 carries the force term,
//   P_k, k>=1, carries force index k-1, as in fortran/fibers.f95:403-408).
struct Tables {
  float pts[kMaxQuad];
  float W[kMaxTerms + 1][kMaxQuad];   // W[0][q] = w_q
  // W2[k][q] = (W[k][q], W[k][q]) for q < Q/2: the weight as the second
  // operand of a packed two-lane FP32 multiply-add
  float2 W2[kMaxTerms + 1][kMaxQuad / 2];
  float gamma[kMaxTerms];   // gamma[0] = D1 (force index 0), gamma[k] for k>=1
  float eigen[kMaxTerms];   // E_k; unused for k = 0
  float e2;                 // 2 * eps^2
  float fz_half;            // external force z / 2 = -0.5 (fortran/fibers.f95:149)
  float d;                  // -log(eps^2 e)
  float eps;                // slenderness
  int M, Q;
};


// Error plumbing: every launch is checked; the C ABI maps failures to codes.
#define RF_CUDA_TRY(expr)                                                          \
  do {                                                                             \
    cudaError_t _e = (expr);                                                       \
    if (_e != cudaSuccess) {                                                       \
      ::rf::set_last_error(cudaGetErrorString(_e), __FILE__, __LINE__);            \
      return _e == cudaErrorMemoryAllocation ? RF_E_OOM : RF_E_CUDA;               \
    }                                                                              \
  } while (0)

#define RF_LAUNCH_CHECK() RF_CUDA_TRY(cudaGetLastError())

// propagate a non-zero rf_status
#define RF_TRY_RF(expr)             \
  do {                              \
    int _rc = (expr);               \
    if (_rc != RF_OK) return _rc;   \
  } while (0)

void set_last_error(const char* msg, const char* file, int line);
void set_last_error_str(const char* msg);
// Fault injection (tests): limit of the first bounded device-side wait of the
// TMA and tensor-core kernels (polls for the TMA pipeline, nanoseconds for the
// tensor-core commit); -1 keeps the defaults.  Waits that drain in-flight work
// after a failure always use the defaults.
int64_t device_wait_limit();

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Host wait for the work queued on st so far.  ev null: cudaStreamSynchronize
// (the thread polls); else ev, an event created with cudaEventBlockingSync, is
// recorded and waited on, which puts the thread to sleep until the work is
// done -- many threads waiting at once (a serving loop) then leave the host
// cores to the threads that launch.
inline cudaError_t host_wait(cudaStream_t st, cudaEvent_t ev) {
  if (!ev) return cudaStreamSynchronize(st);
  const cudaError_t e = cudaEventRecord(ev, st);
  return e != cudaSuccess ? e : cudaEventSynchronize(ev);
}

// FP32 -> FP64 without flushing subnormal inputs: with -ftz=true a plain cast
// becomes a conversion plus a flushing multiply; the conversion alone is exact
// for every FP32 value
__device__ __forceinline__ double f2d(float v) {
  double d;
  asm("cvt.f64.f32 %0, %1;" : "=d"(d) : "f"(v));
  return d;
}

// Symmetric 3x3 stored as (11, 22, 33, 12, 13, 23) -- the order of
// fortran/compute_inner_integral_numerically.incl:179-184.
__device__ __forceinline__ float sym_get(const float* s6, int a, int b) {
  const int idx[3][3] = {{0, 3, 4}, {3, 1, 5}, {4, 5, 2}};
  return s6[idx[a][b]];
}

}  // namespace rf
