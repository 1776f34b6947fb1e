// Kernel launchers shared between translation units of the library.
#pragma once
#include "rf_common.cuh"

// (M, Q) instantiations of the templated pair kernels: M Legendre terms,
// Q = 3 * intervals quadrature points per fiber (Q must be even).
#define RF_FOR_EACH_MQ(X) \
  X(1, 24) X(2, 24) X(3, 24) X(4, 24) X(5, 24) X(6, 24) X(7, 24) X(8, 24) X(5, 12) X(5, 48)

namespace rf {

bool mq_supported(int M, int Q);
// out[r] = sum_p part[p*R + r], fixed order
int launch_reduce_rows(const float* part, int nparts, int64_t R, float* out, cudaStream_t st);
int assemble_tiles(int M, int Q, int N);

// Numerical assembly into dense column-major A (leading dimension lda) and b.
// bpart: assemble_tiles(M,Q,N) x R floats of scratch.
int launch_assemble_numerical(const Tables& tab, int N, const float4* pos, const float4* ori, float* A,
                              int64_t lda, float* bpart, float* b, cudaStream_t st);

}  // namespace rf

namespace rf {
int velocity_chunks(int N);
// fw: N*Q float4 scratch; vpart: velocity_chunks(N) * N * 6 floats scratch.
int launch_velocity_numerical(const Tables& tab, int N, const float4* pos, const float4* ori, const float* x,
                              float4* fw, float* vpart, float4* tvel, float4* rvel, cudaStream_t st);
int launch_update_fibers(int N, int first, double dt, const double4* pp, const double4* cp, const double4* po,
                         const double4* co, const float4* ptv, const float4* ctv, const float4* prv,
                         const float4* crv, double4* np, double4* no, float4* pos32, float4* ori32,
                         cudaStream_t st);
}  // namespace rf
