// Kernel launchers shared between translation units of the library.
#pragma once
#include "rf_common.cuh"

// (M, Q) instantiations of the templated pair kernels: M Legendre terms,
// Q = 3 * intervals quadrature points per fiber (Q must be even).
#define RF_FOR_EACH_MQ(X) \
  X(1, 24) X(2, 24) X(3, 24) X(4, 24) X(5, 24) X(6, 24) X(7, 24) X(8, 24) X(5, 12) X(5, 48)

namespace rf {

// Structured storage tile: 16 x 16 fibers (a multiple of every assembly tile side).
constexpr int kStoreTile = 16;
// 16-bit storage: one record per pair, the 3 M^2 words (two 16-bit values each:
// block kI*M + kJ, values (0,1), (2,3), (4,5) of its symmetric 3x3) padded to a
// multiple of 4 words so that every record starts on a 16-byte boundary.
__host__ __device__ constexpr int s16_record_words(int M) { return (3 * M * M + 3) / 4 * 4; }
// FP32 storage: block (row, col) of a pair (Legendre indices 0..M, 0 = P_0) is
// stored at block position s32_block(M, row, col) of its (M+1)^2 blocks of 6
// values: the M^2 operator blocks (row, col >= 1) first, row-major, so that
// they are one contiguous run per pair; then row 0; then column 0.
__host__ __device__ constexpr int s32_block(int M, int row, int col) {
  return (row >= 1 && col >= 1) ? (row - 1) * M + (col - 1) : row == 0 ? M * M + col : M * M + M + row;
}

bool mq_supported(int M, int Q);
// out[r] = sum_p part[p*R + r], fixed order
int launch_reduce_rows(const float* part, int nparts, int64_t R, float* out, cudaStream_t st);
int assemble_tiles(int M, int Q, int N);

// Numerical assembly.  ffpart: assemble_tiles(M,Q,N) x N x 3(M+1) floats of
// scratch; F: N x 3(M+1) force terms sum_j T^{ij}[k][P0] F/2; b: R.  pos64:
// the FP64 centres, from which the pair separations are formed.
int launch_assemble_numerical(const Tables& tab, int N, const float4* pos, const float4* ori, const double4* pos64,
                              float* A, int64_t lda, float* ffpart, float* F, float* b, cudaStream_t st);
// Analytical integration (closed-form inner integral in FP64), dense A.
int launch_assemble_analytical(const Tables& tab, int N, const float4* pos, const float4* ori,
                               const double4* pos64, const double4* ori64, float* A, int64_t lda, float* ffpart,
                               float* F, float* b, cudaStream_t st);
// Structured storage: S32 struct_floats32(M,N) floats, S16 struct_words16(M,N) words.
int launch_assemble_structured(const Tables& tab, int N, const float4* pos, const float4* ori, const double4* pos64,
                               float* S32, uint32_t* S16, bool bf16, float* ffpart, float* F, float* b,
                               cudaStream_t st);
int64_t struct_store_tiles(int N);
int64_t struct_floats32(int M, int N);
int64_t struct_words16(int M, int N);
// y = A v on the structured operator (smode 0 FP32 / 1 FP16 / 2 BF16 storage, FP32 accumulation);
// zpart: (ceil(N/16) + 1) x R floats.
// err: device word set to 1 if a bounded wait inside the kernel gave up (may be null:
// then the register-staged kernel is used)
// variant: 0 the TMA-staged kernel where it is built (M <= 5, Q = 24, 16 bit, err
// given), else the register-staged one; 2 always the register-staged one.
int launch_struct_matvec(const Tables& tab, int N, int smode, const float* S32, const uint32_t* S16,
                         const float4* ori, const float* x, float* zpart, float* y, const int* skip, int* err,
                         cudaStream_t st, int variant = 0);
// r = b - A x with the FP32 blocks, x and accumulation in FP64; zpart64: (ceil(N/16) + 1) x R doubles.
// err as for launch_struct_matvec (null: the register-staged kernel).
int launch_struct_residual64(const Tables& tab, int N, const float* S32, const float4* ori, const double* x,
                             double* zpart64, const float* b, float* r, const int* skip, int* err, cudaStream_t st);
// y = A x with the FP32 blocks, x and accumulation in FP64 (err as for the residual).
int launch_struct_apply64(const Tables& tab, int N, const float* S32, const float4* ori, const double* x,
                          double* zpart64, float* y, int* err, cudaStream_t st);
// velocities from the FP32 blocks; vpart: ceil(N/16) x N x 6 floats.
int launch_struct_velocity(const Tables& tab, int N, const float* S32, const float4* ori, const float* F,
                           const float* x, float* vpart, float4* tvel, float4* rvel, cudaStream_t st);
int launch_cast_to_float(const double* in, float* out, int64_t n, cudaStream_t st);

// Packed mixed-precision solves (csrc/rf_pack.cu): one CTA per suspension of
// at most kPackMaxFibers fibers, M = 5, Q = 24 storage.
constexpr int kPackMaxFibers = 128;
struct PackMember {
  int N, smode, maxit, pad;      // smode 1 FP16, 2 BF16 blocks; maxit: Arnoldi steps in total
  double tol;                    // relative to ||b||
  const uint32_t* S16;
  const float* S32;
  const float4* ori;
  const float* b;
  double* x64;                   // solution (FP64)
  float* x;                      // solution (FP32 copy)
  float* V;                      // Krylov basis, m + 1 columns of ldv floats
  int64_t ldv;
  int* out;                      // iterations, restarts, refinements, status (0 ok, 1 no convergence, 2 non-finite)
  double* relres;                // ||b - A x|| / ||b|| at the last check
  float coef[5], eig[5];         // C_k = coef_k (I - E_k t t^T), k >= 1; coef_0 t t^T
};
size_t pack_smem_bytes(int Rmax, int m);
int launch_pack_gmres_ir(const PackMember* members, int n, int Rmax, int m, cudaStream_t st);

}  // namespace rf

namespace rf {
int velocity_chunks(int N);
// fw: N*Q float4 scratch; vpart: velocity_chunks(N) * N * 6 floats scratch.
int launch_check_finite(const float4* a, const float4* b, int N, int* flag, cudaStream_t st);
// pos64: the FP64 centres, from which the pair separations are formed
int launch_velocity_numerical(const Tables& tab, int N, const double4* pos64, const float4* ori, const float* x,
                              float4* fw, float* vpart, float4* tvel, float4* rvel, cudaStream_t st);
// analytical inner integrals (FP64 moments); vpart as for the numerical kernel
int launch_velocity_analytical(const Tables& tab, int N, const float4* ori, const double4* pos64,
                               const double4* ori64, const float* x, float* vpart, float4* tvel, float4* rvel,
                               cudaStream_t st);
// The second-order (or first-step Euler) update; rotates the state in place:
// prev <- cur, cur <- new, previous velocities <- current ones.  halt (may be
// null): a device word that, when set, leaves the state untouched.
int launch_update_fibers(int N, int first, double dt, double4* pp, double4* cp, double4* po, double4* co,
                         float4* ptv, const float4* ctv, float4* prv, const float4* crv, float4* pos32, float4* ori32,
                         const int* halt, cudaStream_t st);
}  // namespace rf
