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

// Kernel variants of the numerical pair tiles (rf_autotune picks one; both
// give bit-identical results): 0 scalar FP32, 1 packed two-lane FP32
// (add/mul/fma .f32x2) for the two mirror points of each folded pair.
constexpr int kAsmVariants = 2;
// Numerical assembly.  ffpart: assemble_tiles(M,Q,N) x N x 3(M+1) floats of
// scratch; F: N x 3(M+1) force terms sum_j T^{ij}[k][P0] F/2; b: R.  pos64:
// the FP64 centres, from which the pair separations are formed.
int launch_assemble_numerical(const Tables& tab, int N, const float4* pos, const float4* ori, const double4* pos64,
                              float* A, int64_t lda, float* ffpart, float* F, float* b, cudaStream_t st,
                              int variant = 0);
// Analytical integration (closed-form inner integral in FP64), dense A.
int launch_assemble_analytical(const Tables& tab, int N, const float4* pos, const float4* ori,
                               const double4* pos64, const double4* ori64, float* A, int64_t lda, float* ffpart,
                               float* F, float* b, cudaStream_t st);
// Matrix-free (nothing stored): with x, z partial rows of T x into zpart
// ((assemble_tiles(M,Q,N) + 1) x R floats, every row written) -- finish the
// product with launch_parts_finalize; with x null, the force terms F and b
// (ffpart as for the numerical assembly).  skip as for the structured matvec.
int launch_assemble_apply(const Tables& tab, int N, const float4* pos, const float4* ori, const double4* pos64,
                          const float* x, float* zpart, const int* skip, float* ffpart, float* F, float* b,
                          cudaStream_t st, int variant = 0);
// y = x + C z with z the fixed-order sum of nparts partial rows of zpart
// (zpart holds nparts + 1 rows: the sum goes to row nparts).
int launch_parts_finalize(const Tables& tab, int N, const float4* ori, const float* x, float* zpart, int nparts,
                          float* y, const int* skip, cudaStream_t st);
// r = b - (x + C z) with z the sum of nparts FP32 partial-row slots of a
// matrix-free product (launch_assemble_apply), summed in FP64, x in FP64
int launch_parts_residual64(const Tables& tab, int N, const float4* ori, const double* x, const float* zpart,
                            int nparts, const float* b, float* r, const int* skip, cudaStream_t st);
// Structured storage: S32 struct_floats32(M,N) floats, S16 struct_words16(M,N) words.
int launch_assemble_structured(const Tables& tab, int N, const float4* pos, const float4* ori, const double4* pos64,
                               float* S32, uint32_t* S16, bool bf16, float* ffpart, float* F, float* b,
                               cudaStream_t st, int variant = 0);
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

// Near-field preconditioner (csrc/rf_precond.cu; M = 5, stored FP32 blocks):
// nb (N x (k+1) ints) the k nearest fibers of each fiber, W (nf_w_floats(N)
// floats) each fiber's rows of the inverse of its neighbourhood block; the
// apply writes z = P v (every row).
constexpr int kNfMaxNeighbours = 8;
int64_t nf_w_floats(int N);
int launch_nf_setup(const Tables& tab, int N, int k, const float4* pos, const float4* ori, const float* S32, int* nb,
                    float* W, cudaStream_t st);
int launch_nf_apply(int N, int k, const int* nb, const float* W, const float* v, float* z, const int* skip,
                    cudaStream_t st);

// Packed mixed-precision solves (csrc/rf_pack.cu): one thread-block cluster
// per suspension of at most kPackMaxFibers fibers, M = 5, Q = 24 storage.
constexpr int kPackMaxFibers = 256;
// the largest member one CTA takes (its 8 partitions' rows in shared memory);
// larger members run on clusters of at least two CTAs
constexpr int kPackSingleMaxFibers = 128;
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
// CTAs (a thread-block cluster of 1, 2, 4 or 8) per member of a packed solve:
// starting from one each (two above kPackSingleMaxFibers fibers), the member
// with the most storage tiles per CTA doubles its cluster while the pack's
// CTAs stay within sms, each CTA keeps at least two tiles and the cluster
// stays within max_cluster.  A member's result does not depend on its
// cluster size.
void pack_plan_ctas(const int* fibers, int n, int sms, int* ctas, int max_cluster);
// the largest cluster of the packed solve this device can schedule (8, 4, 2 or 1)
int pack_max_cluster();
size_t pack_smem_bytes(int Rmax, int m, int csize);
// Streams and events the packed solve forks its cluster-size classes onto.
struct PackLanes {
  cudaStream_t aux[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t fork = nullptr, join[3] = {nullptr, nullptr, nullptr};
};
void pack_lanes_release(PackLanes& lanes);
// members: counts[0] members with clusters of 8, then counts[1] of 4,
// counts[2] of 2 and counts[3] of 1 CTA; rmax[c]: the largest system (rows)
// of class c
int launch_pack_gmres_ir(const PackMember* members, const int (&counts)[4], const int (&rmax)[4], int m,
                         cudaStream_t st, PackLanes& lanes);

// One suspension of a packed step: the buffers its assembly, velocities and
// update read and write.  The packed stage kernels launch once per group of
// members with the same Tables (slenderness); within a group, member m owns
// blocks [asm_start, asm_start + its tile pairs) of the assembly grid and
// [vel_start, ...) of the velocity grid.
struct PackStepMember {
  int N, first;               // fibers; 1 on a first (Euler) step
  int asm_start, vel_start;   // first block of the member in the group's grids
  double dt;
  const int* solve_status;    // the packed solve's status word (2: non-finite, the member sits out)
  int* vbad;                  // set to 1 when a velocity is not finite, else 0
  double4 *pos64, *pos64_prev, *ori64, *ori64_prev;   // FP64 state: current, previous
  float4 *pos32, *ori32;      // FP32 copies of the current state
  float4 *tv, *tv_prev, *rv, *rv_prev;                 // velocities: current, previous
  float* S32;
  uint32_t* S16;
  float *ffpart, *F, *b;      // assembly scratch, force terms, right-hand side
  const float* x;             // the solve's FP32 solution
  float* vpart;               // velocity partials
};
// The member of a packed group that owns block L of a grid whose members'
// first blocks (ascending) are starts(m): the last member with starts(m) <= L.
template <class StartOf>
__device__ __forceinline__ int pack_member_of(int n, int L, StartOf starts) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (starts(mid) <= L) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
// numerical structured assembly + force terms of every member of one group
int launch_pack_assemble(const Tables& tab, const PackStepMember* members, int n, int64_t blocks, bool bf16,
                         cudaStream_t st);
// velocities, the non-finite guard and the fiber update of every member of one group
int launch_pack_velocity_update(const Tables& tab, const PackStepMember* members, int n, int64_t blocks,
                                cudaStream_t st);

}  // namespace rf

namespace rf {
// The handles' device memory pool of device dev (csrc/rf_capi.cu), and the
// count of its users (handles and servers) that keeps freed memory in it.
cudaError_t handle_pool(int dev, cudaMemPool_t* out);
void pools_acquire();
void pools_release();
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
// Fiber i's second-order step (fortran/update_fibers.incl; the first step,
// fortran/update_fibers_firststep.incl, is explicit Euler):
// x' = 4/3 x - 1/3 x_prev + 2/3 dt (2 U - U_prev), the same for t with W, then
// t' normalised.  Writes the rotated state: prev <- current, current <- new.
// Every rounding is explicit (fma, __dmul_rn), so kernels that inline this
// agree bit for bit whatever the compiler would contract.
__device__ __forceinline__ double bdf2_coord(double c43, double c13, double c23, double xc, double xp, float u,
                                             float up) {
  return fma(c23, fma(2.0, (double)u, -(double)up), fma(c43, xc, __dmul_rn(-c13, xp)));
}
__device__ __forceinline__ void update_fiber(int i, int first, double dt, double4* __restrict__ prev_pos,
                                             double4* __restrict__ cur_pos, double4* __restrict__ prev_ori,
                                             double4* __restrict__ cur_ori, float4* __restrict__ prev_tv,
                                             float4 u, float4* __restrict__ prev_rv, float4 w,
                                             float4* __restrict__ pos32, float4* __restrict__ ori32) {
  const double4 xc = cur_pos[i], tc = cur_ori[i];
  double4 xn, tn;
  if (first) {
    xn = make_double4(fma(dt, (double)u.x, xc.x), fma(dt, (double)u.y, xc.y), fma(dt, (double)u.z, xc.z), 0.0);
    tn = make_double4(fma(dt, (double)w.x, tc.x), fma(dt, (double)w.y, tc.y), fma(dt, (double)w.z, tc.z), 0.0);
  } else {
    const double4 xp = prev_pos[i], tp = prev_ori[i];
    const float4 up = prev_tv[i], wp = prev_rv[i];
    const double c43 = 4.0 / 3.0, c13 = 1.0 / 3.0, c23 = (2.0 / 3.0) * dt;
    xn = make_double4(bdf2_coord(c43, c13, c23, xc.x, xp.x, u.x, up.x), bdf2_coord(c43, c13, c23, xc.y, xp.y, u.y, up.y),
                      bdf2_coord(c43, c13, c23, xc.z, xp.z, u.z, up.z), 0.0);
    tn = make_double4(bdf2_coord(c43, c13, c23, tc.x, tp.x, w.x, wp.x), bdf2_coord(c43, c13, c23, tc.y, tp.y, w.y, wp.y),
                      bdf2_coord(c43, c13, c23, tc.z, tp.z, w.z, wp.z), 0.0);
  }
  const double inv = 1.0 / sqrt(fma(tn.z, tn.z, fma(tn.y, tn.y, __dmul_rn(tn.x, tn.x))));
  tn.x = __dmul_rn(tn.x, inv);
  tn.y = __dmul_rn(tn.y, inv);
  tn.z = __dmul_rn(tn.z, inv);
  prev_pos[i] = xc;
  prev_ori[i] = tc;
  cur_pos[i] = xn;
  cur_ori[i] = tn;
  prev_tv[i] = u;
  prev_rv[i] = w;
  pos32[i] = make_float4((float)xn.x, (float)xn.y, (float)xn.z, 0.f);
  ori32[i] = make_float4((float)tn.x, (float)tn.y, (float)tn.z, 0.f);
}

// The second-order (or first-step Euler) update; rotates the state in place:
// prev <- cur, cur <- new, previous velocities <- current ones.  halt (may be
// null): a device word that, when set, leaves the state untouched.
int launch_update_fibers(int N, int first, double dt, double4* pp, double4* cp, double4* po, double4* co,
                         float4* ptv, const float4* ctv, float4* prv, const float4* crv, float4* pos32, float4* ori32,
                         const int* halt, cudaStream_t st);
}  // namespace rf
