// Direct solver interface (blocked LU with partial pivoting + refinement).
#pragma once
#include "rf_common.cuh"

namespace rf {

// column splits of the refinement residual (bounds the rpart buffer)
constexpr int kLuResidualSplits = 32;

struct LuSetup {
  int64_t R;
  int64_t lda;        // leading dimension of A
  int64_t ldlu = 0;   // leading dimension of LU (0: lda); a multiple of 4 for the tensor-core path
  float* LU;          // ldlu x R: the factors (a copy of A is factored)
  int* ipiv;          // R: row swapped with row j at step j (0-based, LAPACK order)
  int* perm;          // R: final row permutation, perm[i] = original row of row i
  int* host_ipiv;     // R pinned (permutation composed on the host)
  int* host_perm;     // R pinned
  float* pmax;        // 2 x coop_blocks
  int* pidx;          // 2 x coop_blocks
  float* prow;        // 2 x coop_blocks x 64: candidate pivot rows (shared-memory panel)
  float* jrow;        // 2 x 64: the diagonal row of the current column
  int* info;          // 1
  float* d;           // R: right-hand side / correction
  double* x64;        // R: refined solution
  double* r64;        // R: FP64 residual
  double* rpart;      // kLuResidualSplits x R: FP64 partial rows of A x
  double* norms;      // 2
  double tol;         // refinement target on ||b - A x|| / ||b||
  int max_refine;
  int coop_blocks;
  int panel_blocks = 0;   // blocks of the shared-memory panel kernel (0: one per SM)
  // tensor-core factorization without row exchanges (used when it gives the
  // factors of partial pivoting; null buffers: the pivoted path only)
  float* LT = nullptr;     // lu_tc_lt_floats(R): row-major copy of one pass's panels' L21
  float* inv = nullptr;    // lu_tc_inv_floats(): the diagonal block's L^-1 and U^-T
  int* flags = nullptr;    // 2: largest |l| (float bits), status
  float* sinv = nullptr;   // lu_tc_sinv_floats(R): each diagonal block's L^-1 and U^-1 (triangular solves)
  bool use_tc = true;
};

struct LuResult {
  int refinement_steps = 0;
  int factorizations = 0;   // 2 when the TF32 factors stalled and the split update was used
  int launches = 0;
  double relative_residual = 0.0;
  bool pivoted = false;     // the row-exchanging factorization ran
  double max_multiplier = 0.0;   // largest |l_ij| of the factorization without row exchanges
};

int64_t lu_tc_lt_floats(int64_t R);
int64_t lu_tc_inv_floats();
int64_t lu_tc_sinv_floats(int64_t R);
// x = (LU)^-1 rhs with the factors of lu_factor_tc (no permutation)
int lu_solve_tc(const LuSetup& s, const float* rhs, float* x, cudaStream_t st);
// The blocked factorization without row exchanges, all products on tcgen05
// (s.LU holds a copy of A): *clean when no pivot vanished and every |l_ij|
// stays within the static-pivoting limit (at most 1: the factors partial
// pivoting would produce); *max_l the largest |l_ij|.
int lu_factor_tc(const LuSetup& s, cudaStream_t st, bool* clean, int* launches, float* max_l);

// Factor A (column-major, lda) into s.LU and solve A x = b with refinement.
int lu_factor_solve(const LuSetup& s, const float* A, const float* b, float* x, cudaStream_t st, LuResult* res);
// Time the first panel factorisation (k = 0) of A with `blocks` panel blocks
// (A is copied into s.LU first); RF_E_UNSUPPORTED if the rows do not fit.
int lu_time_panel(const LuSetup& s, const float* A, int blocks, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1,
                  float* ms);

}  // namespace rf
