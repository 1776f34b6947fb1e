// Direct solver interface (blocked LU with partial pivoting + refinement).
#pragma once
#include "rf_common.cuh"

namespace rf {

struct LuSetup {
  int64_t R;
  int64_t lda;
  float* LU;          // lda x R: the factors (a copy of A is factored)
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
  double* norms;      // 2
  double tol;         // refinement target on ||b - A x|| / ||b||
  int max_refine;
  int coop_blocks;
  int panel_blocks = 0;   // blocks of the shared-memory panel kernel (0: one per SM)
};

struct LuResult {
  int refinement_steps = 0;
  int factorizations = 0;   // 2 when the TF32 factors stalled and the split update was used
  int launches = 0;
  double relative_residual = 0.0;
};

// Factor A (column-major, lda) into s.LU and solve A x = b with refinement.
int lu_factor_solve(const LuSetup& s, const float* A, const float* b, float* x, cudaStream_t st, LuResult* res);
// Time the first panel factorisation (k = 0) of A with `blocks` panel blocks
// (A is copied into s.LU first); RF_E_UNSUPPORTED if the rows do not fit.
int lu_time_panel(const LuSetup& s, const float* A, int blocks, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1,
                  float* ms);

}  // namespace rf
