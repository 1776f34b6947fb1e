// Krylov solver interfaces (device-resident GMRES / BiCGSTAB).
#pragma once
#include <functional>

#include "rf_common.cuh"

namespace rf {

constexpr int kMaxRestart = 64;

// Device control block of one solve; the host reads it once per cycle.
struct GmresCtl {
  int cycle_done;     // skip the rest of this restart cycle
  int converged;      // true residual <= tol * ||b||
  int nan;            // non-finite residual seen
  int jconv;          // Arnoldi steps taken in the current cycle
  int total_iters;
  int maxit;
  int restarts;
  int timeout;        // a bounded device-side wait gave up (set by kernels)
  int heads;          // restart cycles opened from the residual of x (after the first)
  int halt;           // the solve failed (non-finite or timed out): later stages skip
  double tol;
  double bnorm;
  double beta;        // true residual norm at the last cycle start
  double estimate;    // Arnoldi residual estimate after the last step
};

// ypart = partial rows of A x (nsplit of them); `skip` is a device flag the
// matvec kernels read first and return on when set.
using MatvecFn = std::function<int(const float* x, const int* skip, cudaStream_t st)>;
// r = b - A x written to `r` (FP32), for refinement with a more accurate
// operator / accumulation than the matvec's.
using ResidualFn = std::function<int(const void* x, float* r, const int* skip, cudaStream_t st)>;

// Pieces of the GMRES restart cycles captured as CUDA graphs: [0] the first
// cycle (x = 0), [1] the head of a later one (residual of the current x),
// [2 + c] its c-th chunk of kGmresChunk Arnoldi steps.  Kernel
// arguments and buffers are fixed per handle and the tolerance / iteration
// limit live in the device control block, so a replay is exactly the launch
// sequence it was captured from.  state: 0 not run yet, 2 run once directly
// (captured on the next use), 1 ready, -1 capture not possible here (the cycle
// is then launched directly).
// Arnoldi steps between host checks in the cycles after the first
constexpr int kGmresChunk = 4;
// graph variants: the first cycle, a later cycle's head, its chunks
constexpr int kGmresGraphVariants = 2 + (kMaxRestart + kGmresChunk - 1) / kGmresChunk;
struct GmresGraphCache {
  cudaGraphExec_t exec[kGmresGraphVariants] = {};
  int state[kGmresGraphVariants] = {};
  int kernels[kGmresGraphVariants] = {};   // kernel nodes per replay
  void release();
};

struct GmresSetup {
  int64_t R;
  int m;               // restart length
  int maxit;
  double tol;
  float* V;            // (m+1) x ldv
  int64_t ldv;
  // right-preconditioned (flexible) GMRES: the matvec of column j stores
  // z_j = P v_j here and the solution update reads it; null: x += V y
  const float* Z = nullptr;
  const float* ypart;  // written by the matvec
  int nsplit;
  double* part;        // 3 * coop_blocks * (kMaxRestart + 2)
  double* H;           // (m+1) * m
  double* cs;
  double* sn;
  double* g;
  GmresCtl* ctl;       // device
  GmresCtl* host_ctl;  // pinned host
  int coop_blocks;
  GmresGraphCache* graphs = nullptr;   // null: launch every cycle directly
  cudaEvent_t wait_ev = nullptr;       // host waits (host_wait): null polls
};

struct GmresResult {
  int iterations = 0;
  int restarts = 0;
  double relative_residual = 0.0;
  int launches = 0;       // kernels launched (matvec launches counted by the caller's MatvecFn)
  int matvecs = 0;        // matvecs that did work (launches after convergence return at once)
  int residual_calls = 0; // calls of the ResidualFn (cycles after the first)
  int graph_replays = 0;  // cycles run from a captured graph
};

int krylov_coop_blocks(int64_t R, int num_sms);
// Upper bound on krylov_coop_blocks for handles created on the calling thread
// (0 = none); set by the serving loop, whose handles run concurrently.
void set_coop_block_cap(int cap);
// One cooperative block per SM, within that bound (the LU panel's grid).
int coop_blocks_per_sm_capped(int num_sms);
int gmres_solve(const GmresSetup& s, const MatvecFn& matvec, const float* b, float* x, cudaStream_t st,
                GmresResult* res);
// GMRES with iterative refinement at every restart: the Arnoldi steps use
// `matvec` (e.g. a 16-bit operator), each restart recomputes the true residual
// with `residual` and accumulates the correction into x (FP64 if x_double).
int gmres_solve_ex(const GmresSetup& s, const MatvecFn& matvec, const ResidualFn& residual, const float* b, void* x,
                   bool x_double, cudaStream_t st, GmresResult* res);

// The same solve as launches without host synchronisation, for capture into a
// graph whose restart loop is a conditional WHILE node (handle `cond`):
// gmres_enqueue_first enqueues the control-block set-up, x = 0, ||b||, the
// first cycle and the loop condition; gmres_enqueue_cycle one later cycle
// (residual of x, m Arnoldi steps, update) and the loop condition.  Steps after
// convergence return at once on the device.  *kernels counts the kernels
// these functions launch themselves (the callbacks count theirs).
int gmres_enqueue_first(const GmresSetup& s, const MatvecFn& matvec, const ResidualFn& residual, const float* b,
                        void* x, bool x_double, cudaGraphConditionalHandle cond, cudaStream_t st, int* kernels);
int gmres_enqueue_cycle(const GmresSetup& s, const MatvecFn& matvec, const ResidualFn& residual, const float* b,
                        void* x, bool x_double, cudaGraphConditionalHandle cond, cudaStream_t st, int* kernels);
// The solve's outcome from a host copy of its control block (after such a
// graph ran); returns the status gmres_solve_ex would have returned.
int gmres_result_from_ctl(const GmresCtl& h, bool has_residual, GmresResult* res);

// BiCGSTAB control block (device); stop_word is what the matvec kernels read.
struct BicgCtl {
  int stop_word;
  int converged;
  int nan;
  int need_restart;
  int iters;
  int maxit;
  int last_restart;
  int restart_every;
  int restarts;
  int pad;
  double tol;
  double bnorm;
  double rho;
  double alpha;
  double rnorm;
};

struct BicgSetup {
  int64_t R;
  int maxit;
  int restart_every;   // iterations before a restart from the true residual (ViennaCL: 200)
  double tol;
  float* work;         // 6 x ldv floats: r, r0, p, v, s, t
  int64_t ldv;
  const float* ypart;
  int nsplit;
  double* part;        // 2 * coop_blocks * (kMaxRestart + 2)
  BicgCtl* ctl;
  BicgCtl* host_ctl;
  int coop_blocks;
};

struct BicgResult {
  int iterations = 0;
  int restarts = 0;
  int matvecs = 0;
  int launches = 0;
  int refinements = 0;    // outer corrections (bicgstab_ir_solve)
  double relative_residual = 0.0;
};

int bicgstab_solve(const BicgSetup& s, const MatvecFn& matvec, const float* b, float* x, cudaStream_t st,
                   BicgResult* res);

// Buffers and targets of BiCGSTAB with FP64-residual refinement.
struct BicgIr {
  double* x64;         // R: the solution (FP64)
  float* r;            // R: the residual b - A x (FP32 copy of the FP64 sums)
  float* d;            // R: the correction
  double* norm_dev;    // 1 (device)
  double* norm_host;   // 1 (pinned host)
  double tol;          // outer target on ||b - A x|| / ||b||
  double inner_tol;    // inner BiCGSTAB target relative to ||r||
  int max_outer;       // corrections at most
};
// s.maxit bounds the inner iterations in total; res->iterations counts them,
// res->refinements the corrections.
int bicgstab_ir_solve(const BicgSetup& s, const MatvecFn& matvec, const ResidualFn& residual, const float* b,
                      const BicgIr& ir, cudaStream_t st, BicgResult* res);

struct DenseGemvPlan {
  int row_blocks;
  int splits;
  int64_t cps;  // columns per split
};
DenseGemvPlan plan_dense_gemv(int64_t R, int num_sms, int ctas_per_sm = 8);
int launch_dense_gemv(const DenseGemvPlan& p, const float* A, int64_t lda, int64_t R, const float* x, float* ypart,
                      const int* skip, cudaStream_t st);

}  // namespace rf
