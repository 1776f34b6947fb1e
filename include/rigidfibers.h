/*
 * rigidfibers.h -- C ABI of the B200 rigid-fiber time step.
 *
 * Drop-in boundary for the reference's per-step seam, the C++ class
 * `Simulation` of ericwolter/rigidfibers (src/simulation.h:38-97), whose
 * step() (src/simulation.cu:286-329) calls assembleSystem / solveSystem /
 * updateVelocities / updateFibers.  The reference has no FFI; this header is
 * what such an FFI binds (a C or C++ program, ctypes, cgo, JNI or N-API).
 *
 * Conventions
 *  - Every function returns an int status (RF_OK == 0).  rf_last_error()
 *    returns a message for the last failure on the calling thread.
 *  - Host arrays are owned by the caller and copied in or out; the handle
 *    owns all device memory and one CUDA stream.  A handle is not
 *    thread-safe; distinct handles may be used from distinct threads.
 *  - Fiber arrays are 3N doubles, fiber-major xyz (the layout of the
 *    reference's Fortran path and of its validate dumps,
 *    fortran/fibers.f95:26-35,205-303).  The force-coefficient vector b / x
 *    has R = 3*M*N entries, index j*3M + 3k + d.  The dense matrix A is
 *    column-major R x R, entry (r, c) at A[r + c*R] (src/simulation.cu:64-110).
 */
#ifndef RIGIDFIBERS_H_
#define RIGIDFIBERS_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference prints or asserts instead
 * (src/common.h:11-25, src/simulation.cu:414,441-442). */
enum rf_status {
  RF_OK = 0,
  RF_E_INPUT = 1,       /* invalid argument, size or configuration */
  RF_E_CUDA = 2,        /* CUDA runtime error */
  RF_E_OOM = 3,         /* device allocation failed */
  RF_E_NOCONV = 4,      /* iterative solver hit its iteration limit */
  RF_E_NAN = 5,         /* NaN / Inf in b, x or the velocities */
  RF_E_TIMEOUT = 6,     /* a bounded device-side wait gave up */
  RF_E_UNSUPPORTED = 7, /* combination not built (e.g. M > 8) */
  RF_E_STATE = 8,       /* call out of order (e.g. solve before assemble) */
  RF_E_SINGULAR = 9     /* direct solver met a zero pivot */
};

/* `--gmres | --bicgstab | --magma` of fibers_runner.py (fibers_runner.py:97-100). */
enum rf_solver { RF_SOLVER_GMRES = 0, RF_SOLVER_BICGSTAB = 1, RF_SOLVER_DIRECT = 2 };

/* `--numerical | --analytical` (fibers_runner.py:102-104). */
enum rf_integration { RF_NUMERICAL = 0, RF_ANALYTICAL = 1 };

/* Storage / arithmetic of the solve.
 *  RF_PREC_FP32:  dense FP32 A (the reference's layout), FP32 Krylov solve.
 *  RF_PREC_MIXED_FP16 / _BF16: structured operator A = I + C T, T stored once
 *      per unordered fiber pair in FP32 and in 16 bits; the Krylov matvec runs
 *      on the 16-bit copy with FP32 accumulation inside FP64-residual
 *      iterative refinement, with GMRES or BiCGSTAB (not the direct solver;
 *      numerical integration only).
 *  RF_PREC_MATRIX_FREE: no matrix stored; every Krylov product recomputes the
 *      pair blocks (FP32, the assembly's kernel applied to the vector), for
 *      suspensions whose operator does not fit in device memory (the FP32
 *      path's GMRES / BiCGSTAB semantics; numerical integration only).
 *  RF_PREC_MIXED_FP16_RECOMPUTE / _BF16_RECOMPUTE: the mixed modes with only
 *      the 16-bit copy stored (304 bytes per fiber pair instead of 1168); the
 *      FP64 refinement residual and the velocities recompute the FP32 blocks
 *      from the fibers, for suspensions whose 16-bit operator fits in device
 *      memory but whose FP32 blocks do not.  Each correction costs one
 *      assembly, so these modes want a longer refinement_restart (40). */
enum rf_precision {
  RF_PREC_FP32 = 0,
  RF_PREC_MIXED_FP16 = 1,
  RF_PREC_MIXED_BF16 = 2,
  RF_PREC_MATRIX_FREE = 3,
  RF_PREC_MIXED_FP16_RECOMPUTE = 4,
  RF_PREC_MIXED_BF16_RECOMPUTE = 5
};

/* Mirrors the reference's .ini keys (tests/config.ini:18-37, read by
 * runner/cuda_runner.py:18-47) plus the runtime choices the reference made
 * at compile time (runner/cuda_runner.py:49-117). */
typedef struct rf_config {
  int number_of_timesteps;                      /* [RUN] */
  int state_save_interval;
  int velocity_save_interval;
  double timestep;                              /* [SIMULATION] */
  double slenderness;
  int number_of_terms_in_force_expansion;       /* M, 1..8 */
  int number_of_quadrature_intervals;           /* Q = 3 * intervals */
  int number_of_quadrature_points_per_interval; /* must be 3 */
  int gmres_restart;                            /* [GMRES] */
  int gmres_max_iterations;
  double gmres_tolerance;
  int bicgstab_max_iterations;                  /* [BICGSTAB] */
  double bicgstab_tolerance;
  int solver;                                   /* enum rf_solver */
  int integration;                              /* enum rf_integration */
  int precision;                                /* enum rf_precision */
  int velocity_integration;                     /* -1: same as `integration` (what
                                                   the reference's golden files were
                                                   made with); 0 numerical (what its
                                                   committed code does); 1 analytical */
  double refinement_tolerance;                  /* mixed precision: outer target on
                                                   ||b - A x|| / ||b|| */
  int refinement_max_iterations;
  int refinement_restart;                       /* mixed precision: Arnoldi steps between
                                                   FP64 residual corrections (default 20);
                                                   0 = gmres_restart */
} rf_config;

typedef struct rf_stats {
  int iterations;            /* Krylov iterations of the last solve (inner total) */
  int restarts;
  int refinement_steps;      /* outer FP64-residual corrections (mixed precision) */
  double relative_residual;  /* ||b - A x|| / ||b|| at exit, FP64 */
  /* milliseconds of the last call of each stage, CUDA events on the handle's
   * stream (names as in src/performance.cc: assemble_system, solve_system,
   * update_velocities, update_fibers) */
  double ms_assemble_system;
  double ms_solve_system;
  double ms_update_velocities;
  double ms_update_fibers;
  int64_t device_bytes;      /* device memory held by the handle */
  int kernel_launches;       /* kernels launched by the last rf_step */
  int graph_replays;         /* GMRES restart cycles of the last solve run from a
                                captured CUDA graph (0 while profiling is on) */
  int factorizations;        /* direct solver: 1 = TF32 tensor-core factors refined,
                                2 = refactored with the 3xTF32 split update */
  int pivoted;               /* direct solver: 1 when the factors were computed with
                                row exchanges (partial pivoting) because those without
                                (static pivoting) met a zero pivot, a multiplier above
                                64 or did not refine */
  double max_multiplier;     /* direct solver: largest |l_ij| of the factorization
                                without row exchanges (at most 1: partial pivoting
                                would exchange no row; 0 if it did not run) */
  double ms_step;            /* the whole last rf_step (CUDA events on the handle's
                                stream); when the step ran as one CUDA graph the four
                                stage times above are 0 */
} rf_stats;

typedef struct rf_handle rf_handle;

/* Defaults of tests/config.ini with GMRES, numerical, FP32. */
int rf_config_default(rf_config* cfg);

/* Replaces Simulation::Simulation + initializeGPUMemory +
 * writeFiberStateToDevice + precomputeLegendrePolynomials
 * (src/simulation.cu:44-284).  pos / ori: 3N doubles. */
int rf_create(const rf_config* cfg, int number_of_fibers, const double* pos, const double* ori,
              rf_handle** out);
int rf_destroy(rf_handle* h);

/* Simulation::assembleSystem (src/simulation.cu:331-399). */
int rf_assemble(rf_handle* h);
/* Simulation::solveSystem (src/simulation.cu:401-445). */
int rf_solve(rf_handle* h);
/* Simulation::updateVelocities (src/simulation.cu:447-489). */
int rf_update_velocities(rf_handle* h);
/* Simulation::updateFibers (src/simulation.cu:491-528); first_step selects
 * the Euler step of the first time step.  Also rotates the
 * previous/current/next buffers (src/simulation.cu:307-311). */
int rf_update_fibers(rf_handle* h, int first_step);
/* Simulation::step (src/simulation.cu:286-329): the four stages above. */
int rf_step(rf_handle* h, int current_timestep);
/* rf_step over `nsteps` steps starting at `first_timestep`. */
int rf_run(rf_handle* h, int first_timestep, int nsteps);

/* Packed solves of many small suspensions (no reference counterpart: the
 * ensemble path of the serving loop).  One launch per cluster size solves
 * the assembled systems of n handles, each on a thread-block cluster of 1 to
 * 8 CTAs (rf_debug_pack_plan), with the algorithm rf_solve runs in the mixed
 * modes (GMRES-IR, FP64 residual).  Members: mixed precision, GMRES,
 * 5 force terms, 8x3 quadrature, at most 256 fibers, one restart length.  A
 * member's result depends only on its own data, so it is the same alone and
 * in any pack (it may differ from rf_solve's in the last bits: the sums run
 * in another order).  Returns RF_E_NAN / RF_E_NOCONV if a member ended so;
 * rf_last_stats has each member's counts. */
int rf_solve_packed(rf_handle** handles, int n);
/* One time step of n suspensions with a packed solve: rf_assemble on each,
 * rf_solve_packed, rf_update_velocities and rf_update_fibers on each.
 * status[i] receives each member's result (RF_OK, RF_E_NOCONV, RF_E_NAN, ...). */
int rf_step_packed(rf_handle** handles, const int* timesteps, int n, int* status);

/* State and dumps (src/simulation.cu:530-822 write these to files). */
int rf_get_state(rf_handle* h, double* pos, double* ori);
int rf_set_state(rf_handle* h, const double* pos, const double* ori);
int rf_get_velocities(rf_handle* h, double* tvel, double* rvel);
/* b after assemble (before solve); A (R*R floats, column-major) only in
 * RF_PREC_FP32 mode, pass NULL to skip it. */
int rf_get_system(rf_handle* h, float* A, double* b);
/* x, the force coefficients, after solve. */
int rf_get_solution(rf_handle* h, double* x);
int rf_last_stats(rf_handle* h, rf_stats* s);
int rf_get_config(rf_handle* h, rf_config* cfg);
int rf_number_of_fibers(rf_handle* h);

/* Checkpoint / resume (the reference writes state files only,
 * src/simulation.cu:530-604; it cannot resume a second-order run).  The
 * checkpoint holds the FP64 current and previous fiber states, their FP32
 * copies, both velocity buffers, the buffer rotation and the number of steps
 * taken; loading it into a handle created with the same configuration and
 * fiber count continues the run bit for bit (continue with rf_step(h, t) for
 * t = *steps_taken, ...).  RF_E_INPUT on a mismatch or a corrupt buffer. */
int64_t rf_checkpoint_bytes(rf_handle* h);
int rf_checkpoint_save(rf_handle* h, void* buf, int64_t bytes);
int rf_checkpoint_load(rf_handle* h, const void* buf, int64_t bytes, int64_t* steps_taken);

/* y = A x with the assembled operator (3MN doubles in and out; after
 * rf_assemble).  which = 0: the working-precision operator (dense FP32 A, or
 * the FP32 pair blocks with FP64 accumulation in mixed mode); which = 1: the
 * 16-bit pair blocks of mixed mode.  Replaces the product inside the
 * reference's solver (ViennaCL prod(A, x), fortran/solve_system.incl:152)
 * for callers that run their own iteration.  Invalidates the last solution. */
int rf_operator_apply(rf_handle* h, const double* x, double* y, int which);

/* The handle's CUDA stream (cudaStream_t), for callers that order their
 * own work or events after the handle's (the reference used the default
 * stream synchronously, src/simulation.cu). */
int rf_get_stream(rf_handle* h, void** stream);
/* Per-launch timing of the solve's matvec kernels (CUDA events around each
 * launch, the role of src/performance.cc's trackers for that kernel).
 * rf_matvec_profile returns the matvecs that did work in the last solve
 * (launches issued after convergence return at once and are not counted)
 * and the summed milliseconds of those launches (the longest windows). */
int rf_set_profiling(rf_handle* h, int enable);
/* Autotuning of launch choices that leave the method unchanged: the 16-bit
 * structured matvec kernel (matvec_variant 0 = TMA-staged, 2 = register-staged;
 * matvec_ms[0], [1] their times) in mixed precision, the column splits of the
 * dense FP32 matvec (gemv_ctas_per_sm of 2, 4, 8, 16; gemv_ms[] their times,
 * -1 when not tried) in FP32, and the numerical assembly's pair-tile kernel
 * (asm_variant).  Call after rf_assemble; times each candidate with CUDA events
 * on the assembled operator, keeps the fastest for this handle and caches it
 * per (device, precision and solver, M, Q, N) for later calls (cached = 1).  The
 * summation order, hence the last bits of the solution, follow the choice.
 * (The reference compiles one kernel variant per run, runner/cuda_runner.py:49-117.) */
typedef struct rf_tune_report {
  int matvec_variant;
  double matvec_ms[2];
  int gemv_ctas_per_sm;
  double gemv_ms[4];
  int cached;
  int panel_blocks;         /* direct solver: blocks of the LU panel kernel (one
                               grid sync per column): SMs, SMs/2, SMs/4 tried */
  double panel_ms[3];       /* first panel's time per candidate (-1: rows do not fit) */
  int asm_variant;          /* numerical assembly's pair-tile kernel: 0 scalar FP32,
                               1 packed two-lane FP32 (f32x2) for mirror points; both
                               give bit-identical operators */
  double asm_ms[2];         /* one assembly per candidate (-1: not tried, analytical) */
} rf_tune_report;
int rf_autotune(rf_handle* h, rf_tune_report* report);
/* Near-field preconditioner (no reference counterpart: the reference's
 * GMRES runs unpreconditioned).  neighbours = k in [1, 8]: at every assembly
 * each fiber's k nearest fibers (centre distance) form a small block of the
 * system from the stored FP32 blocks, and the solve applies each fiber's rows
 * of that block's inverse on the right (flexible GMRES: the convergence tests
 * see the true residual, so the tolerance means what it means without it).
 * 0 turns it off (the default).  Stored mixed modes (not the recompute ones),
 * GMRES, 5 force terms; RF_E_UNSUPPORTED otherwise.  Takes effect at the next
 * rf_assemble. */
int rf_set_near_field_preconditioner(rf_handle* h, int neighbours);
/* Select the numerical assembly's pair-tile kernel by hand (the asm_variant
 * values of rf_tune_report); the operator is the same bit for bit either way.
 * RF_E_INPUT for an unknown variant. */
int rf_set_assembly_variant(rf_handle* h, int variant);

/* CUDA graphs; results are identical in every mode.  mode 1 (default): with
 * GMRES, rf_step runs the whole time step as one graph from the second step of
 * its kind on (the first step, and second-order steps): assembly, the restart
 * cycles in a conditional WHILE node that the solve ends on the device,
 * velocities and the fiber update, with one read of the solver's control
 * block afterwards (rf_stats then has ms_step but no stage times).  mode 2:
 * only the GMRES restart cycles replay from graphs (captured on their second
 * use; stage times measured).  mode 0: no graphs.  Stage-by-stage calls
 * (rf_assemble, rf_solve, ...) never use the whole-step graph. */
int rf_set_cuda_graphs(rf_handle* h, int mode);
/* Build the whole-step graphs of mode 1 now instead of on a step's second use
 * (which: 1 the first, Euler, step; 2 the second-order steps; 3 both), so that
 * no later rf_step pays for a capture and an instantiation (a serving loop
 * calls it when it admits a request).  Nothing runs on the device.  RF_OK
 * without building when the handle does not use whole-step graphs (mode 0 or
 * 2, BiCGSTAB or direct solver, profiling on); a graph that cannot be built
 * leaves rf_step on direct launches. */
int rf_prepare_step_graphs(rf_handle* h, int which);
/* How rf_step waits on the host for its results: 0 (default) polls the
 * stream, 1 sleeps on a blocking-sync event.  Polling answers a few
 * microseconds sooner; with many handles stepping from their own threads
 * (a serving loop) the polling threads take the host cores from the threads
 * that launch, so the server's handles sleep. */
int rf_set_host_wait(rf_handle* h, int blocking);
int rf_matvec_profile(rf_handle* h, int* launches, double* total_ms);

/* Device-pointer entry points (no host copies; pointers are device memory
 * on the current device, the stream may be 0).
 * rf_dense_matvec: y = A x for column-major FP32 A (R x R); replaces the
 * ViennaCL prod(A, x) behind the reference's GMRES
 * (lib/viennacl/linalg/cuda/matrix_operations_col.hpp:1251-1278). */
int rf_dense_matvec(const float* A, const float* x, float* y, int64_t R, void* stream);
/* rf_dense_lu_solve: x = A^{-1} b for column-major FP32 A (R x R) by LU and
 * FP64-residual refinement until ||b - A x|| / ||b|| <= tol (RF_E_NOCONV after
 * 20 steps, RF_E_SINGULAR on a zero pivot); A and b are not modified.  The LU
 * is first computed without row exchanges on the tensor cores (static
 * pivoting; with every multiplier at most 1 these are partial pivoting's
 * factors) and recomputed with partial pivoting when a pivot vanishes, a
 * multiplier exceeds 64 or the refinement does not converge.  Replaces
 * MAGMA's magma_sgesv_gpu behind the reference's --magma path
 * (src/simulation.cu:403-418). */
int rf_dense_lu_solve(const float* A, const float* b, float* x, int64_t R, double tol, void* stream);
/* rf_dense_matvec_noalloc: the same y = A x, for callers that cannot let a
 * library allocate device memory (a host program whose pool allocator owns all
 * of HBM, or a loop that cannot afford cudaMalloc's latency).  It has no
 * counterpart in the reference.  Its scratch is a fixed 8 MiB array in the
 * library's device image (held on every GPU that loads the library until the
 * process exits), so R must not exceed 131072 (RF_E_INPUT otherwise).  The
 * first call in a CUDA context (for the primary context: the first call on
 * that device) looks up that array's device address; make that first call
 * before any stream capture.  The address is cached per context, so after
 * cudaDeviceReset the next call looks it up again in the new context.  All
 * calls share the one array: calls that overlap on the GPU (different
 * streams, or different host threads on the same device) race and must be
 * serialised by the caller. */
int rf_dense_matvec_noalloc(const float* A, const float* x, float* y, int64_t R, void* stream);

/* ---- Serving: an ensemble of independent suspensions ------------------------
 * The reference runs one suspension per process (fibers_runner.py:17-162 starts
 * one `fibers` binary per configuration).  The server below runs many at once
 * on one GPU: requests are admitted in arrival order while a slot is free and
 * their device memory (rf_device_bytes_estimate) fits hbm_budget_bytes; each
 * runs on its own handle and stream, so requests overlap on the device, and its
 * result equals that of a lone rf_create + rf_step loop on the same inputs. */
enum rf_request_status { RF_REQ_QUEUED = 0, RF_REQ_RUNNING = 1, RF_REQ_DONE = 2, RF_REQ_FAILED = 3, RF_REQ_CANCELLED = 4 };

typedef struct rf_server rf_server;

typedef struct rf_server_config {
  int max_active;            /* requests running at once on their own handles
                                (default 8; the pack's members are not counted) */
  int64_t hbm_budget_bytes;  /* sum of the running requests' estimates */
  int use_cuda_graphs;       /* rf_set_cuda_graphs mode of every request's handle
                                (default 2: restart cycles; 1: whole-step graphs, built
                                when the request is admitted, rf_prepare_step_graphs) */
  int pack_max_fibers;       /* requests of at most this many fibers (<= 256, mixed
                                precision, GMRES, 5 terms, 8x3 quadrature) step together
                                with packed solves (rf_step_packed); 0: off.
                                Default 128 */
  int pack_max_members;      /* suspensions per pack */
  int64_t reserve_bytes;     /* device memory taken into the handles' pool when the
                                server starts (at most hbm_budget_bytes), so that
                                admitting a large request does not grow the pool while
                                others step: growing it maps new memory, which holds
                                up every stream of the device.  Default: a quarter
                                of the budget; 0: grow on demand */
} rf_server_config;

typedef struct rf_request_stats {
  int steps_done;
  double queue_ms;      /* submit -> admission */
  double run_ms;        /* admission -> last step done */
  double mean_step_ms;  /* host wall time of rf_step, mean */
  int64_t device_bytes; /* admission estimate */
  double setup_ms;      /* admission -> ready to step (handle created, graphs built) */
} rf_request_stats;

typedef struct rf_server_stats {
  int64_t steps;        /* completed steps of completed requests */
  double p50_step_ms;   /* step latency percentiles over those steps */
  double p99_step_ms;
  int64_t fiber_steps;  /* sum of fibers x steps */
  double elapsed_s;     /* server creation -> last completion */
  int peak_active;
  int64_t peak_bytes;
  int completed, failed, queued, active;
  /* the pack (pack_max_fibers > 0): its rf_step_packed calls, their host wall
     time percentiles and maximum, and the mean suspensions per call */
  int64_t pack_steps;
  double pack_p50_ms, pack_p99_ms, pack_max_ms;
  double pack_mean_members;
  /* admission -> ready to step, percentiles over completed requests */
  double p50_setup_ms, p99_setup_ms;
} rf_server_stats;

/* Device bytes a handle of this configuration and size allocates (an upper
 * estimate used for admission). */
int64_t rf_device_bytes_estimate(const rf_config* cfg, int number_of_fibers);
int rf_server_config_default(rf_server_config* cfg);
int rf_server_create(const rf_server_config* cfg, rf_server** server);
/* Queue `nsteps` time steps of a suspension; pos/ori are copied. */
int rf_server_submit(rf_server* s, const rf_config* cfg, int number_of_fibers, const double* pos,
                     const double* ori, int nsteps, int64_t* request_id);
int rf_server_poll(rf_server* s, int64_t request_id, int* status, int* steps_done);
int rf_server_cancel(rf_server* s, int64_t request_id);
int rf_server_wait(rf_server* s, int64_t request_id, double timeout_seconds);
int rf_server_drain(rf_server* s, double timeout_seconds);
/* Final state and last velocities (any pointer may be NULL). */
int rf_server_result(rf_server* s, int64_t request_id, double* pos, double* ori, double* tvel, double* rvel,
                     rf_request_stats* stats);
int rf_server_get_stats(rf_server* s, rf_server_stats* stats);
/* Host wall time of each step of a finished request, in step order: copies
 * min(capacity, steps) values to ms (may be NULL) and the step count to
 * *count.  RF_E_STATE while the request runs. */
int rf_server_step_times(rf_server* s, int64_t request_id, double* ms, int capacity, int* count);
/* Cancels what has not finished, waits for running steps, frees everything. */
int rf_server_destroy(rf_server* s);

/* Fault injection for tests (no counterpart in the reference, which prints and
 * continues).  rf_debug_set_device_wait_limit(0) makes the first bounded
 * device-side wait of the TMA-pipelined matvec and of the tensor-core LU
 * update give up at once, so the calls return RF_E_TIMEOUT and the handle stays
 * usable; -1 restores the limits (2^24 polls, one second).
 * rf_debug_fail_allocation_after(n): the n-th device allocation of rf_create
 * from now on fails (RF_E_OOM); -1 disables. */
int rf_debug_set_device_wait_limit(int64_t limit);
int rf_debug_fail_allocation_after(int n);
/* The column-split plan rf_dense_matvec_noalloc uses for R rows on a GPU with
 * `sms` multiprocessors (no device needed): the number of splits and the
 * columns per split, capped so that splits x R partial rows fit its fixed
 * scratch array.  RF_E_INPUT when R is outside [1, 131072] or sms < 1. */
int rf_debug_noalloc_plan(int64_t R, int sms, int* splits, int64_t* cols_per_split);
/* The CTAs (a thread-block cluster of 1, 2, 4 or 8) that rf_solve_packed and
 * rf_step_packed give each member of a pack of n suspensions of fibers[i]
 * fibers on a GPU with `sms` multiprocessors (no device needed): every member
 * starts at one CTA (two above 128 fibers), then the member with the most
 * 16 x 16-fiber storage tiles per CTA doubles its cluster while the pack's
 * CTAs stay within sms and every CTA keeps two tiles.  A member's result is
 * the same bits for every cluster size.  RF_E_INPUT when n < 1, sms < 1 or a
 * size is outside [1, 256]. */
int rf_debug_pack_plan(const int* fibers, int n, int sms, int* ctas);

const char* rf_status_string(int status);
const char* rf_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* RIGIDFIBERS_H_ */
