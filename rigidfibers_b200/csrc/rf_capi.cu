// C ABI of the rigid-fiber time step: the handle owns the device state and
// one stream, and runs the reference's step
// (src/simulation.cu:286-329: assembleSystem -> solveSystem ->
// updateVelocities -> updateFibers -> buffer rotation).
#include <algorithm>
#include <cmath>
#include <functional>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

#include "rf_common.cuh"
#include "rf_kernels.cuh"
#include "rf_krylov.cuh"
#include "rf_lu.cuh"

#include <nvtx3/nvToolsExt.h>

namespace rf {

static thread_local std::string g_last_error;

void set_last_error(const char* msg, const char* file, int line) {
  g_last_error = std::string(msg) + " (" + file + ":" + std::to_string(line) + ")";
}
void set_last_error_str(const char* msg) { g_last_error = msg; }

static std::atomic<int64_t> g_wait_limit{-1};
static std::atomic<int> g_fail_alloc_after{-1};
int64_t device_wait_limit() { return g_wait_limit.load(); }

// ---- memory for handles that come and go while others step ----------------
// Allocating or freeing page-locked host memory is an implicit synchronisation
// point of the whole device, so the handles' small page-locked control blocks
// come from this process-wide pool: slabs are allocated once and never freed,
// blocks are recycled per power-of-two size class.
class PinnedPool {
 public:
  void* get(size_t bytes) {
    const size_t cls = size_class(bytes);
    std::lock_guard<std::mutex> lk(mu_);
    std::vector<void*>& fl = free_[cls];
    if (!fl.empty()) {
      void* p = fl.back();
      fl.pop_back();
      return p;
    }
    if (cls > left_) {
      const size_t slab = std::max<size_t>(size_t(1) << 20, cls);
      void* m = nullptr;
      if (cudaMallocHost(&m, slab) != cudaSuccess) return nullptr;
      cur_ = static_cast<char*>(m);
      left_ = slab;
    }
    void* p = cur_;
    cur_ += cls;
    left_ -= cls;
    return p;
  }
  void put(void* p, size_t bytes) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(mu_);
    free_[size_class(bytes)].push_back(p);
  }

 private:
  static size_t size_class(size_t bytes) {
    size_t c = 256;
    while (c < bytes) c <<= 1;
    return c;
  }
  std::mutex mu_;
  std::map<size_t, std::vector<void*>> free_;
  char* cur_ = nullptr;
  size_t left_ = 0;
};
static PinnedPool& pinned_pool() {
  static PinnedPool* p = new PinnedPool();   // outlives every handle (never destroyed)
  return *p;
}

// Device memory of the handles comes from one memory pool per device that
// keeps what is freed (release threshold at its maximum) while any handle or
// server is alive, and gives it back when the last one goes.  The default pool
// returns unused memory to the driver at every synchronisation, so each new
// request of a serving loop would map its buffers afresh.
struct DevicePools {
  std::mutex mu;
  std::map<int, cudaMemPool_t> pool;
  int live = 0;   // handles + servers
};
static DevicePools& device_pools() {
  static DevicePools* p = new DevicePools();
  return *p;
}
cudaError_t handle_pool(int dev, cudaMemPool_t* out) {
  DevicePools& d = device_pools();
  std::lock_guard<std::mutex> lk(d.mu);
  auto it = d.pool.find(dev);
  if (it != d.pool.end()) {
    *out = it->second;
    return cudaSuccess;
  }
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t pool = nullptr;
  cudaError_t e = cudaMemPoolCreate(&pool, &props);
  if (e != cudaSuccess) return e;
  uint64_t keep = ~uint64_t(0);
  e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  if (e != cudaSuccess) {
    cudaMemPoolDestroy(pool);
    return e;
  }
  d.pool[dev] = pool;
  *out = pool;
  return cudaSuccess;
}
void pools_acquire() {
  DevicePools& d = device_pools();
  std::lock_guard<std::mutex> lk(d.mu);
  d.live += 1;
}
void pools_release() {
  DevicePools& d = device_pools();
  std::lock_guard<std::mutex> lk(d.mu);
  if (--d.live == 0)
    for (auto& kv : d.pool) cudaMemPoolTrimTo(kv.second, 0);
}

bool mq_supported(int M, int Q) {
#define RF_MQ_CASE(MM, QQ) \
  if (M == MM && Q == QQ) return true;
  RF_FOR_EACH_MQ(RF_MQ_CASE)
#undef RF_MQ_CASE
  return false;
}

// fortran/fibers.f95:141-145,353-476: quadrature, Legendre, lambda and E_k
// in double, then the working-precision constants as the REAL*4 program
// forms them (c, d, D1 and gamma in single precision).
static Tables make_tables(const rf_config& c) {
  Tables t;
  std::memset(&t, 0, sizeof(t));
  const int M = c.number_of_terms_in_force_expansion;
  const int nint = c.number_of_quadrature_intervals;
  const int Q = 3 * nint;
  t.M = M;
  t.Q = Q;
  const double p[3] = {-std::sqrt(15.0) / 5.0, 0.0, std::sqrt(15.0) / 5.0};
  const double w[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
  const double h = 2.0 / nint;
  double lower = -1.0;
  std::vector<double> pts, wts;
  for (int iv = 0; iv < nint; ++iv) {
    for (int k = 0; k < 3; ++k) {
      pts.push_back((2.0 * lower + h + p[k] * h) / 2.0);
      wts.push_back(w[k] / nint);
    }
    lower += h;
  }
  auto P = [](double x, int n) -> double {
    switch (n) {
      case 0: return 1.0;
      case 1: return x;
      case 2: return 0.5 * (3.0 * x * x - 1.0);
      case 3: return 0.5 * (5.0 * x * x * x - 3.0 * x);
      case 4: return 0.125 * (35.0 * std::pow(x, 4) - 30.0 * x * x + 3.0);
      case 5: return 0.125 * (63.0 * std::pow(x, 5) - 70.0 * std::pow(x, 3) + 15.0 * x);
      case 6: return 0.0625 * (231.0 * std::pow(x, 6) - 315.0 * std::pow(x, 4) + 105.0 * x * x - 5.0);
      case 7: return 0.0625 * (429.0 * std::pow(x, 7) - 693.0 * std::pow(x, 5) + 315.0 * std::pow(x, 3) - 35.0 * x);
      case 8:
        return (1.0 / 128.0) *
               (6435.0 * std::pow(x, 8) - 12012.0 * std::pow(x, 6) + 6930.0 * std::pow(x, 4) - 1260.0 * x * x + 35.0);
    }
    return 0.0;
  };
  for (int q = 0; q < Q; ++q) {
    t.pts[q] = (float)pts[q];
    for (int k = 0; k <= M; ++k) {
      // weight and Legendre value rounded separately, as the REAL*4 tables are
      t.W[k][q] = (float)wts[q] * (float)P(pts[q], k);
      if (2 * q < Q) t.W2[k][q] = make_float2(t.W[k][q], t.W[k][q]);
    }
  }
  const double eps = c.slenderness;
  const double cd = std::log(eps * eps * std::exp(1.0));
  const double dd = -cd;
  std::vector<double> lam(M), eig(M);
  lam[0] = 2.0;
  eig[0] = ((dd - 2.0 - lam[0]) / 2.0) / (dd - lam[0]);
  for (int k = 1; k < M; ++k) {
    lam[k] = lam[k - 1] + 2.0 / (k + 1);
    eig[k] = ((dd - 2.0 - lam[k]) / 2.0) / (dd - lam[k]);
  }
  const float epsf = (float)eps;
  const float cf = std::log(epsf * epsf * std::exp(1.0f));
  const float df = -cf;
  t.d = df;
  t.e2 = 2.0f * epsf * epsf;
  t.eps = epsf;
  t.fz_half = -0.5f;
  t.gamma[0] = 0.75f / (df - 2.0f * 1.0f);  // D1
  t.eigen[0] = (float)eig[0];
  for (int k = 1; k < M; ++k) {
    t.gamma[k] = 0.5f * (2.0f * (float)(k + 1) + 1.0f) / (df + 2.0f - 1.0f * (float)lam[k]);
    t.eigen[k] = (float)eig[k];
  }
  return t;
}

}  // namespace rf

using namespace rf;

// 16-bit storage format of the mixed modes: 1 FP16, 2 BF16
static int storage16(const rf_config& c) {
  return c.precision == RF_PREC_MIXED_BF16 || c.precision == RF_PREC_MIXED_BF16_RECOMPUTE ? 2 : 1;
}

struct rf_handle {
  rf_config cfg;
  int N = 0, M = 0, Q = 0;
  int64_t R = 0, lda = 0;
  Tables tab;
  cudaStream_t st = nullptr;
  int dev = 0, num_sms = 148;
  // fiber state: FP64 master copies (prev, cur, next rotate) and FP32 views
  double4* pos64[3] = {nullptr, nullptr, nullptr};
  double4* ori64[3] = {nullptr, nullptr, nullptr};
  int iprev = 0, icur = 1, inext = 2;
  float4* pos32 = nullptr;
  float4* ori32 = nullptr;
  float4* tv[2] = {nullptr, nullptr};
  float4* rv[2] = {nullptr, nullptr};
  int vprev = 0, vcur = 1;   // velocity buffers; vcur is written by update_velocities
  int vlast = -1;            // buffer holding the most recent velocities
  bool vel_fresh = false;    // velocities computed since the last fiber update
  // linear system
  bool mixed = false;        // structured operator + refinement (RF_PREC_MIXED_*)
  bool mfree = false;        // no operator stored (RF_PREC_MATRIX_FREE)
  bool recompute = false;    // mixed with the 16-bit copy only (RF_PREC_MIXED_*_RECOMPUTE)
  float* xcast = nullptr;    // recompute: the FP32 copy of x for the residual's product
  // near-field preconditioner (rf_set_near_field_preconditioner): neighbours per
  // fiber (0: off), neighbour lists, the fibers' rows of the neighbourhood
  // inverses, and the preconditioned basis z_j of flexible GMRES
  int nf_k = 0;
  int* nf_nb = nullptr;
  float* nf_w = nullptr;
  float* nf_z = nullptr;
  int zparts = 0;            // matrix-free: partial-row slots of a product
  float* A = nullptr;        // dense FP32 (RF_PREC_FP32)
  float* S32 = nullptr;      // structured FP32 blocks (mixed)
  uint32_t* S16 = nullptr;   // structured 16-bit blocks (mixed)
  float* zpart = nullptr;    // structured matvec partial rows
  double* zpart64 = nullptr; // FP64 residual partial rows
  double* x64 = nullptr;     // FP64 solution (mixed)
  float* b = nullptr;
  float* x = nullptr;
  float* ffpart = nullptr;   // force-term partials
  float* F = nullptr;        // force terms sum_j T^{ij}[k][P0] F/2
  float* svpart = nullptr;   // structured velocity partials
  int* vflag = nullptr;      // set when a velocity is not finite
  int* host_vflag = nullptr; // its page-locked host copy (a pageable target would make the read synchronous)
  cudaEvent_t wait_ev = nullptr;   // blocking-sync event of the step's host waits (rf_set_host_wait); null polls
  // Krylov scratch
  float* V = nullptr;
  float* ypart = nullptr;
  double* part = nullptr;
  double* H = nullptr;
  double* cs = nullptr;
  double* sn = nullptr;
  double* g = nullptr;
  GmresCtl* ctl = nullptr;
  GmresCtl* host_ctl = nullptr;
  LuSetup lu{};                   // direct solver workspace
  float* bicg_work = nullptr;     // BiCGSTAB vectors r, r0, p, v, s, t
  BicgCtl* bctl = nullptr;
  BicgCtl* host_bctl = nullptr;
  double* ir_norm = nullptr;      // BiCGSTAB refinement (mixed): ||r||^2 on the device
  double* host_ir_norm = nullptr; //   and its pinned host copy
  DenseGemvPlan gemv_plan;
  int coop_blocks = 1;
  // velocity scratch
  float4* fw = nullptr;
  float* vpart = nullptr;
  cudaEvent_t ev[8];
  cudaEvent_t order_ev = nullptr;   // orders this handle's stream before a packed solve
  PackLanes pack_lanes;             // streams of a packed solve this handle leads
  int pack_status = RF_OK;          // this handle's result in the last packed solve
  rf_stats stats;
  // optional per-launch timing of the solve's matvec kernels
  bool profile = false;
  std::vector<cudaEvent_t> mv_events;
  int mv_used = 0;
  int launches = 0;
  int matvecs_done = 0;
  int refinements = 0;
  int restart = 10;          // Krylov dimension per cycle
  int64_t steps_taken = 0;   // completed rf_update_fibers calls (checkpoint metadata)
  GmresGraphCache gmres_graphs;   // captured restart cycles (GMRES)
  // The whole time step as one CUDA graph (GMRES): assembly, the first restart
  // cycle, later cycles in a conditional WHILE node the solve itself ends,
  // velocities and the fiber update; [0] second-order steps, [1] the first
  // step.  state: 0 unused, 2 run once directly (captured on the next use),
  // 1 ready, -1 not capturable here.
  struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    int state = 0;
    int pre_kernels = 0, cycle_kernels = 0, post_kernels = 0;
  } step_graph[2];
  bool use_graphs = true;         // GMRES restart cycles from graphs
  bool use_step_graphs = true;    // rf_step as one graph
  int mv_variant = 0;             // structured matvec kernel (rf_autotune)
  int asm_variant = 0;            // numerical pair-tile kernel (rf_autotune)
  int64_t ypart_floats = 0;       // capacity of ypart
  bool assembled = false, solved = false;
  int64_t device_bytes = 0;
  std::vector<void*> allocations;

  bool dry = false;          // count bytes only (rf_device_bytes_estimate)
  bool pooled = false;       // counted in the device pools' live handles
  // Stream-ordered allocations: creating or destroying a handle does not
  // synchronise the device, so handles of a serving loop come and go without
  // stalling the others.
  int alloc(void** p, size_t bytes) {
    if (dry) {
      *p = nullptr;
      device_bytes += (int64_t)bytes;
      return RF_OK;
    }
    // fault injection: the n-th allocation from now fails (tests)
    int left = g_fail_alloc_after.load();
    while (left >= 0 && !g_fail_alloc_after.compare_exchange_weak(left, left - 1)) {}
    if (left == 0) {
      *p = nullptr;
      set_last_error_str("device allocation failed (injected)");
      return RF_E_OOM;
    }
    cudaMemPool_t pool = nullptr;
    cudaError_t e = handle_pool(dev, &pool);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(p, bytes, pool, st);
    if (e != cudaSuccess) {
      *p = nullptr;
      set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
      return e == cudaErrorMemoryAllocation ? RF_E_OOM : RF_E_CUDA;
    }
    allocations.push_back(*p);
    device_bytes += (int64_t)bytes;
    return RF_OK;
  }
  void release_step_graphs() {
    for (auto& g : step_graph) {
      if (g.exec) cudaGraphExecDestroy(g.exec);
      g = StepGraph();
    }
  }
  ~rf_handle() {
    gmres_graphs.release();
    release_step_graphs();
    for (auto e : mv_events) cudaEventDestroy(e);
    for (void* p : allocations) cudaFreeAsync(p, st);
    if (st) cudaStreamSynchronize(st);
    PinnedPool& pp = pinned_pool();
    pp.put(host_ctl, sizeof(GmresCtl));
    pp.put(host_bctl, sizeof(BicgCtl));
    pp.put(host_ir_norm, sizeof(double));
    pp.put(host_vflag, sizeof(int));
    pp.put(lu.host_ipiv, (size_t)lu.R * sizeof(int));
    pp.put(lu.host_perm, (size_t)lu.R * sizeof(int));
    if (pooled) pools_release();
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (order_ev) cudaEventDestroy(order_ev);
    for (auto& a : pack_lanes.aux)
      if (a) cudaStreamSynchronize(a);
    pack_lanes_release(pack_lanes);
    if (wait_ev) cudaEventDestroy(wait_ev);
    if (st) cudaStreamDestroy(st);
  }
};

#define RF_TRY(expr)        \
  do {                      \
    int _rc = (expr);       \
    if (_rc != RF_OK) return _rc; \
  } while (0)

static int validate_config(const rf_config* c, int N) {
  if (!c || N < 1) { set_last_error_str("rf_create: null config or N < 1"); return RF_E_INPUT; }
  const int M = c->number_of_terms_in_force_expansion;
  if (M < 1 || M > kMaxTerms) { set_last_error_str("M must be in [1, 8]"); return RF_E_INPUT; }
  if (c->number_of_quadrature_points_per_interval != 3) {
    set_last_error_str("only 3 Gauss points per interval are defined (fortran/fibers.f95:370-376)");
    return RF_E_INPUT;
  }
  const int Q = 3 * c->number_of_quadrature_intervals;
  if (Q < 2 || Q > kMaxQuad) { set_last_error_str("quadrature intervals out of range"); return RF_E_INPUT; }
  if (!mq_supported(M, Q)) { set_last_error_str("(M, intervals) combination not built"); return RF_E_UNSUPPORTED; }
  if (!(c->slenderness > 0.0) || !(c->timestep > 0.0)) { set_last_error_str("slenderness / timestep"); return RF_E_INPUT; }
  if (c->solver < 0 || c->solver > 2 || c->integration < 0 || c->integration > 1) {
    set_last_error_str("solver / integration"); return RF_E_INPUT;
  }
  if (c->precision < RF_PREC_FP32 || c->precision > RF_PREC_MIXED_BF16_RECOMPUTE) {
    set_last_error_str("precision");
    return RF_E_INPUT;
  }
  const bool is_mixed = c->precision != RF_PREC_FP32 && c->precision != RF_PREC_MATRIX_FREE;
  if (c->precision != RF_PREC_FP32 && c->integration != RF_NUMERICAL) {
    set_last_error_str("mixed precision and the matrix-free mode use the symmetric pair blocks of numerical integration");
    return RF_E_UNSUPPORTED;
  }
  if (is_mixed && c->number_of_quadrature_intervals != 8) {
    set_last_error_str("mixed precision is built for 8 quadrature intervals (24 points per fiber)");
    return RF_E_UNSUPPORTED;
  }
  if (c->precision != RF_PREC_FP32 && c->solver == RF_SOLVER_DIRECT) {
    set_last_error_str("the direct solver factors the dense FP32 matrix (RF_PREC_FP32 only)");
    return RF_E_UNSUPPORTED;
  }
  if (c->precision != RF_PREC_FP32 && !(c->refinement_tolerance > 0.0)) {
    set_last_error_str("refinement_tolerance must be positive"); return RF_E_INPUT;
  }
  if (c->velocity_integration < -1 || c->velocity_integration > 1) {
    set_last_error_str("velocity_integration must be -1, 0 or 1"); return RF_E_INPUT;
  }
  if (c->solver == RF_SOLVER_BICGSTAB && (c->bicgstab_max_iterations < 1 || !(c->bicgstab_tolerance > 0.0))) {
    set_last_error_str("bicgstab_max_iterations / bicgstab_tolerance"); return RF_E_INPUT;
  }
  if (c->gmres_restart < 1 || c->gmres_restart > kMaxRestart) { set_last_error_str("gmres restart in [1, 64]"); return RF_E_INPUT; }
  if (c->refinement_restart < 0 || c->refinement_restart > kMaxRestart) {
    set_last_error_str("refinement_restart in [0, 64]"); return RF_E_INPUT;
  }
  return RF_OK;
}

extern "C" {

int rf_config_default(rf_config* c) {
  if (!c) return RF_E_INPUT;
  std::memset(c, 0, sizeof(*c));
  c->number_of_timesteps = 10;
  c->state_save_interval = 1;
  c->velocity_save_interval = 1;
  c->timestep = 0.1;
  c->slenderness = 0.01;
  c->number_of_terms_in_force_expansion = 5;
  c->number_of_quadrature_intervals = 8;
  c->number_of_quadrature_points_per_interval = 3;
  c->gmres_restart = 10;
  c->gmres_max_iterations = 1000;
  c->gmres_tolerance = 1e-5;
  c->bicgstab_max_iterations = 1000;
  c->bicgstab_tolerance = 1e-5;
  c->solver = RF_SOLVER_GMRES;
  c->integration = RF_NUMERICAL;
  c->precision = RF_PREC_FP32;
  c->velocity_integration = -1;
  c->refinement_tolerance = 1e-6;
  c->refinement_max_iterations = 20;
  // N=4000, FP16 blocks: 24.3 ms per step with 10 Arnoldi steps between
  // corrections (3.2 corrections, 26.8 iterations), 21.2 ms with 20, 21.3 with 30
  c->refinement_restart = 20;
  return RF_OK;
}

const char* rf_status_string(int s) {
  switch (s) {
    case RF_OK: return "ok";
    case RF_E_INPUT: return "invalid input";
    case RF_E_CUDA: return "CUDA error";
    case RF_E_OOM: return "out of device memory";
    case RF_E_NOCONV: return "solver did not converge";
    case RF_E_NAN: return "non-finite values";
    case RF_E_TIMEOUT: return "device wait timed out";
    case RF_E_UNSUPPORTED: return "unsupported configuration";
    case RF_E_STATE: return "call out of order";
    case RF_E_SINGULAR: return "singular matrix";
  }
  return "unknown status";
}

const char* rf_last_error(void) { return g_last_error.c_str(); }

static void to_double4(const double* src, int N, std::vector<double>& out) {
  out.assign((size_t)N * 4, 0.0);
  for (int i = 0; i < N; ++i)
    for (int a = 0; a < 3; ++a) out[(size_t)i * 4 + a] = src[(size_t)i * 3 + a];
}

int rf_set_state(rf_handle* h, const double* pos, const double* ori) {
  if (!h || !pos || !ori) return RF_E_INPUT;
  std::vector<double> p4, o4;
  to_double4(pos, h->N, p4);
  to_double4(ori, h->N, o4);
  std::vector<float> p32((size_t)h->N * 4), o32((size_t)h->N * 4);
  for (size_t k = 0; k < p4.size(); ++k) { p32[k] = (float)p4[k]; o32[k] = (float)o4[k]; }
  const size_t b64 = (size_t)h->N * sizeof(double4), b32 = (size_t)h->N * sizeof(float4);
  for (int s = 0; s < 2; ++s) {   // previous == current at the first step
    const int idx = s == 0 ? h->icur : h->iprev;
    RF_CUDA_TRY(cudaMemcpyAsync(h->pos64[idx], p4.data(), b64, cudaMemcpyHostToDevice, h->st));
    RF_CUDA_TRY(cudaMemcpyAsync(h->ori64[idx], o4.data(), b64, cudaMemcpyHostToDevice, h->st));
  }
  RF_CUDA_TRY(cudaMemcpyAsync(h->pos32, p32.data(), b32, cudaMemcpyHostToDevice, h->st));
  RF_CUDA_TRY(cudaMemcpyAsync(h->ori32, o32.data(), b32, cudaMemcpyHostToDevice, h->st));
  RF_CUDA_TRY(cudaStreamSynchronize(h->st));
  h->assembled = h->solved = false;
  h->vel_fresh = false;
  return RF_OK;
}

// Every device buffer of a handle.  With h->dry set nothing is allocated and
// h->device_bytes is the exact footprint (admission control of the server).
constexpr int kTuneMaxCtasPerSm = 16;
// Mixed-precision BiCGSTAB: each inner solve on the 16-bit blocks stops when
// its residual has fallen to this fraction of the correction equation's
// right-hand side (the 16-bit operator is accurate to about 1e-4, so going
// further buys little before the next FP64 residual)
constexpr double kBicgInnerTolerance = 1e-3;

static int allocate_buffers(rf_handle* h, const rf_config* cfg) {
  const int64_t R = h->R;
  const int N = h->N;
  const size_t b64 = (size_t)N * sizeof(double4), b32 = (size_t)N * sizeof(float4);
  int rc = RF_OK;
  for (int s = 0; s < 3 && !rc; ++s) {
    rc = h->alloc((void**)&h->pos64[s], b64);
    if (!rc) rc = h->alloc((void**)&h->ori64[s], b64);
  }
  if (!rc) rc = h->alloc((void**)&h->pos32, b32);
  if (!rc) rc = h->alloc((void**)&h->ori32, b32);
  for (int s = 0; s < 2 && !rc; ++s) {
    rc = h->alloc((void**)&h->tv[s], b32);
    if (!rc) rc = h->alloc((void**)&h->rv[s], b32);
  }
  h->recompute = cfg->precision == RF_PREC_MIXED_FP16_RECOMPUTE || cfg->precision == RF_PREC_MIXED_BF16_RECOMPUTE;
  h->mixed = cfg->precision == RF_PREC_MIXED_FP16 || cfg->precision == RF_PREC_MIXED_BF16 || h->recompute;
  h->mfree = cfg->precision == RF_PREC_MATRIX_FREE;
  const int64_t T16 = ceil_div(N, kStoreTile);
  if (h->mfree) {
    // partial rows of a product: one slot per assembly tile, one for the
    // diagonal tiles' j side, one for the sum
    h->zparts = assemble_tiles(h->M, h->Q, N) + 1;
    if (!rc) rc = h->alloc((void**)&h->zpart, (size_t)(h->zparts + 1) * (size_t)R * sizeof(float));
  } else if (!h->mixed) {
    if (!rc) rc = h->alloc((void**)&h->A, (size_t)h->lda * (size_t)R * sizeof(float));
  } else {
    if (!h->recompute && !rc) rc = h->alloc((void**)&h->S32, (size_t)struct_floats32(h->M, N) * sizeof(float));
    if (!rc) rc = h->alloc((void**)&h->S16, (size_t)struct_words16(h->M, N) * sizeof(uint32_t));
    // one extra row slot holds the summed partials; the recompute modes' residual
    // product (launch_assemble_apply) needs one slot per assembly tile and one more
    int64_t slots = T16 + 1;
    if (h->recompute) {
      h->zparts = assemble_tiles(h->M, h->Q, N) + 1;
      slots = std::max<int64_t>(slots, h->zparts + 1);
    }
    if (!rc) rc = h->alloc((void**)&h->zpart, (size_t)slots * (size_t)R * sizeof(float));
    if (!h->recompute && !rc) rc = h->alloc((void**)&h->zpart64, (size_t)(T16 + 1) * (size_t)R * sizeof(double));
    if (!rc) rc = h->alloc((void**)&h->x64, (size_t)R * sizeof(double));
    if (h->recompute) {
      if (!rc) rc = h->alloc((void**)&h->xcast, (size_t)R * sizeof(float));
    } else if (!rc) {
      rc = h->alloc((void**)&h->svpart, (size_t)T16 * N * 6 * sizeof(float));
    }
  }
  if (!rc) rc = h->alloc((void**)&h->b, (size_t)R * sizeof(float));
  if (!rc) rc = h->alloc((void**)&h->x, (size_t)R * sizeof(float));
  const int tiles = assemble_tiles(h->M, h->Q, N);
  const size_t ffn = (size_t)N * 3 * (h->M + 1);
  if (!rc) rc = h->alloc((void**)&h->ffpart, (size_t)tiles * ffn * sizeof(float));
  if (!rc) rc = h->alloc((void**)&h->F, ffn * sizeof(float));
  // Krylov
  const int m = (h->mixed && cfg->refinement_restart > 0) ? cfg->refinement_restart : cfg->gmres_restart;
  h->restart = m;
  h->gemv_plan = plan_dense_gemv(R, h->num_sms);
  if (h->mixed || h->mfree) h->gemv_plan.splits = 1;  // these products write complete rows
  h->coop_blocks = krylov_coop_blocks(R, h->num_sms);
  const int64_t ldv = ceil_div(R, 32) * 32;
  if (!rc) rc = h->alloc((void**)&h->V, (size_t)(m + 1) * (size_t)ldv * sizeof(float));
  // room for the most column splits rf_autotune tries
  h->ypart_floats = (int64_t)(h->mixed || h->mfree ? 1 : plan_dense_gemv(R, h->num_sms, kTuneMaxCtasPerSm).splits) * R;
  h->ypart_floats = std::max<int64_t>(h->ypart_floats, (int64_t)h->gemv_plan.splits * R);
  if (!rc) rc = h->alloc((void**)&h->ypart, (size_t)h->ypart_floats * sizeof(float));
  if (!rc) rc = h->alloc((void**)&h->part, (size_t)3 * h->coop_blocks * (kMaxRestart + 2) * sizeof(double));
  if (!rc) rc = h->alloc((void**)&h->H, (size_t)(m + 1) * m * sizeof(double));
  if (!rc) rc = h->alloc((void**)&h->cs, (size_t)m * sizeof(double));
  if (!rc) rc = h->alloc((void**)&h->sn, (size_t)m * sizeof(double));
  if (!rc) rc = h->alloc((void**)&h->g, (size_t)(m + 1) * sizeof(double));
  if (!rc) rc = h->alloc((void**)&h->ctl, sizeof(GmresCtl));
  if (!rc && !h->dry && !(h->host_ctl = static_cast<GmresCtl*>(pinned_pool().get(sizeof(GmresCtl))))) rc = RF_E_OOM;
  if (cfg->solver == RF_SOLVER_DIRECT) {
    LuSetup& L = h->lu;
    L.R = R;
    L.lda = h->lda;
    L.tol = cfg->refinement_tolerance;
    L.max_refine = cfg->refinement_max_iterations;
    L.coop_blocks = std::max(h->coop_blocks, coop_blocks_per_sm_capped(h->num_sms));
    if (!rc) rc = h->alloc((void**)&L.LU, (size_t)h->lda * (size_t)R * sizeof(float));
    if (!rc) rc = h->alloc((void**)&L.ipiv, (size_t)R * sizeof(int));
    if (!rc) rc = h->alloc((void**)&L.perm, (size_t)R * sizeof(int));
    if (!rc) rc = h->alloc((void**)&L.pmax, (size_t)2 * L.coop_blocks * sizeof(float));
    if (!rc) rc = h->alloc((void**)&L.pidx, (size_t)2 * L.coop_blocks * sizeof(int));
    if (!rc) rc = h->alloc((void**)&L.prow, (size_t)2 * L.coop_blocks * 64 * sizeof(float));
    if (!rc) rc = h->alloc((void**)&L.jrow, (size_t)2 * 64 * sizeof(float));
    if (!rc) rc = h->alloc((void**)&L.info, sizeof(int));
    if (!rc) rc = h->alloc((void**)&L.d, (size_t)R * sizeof(float));
    if (!rc) rc = h->alloc((void**)&L.x64, (size_t)R * sizeof(double));
    if (!rc) rc = h->alloc((void**)&L.r64, (size_t)R * sizeof(double));
    if (!rc) rc = h->alloc((void**)&L.rpart, (size_t)kLuResidualSplits * R * sizeof(double));
    if (!rc) rc = h->alloc((void**)&L.norms, 2 * sizeof(double));
    if (!rc) rc = h->alloc((void**)&L.LT, (size_t)lu_tc_lt_floats(R) * sizeof(float));
    if (!rc) rc = h->alloc((void**)&L.inv, (size_t)lu_tc_inv_floats() * sizeof(float));
    if (!rc) rc = h->alloc((void**)&L.flags, 2 * sizeof(int));
    if (!rc) rc = h->alloc((void**)&L.sinv, (size_t)lu_tc_sinv_floats(R) * sizeof(float));
    if (!rc && !h->dry && !(L.host_ipiv = static_cast<int*>(pinned_pool().get((size_t)R * sizeof(int))))) rc = RF_E_OOM;
    if (!rc && !h->dry && !(L.host_perm = static_cast<int*>(pinned_pool().get((size_t)R * sizeof(int))))) rc = RF_E_OOM;
  }
  if (cfg->solver == RF_SOLVER_BICGSTAB) {
    if (!rc) rc = h->alloc((void**)&h->bicg_work, (size_t)6 * (size_t)ldv * sizeof(float));
    if (!rc) rc = h->alloc((void**)&h->bctl, sizeof(BicgCtl));
    if (!rc && !h->dry && !(h->host_bctl = static_cast<BicgCtl*>(pinned_pool().get(sizeof(BicgCtl))))) rc = RF_E_OOM;
    if (h->mixed) {
      if (!rc) rc = h->alloc((void**)&h->ir_norm, sizeof(double));
      if (!rc && !h->dry && !(h->host_ir_norm = static_cast<double*>(pinned_pool().get(sizeof(double))))) rc = RF_E_OOM;
    }
  }
  // velocities
  if (!rc) rc = h->alloc((void**)&h->fw, (size_t)N * h->Q * sizeof(float4));
  if (!rc) rc = h->alloc((void**)&h->vpart, (size_t)velocity_chunks(N) * N * 6 * sizeof(float));
  if (!rc) rc = h->alloc((void**)&h->vflag, sizeof(int));
  if (!rc && !h->dry && !(h->host_vflag = static_cast<int*>(pinned_pool().get(sizeof(int))))) rc = RF_E_OOM;
  return rc;
}

static void init_dims(rf_handle* h, const rf_config* cfg, int N) {
  h->cfg = *cfg;
  h->N = N;
  h->M = cfg->number_of_terms_in_force_expansion;
  h->Q = 3 * cfg->number_of_quadrature_intervals;
  h->R = (int64_t)3 * h->M * N;
  h->lda = ceil_div(h->R, 32) * 32;
  h->tab = make_tables(*cfg);
  std::memset(&h->stats, 0, sizeof(h->stats));
  for (auto& e : h->ev) e = nullptr;
}

int64_t rf_device_bytes_estimate(const rf_config* cfg, int N) {
  if (validate_config(cfg, N) != RF_OK) return -1;
  rf_handle h;
  init_dims(&h, cfg, N);
  h.dry = true;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&h.num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    h.num_sms = 148;
  cudaGetLastError();
  if (allocate_buffers(&h, cfg) != RF_OK) return -1;
  return h.device_bytes;
}

int rf_create(const rf_config* cfg, int N, const double* pos, const double* ori, rf_handle** out) {
  if (!out) return RF_E_INPUT;
  *out = nullptr;
  RF_TRY(validate_config(cfg, N));
  if (!pos || !ori) { set_last_error_str("rf_create: null fiber arrays"); return RF_E_INPUT; }
  rf_handle* h = new rf_handle();
  init_dims(h, cfg, N);
  auto fail = [&](int rc) { delete h; return rc; };
  cudaError_t e = cudaGetDevice(&h->dev);
  if (e != cudaSuccess) { set_last_error(cudaGetErrorString(e), __FILE__, __LINE__); return fail(RF_E_CUDA); }
  cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->dev);
  if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) return fail(RF_E_CUDA);
  pools_acquire();
  h->pooled = true;
  for (auto& ev : h->ev)
    if (cudaEventCreate(&ev) != cudaSuccess) return fail(RF_E_CUDA);
  int rc = allocate_buffers(h, cfg);
  if (rc) return fail(rc);
  if (h->mixed) {
    // records that the assembly never writes (fibers >= N, the lower sub-tile
    // of a diagonal storage tile) hold zeros rather than whatever the pool had
    if ((h->S32 &&
         cudaMemsetAsync(h->S32, 0, (size_t)struct_floats32(h->M, N) * sizeof(float), h->st) != cudaSuccess) ||
        cudaMemsetAsync(h->S16, 0, (size_t)struct_words16(h->M, N) * sizeof(uint32_t), h->st) != cudaSuccess)
      return fail(RF_E_CUDA);
  }
  h->stats.device_bytes = h->device_bytes;
  rc = rf_set_state(h, pos, ori);
  if (rc) return fail(rc);
  *out = h;
  return RF_OK;
}

int rf_destroy(rf_handle* h) {
  if (!h) return RF_E_INPUT;
  cudaStreamSynchronize(h->st);
  delete h;
  return RF_OK;
}

static float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

static int enqueue_assemble(rf_handle* h) {
  if (h->mfree)   // the force terms and b (the products recompute the blocks)
    return launch_assemble_apply(h->tab, h->N, h->pos32, h->ori32, h->pos64[h->icur], nullptr, h->zpart, nullptr,
                                 h->ffpart, h->F, h->b, h->st, h->asm_variant);
  if (h->mixed) {
    RF_TRY(launch_assemble_structured(h->tab, h->N, h->pos32, h->ori32, h->pos64[h->icur], h->S32, h->S16,
                                      storage16(h->cfg) == 2, h->ffpart, h->F, h->b, h->st,
                                      h->asm_variant));
    // the preconditioner's blocks come from this step's FP32 records
    if (h->nf_k > 0)
      return launch_nf_setup(h->tab, h->N, h->nf_k, h->pos32, h->ori32, h->S32, h->nf_nb, h->nf_w, h->st);
    return RF_OK;
  }
  if (h->cfg.integration == RF_ANALYTICAL)
    return launch_assemble_analytical(h->tab, h->N, h->pos32, h->ori32, h->pos64[h->icur], h->ori64[h->icur], h->A,
                                      h->lda, h->ffpart, h->F, h->b, h->st);
  return launch_assemble_numerical(h->tab, h->N, h->pos32, h->ori32, h->pos64[h->icur], h->A, h->lda, h->ffpart,
                                   h->F, h->b, h->st, h->asm_variant);
}

int rf_assemble(rf_handle* h) {
  if (!h) return RF_E_INPUT;
  RF_CUDA_TRY(cudaEventRecord(h->ev[0], h->st));
  RF_TRY(enqueue_assemble(h));
  h->launches += 2;
  RF_CUDA_TRY(cudaEventRecord(h->ev[1], h->st));
  h->assembled = true;
  h->solved = false;
  return RF_OK;
}

static GmresSetup gmres_setup(rf_handle* h) {
  GmresSetup s;
  s.R = h->R;
  s.m = h->restart;
  s.maxit = h->cfg.gmres_max_iterations;
  s.tol = h->mixed ? h->cfg.refinement_tolerance : h->cfg.gmres_tolerance;
  s.V = h->V;
  s.ldv = ceil_div(h->R, 32) * 32;
  s.Z = h->nf_k > 0 ? h->nf_z : nullptr;
  s.ypart = h->ypart;
  s.nsplit = h->gemv_plan.splits;
  s.part = h->part;
  s.H = h->H;
  s.cs = h->cs;
  s.sn = h->sn;
  s.g = h->g;
  s.ctl = h->ctl;
  s.host_ctl = h->host_ctl;
  s.coop_blocks = h->coop_blocks;
  s.wait_ev = h->wait_ev;
  // per-matvec profiling events are recorded by the callbacks, so profiling runs
  // launch every cycle directly; otherwise the cycles replay captured graphs
  // (an injected device-wait limit is a kernel argument: no capture or replay then)
  s.graphs = (h->profile || !h->use_graphs || device_wait_limit() >= 0) ? nullptr : &h->gmres_graphs;
  return s;
}

// The Krylov matvec of the handle's operator (optionally timed by events),
// counting its kernel launches into *launches
static MatvecFn make_matvec(rf_handle* h, int* launches) {
  return [h, launches](const float* xin, const int* skip, cudaStream_t st) -> int {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (h->profile) {
      while ((int)h->mv_events.size() < h->mv_used + 2) {
        cudaEvent_t e;
        RF_CUDA_TRY(cudaEventCreate(&e));
        h->mv_events.push_back(e);
      }
      e0 = h->mv_events[h->mv_used];
      e1 = h->mv_events[h->mv_used + 1];
      h->mv_used += 2;
      RF_CUDA_TRY(cudaEventRecord(e0, st));
    }
    ++*launches;
    int rc;
    if (h->mixed) {
      const int smode = storage16(h->cfg);
      // flexible GMRES: the product of basis column j is A z_j with z_j = P v_j
      // kept for the solution update (other vectors get the plain product)
      const int64_t ldv = ceil_div(h->R, 32) * 32;
      const int64_t off = ((intptr_t)xin - (intptr_t)h->V) / (int64_t)sizeof(float);
      const float* xa = xin;
      if (h->nf_k > 0 && (intptr_t)xin >= (intptr_t)h->V && off % ldv == 0 && off / ldv <= h->restart) {
        float* zj = h->nf_z + off;
        rc = launch_nf_apply(h->N, h->nf_k, h->nf_nb, h->nf_w, xin, zj, skip, st);
        if (rc != RF_OK) return rc;
        xa = zj;
        ++*launches;
      }
      rc = launch_struct_matvec(h->tab, h->N, smode, h->S32, h->S16, h->ori32, xa, h->zpart, h->ypart, skip,
                                &h->ctl->timeout, st, h->recompute ? 0 : h->mv_variant);
      *launches += 2;
    } else if (h->mfree) {
      rc = launch_assemble_apply(h->tab, h->N, h->pos32, h->ori32, h->pos64[h->icur], xin, h->zpart, skip,
                                 h->ffpart, h->F, h->b, st, h->asm_variant);
      if (rc == RF_OK) rc = launch_parts_finalize(h->tab, h->N, h->ori32, xin, h->zpart, h->zparts, h->ypart, skip, st);
      *launches += 2;
    } else {
      rc = launch_dense_gemv(h->gemv_plan, h->A, h->lda, h->R, xin, h->ypart, skip, st);
    }
    if (h->profile) RF_CUDA_TRY(cudaEventRecord(e1, st));
    return rc;
  };
}

// FP64-accumulated residual r = b - A x over the FP32 pair blocks (mixed modes);
// the recompute modes form the blocks again (the matrix-free product of an FP32
// copy of x, its partial rows summed in FP64)
static ResidualFn make_residual(rf_handle* h) {
  if (h->recompute)
    return [h](const void* xin, float* r, const int* skip, cudaStream_t st) -> int {
      const double* x64 = static_cast<const double*>(xin);
      RF_TRY(launch_cast_to_float(x64, h->xcast, h->R, st));
      RF_TRY(launch_assemble_apply(h->tab, h->N, h->pos32, h->ori32, h->pos64[h->icur], h->xcast, h->zpart, skip,
                                   h->ffpart, h->F, h->b, st, h->asm_variant));
      return launch_parts_residual64(h->tab, h->N, h->ori32, x64, h->zpart, h->zparts, h->b, r, skip, st);
    };
  return [h](const void* xin, float* r, const int* skip, cudaStream_t st) -> int {
    return launch_struct_residual64(h->tab, h->N, h->S32, h->ori32, static_cast<const double*>(xin), h->zpart64,
                                    h->b, r, skip, &h->ctl->timeout, st);
  };
}

int rf_solve(rf_handle* h) {
  if (!h) return RF_E_INPUT;
  if (!h->assembled) { set_last_error_str("rf_solve before rf_assemble"); return RF_E_STATE; }
  RF_CUDA_TRY(cudaEventRecord(h->ev[2], h->st));
  h->stats.graph_replays = 0;
  GmresSetup s = gmres_setup(h);
  h->mv_used = 0;
  int mv_launches = 0;
  MatvecFn mv = make_matvec(h, &mv_launches);
  if (h->cfg.solver == RF_SOLVER_DIRECT) {
    LuResult lr;
    const int lrc = lu_factor_solve(h->lu, h->A, h->b, h->x, h->st, &lr);
    RF_CUDA_TRY(cudaEventRecord(h->ev[3], h->st));
    h->launches += lr.launches;
    h->matvecs_done = 0;
    h->stats.iterations = 0;
    h->stats.restarts = 0;
    h->stats.refinement_steps = lr.refinement_steps;
    h->stats.factorizations = lr.factorizations;
    h->stats.pivoted = lr.pivoted ? 1 : 0;
    h->stats.max_multiplier = lr.max_multiplier;
    h->stats.relative_residual = lr.relative_residual;
    if (lrc != RF_OK && lrc != RF_E_NOCONV) return lrc;
    h->solved = true;
    return lrc;
  }
  if (h->cfg.solver == RF_SOLVER_BICGSTAB) {
    BicgSetup bs;
    bs.R = h->R;
    bs.maxit = h->cfg.bicgstab_max_iterations;
    bs.restart_every = 200;   // ViennaCL's max_iterations_before_restart default (bicgstab.hpp:51)
    bs.tol = h->cfg.bicgstab_tolerance;
    bs.work = h->bicg_work;
    bs.ldv = ceil_div(h->R, 32) * 32;
    bs.ypart = h->ypart;
    bs.nsplit = h->gemv_plan.splits;
    bs.part = h->part;
    bs.ctl = h->bctl;
    bs.host_ctl = h->host_bctl;
    bs.coop_blocks = h->coop_blocks;
    BicgResult br;
    int brc;
    if (h->mixed) {
      // BiCGSTAB on the 16-bit blocks inside FP64-residual refinement: the
      // residual, its correction and the FP64 solution use the Krylov basis
      // buffers (the GMRES basis is idle under this solver)
      RF_CUDA_TRY(cudaMemsetAsync(&h->ctl->timeout, 0, sizeof(int), h->st));
      ResidualFn resid = make_residual(h);
      BicgIr ir;
      ir.x64 = h->x64;
      ir.r = h->V;
      ir.d = h->V + bs.ldv;
      ir.norm_dev = h->ir_norm;
      ir.norm_host = h->host_ir_norm;
      ir.tol = h->cfg.refinement_tolerance;
      ir.inner_tol = kBicgInnerTolerance;
      ir.max_outer = h->cfg.refinement_max_iterations;
      brc = bicgstab_ir_solve(bs, mv, resid, h->b, ir, h->st, &br);
      int timed_out = 0;
      RF_CUDA_TRY(cudaMemcpyAsync(&timed_out, &h->ctl->timeout, sizeof(int), cudaMemcpyDeviceToHost, h->st));
      RF_CUDA_TRY(cudaStreamSynchronize(h->st));
      if (timed_out) {
        set_last_error_str("a bounded device-side wait timed out");
        return RF_E_TIMEOUT;
      }
      if (brc == RF_OK || brc == RF_E_NOCONV) {
        RF_TRY(launch_cast_to_float(h->x64, h->x, h->R, h->st));
        h->launches += 1;
      }
      h->launches += 3 * (br.refinements + 1);   // the FP64 residual of every outer pass
      h->refinements = br.refinements;
    } else {
      brc = bicgstab_solve(bs, mv, h->b, h->x, h->st, &br);
    }
    RF_CUDA_TRY(cudaEventRecord(h->ev[3], h->st));
    h->launches += br.launches + mv_launches;
    h->matvecs_done = br.matvecs;
    h->stats.iterations = br.iterations;
    h->stats.restarts = br.restarts;
    h->stats.refinement_steps = h->mixed ? br.refinements : 0;
    h->stats.relative_residual = br.relative_residual;
    if (brc != RF_OK && brc != RF_E_NOCONV) return brc;
    h->solved = true;
    return brc;
  }
  GmresResult res;
  int rc;
  if (h->mixed) {
    ResidualFn resid = make_residual(h);
    h->refinements = 0;
    rc = gmres_solve_ex(s, mv, resid, h->b, h->x64, true, h->st, &res);
    h->refinements = res.residual_calls;
    if (rc == RF_OK || rc == RF_E_NOCONV) {
      int rc2 = launch_cast_to_float(h->x64, h->x, h->R, h->st);
      if (rc2) return rc2;
      h->launches += 1;
    }
    h->launches += 2 * h->refinements;
  } else {
    rc = gmres_solve(s, mv, h->b, h->x, h->st, &res);
  }
  RF_CUDA_TRY(cudaEventRecord(h->ev[3], h->st));
  h->launches += res.launches + mv_launches;
  h->matvecs_done = res.matvecs;
  h->stats.iterations = res.iterations;
  h->stats.restarts = res.restarts;
  h->stats.refinement_steps = h->mixed ? h->refinements : 0;
  h->stats.relative_residual = res.relative_residual;
  h->stats.graph_replays = res.graph_replays;
  if (rc != RF_OK && rc != RF_E_NOCONV) return rc;
  h->solved = true;
  return rc;
}

// the velocity kernels and the non-finite guard (read by rf_step after its
// sync); returns the number of kernels in *kernels
static int enqueue_velocities(rf_handle* h, int* kernels) {
  const int vint = h->cfg.velocity_integration < 0 ? h->cfg.integration : h->cfg.velocity_integration;
  if (vint == RF_ANALYTICAL) {
    RF_TRY(launch_velocity_analytical(h->tab, h->N, h->ori32, h->pos64[h->icur], h->ori64[h->icur], h->x,
                                      h->vpart, h->tv[h->vcur], h->rv[h->vcur], h->st));
    *kernels += 2;
  } else if (h->mixed && !h->recompute) {
    RF_TRY(launch_struct_velocity(h->tab, h->N, h->S32, h->ori32, h->F, h->x, h->svpart, h->tv[h->vcur],
                                  h->rv[h->vcur], h->st));
    *kernels += 2;
  } else {
    RF_TRY(launch_velocity_numerical(h->tab, h->N, h->pos64[h->icur], h->ori32, h->x, h->fw, h->vpart, h->tv[h->vcur],
                                     h->rv[h->vcur], h->st));
    *kernels += 3;
  }
  RF_TRY(launch_check_finite(h->tv[h->vcur], h->rv[h->vcur], h->N, h->vflag, h->st));
  *kernels += 1;
  return RF_OK;
}

int rf_update_velocities(rf_handle* h) {
  if (!h) return RF_E_INPUT;
  if (!h->solved) { set_last_error_str("rf_update_velocities before rf_solve"); return RF_E_STATE; }
  RF_CUDA_TRY(cudaEventRecord(h->ev[4], h->st));
  RF_TRY(enqueue_velocities(h, &h->launches));
  RF_CUDA_TRY(cudaEventRecord(h->ev[5], h->st));
  h->vlast = h->vcur;
  h->vel_fresh = true;
  return RF_OK;
}

// halt: a device word that, when set, makes the update leave the state as it
// is (the whole-step graph passes the solve's failure word; null otherwise)
static int enqueue_update_fibers(rf_handle* h, int first_step, const int* halt = nullptr) {
  // the state rotates in place inside the kernel (src/simulation.cu:307-311;
  // fortran/fibers.f95:325-341 swap buffers instead)
  return launch_update_fibers(h->N, first_step, h->cfg.timestep, h->pos64[h->iprev], h->pos64[h->icur],
                              h->ori64[h->iprev], h->ori64[h->icur], h->tv[h->vprev], h->tv[h->vcur],
                              h->rv[h->vprev], h->rv[h->vcur], h->pos32, h->ori32, halt, h->st);
}

static bool step_graph_eligible(const rf_handle* h) {
  return h->use_graphs && h->use_step_graphs && !h->profile && device_wait_limit() < 0 &&
         h->cfg.solver == RF_SOLVER_GMRES;
}

// Capture one stream segment into a graph (nothing runs during the capture).
static int capture_segment(cudaStream_t st, const std::function<int()>& fn, cudaGraph_t* out) {
  *out = nullptr;
  if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return RF_E_CUDA;
  }
  int rc = fn();
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(st, &g);
  if (rc == RF_OK && (e != cudaSuccess || !g)) rc = RF_E_CUDA;
  if (rc != RF_OK) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return rc;
  }
  *out = g;
  return RF_OK;
}

// The step graph: [assembly, first GMRES cycle, loop condition] ->
// WHILE(condition) { later cycle, loop condition } -> [solution cast,
// velocities, fiber update].  The WHILE node runs the restart cycles on the
// device, so a step is one graph launch and one read of the control block.
static int build_step_graph(rf_handle* h, int first_step, rf_handle::StepGraph* sg) {
  cudaGraph_t G = nullptr, pre = nullptr, body = nullptr, post = nullptr;
  auto fail = [&](int rc) {
    for (cudaGraph_t g : {pre, body, post, G})
      if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    sg->state = -1;
    return rc;
  };
  if (cudaGraphCreate(&G, 0) != cudaSuccess) return fail(RF_E_CUDA);
  cudaGraphConditionalHandle cond;
  if (cudaGraphConditionalHandleCreate(&cond, G, 1, cudaGraphCondAssignDefault) != cudaSuccess)
    return fail(RF_E_CUDA);
  GmresSetup s = gmres_setup(h);
  s.graphs = nullptr;
  int mvk = 0;
  MatvecFn mv = make_matvec(h, &mvk);
  ResidualFn resid = h->mixed ? make_residual(h) : ResidualFn();
  void* xsol = h->mixed ? static_cast<void*>(h->x64) : static_cast<void*>(h->x);
  int kpre = 2, kcycle = 0, kpost = 1;
  int rc = capture_segment(h->st, [&]() -> int {
    RF_TRY(enqueue_assemble(h));
    return gmres_enqueue_first(s, mv, resid, h->b, xsol, h->mixed, cond, h->st, &kpre);
  }, &pre);
  if (rc) return fail(rc);
  kpre += mvk;
  mvk = 0;
  rc = capture_segment(h->st, [&]() -> int {
    return gmres_enqueue_cycle(s, mv, resid, h->b, xsol, h->mixed, cond, h->st, &kcycle);
  }, &body);
  if (rc) return fail(rc);
  kcycle += mvk + (h->mixed ? 3 : 0);   // the FP64 residual's kernels
  rc = capture_segment(h->st, [&]() -> int {
    if (h->mixed) {
      RF_TRY(launch_cast_to_float(h->x64, h->x, h->R, h->st));
      ++kpost;
    }
    RF_TRY(enqueue_velocities(h, &kpost));
    return enqueue_update_fibers(h, first_step, &h->ctl->halt);
  }, &post);
  if (rc) return fail(rc);
  cudaGraphNode_t npre, ncond, nbody, npost;
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  if (cudaGraphAddChildGraphNode(&npre, G, nullptr, 0, pre) != cudaSuccess ||
      cudaGraphAddNode(&ncond, G, &npre, 1, &cp) != cudaSuccess ||
      cudaGraphAddChildGraphNode(&nbody, cp.conditional.phGraph_out[0], nullptr, 0, body) != cudaSuccess ||
      cudaGraphAddChildGraphNode(&npost, G, &ncond, 1, post) != cudaSuccess ||
      cudaGraphInstantiate(&sg->exec, G, 0) != cudaSuccess) {
    sg->exec = nullptr;
    return fail(RF_E_CUDA);
  }
  for (cudaGraph_t g : {pre, body, post, G}) cudaGraphDestroy(g);
  sg->pre_kernels = kpre;
  sg->cycle_kernels = kcycle;
  sg->post_kernels = kpost;
  sg->state = 1;
  return RF_OK;
}

int rf_prepare_step_graphs(rf_handle* h, int which) {
  if (!h || which < 0 || which > 3) return RF_E_INPUT;
  if (!step_graph_eligible(h)) return RF_OK;
  for (int first = 0; first < 2; ++first) {
    if (!(which & (first ? 1 : 2))) continue;
    rf_handle::StepGraph& g = h->step_graph[first];
    if (g.state == 1 || g.state == -1) continue;
    build_step_graph(h, first, &g);   // state 1, or -1: direct launches
  }
  return RF_OK;
}

int rf_update_fibers(rf_handle* h, int first_step) {
  if (!h) return RF_E_INPUT;
  if (!h->vel_fresh) { set_last_error_str("rf_update_fibers before rf_update_velocities"); return RF_E_STATE; }
  RF_CUDA_TRY(cudaEventRecord(h->ev[6], h->st));
  RF_TRY(enqueue_update_fibers(h, first_step));
  h->launches += 1;
  RF_CUDA_TRY(cudaEventRecord(h->ev[7], h->st));
  h->vel_fresh = false;
  h->assembled = h->solved = false;
  h->steps_taken += 1;
  return RF_OK;
}

// One step as a graph launch (see build_step_graph); the control block and the
// velocity guard are read once afterwards.
static int run_step_graph(rf_handle* h, const rf_handle::StepGraph& g) {
  RF_CUDA_TRY(cudaEventRecord(h->ev[0], h->st));
  RF_CUDA_TRY(cudaGraphLaunch(g.exec, h->st));
  RF_CUDA_TRY(cudaEventRecord(h->ev[7], h->st));
  RF_CUDA_TRY(cudaMemcpyAsync(h->host_ctl, h->ctl, sizeof(GmresCtl), cudaMemcpyDeviceToHost, h->st));
  RF_CUDA_TRY(cudaMemcpyAsync(h->host_vflag, h->vflag, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  RF_CUDA_TRY(host_wait(h->st, h->wait_ev));
  const int vbad = *h->host_vflag;
  const GmresCtl c = *h->host_ctl;
  GmresResult res;
  const int rc = gmres_result_from_ctl(c, h->mixed, &res);
  h->launches = g.pre_kernels + c.heads * g.cycle_kernels + g.post_kernels;
  h->matvecs_done = res.matvecs;
  h->mv_used = 0;
  h->refinements = h->mixed ? res.residual_calls : 0;
  h->stats.iterations = res.iterations;
  h->stats.restarts = res.restarts;
  h->stats.refinement_steps = h->refinements;
  h->stats.relative_residual = res.relative_residual;
  h->stats.graph_replays = 1;
  h->stats.ms_assemble_system = h->stats.ms_solve_system = 0.0;
  h->stats.ms_update_velocities = h->stats.ms_update_fibers = 0.0;
  h->stats.ms_step = elapsed(h->ev[0], h->ev[7]);
  h->stats.kernel_launches = h->launches;
  if (rc == RF_E_NAN || rc == RF_E_TIMEOUT) {
    // the update left the state as it was; the velocities are not valid
    h->assembled = h->solved = false;
    h->vel_fresh = false;
    return rc;
  }
  h->vlast = h->vcur;
  h->vel_fresh = false;
  h->assembled = h->solved = false;
  h->steps_taken += 1;
  if (vbad) {
    set_last_error_str("non-finite velocity");
    return RF_E_NAN;
  }
  return rc;
}

int rf_step(rf_handle* h, int t) {
  if (!h) return RF_E_INPUT;
  h->launches = 0;
  if (step_graph_eligible(h)) {
    rf_handle::StepGraph& g = h->step_graph[t == 0 ? 1 : 0];
    if (g.state == 2) build_step_graph(h, t == 0, &g);   // -1 when not capturable: direct launches
    if (g.state == 1) return run_step_graph(h, g);
    if (g.state == 0) g.state = 2;                         // the next step of this kind is captured
  }
  // NVTX ranges with the reference's step names (src/performance.cc)
  struct Range {
    explicit Range(const char* n) { nvtxRangePushA(n); }
    ~Range() { nvtxRangePop(); }
  };
  Range step_range("rf_step");
  int rc;
  {
    Range r("assemble_system");
    RF_TRY(rf_assemble(h));
  }
  {
    Range r("solve_system");
    rc = rf_solve(h);
  }
  if (rc != RF_OK && rc != RF_E_NOCONV) return rc;
  {
    Range r("update_velocities");
    RF_TRY(rf_update_velocities(h));
  }
  {
    Range r("update_fibers");
    RF_TRY(rf_update_fibers(h, t == 0));
  }
  RF_CUDA_TRY(cudaMemcpyAsync(h->host_vflag, h->vflag, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  RF_CUDA_TRY(host_wait(h->st, h->wait_ev));
  const int vbad = *h->host_vflag;
  if (vbad) {
    set_last_error_str("non-finite velocity");
    return RF_E_NAN;
  }
  h->stats.ms_assemble_system = elapsed(h->ev[0], h->ev[1]);
  h->stats.ms_solve_system = elapsed(h->ev[2], h->ev[3]);
  h->stats.ms_update_velocities = elapsed(h->ev[4], h->ev[5]);
  h->stats.ms_update_fibers = elapsed(h->ev[6], h->ev[7]);
  h->stats.ms_step = elapsed(h->ev[0], h->ev[7]);
  h->stats.kernel_launches = h->launches;
  return rc;
}

// ---- packed solves and steps of many small suspensions --------------------
// The conditions of the packed solve (k_pack_gmres_ir): mixed precision,
// GMRES, M = 5, Q = 24, at most kPackMaxFibers fibers (more than
// kPackSingleMaxFibers only where the device runs clusters), one restart length.
static int pack_check(rf_handle** hs, int n, bool need_assembled, const char* who, int* m_out, int* Rmax_out) {
  int m = -1, Rmax = 0;
  for (int i = 0; i < n; ++i) {
    rf_handle* h = hs[i];
    if (!h) return RF_E_INPUT;
    if (need_assembled && !h->assembled) {
      set_last_error_str((std::string(who) + " before rf_assemble").c_str());
      return RF_E_STATE;
    }
    if (!h->mixed || h->recompute || h->cfg.solver != RF_SOLVER_GMRES || h->M != 5 || h->tab.Q != 24 ||
        h->N > kPackMaxFibers ||
        (h->N > kPackSingleMaxFibers && pack_max_cluster() < 2)) {
      set_last_error_str(
          (std::string(who) + ": mixed precision, GMRES, 5 force terms, 8x3 quadrature, at most 256 fibers").c_str());
      return RF_E_UNSUPPORTED;
    }
    if (m >= 0 && h->restart != m) {
      set_last_error_str((std::string(who) + ": one restart length per pack").c_str());
      return RF_E_INPUT;
    }
    m = h->restart;
    Rmax = std::max<int>(Rmax, (int)h->R);
  }
  *m_out = m;
  *Rmax_out = Rmax;
  return RF_OK;
}

// every member's earlier work on its own stream before the pack's launches on st
static int pack_order_streams(rf_handle** hs, int n, cudaStream_t st) {
  for (int i = 0; i < n; ++i) {
    rf_handle* h = hs[i];
    if (h->st == st) continue;
    if (!h->order_ev) RF_CUDA_TRY(cudaEventCreateWithFlags(&h->order_ev, cudaEventDisableTiming));
    RF_CUDA_TRY(cudaEventRecord(h->order_ev, h->st));
    RF_CUDA_TRY(cudaStreamWaitEvent(st, h->order_ev, 0));
  }
  return RF_OK;
}

// The packed solve's cluster sizes (pack_plan_ctas) and the members' order in
// its descriptor array: clusters of 8 first, then 4, 2 and 1 (counts, and the
// largest system of each class in rmax); pos[i] is member i's place.
static void pack_solve_order(rf_handle** hs, int n, std::vector<int>& pos, int (&counts)[4], int (&rmax)[4]) {
  std::vector<int> fibers((size_t)n), ctas((size_t)n);
  for (int i = 0; i < n; ++i) fibers[(size_t)i] = (int)hs[i]->N;
  pack_plan_ctas(fibers.data(), n, hs[0]->num_sms, ctas.data(), pack_max_cluster());
  pos.assign((size_t)n, 0);
  int k = 0;
  for (int c = 0; c < 4; ++c) {
    counts[c] = 0;
    rmax[c] = 0;
    for (int i = 0; i < n; ++i)
      if (ctas[(size_t)i] == (8 >> c)) {
        pos[(size_t)i] = k++;
        ++counts[c];
        rmax[c] = std::max(rmax[c], (int)hs[i]->R);
      }
  }
}

// the packed solve's descriptor of h (out: 4 ints, relres: 1 double, on the device)
static void pack_member(rf_handle* h, int* out, double* relres, PackMember* q) {
  std::memset(q, 0, sizeof(*q));
  q->N = h->N;
  q->smode = storage16(h->cfg);
  q->maxit = h->cfg.gmres_max_iterations;
  q->tol = h->cfg.refinement_tolerance;
  q->S16 = h->S16;
  q->S32 = h->S32;
  q->ori = h->ori32;
  q->b = h->b;
  q->x64 = h->x64;
  q->x = h->x;
  q->V = h->V;
  q->ldv = ceil_div(h->R, 32) * 32;
  q->out = out;
  q->relres = relres;
  for (int k = 0; k < 5; ++k) {
    q->coef[k] = h->tab.gamma[k];
    q->eig[k] = h->tab.eigen[k];
  }
}

// a member's solve outcome (o: its 4 output ints) into its handle
static int pack_record_solve(rf_handle* h, const int* o, double relres) {
  h->matvecs_done = o[0];
  h->mv_used = 0;   // no per-launch matvec windows: the matvecs ran inside the packed kernel
  h->refinements = o[2];
  h->stats.iterations = o[0];
  h->stats.restarts = o[1];
  h->stats.refinement_steps = o[2];
  h->stats.relative_residual = relres;
  h->stats.graph_replays = 0;
  h->pack_status = o[3] == 0 ? RF_OK : (o[3] == 1 ? RF_E_NOCONV : RF_E_NAN);
  if (h->pack_status != RF_E_NAN) h->solved = true;
  return h->pack_status;
}

// One launch per cluster size solves every handle's assembled system
// (k_pack_gmres_ir: one thread-block cluster per suspension, the rf_solve
// algorithm for the mixed modes); each handle's result depends only on its
// own data.
int rf_solve_packed(rf_handle** hs, int n) {
  if (!hs || n < 1) return RF_E_INPUT;
  int m = 0, Rmax = 0;
  RF_TRY(pack_check(hs, n, true, "rf_solve_packed", &m, &Rmax));
  rf_handle* h0 = hs[0];
  cudaStream_t st = h0->st;
  RF_TRY(pack_order_streams(hs, n, st));
  const size_t bm = (size_t)n * sizeof(PackMember), bo = (size_t)n * 4 * sizeof(int), br = (size_t)n * sizeof(double);
  unsigned char* dbuf = nullptr;
  cudaMemPool_t pool = nullptr;
  RF_CUDA_TRY(handle_pool(h0->dev, &pool));
  RF_CUDA_TRY(cudaMallocFromPoolAsync((void**)&dbuf, bm + bo + br, pool, st));
  PackMember* dm = reinterpret_cast<PackMember*>(dbuf);
  double* drel = reinterpret_cast<double*>(dbuf + bm);
  int* dout = reinterpret_cast<int*>(dbuf + bm + br);
  std::vector<PackMember> pm((size_t)n);
  std::vector<int> pos;
  int counts[4], rmax[4];
  pack_solve_order(hs, n, pos, counts, rmax);
  for (int i = 0; i < n; ++i) {
    pack_member(hs[i], dout + 4 * i, drel + i, &pm[(size_t)pos[(size_t)i]]);
    RF_CUDA_TRY(cudaEventRecord(hs[i]->ev[2], st));
  }
  RF_CUDA_TRY(cudaMemcpyAsync(dm, pm.data(), bm, cudaMemcpyHostToDevice, st));
  int rc = launch_pack_gmres_ir(dm, counts, rmax, m, st, h0->pack_lanes);
  std::vector<int> out((size_t)n * 4, 0);
  std::vector<double> rel((size_t)n, 0.0);
  if (rc == RF_OK) {
    RF_CUDA_TRY(cudaMemcpyAsync(out.data(), dout, bo, cudaMemcpyDeviceToHost, st));
    RF_CUDA_TRY(cudaMemcpyAsync(rel.data(), drel, br, cudaMemcpyDeviceToHost, st));
  }
  for (int i = 0; i < n; ++i) RF_CUDA_TRY(cudaEventRecord(hs[i]->ev[3], st));
  RF_CUDA_TRY(cudaFreeAsync(dbuf, st));
  // the members' next work is enqueued after this returns, so after the solve
  RF_CUDA_TRY(cudaStreamSynchronize(st));
  if (rc != RF_OK) return rc;
  int worst = RF_OK;
  for (int i = 0; i < n; ++i) {
    rf_handle* h = hs[i];
    h->launches += (i == 0) ? 1 : 0;
    const int s = pack_record_solve(h, &out[(size_t)i * 4], rel[(size_t)i]);
    if (s == RF_E_NAN) worst = RF_E_NAN;
    else if (s == RF_E_NOCONV && worst == RF_OK) worst = RF_E_NOCONV;
  }
  return worst;
}

// A whole time step of every member as one launch sequence on the first
// member's stream: per group of members with the same Tables and storage,
// the packed assembly (k_pack_assemble, k_pack_force_terms); the packed solve
// of all members; per group the packed velocities and update (k_pack_velocity,
// k_pack_finish).  One upload of the descriptors, one download of the
// outcomes, one synchronisation.  A member whose solve ends non-finite keeps
// its state; one whose velocities are not finite has taken the step and
// reports RF_E_NAN (as rf_step's stages do).
int rf_step_packed(rf_handle** hs, const int* timesteps, int n, int* status) {
  if (!hs || !timesteps || !status || n < 1) return RF_E_INPUT;
  for (int i = 0; i < n; ++i) {
    if (!hs[i]) return RF_E_INPUT;
    status[i] = RF_OK;
  }
  int m = 0, Rmax = 0;
  const int chk = pack_check(hs, n, false, "rf_step_packed", &m, &Rmax);
  if (chk != RF_OK) {
    for (int i = 0; i < n; ++i) status[i] = chk;
    return chk;
  }
  nvtxRangePushA("rf_step_packed");
  struct Pop {
    ~Pop() { nvtxRangePop(); }
  } pop;
  rf_handle* h0 = hs[0];
  cudaStream_t st = h0->st;
  RF_TRY(pack_order_streams(hs, n, st));

  // groups: members with the same Tables (slenderness) and 16-bit format
  std::vector<int> order;
  std::vector<int> gbeg;   // group g: order[gbeg[g] .. gbeg[g+1])
  {
    std::vector<bool> taken((size_t)n, false);
    for (int i = 0; i < n; ++i) {
      if (taken[(size_t)i]) continue;
      gbeg.push_back((int)order.size());
      for (int j = i; j < n; ++j) {
        if (taken[(size_t)j] || hs[j]->cfg.precision != hs[i]->cfg.precision ||
            std::memcmp(&hs[j]->tab, &hs[i]->tab, sizeof(Tables)) != 0)
          continue;
        taken[(size_t)j] = true;
        order.push_back(j);
      }
    }
    gbeg.push_back(n);
  }
  const int ngroups = (int)gbeg.size() - 1;

  // device block: [PackMember n][PackStepMember n][relres n][out 4n][vbad n]
  const size_t bm = (size_t)n * sizeof(PackMember), bs = (size_t)n * sizeof(PackStepMember);
  const size_t br = (size_t)n * sizeof(double), bo = (size_t)n * 5 * sizeof(int);
  unsigned char* dbuf = nullptr;
  cudaMemPool_t pool = nullptr;
  RF_CUDA_TRY(handle_pool(h0->dev, &pool));
  RF_CUDA_TRY(cudaMallocFromPoolAsync((void**)&dbuf, bm + bs + br + bo, pool, st));
  PackMember* dpm = reinterpret_cast<PackMember*>(dbuf);
  PackStepMember* dsm = reinterpret_cast<PackStepMember*>(dbuf + bm);
  double* drel = reinterpret_cast<double*>(dbuf + bm + bs);
  int* dout = reinterpret_cast<int*>(dbuf + bm + bs + br);
  int* dvbad = dout + 4 * n;
  std::vector<unsigned char> host(bm + bs);
  PackMember* pm = reinterpret_cast<PackMember*>(host.data());
  PackStepMember* sm = reinterpret_cast<PackStepMember*>(host.data() + bm);
  std::vector<int64_t> asm_blocks((size_t)ngroups, 0), vel_blocks((size_t)ngroups, 0);
  std::vector<int> pos;
  int counts[4], rmax[4];
  pack_solve_order(hs, n, pos, counts, rmax);
  for (int g = 0; g < ngroups; ++g) {
    for (int k = gbeg[g]; k < gbeg[g + 1]; ++k) {
      const int i = order[(size_t)k];
      rf_handle* h = hs[i];
      pack_member(h, dout + 4 * i, drel + i, &pm[pos[(size_t)i]]);
      PackStepMember& q = sm[k];
      std::memset(&q, 0, sizeof(q));
      q.N = h->N;
      q.first = timesteps[i] == 0 ? 1 : 0;
      q.asm_start = (int)asm_blocks[(size_t)g];
      q.vel_start = (int)vel_blocks[(size_t)g];
      const int64_t T = ceil_div(h->N, 8);
      asm_blocks[(size_t)g] += T * (T + 1) / 2;
      vel_blocks[(size_t)g] += struct_store_tiles(h->N);
      q.dt = h->cfg.timestep;
      q.solve_status = dout + 4 * i + 3;
      q.vbad = dvbad + i;
      q.pos64 = h->pos64[h->icur];
      q.pos64_prev = h->pos64[h->iprev];
      q.ori64 = h->ori64[h->icur];
      q.ori64_prev = h->ori64[h->iprev];
      q.pos32 = h->pos32;
      q.ori32 = h->ori32;
      q.tv = h->tv[h->vcur];
      q.tv_prev = h->tv[h->vprev];
      q.rv = h->rv[h->vcur];
      q.rv_prev = h->rv[h->vprev];
      q.S32 = h->S32;
      q.S16 = h->S16;
      q.ffpart = h->ffpart;
      q.F = h->F;
      q.b = h->b;
      q.x = h->x;
      q.vpart = h->svpart;
    }
  }
  cudaEvent_t* ev = h0->ev;
  int launches = 1;
  RF_CUDA_TRY(cudaEventRecord(ev[0], st));
  RF_CUDA_TRY(cudaMemcpyAsync(dbuf, host.data(), bm + bs, cudaMemcpyHostToDevice, st));
  int rc = RF_OK;
  for (int g = 0; g < ngroups && rc == RF_OK; ++g) {
    rf_handle* hg = hs[order[(size_t)gbeg[g]]];
    rc = launch_pack_assemble(hg->tab, dsm + gbeg[g], gbeg[g + 1] - gbeg[g], asm_blocks[(size_t)g],
                              storage16(hg->cfg) == 2, st);
    launches += 2;
  }
  RF_CUDA_TRY(cudaEventRecord(ev[1], st));
  if (rc == RF_OK) rc = launch_pack_gmres_ir(dpm, counts, rmax, m, st, h0->pack_lanes);
  RF_CUDA_TRY(cudaEventRecord(ev[3], st));
  for (int g = 0; g < ngroups && rc == RF_OK; ++g) {
    rf_handle* hg = hs[order[(size_t)gbeg[g]]];
    rc = launch_pack_velocity_update(hg->tab, dsm + gbeg[g], gbeg[g + 1] - gbeg[g], vel_blocks[(size_t)g], st);
    launches += 2;
  }
  RF_CUDA_TRY(cudaEventRecord(ev[5], st));
  std::vector<unsigned char> res(br + bo);
  if (rc == RF_OK) RF_CUDA_TRY(cudaMemcpyAsync(res.data(), drel, br + bo, cudaMemcpyDeviceToHost, st));
  RF_CUDA_TRY(cudaFreeAsync(dbuf, st));
  RF_CUDA_TRY(cudaStreamSynchronize(st));
  if (rc != RF_OK) {
    for (int i = 0; i < n; ++i) status[i] = rc;
    return rc;
  }
  const double* rel = reinterpret_cast<const double*>(res.data());
  const int* out = reinterpret_cast<const int*>(res.data() + br);
  const int* vbad = out + 4 * n;
  const float ms_asm = elapsed(ev[0], ev[1]), ms_solve = elapsed(ev[1], ev[3]), ms_vel = elapsed(ev[3], ev[5]);
  int worst = RF_OK;
  for (int i = 0; i < n; ++i) {
    rf_handle* h = hs[i];
    h->launches = i == 0 ? launches : 0;
    h->assembled = true;
    h->solved = false;
    int s = pack_record_solve(h, &out[(size_t)i * 4], rel[i]);
    if (s != RF_E_NAN) {
      // velocities computed, state rotated in place (as rf_update_velocities + rf_update_fibers)
      h->vlast = h->vcur;
      h->vel_fresh = false;
      h->assembled = h->solved = false;
      h->steps_taken += 1;
      if (vbad[i]) {
        set_last_error_str("non-finite velocity");
        s = RF_E_NAN;
      }
    }
    // stage times are the pack's: its assembly, its solve, and its velocities
    // with the update fused into their last kernel
    h->stats.ms_assemble_system = ms_asm;
    h->stats.ms_solve_system = ms_solve;
    h->stats.ms_update_velocities = ms_vel;
    h->stats.ms_update_fibers = 0.0;
    h->stats.ms_step = ms_asm + ms_solve + ms_vel;
    h->stats.kernel_launches = h->launches;
    status[i] = s;
    if (s != RF_OK && s != RF_E_NOCONV && worst == RF_OK) worst = s;
  }
  return worst;
}

int rf_run(rf_handle* h, int first_timestep, int nsteps) {
  for (int k = 0; k < nsteps; ++k) {
    int rc = rf_step(h, first_timestep + k);
    if (rc != RF_OK) return rc;
  }
  return RF_OK;
}

static int fetch3(rf_handle* h, const void* dev, bool is_double, double* out) {
  const int N = h->N;
  if (is_double) {
    std::vector<double> tmp((size_t)N * 4);
    RF_CUDA_TRY(cudaMemcpyAsync(tmp.data(), dev, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    RF_CUDA_TRY(cudaStreamSynchronize(h->st));
    for (int i = 0; i < N; ++i)
      for (int a = 0; a < 3; ++a) out[(size_t)i * 3 + a] = tmp[(size_t)i * 4 + a];
  } else {
    std::vector<float> tmp((size_t)N * 4);
    RF_CUDA_TRY(cudaMemcpyAsync(tmp.data(), dev, tmp.size() * sizeof(float), cudaMemcpyDeviceToHost, h->st));
    RF_CUDA_TRY(cudaStreamSynchronize(h->st));
    for (int i = 0; i < N; ++i)
      for (int a = 0; a < 3; ++a) out[(size_t)i * 3 + a] = tmp[(size_t)i * 4 + a];
  }
  return RF_OK;
}

int rf_get_state(rf_handle* h, double* pos, double* ori) {
  if (!h || !pos || !ori) return RF_E_INPUT;
  RF_TRY(fetch3(h, h->pos64[h->icur], true, pos));
  return fetch3(h, h->ori64[h->icur], true, ori);
}

int rf_get_velocities(rf_handle* h, double* tvel, double* rvel) {
  if (!h || !tvel || !rvel) return RF_E_INPUT;
  if (h->vlast < 0) { set_last_error_str("no velocities computed yet"); return RF_E_STATE; }
  RF_TRY(fetch3(h, h->tv[h->vlast], false, tvel));
  return fetch3(h, h->rv[h->vlast], false, rvel);
}

static int fetch_vec(rf_handle* h, const float* dev, double* out) {
  std::vector<float> tmp((size_t)h->R);
  RF_CUDA_TRY(cudaMemcpyAsync(tmp.data(), dev, tmp.size() * sizeof(float), cudaMemcpyDeviceToHost, h->st));
  RF_CUDA_TRY(cudaStreamSynchronize(h->st));
  for (int64_t r = 0; r < h->R; ++r) out[r] = tmp[r];
  return RF_OK;
}

int rf_get_system(rf_handle* h, float* A, double* b) {
  if (!h) return RF_E_INPUT;
  if (!h->assembled) { set_last_error_str("no assembled system"); return RF_E_STATE; }
  if (A && !h->A) { set_last_error_str("no dense matrix in the mixed-precision and matrix-free modes"); return RF_E_STATE; }
  if (A) {
    RF_CUDA_TRY(cudaMemcpy2DAsync(A, (size_t)h->R * sizeof(float), h->A, (size_t)h->lda * sizeof(float),
                                  (size_t)h->R * sizeof(float), (size_t)h->R, cudaMemcpyDeviceToHost, h->st));
  }
  if (b) RF_TRY(fetch_vec(h, h->b, b));
  RF_CUDA_TRY(cudaStreamSynchronize(h->st));
  return RF_OK;
}

int rf_get_solution(rf_handle* h, double* x) {
  if (!h || !x) return RF_E_INPUT;
  if (!h->solved && h->vlast < 0) { set_last_error_str("no solution yet"); return RF_E_STATE; }
  return fetch_vec(h, h->x, x);
}

int rf_last_stats(rf_handle* h, rf_stats* s) {
  if (!h || !s) return RF_E_INPUT;
  *s = h->stats;
  s->device_bytes = h->device_bytes;
  s->kernel_launches = h->launches;   // since the last rf_step began (or the handle was created)
  return RF_OK;
}

int rf_get_config(rf_handle* h, rf_config* c) {
  if (!h || !c) return RF_E_INPUT;
  *c = h->cfg;
  return RF_OK;
}

int rf_number_of_fibers(rf_handle* h) { return h ? h->N : -1; }

int rf_operator_apply(rf_handle* h, const double* x, double* y, int which) {
  if (!h || !x || !y || which < 0 || which > 1) return RF_E_INPUT;
  if (!h->assembled) { set_last_error_str("rf_operator_apply before rf_assemble"); return RF_E_STATE; }
  if (which == 1 && !h->mixed) { set_last_error_str("no 16-bit operator outside the mixed-precision modes"); return RF_E_STATE; }
  const int64_t R = h->R;
  std::vector<double> hx(x, x + R);
  std::vector<float> hxf(R), hy(R);
  for (int64_t r = 0; r < R; ++r) hxf[r] = (float)hx[r];
  // the Krylov basis and solution buffers serve as staging (the handle is idle)
  float* dxf = h->V;
  float* dy = h->V + ceil_div(R, 32) * 32;
  RF_CUDA_TRY(cudaMemcpyAsync(dxf, hxf.data(), R * sizeof(float), cudaMemcpyHostToDevice, h->st));
  if (h->mfree || (h->recompute && which == 0)) {
    RF_TRY(launch_assemble_apply(h->tab, h->N, h->pos32, h->ori32, h->pos64[h->icur], dxf, h->zpart, nullptr,
                                 h->ffpart, h->F, h->b, h->st, h->asm_variant));
    RF_TRY(launch_parts_finalize(h->tab, h->N, h->ori32, dxf, h->zpart, h->zparts, dy, nullptr, h->st));
  } else if (!h->mixed) {
    RF_TRY(launch_dense_gemv(h->gemv_plan, h->A, h->lda, R, dxf, h->ypart, nullptr, h->st));
    RF_TRY(launch_reduce_rows(h->ypart, h->gemv_plan.splits, R, dy, h->st));
  } else if (which == 1) {
    const int smode = storage16(h->cfg);
    RF_CUDA_TRY(cudaMemsetAsync(&h->ctl->timeout, 0, sizeof(int), h->st));
    RF_TRY(launch_struct_matvec(h->tab, h->N, smode, h->S32, h->S16, h->ori32, dxf, h->zpart, dy, nullptr,
                                &h->ctl->timeout, h->st));
  } else {
    RF_CUDA_TRY(cudaMemcpyAsync(h->x64, hx.data(), R * sizeof(double), cudaMemcpyHostToDevice, h->st));
    RF_CUDA_TRY(cudaMemsetAsync(&h->ctl->timeout, 0, sizeof(int), h->st));
    RF_TRY(launch_struct_apply64(h->tab, h->N, h->S32, h->ori32, h->x64, h->zpart64, dy, &h->ctl->timeout, h->st));
  }
  if (h->mixed) {
    int timed_out = 0;
    RF_CUDA_TRY(cudaMemcpyAsync(&timed_out, &h->ctl->timeout, sizeof(int), cudaMemcpyDeviceToHost, h->st));
    RF_CUDA_TRY(cudaStreamSynchronize(h->st));
    if (timed_out) { set_last_error_str("a bounded device-side wait timed out"); return RF_E_TIMEOUT; }
  }
  RF_CUDA_TRY(cudaMemcpyAsync(hy.data(), dy, R * sizeof(float), cudaMemcpyDeviceToHost, h->st));
  RF_CUDA_TRY(cudaStreamSynchronize(h->st));
  for (int64_t r = 0; r < R; ++r) y[r] = hy[r];
  h->solved = false;
  return RF_OK;
}

// ---- checkpoint / resume --------------------------------------------------
// Everything the next step reads besides the configuration: the FP64 current
// and previous fiber states (second-order update), their FP32 copies, both
// velocity buffers (U^{n-1}, Omega^{n-1}), the buffer rotation and the step
// count.  Host-endian binary; the configuration is stored field by field and
// must match on load, so a resumed run repeats the uninterrupted one bit for bit.
namespace {
struct CkptHeader {
  char magic[8];
  uint32_t version, header_bytes;
  int32_t N, M, Q, solver, integration, precision, velocity_integration;
  int32_t gmres_restart, gmres_max_iterations, bicgstab_max_iterations, refinement_max_iterations,
      refinement_restart;
  double timestep, slenderness, gmres_tolerance, bicgstab_tolerance, refinement_tolerance;
  int64_t steps_taken;
  int32_t iprev, icur, vprev, vcur, vlast, pad;
};
const char kCkptMagic[8] = {'R', 'F', 'C', 'K', 'P', 'T', '0', '1'};

CkptHeader ckpt_header(const rf_handle* h) {
  CkptHeader c;
  std::memset(&c, 0, sizeof(c));
  std::memcpy(c.magic, kCkptMagic, 8);
  c.version = 1;
  c.header_bytes = sizeof(CkptHeader);
  const rf_config& f = h->cfg;
  c.N = h->N; c.M = h->M; c.Q = h->Q;
  c.solver = f.solver; c.integration = f.integration; c.precision = f.precision;
  c.velocity_integration = f.velocity_integration;
  c.gmres_restart = f.gmres_restart; c.gmres_max_iterations = f.gmres_max_iterations;
  c.bicgstab_max_iterations = f.bicgstab_max_iterations;
  c.refinement_max_iterations = f.refinement_max_iterations; c.refinement_restart = f.refinement_restart;
  c.timestep = f.timestep; c.slenderness = f.slenderness; c.gmres_tolerance = f.gmres_tolerance;
  c.bicgstab_tolerance = f.bicgstab_tolerance; c.refinement_tolerance = f.refinement_tolerance;
  c.steps_taken = h->steps_taken;
  c.iprev = h->iprev; c.icur = h->icur; c.vprev = h->vprev; c.vcur = h->vcur; c.vlast = h->vlast;
  return c;
}
}  // namespace

int64_t rf_checkpoint_bytes(rf_handle* h) {
  if (!h) return -1;
  const int64_t n = h->N;
  return (int64_t)sizeof(CkptHeader) + 2 * 2 * n * (int64_t)sizeof(double4) + 2 * n * (int64_t)sizeof(float4) +
         2 * 2 * n * (int64_t)sizeof(float4);
}

// device buffers in checkpoint order: pos64/ori64 of (prev, cur), pos32, ori32, tv[0..1], rv[0..1]
static void ckpt_layout(rf_handle* h, std::vector<std::pair<void*, size_t>>& parts) {
  const size_t b64 = (size_t)h->N * sizeof(double4), b32 = (size_t)h->N * sizeof(float4);
  parts = {{h->pos64[h->iprev], b64}, {h->ori64[h->iprev], b64}, {h->pos64[h->icur], b64},
           {h->ori64[h->icur], b64},  {h->pos32, b32},           {h->ori32, b32},
           {h->tv[0], b32},           {h->tv[1], b32},           {h->rv[0], b32},
           {h->rv[1], b32}};
}

int rf_checkpoint_save(rf_handle* h, void* buf, int64_t bytes) {
  if (!h || !buf || bytes < rf_checkpoint_bytes(h)) {
    set_last_error_str("rf_checkpoint_save: buffer smaller than rf_checkpoint_bytes");
    return RF_E_INPUT;
  }
  const CkptHeader c = ckpt_header(h);
  unsigned char* out = static_cast<unsigned char*>(buf);
  std::memcpy(out, &c, sizeof(c));
  size_t off = sizeof(c);
  std::vector<std::pair<void*, size_t>> parts;
  ckpt_layout(h, parts);
  for (auto& pt : parts) {
    RF_CUDA_TRY(cudaMemcpyAsync(out + off, pt.first, pt.second, cudaMemcpyDeviceToHost, h->st));
    off += pt.second;
  }
  RF_CUDA_TRY(cudaStreamSynchronize(h->st));
  return RF_OK;
}

int rf_checkpoint_load(rf_handle* h, const void* buf, int64_t bytes, int64_t* steps_taken) {
  if (!h || !buf || bytes < (int64_t)sizeof(CkptHeader)) return RF_E_INPUT;
  CkptHeader c;
  std::memcpy(&c, buf, sizeof(c));
  if (std::memcmp(c.magic, kCkptMagic, 8) != 0 || c.version != 1 || c.header_bytes != sizeof(CkptHeader)) {
    set_last_error_str("rf_checkpoint_load: not a checkpoint of this library version");
    return RF_E_INPUT;
  }
  if (bytes < rf_checkpoint_bytes(h)) { set_last_error_str("rf_checkpoint_load: truncated checkpoint"); return RF_E_INPUT; }
  CkptHeader mine = ckpt_header(h);
  // the state fields come from the checkpoint; everything else must match
  mine.steps_taken = c.steps_taken;
  mine.iprev = c.iprev; mine.icur = c.icur; mine.vprev = c.vprev; mine.vcur = c.vcur; mine.vlast = c.vlast;
  if (std::memcmp(&mine, &c, sizeof(c)) != 0) {
    set_last_error_str("rf_checkpoint_load: checkpoint of another configuration or fiber count");
    return RF_E_INPUT;
  }
  const bool idx_ok = c.iprev >= 0 && c.iprev < 3 && c.icur >= 0 && c.icur < 3 && c.iprev != c.icur &&
                      (c.vprev == 0 || c.vprev == 1) && c.vcur == 1 - c.vprev && c.vlast >= -1 && c.vlast < 2;
  if (!idx_ok) { set_last_error_str("rf_checkpoint_load: corrupt buffer indices"); return RF_E_INPUT; }
  // the step graphs hold the buffer roles they were captured with
  if (h->iprev != c.iprev || h->icur != c.icur || h->vprev != c.vprev || h->vcur != c.vcur)
    h->release_step_graphs();
  h->iprev = c.iprev;
  h->icur = c.icur;
  h->inext = 3 - c.iprev - c.icur;
  h->vprev = c.vprev;
  h->vcur = c.vcur;
  h->vel_fresh = false;
  h->vlast = c.vlast;
  h->steps_taken = c.steps_taken;
  const unsigned char* in = static_cast<const unsigned char*>(buf);
  size_t off = sizeof(c);
  std::vector<std::pair<void*, size_t>> parts;
  ckpt_layout(h, parts);
  for (auto& pt : parts) {
    RF_CUDA_TRY(cudaMemcpyAsync(pt.first, in + off, pt.second, cudaMemcpyHostToDevice, h->st));
    off += pt.second;
  }
  RF_CUDA_TRY(cudaStreamSynchronize(h->st));
  h->assembled = h->solved = false;
  if (steps_taken) *steps_taken = c.steps_taken;
  return RF_OK;
}

// ---- autotuning ----------------------------------------------------------
// The matvec of the Krylov solve has launch choices that do not change the
// method: the 16-bit structured kernel (TMA-staged or register-staged) and the
// number of column splits of the dense FP32 kernel.  rf_autotune times each
// candidate with CUDA events on this handle's assembled operator and keeps the
// fastest; the choice is cached per (device, precision, M, N).
namespace {
struct TuneKey {
  int dev, prec, M, Q, N;
  bool operator<(const TuneKey& o) const {
    return std::tie(dev, prec, M, Q, N) < std::tie(o.dev, o.prec, o.M, o.Q, o.N);
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, rf_tune_report> g_tune_cache;
}  // namespace

static void apply_tuning(rf_handle* h, const rf_tune_report& t) {
  if (h->cfg.solver == RF_SOLVER_DIRECT && t.panel_blocks > 0) h->lu.panel_blocks = t.panel_blocks;
  h->asm_variant = t.asm_variant;
  if (h->mixed) {
    h->mv_variant = t.matvec_variant;
  } else if (!h->mfree) {
    h->gemv_plan = plan_dense_gemv(h->R, h->num_sms, t.gemv_ctas_per_sm);
  }
  h->gmres_graphs.release();   // the captured cycles hold the old launch parameters
  h->release_step_graphs();
}

int rf_autotune(rf_handle* h, rf_tune_report* out) {
  if (!h) return RF_E_INPUT;
  if (!h->assembled) { set_last_error_str("rf_autotune needs an assembled system (rf_assemble)"); return RF_E_STATE; }
  const TuneKey key{h->dev, h->cfg.precision * 4 + h->cfg.solver, h->M, h->tab.Q, h->N};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      apply_tuning(h, it->second);
      if (out) { *out = it->second; out->cached = 1; }
      return RF_OK;
    }
  }
  rf_tune_report t;
  std::memset(&t, 0, sizeof(t));
  const int64_t R = h->R;
  const float* xin = h->b;                            // any vector of the right size
  float* y = h->V + ceil_div(R, 32) * 32;             // Krylov basis as scratch (the handle is idle)
  cudaEvent_t e0 = h->ev[2], e1 = h->ev[3];
  auto time_it = [&](auto&& launch, double* ms) -> int {
    for (int r = 0; r < 2; ++r) RF_TRY(launch());
    RF_CUDA_TRY(cudaEventRecord(e0, h->st));
    const int reps = 8;
    for (int r = 0; r < reps; ++r) RF_TRY(launch());
    RF_CUDA_TRY(cudaEventRecord(e1, h->st));
    RF_CUDA_TRY(cudaEventSynchronize(e1));
    float f = 0.f;
    RF_CUDA_TRY(cudaEventElapsedTime(&f, e0, e1));
    *ms = f / reps;
    return RF_OK;
  };
  if (h->mixed) {
    const int smode = storage16(h->cfg);
    RF_CUDA_TRY(cudaMemsetAsync(&h->ctl->timeout, 0, sizeof(int), h->st));
    double best = 1e30;
    for (int v = 0; v < (h->recompute ? 1 : 2); ++v) {   // the register-staged kernel reads the FP32 copy too
      const int variant = v == 0 ? 0 : 2;
      double ms = 0;
      RF_TRY(time_it([&]() {
        return launch_struct_matvec(h->tab, h->N, smode, h->S32, h->S16, h->ori32, xin, h->zpart, y, nullptr,
                                    &h->ctl->timeout, h->st, variant);
      }, &ms));
      t.matvec_ms[v] = ms;
      if (ms < best) { best = ms; t.matvec_variant = variant; }
    }
    int timeout = 0;
    RF_CUDA_TRY(cudaMemcpyAsync(&timeout, &h->ctl->timeout, sizeof(int), cudaMemcpyDeviceToHost, h->st));
    RF_CUDA_TRY(cudaStreamSynchronize(h->st));
    if (timeout) { set_last_error_str("rf_autotune: a bounded device-side wait timed out"); return RF_E_TIMEOUT; }
    t.gemv_ctas_per_sm = 0;
  } else if (h->mfree) {
    t.gemv_ctas_per_sm = 0;
    t.matvec_variant = 0;
  } else {
    const int cand[4] = {2, 4, 8, 16};
    double best = 1e30;
    for (int c = 0; c < 4; ++c) {
      const DenseGemvPlan p = plan_dense_gemv(R, h->num_sms, cand[c]);
      if ((int64_t)p.splits * R > h->ypart_floats) { t.gemv_ms[c] = -1; continue; }
      double ms = 0;
      RF_TRY(time_it([&]() { return launch_dense_gemv(p, h->A, h->lda, R, xin, h->ypart, nullptr, h->st); }, &ms));
      t.gemv_ms[c] = ms;
      if (ms < best) { best = ms; t.gemv_ctas_per_sm = cand[c]; }
    }
    t.matvec_variant = 0;
  }
  // the numerical assembly's pair-tile kernel (the variants' results are bit
  // for bit the same; re-assembling rewrites the same operator)
  t.asm_variant = 0;
  for (int v = 0; v < kAsmVariants; ++v) t.asm_ms[v] = -1;
  if (h->cfg.integration == RF_NUMERICAL) {
    double best = 1e30;
    const int keep = h->asm_variant;
    for (int v = 0; v < kAsmVariants; ++v) {
      h->asm_variant = v;
      double ms = 0;
      const int rc = time_it([&]() { return enqueue_assemble(h); }, &ms);
      if (rc != RF_OK) { h->asm_variant = keep; return rc; }
      t.asm_ms[v] = ms;
      if (ms < best) { best = ms; t.asm_variant = v; }
    }
    h->asm_variant = keep;
  }
  if (h->cfg.solver == RF_SOLVER_DIRECT) {
    // LU panel: fewer blocks make each grid sync cheaper but give each block
    // more rows (they must fit in shared memory); time the first panel
    const int cand[3] = {h->num_sms, std::max(1, h->num_sms / 2), std::max(1, h->num_sms / 4)};
    double best = 1e30;
    for (int c = 0; c < 3; ++c) {
      float ms = 0.f;
      const int rc = lu_time_panel(h->lu, h->A, cand[c], h->st, e0, e1, &ms);
      if (rc == RF_E_UNSUPPORTED) { t.panel_ms[c] = -1; continue; }
      RF_TRY(rc);
      t.panel_ms[c] = ms;
      if (ms < best) { best = ms; t.panel_blocks = cand[c]; }
    }
  }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = t;
  }
  apply_tuning(h, t);
  if (out) *out = t;
  return RF_OK;
}

int rf_debug_set_device_wait_limit(int64_t limit) {
  if (limit < -1) return RF_E_INPUT;
  g_wait_limit.store(limit);
  return RF_OK;
}

int rf_debug_fail_allocation_after(int n) {
  if (n < -1) return RF_E_INPUT;
  g_fail_alloc_after.store(n);
  return RF_OK;
}

int rf_set_near_field_preconditioner(rf_handle* h, int neighbours) {
  if (!h || neighbours < 0 || neighbours > kNfMaxNeighbours) return RF_E_INPUT;
  if (neighbours > 0 && (!h->mixed || h->recompute || h->M != 5 || h->cfg.solver != RF_SOLVER_GMRES)) {
    set_last_error_str("the near-field preconditioner needs a stored mixed mode, GMRES and 5 force terms");
    return RF_E_UNSUPPORTED;
  }
  if (neighbours > 0) {
    const int64_t ldv = ceil_div(h->R, 32) * 32;
    int rc = RF_OK;
    if (!h->nf_nb) rc = h->alloc((void**)&h->nf_nb, (size_t)h->N * (kNfMaxNeighbours + 1) * sizeof(int));
    if (!rc && !h->nf_w) rc = h->alloc((void**)&h->nf_w, (size_t)nf_w_floats(h->N) * sizeof(float));
    if (!rc && !h->nf_z) rc = h->alloc((void**)&h->nf_z, (size_t)(h->restart + 1) * ldv * sizeof(float));
    if (rc) return rc;
    h->stats.device_bytes = h->device_bytes;
  }
  if (neighbours != h->nf_k) {
    // captured cycles and steps hold the old launch parameters; the blocks of
    // the current system are formed at the next rf_assemble
    h->gmres_graphs.release();
    h->release_step_graphs();
    h->assembled = h->solved = false;
  }
  h->nf_k = neighbours;
  return RF_OK;
}

int rf_set_assembly_variant(rf_handle* h, int variant) {
  if (!h || variant < 0 || variant >= kAsmVariants) return RF_E_INPUT;
  if (h->asm_variant != variant) h->release_step_graphs();   // captured steps hold the old kernel
  h->asm_variant = variant;
  return RF_OK;
}

int rf_set_host_wait(rf_handle* h, int blocking) {
  if (!h || blocking < 0 || blocking > 1) return RF_E_INPUT;
  if (blocking && !h->wait_ev)
    RF_CUDA_TRY(cudaEventCreateWithFlags(&h->wait_ev, cudaEventBlockingSync | cudaEventDisableTiming));
  if (!blocking && h->wait_ev) {
    RF_CUDA_TRY(cudaStreamSynchronize(h->st));
    RF_CUDA_TRY(cudaEventDestroy(h->wait_ev));
    h->wait_ev = nullptr;
  }
  return RF_OK;
}

int rf_set_cuda_graphs(rf_handle* h, int mode) {
  if (!h || mode < 0 || mode > 2) return RF_E_INPUT;
  h->use_graphs = mode != 0;
  h->use_step_graphs = mode == 1;
  if (!h->use_step_graphs) h->release_step_graphs();
  return RF_OK;
}

int rf_get_stream(rf_handle* h, void** stream) {
  if (!h || !stream) return RF_E_INPUT;
  *stream = (void*)h->st;
  return RF_OK;
}

int rf_set_profiling(rf_handle* h, int enable) {
  if (!h) return RF_E_INPUT;
  h->profile = enable != 0;
  return RF_OK;
}

int rf_matvec_profile(rf_handle* h, int* launches, double* total_ms) {
  if (!h || !launches || !total_ms) return RF_E_INPUT;
  RF_CUDA_TRY(cudaStreamSynchronize(h->st));
  // launches issued after convergence return at once, so the matvecs that did
  // work are the matvecs_done longest launch windows
  std::vector<double> w;
  for (int k = 0; k + 1 < h->mv_used; k += 2) w.push_back(elapsed(h->mv_events[k], h->mv_events[k + 1]));
  const int n = std::min<int>(h->matvecs_done, (int)w.size());
  std::partial_sort(w.begin(), w.begin() + n, w.end(), std::greater<double>());
  double t = 0.0;
  for (int k = 0; k < n; ++k) t += w[k];
  *launches = n;
  *total_ms = t;
  return RF_OK;
}

int rf_dense_lu_solve(const float* A, const float* b, float* x, int64_t R, double tol, void* stream) {
  if (!A || !b || !x || R < 1 || !(tol > 0.0)) { set_last_error_str("rf_dense_lu_solve: bad arguments"); return RF_E_INPUT; }
  int dev = 0, sms = 148;
  RF_CUDA_TRY(cudaGetDevice(&dev));
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaStream_t st = (cudaStream_t)stream;
  LuSetup L{};
  L.R = R;
  L.lda = R;
  L.ldlu = ceil_div(R, 32) * 32;   // factors with 128-byte aligned columns (the tensor-core path's TMA needs
                                   // 16-byte multiples)
  L.tol = tol;
  L.max_refine = 20;
  L.coop_blocks = std::max(krylov_coop_blocks(R, sms), coop_blocks_per_sm_capped(sms));
  std::vector<void*> mem;
  auto get = [&](void** p, size_t bytes) -> int {
    // fault injection: the n-th allocation from now fails (tests)
    int left = g_fail_alloc_after.load();
    while (left >= 0 && !g_fail_alloc_after.compare_exchange_weak(left, left - 1)) {}
    if (left == 0) {
      *p = nullptr;
      set_last_error_str("device allocation failed (injected)");
      return RF_E_OOM;
    }
    cudaError_t e = cudaMallocAsync(p, bytes, st);
    if (e != cudaSuccess) { set_last_error(cudaGetErrorString(e), __FILE__, __LINE__); return RF_E_OOM; }
    mem.push_back(*p);
    return RF_OK;
  };
  int rc = get((void**)&L.LU, (size_t)L.ldlu * R * sizeof(float));
  if (!rc) rc = get((void**)&L.LT, (size_t)lu_tc_lt_floats(R) * sizeof(float));
  if (!rc) rc = get((void**)&L.inv, (size_t)lu_tc_inv_floats() * sizeof(float));
  if (!rc) rc = get((void**)&L.flags, 2 * sizeof(int));
  if (!rc) rc = get((void**)&L.sinv, (size_t)lu_tc_sinv_floats(R) * sizeof(float));
  if (!rc) rc = get((void**)&L.ipiv, R * sizeof(int));
  if (!rc) rc = get((void**)&L.perm, R * sizeof(int));
  if (!rc) rc = get((void**)&L.pmax, 2 * L.coop_blocks * sizeof(float));
  if (!rc) rc = get((void**)&L.pidx, 2 * L.coop_blocks * sizeof(int));
  if (!rc) rc = get((void**)&L.prow, 2 * L.coop_blocks * 64 * sizeof(float));
  if (!rc) rc = get((void**)&L.jrow, 2 * 64 * sizeof(float));
  if (!rc) rc = get((void**)&L.info, sizeof(int));
  if (!rc) rc = get((void**)&L.d, R * sizeof(float));
  if (!rc) rc = get((void**)&L.x64, R * sizeof(double));
  if (!rc) rc = get((void**)&L.r64, R * sizeof(double));
  if (!rc) rc = get((void**)&L.rpart, (size_t)kLuResidualSplits * R * sizeof(double));
  if (!rc) rc = get((void**)&L.norms, 2 * sizeof(double));
  std::vector<int> hi(R), hp(R);
  L.host_ipiv = hi.data();
  L.host_perm = hp.data();
  LuResult lr;
  if (!rc) rc = lu_factor_solve(L, A, b, x, st, &lr);
  for (void* p : mem) cudaFreeAsync(p, st);
  cudaStreamSynchronize(st);
  return rc;
}

int rf_dense_matvec(const float* A, const float* x, float* y, int64_t R, void* stream) {
  if (!A || !x || !y || R < 1) { set_last_error_str("rf_dense_matvec: bad arguments"); return RF_E_INPUT; }
  int dev = 0, sms = 148;
  RF_CUDA_TRY(cudaGetDevice(&dev));
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaStream_t st = (cudaStream_t)stream;
  DenseGemvPlan p = plan_dense_gemv(R, sms);
  float* ypart = nullptr;
  RF_CUDA_TRY(cudaMallocAsync((void**)&ypart, (size_t)p.splits * R * sizeof(float), st));
  int rc = launch_dense_gemv(p, A, R, R, x, ypart, nullptr, st);
  if (rc == RF_OK) rc = launch_reduce_rows(ypart, p.splits, R, y, st);
  cudaFreeAsync(ypart, st);
  return rc;
}

}  // extern "C"
