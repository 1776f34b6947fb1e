// rf_dense_matvec_noalloc: the dense matvec without any device allocation.
//
// rf_dense_matvec splits the columns of A over CTAs and needs a partial-row
// buffer (splits x R floats), which it allocates on the caller's stream.
// Some callers cannot let a library allocate: a host program that has handed
// the whole device memory to its own pool allocator up front (a framework's
// caching allocator, or a serving process that budgets every byte of HBM),
// where a cudaMalloc from inside the library fails or fragments the pool, or
// a latency-critical loop where cudaMalloc / cudaFree, which may synchronize
// the device, are not acceptable.  This variant takes its scratch from a
// fixed array in device memory that is part of the library image instead.
//
// The scratch array (kNoAllocScratchFloats floats, 8 MiB) is a file-scope
// __device__ variable: every GPU on which the library is loaded holds it
// until the process exits.  Its name is only a host-side stand-in; the device
// address is looked up with cudaGetSymbolAddress, with the device current, on
// the first call made in each CUDA context (for the usual primary context:
// once per device).  The lookup is cached per context by the context's
// unique id, so a context created after cudaDeviceReset gets a fresh lookup
// instead of the address from the destroyed one.
#include <map>
#include <mutex>

#include <cuda.h>

#include "rf_common.cuh"
#include "rf_kernels.cuh"
#include "rf_krylov.cuh"

namespace rf {

// 8 MiB: enough split-partial rows for any system with R <= kNoAllocMaxRows.
constexpr int64_t kNoAllocScratchFloats = 2 * 1024 * 1024;
constexpr int64_t kNoAllocMaxRows = 131072;

static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchFloats];

// The split plan of rf_dense_matvec, with the number of column splits capped
// so that splits x R partial rows fit in the scratch array.  Every column
// belongs to exactly one split: split s covers [s*cps, min(R, (s+1)*cps)).
static DenseGemvPlan noalloc_gemv_plan(int64_t R, int sms) {
  DenseGemvPlan p = plan_dense_gemv(R, sms);
  const int64_t max_splits = kNoAllocScratchFloats / R;
  if (p.splits > max_splits) {
    p.cps = ceil_div(R, max_splits);
    p.splits = (int)ceil_div(R, p.cps);
  }
  return p;
}

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

static std::mutex g_noalloc_mutex;
static std::map<unsigned long long, float*> g_noalloc_by_ctx;
static CtxGetCurrentFn g_ctx_current = nullptr;
static CtxGetIdFn g_ctx_id = nullptr;
static bool g_driver_fns_looked_up = false;

// Unique id of the calling thread's current context (0 when there is none).
static unsigned long long current_context_id() {
  if (!g_driver_fns_looked_up) {
    g_driver_fns_looked_up = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();
  }
  if (!g_ctx_current || !g_ctx_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (g_ctx_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
  if (g_ctx_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of the scratch array in the calling thread's current context.
static int noalloc_scratch(float** out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  unsigned long long id = current_context_id();
  if (id != 0) {
    auto it = g_noalloc_by_ctx.find(id);
    if (it != g_noalloc_by_ctx.end()) {
      *out = it->second;
      return RF_OK;
    }
  }
  // the lookup makes the device's primary context current if the thread has
  // no context yet; the id is read again afterwards
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) {
    set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
    return RF_E_CUDA;
  }
  if (id == 0) id = current_context_id();
  if (id != 0) g_noalloc_by_ctx[id] = static_cast<float*>(p);
  *out = static_cast<float*>(p);
  return RF_OK;
}

}  // namespace rf

extern "C" int rf_dense_matvec_noalloc(const float* A, const float* x, float* y, int64_t R, void* stream) {
  using namespace rf;
  if (!A || !x || !y || R < 1) {
    set_last_error_str("rf_dense_matvec_noalloc: bad arguments");
    return RF_E_INPUT;
  }
  if (R > kNoAllocMaxRows) {
    set_last_error_str("rf_dense_matvec_noalloc: R exceeds the 131072-row limit of the fixed scratch array");
    return RF_E_INPUT;
  }
  int dev = 0, sms = 148;
  RF_CUDA_TRY(cudaGetDevice(&dev));
  RF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  float* scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc != RF_OK) return rc;
  const DenseGemvPlan p = noalloc_gemv_plan(R, sms);
  // every (split, row) partial is written before it is read: nothing in the
  // shared scratch has to start at zero
  cudaStream_t st = (cudaStream_t)stream;
  rc = launch_dense_gemv(p, A, R, R, x, scratch, nullptr, st);
  if (rc == RF_OK) rc = launch_reduce_rows(scratch, p.splits, R, y, st);
  return rc;
}

extern "C" int rf_debug_noalloc_plan(int64_t R, int sms, int* splits, int64_t* cols_per_split) {
  using namespace rf;
  if (R < 1 || R > kNoAllocMaxRows || sms < 1 || !splits || !cols_per_split) return RF_E_INPUT;
  const DenseGemvPlan p = noalloc_gemv_plan(R, sms);
  *splits = p.splits;
  *cols_per_split = p.cps;
  return RF_OK;
}
