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
// address is looked up once per device with cudaGetSymbolAddress, with that
// device current, on the first call made on that device.
#include <mutex>

#include "rf_common.cuh"
#include "rf_kernels.cuh"
#include "rf_krylov.cuh"

namespace rf {

// 8 MiB: enough split-partial rows for any system with R <= kNoAllocMaxRows.
constexpr int64_t kNoAllocScratchFloats = 2 * 1024 * 1024;
constexpr int64_t kNoAllocMaxRows = 131072;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchFloats];

static std::mutex g_noalloc_mutex;
static float* g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};

// Device address of the scratch array on `dev` (the current device).
static int noalloc_scratch(int dev, float** out) {
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    set_last_error_str("rf_dense_matvec_noalloc: device ordinal out of range");
    return RF_E_INPUT;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (g_noalloc_ptr[dev] == nullptr) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      set_last_error(cudaGetErrorString(e), __FILE__, __LINE__);
      return RF_E_CUDA;
    }
    g_noalloc_ptr[dev] = static_cast<float*>(p);
  }
  *out = g_noalloc_ptr[dev];
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
  int rc = noalloc_scratch(dev, &scratch);
  if (rc != RF_OK) return rc;
  // same split plan as rf_dense_matvec, capped so the partial rows fit
  DenseGemvPlan p = plan_dense_gemv(R, sms);
  const int64_t max_splits = kNoAllocScratchFloats / R;
  if (p.splits > max_splits) {
    p.cps = ceil_div(R, max_splits);
    p.splits = (int)ceil_div(R, p.cps);
  }
  // every (split, row) partial is written before it is read: nothing in the
  // shared scratch has to start at zero
  cudaStream_t st = (cudaStream_t)stream;
  rc = launch_dense_gemv(p, A, R, R, x, scratch, nullptr, st);
  if (rc == RF_OK) rc = launch_reduce_rows(scratch, p.splits, R, y, st);
  return rc;
}
