// Blocked LU without row exchanges, every O(R^3) product on the tensor cores.
//
// The systems of this problem have identity diagonal blocks and couplings
// that are mostly well below 1 (largest off-diagonal entry 0.55 at N=1000 in a
// sphere of radius 14), so elimination without row exchanges is stable for
// them.  At step j of LAPACK's sgetrf (MAGMA's magma_sgetrf_gpu behind the
// reference's --magma path, src/simulation.cu:403-418) the pivot is the
// diagonal entry exactly when |a_ij / a_jj| <= 1 for every i > j, i.e. when
// the multipliers l_ij of the unpivoted factorization are at most 1 in
// magnitude: then these are partial pivoting's factors (up to rounding
// order).  Nearly touching fibers give multipliers above 1 (up to ~24 in the
// benchmark layouts); the factors are then kept as a static-pivoting
// factorization (Li & Demmel, "Making sparse Gaussian elimination scalable
// by static pivoting", SC 1998: no row exchanges, accuracy recovered by
// iterative refinement) as long as no pivot vanished and every |l_ij| stays
// within kStaticPivotLimit; the caller's FP64-residual refinement then
// decides, and refactors with partial pivoting if it does not converge.
//
// Per pass of eight 128-column panels k_p = k + 128 p (Golub & Van Loan, the
// right-looking blocked LU, with the pass's later panels updated by its
// earlier ones first, so the trailing matrix is read and written once per 1024
// columns):
//   for p = 0 .. 7:
//     A(k_p.., k_p:k_p+128) -= [L21(k_0..k_p-1)] [U12(...)]    (GEMM, K = 128 p)
//     diag(k_p):  LU of the 128 x 128 diagonal block in shared memory (one
//                 CTA), and the explicit inverses U11^-1, L11^-1 of its factors
//     L21(k_p):   L21 = A21 U11^-1                             (GEMM, K = 128)
//     rows k_p..k_p+128 right of the panel -= L21 U12          (GEMM, K = 128 p)
//     U12(k_p):   U12 = L11^-1 A12                             (GEMM, K = 128)
//   A22 -= [L21(k_0) .. L21(k_7)] [U12(k_0); ..; U12(k_7)]     (GEMM, K = 1024)
//
// The GEMM: C (column-major) = or -= A B with A (M x K) and B (K x N) both
// K-major in shared memory, loaded by TMA (cp.async.bulk.tensor, 128-byte
// swizzle) into a two-stage mbarrier pipeline; one thread issues
// tcgen05.mma kind::tf32 (M = 128, N = BN, K = 8) into a tensor-memory
// accumulator and commits to the stage's "empty" barrier; after the last
// k-block the four warps read the accumulator (thread = row = TMEM lane) and
// update C.  L21 is K-major for that A operand only as a row-major copy (LT,
// R x 256), which the L21 GEMM writes beside the column-major factor; A21 is
// transposed into LT first.  U12 and the trailing columns are read straight
// from the column-major matrix, where each column's k-run is contiguous.
// Every wait is bounded (%globaltimer); a wait that gives up records -1 in
// the status word, and the kernel drains what it issued before freeing TMEM.
#include <cooperative_groups.h>
#include <cuda.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "rf_common.cuh"
#include "rf_lu.cuh"

namespace cg = cooperative_groups;

namespace rf {

namespace {

constexpr int kTcBM = 128;          // rows per tile (TMEM lanes)
constexpr int kTcBK = 32;           // k per pipeline stage: 32 floats = one 128-byte swizzle row
constexpr int kTcStages = 2;
constexpr int kPanel = 128;         // panel width
constexpr int kPassPanels = 8;                 // panels factored per pass of the trailing update
constexpr int kLtCols = kPassPanels * kPanel;  // columns of the row-major L21 copy
constexpr uint64_t kDrainNs = 1000000000ull;
// largest multiplier of factors kept without row exchanges (bounded growth)
constexpr float kStaticPivotLimit = 64.f;

enum TcMode { kTcStore = 0, kTcSub = 1, kTcStoreL = 2 };

struct TcArgs {
  float* C;            // output tile origin (row 0, column 0 of the product)
  int64_t ldc;
  int M, N;            // product size
  int a_x, a_y;        // A operand: k and row coordinates of its origin in tmA
  int b_x, b_y;        // B operand: k and column coordinates of its origin in tmB
  int kblocks;         // K / 32
  int c_x, c_y;        // kTcSub: row and column coordinates of C's origin in tmC
  float* lt;           // kTcStoreL: row-major copy, row r at lt + r * ldlt
  int64_t ldlt;
  unsigned int* lmax;  // kTcStoreL: largest |value| (float bits, values >= 0)
  int* status;         // -1 on a timed-out wait
  uint64_t wait_ns;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bounded wait on an mbarrier phase; false when limit_ns passed
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
  const uint64_t t0 = now_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
    if (now_ns() - t0 > limit_ns) return false;
  }
}

// SW128 K-major shared-memory matrix descriptor: rows of 128 bytes, 8-row
// groups 1024 bytes apart, version 1, layout type 2 (128-byte swizzle)
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, int x, int y, uint32_t src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(src)
               : "memory");
}

// kTcSub stages the whole C tile in shared memory: one TMA load issued before
// the k-loop (so it overlaps the products), the update applied there from
// TMEM, one TMA store (clipped at the matrix edge) at the end
template <int BN, int MODE>
__global__ void __launch_bounds__(128, 1) k_tc_gemm(const __grid_constant__ CUtensorMap tmA,
                                                    const __grid_constant__ CUtensorMap tmB,
                                                    const __grid_constant__ CUtensorMap tmC, TcArgs a) {
  constexpr uint32_t kABytes = kTcBM * kTcBK * 4;   // 16 KB
  constexpr uint32_t kBBytes = BN * kTcBK * 4;
  constexpr uint32_t kStageBytes = kABytes + kBBytes;
  constexpr uint32_t kCBytes = kTcBM * BN * 4;
  // F32 accumulator, TF32 A and B, both K-major, N = BN, M = 128
  constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) |
                              ((uint32_t)(kTcBM >> 4) << 24);
  extern __shared__ __align__(1024) unsigned char dsm[];
  __shared__ __align__(8) uint64_t full[kTcStages], empty[kTcStages], accf, cbar;
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail;
  // 1024-byte alignment of the swizzled tiles
  unsigned char* base = dsm + ((1024 - (smem_u32(dsm) & 1023)) & 1023);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kTcBM, n0 = blockIdx.y * BN;
  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[s])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[s])) : "memory");
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&accf)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&cbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_fail = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  const int KB = a.kblocks;

  int last_kb[kTcStages];
#pragma unroll
  for (int s = 0; s < kTcStages; ++s) last_kb[s] = -1;
  float* sC = reinterpret_cast<float*>(base + kTcStages * kStageBytes);   // [BN][128] (kTcSub)
  if (warp == 0 && lane == 0) {
    if (MODE == kTcSub) {
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&cbar)), "r"(kCBytes)
                   : "memory");
      tma_load_2d(smem_u32(sC), &tmC, a.c_x + m0, a.c_y + n0, smem_u32(&cbar));
    }
    // producer: TMA loads of A and B k-blocks into the ring of stages
    for (int kb = 0; kb < KB; ++kb) {
      const int s = kb % kTcStages;
      if (kb >= kTcStages && !mbar_wait(&empty[s], ((kb / kTcStages) - 1) & 1, a.wait_ns)) {
        atomicExch(&s_fail, 1);
        break;
      }
      if (s_fail) break;
      last_kb[s] = kb;
      unsigned char* st = base + s * kStageBytes;
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&full[s])),
                   "r"(kStageBytes)
                   : "memory");
      tma_load_2d(smem_u32(st), &tmA, a.a_x + kb * kTcBK, a.a_y + m0, smem_u32(&full[s]));
      tma_load_2d(smem_u32(st + kABytes), &tmB, a.b_x + kb * kTcBK, a.b_y + n0, smem_u32(&full[s]));
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    int issued = 0;
    for (int kb = 0; kb < KB; ++kb) {
      const int s = kb % kTcStages;
      if (s_fail || !mbar_wait(&full[s], (kb / kTcStages) & 1, a.wait_ns)) {
        atomicExch(&s_fail, 1);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sa = smem_u32(base + s * kStageBytes), sb = sa + kABytes;
#pragma unroll
      for (int k = 0; k < kTcBK / 8; ++k) {
        const uint64_t da = sw128_desc(sa + 32 * k), db = sw128_desc(sb + 32 * k);
        const uint32_t acc = (kb > 0 || k > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
            "l"(da), "l"(db), "r"(kIdesc), "r"(acc));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&empty[s]))
                   : "memory");
      ++issued;
    }
    // completes when every MMA issued above has (also on the failure path, so
    // that TMEM is not freed under them)
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(&accf))
                 : "memory");
    (void)issued;
  }
  __syncwarp();
  // epilogue: all four warps; thread = row = TMEM lane
  const bool done = mbar_wait(&accf, 0, a.wait_ns);
  const bool ok = __syncthreads_and(done && !s_fail) != 0;
  if (!ok) {
    if (tid == 0) atomicExch(a.status, -1);
    // drain: the last load issued into each stage has landed (at most one
    // use of a stage is outstanding, so its phase parity identifies it)
    // (bounded by one second whatever the injected limit, so a shortened
    // limit never lets the CTA exit under its own copies or MMAs)
    if (warp == 0 && lane == 0) {
      for (int s = 0; s < kTcStages; ++s)
        if (last_kb[s] >= 0) (void)mbar_wait(&full[s], (last_kb[s] / kTcStages) & 1, kDrainNs);
      if (MODE == kTcSub) (void)mbar_wait(&cbar, 0, kDrainNs);
    }
    if (!done && tid == 0) (void)mbar_wait(&accf, 0, kDrainNs);
  } else if (MODE == kTcSub) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int row = warp * 32 + lane;
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
    const bool cok = mbar_wait(&cbar, 0, a.wait_ns);
    const bool all = __syncthreads_and(cok) != 0;
    if (!all) {
      if (tid == 0) {
        atomicExch(a.status, -1);
        (void)mbar_wait(&cbar, 0, kDrainNs);
      }
    } else {
#pragma unroll 1
      for (int cc = 0; cc < BN; cc += 32) {
        if (n0 + cc >= a.N) break;
        uint32_t d[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
              "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15]),
              "=r"(d[16]), "=r"(d[17]), "=r"(d[18]), "=r"(d[19]), "=r"(d[20]), "=r"(d[21]), "=r"(d[22]),
              "=r"(d[23]), "=r"(d[24]), "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]), "=r"(d[29]),
              "=r"(d[30]), "=r"(d[31])
            : "r"(taddr + (uint32_t)cc));
        asm volatile("tcgen05.wait::ld.sync.aligned;"
                     : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3]), "+r"(d[4]), "+r"(d[5]), "+r"(d[6]),
                       "+r"(d[7]), "+r"(d[8]), "+r"(d[9]), "+r"(d[10]), "+r"(d[11]), "+r"(d[12]), "+r"(d[13]),
                       "+r"(d[14]), "+r"(d[15]), "+r"(d[16]), "+r"(d[17]), "+r"(d[18]), "+r"(d[19]), "+r"(d[20]),
                       "+r"(d[21]), "+r"(d[22]), "+r"(d[23]), "+r"(d[24]), "+r"(d[25]), "+r"(d[26]), "+r"(d[27]),
                       "+r"(d[28]), "+r"(d[29]), "+r"(d[30]), "+r"(d[31])
                     :
                     : "memory");
        float* col = sC + cc * kTcBM + row;
#pragma unroll
        for (int j = 0; j < 32; ++j) col[j * kTcBM] -= __uint_as_float(d[j]);
      }
      // generic-proxy writes of the tile -> the TMA store (async proxy)
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        tma_store_2d(&tmC, a.c_x + m0, a.c_y + n0, smem_u32(sC));
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        // the shared-memory source must stay until the store has read it
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
      }
    }
  } else {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int row = warp * 32 + lane;
    const int gr = m0 + row;
    const bool rok = gr < a.M;
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
    float* crow = a.C + (rok ? gr : 0);
    float vmax = 0.f;
    // C of chunk cc + 32 is loaded while chunk cc is combined with the
    // accumulator: every load of a chunk is issued before any store, so each
    // thread keeps 32 reads in flight instead of one at a time
    float cv[32], cn[32];
    auto load_chunk = [&](int cc, float (&dst)[32]) {
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int gc = n0 + cc + j;
        dst[j] = (MODE == kTcSub && rok && gc < a.N) ? __ldcg(crow + (int64_t)gc * a.ldc) : 0.f;
      }
    };
    load_chunk(0, cv);
#pragma unroll 1
    for (int cc = 0; cc < BN; cc += 32) {
      if (n0 + cc >= a.N) break;
      if (cc + 32 < BN && n0 + cc + 32 < a.N) load_chunk(cc + 32, cn);
      uint32_t d[32];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
          "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
          : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
            "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15]),
            "=r"(d[16]), "=r"(d[17]), "=r"(d[18]), "=r"(d[19]), "=r"(d[20]), "=r"(d[21]), "=r"(d[22]), "=r"(d[23]),
            "=r"(d[24]), "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]), "=r"(d[29]), "=r"(d[30]), "=r"(d[31])
          : "r"(taddr + (uint32_t)cc));
      asm volatile("tcgen05.wait::ld.sync.aligned;"
                   : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3]), "+r"(d[4]), "+r"(d[5]), "+r"(d[6]), "+r"(d[7]),
                     "+r"(d[8]), "+r"(d[9]), "+r"(d[10]), "+r"(d[11]), "+r"(d[12]), "+r"(d[13]), "+r"(d[14]),
                     "+r"(d[15]), "+r"(d[16]), "+r"(d[17]), "+r"(d[18]), "+r"(d[19]), "+r"(d[20]), "+r"(d[21]),
                     "+r"(d[22]), "+r"(d[23]), "+r"(d[24]), "+r"(d[25]), "+r"(d[26]), "+r"(d[27]), "+r"(d[28]),
                     "+r"(d[29]), "+r"(d[30]), "+r"(d[31])
                   :
                   : "memory");
      if (rok) {
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int gc = n0 + cc + j;
          if (gc < a.N) {
            const float v = __uint_as_float(d[j]);
            __stcg(crow + (int64_t)gc * a.ldc, MODE == kTcSub ? cv[j] - v : v);
            if (MODE == kTcStoreL) vmax = fmaxf(vmax, fabsf(v));
          }
        }
        if (MODE == kTcStoreL) {
          float* lrow = a.lt + (int64_t)gr * a.ldlt + n0 + cc;
#pragma unroll
          for (int j = 0; j < 32; j += 4) {
            if (n0 + cc + j + 3 < a.N) {
              *reinterpret_cast<float4*>(lrow + j) =
                  make_float4(__uint_as_float(d[j]), __uint_as_float(d[j + 1]), __uint_as_float(d[j + 2]),
                              __uint_as_float(d[j + 3]));
            } else {
              for (int u = 0; u < 4 && n0 + cc + j + u < a.N; ++u) lrow[j + u] = __uint_as_float(d[j + u]);
            }
          }
        }
      }
#pragma unroll
      for (int j = 0; j < 32; ++j) cv[j] = cn[j];
    }
    if (MODE == kTcStoreL) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
      if (lane == 0) atomicMax(a.lmax, __float_as_uint(vmax));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
  }
}

// ---------------------------------------------------------------------------
// The trailing update C -= A B as a persistent, warp-specialized kernel: one
// CTA per SM walks the 128 x BN tiles (m fastest, so CTAs in flight share
// their B tile in L2).  Warp 0 streams the A and B k-blocks by TMA into a ring
// of kUpStages stages; warp 1 issues the tcgen05 MMAs into one of two TMEM
// accumulators (2 x BN columns), so the products of tile t+1 run while tile t
// is being written back; warp 6 streams C in 128 x 32 chunks by TMA into a ring
// of kUpSlots slots ahead of the epilogue; warps 2-5 (one TMEM lane quarter
// each) subtract the accumulator chunk from the C chunk in shared memory and
// write it back with a TMA store (clipped at the matrix edge).  All waits are
// bounded; a failed wait stops every role, which then drains what it issued.
// ---------------------------------------------------------------------------
constexpr int kUpStages = 3;
constexpr int kUpSlots = 4;
constexpr int kUpChunk = 32;                                  // columns per C chunk
constexpr uint32_t kUpChunkBytes = kTcBM * kUpChunk * 4;      // 16 KB

template <int BN>
constexpr size_t up_smem() {
  return (size_t)kUpStages * (kTcBM + BN) * kTcBK * 4 + (size_t)kUpSlots * kUpChunkBytes + 1024;
}

struct UpArgs {
  int M, N;            // product size
  int a_x, a_y;        // A: k and row coordinates of the product's origin in tmA
  int b_x, b_y;        // B: k and column coordinates in tmB
  int c_x, c_y;        // C: row and column coordinates in tmC
  int kblocks;
  int tiles_m, tiles;
  int* status;
  uint64_t wait_ns;
};

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// AND of `v` over the 128 threads of named barrier 1 (the epilogue warps), so
// that they all take the same branch before the next named barrier
__device__ __forceinline__ bool epi_all(bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 q, %1, 0;\n\tbar.red.and.pred p, 1, 128, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v)
      : "memory");
  return r != 0;
}

template <int BN>
__global__ void __launch_bounds__(224, 1) k_tc_update(const __grid_constant__ CUtensorMap tmA,
                                                      const __grid_constant__ CUtensorMap tmB,
                                                      const __grid_constant__ CUtensorMap tmC, UpArgs a) {
  constexpr uint32_t kABytes = kTcBM * kTcBK * 4;
  constexpr uint32_t kStageBytes = kABytes + BN * kTcBK * 4;
  constexpr int kChunks = BN / kUpChunk;
  constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) |
                              ((uint32_t)(kTcBM >> 4) << 24);
  extern __shared__ __align__(1024) unsigned char dsm[];
  __shared__ __align__(8) uint64_t full[kUpStages], empty[kUpStages], accf[2], acce[2], cfull[kUpSlots],
      cempty[kUpSlots], drain;
  __shared__ uint32_t s_tmem;
  __shared__ volatile int fail;
  unsigned char* base = dsm + ((1024 - (smem_u32(dsm) & 1023)) & 1023);
  float* cslots = reinterpret_cast<float*>(base + kUpStages * kStageBytes);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int i = 0; i < kUpStages; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[i])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[i])) : "memory");
    }
    for (int i = 0; i < 2; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&accf[i])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(smem_u32(&acce[i])) : "memory");
    }
    for (int i = 0; i < kUpSlots; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&cfull[i])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&cempty[i])) : "memory");
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&drain)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fail = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(2 * BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  const int KB = a.kblocks;
  auto give_up = [&]() {
    fail = 1;
    atomicExch(a.status, -1);
  };
  auto nchunks = [&](int n0) { return min(kChunks, (a.N - n0 + kUpChunk - 1) / kUpChunk); };

  if (warp == 0) {
    if (lane == 0) {
      // operand producer
      int g = 0;
      for (int t = blockIdx.x; t < a.tiles && !fail; t += gridDim.x) {
        const int m0 = (t % a.tiles_m) * kTcBM, n0 = (t / a.tiles_m) * BN;
        for (int kb = 0; kb < KB; ++kb, ++g) {
          const int st = g % kUpStages;
          if (g >= kUpStages && !mbar_wait(&empty[st], ((g / kUpStages) - 1) & 1, a.wait_ns)) {
            give_up();
            break;
          }
          if (fail) break;
          unsigned char* sp = base + st * kStageBytes;
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&full[st])),
                       "r"(kStageBytes)
                       : "memory");
          tma_load_2d(smem_u32(sp), &tmA, a.a_x + kb * kTcBK, a.a_y + m0, smem_u32(&full[st]));
          tma_load_2d(smem_u32(sp + kABytes), &tmB, a.b_x + kb * kTcBK, a.b_y + n0, smem_u32(&full[st]));
        }
      }
      // drain: the last use of each stage has landed
      for (int st = 0; st < kUpStages; ++st) {
        const int last = g - 1 - ((g - 1 - st) % kUpStages + kUpStages) % kUpStages;
        if (g > 0 && last >= 0 && last % kUpStages == st) (void)mbar_wait(&full[st], (last / kUpStages) & 1, kDrainNs);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issuer
      int g = 0, lt = 0;
      for (int t = blockIdx.x; t < a.tiles && !fail; t += gridDim.x, ++lt) {
        const int b = lt & 1;
        if (lt >= 2 && !mbar_wait(&acce[b], ((lt / 2) - 1) & 1, a.wait_ns)) {
          give_up();
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc_addr = tmem + (uint32_t)(b * BN);
        bool ok = true;
        for (int kb = 0; kb < KB; ++kb, ++g) {
          const int st = g % kUpStages;
          if (fail || !mbar_wait(&full[st], (g / kUpStages) & 1, a.wait_ns)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t sa = smem_u32(base + st * kStageBytes), sb = sa + kABytes;
#pragma unroll
          for (int k = 0; k < kTcBK / 8; ++k) {
            const uint64_t da = sw128_desc(sa + 32 * k), db = sw128_desc(sb + 32 * k);
            const uint32_t acc = (kb > 0 || k > 0) ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(acc_addr),
                "l"(da), "l"(db), "r"(kIdesc), "r"(acc));
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                           smem_u32(&empty[st]))
                       : "memory");
        }
        if (!ok) {
          give_up();
          break;
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&accf[b]))
                     : "memory");
      }
      // every MMA issued above has completed before TMEM is freed
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&drain))
                   : "memory");
      (void)mbar_wait(&drain, 0, kDrainNs);
    }
  } else if (warp == 6) {
    if (lane == 0) {
      // C loader: 128 x 32 chunks into the slot ring, ahead of the epilogue
      int q = 0;
      for (int t = blockIdx.x; t < a.tiles && !fail; t += gridDim.x) {
        const int m0 = (t % a.tiles_m) * kTcBM, n0 = (t / a.tiles_m) * BN;
        const int nch = nchunks(n0);
        for (int c = 0; c < nch; ++c, ++q) {
          const int r = q % kUpSlots;
          if (q >= kUpSlots && !mbar_wait(&cempty[r], ((q / kUpSlots) - 1) & 1, a.wait_ns)) {
            give_up();
            break;
          }
          if (fail) break;
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&cfull[r])),
                       "r"(kUpChunkBytes)
                       : "memory");
          tma_load_2d(smem_u32(cslots + r * (kTcBM * kUpChunk)), &tmC, a.c_x + m0, a.c_y + n0 + c * kUpChunk,
                      smem_u32(&cfull[r]));
        }
      }
      for (int r = 0; r < kUpSlots && q > 0; ++r) {
        const int last = q - 1 - ((q - 1 - r) % kUpSlots + kUpSlots) % kUpSlots;
        if (last >= 0 && last % kUpSlots == r) (void)mbar_wait(&cfull[r], (last / kUpSlots) & 1, kDrainNs);
      }
    }
  } else {
    // epilogue: warps 2..5, TMEM lane quarter warp % 4
    const int quarter = warp & 3;
    const int row = quarter * 32 + lane;
    const bool leader = warp == 2 && lane == 0;
    int q = 0, lt = 0;
    // every branch below is decided by all 128 epilogue threads together
    // (epi_all), so none of them is left waiting at the named barrier
    for (int t = blockIdx.x; t < a.tiles; t += gridDim.x, ++lt) {
      const int n0 = (t / a.tiles_m) * BN;
      const int b = lt & 1;
      const bool got = !fail && mbar_wait(&accf[b], (lt / 2) & 1, a.wait_ns);
      if (!epi_all(got)) {
        if (leader) give_up();
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * BN);
      const int m0 = (t % a.tiles_m) * kTcBM;
      const int nch = nchunks(n0);
      bool ok = true;
      for (int c = 0; c < nch; ++c, ++q) {
        const int r = q % kUpSlots;
        const bool got = !fail && mbar_wait(&cfull[r], (q / kUpSlots) & 1, a.wait_ns);
        if (!epi_all(got)) {
          ok = false;
          break;
        }
        uint32_t d[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
              "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15]),
              "=r"(d[16]), "=r"(d[17]), "=r"(d[18]), "=r"(d[19]), "=r"(d[20]), "=r"(d[21]), "=r"(d[22]),
              "=r"(d[23]), "=r"(d[24]), "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]), "=r"(d[29]),
              "=r"(d[30]), "=r"(d[31])
            : "r"(taddr + (uint32_t)(c * kUpChunk)));
        asm volatile("tcgen05.wait::ld.sync.aligned;"
                     : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3]), "+r"(d[4]), "+r"(d[5]), "+r"(d[6]),
                       "+r"(d[7]), "+r"(d[8]), "+r"(d[9]), "+r"(d[10]), "+r"(d[11]), "+r"(d[12]), "+r"(d[13]),
                       "+r"(d[14]), "+r"(d[15]), "+r"(d[16]), "+r"(d[17]), "+r"(d[18]), "+r"(d[19]), "+r"(d[20]),
                       "+r"(d[21]), "+r"(d[22]), "+r"(d[23]), "+r"(d[24]), "+r"(d[25]), "+r"(d[26]), "+r"(d[27]),
                       "+r"(d[28]), "+r"(d[29]), "+r"(d[30]), "+r"(d[31])
                     :
                     : "memory");
        float* col = cslots + r * (kTcBM * kUpChunk) + row;   // [32 columns][128 rows]
#pragma unroll
        for (int j = 0; j < 32; ++j) col[j * kTcBM] -= __uint_as_float(d[j]);
        // the slot's generic-proxy writes -> the TMA store, once all 128 rows are in
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("bar.sync 1, 128;" ::: "memory");
        if (leader) {
          tma_store_2d(&tmC, a.c_x + m0, a.c_y + n0 + c * kUpChunk, smem_u32(cslots + r * (kTcBM * kUpChunk)));
          asm volatile("cp.async.bulk.commit_group;" ::: "memory");
          asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
          mbar_arrive(&cempty[r]);
        }
      }
      // this accumulator may be overwritten by the next tile's products
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&acce[b]);
      if (!ok) {
        if (leader) give_up();
        break;
      }
    }
    if (leader) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * BN));
  }
}

template <int BN, int MODE>
constexpr size_t tc_smem() {
  return (size_t)kTcStages * (kTcBM + BN) * kTcBK * 4 + (MODE == kTcSub ? (size_t)kTcBM * BN * 4 : 0) + 1024;
}

// ---------------------------------------------------------------------------
// The w x w diagonal block (w <= 128) at (k, k): factored in shared memory
// without row exchanges (multiplier a * (1 / pivot), then fmaf(-l, u, a), as
// the pivoted panel does) and written back; the largest |l| into lmax, a zero
// pivot into status.  The inverses of its factors follow in k_lu_diag_inv.
//
// 32 warps, warp w owning columns w, w + 32, w + 64, w + 96, lane l rows
// l, l + 32, l + 64, l + 96 of each.  No step waits for the whole CTA: the
// owner of column j + 1 applies step j to that column first, scales it and
// publishes it through flag[j + 1] (a bounded spin in shared memory), then
// applies step j to its other columns; every warp applies the steps to its
// columns in order.
// ---------------------------------------------------------------------------
constexpr int kDiagLd = kPanel + 1;
constexpr uint32_t kDiagSpin = 1u << 26;

__global__ void __launch_bounds__(1024) k_lu_diag(float* __restrict__ A, int64_t lda, int64_t k, int w,
                                                  unsigned int* __restrict__ lmax, int* __restrict__ status) {
  extern __shared__ float sm[];
  float* a = sm;                          // [128][129] row-major block
  __shared__ volatile int flag[kPanel];   // 1: column j scaled, 2: abort
  const int tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, lane = tid & 31;
  for (int e = tid; e < kPanel * kPanel; e += nt) {
    const int r = e % kPanel, c = e / kPanel;   // coalesced over r (column-major source)
    a[r * kDiagLd + c] = (r < w && c < w) ? A[(k + r) + (k + c) * lda] : (r == c ? 1.f : 0.f);
  }
  if (tid < kPanel) flag[tid] = 0;
  __syncthreads();
  float vmax = 0.f;
  bool abort = false;
  // scale column j below the diagonal (the warp owning it); false on a zero pivot
  auto scale = [&](int j) -> bool {
    const float piv = a[j * kDiagLd + j];
    if (piv == 0.f) return false;
    const float inv = 1.f / piv;
    for (int r = (j + 1) >> 5; r < 4; ++r) {
      const int i = lane + 32 * r;
      if (i > j && i < w) {
        const float l = a[i * kDiagLd + j] * inv;
        a[i * kDiagLd + j] = l;
        vmax = fmaxf(vmax, fabsf(l));
      }
    }
    return true;
  };
  auto publish = [&](int j, int v) {
    __syncwarp();
    __threadfence_block();
    if (lane == 0) flag[j] = v;
  };
  // step j applied to column c (rows > j)
  auto apply = [&](int j, int c) {
    const float u = a[j * kDiagLd + c];
    for (int r = (j + 1) >> 5; r < 4; ++r) {
      const int i = lane + 32 * r;
      if (i > j && i < w) a[i * kDiagLd + c] = fmaf(-a[i * kDiagLd + j], u, a[i * kDiagLd + c]);
    }
  };
  if (w > 0 && warp == 0) {
    const bool ok = scale(0);
    publish(0, ok ? 1 : 2);
  }
  for (int j = 0; j < w && !abort; ++j) {
    // wait for column j (bounded)
    uint32_t spins = 0;
    int f;
    while ((f = flag[j]) == 0) {
      if (++spins > kDiagSpin) { f = 3; break; }
    }
    __syncwarp();
    __threadfence_block();
    if (f != 1) {
      if (lane == 0) atomicExch(status, f == 3 ? -1 : 2);
      abort = true;
      // the owners of later columns must not wait for this one
      if (j + 1 < w && ((j + 1) & 31) == warp) publish(j + 1, 2);
      break;
    }
    const int jn = j + 1;
    if (jn < w && (jn & 31) == warp) {
      apply(j, jn);
      __syncwarp();
      const bool ok = scale(jn);
      publish(jn, ok ? 1 : 2);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c = warp + 32 * q;
      if (c > j && c < w && c != jn) apply(j, c);
    }
    __syncwarp();
  }
  // every thread leaves here or none does (the barriers below need all of them)
  if (__syncthreads_or(abort)) return;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
  if (lane == 0) atomicMax(lmax, __float_as_uint(vmax));
  for (int e = tid; e < w * w; e += nt) {
    const int r = e % w, c = e / w;
    A[(k + r) + (k + c) * lda] = a[r * kDiagLd + c];
  }
}

// The inverses of the factored diagonal block (written back by k_lu_diag):
// 8 CTAs, CTAs 0-3 columns 32b.. of L11^-1, CTAs 4-7 those of U11^-1, one warp
// per column (lane l: rows l, l + 32, l + 64, l + 96), so the eight run side
// by side on eight SMs.  L11^-1: column c starts as e_c; step j (from c on)
// subtracts l_ij x_jc from the rows below j.  U11^-1: step j (from c down to
// 0) divides x_jc by u_jj and subtracts u_ij x_jc from the rows above j.
// Outputs: Linv row-major, UinvT (row n = column n of U11^-1), LinvC (both
// column-major); zero outside w x w.
__global__ void __launch_bounds__(1024) k_lu_diag_inv(const float* __restrict__ A, int64_t lda, int64_t k, int w,
                                                      float* __restrict__ Linv, float* __restrict__ UinvT,
                                                      float* __restrict__ LinvC, const int* __restrict__ status) {
  if (*status != 0) return;   // a zero pivot: the factors are discarded
  extern __shared__ float sm[];
  float* a = sm;                          // [128][129] the factored block
  float* x = sm + kPanel * kDiagLd;       // [128][33]  this CTA's 32 columns
  constexpr int kXLd = 33;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool upper = blockIdx.x >= 4;
  const int c = (blockIdx.x & 3) * 32 + warp;
  for (int e = tid; e < kPanel * kPanel; e += blockDim.x) {
    const int r = e % kPanel, cc = e / kPanel;
    a[r * kDiagLd + cc] = (r < w && cc < w) ? A[(k + r) + (k + cc) * lda] : (r == cc ? 1.f : 0.f);
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i = lane + 32 * r;
    x[i * kXLd + warp] = (i == c && c < w) ? 1.f : 0.f;
  }
  __syncwarp();
  if (c < w) {
    if (!upper) {
      for (int j = c; j < w - 1; ++j) {
        const float v = x[j * kXLd + warp];
        for (int r = (j + 1) >> 5; r < 4; ++r) {
          const int i = lane + 32 * r;
          if (i > j && i < w) x[i * kXLd + warp] = fmaf(-a[i * kDiagLd + j], v, x[i * kXLd + warp]);
        }
        __syncwarp();
      }
    } else {
      for (int j = c; j >= 0; --j) {
        const float v = x[j * kXLd + warp] / a[j * kDiagLd + j];
        __syncwarp();
        if (lane == (j & 31)) x[j * kXLd + warp] = v;
        for (int r = 0; r <= (j >> 5); ++r) {
          const int i = lane + 32 * r;
          if (i < j) x[i * kXLd + warp] = fmaf(-a[i * kDiagLd + j], v, x[i * kXLd + warp]);
        }
        __syncwarp();
      }
    }
  }
  __syncthreads();
  // write this CTA's 32 columns (rows 0..127)
  const int cb = (blockIdx.x & 3) * 32;
  for (int e = tid; e < kPanel * 32; e += blockDim.x) {
    const int i = e & (kPanel - 1), cl = e >> 7;   // column-major: coalesced over i
    const float v = x[i * kXLd + cl];
    if (!upper) {
      LinvC[(cb + cl) * kPanel + i] = v;
    } else {
      LinvC[kPanel * kPanel + (cb + cl) * kPanel + i] = v;
      UinvT[(cb + cl) * kPanel + i] = v;
    }
  }
  if (!upper) {
    for (int e = tid; e < kPanel * 32; e += blockDim.x) {
      const int cl = e & 31, i = e >> 5;   // row-major rows of L11^-1: 32 consecutive columns
      Linv[i * kPanel + cb + cl] = x[i * kXLd + cl];
    }
  }
}

// ---------------------------------------------------------------------------
// Triangular solves with the factors of lu_factor_tc (no permutation): one
// cooperative kernel per factor, 128-row blocks owned cyclically by the CTAs.
// Step b: the owner of block b turns y_b into x_b = D_b^-1 y_b with the stored
// inverse of the diagonal block (a 128 x 128 matvec), then a grid sync, then
// every CTA subtracts L[rows, block b] x_b (U[rows, block b] x_b) from the
// blocks it owns below (above) block b.  The owner of the next block updated
// that block itself, so one grid sync per block suffices.
// ---------------------------------------------------------------------------
struct TrsvArgs {
  const float* LU;
  int64_t lda, R;
  const float* sinv;   // per block: L^-1 column-major, then U^-1 column-major (2 x 128 x 128)
  float* y;            // right-hand side in, solution out
  int nblocks;
  int lower;
};

// 512 threads: row i = tid % 128 of a block, quarter h = tid / 128 of its
// 128 columns; each thread loads its 32 matrix values before the first
// multiply-add, so a CTA has the whole 128 x 128 block in flight at once
constexpr int kTrsvThreads = 512;

__global__ void __launch_bounds__(kTrsvThreads) k_trsv_tc(TrsvArgs a) {
  cg::grid_group grid = cg::this_grid();
  __shared__ float xs[kPanel];
  __shared__ float part[4][kPanel];
  const int tid = threadIdx.x, i = tid & (kPanel - 1), h = tid >> 7;
  const int P = gridDim.x, nb = a.nblocks;
  const int64_t R = a.R;
  for (int s = 0; s < nb; ++s) {
    const int b = a.lower ? s : nb - 1 - s;
    const int64_t r0 = (int64_t)b * kPanel;
    const int nr = (int)min((int64_t)kPanel, R - r0);
    if (b % P == (int)blockIdx.x) {
      if (tid < kPanel) xs[tid] = tid < nr ? a.y[r0 + tid] : 0.f;
      __syncthreads();
      const float* inv = a.sinv + (int64_t)b * 2 * kPanel * kPanel + (a.lower ? 0 : kPanel * kPanel);
      float m[32];
#pragma unroll
      for (int q = 0; q < 32; ++q) m[q] = __ldcs(inv + (int64_t)(h * 32 + q) * kPanel + i);
      float v = 0.f;
#pragma unroll
      for (int q = 0; q < 32; ++q) v = fmaf(m[q], xs[h * 32 + q], v);
      part[h][i] = v;
      __syncthreads();
      if (tid < nr) a.y[r0 + tid] = (part[0][tid] + part[1][tid]) + (part[2][tid] + part[3][tid]);
    }
    grid.sync();
    // x_b into shared memory, then the owned blocks on the far side of b
    if (tid < kPanel) xs[tid] = tid < nr ? __ldcg(a.y + r0 + tid) : 0.f;
    __syncthreads();
    const int first = a.lower ? b + 1 : 0, last = a.lower ? nb - 1 : b - 1;
    int bb = first + ((int)blockIdx.x - first % P + P) % P;
    for (; bb <= last; bb += P) {
      const int64_t q0 = (int64_t)bb * kPanel;
      const int nq = (int)min((int64_t)kPanel, R - q0);
      float v = 0.f;
      if (i < nq) {
        const float* col = a.LU + (q0 + i) + (r0 + h * 32) * a.lda;
        float m[32];
#pragma unroll
        for (int c = 0; c < 32; ++c) m[c] = (h * 32 + c < nr) ? __ldcs(col + (int64_t)c * a.lda) : 0.f;
#pragma unroll
        for (int c = 0; c < 32; ++c) v = fmaf(m[c], xs[h * 32 + c], v);
      }
      part[h][i] = v;
      __syncthreads();
      if (tid < nq) a.y[q0 + tid] -= (part[0][tid] + part[1][tid]) + (part[2][tid] + part[3][tid]);
      __syncthreads();
    }
  }
}

// LT[r][col0 + c] = A[r0 + r, k + c] for c < w, 0 for w <= c < 128 (rows r < m)
__global__ void k_lu_to_rows(const float* __restrict__ A, int64_t lda, int64_t r0, int64_t k, int w, int64_t m,
                             float* __restrict__ LT, int col0) {
  __shared__ float t[32][33];
  const int64_t rb = (int64_t)blockIdx.x * 32;
  const int cb = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;   // 32 x 8
  for (int yy = ty; yy < 32; yy += 8) {
    const int c = cb + yy;
    const int64_t r = rb + tx;
    t[yy][tx] = (r < m && c < w) ? A[(r0 + r) + (k + c) * lda] : 0.f;
  }
  __syncthreads();
  for (int yy = ty; yy < 32; yy += 8) {
    const int64_t r = rb + yy;
    const int c = cb + tx;
    if (r < m) LT[r * kLtCols + col0 + c] = t[tx][yy];
  }
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static std::once_flag once;
  static EncodeTiledFn fn = nullptr;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
    cudaGetLastError();
  });
  return fn;
}

// A 2-D FP32 map: inner dimension `inner` (contiguous), `outer` rows of
// `stride_bytes`; boxes of 32 inner x box_outer, 128-byte swizzle, zero fill
// outside the extent.
int make_map(CUtensorMap* map, const float* base, uint64_t inner, uint64_t outer, uint64_t stride_bytes,
             uint32_t box_outer, uint32_t box_inner = kTcBK,
             CUtensorMapSwizzle swz = CU_TENSOR_MAP_SWIZZLE_128B) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) {
    set_last_error_str("lu: cuTensorMapEncodeTiled unavailable");
    return RF_E_CUDA;
  }
  const cuuint64_t dims[2] = {inner, outer};
  const cuuint64_t strides[1] = {stride_bytes};
  const cuuint32_t box[2] = {box_inner, box_outer};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_last_error_str("lu: cuTensorMapEncodeTiled failed");
    return RF_E_CUDA;
  }
  return RF_OK;
}

struct TcMaps {
  CUtensorMap mat_b128, mat_b256;   // the factored matrix as a B operand (k = rows, n = columns)
  CUtensorMap mat_c128, mat_c256;   // the factored matrix as a C tile (128 rows x 128 / 256 columns)
  CUtensorMap mat_c32;              // the factored matrix as a C chunk (128 rows x 32 columns)
  CUtensorMap lt;                   // LT as an A operand (k = columns, m = rows)
  CUtensorMap linv;                 // L11^-1 as an A operand
  CUtensorMap uinvT;                // U11^-1 as a B operand (row n = column n)
};

template <int BN, int MODE>
int launch_tc(const CUtensorMap& ta, const CUtensorMap& tb, const CUtensorMap& tc, const TcArgs& a,
              cudaStream_t st) {
  if (a.M <= 0 || a.N <= 0) return RF_OK;
  static const cudaError_t attr = cudaFuncSetAttribute(
      k_tc_gemm<BN, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc_smem<BN, MODE>());
  RF_CUDA_TRY(attr);
  dim3 grid((unsigned)ceil_div(a.M, kTcBM), (unsigned)ceil_div(a.N, BN));
  k_tc_gemm<BN, MODE><<<grid, 128, tc_smem<BN, MODE>(), st>>>(ta, tb, tc, a);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

// C -= A B over the product M x N (coordinates in the three maps) by the
// persistent update kernel; one CTA per SM at most
template <int BN>
int launch_update(const CUtensorMap& ta, const CUtensorMap& tb, const CUtensorMap& tc, UpArgs u, int sms,
                  cudaStream_t st) {
  if (u.M <= 0 || u.N <= 0) return RF_OK;
  static const cudaError_t attr =
      cudaFuncSetAttribute(k_tc_update<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)up_smem<BN>());
  RF_CUDA_TRY(attr);
  u.tiles_m = (int)ceil_div(u.M, kTcBM);
  u.tiles = u.tiles_m * (int)ceil_div(u.N, BN);
  const int grid = std::max(1, std::min(sms, u.tiles));
  k_tc_update<BN><<<grid, 224, up_smem<BN>(), st>>>(ta, tb, tc, u);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

}  // namespace

int64_t lu_tc_lt_floats(int64_t R) { return R * kLtCols; }
int64_t lu_tc_inv_floats() { return 2 * (int64_t)kPanel * kPanel; }
int64_t lu_tc_sinv_floats(int64_t R) { return ceil_div(R, kPanel) * 2 * kPanel * kPanel; }

// x = (LU)^-1 rhs with the factors of lu_factor_tc (rhs and x distinct)
int lu_solve_tc(const LuSetup& s, const float* rhs, float* x, cudaStream_t st) {
  const int64_t R = s.R;
  RF_CUDA_TRY(cudaMemcpyAsync(x, rhs, R * sizeof(float), cudaMemcpyDeviceToDevice, st));
  TrsvArgs t;
  t.LU = s.LU;
  t.lda = s.ldlu ? s.ldlu : s.lda;
  t.R = R;
  t.sinv = s.sinv;
  t.y = x;
  t.nblocks = (int)ceil_div(R, kPanel);
  // every CTA must be resident (grid syncs): at most what the SMs hold
  static int occ = -1;
  static int sms = 0;
  if (occ < 0) {
    int dev = 0;
    RF_CUDA_TRY(cudaGetDevice(&dev));
    RF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    RF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_trsv_tc, kTrsvThreads, 0));
  }
  const int P = std::max(1, std::min(std::min(s.coop_blocks, t.nblocks), std::max(1, occ) * sms));
  for (int lower = 1; lower >= 0; --lower) {
    t.lower = lower;
    void* args[] = {&t};
    RF_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_trsv_tc, dim3(P), dim3(kTrsvThreads), args, 0, st));
  }
  return RF_OK;
}

// The unpivoted factorization of s.LU (already a copy of A).  Returns RF_OK
// with *clean = true when no pivot vanished and every multiplier is at most
// kStaticPivotLimit in magnitude (at most 1: the factors of partial pivoting),
// *max_l the largest |l_ij|; *clean = false otherwise (the caller refactors
// with pivoting).  RF_E_TIMEOUT when a bounded wait gave up.
int lu_factor_tc(const LuSetup& s, cudaStream_t st, bool* clean, int* launches, float* max_l) {
  const int64_t R = s.R, lda = s.ldlu ? s.ldlu : s.lda;
  *clean = false;
  if ((lda % 4) != 0 || (reinterpret_cast<uintptr_t>(s.LU) % 16) != 0 || !s.LT || !s.inv || !s.flags || !s.sinv) {
    set_last_error_str("lu: tensor-core factorization needs a 16-byte aligned matrix and its buffers");
    return RF_E_UNSUPPORTED;
  }
  float* Linv = s.inv;
  float* UinvT = s.inv + kPanel * kPanel;
  unsigned int* lmax = reinterpret_cast<unsigned int*>(s.flags);
  int* status = s.flags + 1;
  RF_CUDA_TRY(cudaMemsetAsync(s.flags, 0, 2 * sizeof(int), st));
  TcMaps mp;
  RF_TRY_RF(make_map(&mp.mat_b128, s.LU, (uint64_t)R, (uint64_t)R, (uint64_t)lda * 4, 128));
  RF_TRY_RF(make_map(&mp.mat_b256, s.LU, (uint64_t)R, (uint64_t)R, (uint64_t)lda * 4, 256));
  RF_TRY_RF(make_map(&mp.mat_c128, s.LU, (uint64_t)R, (uint64_t)R, (uint64_t)lda * 4, 128, kTcBM,
                     CU_TENSOR_MAP_SWIZZLE_NONE));
  RF_TRY_RF(make_map(&mp.mat_c256, s.LU, (uint64_t)R, (uint64_t)R, (uint64_t)lda * 4, 256, kTcBM,
                     CU_TENSOR_MAP_SWIZZLE_NONE));
  RF_TRY_RF(make_map(&mp.mat_c32, s.LU, (uint64_t)R, (uint64_t)R, (uint64_t)lda * 4, kUpChunk, kTcBM,
                     CU_TENSOR_MAP_SWIZZLE_NONE));
  int sms = 148;
  {
    int dev = 0;
    RF_CUDA_TRY(cudaGetDevice(&dev));
    RF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  }
  RF_TRY_RF(make_map(&mp.lt, s.LT, kLtCols, (uint64_t)R, kLtCols * 4, 128));
  RF_TRY_RF(make_map(&mp.linv, Linv, kPanel, kPanel, kPanel * 4, 128));
  RF_TRY_RF(make_map(&mp.uinvT, UinvT, kPanel, kPanel, kPanel * 4, 128));
  const int64_t lim = device_wait_limit();
  const uint64_t wait_ns = lim < 0 ? 1000000000ull : (uint64_t)lim;
  static const cudaError_t diag_attr[2] = {
      cudaFuncSetAttribute(k_lu_diag, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(kPanel * kDiagLd * sizeof(float))),
      cudaFuncSetAttribute(k_lu_diag_inv, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)((kPanel * kDiagLd + kPanel * 33) * sizeof(float)))};
  RF_CUDA_TRY(diag_attr[0]);
  RF_CUDA_TRY(diag_attr[1]);
  int nl = 0;
  auto base_args = [&]() {
    TcArgs t{};
    t.lmax = lmax;
    t.status = status;
    t.wait_ns = wait_ns;
    t.lt = s.LT;
    t.ldlt = kLtCols;
    return t;
  };
  // factor the panel at column k (width w): diagonal block, then L21 for rows
  // k + w .. R into the matrix and into LT columns lt_col .. lt_col + 128
  auto panel = [&](int64_t k, int w, int lt_col) -> int {
    k_lu_diag<<<1, 1024, kPanel * kDiagLd * sizeof(float), st>>>(s.LU, lda, k, w, lmax, status);
    RF_LAUNCH_CHECK();
    k_lu_diag_inv<<<8, 1024, (kPanel * kDiagLd + kPanel * 33) * sizeof(float), st>>>(
        s.LU, lda, k, w, Linv, UinvT, s.sinv + (k / kPanel) * 2 * kPanel * kPanel, status);
    RF_LAUNCH_CHECK();
    ++nl;
    ++nl;
    const int64_t m = R - k - w;
    if (m <= 0) return RF_OK;
    dim3 tg((unsigned)ceil_div(m, 32), (unsigned)(kPanel / 32));
    k_lu_to_rows<<<tg, dim3(32, 8), 0, st>>>(s.LU, lda, k + w, k, w, m, s.LT + (int64_t)(k + w) * kLtCols, lt_col);
    RF_LAUNCH_CHECK();
    ++nl;
    // L21 = A21 U11^-1: A operand LT rows k+w.., B operand U11^-T rows
    TcArgs t = base_args();
    t.C = s.LU + (k + w) + k * lda;
    t.ldc = lda;
    t.M = (int)m;
    t.N = w;
    t.a_x = lt_col;
    t.a_y = (int)(k + w);
    t.b_x = 0;
    t.b_y = 0;
    t.kblocks = kPanel / kTcBK;
    t.lt = s.LT + (int64_t)(k + w) * kLtCols + lt_col;
    ++nl;
    return launch_tc<128, kTcStoreL>(mp.lt, mp.uinvT, mp.mat_c128, t, st);
  };
  // U12 = L11^-1 A12 in place: rows k .. k+w of columns c0 .. R
  auto u12 = [&](int64_t k, int w, int64_t c0) -> int {
    TcArgs t = base_args();
    t.C = s.LU + k + c0 * lda;
    t.ldc = lda;
    t.M = w;
    t.N = (int)(R - c0);
    t.a_x = 0;
    t.a_y = 0;
    t.b_x = (int)k;
    t.b_y = (int)c0;
    t.kblocks = kPanel / kTcBK;
    ++nl;
    return launch_tc<256, kTcStore>(mp.linv, mp.mat_b256, mp.mat_c256, t, st);
  };
  // C -= LT[rows r0.., cols lt_col.. lt_col + K] * U[rows kk.. kk + K, cols c0..]
  auto up_args = [&](int64_t r0, int64_t r1, int64_t c0, int64_t c1, int64_t kk, int K, int lt_col) {
    UpArgs u{};
    u.M = (int)(r1 - r0);
    u.N = (int)(c1 - c0);
    u.a_x = lt_col;
    u.a_y = (int)r0;
    u.b_x = (int)kk;
    u.b_y = (int)c0;
    u.c_x = (int)r0;
    u.c_y = (int)c0;
    u.kblocks = K / kTcBK;
    u.status = status;
    u.wait_ns = wait_ns;
    ++nl;
    return u;
  };
  auto update = [&](int64_t r0, int64_t r1, int64_t c0, int64_t kk, int K, int lt_col) -> int {
    return launch_update<256>(mp.lt, mp.mat_b256, mp.mat_c32, up_args(r0, r1, c0, R, kk, K, lt_col), sms, st);
  };
  auto update_cols = [&](int64_t r0, int64_t c0, int64_t c1, int64_t kk, int K) -> int {
    return launch_update<128>(mp.lt, mp.mat_b128, mp.mat_c32, up_args(r0, R, c0, c1, kk, K, 0), sms, st);
  };
  // One pass: panels p = 0 .. kPassPanels-1 at columns k + 128 p, each brought
  // up to date by the pass's earlier panels (its columns below it, K = 128 p)
  // and factored; the rows of each panel right of it updated the same way and
  // turned into U12; then the trailing matrix by all the pass's panels at once
  // (K = 1024: C is read and written once per 1024 columns of the factorization;
  // N=4000: 706 ms with K = 256, 530 ms with 512, 497 ms with 1024).
  for (int64_t k = 0; k < R;) {
    int64_t end = k;
    for (int p = 0; p < kPassPanels && end < R; ++p) {
      const int64_t kk = end;
      const int w = (int)std::min<int64_t>(kPanel, R - kk);
      if (p > 0) RF_TRY_RF(update_cols(kk, kk, kk + w, k, kPanel * p));
      RF_TRY_RF(panel(kk, w, kPanel * p));
      end = kk + w;
      if (end >= R) break;
      if (p > 0) RF_TRY_RF(update(kk, kk + w, end, k, kPanel * p, 0));
      RF_TRY_RF(u12(kk, w, end));
    }
    if (end >= R) break;
    RF_TRY_RF(update(end, R, end, k, (int)(end - k), 0));
    k = end;
  }
  unsigned int h[2] = {0, 0};
  RF_CUDA_TRY(cudaMemcpyAsync(h, s.flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
  RF_CUDA_TRY(cudaStreamSynchronize(st));
  *launches += nl;
  if ((int)h[1] < 0) {
    set_last_error_str("lu: a bounded device-side wait timed out");
    return RF_E_TIMEOUT;
  }
  float lm;
  std::memcpy(&lm, &h[0], sizeof(float));
  if (max_l) *max_l = lm;
  *clean = h[1] == 0 && lm <= kStaticPivotLimit;
  return RF_OK;
}

}  // namespace rf
