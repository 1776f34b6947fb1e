// Structured operator A = I + C T: matvec, residual and velocities from the
// pair blocks that the assembly stores once per unordered fiber pair.
//
// The reference builds the dense R x R matrix (src/simulation.cu:331-399,
// fortran/assemble_matrix.incl) whose block (i,j) is C_i T^{ij} with C_i the
// per-force-index projector (D1 t t^T, or gamma_k (I - E_k t t^T)) and
// T^{ij}_{k,kj} a symmetric 3x3 block with T^{ji} = (T^{ij})^T.  A matvec is
//   y_{i,k} = x_{i,k} + C_i(k) z_{i,k},   z_{i,k} = sum_{j != i} sum_kj T^{ij}_{k,kj} x_{j,kj}
// and only the M^2 blocks of each unordered pair (150 values at M = 5) have to
// be read: 2.4 GB in FP16 at N = 4000 against 14.4 GB for dense FP32.
//
// Storage (written by k_assemble_numerical in structured mode): 16x16 fiber
// storage tiles over the upper triangle; inside, (16/TI)^2 assembly
// sub-tiles of TI x TI pairs.  FP32 blocks as [j][value][i] (values in
// s32_block order: the operator blocks lead), so a warp reads whole 32-byte
// sectors; 16-bit blocks as [j][i][record], one 16-byte aligned
// record of s16_record_words(M) words per pair (copied whole into shared
// memory and read there with 16-byte loads).  One CTA = one storage tile =
// 256 pairs.
// z is reduced deterministically: per-tile partial rows, fixed-order sums.
// The velocities reuse the FP32 blocks with P_0 / P_1 on the receiving side
// (fortran/update_velocities.incl:64-86: TFA0 and TFA1 are exactly those).
#include <type_traits>

#include "rf_common.cuh"
#include "rf_kernels.cuh"

namespace rf {

__device__ __forceinline__ int64_t struct_store_tiles_dev(int N) {
  const int64_t T16 = (N + kStoreTile - 1) / kStoreTile;
  return T16 * (T16 + 1) / 2;
}

__device__ __forceinline__ void tile_pair16(int64_t L, int& I, int& J) {
  int64_t j = (int64_t)((sqrt(8.0 * (double)L + 1.0) - 1.0) * 0.5);
  while ((j + 1) * (j + 2) / 2 <= L) ++j;
  while (j * (j + 1) / 2 > L) --j;
  J = (int)j;
  I = (int)(L - j * (j + 1) / 2);
}

template <typename T>
__device__ __forceinline__ float2 unpack16(uint32_t w);
template <>
__device__ __forceinline__ float2 unpack16<__half>(uint32_t w) {
  return __half22float2(*reinterpret_cast<const __half2*>(&w));
}
template <>
__device__ __forceinline__ float2 unpack16<__nv_bfloat16>(uint32_t w) {
  return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w));
}

// sym(T6) * v accumulated into acc
template <typename A>
__device__ __forceinline__ A fma_(A a, A b, A c) { return fma(a, b, c); }
template <>
__device__ __forceinline__ float fma_<float>(float a, float b, float c) { return fmaf(a, b, c); }

template <typename A>
__device__ __forceinline__ void sym_mv_acc(const A (&t)[6], const A* v, A* acc) {
  acc[0] = fma_(t[4], v[2], fma_(t[3], v[1], fma_(t[0], v[0], acc[0])));
  acc[1] = fma_(t[5], v[2], fma_(t[1], v[1], fma_(t[3], v[0], acc[1])));
  acc[2] = fma_(t[2], v[2], fma_(t[5], v[1], fma_(t[4], v[0], acc[2])));
}

// Thread -> pair of a storage tile.
template <int TI>
struct TileMap {
  static constexpr int SUB = kStoreTile / TI;
  int sub, jl, tl, a, b;
  __device__ TileMap(int t) {
    sub = t / (TI * TI);
    const int rem = t % (TI * TI);
    jl = rem / TI;
    tl = rem % TI;
    a = sub / SUB;
    b = sub % SUB;
  }
  __device__ int i16() const { return a * TI + tl; }
  __device__ int j16() const { return b * TI + jl; }
};

// z partials.  SMODE: 0 = FP32 storage (inner blocks of S32), 1 = FP16, 2 = BF16.
// XT: type of x; ACC: accumulation type.
// Shared memory: x of both tiles, then per-warp partial sums of z for the 16
// row fibers of each side (zero-filled; warps that do not touch a fiber leave
// zeros), summed in a fixed order at the end.

// Shared memory of the z kernel (8x8 assembly sub-tiles, 8 warps):
//  x rows of both tiles (padded: 20 floats / 17 doubles per fiber so the
//  rows that one warp reads start on distinct banks), then the per-warp
//  partial sums.  Warp w covers row fibers 8(w/4)..+8 on the i side (4
//  warps per row) and 4 fibers 8((w/2)%2) + 4(w%2)..+4 on the j side (2 warps
//  per row), so every slot is written once and nothing is zero-filled.
template <int M, int ACCB>
struct ZSmem {
  static constexpr int M3 = 3 * M;
  static constexpr int XS = ACCB == 4 ? ((M3 + 3) / 4 * 4 + 4) : (M3 + 2) | 1;   // x row stride
  static constexpr size_t kX = (size_t)2 * kStoreTile * XS * ACCB;
  static constexpr size_t kWI = (size_t)kStoreTile * 4 * M3 * ACCB;
  static constexpr size_t kWJ = (size_t)kStoreTile * 2 * M3 * ACCB;
  static constexpr size_t kBytes = kX + kWI + kWJ;
};

// The words of block row kI of one pair (M blocks of 6 values).
template <int M, int TI, int SMODE>
struct RowLoader {
  static constexpr int K1 = M + 1;
  static constexpr int NW = SMODE == 0 ? 6 * M : 3 * M;   // 4-byte words per row
  __device__ static void load(uint32_t (&w)[NW], const void* base, int kI) {
    if constexpr (SMODE == 0) {
      const float* p = static_cast<const float*>(base);
#pragma unroll
      for (int kJ = 0; kJ < M; ++kJ)
#pragma unroll
        for (int c = 0; c < 6; ++c)
          w[kJ * 6 + c] = __float_as_uint(__ldcs(p + ((kI * M + kJ) * 6 + c) * TI));
    } else {
      const uint32_t* p = static_cast<const uint32_t*>(base);   // this pair's record (L1 keeps its sectors)
#pragma unroll
      for (int q = 0; q < 3 * M; ++q) w[q] = __ldg(p + kI * 3 * M + q);
    }
  }
  template <typename ACC>
  __device__ static void values(const uint32_t (&w)[NW], int kJ, ACC (&tv)[6]) {
    if constexpr (SMODE == 0) {
#pragma unroll
      for (int c = 0; c < 6; ++c) tv[c] = (ACC)__uint_as_float(w[kJ * 6 + c]);
    } else {
      using H16 = typename std::conditional<SMODE == 1, __half, __nv_bfloat16>::type;
#pragma unroll
      for (int h = 0; h < 3; ++h) {
        const float2 f = unpack16<H16>(w[kJ * 3 + h]);
        tv[2 * h] = (ACC)f.x;
        tv[2 * h + 1] = (ACC)f.y;
      }
    }
  }
};

template <typename ACC>
__device__ __forceinline__ ACC shfl_xor(ACC v, int m) {
  return __shfl_xor_sync(0xffffffffu, v, m);
}

// x row of a fiber from shared memory (padded rows, 16-byte aligned)
template <typename ACC, int M3P>
__device__ __forceinline__ void load_xrow(const ACC* src, ACC (&dst)[M3P]) {
  if constexpr (sizeof(ACC) == 4) {
#pragma unroll
    for (int k = 0; k < M3P / 4; ++k) {
      const float4 v = reinterpret_cast<const float4*>(src)[k];
      dst[4 * k] = v.x; dst[4 * k + 1] = v.y; dst[4 * k + 2] = v.z; dst[4 * k + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < M3P / 2; ++k) {
      const double2 v = reinterpret_cast<const double2*>(src)[k];
      dst[2 * k] = v.x; dst[2 * k + 1] = v.y;
    }
  }
}

template <int M, int TI, int SMODE, typename XT, typename ACC, bool PREFETCH>
__global__ void __launch_bounds__(256, SMODE == 0 ? 2 : 3)
k_struct_z(int N, const float* __restrict__ S32, const uint32_t* __restrict__ S16, const XT* __restrict__ x,
           ACC* __restrict__ zpart, const int* __restrict__ skip) {
  static_assert(TI == 8, "structured operator kernels are specialised to 8x8 assembly sub-tiles (Q = 24)");
  if (skip != nullptr && *skip) return;
  constexpr int K1 = M + 1, M3 = 3 * M;
  constexpr int XS = ZSmem<M, sizeof(ACC)>::XS;
  constexpr int NQ32 = K1 * K1 * 6;
  constexpr int SUB = kStoreTile / TI;
  using RL = RowLoader<M, TI, SMODE>;
  extern __shared__ __align__(16) unsigned char zsm[];
  ACC (*sx)[kStoreTile][XS] = reinterpret_cast<ACC (*)[kStoreTile][XS]>(zsm);
  ACC (*swi)[4][M3] = reinterpret_cast<ACC (*)[4][M3]>(zsm + ZSmem<M, sizeof(ACC)>::kX);
  ACC (*swj)[2][M3] =
      reinterpret_cast<ACC (*)[2][M3]>(zsm + ZSmem<M, sizeof(ACC)>::kX + ZSmem<M, sizeof(ACC)>::kWI);
  int I16, J16;
  tile_pair16(blockIdx.x, I16, J16);
  const bool diag = I16 == J16;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int64_t R = (int64_t)M3 * N;
  const TileMap<TI> mp(t);
  const int i = I16 * kStoreTile + mp.i16(), j = J16 * kStoreTile + mp.j16();
  const bool active = i < j && j < N;
  const int64_t rec = ((int64_t)blockIdx.x * SUB * SUB + mp.sub) * TI + mp.jl;
  const void* base = SMODE == 0 ? (const void*)(S32 + rec * (int64_t)(NQ32 * TI) + mp.tl)
                                : (const void*)(S16 + (rec * TI + mp.tl) * (int64_t)s16_record_words(M));
  // first block row in flight before the x prologue
  uint32_t wa[RL::NW], wb[RL::NW];
  if (active) RL::load(wa, base, 0);
  for (int k = t; k < 2 * kStoreTile * M3; k += blockDim.x) {
    const int side = k / (kStoreTile * M3), rem = k % (kStoreTile * M3);
    const int f = (side == 0 ? I16 : J16) * kStoreTile + rem / M3, v = rem % M3;
    sx[side][rem / M3][v] = f < N ? (ACC)x[(int64_t)f * M3 + v] : (ACC)0;
  }
  __syncthreads();
  ACC zj[M3];
#pragma unroll
  for (int k = 0; k < M3; ++k) zj[k] = (ACC)0;
  // x_j in registers for FP32 accumulation; read from shared memory for FP64
  constexpr int M3P = (M3 + 3) / 4 * 4;
  ACC xjr[sizeof(ACC) == 4 ? M3P : 1];
  if constexpr (sizeof(ACC) == 4) load_xrow<ACC, M3P>(sx[1][mp.j16()], xjr);
  const ACC* xjs = sx[1][mp.j16()];
  const ACC* xi = sx[0][mp.i16()];
  const bool owner_i = lane < TI;           // lanes 0..7 hold the i-side warp sums
  const int slot_i = warp & 3;
  auto row = [&](const uint32_t (&w)[RL::NW], int kI) {
    ACC ziv[3] = {(ACC)0, (ACC)0, (ACC)0};
    const ACC xik[3] = {xi[3 * kI], xi[3 * kI + 1], xi[3 * kI + 2]};
    if (active) {
#pragma unroll
      for (int kJ = 0; kJ < M; ++kJ) {
        ACC tv[6];
        RL::values(w, kJ, tv);
        if constexpr (sizeof(ACC) == 4) sym_mv_acc(tv, xjr + 3 * kJ, ziv);
        else sym_mv_acc(tv, xjs + 3 * kJ, ziv);
        sym_mv_acc(tv, xik, zj + 3 * kJ);
      }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      ACC v = ziv[a];
      v += shfl_xor(v, 8);
      v += shfl_xor(v, 16);
      if (owner_i) swi[mp.i16()][slot_i][3 * kI + a] = v;
    }
  };
  // ping-pong over the block rows: the next row's loads overlap this row's math
#pragma unroll 1
  for (int kI = 0; kI < M; kI += 2) {
    if (PREFETCH && active && kI + 1 < M) RL::load(wb, base, kI + 1);
    row(wa, kI);
    if (kI + 1 < M) {
      if (!PREFETCH && active) RL::load(wb, base, kI + 1);
      if (PREFETCH && active && kI + 2 < M) RL::load(wa, base, kI + 2);
      row(wb, kI + 1);
      if (!PREFETCH && active && kI + 2 < M) RL::load(wa, base, kI + 2);
    }
  }
  // z_j over the row lanes (lane bits 0..2)
#pragma unroll
  for (int k = 0; k < M3; ++k) {
    ACC b = zj[k];
    b += shfl_xor(b, 1);
    b += shfl_xor(b, 2);
    b += shfl_xor(b, 4);
    zj[k] = b;
  }
  if ((lane & (TI - 1)) == 0) {
#pragma unroll
    for (int k = 0; k < M3; ++k) swj[mp.j16()][warp >> 2][k] = zj[k];
  }
  __syncthreads();
  for (int task = t; task < kStoreTile * M3; task += blockDim.x) {
    const int rf = task / M3, rv = task % M3;
    const ACC si = ((swi[rf][0][rv] + swi[rf][1][rv]) + swi[rf][2][rv]) + swi[rf][3][rv];
    const ACC sj = swj[rf][0][rv] + swj[rf][1][rv];
    const int fi = I16 * kStoreTile + rf, fj = J16 * kStoreTile + rf;
    if (diag) {
      if (fi < N) zpart[(int64_t)I16 * R + (int64_t)fi * M3 + rv] = si + sj;
    } else {
      if (fi < N) zpart[(int64_t)J16 * R + (int64_t)fi * M3 + rv] = si;
      if (fj < N) zpart[(int64_t)I16 * R + (int64_t)fj * M3 + rv] = sj;
    }
  }
}

// ---------------------------------------------------------------------------
// 16-bit matvec with whole tiles staged through shared memory by TMA bulk
// copies (cp.async.bulk + mbarrier transaction counts): persistent CTAs,
// one per SM, two tiles in flight per CTA (~150 KB per SM), so the copy
// engine keeps HBM busy while the threads compute the previous tile.
// Every mbarrier wait is bounded: on timeout the CTA records the fault in
// *err, waits (bounded) for its own copies in flight, and returns.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait; returns false on timeout
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t polls = (1u << 24)) {
  for (uint32_t it = 0; it < polls; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

template <int M>
struct BulkShape {
  static constexpr int M3 = 3 * M;
  static constexpr int NW = s16_record_words(M);                                   // words per pair record
  static constexpr uint32_t kTileBytes = 4u * kStoreTile * kStoreTile * NW;       // 256 records
  static constexpr int M3P = (M3 + 3) / 4 * 4;
  static constexpr int XS = M3P + 4;                                              // x row stride (floats)
  // the M^2 blocks of a pair are split between two threads at a 16-byte
  // boundary of the record: blocks [0, B0) and [B0, M^2), B0 a multiple of 4
  static constexpr int B0 = 4 * ((M * M + 4) / 8);
  static constexpr int ZW = 12;                                                   // z_i values per half (<= 3 rows + pad)
  static constexpr size_t kX = (size_t)2 * 2 * kStoreTile * XS * 4;              // double-buffered x rows
  static constexpr size_t kWI = (size_t)2 * kStoreTile * 4 * ZW * 4;
  static constexpr size_t kWJ = (size_t)kStoreTile * 4 * 16 * 4;
  static constexpr size_t kBytes = 2 * (size_t)kTileBytes + kX + kWI + kWJ;
  static constexpr int kThreads = 512;                                            // two threads per pair
  static_assert(M3 <= 16, "z_j is reduced as 16 values");
};

template <int M, int H>
struct BulkHalf {
  static constexpr int BB = H ? BulkShape<M>::B0 : 0, BE = H ? M * M : BulkShape<M>::B0;   // blocks [BB, BE)
  static constexpr int NBLK = BE - BB;
  static constexpr int R0 = NBLK > 0 ? BB / M : 0;
  static constexpr int NR = NBLK > 0 ? (BE - 1) / M - R0 + 1 : 0;                // block rows touched
  static constexpr int NU = (3 * NBLK + 3) / 4;                                  // 16-byte loads
  static_assert(3 * NR <= BulkShape<M>::ZW, "at most three block rows per half");
};

// v[16] summed over the 8 lanes that differ in lane bits 0..2; lane l keeps
// the sums of v[2l] and v[2l+1] (three halving exchanges instead of 16 x 3).
template <typename T>
__device__ __forceinline__ void reduce_scatter8(const T (&v)[16], int lane, T& y0, T& y1) {
  const bool b2 = lane & 4, b1 = lane & 2, b0 = lane & 1;
  T u[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const T send = b2 ? v[k] : v[k + 8], keep = b2 ? v[k + 8] : v[k];
    u[k] = keep + shfl_xor(send, 4);
  }
  T w[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const T send = b1 ? u[k] : u[k + 4], keep = b1 ? u[k + 4] : u[k];
    w[k] = keep + shfl_xor(send, 2);
  }
  T y[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const T send = b0 ? w[k] : w[k + 2], keep = b0 ? w[k + 2] : w[k];
    y[k] = keep + shfl_xor(send, 1);
  }
  y0 = y[0];
  y1 = y[1];
}

// v[12] summed over the 4 lanes that differ in lane bits 3, 4 (two halving
// exchanges); lane group g = lane / 8 stores the sums of v[3g..3g+2] to dst.
template <typename T>
__device__ __forceinline__ void reduce_scatter4x3(const T (&v)[12], int lane, T* dst) {
  const bool b4 = lane & 16, b3 = lane & 8;
  T u[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const T send = b4 ? v[k] : v[k + 6], keep = b4 ? v[k + 6] : v[k];
    u[k] = keep + shfl_xor(send, 16);
  }
  const int g = lane >> 3;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const T send = b3 ? u[k] : u[k + 3], keep = b3 ? u[k + 3] : u[k];
    dst[3 * g + k] = keep + shfl_xor(send, 8);
  }
}

// The blocks of half H of one pair: z_i rows of this half reduced over the
// warp's 4 j lanes into swi (lane group g = lane / 8 stores values 3g..3g+2,
// i.e. row R0 + g), z_j (16 values, this pair's contribution) returned for
// the caller's reduction.
template <int M, int SMODE, int H>
__device__ __forceinline__ void z16_half(const uint32_t* rec, const float* xjs, const float* xis, bool active,
                                         float (&zj)[16], float* swi_slot, int lane) {
  using HF = BulkHalf<M, H>;
  using H16 = typename std::conditional<SMODE == 1, __half, __nv_bfloat16>::type;
  constexpr int M3P = BulkShape<M>::M3P;
  float zi[12];
#pragma unroll
  for (int q = 0; q < 12; ++q) zi[q] = 0.f;
  if constexpr (HF::NBLK > 0) {
    if (active) {
      uint32_t w[4 * HF::NU];
      const uint4* p = reinterpret_cast<const uint4*>(rec + 3 * HF::BB);
#pragma unroll
      for (int u = 0; u < HF::NU; ++u) {
        const uint4 v = p[u];
        w[4 * u] = v.x; w[4 * u + 1] = v.y; w[4 * u + 2] = v.z; w[4 * u + 3] = v.w;
      }
      float xj[M3P], xi[12];
      load_xrow<float, M3P>(xjs, xj);
#pragma unroll
      for (int q = 0; q < 3 * HF::NR; ++q) xi[q] = xis[3 * HF::R0 + q];
#pragma unroll
      for (int b = 0; b < HF::NBLK; ++b) {
        const int blk = HF::BB + b, kI = blk / M, kJ = blk % M;
        float tv[6];
#pragma unroll
        for (int h = 0; h < 3; ++h) {
          const float2 f = unpack16<H16>(w[3 * b + h]);
          tv[2 * h] = f.x;
          tv[2 * h + 1] = f.y;
        }
        sym_mv_acc(tv, xj + 3 * kJ, zi + 3 * (kI - HF::R0));
        sym_mv_acc(tv, xi + 3 * (kI - HF::R0), zj + 3 * kJ);
      }
    }
  }
  // z_i (12 values, rows R0.. padded) summed over the 4 j lanes of the warp
  reduce_scatter4x3(zi, lane, swi_slot);
}

// (I, J) of storage tile L (L = J (J + 1) / 2 + I, I <= J) without FP64
__device__ __forceinline__ void tile_pair16f(int64_t L, int& I, int& J) {
  int64_t j = (int64_t)((sqrtf(8.f * (float)L + 1.f) - 1.f) * 0.5f);
  while ((j + 1) * (j + 2) / 2 <= L) ++j;
  while (j * (j + 1) / 2 > L) --j;
  J = (int)j;
  I = (int)(L - j * (j + 1) / 2);
}

// Thread t: half h = t / 256 takes blocks [BB, BE) of pair tt = t % 256
// (TileMap).  z_i of a block row comes from one or both halves (4 warp
// slots each), z_j from both halves (2 warp slots each).  Partial rows go to
// zpart slot J (i side of tile (I, J)) and I (j side); the j side of a
// diagonal tile goes to slot ceil(N/16), so every slot has one writer.
template <int M, int SMODE>
__global__ void __launch_bounds__(512, 1)
k_struct_z16_bulk(int N, const uint32_t* __restrict__ S16, const float* __restrict__ x, float* __restrict__ zpart,
                  const int* __restrict__ skip, int* __restrict__ err, uint32_t wait_polls) {
  constexpr int TI = 8, M3 = 3 * M;
  using B = BulkShape<M>;
  using H0 = BulkHalf<M, 0>;
  using H1 = BulkHalf<M, 1>;
  constexpr int XS = B::XS, ZW = B::ZW;
  if (skip != nullptr && *skip) return;
  extern __shared__ __align__(128) unsigned char bsm[];
  auto stage = [&](int s) { return reinterpret_cast<uint32_t*>(bsm + (size_t)s * B::kTileBytes); };
  float (*sx)[2][kStoreTile][XS] = reinterpret_cast<float (*)[2][kStoreTile][XS]>(bsm + 2 * B::kTileBytes);
  float (*swi)[kStoreTile][4][ZW] = reinterpret_cast<float (*)[kStoreTile][4][ZW]>(bsm + 2 * B::kTileBytes + B::kX);
  float (*swj)[4][16] = reinterpret_cast<float (*)[4][16]>(bsm + 2 * B::kTileBytes + B::kX + B::kWI);
  __shared__ __align__(8) uint64_t bar[2];
  const int64_t ntiles = struct_store_tiles_dev(N);
  const int t = threadIdx.x, lane = t & 31;
  const int half = t >> 8, tt = t & 255, hw = tt >> 5;   // warp index within the half
  const int64_t R = (int64_t)M3 * N;
  const TileMap<TI> mp(tt);
  if (t == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  auto issue = [&](int64_t L, int s) {
    mbar_expect_tx(&bar[s], B::kTileBytes);
    bulk_g2s(stage(s), S16 + L * (int64_t)(B::kTileBytes / 4), B::kTileBytes, &bar[s]);
  };
  // x rows of a tile: thread t < 2*16*M3 owns one value
  auto xval = [&](bool valid, int I16, int J16) -> float {
    if (t >= 2 * kStoreTile * M3 || !valid) return 0.f;
    const int side = t / (kStoreTile * M3), rem = t % (kStoreTile * M3);
    const int f = (side == 0 ? I16 : J16) * kStoreTile + rem / M3;
    return f < N ? x[(int64_t)f * M3 + rem % M3] : 0.f;
  };
  auto xstore = [&](int buf, float v) {
    if (t < 2 * kStoreTile * M3) {
      const int side = t / (kStoreTile * M3), rem = t % (kStoreTile * M3);
      sx[buf][side][rem / M3][rem % M3] = v;
    }
  };
  int cI = 0, cJ = 0;
  tile_pair16f(blockIdx.x, cI, cJ);
  xstore(0, xval(true, cI, cJ));
  __syncthreads();
  if (t == 0) {
    for (int s = 0; s < 2; ++s) {
      const int64_t L = blockIdx.x + (int64_t)s * gridDim.x;
      if (L < ntiles) issue(L, s);
    }
  }
  bool failed = false;
  int k = 0;
  for (int64_t L = blockIdx.x; L < ntiles; L += gridDim.x, ++k) {
    const int s = k & 1, xb = k & 1;
    const uint32_t parity = (k >> 1) & 1;
    const int I16 = cI, J16 = cJ;
    const bool diag = I16 == J16;
    const bool more = L + gridDim.x < ntiles;
    if (more) tile_pair16f(L + gridDim.x, cI, cJ);
    const float xnext = xval(more, cI, cJ);   // in flight while this tile is computed
    const bool ok_wait = mbar_wait_bounded(&bar[s], parity, wait_polls);
    if (__syncthreads_or(!ok_wait)) {
      failed = true;
      break;
    }
    const int i = I16 * kStoreTile + mp.i16(), j = J16 * kStoreTile + mp.j16();
    const bool active = i < j && j < N;
    const uint32_t* rec = stage(s) + ((mp.sub * TI + mp.jl) * TI + mp.tl) * B::NW;
    const float* xjs = sx[xb][1][mp.j16()];
    const float* xis = sx[xb][0][mp.i16()];
    float zj[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) zj[q] = 0.f;
    if (half == 0) z16_half<M, SMODE, 0>(rec, xjs, xis, active, zj, swi[0][mp.i16()][hw & 3], lane);
    else z16_half<M, SMODE, 1>(rec, xjs, xis, active, zj, swi[1][mp.i16()][hw & 3], lane);
    // z_j over the 8 i lanes (lane bits 0..2): lane tl keeps values 2 tl, 2 tl + 1
    float2 zs;
    reduce_scatter8(zj, lane, zs.x, zs.y);
    *reinterpret_cast<float2*>(&swj[mp.j16()][2 * half + (hw >> 2)][2 * (lane & 7)]) = zs;
    xstore(xb ^ 1, xnext);
    __syncthreads();
    // stage s is free again: refill it with the tile two steps ahead
    if (t == 0) {
      const int64_t Ln = L + 2 * (int64_t)gridDim.x;
      if (Ln < ntiles) issue(Ln, s);
    }
    // half 0 writes the i side, half 1 the j side (fixed-order slot sums)
    if (tt < kStoreTile * M3) {
      const int rf = tt / M3, rv = tt % M3;
      if (half == 0) {
        const int kI = rv / 3;
        const bool in0 = H0::NR > 0 && kI >= H0::R0 && kI < H0::R0 + H0::NR;
        const bool in1 = H1::NR > 0 && kI >= H1::R0 && kI < H1::R0 + H1::NR;
        const int q0 = in0 ? rv - 3 * H0::R0 : 0, q1 = in1 ? rv - 3 * H1::R0 : 0;
        const float s0 = ((swi[0][rf][0][q0] + swi[0][rf][1][q0]) + swi[0][rf][2][q0]) + swi[0][rf][3][q0];
        const float s1 = ((swi[1][rf][0][q1] + swi[1][rf][1][q1]) + swi[1][rf][2][q1]) + swi[1][rf][3][q1];
        const float si = in0 ? (in1 ? s0 + s1 : s0) : s1;
        const int fi = I16 * kStoreTile + rf;
        if (fi < N) zpart[(int64_t)J16 * R + (int64_t)fi * M3 + rv] = si;
      } else {
        const float sj = ((swj[rf][0][rv] + swj[rf][1][rv]) + swj[rf][2][rv]) + swj[rf][3][rv];
        const int fj = J16 * kStoreTile + rf;
        const int64_t slot = diag ? (int64_t)((N + kStoreTile - 1) / kStoreTile) : (int64_t)I16;
        if (fj < N) zpart[slot * R + (int64_t)fj * M3 + rv] = sj;
      }
    }
  }
  if (failed) {
    if (t == 0) {
      atomicExch(err, 1);
      // drain: wait (bounded) for the copies this CTA still has in flight
      for (int kk = k; kk < k + 2; ++kk) {
        const int64_t L = blockIdx.x + (int64_t)kk * gridDim.x;
        if (L < ntiles) (void)mbar_wait_bounded(&bar[kk & 1], (kk >> 1) & 1);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// A x with the FP32 blocks, x and accumulation in FP64 (the refinement
// residual), staged by TMA bulk copies.  A storage tile comes in as two
// halves (assembly sub-tile row a = 0, 1: 16 records of 8 pairs), and of
// every record only its M^2 operator blocks, which lead the record
// (s32_block order: 6 M^2 values x 8 pairs, one copy per record; the P_0 row
// and column stay in HBM).  Persistent CTAs, one per SM; while one half is
// computed the other is in flight.
// ---------------------------------------------------------------------------
template <int M>
struct R64Shape {
  static constexpr int M3 = 3 * M, K1 = M + 1;
  static constexpr int NQ32 = K1 * K1 * 6;                 // FP32 values per pair in storage
  static constexpr int CHF = 6 * M * 8;                    // floats of one block row of a record
  static constexpr uint32_t kRecBytes = M * CHF * 4;       // operator blocks of one record
  static constexpr int RECF = M * CHF + 8;                 // record stride in shared memory: 4
                                                           // consecutive records start on distinct banks
  static constexpr int kRecs = 16;                         // records per half tile
  static constexpr uint32_t kStageBytes = kRecs * RECF * 4;
  static constexpr uint32_t kTxBytes = kRecs * kRecBytes;
  static constexpr int XS = 18;                            // x row stride (doubles, 16-byte aligned rows)
  static constexpr size_t kX = (size_t)2 * 2 * kStoreTile * XS * 8;     // [buf][side][16][XS]
  static constexpr size_t kWI = (size_t)2 * 2 * 8 * 4 * 12 * 8;        // [h][split][8][warp][12]
  static constexpr size_t kWJ = (size_t)kStoreTile * 4 * 16 * 8;        // [16][h*2+split][16]
  static constexpr size_t kBytes = 2 * (size_t)kStageBytes + kX + kWI + kWJ;
  static constexpr int kThreads = 256;                     // two threads per pair of a half tile
  static_assert(M3 <= 15, "z_j is reduced as 16 values");
  static_assert(kRecs == 2 * (kThreads / 32), "lanes 0 and 1 of every warp copy one record each");
};

// Blocks [BB, BE) of split S (the 16-bit kernel's split) of one pair:
// rec points at this pair's column (tl) of its record in shared memory.
template <int M, int S>
__device__ __forceinline__ void r64_half(const float* rec, const double* xjs, const double* xis, bool active,
                                         double (&zj)[16], double* swi_slot, int lane) {
  using HF = BulkHalf<M, S>;
  using RS = R64Shape<M>;
  double zi[12];
#pragma unroll
  for (int q = 0; q < 12; ++q) zi[q] = 0.0;
  if constexpr (HF::NBLK > 0) {
    if (active) {
      double xj[16], xi[12];
      load_xrow<double, 16>(xjs, xj);
#pragma unroll
      for (int q = 0; q < 3 * HF::NR; ++q) xi[q] = xis[3 * HF::R0 + q];
#pragma unroll
      for (int b = 0; b < HF::NBLK; ++b) {
        const int blk = HF::BB + b, kI = blk / M, kJ = blk % M;
        double tv[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) tv[c] = f2d(rec[kI * RS::CHF + (kJ * 6 + c) * 8]);
        sym_mv_acc(tv, xj + 3 * kJ, zi + 3 * (kI - HF::R0));
        sym_mv_acc(tv, xi + 3 * (kI - HF::R0), zj + 3 * kJ);
      }
    }
  }
  reduce_scatter4x3(zi, lane, swi_slot);
}

template <int M>
__global__ void __launch_bounds__(256, 1)
k_struct_r64_bulk(int N, const float* __restrict__ S32, const double* __restrict__ x, double* __restrict__ zpart,
                  const int* __restrict__ skip, int* __restrict__ err, uint32_t wait_polls) {
  constexpr int M3 = 3 * M;
  using RS = R64Shape<M>;
  using H0 = BulkHalf<M, 0>;
  using H1 = BulkHalf<M, 1>;
  constexpr int XS = RS::XS;
  if (skip != nullptr && *skip) return;
  extern __shared__ __align__(128) unsigned char rsm[];
  auto stage = [&](int s) { return reinterpret_cast<float*>(rsm + (size_t)s * RS::kStageBytes); };
  double (*sx)[2][kStoreTile][XS] = reinterpret_cast<double (*)[2][kStoreTile][XS]>(rsm + 2 * RS::kStageBytes);
  double (*swi)[2][8][4][12] =
      reinterpret_cast<double (*)[2][8][4][12]>(rsm + 2 * RS::kStageBytes + RS::kX);
  double (*swj)[4][16] = reinterpret_cast<double (*)[4][16]>(rsm + 2 * RS::kStageBytes + RS::kX + RS::kWI);
  __shared__ __align__(8) uint64_t bar[2];
  const int64_t ntiles = struct_store_tiles_dev(N);
  const int64_t T16 = (N + kStoreTile - 1) / kStoreTile;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int split = t >> 7, p = t & 127, wq = (t >> 5) & 3;
  const int subj = p >> 6, jl = (p >> 3) & 7, tl = p & 7;   // j side 8-group, j and i within it
  const int j16 = subj * 8 + jl;
  const int64_t R = (int64_t)M3 * N;
  if (t == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    mbar_expect_tx(&bar[0], RS::kTxBytes);
    mbar_expect_tx(&bar[1], RS::kTxBytes);
  }
  // half h of tile L into stage h: record r = 2 warp + lane (lanes 0, 1 of
  // every warp), after thread 0 registered the bytes (expect) and a barrier
  auto expect = [&](int h) {
    if (t == 0) mbar_expect_tx(&bar[h], RS::kTxBytes);
  };
  auto issue = [&](int64_t L, int h) {
    if (lane < 2) {
      const int r = 2 * warp + lane;
      const float* src = S32 + (L * 32 + 16 * h + r) * (int64_t)RS::NQ32 * 8;
      bulk_g2s(stage(h) + r * RS::RECF, src, RS::kRecBytes, &bar[h]);
    }
  };
  // x rows of a tile: element e < 2*16*M3 (thread t owns e = t and t + 256)
  auto xval = [&](int e, bool valid, int I16, int J16) -> double {
    if (e >= 2 * kStoreTile * M3 || !valid) return 0.0;
    const int side = e / (kStoreTile * M3), rem = e % (kStoreTile * M3);
    const int f = (side == 0 ? I16 : J16) * kStoreTile + rem / M3;
    return f < N ? x[(int64_t)f * M3 + rem % M3] : 0.0;
  };
  auto xstore = [&](int buf, int e, double v) {
    if (e < 2 * kStoreTile * M3) {
      const int side = e / (kStoreTile * M3), rem = e % (kStoreTile * M3);
      sx[buf][side][rem / M3][rem % M3] = v;
    }
  };
  int cI = 0, cJ = 0;
  tile_pair16f(blockIdx.x, cI, cJ);
  xstore(0, t, xval(t, true, cI, cJ));
  xstore(0, t + 256, xval(t + 256, true, cI, cJ));
  __syncthreads();
  issue(blockIdx.x, 0);
  issue(blockIdx.x, 1);
  bool failed = false, fail_more = false;
  int k = 0, fail_h = 0;
  for (int64_t L = blockIdx.x; L < ntiles; L += gridDim.x, ++k) {
    const int xb = k & 1;
    const uint32_t parity = k & 1;
    const int I16 = cI, J16 = cJ;
    const bool diag = I16 == J16;
    const bool more = L + gridDim.x < ntiles;
    if (more) tile_pair16f(L + gridDim.x, cI, cJ);
    const double xn0 = xval(t, more, cI, cJ), xn1 = xval(t + 256, more, cI, cJ);
    const int j = J16 * kStoreTile + j16;
    const double* xjs = sx[xb][1][j16];
    for (int h = 0; h < 2; ++h) {
      const bool ok_wait = mbar_wait_bounded(&bar[h], parity, wait_polls);
      if (__syncthreads_or(!ok_wait)) {
        failed = true;
        fail_h = h;
        fail_more = more;
        break;
      }
      const int i = I16 * kStoreTile + 8 * h + tl;
      const bool active = i < j && j < N;
      const float* rec = stage(h) + (subj * 8 + jl) * RS::RECF + tl;
      const double* xis = sx[xb][0][8 * h + tl];
      double zj[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) zj[q] = 0.0;
      if (split == 0) r64_half<M, 0>(rec, xjs, xis, active, zj, swi[h][0][tl][wq], lane);
      else r64_half<M, 1>(rec, xjs, xis, active, zj, swi[h][1][tl][wq], lane);
      double y0, y1;
      reduce_scatter8(zj, lane, y0, y1);
      swj[j16][2 * h + split][2 * tl] = y0;
      swj[j16][2 * h + split][2 * tl + 1] = y1;
      if (h == 1) {
        xstore(xb ^ 1, t, xn0);
        xstore(xb ^ 1, t + 256, xn1);
      }
      if (more) expect(h);
      __syncthreads();
      // stage h is free again: the same half of the next tile
      if (more) issue(L + gridDim.x, h);
    }
    if (failed) break;
    // partial rows of this tile: i side to slot J, j side to slot I (diagonal: slot T16)
    for (int task = t; task < 2 * kStoreTile * M3; task += blockDim.x) {
      const int side = task / (kStoreTile * M3), rem = task % (kStoreTile * M3);
      const int rf = rem / M3, rv = rem % M3;
      if (side == 0) {
        const int h = rf >> 3, il = rf & 7, kI = rv / 3;
        const bool in0 = H0::NR > 0 && kI >= H0::R0 && kI < H0::R0 + H0::NR;
        const bool in1 = H1::NR > 0 && kI >= H1::R0 && kI < H1::R0 + H1::NR;
        const int q0 = in0 ? rv - 3 * H0::R0 : 0, q1 = in1 ? rv - 3 * H1::R0 : 0;
        const double s0 = ((swi[h][0][il][0][q0] + swi[h][0][il][1][q0]) + swi[h][0][il][2][q0]) + swi[h][0][il][3][q0];
        const double s1 = ((swi[h][1][il][0][q1] + swi[h][1][il][1][q1]) + swi[h][1][il][2][q1]) + swi[h][1][il][3][q1];
        const double si = in0 ? (in1 ? s0 + s1 : s0) : s1;
        const int fi = I16 * kStoreTile + rf;
        if (fi < N) zpart[(int64_t)J16 * R + (int64_t)fi * M3 + rv] = si;
      } else {
        const double sj = ((swj[rf][0][rv] + swj[rf][1][rv]) + swj[rf][2][rv]) + swj[rf][3][rv];
        const int fj = J16 * kStoreTile + rf;
        if (fj < N) zpart[(diag ? T16 : (int64_t)I16) * R + (int64_t)fj * M3 + rv] = sj;
      }
    }
  }
  if (failed) {
    if (t == 0) {
      atomicExch(err, 1);
      // drain (bounded): the copies this CTA still has in flight
      const uint32_t ph = k & 1;
      (void)mbar_wait_bounded(&bar[fail_h], ph);                       // the half that timed out
      if (fail_h == 0) (void)mbar_wait_bounded(&bar[1], ph);           // this tile's second half
      else if (fail_more) (void)mbar_wait_bounded(&bar[0], ph ^ 1u);   // the next tile's first half
    }
    __syncthreads();
  }
}

// zsum[r] = sum_p zpart[p][r] (fixed order within each of 4 p-groups, then
// the 4 groups in order).  256 threads = 64 consecutive rows x 4 groups, the
// p loop unrolled so that 8 loads per thread are in flight.
template <typename ACC>
__global__ void __launch_bounds__(256)
k_sum_parts(const ACC* part, int nparts, int64_t R, ACC* out, const int* __restrict__ skip) {
  // out may be the last partial row (read by this block before it is written)
  if (skip != nullptr && *skip) return;
  __shared__ ACC red[4][64];
  const int rr = threadIdx.x & 63, g = threadIdx.x >> 6;
  const int64_t r = (int64_t)blockIdx.x * 64 + rr;
  ACC s = (ACC)0;
  if (r < R) {
    int p = g;
    for (; p + 28 < nparts; p += 32) {
      ACC v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = part[(int64_t)(p + 4 * u) * R + r];
#pragma unroll
      for (int u = 0; u < 8; ++u) s += v[u];
    }
    for (; p < nparts; p += 4) s += part[(int64_t)p * R + r];
  }
  red[g][rr] = s;
  __syncthreads();
  if (g == 0 && r < R) out[r] = ((red[0][rr] + red[1][rr]) + red[2][rr]) + red[3][rr];
}

// y = x + C z (z = sum of partials, added in ACC), or r = b - (x + C z).  One
// thread per (fiber, k).
template <typename XT, typename ACC, bool RESIDUAL, typename ZT = ACC>
__global__ void k_struct_finalize(const Tables tab, int N, const float4* __restrict__ ori, const XT* __restrict__ x,
                                  const ZT* __restrict__ zpart, int nparts, const float* __restrict__ b,
                                  float* __restrict__ out, const int* __restrict__ skip) {
  if (skip != nullptr && *skip) return;
  const int M = tab.M;
  const int64_t R = (int64_t)3 * M * N;
  const int64_t n = (int64_t)N * M;
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(u / M), k = (int)(u % M);
    const int64_t r0 = (int64_t)i * 3 * M + 3 * k;
    ACC z[3] = {0, 0, 0};
    for (int p = 0; p < nparts; ++p) {
      const ZT* s = zpart + (int64_t)p * R + r0;
      z[0] += (ACC)s[0]; z[1] += (ACC)s[1]; z[2] += (ACC)s[2];
    }
    const float4 t = ori[i];
    const ACC t3[3] = {(ACC)t.x, (ACC)t.y, (ACC)t.z};
    const ACC tz = t3[0] * z[0] + t3[1] * z[1] + t3[2] * z[2];
    const ACC coef = (ACC)tab.gamma[k], E = (ACC)tab.eigen[k];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const ACC cz = k == 0 ? coef * t3[a] * tz : coef * (z[a] - E * t3[a] * tz);
      const ACC y = (ACC)x[r0 + a] + cz;
      out[r0 + a] = RESIDUAL ? (float)((ACC)b[r0 + a] - y) : (float)y;
    }
  }
}

// Velocity partials from the FP32 blocks:
//   u_i += sum_kJ T^{ij}[P0][kJ+1] x_{j,kJ},  w_i += sum_kJ T^{ij}[P1][kJ+1] x_{j,kJ}
//   u_j += sum_kI T^{ij}[kI+1][P0] x_{i,kI},  w_j += sum_kI T^{ij}[kI+1][P1] x_{i,kI}
// (storage tile L of one suspension: the body of k_struct_velocity and of the
// packed velocities)
template <int M, int TI>
__device__ __forceinline__ void struct_velocity_tile(int N, const float* __restrict__ S32,
                                                     const float* __restrict__ x, float* __restrict__ vpart,
                                                     unsigned L) {
  constexpr int K1 = M + 1, M3 = 3 * M;
  constexpr int NQ32 = K1 * K1 * 6;
  constexpr int SUB = kStoreTile / TI;
  __shared__ float sx[2][kStoreTile][M3];
  __shared__ float sz[2][kStoreTile][kStoreTile][7];
  int I16, J16;
  tile_pair16(L, I16, J16);
  const bool diag = I16 == J16;
  const int t = threadIdx.x;
  for (int k = t; k < 2 * kStoreTile * M3; k += blockDim.x) {
    const int side = k / (kStoreTile * M3), rem = k % (kStoreTile * M3);
    const int f = (side == 0 ? I16 : J16) * kStoreTile + rem / M3;
    sx[side][rem / M3][rem % M3] = f < N ? x[(int64_t)f * M3 + rem % M3] : 0.f;
  }
  __syncthreads();
  const TileMap<TI> mp(t);
  const int i = I16 * kStoreTile + mp.i16(), j = J16 * kStoreTile + mp.j16();
  float vi[6] = {0, 0, 0, 0, 0, 0}, vj[6] = {0, 0, 0, 0, 0, 0};
  if (i < j && j < N) {
    const int64_t rec = ((int64_t)L * SUB * SUB + mp.sub) * TI + mp.jl;
    const float* p = S32 + rec * (int64_t)(NQ32 * TI) + mp.tl;
    const float* xi = sx[0][mp.i16()];
    const float* xj = sx[1][mp.j16()];
#pragma unroll
    for (int kk = 0; kk < M; ++kk) {
      float tv[6];
      // receiving side i: rows P0 and P1 against x_j
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int q0 = s32_block(M, r, kk + 1) * 6;
#pragma unroll
        for (int c = 0; c < 6; ++c) tv[c] = __ldcs(p + (q0 + c) * TI);
        sym_mv_acc(tv, xj + 3 * kk, vi + 3 * r);
      }
      // receiving side j: columns P0 and P1 against x_i
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int q0 = s32_block(M, kk + 1, r) * 6;
#pragma unroll
        for (int c = 0; c < 6; ++c) tv[c] = __ldcs(p + (q0 + c) * TI);
        sym_mv_acc(tv, xi + 3 * kk, vj + 3 * r);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    sz[0][mp.i16()][mp.j16()][k] = vi[k];
    sz[1][mp.j16()][mp.i16()][k] = vj[k];
  }
  __syncthreads();
  for (int k = t; k < 2 * kStoreTile * 6; k += blockDim.x) {
    const int side = k / (kStoreTile * 6), rem = k % (kStoreTile * 6);
    const int f = rem / 6, v = rem % 6;
    float s = 0.f;
    for (int p = 0; p < kStoreTile; ++p) s += sz[side][f][p][v];
    if (diag) {
      if (side == 1) continue;
      for (int p = 0; p < kStoreTile; ++p) s += sz[1][f][p][v];
    }
    const int fib = (side == 0 ? I16 : J16) * kStoreTile + f;
    if (fib < N) vpart[((int64_t)(side == 0 ? J16 : I16) * N + fib) * 6 + v] = s;
  }
}

template <int M, int TI>
__global__ void __launch_bounds__(256)
k_struct_velocity(int N, const float* __restrict__ S32, const float* __restrict__ x, float* __restrict__ vpart) {
  struct_velocity_tile<M, TI>(N, S32, x, vpart, blockIdx.x);
}

// U_i = (0.5/d) [ (d+2)F + (d-2)(t.F)t + F_i[P0] + sum u ],
// W_i = (1.5/d) (I - t t^T) [ F_i[P1] + sum w ]   (fiber i < N).
// Every rounding is spelled out (fmaf, __fmul_rn, __fadd_rn), so the result
// does not depend on which multiply-adds the compiler would contract in the
// kernel it is inlined into: the single-suspension and packed kernels agree
// bit for bit.
__device__ __forceinline__ void struct_velocity_fiber(const Tables& tab, int N, const float4* __restrict__ ori,
                                                      const float* __restrict__ F, const float* __restrict__ vpart,
                                                      int nparts, int i, float4& tv, float4& rv) {
  const int FFn = 3 * (tab.M + 1);
  const float4 t = ori[i];
  const float d = tab.d;
  const float Fz = 2.f * tab.fz_half;
  const float tF = __fmul_rn(t.z, Fz);
  const float cF = __fmul_rn(d - 2.f, tF);
  const float* Fi = F + (int64_t)i * FFn;
  float U[3] = {fmaf(cF, t.x, Fi[0]), fmaf(cF, t.y, Fi[1]), __fadd_rn(fmaf(cF, t.z, __fmul_rn(d + 2.f, Fz)), Fi[2])};
  float W[3] = {Fi[3], Fi[4], Fi[5]};
  for (int p = 0; p < nparts; ++p) {
    const float* v = vpart + ((int64_t)p * N + i) * 6;
    U[0] += v[0]; U[1] += v[1]; U[2] += v[2];
    W[0] += v[3]; W[1] += v[4]; W[2] += v[5];
  }
  const float tW = fmaf(t.z, W[2], fmaf(t.y, W[1], __fmul_rn(t.x, W[0])));
  const float su = 0.5f / d, sr = 1.5f / d;
  tv = make_float4(__fmul_rn(U[0], su), __fmul_rn(U[1], su), __fmul_rn(U[2], su), 0.f);
  rv = make_float4(__fmul_rn(fmaf(-t.x, tW, W[0]), sr), __fmul_rn(fmaf(-t.y, tW, W[1]), sr),
                   __fmul_rn(fmaf(-t.z, tW, W[2]), sr), 0.f);
}

__global__ void k_struct_velocity_finalize(const Tables tab, int N, const float4* __restrict__ ori,
                                           const float* __restrict__ F, const float* __restrict__ vpart, int nparts,
                                           float4* __restrict__ tvel, float4* __restrict__ rvel) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  float4 tv, rv;
  struct_velocity_fiber(tab, N, ori, F, vpart, nparts, i, tv, rv);
  tvel[i] = tv;
  rvel[i] = rv;
}

// ---- packed step: velocities and update of every member of one group -----
// Members whose packed solve ended non-finite (status 2) sit out: their state
// stays as it is.  Per member the arithmetic is the single-suspension path's
// (k_struct_velocity, k_struct_velocity_finalize, the non-finite guard,
// k_update_fibers), so a member's step is bit for bit the one it takes alone.
__global__ void __launch_bounds__(256)
k_pack_velocity(const PackStepMember* __restrict__ mem, int n) {
  const int L = (int)blockIdx.x;
  const PackStepMember& p = mem[pack_member_of(n, L, [&](int m) { return mem[m].vel_start; })];
  if (*p.solve_status == 2) return;
  struct_velocity_tile<5, 8>(p.N, p.S32, p.x, p.vpart, (unsigned)(L - p.vel_start));
}

// one block per member: velocities, the guard and the second-order update
__global__ void __launch_bounds__(128)
k_pack_finish(const Tables tab, const PackStepMember* __restrict__ mem) {
  const PackStepMember& p = mem[blockIdx.x];
  if (*p.solve_status == 2) return;
  const int N = p.N, nparts = (N + kStoreTile - 1) / kStoreTile;
  int bad = 0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    float4 u, w;
    struct_velocity_fiber(tab, N, p.ori32, p.F, p.vpart, nparts, i, u, w);
    p.tv[i] = u;
    p.rv[i] = w;
    bad |= !(isfinite(u.x) && isfinite(u.y) && isfinite(u.z) && isfinite(w.x) && isfinite(w.y) && isfinite(w.z));
    update_fiber(i, p.first, p.dt, p.pos64_prev, p.pos64, p.ori64_prev, p.ori64, p.tv_prev, u, p.rv_prev, w,
                 p.pos32, p.ori32);
  }
  bad = __syncthreads_or(bad);
  if (threadIdx.x == 0) *p.vbad = bad ? 1 : 0;
}

int launch_pack_velocity_update(const Tables& tab, const PackStepMember* members, int n, int64_t blocks,
                                cudaStream_t st) {
  if (tab.M != 5 || tab.Q != 24 || n < 1 || blocks < 1) return RF_E_UNSUPPORTED;
  k_pack_velocity<<<(unsigned)blocks, 256, 0, st>>>(members, n);
  RF_LAUNCH_CHECK();
  k_pack_finish<<<(unsigned)n, 128, 0, st>>>(tab, members);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

template <typename XT>
__global__ void k_cast_to_float(const XT* __restrict__ in, float* __restrict__ out, int64_t n) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
    out[r] = (float)in[r];
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static unsigned fin_blocks(int64_t n) { return (unsigned)std::min<int64_t>(ceil_div(n, 256), 148 * 8); }

template <int M, int TI, int SMODE, typename XT, typename ACC>
static int launch_z_one(int N, const float* S32, const uint32_t* S16, const XT* x, ACC* zpart, const int* skip,
                        cudaStream_t st) {
  constexpr bool kPrefetch = true;   // the next block row in flight while this one is computed
  constexpr size_t smem = ZSmem<M, sizeof(ACC)>::kBytes;
  static const cudaError_t attr = cudaFuncSetAttribute(k_struct_z<M, TI, SMODE, XT, ACC, kPrefetch>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  RF_CUDA_TRY(attr);
  const unsigned grid = (unsigned)struct_store_tiles(N);
  k_struct_z<M, TI, SMODE, XT, ACC, kPrefetch><<<grid, 256, smem, st>>>(N, S32, S16, x, zpart, skip);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

template <int M, int TI>
static int launch_z(int smode, bool fp64, int N, const float* S32, const uint32_t* S16, const void* x, void* zpart,
                    const int* skip, cudaStream_t st) {
  if (fp64) return launch_z_one<M, TI, 0, double, double>(N, S32, S16, (const double*)x, (double*)zpart, skip, st);
  if (smode == 0) return launch_z_one<M, TI, 0, float, float>(N, S32, S16, (const float*)x, (float*)zpart, skip, st);
  if (smode == 1) return launch_z_one<M, TI, 1, float, float>(N, S32, S16, (const float*)x, (float*)zpart, skip, st);
  return launch_z_one<M, TI, 2, float, float>(N, S32, S16, (const float*)x, (float*)zpart, skip, st);
}

template <int M, int SMODE>
static int launch_z16_bulk(int N, const uint32_t* S16, const float* x, float* zpart, const int* skip, int* err,
                           cudaStream_t st) {
  using B = BulkShape<M>;
  static const cudaError_t attr = cudaFuncSetAttribute(k_struct_z16_bulk<M, SMODE>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)B::kBytes);
  RF_CUDA_TRY(attr);
  int dev = 0, nsm = 0;
  RF_CUDA_TRY(cudaGetDevice(&dev));
  RF_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int64_t ntiles = struct_store_tiles(N);
  const unsigned grid = (unsigned)std::min<int64_t>(ntiles, nsm);
  const int64_t lim = device_wait_limit();
  const uint32_t polls = lim < 0 ? (1u << 24) : (uint32_t)std::min<int64_t>(lim, 1 << 24);
  k_struct_z16_bulk<M, SMODE><<<grid, B::kThreads, B::kBytes, st>>>(N, S16, x, zpart, skip, err, polls);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

int launch_struct_matvec(const Tables& tab, int N, int smode, const float* S32, const uint32_t* S16,
                         const float4* ori, const float* x, float* zpart, float* y, const int* skip, int* err,
                         cudaStream_t st, int variant) {
  int rc = RF_E_UNSUPPORTED;
  const bool bulk = variant != 2 && tab.Q == 24 && smode != 0 && err != nullptr && tab.M <= 5;
  if (bulk) {
    // tiles staged by TMA bulk copies (two 3072*M-byte tiles per SM fit in shared memory for M <= 5)
    switch (tab.M) {
      case 1: rc = smode == 1 ? launch_z16_bulk<1, 1>(N, S16, x, zpart, skip, err, st) : launch_z16_bulk<1, 2>(N, S16, x, zpart, skip, err, st); break;
      case 2: rc = smode == 1 ? launch_z16_bulk<2, 1>(N, S16, x, zpart, skip, err, st) : launch_z16_bulk<2, 2>(N, S16, x, zpart, skip, err, st); break;
      case 3: rc = smode == 1 ? launch_z16_bulk<3, 1>(N, S16, x, zpart, skip, err, st) : launch_z16_bulk<3, 2>(N, S16, x, zpart, skip, err, st); break;
      case 4: rc = smode == 1 ? launch_z16_bulk<4, 1>(N, S16, x, zpart, skip, err, st) : launch_z16_bulk<4, 2>(N, S16, x, zpart, skip, err, st); break;
      case 5: rc = smode == 1 ? launch_z16_bulk<5, 1>(N, S16, x, zpart, skip, err, st) : launch_z16_bulk<5, 2>(N, S16, x, zpart, skip, err, st); break;
    }
  } else {
#define RF_Z_CASE(MM, QQ) \
  if (tab.M == MM && tab.Q == QQ && QQ == 24) rc = launch_z<MM, 8>(smode, false, N, S32, S16, x, zpart, skip, st);
    RF_FOR_EACH_MQ(RF_Z_CASE)
#undef RF_Z_CASE
  }
  if (rc != RF_OK) return rc;
  const int64_t n = (int64_t)N * tab.M;
  const int64_t R = 3 * n;
  const int nparts = (int)ceil_div(N, kStoreTile);
  // the summed rows go to partial slot nparts, which the TMA-staged kernel
  // also fills (diagonal tiles' j side): each row is read before it is written
  k_sum_parts<float><<<(unsigned)ceil_div(R, 64), 256, 0, st>>>(zpart, bulk ? nparts + 1 : nparts, R,
                                                                zpart + (int64_t)nparts * R, skip);
  RF_LAUNCH_CHECK();
  k_struct_finalize<float, float, false><<<fin_blocks(n), 256, 0, st>>>(
      tab, N, ori, x, zpart + (int64_t)nparts * R, 1, nullptr, y, skip);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

int launch_parts_finalize(const Tables& tab, int N, const float4* ori, const float* x, float* zpart, int nparts,
                          float* y, const int* skip, cudaStream_t st) {
  const int64_t n = (int64_t)N * tab.M;
  const int64_t R = 3 * n;
  k_sum_parts<float><<<(unsigned)ceil_div(R, 64), 256, 0, st>>>(zpart, nparts, R, zpart + (int64_t)nparts * R, skip);
  RF_LAUNCH_CHECK();
  k_struct_finalize<float, float, false><<<fin_blocks(n), 256, 0, st>>>(tab, N, ori, x, zpart + (int64_t)nparts * R,
                                                                        1, nullptr, y, skip);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

int launch_parts_residual64(const Tables& tab, int N, const float4* ori, const double* x, const float* zpart,
                            int nparts, const float* b, float* r, const int* skip, cudaStream_t st) {
  const int64_t n = (int64_t)N * tab.M;
  k_struct_finalize<double, double, true, float><<<fin_blocks(n), 256, 0, st>>>(tab, N, ori, x, zpart, nparts, b, r,
                                                                                skip);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

template <int M>
static int launch_r64_bulk(int N, const float* S32, const double* x, double* zpart, const int* skip, int* err,
                           cudaStream_t st) {
  using RS = R64Shape<M>;
  static const cudaError_t attr = cudaFuncSetAttribute(k_struct_r64_bulk<M>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RS::kBytes);
  RF_CUDA_TRY(attr);
  int dev = 0, nsm = 0;
  RF_CUDA_TRY(cudaGetDevice(&dev));
  RF_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int64_t ntiles = struct_store_tiles(N);
  const unsigned grid = (unsigned)std::min<int64_t>(ntiles, nsm);
  const int64_t lim = device_wait_limit();
  const uint32_t polls = lim < 0 ? (1u << 24) : (uint32_t)std::min<int64_t>(lim, 1 << 24);
  k_struct_r64_bulk<M><<<grid, RS::kThreads, RS::kBytes, st>>>(N, S32, x, zpart, skip, err, polls);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

int launch_struct_residual64(const Tables& tab, int N, const float* S32, const float4* ori, const double* x,
                             double* zpart64, const float* b, float* r, const int* skip, int* err, cudaStream_t st) {
  int rc = RF_E_UNSUPPORTED;
  // FP32 blocks staged by TMA bulk copies where that kernel is built (M <= 5, Q = 24, err given)
  const bool bulk = err != nullptr && tab.Q == 24 && tab.M <= 5;
  if (bulk) {
    switch (tab.M) {
      case 1: rc = launch_r64_bulk<1>(N, S32, x, zpart64, skip, err, st); break;
      case 2: rc = launch_r64_bulk<2>(N, S32, x, zpart64, skip, err, st); break;
      case 3: rc = launch_r64_bulk<3>(N, S32, x, zpart64, skip, err, st); break;
      case 4: rc = launch_r64_bulk<4>(N, S32, x, zpart64, skip, err, st); break;
      case 5: rc = launch_r64_bulk<5>(N, S32, x, zpart64, skip, err, st); break;
    }
  } else {
#define RF_Z_CASE(MM, QQ) \
  if (tab.M == MM && tab.Q == QQ && QQ == 24) rc = launch_z<MM, 8>(0, true, N, S32, nullptr, x, zpart64, skip, st);
    RF_FOR_EACH_MQ(RF_Z_CASE)
#undef RF_Z_CASE
  }
  if (rc != RF_OK) return rc;
  const int64_t n = (int64_t)N * tab.M;
  const int64_t R = 3 * n;
  const int nparts = (int)ceil_div(N, kStoreTile);
  // the bulk kernel also fills slot nparts (diagonal tiles' j side), which is the output row
  k_sum_parts<double><<<(unsigned)ceil_div(R, 64), 256, 0, st>>>(zpart64, bulk ? nparts + 1 : nparts, R,
                                                                 zpart64 + (int64_t)nparts * R, skip);
  RF_LAUNCH_CHECK();
  k_struct_finalize<double, double, true><<<fin_blocks(n), 256, 0, st>>>(
      tab, N, ori, x, zpart64 + (int64_t)nparts * R, 1, b, r, skip);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

int launch_struct_apply64(const Tables& tab, int N, const float* S32, const float4* ori, const double* x,
                          double* zpart64, float* y, int* err, cudaStream_t st) {
  int rc = RF_E_UNSUPPORTED;
  const bool bulk = err != nullptr && tab.Q == 24 && tab.M <= 5;
  if (bulk) {
    switch (tab.M) {
      case 1: rc = launch_r64_bulk<1>(N, S32, x, zpart64, nullptr, err, st); break;
      case 2: rc = launch_r64_bulk<2>(N, S32, x, zpart64, nullptr, err, st); break;
      case 3: rc = launch_r64_bulk<3>(N, S32, x, zpart64, nullptr, err, st); break;
      case 4: rc = launch_r64_bulk<4>(N, S32, x, zpart64, nullptr, err, st); break;
      case 5: rc = launch_r64_bulk<5>(N, S32, x, zpart64, nullptr, err, st); break;
    }
  } else {
#define RF_Z_CASE(MM, QQ) \
  if (tab.M == MM && tab.Q == QQ && QQ == 24) rc = launch_z<MM, 8>(0, true, N, S32, nullptr, x, zpart64, nullptr, st);
    RF_FOR_EACH_MQ(RF_Z_CASE)
#undef RF_Z_CASE
  }
  if (rc != RF_OK) return rc;
  const int64_t n = (int64_t)N * tab.M;
  const int64_t R = 3 * n;
  const int nparts = (int)ceil_div(N, kStoreTile);
  k_sum_parts<double><<<(unsigned)ceil_div(R, 64), 256, 0, st>>>(zpart64, bulk ? nparts + 1 : nparts, R,
                                                                 zpart64 + (int64_t)nparts * R, nullptr);
  RF_LAUNCH_CHECK();
  k_struct_finalize<double, double, false><<<fin_blocks(n), 256, 0, st>>>(
      tab, N, ori, x, zpart64 + (int64_t)nparts * R, 1, nullptr, y, nullptr);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

int launch_struct_velocity(const Tables& tab, int N, const float* S32, const float4* ori, const float* F,
                           const float* x, float* vpart, float4* tvel, float4* rvel, cudaStream_t st) {
  const unsigned grid = (unsigned)struct_store_tiles(N);
  bool done = false;
#define RF_V_CASE(MM, QQ)                                                                 \
  if (!done && tab.M == MM && tab.Q == QQ) {                                              \
    k_struct_velocity<MM, 192 / QQ><<<grid, 256, 0, st>>>(N, S32, x, vpart);              \
    done = true;                                                                          \
  }
  RF_FOR_EACH_MQ(RF_V_CASE)
#undef RF_V_CASE
  if (!done) return RF_E_UNSUPPORTED;
  RF_LAUNCH_CHECK();
  k_struct_velocity_finalize<<<(unsigned)ceil_div(N, 128), 128, 0, st>>>(tab, N, ori, F, vpart,
                                                                          (int)ceil_div(N, kStoreTile), tvel, rvel);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

int launch_cast_to_float(const double* in, float* out, int64_t n, cudaStream_t st) {
  k_cast_to_float<double><<<fin_blocks(n), 256, 0, st>>>(in, out, n);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

}  // namespace rf
