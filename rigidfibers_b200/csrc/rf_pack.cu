// Packed solves of many small suspensions.  A thread-block cluster of C
// CTAs (C = 1, 2, 4 or 8, chosen per member by pack_plan_ctas) runs one
// suspension's whole mixed-precision GMRES-IR -- the algorithm rf_solve runs
// for RF_PREC_MIXED_*: restart cycles of up to m Arnoldi steps on the 16-bit
// pair blocks with FP32 sums, CGS2 with FP64 dot products, Givens rotations
// and the least-squares update in FP64, x in FP64, and the residual b - A x
// recomputed from the FP32 pair blocks with FP64 sums at every restart -- so
// an ensemble of small systems is solved by a few launches instead of several
// hundred per suspension.
//
// Work of a member is cut into kParts = 8 fixed parts whatever C is: storage
// tile L belongs to partition L mod 8, whose partial rows are summed in tile
// order; row slice s is fibers [s N / 8, (s + 1) N / 8), whose dot-product
// partial one warp sums.  A CTA of the cluster owns 8 / C consecutive
// partitions and slices; the partitions' partial rows and the slices'
// partials are added in part order through distributed shared memory after a
// cluster barrier.  So a member's solution is the same bits for any C, alone
// and in any pack (it differs from rf_solve's in summation order only), and a
// pack can give its large members more SMs when the GPU has them to spare.
//
// Per Arnoldi step each CTA stages v in shared memory, walks its storage
// tiles (one thread per pair of a 16 x 16 tile, the pair's 16-byte aligned
// record read with 16-byte loads), reduces z over the tile's lanes (halving
// exchanges) and adds the tile's partial rows into its partition's rows; the
// Krylov basis stays in the suspension's V (L2-resident at these sizes), each
// CTA writing its own rows of it.
#include <algorithm>
#include <map>
#include <mutex>
#include <type_traits>

#include <cooperative_groups.h>

#include "rf_common.cuh"
#include "rf_kernels.cuh"
#include "rf_krylov.cuh"

namespace rf {
namespace cg = cooperative_groups;
namespace {

constexpr int kPT = 256;                              // threads per CTA
constexpr int kParts = 8;                             // tile partitions and row slices of a member
constexpr int kPM = 5;                                // force terms of the packed kernel
constexpr int kPM3 = 3 * kPM;
constexpr int kNW = s16_record_words(kPM);            // 16-bit record words per pair
constexpr int kNQ32 = (kPM + 1) * (kPM + 1) * 6;      // FP32 values per pair

__device__ __forceinline__ void pack_tile(int L, int& I, int& J) {
  int j = (int)((sqrtf(8.f * (float)L + 1.f) - 1.f) * 0.5f);
  while ((j + 1) * (j + 2) / 2 <= L) ++j;
  while (j * (j + 1) / 2 > L) --j;
  J = j;
  I = L - j * (j + 1) / 2;
}

template <typename T>
__device__ __forceinline__ T pshfl(T v, int m) {
  return __shfl_xor_sync(0xffffffffu, v, m);
}

__device__ __forceinline__ float pfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double pfma(double a, double b, double c) { return fma(a, b, c); }

// acc += sym(t) v, t = (t00, t11, t22, t01, t02, t12)
template <typename T>
__device__ __forceinline__ void psym(const T (&t)[6], const T* v, T* acc) {
  acc[0] = pfma(t[4], v[2], pfma(t[3], v[1], pfma(t[0], v[0], acc[0])));
  acc[1] = pfma(t[5], v[2], pfma(t[1], v[1], pfma(t[3], v[0], acc[1])));
  acc[2] = pfma(t[2], v[2], pfma(t[5], v[1], pfma(t[4], v[0], acc[2])));
}

// v[16] summed over the 16 lanes that differ in lane bits 0..3 (four halving
// exchanges); lane l gets the sum of v[l & 15].
template <typename T>
__device__ __forceinline__ T psum16(const T (&v)[16], int lane) {
  const bool b3 = lane & 8, b2 = lane & 4, b1 = lane & 2, b0 = lane & 1;
  T a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const T s = b3 ? v[k] : v[k + 8], kp = b3 ? v[k + 8] : v[k];
    a[k] = kp + pshfl(s, 8);
  }
  T b[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const T s = b2 ? a[k] : a[k + 4], kp = b2 ? a[k + 4] : a[k];
    b[k] = kp + pshfl(s, 4);
  }
  T c[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const T s = b1 ? b[k] : b[k + 2], kp = b1 ? b[k + 2] : b[k];
    c[k] = kp + pshfl(s, 2);
  }
  const T s = b0 ? c[0] : c[1], kp = b0 ? c[1] : c[0];
  return kp + pshfl(s, 1);
}

template <typename H16>
__device__ __forceinline__ float2 punpack(uint32_t w) {
  if constexpr (std::is_same<H16, __half>::value) return __half22float2(*reinterpret_cast<const __half2*>(&w));
  else return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w));
}

// z_i += T x_j, z_j += T^T x_i over the 25 blocks of one pair record
template <typename H16>
__device__ __forceinline__ void ppair16(const uint32_t (&w)[kNW], const float (&xi)[kPM3], const float (&xj)[kPM3],
                                        float (&zi)[16], float (&zj)[16]) {
#pragma unroll
  for (int kI = 0; kI < kPM; ++kI)
#pragma unroll
    for (int kJ = 0; kJ < kPM; ++kJ) {
      const int blk = kI * kPM + kJ;
      float tv[6];
#pragma unroll
      for (int h = 0; h < 3; ++h) {
        const float2 f = punpack<H16>(w[3 * blk + h]);
        tv[2 * h] = f.x;
        tv[2 * h + 1] = f.y;
      }
      psym(tv, xj + 3 * kJ, zi + 3 * kI);
      psym(tv, xi + 3 * kI, zj + 3 * kJ);
    }
}

// Shared memory (doubles): [staged vector Rmax][partition rows: 8/C x Rmax]
// [i-side tile partials 8 x 16 x 16][j-side tile sums 16 x 16][H (m+1) x m]
// [cs m][sn m][g m+1][y m][h m+1][h2 m+1][reduction partials 3 x 8 x (m+1)]
// [scalar 2][flags]
// kClustered: launched with clusters of 2, 4 or 8 CTAs; otherwise one CTA per
// member (the same arithmetic in the same order, without cluster barriers and
// distributed shared memory)
template <bool kClustered>
__global__ void __launch_bounds__(kPT) k_pack_gmres_ir(const PackMember* __restrict__ members, int Rmax, int m) {
  extern __shared__ __align__(16) unsigned char psm[];
  int C = 1, rank = 0;
  if constexpr (kClustered) {
    C = (int)cg::this_cluster().num_blocks();
    rank = (int)cg::this_cluster().block_rank();
  }
  const PackMember& P = members[blockIdx.x / C];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int N = P.N;
  const int R = kPM3 * N;
  const int T16 = (N + 15) / 16;
  const int ntiles = T16 * (T16 + 1) / 2;
  const int ldh = m + 1;
  const int spc = kParts / C;                                   // partitions (and row slices) per CTA
  const int p0 = rank * spc;                                    // this CTA's first partition
  const int q0 = kPM3 * ((rank * N) / C), q1 = kPM3 * (((rank + 1) * N) / C);   // its rows
  double* sxd = reinterpret_cast<double*>(psm);
  float* sxf = reinterpret_cast<float*>(psm);
  double* zpd = sxd + Rmax;                                     // partition rows, slot stride Rmax
  float* zpf = reinterpret_cast<float*>(zpd);
  double* tail = zpd + (size_t)spc * Rmax;
  double (*zip)[16][16] = reinterpret_cast<double (*)[16][16]>(tail);
  float (*zipf)[16][16] = reinterpret_cast<float (*)[16][16]>(tail);
  double (*zjs)[16] = reinterpret_cast<double (*)[16]>(tail + 8 * 16 * 16);
  float (*zjsf)[16] = reinterpret_cast<float (*)[16]>(tail + 8 * 16 * 16);
  double* H = tail + 8 * 16 * 16 + 16 * 16;
  double* cs = H + (size_t)ldh * m;
  double* sn = cs + m;
  double* g = sn + m;
  double* yv = g + m + 1;
  double* hh = yv + m;
  double* hh2 = hh + m + 1;
  double* dpart = hh2 + m + 1;                                  // [3][kParts][m+1]
  double* scal = dpart + 3 * kParts * (m + 1);
  int* flags = reinterpret_cast<int*>(scal + 2);                // [0] cycle done, [1] converged, [2] non-finite
  float* V = P.V;
  const int64_t ldv = P.ldv;
  const int i16 = t & 15, j16 = t >> 4;
  const int sub = (i16 >> 3) * 2 + (j16 >> 3);
  const int rec16 = (sub * 8 + (j16 & 7)) * 8 + (i16 & 7);   // record of pair (i16, j16) in a storage tile
  const int rec32 = sub * 8 + (j16 & 7);                       // FP32 record (8 pairs, [value][i])
  int rb = 0;                                                  // reduction buffer in use (of 3)
  // a cluster barrier, or the block barrier when the member has one CTA
  auto csync = [&]() {
    if constexpr (kClustered) cg::this_cluster().sync();
    else __syncthreads();
  };
  // a pointer into CTA r's shared memory at the offset of p in this CTA's
  auto at_rank = [&](auto* p, int r) {
    if constexpr (kClustered) return cg::this_cluster().map_shared_rank(p, r);
    else return p;
  };

  // out[k] = sum over the member's rows of a[r] * V_k[r] for k < nv (square:
  // nv = 1 and a[r]^2), FP64.  Slice s's partial is one warp's (lane-strided
  // sums, then a butterfly), written into the owning CTA's buffer; after the
  // cluster barrier every CTA adds the 8 partials in slice order.  Three
  // buffers in turn: a buffer is written again only after two more cluster
  // barriers, when every CTA has read it.
  auto cdots = [&](const float* a, int nv, bool square, double* out) {
    __syncthreads();                                           // this CTA's rows of a are written
    double* part = dpart + (size_t)rb * kParts * (m + 1);
    const int ng = (nv + 3) / 4;
    for (int task = warp; task < spc * ng; task += kPT / 32) {
      const int s = p0 + task % spc, k0 = 4 * (task / spc);
      const int r0 = kPM3 * ((s * N) / kParts), r1 = kPM3 * (((s + 1) * N) / kParts);
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      for (int r = r0 + lane; r < r1; r += 32) {
        const double ar = (double)a[r];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (k0 + u < nv) {
            const float* vk = square ? a : V + (int64_t)(k0 + u) * ldv;
            acc[u] = fma(ar, (double)vk[r], acc[u]);
          }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        double v = acc[u];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += pshfl(v, o);
        if (lane == 0 && k0 + u < nv) part[s * (m + 1) + k0 + u] = v;
      }
    }
    csync();
    for (int k = t; k < nv; k += kPT) {
      double sum = 0.0;
      for (int s = 0; s < kParts; ++s) sum += at_rank(part, s / spc)[s * (m + 1) + k];
      out[k] = sum;
    }
    __syncthreads();
    rb = rb == 2 ? 0 : rb + 1;
  };
  auto sumsq = [&](const float* a) -> double {
    cdots(a, 1, true, scal);
    return scal[0];
  };
  // w = v + C (T v) with the 16-bit blocks, FP32 sums; this CTA writes its rows of w
  auto matvec16 = [&](const float* v, float* w) {
    for (int q = t; q < spc * Rmax; q += kPT) zpf[q] = 0.f;
    csync();                                                   // every CTA's rows of v are written
    for (int r = t; r < R; r += kPT) sxf[r] = v[r];
    __syncthreads();
    for (int L = 0; L < ntiles; ++L) {
      const int p = L % kParts;
      if (p / spc != rank) continue;
      float* zs = zpf + (size_t)(p - p0) * Rmax;
      int I, J;
      pack_tile(L, I, J);
      const int i = I * 16 + i16, j = J * 16 + j16;
      float zi[16], zj[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) zi[q] = zj[q] = 0.f;
      if (i < j && j < N) {
        uint32_t wv[kNW];
        const uint4* pw = reinterpret_cast<const uint4*>(P.S16 + ((int64_t)L * 256 + rec16) * kNW);
#pragma unroll
        for (int u = 0; u < kNW / 4; ++u) {
          const uint4 q4 = pw[u];
          wv[4 * u] = q4.x; wv[4 * u + 1] = q4.y; wv[4 * u + 2] = q4.z; wv[4 * u + 3] = q4.w;
        }
        float xi[kPM3], xj[kPM3];
#pragma unroll
        for (int q = 0; q < kPM3; ++q) {
          xi[q] = sxf[i * kPM3 + q];
          xj[q] = sxf[j * kPM3 + q];
        }
        if (P.smode == 2) ppair16<__nv_bfloat16>(wv, xi, xj, zi, zj);
        else ppair16<__half>(wv, xi, xj, zi, zj);
      }
      const float sj = psum16(zj, lane);   // z_j over this half-warp's 16 i
      const bool b4 = lane & 16;
      float u8[8];                          // z_i over this warp's two j: one halving exchange
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const float s = b4 ? zi[k] : zi[k + 8], kp = b4 ? zi[k + 8] : zi[k];
        u8[k] = kp + pshfl(s, 16);
      }
      __syncthreads();   // the previous tile's sums have been read
      zjsf[j16][lane & 15] = sj;
#pragma unroll
      for (int k = 0; k < 8; ++k) zipf[warp][i16][8 * (b4 ? 1 : 0) + k] = u8[k];
      __syncthreads();
      if (t < 16 * kPM3) {
        const int f = t / kPM3, q = t % kPM3;
        float si = 0.f;
        for (int w8 = 0; w8 < 8; ++w8) si += zipf[w8][f][q];
        const int fi = I * 16 + f, fj = J * 16 + f;
        if (fi < N) zs[fi * kPM3 + q] += si;
        if (fj < N) zs[fj * kPM3 + q] += zjsf[f][q];
      }
    }
    csync();                                                   // every partition's rows are complete
    for (int u = t; u < (q1 - q0) / 3; u += kPT) {
      const int r0 = q0 + 3 * u, i = r0 / kPM3, k = (r0 % kPM3) / 3;
      float z3[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int p = 0; p < kParts; ++p) {
        const float* zr = at_rank(zpf, p / spc) + (size_t)(p % spc) * Rmax + r0;
        z3[0] += zr[0];
        z3[1] += zr[1];
        z3[2] += zr[2];
      }
      const float4 o = P.ori[i];
      const float t3[3] = {o.x, o.y, o.z};
      const float tz = t3[0] * z3[0] + t3[1] * z3[1] + t3[2] * z3[2];
      const float coef = P.coef[k], E = P.eig[k];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const float cz = k == 0 ? coef * t3[a] * tz : coef * (z3[a] - E * t3[a] * tz);
        w[r0 + a] = sxf[r0 + a] + cz;
      }
    }
  };
  // r = b - (x + C (T x)) with the FP32 blocks, x and sums in FP64; this CTA writes its rows of r
  auto residual64 = [&](float* r) {
    for (int q = t; q < spc * Rmax; q += kPT) zpd[q] = 0.0;
    csync();                                                   // every CTA's rows of x are written
    for (int q = t; q < R; q += kPT) sxd[q] = P.x64[q];
    __syncthreads();
    for (int L = 0; L < ntiles; ++L) {
      const int p = L % kParts;
      if (p / spc != rank) continue;
      double* zs = zpd + (size_t)(p - p0) * Rmax;
      int I, J;
      pack_tile(L, I, J);
      const int i = I * 16 + i16, j = J * 16 + j16;
      double zi[16], zj[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) zi[q] = zj[q] = 0.0;
      if (i < j && j < N) {
        const float* base = P.S32 + ((int64_t)L * 32 + rec32) * (kNQ32 * 8) + (i16 & 7);
        const double* xi = sxd + i * kPM3;
        const double* xj = sxd + j * kPM3;
#pragma unroll
        for (int kI = 0; kI < kPM; ++kI)
#pragma unroll
          for (int kJ = 0; kJ < kPM; ++kJ) {
            double tv[6];
#pragma unroll
            for (int c = 0; c < 6; ++c) tv[c] = (double)base[((kI * kPM + kJ) * 6 + c) * 8];
            psym(tv, xj + 3 * kJ, zi + 3 * kI);
            psym(tv, xi + 3 * kI, zj + 3 * kJ);
          }
      }
      const double sj = psum16(zj, lane);
      const bool b4 = lane & 16;
      double u8[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const double s = b4 ? zi[k] : zi[k + 8], kp = b4 ? zi[k + 8] : zi[k];
        u8[k] = kp + pshfl(s, 16);
      }
      __syncthreads();
      zjs[j16][lane & 15] = sj;
#pragma unroll
      for (int k = 0; k < 8; ++k) zip[warp][i16][8 * (b4 ? 1 : 0) + k] = u8[k];
      __syncthreads();
      if (t < 16 * kPM3) {
        const int f = t / kPM3, q = t % kPM3;
        double si = 0.0;
        for (int w8 = 0; w8 < 8; ++w8) si += zip[w8][f][q];
        const int fi = I * 16 + f, fj = J * 16 + f;
        if (fi < N) zs[fi * kPM3 + q] += si;
        if (fj < N) zs[fj * kPM3 + q] += zjs[f][q];
      }
    }
    csync();
    for (int u = t; u < (q1 - q0) / 3; u += kPT) {
      const int r0 = q0 + 3 * u, i = r0 / kPM3, k = (r0 % kPM3) / 3;
      double z3[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int p = 0; p < kParts; ++p) {
        const double* zr = at_rank(zpd, p / spc) + (size_t)(p % spc) * Rmax + r0;
        z3[0] += zr[0];
        z3[1] += zr[1];
        z3[2] += zr[2];
      }
      const float4 o = P.ori[i];
      const double t3[3] = {(double)o.x, (double)o.y, (double)o.z};
      const double tz = t3[0] * z3[0] + t3[1] * z3[1] + t3[2] * z3[2];
      const double coef = (double)P.coef[k], E = (double)P.eig[k];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const double cz = k == 0 ? coef * t3[a] * tz : coef * (z3[a] - E * t3[a] * tz);
        const double yr = sxd[r0 + a] + cz;
        r[r0 + a] = (float)((double)P.b[r0 + a] - yr);
      }
    }
  };

  for (int q = q0 + t; q < q1; q += kPT) P.x64[q] = 0.0;
  const double bnorm = sqrt(sumsq(P.b));
  const double tol = P.tol * bnorm;
  int total = 0, restarts = 0, refinements = 0, status = 0;
  double beta = bnorm;
  bool conv = bnorm == 0.0, bad = !isfinite(bnorm);
  float* V0 = V;
  for (int cycle = 0; !conv && !bad; ++cycle) {
    if (cycle == 0) {
      for (int q = q0 + t; q < q1; q += kPT) V0[q] = P.b[q];
    } else {
      residual64(V0);
      ++refinements;
    }
    beta = sqrt(sumsq(V0));
    conv = beta <= tol;
    bad = !isfinite(beta);
    if (conv || bad || total >= P.maxit) break;
    const float inv = (float)(1.0 / beta);
    for (int q = q0 + t; q < q1; q += kPT) V0[q] *= inv;
    if (t == 0) {
      g[0] = beta;
      for (int k = 1; k <= m; ++k) g[k] = 0.0;
    }
    __syncthreads();
    int jc = 0;
    for (int j = 0; j < m; ++j) {
      float* w = V + (int64_t)(j + 1) * ldv;
      matvec16(V + (int64_t)j * ldv, w);
      const int nv = j + 1;
      cdots(w, nv, false, hh);
      for (int q = q0 + t; q < q1; q += kPT) {
        double s = (double)w[q];
        for (int k = 0; k < nv; ++k) s -= hh[k] * (double)V[(int64_t)k * ldv + q];
        w[q] = (float)s;
      }
      cdots(w, nv, false, hh2);
      for (int q = q0 + t; q < q1; q += kPT) {
        double s = (double)w[q];
        for (int k = 0; k < nv; ++k) s -= hh2[k] * (double)V[(int64_t)k * ldv + q];
        w[q] = (float)s;
      }
      const double nrm = sqrt(sumsq(w));
      if (nrm > 0.0 && isfinite(nrm)) {
        const float winv = (float)(1.0 / nrm);
        for (int q = q0 + t; q < q1; q += kPT) w[q] *= winv;
      }
      if (t == 0) {   // the same values in every CTA of the cluster: the same decisions
        double* Hc = H + (int64_t)j * ldh;
        for (int k = 0; k < nv; ++k) Hc[k] = hh[k] + hh2[k];
        Hc[j + 1] = nrm;
        for (int k = 0; k < j; ++k) {
          const double x0 = Hc[k], x1 = Hc[k + 1];
          Hc[k] = cs[k] * x0 + sn[k] * x1;
          Hc[k + 1] = -sn[k] * x0 + cs[k] * x1;
        }
        const double x0 = Hc[j], x1 = Hc[j + 1];
        const double rr = hypot(x0, x1);
        const double c = rr > 0.0 ? x0 / rr : 1.0, s = rr > 0.0 ? x1 / rr : 0.0;
        cs[j] = c;
        sn[j] = s;
        Hc[j] = rr;
        Hc[j + 1] = 0.0;
        g[j + 1] = -s * g[j];
        g[j] = c * g[j];
        const double est = fabs(g[j + 1]);
        const bool nf = !isfinite(est);
        flags[2] = nf ? 1 : 0;
        flags[0] = (nf || est <= tol || j + 1 >= m || total + 1 >= P.maxit || nrm == 0.0) ? 1 : 0;
      }
      __syncthreads();
      ++total;
      jc = j + 1;
      if (flags[2]) bad = true;
      if (flags[0]) break;
    }
    if (bad) break;
    // x += V y, H y = g (upper triangular, jc x jc)
    if (t == 0) {
      for (int i = jc - 1; i >= 0; --i) {
        double s = g[i];
        for (int k = i + 1; k < jc; ++k) s -= H[(int64_t)k * ldh + i] * yv[k];
        yv[i] = s / H[(int64_t)i * ldh + i];
      }
    }
    __syncthreads();
    for (int q = q0 + t; q < q1; q += kPT) {
      double s = 0.0;
      for (int k = 0; k < jc; ++k) s += yv[k] * (double)V[(int64_t)k * ldv + q];
      P.x64[q] += s;
    }
    ++restarts;
  }
  status = bad ? 2 : (conv ? 0 : 1);
  for (int q = q0 + t; q < q1; q += kPT) P.x[q] = (float)P.x64[q];
  if (rank == 0 && t == 0) {
    P.out[0] = total;
    P.out[1] = restarts;
    P.out[2] = refinements;
    P.out[3] = status;
    P.relres[0] = bnorm > 0.0 ? beta / bnorm : 0.0;
  }
  csync();   // the other CTAs may still read this CTA's shared memory
}

}  // namespace

void pack_plan_ctas(const int* fibers, int n, int sms, int* ctas, int max_cluster) {
  int total = 0;
  for (int i = 0; i < n; ++i) {
    ctas[i] = fibers[i] > kPackSingleMaxFibers ? 2 : 1;
    total += ctas[i];
  }
  for (;;) {
    int best = -1;
    double most = 0.0;
    for (int i = 0; i < n; ++i) {
      const int T = (fibers[i] + 15) / 16, tiles = T * (T + 1) / 2;
      if (2 * ctas[i] > max_cluster || tiles < 4 * ctas[i]) continue;   // at least two tiles per CTA after doubling
      const double w = (double)tiles / ctas[i];
      if (w > most) {
        most = w;
        best = i;
      }
    }
    if (best < 0 || total + ctas[best] > sms) break;
    total += ctas[best];
    ctas[best] *= 2;
  }
}

size_t pack_smem_bytes(int Rmax, int m, int csize) {
  const size_t slots = (size_t)(kParts / csize);
  const size_t doubles = (1 + slots) * (size_t)Rmax + 8 * 16 * 16 + 16 * 16 + (size_t)(m + 1) * m + 2 * (size_t)m +
                         (size_t)(m + 1) + (size_t)m + 2 * (size_t)(m + 1) + 3 * kParts * (size_t)(m + 1) + 2;
  return doubles * sizeof(double) + 4 * sizeof(int);
}

int pack_max_cluster() {
  // one query per device and cluster size with the largest shared memory a
  // pack can ask for (kPackMaxFibers rows, restart kMaxRestart): smaller packs
  // fit wherever it does.  The answer is the largest C with every size from 2
  // to C schedulable.
  static std::mutex mu;
  static std::map<int, int> known;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 1;
  std::lock_guard<std::mutex> lk(mu);
  auto it = known.find(dev);
  if (it != known.end()) return it->second;
  int best = 1;
  for (int c = 2; c <= kParts && best == c / 2; c *= 2) {
    const size_t smem = pack_smem_bytes(kPM3 * kPackMaxFibers, kMaxRestart, c);
    if (cudaFuncSetAttribute(k_pack_gmres_ir<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      break;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)c);
    cfg.blockDim = dim3(kPT);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)c;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, k_pack_gmres_ir<true>, &cfg) == cudaSuccess && clusters > 0)
      best = c;
  }
  cudaGetLastError();   // a refused query leaves no error behind
  known[dev] = best;
  return best;
}

void pack_lanes_release(PackLanes& l) {
  for (auto& s : l.aux)
    if (s) cudaStreamDestroy(s), s = nullptr;
  for (auto& e : l.join)
    if (e) cudaEventDestroy(e), e = nullptr;
  if (l.fork) cudaEventDestroy(l.fork), l.fork = nullptr;
}

int launch_pack_gmres_ir(const PackMember* members, const int (&counts)[4], const int (&rmax)[4], int m,
                         cudaStream_t st, PackLanes& lanes) {
  int n = 0;
  bool sizes_ok = m >= 1 && m <= kMaxRestart;
  size_t smax = 0;
  for (int c = 0; c < 4; ++c) {
    if (counts[c] < 0) sizes_ok = false;
    if (counts[c] <= 0) continue;
    n += counts[c];
    // one CTA holds all 8 partitions' rows: at most kPackSingleMaxFibers fibers
    const int limit = kPM3 * (c == 3 ? kPackSingleMaxFibers : kPackMaxFibers);
    if (rmax[c] < 1 || rmax[c] > limit) sizes_ok = false;
    else smax = std::max(smax, pack_smem_bytes(rmax[c], m, kParts >> c));
  }
  if (n < 1 || !sizes_ok) {
    set_last_error_str("packed solve: bad sizes");
    return RF_E_INPUT;
  }
  RF_CUDA_TRY(cudaFuncSetAttribute(k_pack_gmres_ir<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax));
  RF_CUDA_TRY(cudaFuncSetAttribute(k_pack_gmres_ir<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax));
  // one launch per cluster size, the largest first; the classes after the
  // first on their own streams, forked from st before the first launch, so
  // that they run beside it
  int classes = 0;
  for (int c = 0; c < 4; ++c) classes += counts[c] > 0 ? 1 : 0;
  if (classes > 1) {
    if (!lanes.fork) RF_CUDA_TRY(cudaEventCreateWithFlags(&lanes.fork, cudaEventDisableTiming));
    for (int k = 0; k < classes - 1; ++k)
      if (!lanes.aux[k]) {
        RF_CUDA_TRY(cudaStreamCreateWithFlags(&lanes.aux[k], cudaStreamNonBlocking));
        RF_CUDA_TRY(cudaEventCreateWithFlags(&lanes.join[k], cudaEventDisableTiming));
      }
    RF_CUDA_TRY(cudaEventRecord(lanes.fork, st));
  }
  int used = 0, off = 0;
  for (int c = 0; c < 4; ++c) {
    if (counts[c] == 0) continue;
    const int csize = kParts >> c;
    cudaStream_t s = st;
    if (used > 0) {
      s = lanes.aux[used - 1];
      RF_CUDA_TRY(cudaStreamWaitEvent(s, lanes.fork, 0));
    }
    const int Rmax = rmax[c];
    if (csize == 1) {
      k_pack_gmres_ir<false><<<counts[c], kPT, pack_smem_bytes(Rmax, m, 1), s>>>(members + off, Rmax, m);
      RF_LAUNCH_CHECK();
    } else {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)(counts[c] * csize));
      cfg.blockDim = dim3(kPT);
      cfg.dynamicSmemBytes = pack_smem_bytes(Rmax, m, csize);
      cfg.stream = s;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = (unsigned)csize;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      RF_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_pack_gmres_ir<true>, members + off, Rmax, m));
    }
    if (used > 0) RF_CUDA_TRY(cudaEventRecord(lanes.join[used - 1], s));
    off += counts[c];
    ++used;
  }
  for (int k = 1; k < used; ++k) RF_CUDA_TRY(cudaStreamWaitEvent(st, lanes.join[k - 1], 0));
  return RF_OK;
}

}  // namespace rf

extern "C" int rf_debug_pack_plan(const int* fibers, int n, int sms, int* ctas) {
  if (!fibers || !ctas || n < 1 || sms < 1) return RF_E_INPUT;
  for (int i = 0; i < n; ++i)
    if (fibers[i] < 1 || fibers[i] > rf::kPackMaxFibers) return RF_E_INPUT;
  rf::pack_plan_ctas(fibers, n, sms, ctas, 8);
  return RF_OK;
}
