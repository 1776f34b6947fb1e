// Packed solves of many small suspensions.  One CTA runs one suspension's
// whole mixed-precision GMRES-IR -- the algorithm rf_solve runs for
// RF_PREC_MIXED_*: restart cycles of up to m Arnoldi steps on the 16-bit pair
// blocks with FP32 sums, CGS2 with FP64 dot products, Givens rotations and
// the least-squares update in FP64, x in FP64, and the residual b - A x
// recomputed from the FP32 pair blocks with FP64 sums at every restart -- so
// an ensemble of small systems is solved by one launch instead of several
// hundred per suspension.  A CTA reads and writes only its own suspension's
// buffers and sums in a fixed order, so a suspension's solution is the same
// alone and in any pack (it differs from rf_solve's in summation order only).
//
// Per Arnoldi step the CTA stages v in shared memory, walks the suspension's
// storage tiles (one thread per pair of a 16 x 16 tile, the pair's 16-byte
// aligned record read with 16-byte loads), reduces z over the tile's lanes
// (halving exchanges) and adds the tile's partial rows into a shared-memory z
// in tile order; the Krylov basis stays in the suspension's V (L2-resident at
// these sizes).
#include <type_traits>

#include "rf_common.cuh"
#include "rf_kernels.cuh"

namespace rf {
namespace {

constexpr int kPT = 256;                              // threads per suspension
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

// Shared memory: [staged vector: Rmax doubles][z: Rmax doubles][i-side
// partials 8 x 16 x 16 doubles][j-side sums 16 x 16 doubles][H (m+1) x m]
// [cs m][sn m][g m+1][y m][h m+1][h2 m+1][dot partials 8 x (m+1)][flags]
__global__ void __launch_bounds__(kPT) k_pack_gmres_ir(const PackMember* __restrict__ members, int Rmax, int m) {
  extern __shared__ __align__(16) unsigned char psm[];
  const PackMember& P = members[blockIdx.x];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int N = P.N;
  const int R = kPM3 * N;
  const int T16 = (N + 15) / 16;
  const int ntiles = T16 * (T16 + 1) / 2;
  const int ldh = m + 1;
  double* sxd = reinterpret_cast<double*>(psm);
  float* sxf = reinterpret_cast<float*>(psm);
  double* szd = sxd + Rmax;
  float* szf = reinterpret_cast<float*>(szd);
  double (*zip)[16][16] = reinterpret_cast<double (*)[16][16]>(szd + Rmax);
  float (*zipf)[16][16] = reinterpret_cast<float (*)[16][16]>(szd + Rmax);
  double (*zjs)[16] = reinterpret_cast<double (*)[16]>(szd + Rmax + 8 * 16 * 16);
  float (*zjsf)[16] = reinterpret_cast<float (*)[16]>(szd + Rmax + 8 * 16 * 16);
  double* H = szd + Rmax + 8 * 16 * 16 + 16 * 16;
  double* cs = H + (size_t)ldh * m;
  double* sn = cs + m;
  double* g = sn + m;
  double* yv = g + m + 1;
  double* hh = yv + m;
  double* hh2 = hh + m + 1;
  double* red = hh2 + m + 1;                                // [8][m+1]
  int* flags = reinterpret_cast<int*>(red + 8 * (m + 1));   // [0] cycle done, [1] converged, [2] non-finite
  float* V = P.V;
  const int64_t ldv = P.ldv;
  const int i16 = t & 15, j16 = t >> 4;
  const int sub = (i16 >> 3) * 2 + (j16 >> 3);
  const int rec16 = (sub * 8 + (j16 & 7)) * 8 + (i16 & 7);   // record of pair (i16, j16) in a storage tile
  const int rec32 = sub * 8 + (j16 & 7);                       // FP32 record (8 pairs, [value][i])

  // out[k] = a . V_k for k < nv (FP64, fixed order); ends with a barrier
  auto dots = [&](const float* a, int nv, double* out) {
    for (int k = 0; k < nv; ++k) {
      const float* vk = V + (int64_t)k * ldv;
      double s = 0.0;
      for (int r = t; r < R; r += kPT) s = fma((double)a[r], (double)vk[r], s);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += pshfl(s, o);
      if (lane == 0) red[warp * (m + 1) + k] = s;
    }
    __syncthreads();
    for (int k = t; k < nv; k += kPT) {
      double s = 0.0;
      for (int w8 = 0; w8 < 8; ++w8) s += red[w8 * (m + 1) + k];
      out[k] = s;
    }
    __syncthreads();
  };
  // sum of a[r]^2 (FP64, fixed order); ends with a barrier
  auto sumsq = [&](const float* a) -> double {
    double s = 0.0;
    for (int r = t; r < R; r += kPT) s = fma((double)a[r], (double)a[r], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += pshfl(s, o);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    double tot = 0.0;
    for (int w8 = 0; w8 < 8; ++w8) tot += red[w8];
    __syncthreads();
    return tot;
  };
  // w = v + C (T v) with the 16-bit blocks, FP32 sums
  auto matvec16 = [&](const float* v, float* w) {
    for (int r = t; r < R; r += kPT) {
      sxf[r] = v[r];
      szf[r] = 0.f;
    }
    __syncthreads();
    for (int L = 0; L < ntiles; ++L) {
      int I, J;
      pack_tile(L, I, J);
      const int i = I * 16 + i16, j = J * 16 + j16;
      float zi[16], zj[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) zi[q] = zj[q] = 0.f;
      if (i < j && j < N) {
        uint32_t wv[kNW];
        const uint4* p = reinterpret_cast<const uint4*>(P.S16 + ((int64_t)L * 256 + rec16) * kNW);
#pragma unroll
        for (int u = 0; u < kNW / 4; ++u) {
          const uint4 q4 = p[u];
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
        if (fi < N) szf[fi * kPM3 + q] += si;
        if (fj < N) szf[fj * kPM3 + q] += zjsf[f][q];
      }
    }
    __syncthreads();
    for (int u = t; u < N * kPM; u += kPT) {
      const int i = u / kPM, k = u % kPM, r0 = i * kPM3 + 3 * k;
      const float4 o = P.ori[i];
      const float t3[3] = {o.x, o.y, o.z};
      const float z3[3] = {szf[r0], szf[r0 + 1], szf[r0 + 2]};
      const float tz = t3[0] * z3[0] + t3[1] * z3[1] + t3[2] * z3[2];
      const float coef = P.coef[k], E = P.eig[k];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const float cz = k == 0 ? coef * t3[a] * tz : coef * (z3[a] - E * t3[a] * tz);
        w[r0 + a] = sxf[r0 + a] + cz;
      }
    }
    __syncthreads();
  };
  // r = b - (x + C (T x)) with the FP32 blocks, x and sums in FP64
  auto residual64 = [&](float* r) {
    for (int q = t; q < R; q += kPT) {
      sxd[q] = P.x64[q];
      szd[q] = 0.0;
    }
    __syncthreads();
    for (int L = 0; L < ntiles; ++L) {
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
        if (fi < N) szd[fi * kPM3 + q] += si;
        if (fj < N) szd[fj * kPM3 + q] += zjs[f][q];
      }
    }
    __syncthreads();
    for (int u = t; u < N * kPM; u += kPT) {
      const int i = u / kPM, k = u % kPM, r0 = i * kPM3 + 3 * k;
      const float4 o = P.ori[i];
      const double t3[3] = {(double)o.x, (double)o.y, (double)o.z};
      const double z3[3] = {szd[r0], szd[r0 + 1], szd[r0 + 2]};
      const double tz = t3[0] * z3[0] + t3[1] * z3[1] + t3[2] * z3[2];
      const double coef = (double)P.coef[k], E = (double)P.eig[k];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const double cz = k == 0 ? coef * t3[a] * tz : coef * (z3[a] - E * t3[a] * tz);
        const double yr = sxd[r0 + a] + cz;
        r[r0 + a] = (float)((double)P.b[r0 + a] - yr);
      }
    }
    __syncthreads();
  };

  for (int q = t; q < R; q += kPT) P.x64[q] = 0.0;
  const double bnorm = sqrt(sumsq(P.b));
  const double tol = P.tol * bnorm;
  int total = 0, restarts = 0, refinements = 0, status = 0;
  double beta = bnorm;
  bool conv = bnorm == 0.0, bad = !isfinite(bnorm);
  float* V0 = V;
  for (int cycle = 0; !conv && !bad; ++cycle) {
    if (cycle == 0) {
      for (int q = t; q < R; q += kPT) V0[q] = P.b[q];
      __syncthreads();
    } else {
      residual64(V0);
      ++refinements;
    }
    beta = sqrt(sumsq(V0));
    conv = beta <= tol;
    bad = !isfinite(beta);
    if (conv || bad || total >= P.maxit) break;
    const float inv = (float)(1.0 / beta);
    for (int q = t; q < R; q += kPT) V0[q] *= inv;
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
      dots(w, nv, hh);
      for (int q = t; q < R; q += kPT) {
        double s = (double)w[q];
        for (int k = 0; k < nv; ++k) s -= hh[k] * (double)V[(int64_t)k * ldv + q];
        w[q] = (float)s;
      }
      __syncthreads();
      dots(w, nv, hh2);
      for (int q = t; q < R; q += kPT) {
        double s = (double)w[q];
        for (int k = 0; k < nv; ++k) s -= hh2[k] * (double)V[(int64_t)k * ldv + q];
        w[q] = (float)s;
      }
      __syncthreads();
      const double nrm = sqrt(sumsq(w));
      if (nrm > 0.0 && isfinite(nrm)) {
        const float winv = (float)(1.0 / nrm);
        for (int q = t; q < R; q += kPT) w[q] *= winv;
      }
      if (t == 0) {
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
    for (int q = t; q < R; q += kPT) {
      double s = 0.0;
      for (int k = 0; k < jc; ++k) s += yv[k] * (double)V[(int64_t)k * ldv + q];
      P.x64[q] += s;
    }
    __syncthreads();
    ++restarts;
  }
  status = bad ? 2 : (conv ? 0 : 1);
  for (int q = t; q < R; q += kPT) P.x[q] = (float)P.x64[q];
  if (t == 0) {
    P.out[0] = total;
    P.out[1] = restarts;
    P.out[2] = refinements;
    P.out[3] = status;
    P.relres[0] = bnorm > 0.0 ? beta / bnorm : 0.0;
  }
}

}  // namespace

size_t pack_smem_bytes(int Rmax, int m) {
  const size_t doubles = 2 * (size_t)Rmax + 8 * 16 * 16 + 16 * 16 + (size_t)(m + 1) * m + 2 * (size_t)m +
                         (size_t)(m + 1) + (size_t)m + 2 * (size_t)(m + 1) + 8 * (size_t)(m + 1);
  return doubles * sizeof(double) + 4 * sizeof(int);
}

int launch_pack_gmres_ir(const PackMember* members, int n, int Rmax, int m, cudaStream_t st) {
  if (n < 1 || Rmax < 1 || Rmax > kPM3 * kPackMaxFibers || m < 1) {
    set_last_error_str("packed solve: bad sizes");
    return RF_E_INPUT;
  }
  const size_t smem = pack_smem_bytes(Rmax, m);
  RF_CUDA_TRY(cudaFuncSetAttribute(k_pack_gmres_ir, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_pack_gmres_ir<<<n, kPT, smem, st>>>(members, Rmax, m);
  RF_LAUNCH_CHECK();
  return RF_OK;
}

}  // namespace rf
