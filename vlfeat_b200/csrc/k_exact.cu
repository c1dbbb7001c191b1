// Exact-arithmetic kernels (CUDA cores, float or double).  These evaluate the
// reference's own formulation -- sum_d (x-mu)^2 / sigma^2 per (descriptor,
// component), thresholded statistics, etc. -- and serve VL_TYPE_DOUBLE calls,
// the EXACT precision mode and the M-step / restart machinery of EM.
//
// Determinism: every reduction runs in a fixed order (per-block partials,
// then a fixed-shape final reduction), so results are bitwise reproducible
// run to run, unlike the reference's OpenMP critical-section merge
// (vl/gmm.c:1152-1166).
#include <cmath>
#include <cstring>
#include <type_traits>

#include "engine.h"
#include "exact_math.cuh"
#include "tc_common.cuh"

namespace vlb {

namespace {

constexpr int kThreads = 256;

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float dexp(float x) { return expf(x); }
__device__ __forceinline__ double dexp(double x) { return exp(x); }

// ------------------------------------------------------------ prepare
// Per-component constants, vl/gmm.c:741-756 and vl/fisher.c:386-390.
template <typename T>
__global__ void k_prepare(const T *__restrict__ priors, const T *__restrict__ covs, int K, int D,
                          T halfDimLog2Pi, T *__restrict__ inv, double *__restrict__ cst,
                          T *__restrict__ sis) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  T acc = 0;
  for (int d = 0; d < D; ++d) {
    T c = covs[(i64)k * D + d];
    acc += (T)log((double)c);
    inv[(i64)k * D + d] = (T)1 / c;
    sis[(i64)k * D + d] = (T)sqrt(1.0 / (double)c);
  }
  T logw = ((double)priors[k] < 1e-6) ? (T)(-INFINITY) : (T)log((double)priors[k]);
  cst[k] = (double)(T)(logw - halfDimLog2Pi) - 0.5 * (double)acc;
}

// ------------------------------------------------------------ E-step
// Log-densities of a TM x TK tile of (descriptor, component) pairs.  The
// dimension is streamed through shared memory in chunks of DC.  Each thread
// owns a register tile of 8 descriptors x 4 components: per dimension, 16-byte
// shared loads of its 8 x values, 4 means and 4 inverse variances feed 32
// updates acc += (x - mu)^2 / sigma^2.  Per (descriptor, component) the sum
// runs over the dimensions in ascending order.
template <typename T, int TM, int TK, int DC>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? 3 : 2) k_logp(const T *__restrict__ X, i64 N, int D, int K,
                                                  const T *__restrict__ means,
                                                  const T *__restrict__ inv,
                                                  const double *__restrict__ cst,
                                                  T *__restrict__ q) {
  constexpr int RR = 8, CC = 4, NCG = TK / CC;
  static_assert(TM * TK == kThreads * RR * CC, "one 8 x 4 register tile per thread");
  constexpr int XP = TM + 16 / (int)sizeof(T), MP = TK + 16 / (int)sizeof(T);  // padded, 16-byte rows
  constexpr int VW = 16 / (int)sizeof(T);                                     // elements per vector
  using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  __shared__ __align__(16) T sx[DC][XP];
  __shared__ __align__(16) T smu[DC][MP];
  __shared__ __align__(16) T siv[DC][MP];
  const int tid = threadIdx.x;
  const int tc = tid % NCG, tr = tid / NCG;
  const i64 i0 = (i64)blockIdx.x * TM;
  const int k0 = blockIdx.y * TK;
  T acc[RR][CC];
#pragma unroll
  for (int r = 0; r < RR; ++r)
#pragma unroll
    for (int c = 0; c < CC; ++c) acc[r][c] = 0;

  for (int d0 = 0; d0 < D; d0 += DC) {
    for (int e = tid; e < TM * DC; e += kThreads) {
      int r = e / DC, dd = e % DC;
      i64 i = i0 + r;
      int d = d0 + dd;
      sx[dd][r] = (i < N && d < D) ? X[i * D + d] : (T)0;
    }
    for (int e = tid; e < TK * DC; e += kThreads) {
      int c = e / DC, dd = e % DC;
      int k = k0 + c, d = d0 + dd;
      bool ok = (k < K && d < D);
      smu[dd][c] = ok ? means[(i64)k * D + d] : (T)0;
      siv[dd][c] = ok ? inv[(i64)k * D + d] : (T)0;
    }
    __syncthreads();
    const int dl = min(DC, D - d0);
    for (int dd = 0; dd < dl; ++dd) {
      T x[RR], m[CC], iv[CC];
#pragma unroll
      for (int u = 0; u < RR / VW; ++u) {
        const V w = *reinterpret_cast<const V *>(&sx[dd][tr * RR + u * VW]);
        const T *wp = reinterpret_cast<const T *>(&w);
#pragma unroll
        for (int e = 0; e < VW; ++e) x[u * VW + e] = wp[e];
      }
#pragma unroll
      for (int u = 0; u < CC / VW; ++u) {
        const V a = *reinterpret_cast<const V *>(&smu[dd][tc * CC + u * VW]);
        const V b = *reinterpret_cast<const V *>(&siv[dd][tc * CC + u * VW]);
        const T *ap = reinterpret_cast<const T *>(&a);
        const T *bp = reinterpret_cast<const T *>(&b);
#pragma unroll
        for (int e = 0; e < VW; ++e) {
          m[u * VW + e] = ap[e];
          iv[u * VW + e] = bp[e];
        }
      }
      if constexpr (sizeof(T) == 4) {
        // Packed fp32x2 over component pairs: each half is the scalar
        // x - mu, (x - mu)^2 and the fused (x - mu)^2 iv + acc.
        constexpr unsigned long long kNeg = 0x8000000080000000ull;
#pragma unroll
        for (int c = 0; c < CC; c += 2) {
          const unsigned long long mn = tc::f2u(m[c], m[c + 1]) ^ kNeg, ivp = tc::f2u(iv[c], iv[c + 1]);
#pragma unroll
          for (int r = 0; r < RR; ++r) {
            const unsigned long long df = tc::add2(tc::f2u(x[r], x[r]), mn);
            const unsigned long long a = tc::fma2(tc::mul2(df, df), ivp, tc::f2u(acc[r][c], acc[r][c + 1]));
            acc[r][c] = tc::lo32(a);
            acc[r][c + 1] = tc::hi32(a);
          }
        }
      } else {
#pragma unroll
        for (int r = 0; r < RR; ++r)
#pragma unroll
          for (int c = 0; c < CC; ++c) {
            T diff = x[r] - m[c];
            acc[r][c] += diff * diff * iv[c];
          }
      }
    }
    __syncthreads();
  }
  if constexpr (sizeof(T) == 4 && CC == 4) {
    // The thread's 4 components of a row in one 16-byte store.
    const int kb = k0 + tc * CC;
    if ((K & 3) == 0 && kb + CC <= K && ((uintptr_t)q & 15) == 0) {
      const double c0 = cst[kb], c1 = cst[kb + 1], c2 = cst[kb + 2], c3 = cst[kb + 3];
#pragma unroll
      for (int r = 0; r < RR; ++r) {
        const i64 i = i0 + tr * RR + r;
        if (i < N)
          *reinterpret_cast<float4 *>(q + i * K + kb) =
              make_float4((float)(c0 - 0.5 * (double)acc[r][0]), (float)(c1 - 0.5 * (double)acc[r][1]),
                          (float)(c2 - 0.5 * (double)acc[r][2]), (float)(c3 - 0.5 * (double)acc[r][3]));
      }
      return;
    }
  }
#pragma unroll
  for (int c = 0; c < CC; ++c) {
    const int k = k0 + tc * CC + c;
    if (k >= K) continue;
    const double cc = cst[k];
#pragma unroll
    for (int r = 0; r < RR; ++r) {
      const i64 i = i0 + tr * RR + r;
      if (i < N) q[i * K + k] = (T)(cc - 0.5 * (double)acc[r][c]);
    }
  }
}

// Row-wise log-sum-exp normalisation (vl/gmm.c:776-790), one warp per row,
// plus the optional FAST one-hot (vl/fisher.c:398-417: first arg-max wins).
template <typename T>
__global__ void __launch_bounds__(kThreads) k_normalize(T *__restrict__ q, i64 N, int K, int fast,
                                                       double *__restrict__ ll_part) {
  constexpr int W = kThreads / 32;
  __shared__ double sll[W];
  const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
  const i64 i = (i64)blockIdx.x * W + w;
  double llrow = 0;
  if (i < N) {
    T *row = q + i * K;
    T mx = (T)(-INFINITY);
    for (int k = lane; k < K; k += 32) mx = max(mx, row[k]);
    mx = warp_max(mx);
    T sum = 0;
    for (int k = lane; k < K; k += 32) {
      T e = dexp(row[k] - mx);
      row[k] = e;
      sum += e;
    }
    sum = warp_sum(sum);
    llrow = log((double)sum) + (double)mx;
    T bv = (T)(-INFINITY);
    int bi = 0x7fffffff;
    for (int k = lane; k < K; k += 32) {
      T v = row[k] / sum;
      row[k] = v;
      if (v > bv) { bv = v; bi = k; }
    }
    if (fast) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        T ov = __shfl_xor_sync(0xffffffffu, bv, o);
        int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
      }
      if (bi == 0x7fffffff) bi = 0;  // all-NaN row: the reference keeps index 0
      for (int k = lane; k < K; k += 32) row[k] = (T)(k == bi);
    }
  }
  if (lane == 0) sll[w] = llrow;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int j = 0; j < W; ++j) s += sll[j];
    ll_part[blockIdx.x] = s;
  }
}

// One-hot of each row's first arg-max (vl/fisher.c:398-417), one warp per row.
__global__ void __launch_bounds__(kThreads) k_onehot(float *__restrict__ q, i64 N, int K) {
  const i64 i = (i64)blockIdx.x * (kThreads / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (i >= N) return;
  float *row = q + i * K;
  float bv = -INFINITY;
  int bi = 0x7fffffff;
  for (int k = lane; k < K; k += 32)
    if (row[k] > bv) { bv = row[k]; bi = k; }
  for (int o = 16; o > 0; o >>= 1) {
    const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
  }
  if (bi == 0x7fffffff) bi = 0;
  __syncwarp();
  for (int k = lane; k < K; k += 32) row[k] = (float)(k == bi);
}

__global__ void k_sum_doubles(const double *__restrict__ part, i64 n, double *__restrict__ out) {
  __shared__ double sh[kThreads];
  double s = 0;
  for (i64 j = threadIdx.x; j < n; j += kThreads) s += part[j];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = kThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

// ------------------------------------------------------------ M-step
// Thresholded sufficient statistics over one slab of rows for TKC components
// and a block of 8*JMAX dimensions (vl/gmm.c:1093-1149):
//   mass = sum q, S1 = sum q x, S2 = sum q (x - mu_old)^2, with q < 1e-2/K
//   skipped.  Partials are written per slab in double.
template <typename T, int TKC, int RC, int JMAX>
__global__ void __launch_bounds__(kThreads) k_mstep_stats(
    const T *__restrict__ X, const T *__restrict__ q, i64 N, int K, int D, i64 rowsPerSlab,
    const T *__restrict__ oldMeans, double *__restrict__ pmass, double *__restrict__ ps1,
    double *__restrict__ ps2) {
  constexpr int DB = 8 * JMAX;
  __shared__ __align__(16) T sx[RC][DB];
  __shared__ T sq[RC][TKC];
  __shared__ T smo[DB][TKC + 1];
  const int tid = threadIdx.x, c = tid % TKC, dg = tid / TKC;
  const int slab = blockIdx.x, k0 = blockIdx.y * TKC, dbase = blockIdx.z * DB;
  const i64 r0 = (i64)slab * rowsPerSlab;
  const i64 r1 = min(N, r0 + rowsPerSlab);
  const double thr = 1e-2 / (double)K;
  for (int e = tid; e < TKC * DB; e += kThreads) {
    int cc = e / DB, dd = e % DB;
    int k = k0 + cc, d = dbase + dd;
    smo[dd][cc] = (k < K && d < D) ? oldMeans[(i64)k * D + d] : (T)0;
  }
  T s1[JMAX], s2[JMAX], mass = 0;
#pragma unroll
  for (int j = 0; j < JMAX; ++j) s1[j] = s2[j] = 0;
  for (i64 rb = r0; rb < r1; rb += RC) {
    const int rc = (int)min((i64)RC, r1 - rb);
    __syncthreads();
    for (int e = tid; e < RC * DB; e += kThreads) {
      int r = e / DB, dd = e % DB, d = dbase + dd;
      sx[r][dd] = (r < rc && d < D) ? X[(rb + r) * D + d] : (T)0;
    }
    for (int e = tid; e < RC * TKC; e += kThreads) {
      int r = e / TKC, cc = e % TKC, k = k0 + cc;
      T v = (r < rc && k < K) ? q[(rb + r) * K + k] : (T)0;
      sq[r][cc] = ((double)v < thr) ? (T)0 : v;
    }
    __syncthreads();
    if constexpr (sizeof(T) == 4 && JMAX % 2 == 0) {
      // Packed fp32x2 over dimension pairs (j, j + 1): each half is the
      // scalar x - mu_old, its square, p x + s1 and p (x - mu_old)^2 + s2.
      constexpr unsigned long long kNeg = 0x8000000080000000ull;
      unsigned long long mo[JMAX / 2], a1[JMAX / 2], a2[JMAX / 2];
#pragma unroll
      for (int j = 0; j < JMAX; j += 2) {
        mo[j / 2] = tc::f2u(smo[dg + 8 * j][c], smo[dg + 8 * j + 8][c]) ^ kNeg;
        a1[j / 2] = tc::f2u(s1[j], s1[j + 1]);
        a2[j / 2] = tc::f2u(s2[j], s2[j + 1]);
      }
      for (int r = 0; r < rc; ++r) {
        const T p = sq[r][c];
        if (p == (T)0) continue;
        mass += p;
        const unsigned long long pp = tc::f2u(p, p);
#pragma unroll
        for (int j = 0; j < JMAX; j += 2) {
          const unsigned long long xp = tc::f2u(sx[r][dg + 8 * j], sx[r][dg + 8 * j + 8]);
          const unsigned long long df = tc::add2(xp, mo[j / 2]);
          a1[j / 2] = tc::fma2(pp, xp, a1[j / 2]);
          a2[j / 2] = tc::fma2(pp, tc::mul2(df, df), a2[j / 2]);
        }
      }
#pragma unroll
      for (int j = 0; j < JMAX; j += 2) {
        s1[j] = tc::lo32(a1[j / 2]);
        s1[j + 1] = tc::hi32(a1[j / 2]);
        s2[j] = tc::lo32(a2[j / 2]);
        s2[j + 1] = tc::hi32(a2[j / 2]);
      }
    } else {
      for (int r = 0; r < rc; ++r) {
        const T p = sq[r][c];
        if (p == (T)0) continue;
        mass += p;
#pragma unroll
        for (int j = 0; j < JMAX; ++j) {
          const int dd = dg + 8 * j;
          const T x = sx[r][dd];
          const T diff = x - smo[dd][c];
          s1[j] += p * x;
          s2[j] += p * (diff * diff);
        }
      }
    }
  }
  const int k = k0 + c;
  if (k < K) {
    const i64 base = ((i64)slab * K + k) * D;
#pragma unroll
    for (int j = 0; j < JMAX; ++j) {
      const int d = dbase + dg + 8 * j;
      if (d < D) {
        ps1[base + d] = (double)s1[j];
        ps2[base + d] = (double)s2[j];
      }
    }
    if (dg == 0 && blockIdx.z == 0) pmass[(i64)slab * K + k] = (double)mass;
  }
}

// Normalisation, old-to-new mean correction and bounds (vl/gmm.c:1169-1194);
// priors receive the mass, normalised by k_normalize_priors.
template <typename T>
__global__ void k_mstep_finalize(int nslab, int K, int D, const double *__restrict__ pmass,
                                 const double *__restrict__ ps1, const double *__restrict__ ps2,
                                 const double *__restrict__ lb, T *__restrict__ means,
                                 T *__restrict__ covs, T *__restrict__ priors) {
  i64 idx = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (i64)K * D) return;
  const int k = (int)(idx / D), d = (int)(idx % D);
  double mass = 0, S1 = 0, S2 = 0;
  for (int s = 0; s < nslab; ++s) {
    mass += pmass[(i64)s * K + k];
    S1 += ps1[((i64)s * K + k) * D + d];
    S2 += ps2[((i64)s * K + k) * D + d];
  }
  const double oldmu = (double)means[idx];
  double mu = S1, v = S2;
  if (mass >= 1e-6 / (double)K) {
    mu = S1 / mass;
    v = S2 / mass;
    const double df = mu - oldmu;
    v -= df * df;
  }
  T vt = (T)v;
  if ((double)vt < lb[d]) vt = (T)lb[d];
  means[idx] = (T)mu;
  covs[idx] = vt;
  if (d == 0) priors[k] = (T)mass;
}

template <typename T>
__global__ void k_normalize_priors(T *__restrict__ priors, int K) {
  __shared__ double sh[kThreads];
  double s = 0;
  for (int k = threadIdx.x; k < K; k += kThreads) s += (double)priors[k];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = kThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  double tot = sh[0];
  if (tot < 1e-12) tot = 1e-12;
  for (int k = threadIdx.x; k < K; k += kThreads) priors[k] = (T)((double)priors[k] / tot);
}

template <typename T>
__global__ void k_apply_bounds(T *__restrict__ covs, i64 n, int D, const double *__restrict__ lb) {
  i64 idx = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const int d = (int)(idx % D);
  if ((double)covs[idx] < lb[d]) covs[idx] = (T)lb[d];
}

// Column sums of the posteriors per slab (vl/gmm.c:835-844).
template <typename T>
__global__ void k_colmass(const T *__restrict__ q, i64 N, int K, i64 rowsPerSlab,
                          double *__restrict__ part) {
  const i64 r0 = (i64)blockIdx.x * rowsPerSlab, r1 = min(N, r0 + rowsPerSlab);
  for (int k = threadIdx.x; k < K; k += kThreads) {
    double s = 0;
    for (i64 i = r0; i < r1; ++i) s += (double)q[i * K + k];
    part[(i64)blockIdx.x * K + k] = s;
  }
}

// The same sums for fp32 posteriors with K a multiple of 4 (K <= 1024):
// each thread reads four columns as a float4, the block covers
// 1024 / K rows per pass (coalesced 16-byte loads), four rows per thread are
// in flight, and the row groups are summed in index order at the end.
__global__ void __launch_bounds__(kThreads) k_colmass4(const float *__restrict__ q, i64 N, int K,
                                                       i64 rowsPerSlab, double *__restrict__ part) {
  __shared__ double sh[4 * kThreads];  // [row group][column]
  const int tpr = K / 4, rpb = kThreads / tpr;
  const int rg = threadIdx.x / tpr, c4 = threadIdx.x % tpr;
  const i64 r0 = (i64)blockIdx.x * rowsPerSlab, r1 = min(N, r0 + rowsPerSlab);
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  if (rg < rpb) {
    i64 i = r0 + rg;
    for (; i + 3 * rpb < r1; i += 4 * rpb) {
      float4 v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) v[u] = __ldg((const float4 *)(q + (i + u * rpb) * K) + c4);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        s0 += (double)v[u].x;
        s1 += (double)v[u].y;
        s2 += (double)v[u].z;
        s3 += (double)v[u].w;
      }
    }
    for (; i < r1; i += rpb) {
      const float4 v = __ldg((const float4 *)(q + i * K) + c4);
      s0 += (double)v.x;
      s1 += (double)v.y;
      s2 += (double)v.z;
      s3 += (double)v.w;
    }
    double *row = sh + rg * K + 4 * c4;
    row[0] = s0;
    row[1] = s1;
    row[2] = s2;
    row[3] = s3;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < K; k += kThreads) {
    double t = 0;
    for (int g = 0; g < rpb; ++g) t += sh[g * K + k];
    part[(i64)blockIdx.x * K + k] = t;
  }
}

__global__ void k_sum_slabs(const double *__restrict__ part, int nslab, int K,
                            double *__restrict__ out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  double s = 0;
  for (int j = 0; j < nslab; ++j) s += part[(i64)j * K + k];
  out[k] = s;
}

template <typename T>
__global__ void k_restart_split(T *__restrict__ q, const T *__restrict__ X, i64 N, int K, int D,
                                int icl, int best, int dim, T cut) {
  i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  T p = q[i * K + best], r = q[i * K + icl];
  if (X[i * D + dim] < cut) {
    q[i * K + icl] = p + r;
    q[i * K + best] = 0;
  } else {
    q[i * K + icl] = 0;
    q[i * K + best] = p + r;
  }
}

// ------------------------------------------------------------ Fisher
// Fisher statistics of one segment for TKC components and a block of
// 8*JMAX dimensions (vl/fisher.c:419-449): for pi_k >= 1e-6 and q >= 1e-6,
// u += q (x-mu) s, v += q ((x-mu)^2 s^2 - 1); counts the accumulated terms.
template <typename T, int TKC, int RC, int JMAX>
__global__ void __launch_bounds__(kThreads) k_fisher_stats(
    const T *__restrict__ X, const T *__restrict__ q, i64 qbase, int K, int D,
    const Segment *__restrict__ segs, const T *__restrict__ means, const T *__restrict__ sis,
    const T *__restrict__ priors, double *__restrict__ pu, double *__restrict__ pv,
    unsigned long long *__restrict__ pnt) {
  constexpr int DB = 8 * JMAX;
  __shared__ __align__(16) T sx[RC][DB];
  __shared__ T sq[RC][TKC];
  __shared__ T smu[DB][TKC + 1];
  __shared__ T ssi[DB][TKC + 1];
  const int tid = threadIdx.x, c = tid % TKC, dg = tid / TKC;
  const int sidx = blockIdx.x, k0 = blockIdx.y * TKC, dbase = blockIdx.z * DB;
  const Segment sg = segs[sidx];
  for (int e = tid; e < TKC * DB; e += kThreads) {
    int cc = e / DB, dd = e % DB;
    int k = k0 + cc, d = dbase + dd;
    bool ok = (k < K && d < D);
    smu[dd][cc] = ok ? means[(i64)k * D + d] : (T)0;
    ssi[dd][cc] = ok ? sis[(i64)k * D + d] : (T)0;
  }
  const int k = k0 + c;
  const bool active = (k < K) && ((double)priors[k] >= 1e-6);
  T u[JMAX], v[JMAX];
#pragma unroll
  for (int j = 0; j < JMAX; ++j) u[j] = v[j] = 0;
  unsigned long long nt = 0;
  for (i64 rb = sg.row0; rb < sg.row1; rb += RC) {
    const int rc = (int)min((i64)RC, sg.row1 - rb);
    __syncthreads();
    for (int e = tid; e < RC * DB; e += kThreads) {
      int r = e / DB, dd = e % DB, d = dbase + dd;
      sx[r][dd] = (r < rc && d < D) ? X[(rb + r) * D + d] : (T)0;
    }
    for (int e = tid; e < RC * TKC; e += kThreads) {
      int r = e / TKC, cc = e % TKC, kk = k0 + cc;
      T val = (r < rc && kk < K) ? q[(rb + r - qbase) * K + kk] : (T)0;
      sq[r][cc] = ((double)val < 1e-6) ? (T)0 : val;
    }
    __syncthreads();
    if (!active) continue;
    if constexpr (sizeof(T) == 4 && JMAX % 2 == 0) {
      // Packed fp32x2 over dimension pairs (j, j + 1): each half is the
      // scalar (x - mu) sigma^-1, p df + u and p (df^2 - 1) + v.
      constexpr unsigned long long kNeg = 0x8000000080000000ull, kMinus1 = 0xbf800000bf800000ull;
      unsigned long long mn[JMAX / 2], si[JMAX / 2], au[JMAX / 2], av[JMAX / 2];
#pragma unroll
      for (int j = 0; j < JMAX; j += 2) {
        mn[j / 2] = tc::f2u(smu[dg * JMAX + j][c], smu[dg * JMAX + j + 1][c]) ^ kNeg;
        si[j / 2] = tc::f2u(ssi[dg * JMAX + j][c], ssi[dg * JMAX + j + 1][c]);
        au[j / 2] = tc::f2u(u[j], u[j + 1]);
        av[j / 2] = tc::f2u(v[j], v[j + 1]);
      }
      for (int r = 0; r < rc; ++r) {
        const T p = sq[r][c];
        if (p == (T)0) continue;
        ++nt;
        const unsigned long long pp = tc::f2u(p, p);
        const unsigned long long *xr = reinterpret_cast<const unsigned long long *>(&sx[r][dg * JMAX]);
#pragma unroll
        for (int j = 0; j < JMAX; j += 2) {
          const unsigned long long xp = xr[j / 2];
          const unsigned long long df = tc::mul2(tc::add2(xp, mn[j / 2]), si[j / 2]);
          au[j / 2] = tc::fma2(pp, df, au[j / 2]);
          av[j / 2] = tc::fma2(pp, tc::fma2(df, df, kMinus1), av[j / 2]);
        }
      }
#pragma unroll
      for (int j = 0; j < JMAX; j += 2) {
        u[j] = tc::lo32(au[j / 2]);
        u[j + 1] = tc::hi32(au[j / 2]);
        v[j] = tc::lo32(av[j / 2]);
        v[j + 1] = tc::hi32(av[j / 2]);
      }
    } else {
      for (int r = 0; r < rc; ++r) {
        const T p = sq[r][c];
        if (p == (T)0) continue;
        ++nt;
#pragma unroll
        for (int j = 0; j < JMAX; ++j) {
          const int dd = dg * JMAX + j;
          const T df = (sx[r][dd] - smu[dd][c]) * ssi[dd][c];
          u[j] += p * df;
          v[j] += p * (df * df - (T)1);
        }
      }
    }
  }
  if (k < K) {
    const i64 base = ((i64)sidx * K + k) * D;
#pragma unroll
    for (int j = 0; j < JMAX; ++j) {
      const int d = dbase + dg * JMAX + j;
      if (d < D) {
        pu[base + d] = (double)u[j];
        pv[base + d] = (double)v[j];
      }
    }
    if (dg == 0 && blockIdx.z == 0) pnt[(i64)sidx * K + k] = nt;
  }
}

// Asynchronous global -> shared copies (16 or 4 bytes; bytes past srcBytes
// are zero-filled and nothing is read for them).
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t srcBytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(srcBytes) : "memory");
}
__device__ __forceinline__ void cp_async4(uint32_t dst, const void *src, uint32_t srcBytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src), "r"(srcBytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Thresholded statistics visiting only the (row, component) pairs that pass
// the skip, for float data up to 128 dimensions:
//  - kSpFisher: k_fisher_stats' statistics (vl/fisher.c:419-449): per segment,
//    for pi_k >= 1e-6 and q >= 1e-6, u += q df, v += q (df^2 - 1) with
//    df = (x - mu) s, and the term counts;
//  - kSpMstep: k_mstep_stats' statistics (vl/gmm.c:1093-1149): per slab, for
//    q >= 1e-2/K, mass += q, S1 += q x, S2 += q (x - mu_old)^2.
// A block takes one segment (or slab) and KB components, all dimensions;
// 32-row chunks of x and of the block's posterior columns are double-buffered
// in shared memory by cp.async.  Warp w owns the components w, w + 16, ...:
// per chunk and component it ballots the rows that pass and walks them in row
// order, lanes over dimensions, with the accumulators in registers.  Per
// (component, dimension) the operations and their order are the dense
// kernels' (fused multiply-adds as there, rows ascending), so the partials are
// the same bits; the dense kernels spend their time on the pairs the skip
// removes (about 94% of them on typical posteriors).
constexpr int kFsThreads = 512, kFsRC = 32;
enum { kSpFisher = 0, kSpMstep = 1 };

struct SparseStatsArgs {
  const float *X;        // rows indexed from the call's first row
  const float *q;        // N x K posteriors, row (r - qbase)
  i64 qbase;
  float thr;             // the smallest float >= the skip threshold
  int K, D;
  const Segment *segs;   // kSpFisher: the segments
  i64 N, rowsPerSlab;    // kSpMstep: slab s is rows [s rps, min(N, (s + 1) rps))
  const float *mu;       // means (kSpFisher) or old means (kSpMstep)
  const float *sis;      // kSpFisher: 1 / sigma
  const float *priors;   // kSpFisher
  double *p1, *p2;       // u, v (kSpFisher) or S1, S2 (kSpMstep): [block][K][D]
  unsigned long long *pnt;  // kSpFisher: term counts [segment][K]
  double *pmass;            // kSpMstep: [slab][K]
  int vec16;
};

// KB: components per block (128, or 64 above 96 dimensions, where the
// accumulators of 8 components per warp would not fit in registers).
size_t sparse_stats_smem(int D, int KB) {
  return sizeof(float) * ((size_t)2 * KB * D + (size_t)2 * kFsRC * D + (size_t)2 * kFsRC * (KB + 4));
}

template <int MODE, int DPL, int kFsKB>
__global__ void __launch_bounds__(kFsThreads, 1) k_stats_sparse(const SparseStatsArgs a) {
  constexpr int NW = kFsThreads / 32, CPW = kFsKB / NW, kFsQP = kFsKB + 4;
  extern __shared__ __align__(16) float fs_smem[];
  const int K = a.K, D = a.D;
  const float *__restrict__ X = a.X;
  const float *__restrict__ q = a.q;
  float *smu = fs_smem;               // [KB][D]
  float *ssi = smu + kFsKB * D;       // [KB][D] (kSpFisher)
  float *sx = ssi + kFsKB * D;        // [2][RC][D]
  float *sq = sx + 2 * kFsRC * D;     // [2][RC][QP]
  const int tid = threadIdx.x, w = tid / 32, lane = tid % 32;
  const int sidx = blockIdx.x, k0 = blockIdx.y * kFsKB;
  i64 row0, row1;
  if constexpr (MODE == kSpFisher) {
    const Segment sg = a.segs[sidx];
    row0 = sg.row0;
    row1 = sg.row1;
  } else {
    row0 = (i64)sidx * a.rowsPerSlab;
    row1 = min(a.N, row0 + a.rowsPerSlab);
  }
  const i64 rows = row1 - row0;
  const int nch = (int)((rows + kFsRC - 1) / kFsRC);
  const i64 qbase = a.qbase;

  auto issue = [&](int ch) {
    const int b = ch & 1;
    const i64 rb = row0 + (i64)ch * kFsRC;
    const int rc = (int)min((i64)kFsRC, row1 - rb);
    float *bx = sx + b * kFsRC * D, *bq = sq + b * kFsRC * kFsQP;
    // The chunk's x rows are one contiguous range (rows past rc are never read).
    const float *xs = X + rb * D;
    if (a.vec16) {
      for (int e = tid; e < rc * D / 4; e += kFsThreads) cp_async16(tc::smem_u32(bx + 4 * e), xs + 4 * e, 16u);
      for (int e = tid; e < kFsRC * (kFsKB / 4); e += kFsThreads) {
        const int r = e / (kFsKB / 4), c4 = e % (kFsKB / 4), kk = k0 + 4 * c4;
        const bool ok = r < rc && kk < K;
        cp_async16(tc::smem_u32(bq + r * kFsQP + 4 * c4), ok ? q + (rb + r - qbase) * K + kk : q, ok ? 16u : 0u);
      }
    } else {
      for (int e = tid; e < rc * D; e += kFsThreads) cp_async4(tc::smem_u32(bx + e), xs + e, 4u);
      for (int e = tid; e < kFsRC * kFsKB; e += kFsThreads) {
        const int r = e / kFsKB, c = e % kFsKB, kk = k0 + c;
        const bool ok = r < rc && kk < K;
        cp_async4(tc::smem_u32(bq + r * kFsQP + c), ok ? q + (rb + r - qbase) * K + kk : q, ok ? 4u : 0u);
      }
    }
    cp_async_commit();
  };

  if (nch > 0) issue(0);
  for (int e = tid; e < kFsKB * D; e += kFsThreads) {
    const int kl = e / D, d = e - kl * D, k = k0 + kl;
    smu[e] = k < K ? a.mu[(i64)k * D + d] : 0.f;
    if constexpr (MODE == kSpFisher) ssi[e] = k < K ? a.sis[(i64)k * D + d] : 0.f;
  }
  // The skip: values below thr (compared in double, i.e. below a.thr as
  // floats; NaN passes in both) and zeros.
  const float thr = a.thr;
  bool act[CPW];
  float u[CPW][DPL], v[CPW][DPL], mass[CPW];
  unsigned nt[CPW];  // at most the segment's rows
#pragma unroll
  for (int c = 0; c < CPW; ++c) {
    const int k = k0 + w + NW * c;
    if constexpr (MODE == kSpFisher) act[c] = k < K && (double)a.priors[k] >= 1e-6;
    else act[c] = k < K;
    nt[c] = 0;
    mass[c] = 0.f;
#pragma unroll
    for (int j = 0; j < DPL; ++j) u[c][j] = v[c][j] = 0.f;
  }
  for (int ch = 0; ch < nch; ++ch) {
    if (ch + 1 < nch) {
      issue(ch + 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const float *bx = sx + (ch & 1) * kFsRC * D, *bq = sq + (ch & 1) * kFsRC * kFsQP;
    const int rc = (int)min((i64)kFsRC, rows - (i64)ch * kFsRC);
#pragma unroll
    for (int c = 0; c < CPW; ++c) {
      if (!act[c]) continue;  // warp-uniform
      const int kl = w + NW * c;
      const float val = bq[lane * kFsQP + kl];
      unsigned m = __ballot_sync(0xffffffffu, lane < rc && !(val < thr) && val != 0.f);
      nt[c] += (unsigned)__popc(m);
      float mu[DPL], si[DPL];
#pragma unroll
      for (int j = 0; j < DPL; ++j) {
        const int d = lane + 32 * j;
        mu[j] = d < D ? smu[kl * D + d] : 0.f;
        if constexpr (MODE == kSpFisher) si[j] = d < D ? ssi[kl * D + d] : 0.f;
      }
      while (m) {
        const int r = __ffs(m) - 1;
        m &= m - 1;
        const float p = bq[r * kFsQP + kl];
        if constexpr (MODE == kSpMstep) mass[c] += p;
#pragma unroll
        for (int j = 0; j < DPL; ++j) {
          const int d = lane + 32 * j;
          if (d < D) {
            const float x = bx[r * D + d];
            if constexpr (MODE == kSpFisher) {
              const float df = (x - mu[j]) * si[j];
              u[c][j] = fmaf(p, df, u[c][j]);
              v[c][j] = fmaf(p, fmaf(df, df, -1.f), v[c][j]);
            } else {
              const float df = x - mu[j];
              u[c][j] = fmaf(p, x, u[c][j]);
              v[c][j] = fmaf(p, df * df, v[c][j]);
            }
          }
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int c = 0; c < CPW; ++c) {
    const int k = k0 + w + NW * c;
    if (k >= K) continue;
    const i64 base = ((i64)sidx * K + k) * D;
#pragma unroll
    for (int j = 0; j < DPL; ++j) {
      const int d = lane + 32 * j;
      if (d < D) {
        a.p1[base + d] = (double)u[c][j];
        a.p2[base + d] = (double)v[c][j];
      }
    }
    if (lane == 0) {
      if constexpr (MODE == kSpFisher) a.pnt[(i64)sidx * K + k] = (unsigned long long)nt[c];
      else a.pmass[(i64)sidx * K + k] = (double)mass[c];
    }
  }
}

// Launches k_stats_sparse over nblk segments (or slabs); false when the shape
// is outside it (the dense kernel runs instead).
template <int MODE>
bool launch_stats_sparse(SparseStatsArgs a, i64 nblk, cudaStream_t s) {
  if (a.D > 128 || nblk <= 0) return false;
  const int dpl = (a.D + 31) / 32, kb = dpl == 4 ? 64 : 128;
  auto kern = dpl == 1 ? k_stats_sparse<MODE, 1, 128>
              : dpl == 2 ? k_stats_sparse<MODE, 2, 128>
              : dpl == 3 ? k_stats_sparse<MODE, 3, 128>
                         : k_stats_sparse<MODE, 4, 64>;
  const size_t smem = sparse_stats_smem(a.D, kb);
  VLB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  a.vec16 = (a.D % 4 == 0 && a.K % 4 == 0 && ((uintptr_t)a.X & 15) == 0 && ((uintptr_t)a.q & 15) == 0) ? 1 : 0;
  // (double)v < t for a float v exactly when v < tf, tf the smallest float >= t.
  const double t = MODE == kSpFisher ? 1e-6 : 1e-2 / (double)a.K;
  float tf = (float)t;
  if ((double)tf < t) tf = std::nextafter(tf, INFINITY);
  a.thr = tf;
  dim3 g((unsigned)nblk, (unsigned)((a.K + kb - 1) / kb));
  VLB_LAUNCH(MODE == kSpFisher ? "exact_fisher_stats" : "exact_mstep_stats", s,
             kern<<<g, kFsThreads, smem, s>>>(a));
  return true;
}

// Per-image Fisher finalisation (vl/fisher.c:450-485): sum the image's
// segment partials, scale u by 1/(N sqrt pi) and v by 1/(N sqrt(2 pi)),
// signed square root, global L2 normalisation.  One block per image.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_fisher_finalize(
    int K, int D, const int *__restrict__ imgSegBegin, const i64 *__restrict__ imgRows,
    const double *__restrict__ pu, const double *__restrict__ pv,
    const unsigned long long *__restrict__ pnt, const T *__restrict__ priors, int flags,
    i64 imgBase, T *__restrict__ enc, unsigned long long *__restrict__ nterms) {
  __shared__ double sh[kThreads];
  __shared__ unsigned long long shn[kThreads];
  // Per-component factors 1 / (n sqrt(pi_k)) and 1 / (n sqrt(2 pi_k)), formed
  // once per image (-1: the component is skipped, its entries are 0).
  constexpr int kFinK = 2048;
  __shared__ double sfu[kFinK], sfv[kFinK];
  const int img = blockIdx.x;
  const int s0 = imgSegBegin[img], s1 = imgSegBegin[img + 1];
  const i64 n = imgRows[img];
  const i64 KD = (i64)K * D;
  T *out = enc + (imgBase + img) * 2 * KD;
  auto factor = [&](int k, bool isv) -> double {
    const double pk = (double)priors[k];
    if (!(pk >= 1e-6 && n > 0)) return -1.0;
    return isv ? 1.0 / ((double)n * sqrt(2.0 * pk)) : 1.0 / ((double)n * sqrt(pk));
  };
  const bool cached = K <= kFinK;
  if (cached) {
    for (int k = threadIdx.x; k < K; k += kThreads) {
      sfu[k] = factor(k, false);
      sfv[k] = factor(k, true);
    }
    __syncthreads();
  }
  const bool small = KD <= (i64)INT32_MAX;
  double sq = 0;
  for (i64 e = threadIdx.x; e < 2 * KD; e += kThreads) {
    const bool isv = e >= KD;
    const i64 kd = isv ? e - KD : e;
    const int k = small ? (int)((unsigned)kd / (unsigned)D) : (int)(kd / D);
    double acc = 0;
    for (int s = s0; s < s1; ++s) acc += isv ? pv[(i64)s * KD + kd] : pu[(i64)s * KD + kd];
    const double f = cached ? (isv ? sfv[k] : sfu[k]) : factor(k, isv);
    const double z = f >= 0.0 ? acc * f : 0.0;
    T zt = (T)z;
    // For float, sqrtf is the float rounding of the double square root (double
    // rounding is innocuous for sqrt with 53 >= 2 x 24 + 2 bits).
    if (flags & 1) {
      if constexpr (sizeof(T) == 4) zt = zt >= 0.f ? sqrtf(zt) : -sqrtf(-zt);
      else zt = zt >= (T)0 ? (T)sqrt((double)zt) : -(T)sqrt(-(double)zt);
    }
    out[e] = zt;
    sq += (double)zt * (double)zt;
  }
  unsigned long long nt = 0;
  for (i64 e = threadIdx.x; e < K; e += kThreads)
    for (int s = s0; s < s1; ++s) nt += pnt[(i64)s * K + e];
  sh[threadIdx.x] = sq;
  shn[threadIdx.x] = nt;
  __syncthreads();
  for (int o = kThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sh[threadIdx.x] += sh[threadIdx.x + o];
      shn[threadIdx.x] += shn[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && nterms) nterms[imgBase + img] = shn[0];
  if (flags & 2) {
    double nrm = sqrt(sh[0]);
    if (nrm < 1e-12) nrm = 1e-12;
    const T nt_ = (T)nrm;
    for (i64 e = threadIdx.x; e < 2 * KD; e += kThreads) out[e] = out[e] / nt_;
  }
}

template <typename T>
T half_dim_log_2pi(i64 D) {
  return (T)(((double)D / 2.0) * log(2.0 * 3.141592653589793));
}

inline unsigned grid1(i64 n, int b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

// ================================================================ launchers

template <typename T>
void exact_prepare(const DevModel<T> &m, DevDerived<T> &der, cudaStream_t s) {
  VLB_LAUNCH("exact_prepare", s,
             k_prepare<T><<<grid1(m.K, 128), 128, 0, s>>>(m.priors, m.covs, (int)m.K, (int)m.D,
                                                          half_dim_log_2pi<T>(m.D), der.inv,
                                                          der.cst, der.sis));
}

// Capacity bound for any E-step kernel: the exact kernels write one partial
// per 8 rows; the tensor-core E-step 8 per 128-row tile.
i64 estep_ll_parts(i64 N) { return std::max<i64>((N + 7) / 8 + 1, 8 * ((N + 127) / 128) + 8); }

template <typename T>
i64 exact_estep(const T *X, i64 N, const DevModel<T> &m, const DevDerived<T> &der, T *q,
                double *ll_part, bool fast, cudaStream_t s) {
  if (N <= 0) return 0;
  constexpr int TM = 128, TK = 64, DC = sizeof(T) == 4 ? 32 : 16;  // 34 KB of tiles either way
  dim3 g(grid1(N, TM), grid1(m.K, TK));
  VLB_LAUNCH("exact_logp", s,
             (k_logp<T, TM, TK, DC><<<g, kThreads, 0, s>>>(X, N, (int)m.D, (int)m.K, m.means,
                                                           der.inv, der.cst, q)));
  VLB_LAUNCH("exact_normalize", s,
             k_normalize<T><<<grid1(N, 8), kThreads, 0, s>>>(q, N, (int)m.K, fast ? 1 : 0,
                                                             ll_part));
  return (i64)grid1(N, 8);
}

void sum_doubles(const double *part, i64 n, double *out, cudaStream_t s) {
  VLB_LAUNCH("sum_doubles", s, k_sum_doubles<<<1, kThreads, 0, s>>>(part, n, out));
}

namespace {
i64 pick_slab_rows(i64 N) {
  // About 2 slabs per SM for large N; at least 256 rows per slab.
  i64 slabs = 296;
  i64 r = (N + slabs - 1) / slabs;
  if (r < 256) r = 256;
  return r;
}
}  // namespace

// The M-step statistics of nslab slabs of rows by the sparse kernel (float
// data up to 128 dimensions); false when the dense kernel is to run.
template <typename T>
bool mstep_stats_sparse(const T *X, const T *q, i64 N, i64 K, i64 D, i64 rps, i64 nslab, const T *oldMeans,
                        double *pmass, double *ps1, double *ps2, cudaStream_t s) {
  if constexpr (sizeof(T) == 4) {
    SparseStatsArgs a{};
    a.X = X; a.q = q; a.qbase = 0; a.K = (int)K; a.D = (int)D; a.N = N; a.rowsPerSlab = rps;
    a.mu = oldMeans; a.p1 = ps1; a.p2 = ps2; a.pmass = pmass;
    return launch_stats_sparse<kSpMstep>(a, nslab, s);
  }
  return false;
}

template <typename T>
void exact_mstep(const T *X, i64 N, const T *q, T *means, T *covs, T *priors, i64 K, i64 D,
                 const double *lb, cudaStream_t s) {
  constexpr int TKC = 32, RC = 32, JMAX = sizeof(T) == 8 ? 8 : 16, DB = 8 * JMAX;
  const i64 rps = pick_slab_rows(N > 0 ? N : 1);
  const int nslab = (int)((N + rps - 1) / rps > 0 ? (N + rps - 1) / rps : 1);
  Scratch &sc = thread_scratch(kArenaExact);
  double *pmass = sc.slot[10].get<double>((size_t)nslab * K);
  double *ps1 = sc.slot[11].get<double>((size_t)nslab * K * D);
  double *ps2 = sc.slot[12].get<double>((size_t)nslab * K * D);
  if (N > 0) {
    if (!mstep_stats_sparse<T>(X, q, N, K, D, rps, nslab, means, pmass, ps1, ps2, s)) {
      dim3 g(nslab, grid1(K, TKC), grid1(D, DB));
      VLB_LAUNCH("exact_mstep_stats", s,
                 (k_mstep_stats<T, TKC, RC, JMAX><<<g, kThreads, 0, s>>>(
                     X, q, N, (int)K, (int)D, rps, means, pmass, ps1, ps2)));
    }
  } else {
    VLB_CUDA(cudaMemsetAsync(pmass, 0, sizeof(double) * nslab * K, s));
    VLB_CUDA(cudaMemsetAsync(ps1, 0, sizeof(double) * nslab * K * D, s));
    VLB_CUDA(cudaMemsetAsync(ps2, 0, sizeof(double) * nslab * K * D, s));
  }
  VLB_LAUNCH("exact_mstep_finalize", s,
             k_mstep_finalize<T><<<grid1(K * D, kThreads), kThreads, 0, s>>>(
                 nslab, (int)K, (int)D, pmass, ps1, ps2, lb, means, covs, priors));
  VLB_LAUNCH("normalize_priors", s, k_normalize_priors<T><<<1, kThreads, 0, s>>>(priors, (int)K));
}

i64 exact_mstep_slab_rows(i64 N) { return pick_slab_rows(N > 0 ? N : 1); }

template <typename T>
void exact_mstep_stats_rows(const T *X, i64 row0, i64 n, i64 rps, const T *q, const T *oldMeans, i64 K,
                            i64 D, double *pmass, double *ps1, double *ps2, cudaStream_t s) {
  constexpr int TKC = 32, RC = 32, JMAX = sizeof(T) == 8 ? 8 : 16, DB = 8 * JMAX;
  if (n <= 0) return;
  VLB_CHECK(row0 % rps == 0, VL_ERR_BAD_ARG, "M-step chunk must start on a slab boundary");
  const i64 s0 = row0 / rps, nslab = (n + rps - 1) / rps;
  if (mstep_stats_sparse<T>(X + row0 * D, q, n, K, D, rps, nslab, oldMeans, pmass + s0 * K, ps1 + s0 * K * D,
                            ps2 + s0 * K * D, s))
    return;
  dim3 g((unsigned)nslab, grid1(K, TKC), grid1(D, DB));
  VLB_LAUNCH("exact_mstep_stats", s,
             (k_mstep_stats<T, TKC, RC, JMAX><<<g, kThreads, 0, s>>>(
                 X + row0 * D, q, n, (int)K, (int)D, rps, oldMeans, pmass + s0 * K, ps1 + s0 * K * D,
                 ps2 + s0 * K * D)));
}

template <typename T>
void exact_mstep_finalize_slabs(int nslab, const double *pmass, const double *ps1, const double *ps2,
                                const double *lb, T *means, T *covs, T *priors, i64 K, i64 D,
                                cudaStream_t s) {
  VLB_LAUNCH("exact_mstep_finalize", s,
             k_mstep_finalize<T><<<grid1(K * D, kThreads), kThreads, 0, s>>>(
                 nslab, (int)K, (int)D, pmass, ps1, ps2, lb, means, covs, priors));
  VLB_LAUNCH("normalize_priors", s, k_normalize_priors<T><<<1, kThreads, 0, s>>>(priors, (int)K));
}

// Slab partials summed into slab 0 in slab order (the order the finalize
// kernel uses), so that the finalize over one slab gives the same values.
__global__ void k_sum_slabs(int nslab, i64 K, i64 KD, double *__restrict__ pmass, double *__restrict__ ps1,
                            double *__restrict__ ps2) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= KD) return;
  double a = 0, b = 0, c = 0;
  for (int sl = 0; sl < nslab; ++sl) {
    if (i < K) a += pmass[(i64)sl * K + i];
    b += ps1[(i64)sl * KD + i];
    c += ps2[(i64)sl * KD + i];
  }
  if (i < K) pmass[i] = a;
  ps1[i] = b;
  ps2[i] = c;
}

void exact_sum_slabs(int nslab, double *pmass, double *ps1, double *ps2, i64 K, i64 D, cudaStream_t s) {
  VLB_LAUNCH("sum_slabs", s,
             k_sum_slabs<<<grid1(K * D, kThreads), kThreads, 0, s>>>(nslab, K, K * D, pmass, ps1, ps2));
}

template <typename T>
void normalize_priors(T *priors, i64 K, cudaStream_t s) {
  VLB_LAUNCH("normalize_priors", s, k_normalize_priors<T><<<1, kThreads, 0, s>>>(priors, (int)K));
}

template <typename T>
void column_mass(const T *q, i64 N, i64 K, double *mass, cudaStream_t s) {
  const i64 rps = pick_slab_rows(N > 0 ? N : 1);
  const int nslab = (int)((N + rps - 1) / rps > 0 ? (N + rps - 1) / rps : 1);
  double *part = thread_scratch(kArenaExact).slot[13].get<double>((size_t)nslab * K);
  if (N > 0) {
    bool done = false;
    if constexpr (sizeof(T) == 4) {
      if (K % 4 == 0 && K <= 4 * kThreads) {
        VLB_LAUNCH("column_mass", s, k_colmass4<<<nslab, kThreads, 0, s>>>((const float *)q, N, (int)K, rps, part));
        done = true;
      }
    }
    if (!done) VLB_LAUNCH("column_mass", s, k_colmass<T><<<nslab, kThreads, 0, s>>>(q, N, (int)K, rps, part));
  } else {
    VLB_CUDA(cudaMemsetAsync(part, 0, sizeof(double) * nslab * K, s));
  }
  VLB_LAUNCH("sum_slabs", s, k_sum_slabs<<<grid1(K, 128), 128, 0, s>>>(part, nslab, (int)K, mass));
}

template <typename T>
void restart_split(T *q, const T *X, i64 N, i64 K, i64 D, i64 icl, i64 best, i64 dim, T cut,
                   cudaStream_t s) {
  if (N <= 0) return;
  VLB_LAUNCH("restart_split", s,
             k_restart_split<T><<<grid1(N, kThreads), kThreads, 0, s>>>(
                 q, X, N, (int)K, (int)D, (int)icl, (int)best, (int)dim, cut));
}

template <typename T>
void apply_bounds(T *covs, i64 K, i64 D, const double *lb, cudaStream_t s) {
  VLB_LAUNCH("apply_bounds", s,
             k_apply_bounds<T><<<grid1(K * D, kThreads), kThreads, 0, s>>>(covs, K * D, (int)D, lb));
}

// Batched Fisher encoding with the exact kernels.  Images are processed in
// chunks bounded by a row budget; each image is cut into segments of at most
// kSegRows rows so long images still spread over many blocks.
template <typename T>
void exact_fisher_batch(const T *X, const i64 *h_offsets, i64 numImages, const DevModel<T> &m,
                        T *enc, unsigned long long *nterms, int flags, cudaStream_t s,
                        bool use_router) {
  const i64 K = m.K, D = m.D;
  constexpr int TKC = 32, RC = 32, JMAX = sizeof(T) == 8 ? 5 : 10, DB = 8 * JMAX;
  constexpr i64 kSegRows = 2048;
  const i64 kRowBudget = std::max<i64>(4096, (i64)(1u << 30) / (K * (i64)sizeof(T)));
  const i64 kSegBudget = std::max<i64>(64, (i64)(256u << 20) / (2 * K * D * 8));
  Scratch &sc = thread_scratch(kArenaExact);
  DevDerived<T> der;
  der.inv = sc.slot[0].get<T>(K * D);
  der.sis = sc.slot[1].get<T>(K * D);
  der.cst = sc.slot[2].get<double>(K);
  exact_prepare(m, der, s);

  i64 img = 0;
  while (img < numImages) {
    // Form one chunk of images.
    std::vector<Segment> segs;
    std::vector<int> segBegin;
    std::vector<i64> rows;
    const i64 chunkImg0 = img, row0 = h_offsets[img];
    while (img < numImages) {
      const i64 a = h_offsets[img], b = h_offsets[img + 1];
      const i64 nseg = std::max<i64>(1, (b - a + kSegRows - 1) / kSegRows);
      if (!segs.empty() && ((b - row0) > kRowBudget || (i64)segs.size() + nseg > kSegBudget)) break;
      segBegin.push_back((int)segs.size());
      rows.push_back(b - a);
      for (i64 j = 0; j < nseg; ++j) {
        i64 s0 = a + j * kSegRows, s1 = std::min(b, s0 + kSegRows);
        segs.push_back({img - chunkImg0, s0, s1});
      }
      ++img;
    }
    segBegin.push_back((int)segs.size());
    const i64 nimg = img - chunkImg0;
    const i64 row1 = h_offsets[img];
    const i64 nrows = row1 - row0;
    const i64 nseg = (i64)segs.size();

    T *q = sc.slot[3].get<T>(std::max<i64>(1, nrows) * K);
    double *llp = sc.slot[4].get<double>(estep_ll_parts(nrows));
    if (nrows > 0) {
      if constexpr (sizeof(T) == 4) {
        if (use_router) {
          router_default_posteriors(X + row0 * D, nrows, m, q, s);
          if (flags & 4) {  // FAST: one-hot of each row's arg-max
            VLB_LAUNCH("exact_onehot", s,
                       k_onehot<<<grid1(nrows, 8), kThreads, 0, s>>>(q, nrows, (int)K));
          }
        } else {
          exact_estep(X + row0 * D, nrows, m, der, q, llp, (flags & 4) != 0, s);
        }
      } else {
        exact_estep(X + row0 * D, nrows, m, der, q, llp, (flags & 4) != 0, s);
      }
    }

    Segment *dsegs = sc.slot[5].get<Segment>(nseg);
    int *dbeg = sc.slot[6].get<int>(nimg + 1);
    i64 *drows = sc.slot[7].get<i64>(nimg);
    double *pu = sc.slot[8].get<double>(nseg * K * D);
    double *pv = sc.slot[9].get<double>(nseg * K * D);
    unsigned long long *pnt = sc.slot[14].get<unsigned long long>(nseg * K);
    VLB_CUDA(cudaMemcpyAsync(dsegs, segs.data(), sizeof(Segment) * nseg, cudaMemcpyHostToDevice, s));
    VLB_CUDA(cudaMemcpyAsync(dbeg, segBegin.data(), sizeof(int) * (nimg + 1), cudaMemcpyHostToDevice, s));
    VLB_CUDA(cudaMemcpyAsync(drows, rows.data(), sizeof(i64) * nimg, cudaMemcpyHostToDevice, s));
    bool sparse = false;
    if constexpr (sizeof(T) == 4) {
      // The sparse statistics kernel (same partials, float data up to 128 dimensions).
      SparseStatsArgs a{};
      a.X = X; a.q = q; a.qbase = row0; a.K = (int)K; a.D = (int)D; a.segs = dsegs;
      a.mu = m.means; a.sis = der.sis; a.priors = m.priors; a.p1 = pu; a.p2 = pv; a.pnt = pnt;
      sparse = launch_stats_sparse<kSpFisher>(a, nseg, s);
    }
    if (!sparse) {
      dim3 g((unsigned)nseg, grid1(K, TKC), grid1(D, DB));
      VLB_LAUNCH("exact_fisher_stats", s,
                 (k_fisher_stats<T, TKC, RC, JMAX><<<g, kThreads, 0, s>>>(
                     X, q, row0, (int)K, (int)D, dsegs, m.means, der.sis, m.priors, pu, pv, pnt)));
    }
    VLB_LAUNCH("exact_fisher_finalize", s,
               k_fisher_finalize<T><<<(unsigned)nimg, kThreads, 0, s>>>(
                   (int)K, (int)D, dbeg, drows, pu, pv, pnt, m.priors, flags, chunkImg0, enc,
                   nterms));
  }
}

namespace {
constexpr i64 kFixedSegRows = 2048;

// Segment tables of one image, written on the device so a call needs no
// host-to-device copy.
__global__ void k_single_segments(i64 N, i64 nseg, Segment *segs, int *segBegin, i64 *rows) {
  for (i64 j = threadIdx.x; j < nseg; j += blockDim.x) {
    const i64 a = j * kFixedSegRows;
    segs[j] = Segment{0, a, a + kFixedSegRows < N ? a + kFixedSegRows : N};
  }
  if (threadIdx.x == 0) {
    segBegin[0] = 0;
    segBegin[1] = (int)nseg;
    rows[0] = N;
  }
}
}  // namespace

i64 exact_fv_segments(i64 N) { return N > 0 ? (N + kFixedSegRows - 1) / kFixedSegRows : 1; }

void exact_fisher_single_fixed(const float *X, i64 N, const DevModel<float> &m, float *enc,
                               unsigned long long *nterms, int flags, const ExactFvScratch &sc,
                               cudaStream_t s) {
  constexpr int TKC = 32, RC = 32, JMAX = 10, DB = 8 * JMAX;
  constexpr int TM = 128, TK = 64, DC = 32;
  const i64 K = m.K, D = m.D, nseg = exact_fv_segments(N);
  VLB_LAUNCH_PLAIN(s, k_single_segments<<<1, 32, 0, s>>>(N, nseg, sc.segs, sc.segBegin, sc.rows));
  VLB_LAUNCH_PLAIN(s, k_prepare<float><<<grid1(K, 128), 128, 0, s>>>(
                          m.priors, m.covs, (int)K, (int)D, half_dim_log_2pi<float>(D), sc.inv,
                          sc.cst, sc.sis));
  if (N > 0) {
    dim3 g(grid1(N, TM), grid1(K, TK));
    VLB_LAUNCH_PLAIN(s, (k_logp<float, TM, TK, DC><<<g, kThreads, 0, s>>>(X, N, (int)D, (int)K, m.means,
                                                                         sc.inv, sc.cst, sc.q)));
    VLB_LAUNCH_PLAIN(s, k_normalize<float><<<grid1(N, 8), kThreads, 0, s>>>(sc.q, N, (int)K,
                                                                         (flags & 4) ? 1 : 0, sc.llp));
  }
  dim3 g2((unsigned)nseg, grid1(K, TKC), grid1(D, DB));
  VLB_LAUNCH_PLAIN(s, (k_fisher_stats<float, TKC, RC, JMAX><<<g2, kThreads, 0, s>>>(
                          X, sc.q, 0, (int)K, (int)D, sc.segs, m.means, sc.sis, m.priors, sc.pu,
                          sc.pv, sc.pnt)));
  VLB_LAUNCH_PLAIN(s, k_fisher_finalize<float><<<1, kThreads, 0, s>>>(
                          (int)K, (int)D, sc.segBegin, sc.rows, sc.pu, sc.pv, sc.pnt, m.priors,
                          flags, 0, enc, nterms));
}

// ------------------------------------------------- Rand initialisation
// The reference's Rand initialisation (vl/gmm.c:1376-1443, vl/kmeans.c:
// 588-649) reproduced operation for operation: every sum runs in the data
// type and in the reference's order, multiplies and adds stay separate (the
// explicitly rounded intrinsics of exact_math.cuh never contract into a fused
// multiply-add), so the centres and variances are the reference's bits.

// Global data variance, vl/gmm.c:1376-1413: per dimension the mean, then the
// sum of squared deviations, each accumulated over the rows in order and
// divided by N and N - 1 (0 when N <= 1).  One thread per dimension.
template <typename T>
__global__ void k_global_variance(const T *__restrict__ X, i64 N, int D, T *__restrict__ sigma) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= D) return;
  if (N <= 1) {
    sigma[d] = (T)0;
    return;
  }
  T mean = (T)0;
  for (i64 i = 0; i < N; ++i) mean = add_rn(mean, X[i * D + d]);
  mean = div_rn(mean, (T)N);
  T ss = (T)0;
  for (i64 i = 0; i < N; ++i) {
    const T diff = sub_rn(X[i * D + d], mean);
    ss = add_rn(ss, mul_rn(diff, diff));
  }
  sigma[d] = div_rn(ss, (T)(N - 1));
}

// minDist[x] = min(minDist[x], ||c - x||^2) with the reference's VL_MIN.
template <typename T, int L>
__global__ void k_kpp_update(const T *__restrict__ X, i64 N, int D, const T *__restrict__ center,
                             T *__restrict__ minDist) {
  extern __shared__ unsigned char kpp_smem[];
  T *c = (T *)kpp_smem;
  for (int d = threadIdx.x; d < D; d += blockDim.x) c[d] = center[d];
  __syncthreads();
  const i64 x = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= N) return;
  const T dist = l2_ordered<T, L>(c, X + x * D, D);
  const T m = minDist[x];
  minDist[x] = m < dist ? m : dist;
}

template <typename T>
__global__ void k_fill(T *__restrict__ p, i64 n, T v) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// The next centre, vl/kmeans.c:631-641: the energy (sum of minDist in
// order), then the first x with acc >= thresh * energy, or N - 1.
// The scan's running sum acc is the energy's own prefix sum (both add minDist
// in order from 0).  So the energy pass keeps every 32nd prefix; the scan
// bisects these checkpoints (prefixes of non-negative terms never decrease, and
// a NaN prefix, then every later one, fails the test as in the loop) and
// re-adds at most 32 terms from the checkpoint before, which reproduces the
// prefixes exactly.  One sequential pass of N additions instead of two.
// One block: thread 0 adds in order out of shared memory while the warps on
// the other three schedulers stage the next chunk of minDist, so the chain
// waits on no load and shares its scheduler with no loader.
constexpr int kKppCk = 32;  // terms per checkpoint

template <typename T>
__global__ void __launch_bounds__(1024) k_kpp_select(const T *__restrict__ minDist, i64 N, T thresh,
                                                     T *__restrict__ ck, i64 *__restrict__ xOut) {
  constexpr int kChunk = 16384 / (int)sizeof(T);  // 32 KB of staging in all
  __shared__ T buf[2][kChunk];
  const int tid = threadIdx.x;
  const i64 nch = (N + kChunk - 1) / kChunk;
  auto stage = [&](i64 ch, int b, int t0, int nt) {
    const i64 base = ch * kChunk;
    const int n = (int)min((i64)kChunk, N - base);
    for (int e = t0; e < n; e += nt) buf[b][e] = minDist[base + e];
  };
  stage(0, 0, tid, blockDim.x);
  __syncthreads();
  T energy = (T)0;
  for (i64 ch = 0; ch < nch; ++ch) {
    const int b = (int)(ch & 1);
    if (tid == 0) {
      const i64 base = ch * kChunk;
      const int n = (int)min((i64)kChunk, N - base);
      int e = 0;
      for (; e + kKppCk <= n; e += kKppCk) {  // kChunk is a multiple of kKppCk
#pragma unroll
        for (int g = 0; g < kKppCk; g += 8) {
          T v[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) v[u] = buf[b][e + g + u];
#pragma unroll
          for (int u = 0; u < 8; ++u) energy = add_rn(energy, v[u]);
        }
        ck[(base + e) / kKppCk] = energy;
      }
      for (; e < n; ++e) energy = add_rn(energy, buf[b][e]);
    } else if ((tid >> 5) & 3) {
      const int w = tid >> 5, li = (w - w / 4 - 1) * 32 + (tid & 31), nl = (int)blockDim.x / 4 * 3;
      if (ch + 1 < nch) stage(ch + 1, b ^ 1, li, nl);
    }
    __syncthreads();
  }
  if (tid != 0) return;
  const T t = mul_rn(thresh, energy);
  // The first checkpoint j with ck[j] >= t (nck if none); the answer lies in
  // terms [32 j, 32 j + 32), re-added from checkpoint j - 1.
  const i64 nck = N / kKppCk;
  i64 lo = 0, hi = nck;
  while (lo < hi) {
    const i64 mid = lo + (hi - lo) / 2;
    if (ck[mid] >= t) hi = mid;
    else lo = mid + 1;
  }
  T acc = lo > 0 ? ck[lo - 1] : (T)0;
  i64 x = lo * kKppCk;
  const i64 end = min(N, x + kKppCk);
  for (; x < end; ++x) {
    acc = add_rn(acc, minDist[x]);
    if (acc >= t) break;
  }
  *xOut = min(x, N - 1);  // none before N - 1: the last row
}

// centers[c] = X[x] with x the selected row (device) or the first row (host).
template <typename T>
__global__ void k_kpp_copy(const T *__restrict__ X, int D, const i64 *__restrict__ xDev, i64 xHost,
                           T *__restrict__ dst) {
  const i64 x = xDev ? *xDev : xHost;
  for (int d = threadIdx.x; d < D; d += blockDim.x) dst[d] = X[x * D + d];
}

template <typename T>
void global_variance(const T *X, i64 N, i64 D, T *sigma, cudaStream_t s) {
  VLB_LAUNCH("global_variance", s, k_global_variance<T><<<grid1(D, 128), 128, 0, s>>>(X, N, (int)D, sigma));
}

template <typename T>
void kmeanspp(const T *X, i64 N, i64 D, i64 K, T *centers, i64 x0, const std::vector<T> &thresh, int lanes,
              cudaStream_t s) {
  VLB_CHECK((i64)thresh.size() >= K && N > 0 && K > 0 && x0 >= 0 && x0 < N, VL_ERR_BAD_ARG,
            "kmeans++: bad arguments");
  Scratch &sc = thread_scratch(kArenaExact);
  T *minDist = sc.slot[20].get<T>(N);
  i64 *xdev = sc.slot[21].get<i64>(1);
  T *ck = sc.slot[22].get<T>(N / kKppCk + 1);
  const T inf = (T)INFINITY;
  VLB_LAUNCH("kpp_fill", s, k_fill<T><<<grid1(N, kThreads), kThreads, 0, s>>>(minDist, N, inf));
  const size_t smem = sizeof(T) * D;
  for (i64 c = 0; c < K; ++c) {
    VLB_LAUNCH("kpp_copy", s, k_kpp_copy<T><<<1, 128, 0, s>>>(X, (int)D, c == 0 ? nullptr : xdev, x0,
                                                               centers + c * D));
    if (c + 1 == K) break;
    const T *ctr = centers + c * D;
    switch (lanes) {
      case 8: VLB_LAUNCH("kpp_update", s, (k_kpp_update<T, 8><<<grid1(N, kThreads), kThreads, smem, s>>>(X, N, (int)D, ctr, minDist))); break;
      case 4: VLB_LAUNCH("kpp_update", s, (k_kpp_update<T, 4><<<grid1(N, kThreads), kThreads, smem, s>>>(X, N, (int)D, ctr, minDist))); break;
      case 2: VLB_LAUNCH("kpp_update", s, (k_kpp_update<T, 2><<<grid1(N, kThreads), kThreads, smem, s>>>(X, N, (int)D, ctr, minDist))); break;
      default: VLB_LAUNCH("kpp_update", s, (k_kpp_update<T, 1><<<grid1(N, kThreads), kThreads, smem, s>>>(X, N, (int)D, ctr, minDist))); break;
    }
    VLB_LAUNCH("kpp_select", s, k_kpp_select<T><<<1, 1024, 0, s>>>(minDist, N, thresh[c], ck, xdev));
  }
}

// ------------------------------------------------------ instantiations
#define VLB_INST(T)                                                                          \
  template void exact_prepare<T>(const DevModel<T> &, DevDerived<T> &, cudaStream_t);        \
  template i64 exact_estep<T>(const T *, i64, const DevModel<T> &, const DevDerived<T> &,    \
                              T *, double *, bool, cudaStream_t);                            \
  template void exact_mstep<T>(const T *, i64, const T *, T *, T *, T *, i64, i64,           \
                               const double *, cudaStream_t);                                \
  template void column_mass<T>(const T *, i64, i64, double *, cudaStream_t);                 \
  template void exact_mstep_stats_rows<T>(const T *, i64, i64, i64, const T *, const T *, i64, i64, \
                                          double *, double *, double *, cudaStream_t);       \
  template void exact_mstep_finalize_slabs<T>(int, const double *, const double *, const double *, \
                                              const double *, T *, T *, T *, i64, i64, cudaStream_t); \
  template void normalize_priors<T>(T *, i64, cudaStream_t);                                 \
  template void global_variance<T>(const T *, i64, i64, T *, cudaStream_t);                  \
  template void kmeanspp<T>(const T *, i64, i64, i64, T *, i64, const std::vector<T> &, int,  \
                            cudaStream_t);                                                   \
  template void restart_split<T>(T *, const T *, i64, i64, i64, i64, i64, i64, T,           \
                                 cudaStream_t);                                              \
  template void apply_bounds<T>(T *, i64, i64, const double *, cudaStream_t);                \
  template void exact_fisher_batch<T>(const T *, const i64 *, i64, const DevModel<T> &, T *, \
                                      unsigned long long *, int, cudaStream_t, bool);
VLB_INST(float)
VLB_INST(double)

}  // namespace vlb
