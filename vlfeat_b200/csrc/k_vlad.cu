// VLAD encoding (vl/vlad.c:163-242) on the GPU, with the reference's
// arithmetic operation for operation so that the encodings are its bits:
//
//   enc_k = sum_{i: a_ik > 0} a_ik x_i (each step (T)((double)enc + a * x),
//           rows in order), mass_k = sum a_ik in double;
//   mass_k > 0: enc_k = enc_k / mass_k - mu_k   (VL_VLAD_FLAG_NORMALIZE_MASS)
//               enc_k = enc_k - mass_k mu_k     (otherwise);
//   signed square root (VL_VLAD_FLAG_SQUARE_ROOT);
//   per-component L2 (VL_VLAD_FLAG_NORMALIZE_COMPONENTS) and global L2
//   (unless VL_VLAD_FLAG_UNNORMALIZED), each norm a sum of squares in the
//   data type in element order, floored at 1e-12.
//
// Multiplies and adds are explicitly rounded (no fused multiply-add, as in
// the reference build).  A batch of images is one call; image j owns rows
// [offsets[j], offsets[j+1]) of the data and of the assignments (row-major,
// numClusters per row, vl/vlad.c:173-176).
#include <algorithm>
#include <type_traits>
#include <vector>

#include "engine.h"
#include "tc_common.cuh"

extern "C" {
#include "vl/vlad.h"
#include "vlb200.h"
}

namespace vlb {
namespace {

constexpr int kVladThreads = 128;
constexpr int kVladKT = 8;  // components per block: x loads are reused across them

__device__ __forceinline__ float acc_step(float e, float a, float x) {
  return __double2float_rn(__dadd_rn((double)e, __dmul_rn((double)a, (double)x)));
}
__device__ __forceinline__ double acc_step(double e, double a, double x) { return __dadd_rn(e, __dmul_rn(a, x)); }
__device__ __forceinline__ float add_t(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_t(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_t(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_t(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul_t(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_t(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float div_t(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_t(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float sqrt_t(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double sqrt_t(double a) { return __dsqrt_rn(a); }

// One block per (image, tile of kVladKT components); thread t owns dimensions
// t + kVladThreads j, j < JD.  smem: kVladKT x D values for the component norms.
template <typename T, int JD>
__global__ void __launch_bounds__(kVladThreads) k_vlad_accum(
    T *__restrict__ enc, const T *__restrict__ means, int D, int K, const T *__restrict__ X,
    const T *__restrict__ A, const i64 *__restrict__ offs, i64 img0, int flags) {
  extern __shared__ unsigned char vlad_smem[];
  T *zs = (T *)vlad_smem;
  // The component tiles of one image are adjacent in launch order, so the
  // image's rows are read from HBM once and then from L2.
  const i64 img = img0 + blockIdx.y;
  const int k0 = blockIdx.x * kVladKT, tid = threadIdx.x;
  const int nk = min(kVladKT, K - k0);
  const i64 r0 = offs[img], r1 = offs[img + 1];
  T acc[kVladKT][JD];
  double mass[kVladKT];
#pragma unroll
  for (int c = 0; c < kVladKT; ++c) {
    mass[c] = 0.0;
#pragma unroll
    for (int j = 0; j < JD; ++j) acc[c][j] = (T)0;
  }
  // Row i+1's values are loaded while row i is accumulated.  Components past
  // the tile's end read weight 0, which the positivity test skips.
  T xn[JD], an[kVladKT];
  auto load_row = [&](i64 i) {
#pragma unroll
    for (int j = 0; j < JD; ++j) {
      const int d = tid + kVladThreads * j;
      xn[j] = d < D ? X[i * D + d] : (T)0;
    }
#pragma unroll
    for (int c = 0; c < kVladKT; ++c) an[c] = c < nk ? A[i * K + k0 + c] : (T)0;
  };
  if (r0 < r1) load_row(r0);
  for (i64 i = r0; i < r1; ++i) {
    T x[JD], a[kVladKT];
#pragma unroll
    for (int j = 0; j < JD; ++j) x[j] = xn[j];
#pragma unroll
    for (int c = 0; c < kVladKT; ++c) a[c] = an[c];
    if (i + 1 < r1) load_row(i + 1);
#pragma unroll
    for (int c = 0; c < kVladKT; ++c) {
      if (a[c] > (T)0) {  // vl/vlad.c:182
        mass[c] += (double)a[c];
#pragma unroll
        for (int j = 0; j < JD; ++j) acc[c][j] = acc_step(acc[c][j], a[c], x[j]);
      }
    }
  }
  // Per component: mass step and signed square root per element, then the
  // component's norm (one thread per component sums its D squares in order).
#pragma unroll
  for (int c = 0; c < kVladKT; ++c) {
    if (c >= nk) continue;
    const int k = k0 + c;
#pragma unroll
    for (int j = 0; j < JD; ++j) {
      const int d = tid + kVladThreads * j;
      if (d >= D) continue;
      T z = acc[c][j];
      const T mu = means[(i64)k * D + d];
      if (mass[c] > 0) {
        if (flags & VL_VLAD_FLAG_NORMALIZE_MASS) {
          if constexpr (sizeof(T) == 4) z = __double2float_rn(__ddiv_rn((double)z, mass[c]));
          else z = __ddiv_rn(z, mass[c]);
          z = sub_t(z, mu);
        } else {
          if constexpr (sizeof(T) == 4) z = __double2float_rn(__dsub_rn((double)z, __dmul_rn(mass[c], (double)mu)));
          else z = __dsub_rn(z, __dmul_rn(mass[c], mu));
        }
      }
      if (flags & VL_VLAD_FLAG_SQUARE_ROOT) z = z >= (T)0 ? sqrt_t(z) : -sqrt_t(-z);
      zs[c * D + d] = z;
    }
  }
  __syncthreads();
  __shared__ T s_norm[kVladKT];
  if (flags & VL_VLAD_FLAG_NORMALIZE_COMPONENTS) {
    if (tid < nk) {
      T n = (T)0;
      for (int d = 0; d < D; ++d) n = add_t(n, mul_t(zs[tid * D + d], zs[tid * D + d]));
      n = sqrt_t(n);
      s_norm[tid] = (T)fmax((double)n, 1e-12);
    }
    __syncthreads();
  }
  T *out = enc + img * (i64)K * D;
  for (int c = 0; c < nk; ++c) {
    for (int d = tid; d < D; d += kVladThreads) {
      T z = zs[c * D + d];
      if (flags & VL_VLAD_FLAG_NORMALIZE_COMPONENTS) z = div_t(z, s_norm[c]);
      out[(i64)(k0 + c) * D + d] = z;
    }
  }
}

// Global L2 of each image (vl/vlad.c:226-240), one warp per image: per chunk
// of 256 values (8 loads per lane, issued while lane 0 sums the previous
// chunk) the lanes square their values into shared memory and lane 0 adds the
// squares in element order; the warp then divides its image by the floored
// norm.
constexpr int kGnChunk = 256;

template <typename T>
__global__ void __launch_bounds__(256) k_vlad_global_norm(T *__restrict__ enc, i64 KD, i64 nimg) {
  __shared__ __align__(16) T sq[8][kGnChunk];
  __shared__ T s_n[8];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const i64 img = (i64)blockIdx.x * 8 + w;
  if (img >= nimg) return;
  T *e = enc + img * KD;
  T n = (T)0;
  T z[kGnChunk / 32];
  auto load = [&](i64 i0) {
#pragma unroll
    for (int q = 0; q < kGnChunk / 32; ++q) {
      const i64 i = i0 + q * 32 + lane;
      z[q] = i < KD ? e[i] : (T)0;
    }
  };
  load(0);
  for (i64 i0 = 0; i0 < KD; i0 += kGnChunk) {
#pragma unroll
    for (int q = 0; q < kGnChunk / 32; ++q) sq[w][q * 32 + lane] = mul_t(z[q], z[q]);
    __syncwarp();
    if (i0 + kGnChunk < KD) load(i0 + kGnChunk);  // next chunk in flight during the sum
    if (lane == 0) {
      const int lim = KD - i0 < kGnChunk ? (int)(KD - i0) : kGnChunk;
      if (lim == kGnChunk) {
        if constexpr (sizeof(T) == 4) {
          const float4 *v4 = (const float4 *)sq[w];
#pragma unroll 16
          for (int l = 0; l < kGnChunk / 4; ++l) {
            const float4 v = v4[l];
            n = add_t(add_t(add_t(add_t(n, v.x), v.y), v.z), v.w);
          }
        } else {
#pragma unroll 32
          for (int l = 0; l < kGnChunk; ++l) n = add_t(n, sq[w][l]);
        }
      } else {
        for (int l = 0; l < lim; ++l) n = add_t(n, sq[w][l]);
      }
    }
    __syncwarp();
  }
  if (lane == 0) s_n[w] = (T)fmax((double)sqrt_t(n), 1e-12);
  __syncwarp();
  n = s_n[w];
  // Eight loads in flight before their divisions and stores.
  for (i64 i0 = lane; i0 < KD; i0 += 32 * 8) {
    T v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const i64 i = i0 + 32 * u;
      v[u] = i < KD ? e[i] : (T)0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const i64 i = i0 + 32 * u;
      if (i < KD) e[i] = div_t(v[u], n);
    }
  }
}

// ------------------------------------------------------------ streaming path
// One block per (image, run of kVsWarps x CPW components).  A producer warp
// streams the image's rows through shared memory with bulk asynchronous
// copies (kVsStages stages of R rows: the block's slice of each assignment
// row and the descriptor rows); kVsWarps consumer warps each own CPW
// components with their accumulators in registers (lane l holds dimensions
// l + 32j).  Per step a warp loads 32 weights, one per lane (32/CPW rows of
// its CPW components), and a ballot skips the rows whose weights are all
// <= 0, so hard assignments cost one shared-memory load per row and component
// group.  Positive weights update the accumulators in row order, as the
// reference's loop does: few per row through a branch tree on the component
// index, many through a pass over all CPW components.  The mass step, signed
// square root and the component norm (a serial sum in dimension order,
// broadcast by shuffles) run in registers before the store.
constexpr int kVsWarps = 8;
constexpr int kVsThreads = (kVsWarps + 1) * 32;
constexpr int kVsStages = 4;
constexpr int kVsUnroll = 8;  // steps whose weights are loaded together

struct VsParams {
  void *enc;
  const void *means, *X, *A;
  const i64 *offs;
  i64 img0;
  int D, K, flags, R;
  int *err;
  const int *only;  // when set, the images with only[img] != 0 (the others are done elsewhere)
};

template <typename T>
__device__ __forceinline__ T vlad_mass_step(T z, T mu, double mass, int flags) {
  if (!(mass > 0)) return z;
  if (flags & VL_VLAD_FLAG_NORMALIZE_MASS) {
    if constexpr (sizeof(T) == 4) z = __double2float_rn(__ddiv_rn((double)z, mass));
    else z = __ddiv_rn(z, mass);
    return sub_t(z, mu);
  }
  if constexpr (sizeof(T) == 4) return __double2float_rn(__dsub_rn((double)z, __dmul_rn(mass, (double)mu)));
  else return __dsub_rn(z, __dmul_rn(mass, mu));
}

__device__ __forceinline__ bool vs_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag, int *err) {
  return tc::mbar_wait(bar, parity, abort_flag, err, 0x5600);
}

// acc[c] += av * xv for the component c in [LO, HI) (warp-uniform c): a
// binary branch tree keeps every accumulator index static.  UNIT: float data
// and av == 1, where (float)((double)acc + (double)x) is the float sum itself
// (a sum of two floats rounded to double and then to float rounds as once to
// float, since 53 >= 2 * 24 + 2: Figueroa, "When is double rounding
// innocuous?", 1995).
template <int LO, int HI, bool UNIT, typename T, int CPW, int JD>
__device__ __forceinline__ void vs_update(int c, T (&acc)[CPW][JD], T av, const T (&xv)[JD]) {
  if constexpr (HI - LO == 1) {
#pragma unroll
    for (int j = 0; j < JD; ++j) {
      if constexpr (UNIT) acc[LO][j] = add_t(acc[LO][j], xv[j]);
      else acc[LO][j] = acc_step(acc[LO][j], av, xv[j]);
    }
  } else {
    constexpr int MID = (LO + HI) / 2;
    if (c < MID) vs_update<LO, MID, UNIT>(c, acc, av, xv);
    else vs_update<MID, HI, UNIT>(c, acc, av, xv);
  }
}

// One step of a consumer warp: the 32/CPW rows whose weights gave the ballot
// m (bit h*CPW + c: row h, component c of the warp); sa: the warp's first
// weight of the first row (rows nkb apart), sx: the first row's descriptor,
// both in shared memory.  Rows in order, components in any order (each
// accumulator sees its rows in order).
template <typename T, int JD, int CPW>
__device__ __forceinline__ void vs_rows_step(T (&acc)[CPW][JD], unsigned m, const T *sa, int nkb, const T *sx,
                                             int D, int lane) {
  constexpr int RPS = 32 / CPW;
  constexpr unsigned kMask = CPW == 32 ? 0xffffffffu : ((1u << CPW) - 1u);
#pragma unroll
  for (int h = 0; h < RPS; ++h) {
    unsigned bits = (m >> (CPW * h)) & kMask;
    if (bits == 0) continue;
    const T *wa = sa + (size_t)h * nkb;
    T xv[JD];
#pragma unroll
    for (int j = 0; j < JD; ++j) {
      const int d = lane + 32 * j;
      xv[j] = d < D ? sx[h * D + d] : (T)0;
    }
    if (__popc(bits) > 4) {
#pragma unroll
      for (int c = 0; c < CPW; ++c) {
        if (bits & (1u << c)) {
          const T av = wa[c];
#pragma unroll
          for (int j = 0; j < JD; ++j) acc[c][j] = acc_step(acc[c][j], av, xv[j]);
        }
      }
    } else {
      while (bits) {
        const int c = __ffs(bits) - 1;
        bits &= bits - 1;
        const T av = wa[c];
        if (sizeof(T) == 4 && av == (T)1) vs_update<0, CPW, true>(c, acc, av, xv);
        else vs_update<0, CPW, false>(c, acc, av, xv);
      }
    }
  }
}

template <typename T, int JD, int CPW>
__global__ void __launch_bounds__(kVsThreads, sizeof(T) == 4 && JD <= 3 ? 2 : 1) k_vlad_stream(const VsParams p) {
  constexpr int RPS = 32 / CPW;  // rows per step
  extern __shared__ __align__(128) unsigned char vs_smem[];
  uint64_t *full = (uint64_t *)vs_smem;
  uint64_t *empty = full + kVsStages;
  volatile int *s_abort = (volatile int *)(empty + kVsStages);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int D = p.D, K = p.K, R = p.R;
  const int k0 = blockIdx.x * (kVsWarps * CPW), nkb = min(kVsWarps * CPW, K - k0);
  const i64 img = p.img0 + blockIdx.y;
  if (p.only && !p.only[img]) return;
  const i64 r0 = p.offs[img], r1 = p.offs[img + 1];
  const int ntiles = (int)((r1 - r0 + R - 1) / R);
  const uint32_t aBytes = (uint32_t)(R * nkb * sizeof(T)), stageBytes = aBytes + (uint32_t)(R * D * sizeof(T));
  unsigned char *stage0 = vs_smem + 128;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kVsStages; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], kVsWarps);
    }
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const T *X = (const T *)p.X, *A = (const T *)p.A;
  if (warp == kVsWarps) {
    // Producer: one lane issues the copies of tile t into stage t % kVsStages.
    if (lane == 0) {
      int t = 0;
      for (; t < ntiles; ++t) {
        const int s = t % kVsStages;
        if (t >= kVsStages && !vs_wait(&empty[s], ((t / kVsStages) + 1) & 1, s_abort, p.err)) break;
        const i64 row0 = r0 + (i64)t * R;
        const int rows = (int)(r1 - row0 < (i64)R ? r1 - row0 : (i64)R);
        unsigned char *st = stage0 + (size_t)s * stageBytes;
        const uint32_t ab = (uint32_t)(rows * nkb * sizeof(T)), xb = (uint32_t)(rows * D * sizeof(T));
        tc::mbar_arrive_expect_tx(&full[s], ab + xb);
        if (nkb == K) {
          tc::bulk_g2s(tc::smem_u32(st), A + row0 * K, ab, &full[s]);
        } else {
          for (int r = 0; r < rows; ++r)
            tc::bulk_g2s(tc::smem_u32(st + (size_t)r * nkb * sizeof(T)), A + (row0 + r) * K + k0,
                         (uint32_t)(nkb * sizeof(T)), &full[s]);
        }
        tc::bulk_g2s(tc::smem_u32(st + aBytes), X + row0 * D, xb, &full[s]);
      }
      // The copies already issued land before the block exits (on an abort too).
      for (int u = max(0, t - kVsStages); u < t; ++u) {
        const unsigned long long t0 = tc::global_ns();
        while (!tc::mbar_try_wait(&full[u % kVsStages], (u / kVsStages) & 1) &&
               tc::global_ns() - t0 < tc::kWaitNs) {
        }
      }
    }
    return;
  }
  // Consumers.
  const int cw = warp * CPW;  // first component of this warp within the block
  T acc[CPW][JD];
#pragma unroll
  for (int c = 0; c < CPW; ++c)
#pragma unroll
    for (int j = 0; j < JD; ++j) acc[c][j] = (T)0;
  double mass = 0.0;  // lane c < CPW: component cw + c
  const int myc = cw + (lane % CPW);
  const bool cvalid = myc < nkb;
  for (int t = 0; t < ntiles; ++t) {
    const int s = t % kVsStages;
    if (!vs_wait(&full[s], (t / kVsStages) & 1, s_abort, p.err)) break;
    const unsigned char *st = stage0 + (size_t)s * stageBytes;
    const T *sA = (const T *)st, *sX = (const T *)(st + aBytes);
    const i64 left = r1 - (r0 + (i64)t * R);
    const int rows = (int)(left < (i64)R ? left : (i64)R);
    // This lane's weight column, one row per step of RPS rows.
    const T *pa = sA + (lane / CPW) * nkb + (cvalid ? myc : 0);
    const int stride = RPS * nkb;
    for (int r = 0; r < rows; r += RPS * kVsUnroll, pa += kVsUnroll * stride) {
      T a[kVsUnroll];
      unsigned m[kVsUnroll];
      if (r + RPS * kVsUnroll <= rows && cvalid) {
#pragma unroll
        for (int u = 0; u < kVsUnroll; ++u) a[u] = pa[u * stride];
      } else {
#pragma unroll
        for (int u = 0; u < kVsUnroll; ++u)
          a[u] = (r + u * RPS + lane / CPW < rows && cvalid) ? pa[u * stride] : (T)0;
      }
      unsigned rowbits = 0;  // bit u: step u has a positive weight
#pragma unroll
      for (int u = 0; u < kVsUnroll; ++u) {
        m[u] = __ballot_sync(0xffffffffu, a[u] > (T)0);  // vl/vlad.c:182
        rowbits |= (m[u] != 0u) << u;
      }
      while (rowbits) {  // steps with a positive weight, in row order
        const int u = __ffs(rowbits) - 1;
        rowbits &= rowbits - 1;
        unsigned mu = m[0];
#pragma unroll
        for (int v = 1; v < kVsUnroll; ++v) mu = u == v ? m[v] : mu;
        // The step's weights are still in the stage: this lane's own (for the
        // mass) and, per positive component, a broadcast read.
        const T au = (cvalid && r + u * RPS + lane / CPW < rows) ? pa[u * stride] : (T)0;
        // The mass of a component sums its positive weights in row order;
        // the other weights would add 0.0, which leaves it unchanged.
        const double am = au > (T)0 ? (double)au : 0.0;
        mass += am;
        if constexpr (RPS == 2) mass += __shfl_down_sync(0xffffffffu, am, 16);
        const int rs = r + u * RPS;
        vs_rows_step<T, JD, CPW>(acc, mu, sA + (size_t)rs * nkb + cw, nkb, sX + (size_t)rs * D, D, lane);
      }
    }
    __syncwarp();
    if (lane == 0) tc::mbar_arrive(&empty[s]);
  }
  // Epilogue through shared memory (the stage area, free once every consumer
  // warp is past its last tile; the producer has seen all its copies land):
  // the warp stores its raw sums as rows of D + 1 values, lane c < CPW
  // finishes component cw + c there (mass step, signed square root and the
  // component norm in dimension order), and the warp writes the rows out
  // coalesced.
  tc::named_barrier(1, kVsWarps * 32);
  if (*s_abort) return;
  const int ncw = min(CPW, nkb - cw);
  const int ld = D + 1;
  T *zs = (T *)stage0 + (size_t)cw * ld;
#pragma unroll
  for (int c = 0; c < CPW; ++c) {
#pragma unroll
    for (int j = 0; j < JD; ++j) {
      const int d = lane + 32 * j;
      if (c < ncw && d < D) zs[c * ld + d] = acc[c][j];
    }
  }
  __syncwarp();
  if (lane < ncw) {
    const T *mu = (const T *)p.means + (i64)(k0 + cw + lane) * D;
    T *o = zs + lane * ld;
    T n = (T)0;
    for (int d = 0; d < D; ++d) {
      T z = vlad_mass_step<T>(o[d], mu[d], mass, p.flags);
      if (p.flags & VL_VLAD_FLAG_SQUARE_ROOT) z = z >= (T)0 ? sqrt_t(z) : -sqrt_t(-z);
      n = add_t(n, mul_t(z, z));
      o[d] = z;
    }
    if (p.flags & VL_VLAD_FLAG_NORMALIZE_COMPONENTS) {
      n = (T)fmax((double)sqrt_t(n), 1e-12);
      for (int d = 0; d < D; ++d) o[d] = div_t(o[d], n);
    }
  }
  __syncwarp();
  T *out = (T *)p.enc + img * (i64)K * D + (i64)(k0 + cw) * D;
  for (int c = 0; c < ncw; ++c)
    for (int d = lane; d < D; d += 32) out[(i64)c * D + d] = zs[c * ld + d];
}

// -------------------------------------------- grouped path (one weight per row)
// When each row has at most one positive weight (hard assignments), the rows
// of an image are first grouped by that component, in row order; then one
// warp per (image, component) walks its rows.  Every chain sees the same
// rows in the same order as in the reference's loop, so the bits are the
// same; the assignment matrix is read once, by a streaming pass.

// Per row: its only positive weight's component and value (comp -1: no
// positive weight; -2: more than one, and its image takes the streaming
// kernel).  One warp per row, 16-byte loads.
template <typename T>
__global__ void __launch_bounds__(256) k_vlad_pick(const T *__restrict__ A, i64 N, int K, int *__restrict__ comp,
                                                    T *__restrict__ wgt) {
  constexpr int V = 16 / (int)sizeof(T);
  using L = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  const int lane = threadIdx.x & 31;
  const i64 w0 = ((i64)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((i64)gridDim.x * blockDim.x) >> 5;
  // Two rows per warp and pass, their loads in flight together.
  for (i64 i0 = 2 * w0; i0 < N; i0 += 2 * nw) {
    int cnt[2] = {0, 0}, kk[2] = {-1, -1};
    T av[2] = {(T)0, (T)0};
    for (int k0 = lane * V; k0 < K; k0 += 32 * V) {
      L v[2];
#pragma unroll
      for (int h = 0; h < 2; ++h)
        if (i0 + h < N) v[h] = *reinterpret_cast<const L *>(A + (i0 + h) * K + k0);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (i0 + h >= N) continue;
        const T *e = reinterpret_cast<const T *>(&v[h]);
#pragma unroll
        for (int u = 0; u < V; ++u)
          if (e[u] > (T)0) {  // vl/vlad.c:182
            ++cnt[h];
            kk[h] = k0 + u;
            av[h] = e[u];
          }
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const i64 i = i0 + h;
      const int tot = __reduce_add_sync(0xffffffffu, cnt[h]);
      if (i >= N) continue;
      if (tot == 1 && cnt[h] == 1) {
        comp[i] = kk[h];
        wgt[i] = av[h];
      }
      if (lane == 0 && tot != 1) comp[i] = tot == 0 ? -1 : -2;
    }
  }
}

constexpr int kSortWarps = 16;

// Per image (one block): a stable counting sort of its rows by component.
// Warp w takes a contiguous run of the rows; per-warp counts give each
// (warp, component) its first slot, so rows keep their order within a
// component.  cstart[img][k] .. cstart[img][k + 1]: the component's slots in
// sorted (rows relative to the image's first); soft[img]: a row with more
// than one positive weight.
__global__ void __launch_bounds__(kSortWarps * 32) k_vlad_sort(const i64 *__restrict__ offs, const int *__restrict__ comp,
                                                              int K, int *__restrict__ sorted, int *__restrict__ cstart,
                                                              int *__restrict__ soft) {
  extern __shared__ int sh[];
  int *hist = sh;                   // [warp][K]: counts, then first slots
  int *base = sh + kSortWarps * K;  // [K + 1]
  __shared__ int s_soft;
  const i64 img = blockIdx.x;
  const i64 r0 = offs[img], n = offs[img + 1] - r0;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < kSortWarps * K; i += kSortWarps * 32) hist[i] = 0;
  if (tid == 0) s_soft = 0;
  __syncthreads();
  const i64 w0 = r0 + n * warp / kSortWarps, w1 = r0 + n * (warp + 1) / kSortWarps;
  for (i64 r = w0 + lane; r < w1; r += 32) {
    const int c = comp[r];
    if (c >= 0) atomicAdd(&hist[warp * K + c], 1);
    else if (c == -2) s_soft = 1;
  }
  __syncthreads();
  for (int k = tid; k < K; k += kSortWarps * 32) {
    int t = 0;
    for (int w = 0; w < kSortWarps; ++w) {
      const int h = hist[w * K + k];
      hist[w * K + k] = t;
      t += h;
    }
    base[k] = t;
  }
  __syncthreads();
  if (warp == 0) {  // exclusive prefix of the component totals
    const int per = (K + 31) / 32;
    int sum = 0;
    for (int j = 0; j < per; ++j) {
      const int k = lane * per + j;
      if (k < K) sum += base[k];
    }
    int pre = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, pre, o);
      if (lane >= o) pre += v;
    }
    int run = pre - sum;
    for (int j = 0; j < per; ++j) {
      const int k = lane * per + j;
      if (k < K) {
        const int t = base[k];
        base[k] = run;
        run += t;
      }
    }
    if (lane == 31) base[K] = run;
  }
  __syncthreads();
  for (int k = tid; k <= K; k += kSortWarps * 32) cstart[img * (K + 1) + k] = base[k];
  if (tid == 0) soft[img] = s_soft;
  // Stable scatter: 32 consecutive rows at a time; lanes with the same
  // component take consecutive slots in lane order.
  for (i64 rb = w0; rb < w1; rb += 32) {
    const i64 r = rb + lane;
    const int c = r < w1 ? comp[r] : -1;
    const unsigned same = __match_any_sync(0xffffffffu, c);
    const int first = c >= 0 ? base[c] + hist[warp * K + c] : 0;
    __syncwarp();
    if (c >= 0) {
      sorted[r0 + first + __popc(same & ((1u << lane) - 1u))] = (int)(r - r0);
      if ((same >> lane) == 1u) hist[warp * K + c] += __popc(same);  // the group's last lane
    }
    __syncwarp();
  }
}

struct VgParams {
  void *enc;
  const void *means, *X, *wgt;
  const i64 *offs;
  const int *sorted, *cstart, *soft;
  i64 img0;
  int D, K, flags;
};

constexpr int kVgWarps = 8;
constexpr int kVgPrefetch = 8;  // rows whose descriptors are loaded together

// One warp per (image, component): the component's rows in order (lane l
// holds dimensions l + 32 j), the chain step and the mass as in the
// reference's loop, then the mass step, the signed square root and the
// component norm (a sum of squares in dimension order, by lane 0 through
// shared memory), and the coalesced store.  Images with a multi-weight row
// are left to the streaming kernel.
template <typename T, int JD>
__global__ void __launch_bounds__(kVgWarps * 32) k_vlad_group(const VgParams p) {
  __shared__ T zs[kVgWarps][128];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const i64 img = p.img0 + blockIdx.y;
  if (p.soft[img]) return;
  const int K = p.K, D = p.D, k = blockIdx.x * kVgWarps + warp;
  if (k >= K) return;
  const T *X = (const T *)p.X, *W = (const T *)p.wgt;
  const i64 r0 = p.offs[img];
  const int b = p.cstart[img * (K + 1) + k], e = p.cstart[img * (K + 1) + k + 1];
  const int *rows = p.sorted + r0;
  T acc[JD];
#pragma unroll
  for (int j = 0; j < JD; ++j) acc[j] = (T)0;
  double mass = 0.0;
  // 32 of the component's rows at a time: lane j loads the j-th row index and
  // weight; the rows' descriptors are loaded kVgPrefetch rows ahead.
  for (int t = b; t < e; t += 32) {
    const int cnt = min(32, e - t);
    const int myrow = lane < cnt ? rows[t + lane] : 0;
    const T mya = lane < cnt ? W[r0 + myrow] : (T)0;
    for (int u0 = 0; u0 < cnt; u0 += kVgPrefetch) {
      T av[kVgPrefetch], xv[kVgPrefetch][JD];
#pragma unroll
      for (int u = 0; u < kVgPrefetch; ++u) {
        const int rr = __shfl_sync(0xffffffffu, myrow, (u0 + u) & 31);
        av[u] = __shfl_sync(0xffffffffu, mya, (u0 + u) & 31);
        if (u0 + u < cnt) {
          const i64 row = r0 + rr;
#pragma unroll
          for (int j = 0; j < JD; ++j) {
            const int d = lane + 32 * j;
            xv[u][j] = d < D ? X[row * D + d] : (T)0;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < kVgPrefetch; ++u) {
        if (u0 + u < cnt) {
          mass += (double)av[u];
          if (sizeof(T) == 4 && av[u] == (T)1) {
#pragma unroll
            for (int j = 0; j < JD; ++j) acc[j] = add_t(acc[j], xv[u][j]);
          } else {
#pragma unroll
            for (int j = 0; j < JD; ++j) acc[j] = acc_step(acc[j], av[u], xv[u][j]);
          }
        }
      }
    }
  }
  const T *mu = (const T *)p.means + (i64)k * D;
  T z[JD];
#pragma unroll
  for (int j = 0; j < JD; ++j) {
    const int d = lane + 32 * j;
    z[j] = (T)0;
    if (d < D) {
      T v = vlad_mass_step<T>(acc[j], mu[d], mass, p.flags);
      if (p.flags & VL_VLAD_FLAG_SQUARE_ROOT) v = v >= (T)0 ? sqrt_t(v) : -sqrt_t(-v);
      z[j] = v;
      zs[warp][d] = v;
    }
  }
  if (p.flags & VL_VLAD_FLAG_NORMALIZE_COMPONENTS) {
    __syncwarp();
    T nrm = (T)0;
    if (lane == 0) {
      for (int d = 0; d < D; ++d) nrm = add_t(nrm, mul_t(zs[warp][d], zs[warp][d]));
      nrm = (T)fmax((double)sqrt_t(nrm), 1e-12);
    }
    nrm = __shfl_sync(0xffffffffu, nrm, 0);
#pragma unroll
    for (int j = 0; j < JD; ++j) z[j] = div_t(z[j], nrm);
  }
  T *out = (T *)p.enc + img * (i64)K * D + (i64)k * D;
#pragma unroll
  for (int j = 0; j < JD; ++j) {
    const int d = lane + 32 * j;
    if (d < D) out[d] = z[j];
  }
}

// Components per consumer warp.  16 (two rows per step) keeps float
// accumulators within the register budget of two blocks per SM.
constexpr int kVsCpw = 16;

// Rows per stage: stages of about 24 KB where two blocks share an SM (float
// data, D <= 96), 32 KB otherwise.
template <typename T>
int vs_rows(int D, int K) {
  const int rowBytes = (int)((std::min(K, kVsWarps * kVsCpw) + D) * sizeof(T));
  const int target = sizeof(T) == 4 && D <= 96 ? 24 * 1024 : 32 * 1024;
  return std::max(8, std::min(64, (target / rowBytes) & ~1));
}

template <typename T>
bool vs_eligible(int D, int K, const void *X, const void *A) {
  return D <= 128 && (D * sizeof(T)) % 16 == 0 && (K * sizeof(T)) % 16 == 0 && ((uintptr_t)X % 16) == 0 &&
         ((uintptr_t)A % 16) == 0;
}

template <typename T, int JD, int CPW>
void launch_stream_cpw(const VsParams &p0, i64 nimg, cudaStream_t s) {
  constexpr int comps = kVsWarps * CPW;
  VsParams p = p0;
  const size_t stages = (size_t)kVsStages * p.R * (std::min(p.K, comps) + p.D) * sizeof(T);
  const size_t epi = (size_t)std::min(p.K, comps) * (p.D + 1) * sizeof(T);
  const size_t smem = 128 + std::max(stages, epi);
  auto kern = k_vlad_stream<T, JD, CPW>;
  VLB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (i64 img0 = 0; img0 < nimg; img0 += 65535) {
    p.img0 = img0;
    dim3 grid((unsigned)((p.K + comps - 1) / comps), (unsigned)std::min<i64>(65535, nimg - img0));
    VLB_LAUNCH("vlad_stream", s, kern<<<grid, kVsThreads, smem, s>>>(p));
  }
}

template <typename T, int JD>
void launch_stream(T *enc, const T *means, int D, int K, const T *X, const T *A, const i64 *doffs, i64 nimg,
                   int flags, int *derr, const int *only, cudaStream_t s) {
  VsParams p;
  p.enc = enc; p.means = means; p.X = X; p.A = A; p.offs = doffs;
  p.D = D; p.K = K; p.flags = flags; p.R = vs_rows<T>(D, K); p.err = derr; p.only = only;
  launch_stream_cpw<T, JD, kVsCpw>(p, nimg, s);
}

template <typename T, int JD>
void launch_group(const VgParams &p0, i64 nimg, cudaStream_t s) {
  VgParams p = p0;
  for (i64 img0 = 0; img0 < nimg; img0 += 65535) {
    p.img0 = img0;
    dim3 grid((unsigned)((p.K + kVgWarps - 1) / kVgWarps), (unsigned)std::min<i64>(65535, nimg - img0));
    VLB_LAUNCH("vlad_group", s, (k_vlad_group<T, JD><<<grid, kVgWarps * 32, 0, s>>>(p)));
  }
}

// The grouped path's pre-passes: per row its one positive weight, then per
// image the rows sorted by component (scratch slots 7-11 of the VLAD arena).
// Returns the per-image flags of images that need the streaming kernel.
template <typename T>
const int *group_rows(Scratch &sc, const T *A, i64 N, int K, const i64 *doffs, i64 nimg, VgParams &g,
                      cudaStream_t s) {
  int *comp = sc.slot[7].get<int>((size_t)std::max<i64>(1, N));
  T *wgt = sc.slot[8].get<T>((size_t)std::max<i64>(1, N));
  int *sorted = sc.slot[9].get<int>((size_t)std::max<i64>(1, N));
  int *cstart = sc.slot[10].get<int>((size_t)nimg * (K + 1));
  int *soft = sc.slot[11].get<int>((size_t)nimg);
  if (N > 0) {
    const unsigned blocks = (unsigned)std::min<i64>((N + 7) / 8, 16 * 148);
    VLB_LAUNCH("vlad_pick", s, k_vlad_pick<T><<<blocks, 256, 0, s>>>(A, N, K, comp, wgt));
  }
  const size_t smem = sizeof(int) * ((size_t)kSortWarps * K + K + 1);
  VLB_CUDA(cudaFuncSetAttribute(k_vlad_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  VLB_LAUNCH("vlad_sort", s, k_vlad_sort<<<(unsigned)nimg, kSortWarps * 32, smem, s>>>(doffs, comp, K, sorted, cstart, soft));
  g.wgt = wgt;
  g.sorted = sorted;
  g.cstart = cstart;
  g.soft = soft;
  return soft;
}

template <typename T, int JD>
void launch_accum(T *enc, const T *means, int D, int K, const T *X, const T *A, const i64 *doffs, i64 nimg,
                  int flags, cudaStream_t s) {
  const size_t smem = sizeof(T) * kVladKT * D;
  auto kern = k_vlad_accum<T, JD>;
  VLB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (i64 img0 = 0; img0 < nimg; img0 += 65535) {
    dim3 grid((unsigned)((K + kVladKT - 1) / kVladKT), (unsigned)std::min<i64>(65535, nimg - img0));
    VLB_LAUNCH("vlad_accum", s, kern<<<grid, kVladThreads, smem, s>>>(enc, means, D, K, X, A, doffs, img0, flags));
  }
}

template <typename T>
void vlad_tiles(T *enc, const T *means, i64 D, i64 K, const T *X, const T *A, const i64 *doffs, i64 nimg, int flags,
                cudaStream_t s) {
  const int jd = (int)((D + kVladThreads - 1) / kVladThreads);
  if (jd <= 1) launch_accum<T, 1>(enc, means, (int)D, (int)K, X, A, doffs, nimg, flags, s);
  else if (jd <= 2) launch_accum<T, 2>(enc, means, (int)D, (int)K, X, A, doffs, nimg, flags, s);
  else if (jd <= 4) launch_accum<T, 4>(enc, means, (int)D, (int)K, X, A, doffs, nimg, flags, s);
  else launch_accum<T, 8>(enc, means, (int)D, (int)K, X, A, doffs, nimg, flags, s);
}

}  // namespace

template <typename T>
void vlad_batch(T *enc, const T *means, i64 D, i64 K, const T *X, const T *A, const i64 *h_offsets, i64 nimg,
                int flags, cudaStream_t s) {
  VLB_CHECK(D >= 1 && K >= 1, VL_ERR_BAD_ARG, "VLAD: dimension and numClusters must be >= 1");
  VLB_CHECK(D <= 8 * kVladThreads, VL_ERR_BAD_ARG, "VLAD: dimension above 1024 is not supported");
  if (nimg <= 0) return;
  // VLAD arena slots: 0 offsets, 6 error word (here); 2-5 the
  // host entry point's staged inputs and output.
  Scratch &sc = thread_scratch(kArenaVlad);
  // Offsets relative to the first image's first row (data and assignments
  // rebased with them), so that the per-row scratch starts at the batch.
  const i64 base0 = h_offsets[0];
  std::vector<i64> rel(nimg + 1);
  for (i64 j = 0; j <= nimg; ++j) rel[j] = h_offsets[j] - base0;
  X += base0 * D;
  A += base0 * K;
  const i64 N = rel[nimg];
  i64 *doffs = sc.slot[0].get<i64>(nimg + 1);
  VLB_CUDA(cudaMemcpyAsync(doffs, rel.data(), sizeof(i64) * (nimg + 1), cudaMemcpyHostToDevice, s));
  int *herr = (int *)pinned_host(sizeof(int));
  *herr = 0;
  if (vs_eligible<T>((int)D, (int)K, X, A)) {
    int *derr = sc.slot[6].get<int>(1);
    VLB_CUDA(cudaMemsetAsync(derr, 0, sizeof(int), s));
    const int jd = (int)((D + 31) / 32);
    // Up to 1,024 components, rows with one positive weight are grouped by
    // component first; the streaming kernel takes only the images with a
    // row of several.
    const int *only = nullptr;
    if (K <= 1024 && N < (i64)INT32_MAX) {
      VgParams g;
      g.enc = enc; g.means = means; g.X = X; g.offs = doffs; g.D = (int)D; g.K = (int)K; g.flags = flags;
      only = group_rows<T>(sc, A, N, (int)K, doffs, nimg, g, s);
      if (jd <= 1) launch_group<T, 1>(g, nimg, s);
      else if (jd == 2) launch_group<T, 2>(g, nimg, s);
      else if (jd == 3) launch_group<T, 3>(g, nimg, s);
      else launch_group<T, 4>(g, nimg, s);
    }
    if (jd <= 1) launch_stream<T, 1>(enc, means, (int)D, (int)K, X, A, doffs, nimg, flags, derr, only, s);
    else if (jd == 2) launch_stream<T, 2>(enc, means, (int)D, (int)K, X, A, doffs, nimg, flags, derr, only, s);
    else if (jd == 3) launch_stream<T, 3>(enc, means, (int)D, (int)K, X, A, doffs, nimg, flags, derr, only, s);
    else launch_stream<T, 4>(enc, means, (int)D, (int)K, X, A, doffs, nimg, flags, derr, only, s);
    VLB_CUDA(cudaMemcpyAsync(herr, derr, sizeof(int), cudaMemcpyDeviceToHost, s));
  } else {
    vlad_tiles<T>(enc, means, D, K, X, A, doffs, nimg, flags, s);
  }
  if (!(flags & VL_VLAD_FLAG_UNNORMALIZED))
    VLB_LAUNCH("vlad_global_norm", s,
               k_vlad_global_norm<T><<<(unsigned)((nimg + 7) / 8), 256, 0, s>>>(enc, K * D, nimg));
  // The scratch above is reused by the next call on this thread, which may
  // use another stream: finish before returning.
  VLB_CUDA(cudaStreamSynchronize(s));
  VLB_CHECK(*herr == 0, VL_ERR_ALLOC, "VLAD: a pipeline wait timed out on the device");
}

template void vlad_batch<float>(float *, const float *, i64, i64, const float *, const float *, const i64 *, i64,
                                int, cudaStream_t);
template void vlad_batch<double>(double *, const double *, i64, i64, const double *, const double *, const i64 *,
                                 i64, int, cudaStream_t);

}  // namespace vlb

using vlb::i64;

namespace {
template <typename F>
int guarded(F &&f) {
  try {
    f();
    return 0;
  } catch (const vlb::Error &e) {
    vl_set_last_error(e.code, "%s", e.what());
    return e.code;
  } catch (const std::exception &e) {
    vl_set_last_error(VL_ERR_ALLOC, "%s", e.what());
    return VL_ERR_ALLOC;
  }
}

template <typename T>
void vlad_host(T *enc, const T *means, vl_size D, vl_size K, const T *data, vl_size N, const T *assign,
               int flags) {
  VLB_CHECK(D >= 1 && K >= 1, VL_ERR_BAD_ARG, "vl_vlad_encode: dimension and numClusters must be >= 1");
  cudaStream_t s = vlb::thread_stream();
  vlb::Scratch &sc = vlb::thread_scratch(vlb::kArenaVlad);
  T *dX = sc.slot[2].get<T>(std::max<vl_size>(1, N) * D);
  T *dA = sc.slot[3].get<T>(std::max<vl_size>(1, N) * K);
  T *dm = sc.slot[4].get<T>(K * D);
  T *de = sc.slot[5].get<T>(K * D);
  if (N) {
    VLB_CUDA(cudaMemcpyAsync(dX, data, sizeof(T) * N * D, cudaMemcpyHostToDevice, s));
    VLB_CUDA(cudaMemcpyAsync(dA, assign, sizeof(T) * N * K, cudaMemcpyHostToDevice, s));
  }
  VLB_CUDA(cudaMemcpyAsync(dm, means, sizeof(T) * K * D, cudaMemcpyHostToDevice, s));
  const i64 offs[2] = {0, (i64)N};
  vlb::vlad_batch<T>(de, dm, (i64)D, (i64)K, dX, dA, offs, 1, flags, s);
  VLB_CUDA(cudaMemcpyAsync(enc, de, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaStreamSynchronize(s));
}
}  // namespace

extern "C" {

void vl_vlad_encode(void *enc, vl_type dataType, void const *means, vl_size dimension, vl_size numClusters,
                    void const *data, vl_size numData, void const *assignments, int flags) {
  guarded([&] {
    VLB_CHECK(dataType == VL_TYPE_FLOAT || dataType == VL_TYPE_DOUBLE, VL_ERR_BAD_ARG,
              "vl_vlad_encode: data type must be VL_TYPE_FLOAT or VL_TYPE_DOUBLE");
    if (dataType == VL_TYPE_FLOAT)
      vlad_host<float>((float *)enc, (const float *)means, dimension, numClusters, (const float *)data, numData,
                       (const float *)assignments, flags);
    else
      vlad_host<double>((double *)enc, (const double *)means, dimension, numClusters, (const double *)data,
                        numData, (const double *)assignments, flags);
  });
}

int vlb200_vlad_encode_batch_device(void *enc, vl_type dataType, void const *means, vl_size dimension,
                                    vl_size numClusters, void const *data, void const *assignments,
                                    vl_int64 const *offsets, vl_size numImages, int flags, void *stream) {
  return guarded([&] {
    VLB_CHECK(dataType == VL_TYPE_FLOAT || dataType == VL_TYPE_DOUBLE, VL_ERR_BAD_ARG,
              "data type must be VL_TYPE_FLOAT or VL_TYPE_DOUBLE");
    VLB_CHECK(offsets != nullptr && offsets[0] >= 0, VL_ERR_BAD_ARG, "bad offsets");
    for (vl_size j = 0; j < numImages; ++j)
      VLB_CHECK(offsets[j + 1] >= offsets[j], VL_ERR_BAD_ARG, "offsets must be non-decreasing");
    cudaStream_t s = vlb::pick_stream(stream);
    if (dataType == VL_TYPE_FLOAT)
      vlb::vlad_batch<float>((float *)enc, (const float *)means, (i64)dimension, (i64)numClusters,
                             (const float *)data, (const float *)assignments, (const i64 *)offsets,
                             (i64)numImages, flags, s);
    else
      vlb::vlad_batch<double>((double *)enc, (const double *)means, (i64)dimension, (i64)numClusters,
                              (const double *)data, (const double *)assignments, (const i64 *)offsets,
                              (i64)numImages, flags, s);
  });
}

}  // extern "C"
