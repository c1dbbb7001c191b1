// Tensor-core (tcgen05) path for float data.
//
// The two contractions of the GMM / Fisher path run on the 5th-generation
// tensor cores with fp32 accumulators in TMEM:
//
//  E-step   S = [x', x'^2] . W^T,  W_k = [mu'_k / sigma2_k, -1 / (2 sigma2_k)] * log2(e)
//           x' = x - m (m: mean of the component means), so that
//           log2 p_ik = cst2_k + S_ik with cst2_k the per-component constant of
//           vl/gmm.c:741-774 in base 2.  The epilogue (4 warps, one row per
//           thread) turns the TMEM row into posteriors with a log-sum-exp:
//           max, exp2 + sum (written back to TMEM), normalise, store.
//  Stats    T = q^T . [x', x'^2, 1]  (per component: sum q x', sum q x'^2, sum q)
//           accumulated over a work item (a run of rows of one image) in TMEM
//           and drained to a per-item fp32 partial; a finalize kernel reduces
//           an image's partials in double and forms the Fisher vector
//           (vl/fisher.c:419-485) or the M-step update (vl/gmm.c:1169-1205).
//
// Precision: both operands are split into fp16 hi + lo parts (22 bits) and
// each product is formed as hi.hi + hi.lo + lo.hi (fp16x3, ~2^-21 relative per
// product, fp32 accumulation).  Power-of-two scales keep the operands in
// fp16's normal range: x' is multiplied by scale_d per dimension, W by one
// global 2^-g (undone by the epilogue's fused multiply-add), q by 2^14 in the
// image (undone by the finalizers).  The BF16 mode keeps the split on the
// E-step (the expanded quadratic cancels) and uses a single fp16 q part for
// the statistics.
//
// Both kernels are persistent and warp-specialised (288 threads):
//   warps 0-3  producers: load fp32 rows, centre/square, split, and write the
//              swizzled fp16 operand tiles into a ring of shared-memory stages;
//   warps 4-7  epilogue: TMEM -> registers -> global;
//   warp 8     TMEM allocation and, from one lane, tcgen05.mma issue.
// Operand layouts: E-step A and W are K-major with the 64-byte swizzle (one
// 32-element k-atom per stage); statistics A (q^T) and B are MN-major with the
// 128-byte swizzle, which matches the row-major q and x in global memory.
#include <cmath>
#include <cstring>
#include <algorithm>
#include <functional>
#include <memory>
#include <numeric>
#include <vector>

#include <cooperative_groups.h>

#include "engine.h"
#include "tc_common.cuh"

extern "C" {
#include "vlb200.h"
}

namespace vlb {

namespace {

using namespace tc;
namespace cg = cooperative_groups;

// E-step block: 4 producer, 8 epilogue and 1 MMA warp; with W streamed (SW)
// one more warp loads the descriptor rows and the W k-atoms.
__host__ __device__ constexpr int tc_threads(bool sw) { return sw ? 448 : 416; }
constexpr int kSmemLimit = 232448;  // 227 KB opt-in per block
constexpr int kMaxXs = 8;           // E-step ring of descriptor-row boxes: at most 8
constexpr double kLn2 = 0.6931471805599453;

int num_sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    VLB_CUDA(cudaGetDevice(&dev));
    VLB_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  }
  return n;
}

// Rounds a dynamic shared-memory pointer up to 1 KB by pointer arithmetic,
// so the compiler keeps treating derived pointers as shared memory.
__device__ __forceinline__ uint8_t *align1024(uint8_t *p) {
  return p + ((1024u - (smem_u32(p) & 1023u)) & 1023u);
}

// ================================================================ prep
// Sum over the 32 lanes in a fixed butterfly order (the same bits every run).
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Centre m_d = mean over components of mu_kd.  One warp per dimension.
__global__ void k_tc_center(const float *__restrict__ means, int K, int D, float *__restrict__ ctr) {
  const int d = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x % 32;
  if (d >= D) return;
  double s = 0;
  for (int k = lane; k < K; k += 32) s += (double)means[(i64)k * D + d];
  s = warp_sum(s);
  if (lane == 0) ctr[d] = (float)(s / (double)K);
}

// The x''^2 weight of component k and dimension d, -1/2 / s2_kd / scale_d^2
// log2(e), before the common part is taken out.
__device__ __forceinline__ double tc_weight2(const float *__restrict__ covs, const float *__restrict__ scale,
                                             int k, int d, int D) {
  const double s2 = (double)covs[(i64)k * D + d], sc = (double)scale[d];
  return -0.5 / s2 / (sc * sc) * 1.4426950408889634;
}

// Common part of the x''^2 weights: wbar_d = mean over the components of
// tc_weight2 (fixed-order sums, one warp per dimension).  The logits of a
// row change by the same amount sum_d wbar_d x''_d^2 when it is taken out of
// every component's weights, so the posteriors do not change, while the
// terms the fp32 accumulator adds (and the logit it rounds) shrink by about
// an order of magnitude; the log-likelihood adds the common part back.
__global__ void k_tc_wbar(const float *__restrict__ covs, const float *__restrict__ scale, int K, int D,
                          float *__restrict__ wbar) {
  const int d = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x % 32;
  if (d >= D) return;
  double s = 0;
  for (int k = lane; k < K; k += 32) s += tc_weight2(covs, scale, k, d, D);
  s = warp_sum(s);
  if (lane == 0) wbar[d] = (float)(s / (double)K);
}

// Entries of the E-step's weight matrix for component k and K-order element
// e (chunk c = e / 32 holds x''_d for d = 16c .. 16c+15, then x''_d^2 for the
// same d, so that the producers read each element of x once):
//   [mu'_kd / s2_kd / scale_d, -1/2 / s2_kd / scale_d^2 - wbar_d] log2(e),
// the producers multiplying x' by the power of two scale_d.
__device__ __forceinline__ double tc_weight(const float *__restrict__ means, const float *__restrict__ covs,
                                            const float *__restrict__ ctr, const float *__restrict__ scale,
                                            const float *__restrict__ wbar, int k, int e, int D) {
  const int c = e / 32, ee = e % 32, d = 16 * c + (ee & 15);
  if (ee >= 16) return tc_weight2(covs, scale, k, d, D) - (double)wbar[d];
  const double s2 = (double)covs[(i64)k * D + d], sc = (double)scale[d];
  const double mup = (double)means[(i64)k * D + d] - (double)ctr[d];
  return mup / s2 / sc * 1.4426950408889634;
}

// max |w| over the model: one element per thread, a warp maximum, then an
// atomic maximum on the float's bits (non-negative floats order as their bits;
// *wmax is zeroed before the launch).  The maximum does not depend on order.
__global__ void k_tc_wmax(const float *__restrict__ means, const float *__restrict__ covs,
                          const float *__restrict__ ctr, const float *__restrict__ scale,
                          const float *__restrict__ wbar, int K, int D, float *__restrict__ wmax) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  float m = 0.f;
  if (i < (i64)K * 2 * D)
    m = (float)fabs(tc_weight(means, covs, ctr, scale, wbar, (int)(i / (2 * D)), (int)(i % (2 * D)), D));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax((unsigned *)wmax, __float_as_uint(m));
}

// W image (hi then lo, fp16), K-major 64-byte-swizzled k-atoms of 32 elements:
// part p, atom c, row k, element e -> p*wbytes + c*Kp*64 + swizzled(k, e).
// The entries are divided by 2^g, the power of two that puts max |w| in
// [2^14, 2^15) (fp16 keeps 11 bits per part there); *wsc = 2^g, which the
// E-step multiplies back onto every logit.
__global__ void k_tc_wimg(const float *__restrict__ means, const float *__restrict__ covs,
                          const float *__restrict__ ctr, const float *__restrict__ scale,
                          const float *__restrict__ wbar, const float *__restrict__ wmax, int K, int Kp,
                          int D, __half *__restrict__ wimg, float *__restrict__ wsc) {
  const int KD2 = 2 * D;
  i64 idx = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  int g = 0;
  const float mx = *wmax;
  if (mx > 0.f) {
    frexpf(mx, &g);  // mx = m 2^g, m in [0.5, 1)
    g -= 15;
  }
  if (idx == 0) *wsc = ldexpf(1.f, g);
  if (idx >= (i64)Kp * KD2) return;
  const int k = (int)(idx / KD2), e = (int)(idx % KD2);
  const int c = e / 32, ee = e % 32;
  float w = 0.f;
  if (k < K) w = (float)ldexp(tc_weight(means, covs, ctr, scale, wbar, k, e, D), -g);
  const __half hi = __float2half_rn(w);
  const __half lo = __float2half_rn(w - __half2float(hi));
  const size_t wbytes = (size_t)(KD2 / 32) * Kp * 64;
  const size_t off = (size_t)c * Kp * 64 + kmajor_sw64_off(k, ee / 8) + (ee % 8) * 2;
  char *base = (char *)wimg;
  *(__half *)(base + off) = hi;
  *(__half *)(base + wbytes + off) = lo;
}

// c_k = log2(e) * (log pi_k - D/2 log 2pi - 1/2 sum log s2 - 1/2 sum mu'^2/s2)
// in double, -inf for padding and for priors below 1e-6 (vl/gmm.c:746-747).
__global__ void k_tc_cst(const float *__restrict__ priors, const float *__restrict__ means,
                         const float *__restrict__ covs, const float *__restrict__ ctr, int K,
                         int Kp, int D, double *__restrict__ cst64) {
  // One warp per component; lanes take dimensions d = lane, lane + 32, ...
  const int k = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x % 32;
  if (k >= Kp) return;
  if (k >= K || (double)priors[k] < 1e-6) {
    if (lane == 0) cst64[k] = -INFINITY;
    return;
  }
  double c = 0;
  for (int d = lane; d < D; d += 32) {
    const double s2 = (double)covs[(i64)k * D + d];
    const double mup = (double)means[(i64)k * D + d] - (double)ctr[d];
    c += 0.5 * log(s2) + 0.5 * mup * mup / s2;
  }
  c = log((double)priors[k]) - 0.5 * (double)D * log(2.0 * 3.141592653589793) - warp_sum(c);
  if (lane == 0) cst64[k] = c * 1.4426950408889634;
}

// cst2_k = c_k - cbar in float, with cbar the mean of the finite c_k (one
// warp, fixed-order sums; 0 when every component is skipped).  Like wbar,
// cbar is common to all components: the posteriors do not see it, the float
// constants carry less rounding, and the log-likelihood adds it back.
__global__ void k_tc_cst_center(const double *__restrict__ cst64, int Kp, float *__restrict__ cst2,
                                double *__restrict__ cbar) {
  const int lane = threadIdx.x;
  double s = 0, n = 0;
  for (int k = lane; k < Kp; k += 32)
    if (cst64[k] != -INFINITY) {
      s += cst64[k];
      n += 1;
    }
  s = warp_sum(s);
  n = warp_sum(n);
  const double c = n > 0 ? s / n : 0.0;
  for (int k = lane; k < Kp; k += 32) cst2[k] = cst64[k] == -INFINITY ? -INFINITY : (float)(cst64[k] - c);
  if (lane == 0) *cbar = c;
}

// Per-dimension power-of-two scale for fp16 statistics operands, chosen from
// the model so that x'' = x' * scale is O(1) for data the model describes:
// scale_d = 2^-ceil(log2(max_k |mu'_kd| + 4 sigma_kd)).
__global__ void k_tc_scale(const float *__restrict__ means, const float *__restrict__ covs,
                           const float *__restrict__ ctr, int K, int D, float *__restrict__ scale) {
  // One warp per dimension; the maximum does not depend on the order.
  const int d = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x % 32;
  if (d >= D) return;
  double b = 0;
  for (int k = lane; k < K; k += 32) {
    const double v = fabs((double)means[(i64)k * D + d] - (double)ctr[d]) + 4.0 * sqrt((double)covs[(i64)k * D + d]);
    b = v > b ? v : b;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
  if (lane != 0) return;
  int e = 0;
  if (b > 0) frexp(b, &e);
  scale[d] = (float)ldexp(1.0, -e);
}

// ============================================================ E-step
// Finite values beyond fp16's range are clamped to it; NaN and +-inf pass
// through, so that a non-finite descriptor gives a non-finite result, as in
// the reference's float arithmetic.
__device__ __forceinline__ float clamp_f16(float v) {
  return fabsf(v) < INFINITY ? fminf(fmaxf(v, -65504.f), 65504.f) : v;
}

// The q image holds q * 2^14 in fp16 (one part, or hi and lo parts): every
// posterior the statistics keep (q >= 1e-6) is then a normal fp16 number.
// The statistics' finalizers multiply by 2^-14.
constexpr float kQScale = 16384.f;

// Output layouts of the posteriors written by the E-step.
//   kQRow    fp32, row-major q[i * ldq + k] (VLFeat's layout; EM and API).
//   kQImg16  fp16 operand image of q^T (times 2^14) for the statistics GEMM: per
//            32-component block, the 8-row groups of all rows in order, each
//            an MN-major 64-byte-swizzled 512-byte atom (32 components x 8
//            rows; qimg_off).  An E-step warp's 32 rows x 32 components are
//            one 2 KB block, written by one bulk copy from shared memory, and
//            the statistics' A operand for 32 rows (4 groups of each of its
//            blocks) is one 4-D TMA box of the image.
//   kQImg32  the same image as two fp16 parts (hi, lo) for fp16x3 statistics.
//   kQRowImg16, kQRowImg32  both: the row-major posteriors (unthresholded)
//            and the image (thresholded), for EM with the tensor-core M-step.
constexpr int kQRow = 0, kQImg16 = 1, kQImg32 = 2, kQRowImg16 = 3, kQRowImg32 = 4;
// Byte offset in an image part of `ngroups` 8-row groups of the 16-byte chunk
// with components [8 k8, 8 k8 + 8) of row r.
__host__ __device__ __forceinline__ size_t qimg_off(i64 ngroups, i64 r, uint32_t k8) {
  return ((size_t)(k8 >> 2) * (size_t)ngroups + (size_t)(r >> 3)) * 512u + mnmajor_sw64_off((uint32_t)(r & 7), k8 & 3u);
}
__host__ __device__ constexpr bool q_rows(int qf) { return qf == kQRow || qf == kQRowImg16 || qf == kQRowImg32; }
__host__ __device__ constexpr bool q_image(int qf) { return qf != kQRow; }
__host__ __device__ constexpr bool q_image32(int qf) { return qf == kQImg32 || qf == kQRowImg32; }

struct EParams {
  CUtensorMap xmap;  // SW: X as a {D, N} fp32 tensor, boxes of 16 dimensions x 128 rows
  const float *X;
  i64 N;
  // Kp: this CTA's components (at most 256); Kg: all padded components (the
  // W image's and cst2's extent; Kp times the cluster size); Kq: components in
  // the q image (Kg rounded up to 128).
  int K, Kp, Kg, Kq, nst;
  int nxs;    // SW: boxes in the ring of descriptor rows
  i64 qpart;  // bytes of one part of the q image
  const uint4 *wimg;
  const float *cst2;
  const float *ctr;
  const float *scl;  // per-dimension power-of-two scale of x' (the operands are x'' = x' scale)
  const float *wsc;  // the W image's power-of-two scale (one float, device)
  const float *wbar;   // common part of the x''^2 weights (log2 units), taken out of W
  const double *cbar;  // common part of the constants (log2 units), taken out of cst2
  void *q;     // row-major posteriors (kQRow*) or the image (kQImg*)
  void *qimg;  // the image of the combined formats
  int ldq;
  int fast;
  float qthr;  // image outputs: posteriors below this are stored as 0 (vl/fisher.c:440)
  unsigned *rowcnt;
  double *ll_part;
  int *err;
  i64 ntiles;
};

// Shared-memory layout of the E-step.  With W resident (SW false) the W
// image (hi + lo) is copied in once and the producers load the descriptor
// rows into registers.  With W streamed (SW true) each operand stage also
// holds the k-atom of W its MMAs read, bulk-copied from global memory (L2)
// when the stage is filled, and the freed space holds a ring of TMA boxes of
// descriptor rows (128 rows x 16 dimensions, fp32) that the producers read.
template <int DIM, bool SW = false, bool CL = false>
struct ELayout {
  static constexpr int KD2 = 2 * DIM;
  static constexpr int NKA = KD2 / 32;
  static constexpr int kStage = 2 * 8192;  // hi + lo parts of one 128 x 32 chunk
  // Epilogue staging: each of the 8 epilogue warps lays out its 32 rows x 32
  // components of the q image (one 2 KB block) in shared memory for one bulk
  // copy to global memory; two buffers per warp (one with W resident) so the
  // next block is formed while the previous copy reads its buffer.
  static constexpr int kStageBufs = SW ? 2 : 1;
  static constexpr int kStaging = 8 * 2048 * kStageBufs;
  __host__ __device__ static size_t wbytes(int Kp) { return (size_t)NKA * Kp * 64; }
  __host__ __device__ static size_t wstage(int Kp) { return SW ? (size_t)2 * Kp * 64 : 0; }
  __host__ __device__ static size_t stage(int Kp) { return kStage + wstage(Kp); }
  // Cluster exchange slots: per TMEM buffer, 128 rows of (max, sum, argmax).
  static constexpr int kXch = CL ? 2 * 128 * 16 : 0;
  static constexpr int kXBox = 128 * 16 * 4;  // one box of descriptor rows
  static size_t fixed(int Kp) {
    return (SW ? 0 : 2 * wbytes(Kp)) + 1024 /*cst*/ + 2048 /*ctr, bars*/ + kStaging + kXch + 1024 /*alignment*/;
  }
  static int max_stages(int Kp, int nxs = 0) {
    const size_t f = fixed(Kp) + (size_t)nxs * kXBox;
    return f >= (size_t)kSmemLimit ? 0 : (int)((kSmemLimit - f) / stage(Kp));
  }
  static size_t bytes(int Kp, int nst, int nxs = 0) { return fixed(Kp) + (size_t)nst * stage(Kp) + (size_t)nxs * kXBox; }
};

// CL: the components are split over the CTAs of a thread-block cluster (K
// above 256): CTA r computes the logits of components [r Kp, (r+1) Kp) for
// every tile of its cluster, and after pass A the CTAs exchange each row's
// running maximum and sum through distributed shared memory, so that pass B
// normalises with the row's log-sum-exp over all K.
template <int DIM, int QF, bool FAST, bool SW = false, bool CL = false>
__global__ void __launch_bounds__(tc_threads(SW), 1) k_tc_estep(const __grid_constant__ EParams p) {
  using L = ELayout<DIM, SW, CL>;
  constexpr int NKA = L::NKA;
  constexpr int NT = tc_threads(SW);
  extern __shared__ uint8_t smem_raw[];
  uint8_t *base = align1024(smem_raw);
  const uint32_t wbytes = (uint32_t)L::wbytes(p.Kp);
  const uint32_t stageBytes = (uint32_t)L::stage(p.Kp);
  const uint32_t wpart = (uint32_t)p.Kp * 64;  // one k-atom of one W part
  uint8_t *sW = base;
  uint8_t *sA = sW + (SW ? 0 : 2 * wbytes);
  uint8_t *sX = sA + (size_t)p.nst * stageBytes;  // SW: ring of nxs boxes of descriptor rows
  float *s_cst = (float *)(sX + (SW ? (size_t)p.nxs * L::kXBox : 0));
  float *s_ctr = s_cst + 256;                     // DIM <= 128 floats
  uint64_t *bars = (uint64_t *)(s_ctr + 128);     // 84 barriers, then TMEM base and abort flag
  uint64_t *full = bars, *empty = bars + 16, *accf = bars + 32, *acce = bars + 34;
  uint64_t *xready = bars + 36, *xcons = bars + 44;  // cluster exchange: [buffer][epilogue warp]
  uint64_t *xfull = bars + 52, *xempty = bars + 60;  // SW: descriptor-row boxes
  uint64_t *wfull = bars + 68;                       // SW: W k-atoms, per stage
  uint32_t *s_tmem = (uint32_t *)(bars + 84);
  volatile int *s_abort = (volatile int *)(s_tmem + 1);
  uint8_t *s_stage = (uint8_t *)(s_cst + 768);   // 8 x 2 KB epilogue staging
  float4 *s_xch = (float4 *)(s_stage + L::kStaging);  // [buffer][row] (max, sum, argmax) when CL
  // This CTA's components and tiles: with CL the cluster shares each tile.
  const int crank = CL ? (int)cluster_rank() : 0, ncta = CL ? (int)cluster_size() : 1;
  const int kbase = crank * p.Kp;
  const i64 tile0 = blockIdx.x / ncta, tstep = gridDim.x / ncta;
  const size_t wbytesG = (size_t)NKA * p.Kg * 64;  // the global W image's part size

  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  if (tid == 0) {
    for (int s = 0; s < p.nst; ++s) {
      mbar_init(&full[s], 128);
      mbar_init(&empty[s], 1);
      if (SW) mbar_init(&wfull[s], 1);
    }
    if (SW)
      for (int b = 0; b < p.nxs; ++b) {
        mbar_init(&xfull[b], 1);
        mbar_init(&xempty[b], 128);
      }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 128);
    }
    if (CL)
      for (int b = 0; b < 8; ++b) {
        mbar_init(&xready[b], ncta);
        mbar_init(&xcons[b], ncta);
      }
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 12) {
    tmem_alloc(s_tmem, 512);
    tmem_relinquish();
  }
  // Resident W (this CTA's rows of the pre-swizzled image: per part and
  // k-atom, Kp rows of 64 bytes) and per-component constants.
  {
    const uint4 *src = p.wimg;
    uint4 *dst = (uint4 *)sW;
    const int n16 = SW ? 0 : (int)(2 * wbytes / 16);
    const int part16 = (int)(wbytes / 16), atom16 = (int)(wpart / 16);
    for (int i = tid; i < n16; i += NT) {
      const int part = i / part16, rem = i % part16, c = rem / atom16, o = rem % atom16;
      dst[i] = src[(part * wbytesG + (size_t)c * p.Kg * 64 + (size_t)kbase * 64) / 16 + o];
    }
    for (int k = tid; k < 256; k += NT) s_cst[k] = k < p.Kp ? p.cst2[kbase + k] : -INFINITY;
    fence_proxy_async_smem();
  }
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;

  if (warp < 4) {
    // ---------------------------------------------------- producers
    // Warp w owns rows [32w, 32w+32) of each tile.  Chunk c of the A row is
    // [x'_d, x'_d^2] for d = 16c .. 16c+15 (the K order of the W image), so
    // lane (rg, part) reads dimensions 16c + 4 part .. +3 of rows
    // 32w + 8s + rr, s = 0..3, once and writes both the x' and the x'^2
    // elements: each load instruction reads 8 rows x 64 contiguous bytes.
    // rr permutes rg so that the 16 lanes of each half-warp store to 16
    // distinct bank groups of the 64-byte-swizzled stage.  With W resident
    // the rows come from global memory, the next chunks' rows prefetched into
    // registers while the current chunk is converted; with W streamed they
    // come from the loader warp's ring of TMA boxes (one box per chunk: 128
    // rows x 64 bytes, rows past N zero-filled), read 8 rows x 64 contiguous
    // bytes per instruction.
    const int part = lane & 3, rg = lane >> 2;
    const int rr = (rg & 1) | ((rg & 2) << 1) | ((rg & 4) >> 1);
    auto load = [&](float4(&buf)[4], i64 t, int c) {
      const int d0 = 16 * c + 4 * part;
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const i64 row = t * 128 + 32 * warp + 8 * s + rr;
        buf[s] = row < p.N ? __ldg((const float4 *)(p.X + row * DIM + d0)) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
    };
    // Position (tile, chunk) of the chunk being converted and, with W
    // resident, of the next two, whose rows are already in flight (a 3-deep
    // register prefetch ring).
    i64 t0 = tile0, t1, t2;
    int c0 = 0, c1, c2, it = 0;
    // Log-likelihood: the common parts taken out of the logits, per row
    // sum_d wbar_d x''_d^2 + cbar (log2 units), summed in double in a fixed
    // order (this lane's rows and dimensions over the tile's chunks, then the
    // warp's butterfly) and written as the warp's partial for the tile, after
    // the epilogue's partials (ll_part[4 ntiles + 4 tile + warp]).
    const bool want_ll = p.ll_part != nullptr && crank == 0;
    const double cb = want_ll ? *p.cbar : 0.0;
    double cacc = 0.0;
    auto adv = [&](i64 t, int c, i64 &tn, int &cn) {
      tn = t;
      cn = c + 1;
      if (cn == NKA) {
        cn = 0;
        tn += tstep;
      }
    };
    // Converts chunk (t0, c0), whose rows are in cur, into operand stage it % nst.
    auto put = [&](const float4(&cur)[4]) -> bool {
      const int stage = it % p.nst;
      if (!mbar_wait(&empty[stage], ((it / p.nst) & 1) ^ 1, s_abort, p.err, 1)) return false;
      const uint32_t a_hi = smem_u32(sA + (size_t)stage * stageBytes);
      const int d0 = 16 * c0 + 4 * part;
      const float4 mm = __ldg((const float4 *)(p.ctr + d0)), sc = __ldg((const float4 *)(p.scl + d0));
      const float4 wb = want_ll ? __ldg((const float4 *)(p.wbar + d0)) : make_float4(0.f, 0.f, 0.f, 0.f);
      const unsigned long long m01 = f2u(mm.x, mm.y), m23 = f2u(mm.z, mm.w);
      const unsigned long long s01 = f2u(sc.x, sc.y), s23 = f2u(sc.z, sc.w);
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        // x'' = (x - ctr) scale (packed pairs, the scalar roundings), clamped
        // to fp16's finite range (an x'' beyond it is more than 255 model
        // scales from the centre); NaN passes.
        const unsigned long long d01 = mul2(sub2(f2u(cur[s].x, cur[s].y), m01), s01);
        const unsigned long long d23 = mul2(sub2(f2u(cur[s].z, cur[s].w), m23), s23);
        const float v0 = clamp_f16n(lo32(d01)), v1 = clamp_f16n(hi32(d01));
        const float v2 = clamp_f16n(lo32(d23)), v3 = clamp_f16n(hi32(d23));
        if (want_ll && t0 * 128 + 32 * warp + 8 * s + rr < p.N)
          cacc += (double)wb.x * ((double)v0 * v0) + (double)wb.y * ((double)v1 * v1) +
                  (double)wb.z * ((double)v2 * v2) + (double)wb.w * ((double)v3 * v3);
        // x''^2, at most fp16's max; plus d * 0, which is +-0 for a finite
        // difference and NaN for an infinite one, so that a non-finite x
        // still makes the row's logits NaN (as the reference's arithmetic
        // makes its posteriors).
        const unsigned long long p01 = mul2(f2u(v0, v1), f2u(v0, v1)), p23 = mul2(f2u(v2, v3), f2u(v2, v3));
        const unsigned long long q01 = add2(f2u(fminf(lo32(p01), 65504.f), fminf(hi32(p01), 65504.f)), mul2(d01, 0ull));
        const unsigned long long q23 = add2(f2u(fminf(lo32(p23), 65504.f), fminf(hi32(p23), 65504.f)), mul2(d23, 0ull));
        uint32_t h0, l0, h1, l1, h2, l2, h3, l3;
        split2<true>(v0, v1, h0, l0);
        split2<true>(v2, v3, h1, l1);
        split2<true>(lo32(q01), hi32(q01), h2, l2);
        split2<true>(lo32(q23), hi32(q23), h3, l3);
        const uint32_t row = (uint32_t)(32 * warp + 8 * s + rr);
        const uint32_t o1 = kmajor_sw64_off(row, (uint32_t)(part >> 1)) + (part & 1) * 8;
        const uint32_t o2 = kmajor_sw64_off(row, (uint32_t)(2 + (part >> 1))) + (part & 1) * 8;
        st_shared_v2(a_hi + o1, h0, h1);
        st_shared_v2(a_hi + 8192 + o1, l0, l1);
        st_shared_v2(a_hi + o2, h2, h3);
        st_shared_v2(a_hi + 8192 + o2, l2, l3);
      }
      fence_proxy_async_smem();
      mbar_arrive(&full[stage]);
      if (want_ll && c0 == NKA - 1) {
        const double v = warp_sum(cacc);
        if (lane == 0) {
          const i64 r0 = t0 * 128 + 32 * warp;
          const i64 nv = p.N - r0 < 0 ? 0 : (p.N - r0 > 32 ? 32 : p.N - r0);
          p.ll_part[p.ntiles * 4 + t0 * 4 + warp] = (v + (double)nv * cb) * kLn2;
        }
        cacc = 0.0;
      }
      return true;
    };
    if constexpr (SW) {
      while (t0 < p.ntiles) {
        const int xs = it % p.nxs;
        if (!mbar_wait(&xfull[xs], (it / p.nxs) & 1, s_abort, p.err, 9)) break;
        float4 cur[4];
        const uint8_t *xb = sX + (size_t)xs * L::kXBox + (size_t)(32 * warp + rr) * 64 + part * 16;
#pragma unroll
        for (int s = 0; s < 4; ++s) cur[s] = *(const float4 *)(xb + s * 8 * 64);
        if (!put(cur)) break;
        // The slot is released after put()'s proxy fence: these generic reads
        // of the box must be ordered before the loader's next TMA (async
        // proxy) write into it, which the mbarrier alone does not do.
        mbar_arrive(&xempty[xs]);
        ++it;
        adv(t0, c0, t0, c0);
      }
    } else {
      float4 b0[4], b1[4], b2[4];
      adv(t0, c0, t1, c1);
      adv(t1, c1, t2, c2);
      if (t0 < p.ntiles) load(b0, t0, c0);
      if (t1 < p.ntiles) load(b1, t1, c1);
      auto step = [&](float4(&cur)[4], float4(&fut)[4]) -> bool {
        if (t0 >= p.ntiles) return false;
        if (t2 < p.ntiles) load(fut, t2, c2);
        if (!put(cur)) return false;
        ++it;
        t0 = t1; c0 = c1;
        t1 = t2; c1 = c2;
        adv(t1, c1, t2, c2);
        return true;
      };
      while (step(b0, b2) && step(b1, b0) && step(b2, b1)) {
      }
    }
  } else if (warp < 12) {
    // ----------------------------------------------------- epilogue
    // Two warpgroups: group g drains the tiles whose accumulator is TMEM
    // buffer g (alternate tiles), so one tile's log-sum-exp overlaps the
    // next tile's stores and the two groups keep different pipes busy.
    // Warp w reads TMEM lanes 32 (w % 4) .. +31, i.e. rows of the tile.
    // Arithmetic on pairs of columns uses packed f32x2 instructions.
    const int eg = (warp - 4) >> 2, ew = warp & 3;
    const int r = ew * 32 + lane;
    const int nch = p.Kp / 32;
    // Image chunks this CTA writes: its own, and (last CTA) the zero padding
    // from Kg to Kq.
    const int ncw = q_image(QF) ? nch + (crank == ncta - 1 ? (p.Kq - p.Kg) / 32 : 0) : nch;
    const unsigned long long *cst2v = (const unsigned long long *)s_cst;
    const float wsc = *p.wsc;
    const unsigned long long wsc2 = f2u(wsc, wsc);
    uint8_t *stg = s_stage + (warp - 4) * 2048 * L::kStageBufs;
    int sb = 0;  // staging buffer the next image block is formed in
    int tt = 0;
    for (i64 tile = tile0; tile < p.ntiles; tile += tstep, ++tt) {
      const int buf = tt & 1;
      if (buf != eg) continue;
      if (!mbar_wait(&accf[buf], (tt >> 1) & 1, s_abort, p.err, 2)) break;
      tc_fence_after();
      const uint32_t tb = tmem + ((uint32_t)(ew * 32) << 16) + (uint32_t)(buf * 256);
      // Pass A: online log-sum-exp over 64-column groups.  e = 2^(s - m_g)
      // is written back to TMEM with the running maximum m_g of its group.
      float m = -INFINITY, sum = 0.f, mg[4];
      int am = 0;
#pragma unroll 1
      for (int pc = 0; pc < nch; pc += 2) {
        const bool two = pc + 1 < nch;
        uint32_t va[32], vb[32];
        tmem_ld32(tb + pc * 32, va);
        if (two) tmem_ld32(tb + pc * 32 + 32, vb);
        tmem_wait_ld();
        float cm = -INFINITY;
        int cam = 0;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const unsigned long long s = fma2(f2u(__uint_as_float(va[2 * j]), __uint_as_float(va[2 * j + 1])),
                                            wsc2, cst2v[pc * 16 + j]);
          va[2 * j] = __float_as_uint(lo32(s));
          va[2 * j + 1] = __float_as_uint(hi32(s));
          if (FAST) {
            if (lo32(s) > cm) { cm = lo32(s); cam = pc * 32 + 2 * j; }
            if (hi32(s) > cm) { cm = hi32(s); cam = pc * 32 + 2 * j + 1; }
          } else {
            cm = max3f(cm, lo32(s), hi32(s));
          }
        }
        if (two) {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const unsigned long long s = fma2(f2u(__uint_as_float(vb[2 * j]), __uint_as_float(vb[2 * j + 1])),
                                              wsc2, cst2v[pc * 16 + 16 + j]);
            vb[2 * j] = __float_as_uint(lo32(s));
            vb[2 * j + 1] = __float_as_uint(hi32(s));
            if (FAST) {
              if (lo32(s) > cm) { cm = lo32(s); cam = pc * 32 + 32 + 2 * j; }
              if (hi32(s) > cm) { cm = hi32(s); cam = pc * 32 + 32 + 2 * j + 1; }
            } else {
              cm = max3f(cm, lo32(s), hi32(s));
            }
          }
        }
        if (cm > m) {
          sum = (m == -INFINITY) ? 0.f : sum * ex2_approx(m - cm);
          m = cm;
          if (FAST) am = cam;
        }
        const unsigned long long nm = f2u(-m, -m);
        unsigned long long acc = 0ull;  // two partial sums (+0.0f, +0.0f)
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const unsigned long long d = add2(f2u(__uint_as_float(va[2 * j]), __uint_as_float(va[2 * j + 1])), nm);
          const float e0 = ex2_approx(lo32(d)), e1 = ex2_approx(hi32(d));
          acc = add2(acc, f2u(e0, e1));
          va[2 * j] = __float_as_uint(e0);
          va[2 * j + 1] = __float_as_uint(e1);
        }
        tmem_st32(tb + pc * 32, va);
        if (two) {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const unsigned long long d = add2(f2u(__uint_as_float(vb[2 * j]), __uint_as_float(vb[2 * j + 1])), nm);
            const float e0 = ex2_approx(lo32(d)), e1 = ex2_approx(hi32(d));
            acc = add2(acc, f2u(e0, e1));
            vb[2 * j] = __float_as_uint(e0);
            vb[2 * j + 1] = __float_as_uint(e1);
          }
          tmem_st32(tb + pc * 32 + 32, vb);
        }
        sum += lo32(acc) + hi32(acc);
        mg[pc >> 1] = m;
      }
      tmem_wait_st();
      float mt = m, st = sum;
      if constexpr (CL) {
        // Exchange (max, sum, argmax) of each row with the cluster and
        // combine them in rank order, identically in every CTA.
        uint64_t *xr = &xready[buf * 4 + ew], *xc = &xcons[buf * 4 + ew];
        float4 *slot = s_xch + buf * 128;
        const int use = tt >> 1;
        if (use > 0 && !mbar_wait_cluster(xc, (use + 1) & 1, s_abort, p.err, 5)) break;
        slot[r] = make_float4(m, sum, __int_as_float(kbase + am), 0.f);
        fence_acq_rel_cluster();
        __syncwarp();
        if (lane < ncta) mbar_arrive_remote(xr, (uint32_t)lane);
        if (!mbar_wait_cluster(xr, use & 1, s_abort, p.err, 6)) break;
        float4 v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (q < ncta) v[q] = ld_dsmem_f4(&slot[r], (uint32_t)q);
        float M = -INFINITY, S = 0.f;
        int amg = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (q < ncta && v[q].x > M) {  // first rank wins ties: first index, vl/fisher.c:406
            M = v[q].x;
            amg = __float_as_int(v[q].z);
          }
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (q < ncta && v[q].x != -INFINITY) S += v[q].y * ex2_approx(v[q].x - M);
        __syncwarp();
        if (lane < ncta) mbar_arrive_remote(xc, (uint32_t)lane);
        mt = M;
        st = S;
        if (FAST) am = amg - kbase;
      }
      const float inv = 1.f / st;
      const i64 row = tile * 128 + r;
      const bool valid = row < p.N;
      unsigned long long cnt2 = 0ull;  // (+0.0f, +0.0f): per-row term counts, exact below 2^24
      // The image-only formats form q 2^14 directly (the scale folded into the
      // row's normaliser) and test it against qthr 2^14: power-of-two scaling
      // keeps every comparison, and the flags, exact.
      constexpr bool kImgOnly = (QF == kQImg16 || QF == kQImg32);
      constexpr float kQs = kImgOnly ? kQScale : 1.f;   // scale of qv below
      constexpr float kPack = kImgOnly ? 1.f : kQScale;  // still to apply when packing the image
      // -prev(qthr) * 2^64 (times the scale), prev(qthr) the largest float below qthr (> 0).
      const float nthr = -__uint_as_float(__float_as_uint(p.qthr) - 1u) * (0x1p64f * kQs);
      // q image; this warp's rows are the tile's 8-row groups 4 ew .. 4 ew + 3.
      uint8_t *ib = (uint8_t *)(q_rows(QF) ? p.qimg : p.q);
      const size_t blockBytes = (size_t)p.ntiles * 16 * 512;  // one 32-component block of all rows
      // Image blocks: lane = row writes its 64 bytes (four 16-byte chunks)
      // into the staging buffer in the image's own layout (the 64-byte
      // swizzle keeps each 8-lane group on distinct banks), then lane 0 copies
      // the 2 KB block to the image with one bulk copy (component block
      // kbase / 32 + cc, the tile's row groups 4 ew .. 4 ew + 3).  Before a
      // buffer is refilled, the copy that last read it has finished reading.
      auto stage_put = [&](int j, const uint4 &w) {
        *(uint4 *)(stg + sb * 2048 + (lane >> 3) * 512 + mnmajor_sw64_off((uint32_t)(lane & 7), (uint32_t)j)) = w;
      };
      auto stage_out = [&](int cc, size_t part_off) {
        fence_proxy_async_smem();  // this lane's staging writes, before the copy reads them
        __syncwarp();
        if (lane == 0) {
          bulk_s2g(ib + part_off + (size_t)(kbase / 32 + cc) * blockBytes + ((size_t)tile * 16 + 4 * ew) * 512,
                   smem_u32(stg + sb * 2048), 2048);
          bulk_commit();
          bulk_wait_read<L::kStageBufs - 1>();
        }
        __syncwarp();
        sb = sb + 1 == L::kStageBufs ? 0 : sb + 1;
      };
      // Pass B: q = e * 2^(m_g - m) / sum, thresholded, one 32-column chunk at
      // a time.  TMEM loads and staging stay warp-uniform; rows past N (tile
      // padding) and image columns past Kp are zeros.
#pragma unroll 1
      for (int cc = 0; cc < ncw; ++cc) {
        float qv[32];
        const bool ha = cc < nch;
        const bool live = valid && ha;
        if (ha) {
          uint32_t va[32];
          tmem_ld32(tb + cc * 32, va);
          tmem_wait_ld();
          const float sc = live ? ex2_approx(mg[cc >> 1] - mt) * (inv * kQs) : 0.f;
          const unsigned long long sc2 = f2u(sc, sc);
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            float x0, x1;
            if (FAST) {
              x0 = (live && cc * 32 + 2 * j == am) ? kQs : 0.f;  // am: this CTA's columns
              x1 = (live && cc * 32 + 2 * j + 1 == am) ? kQs : 0.f;
            } else {
              const unsigned long long q2 = mul2(f2u(__uint_as_float(va[2 * j]), __uint_as_float(va[2 * j + 1])), sc2);
              x0 = lo32(q2);
              x1 = hi32(q2);
            }
            // Keep flags (1.0 / 0.0) for q >= qthr, counted in packed float
            // pairs and, for the image, applied by a packed multiply.  The
            // flag is sat((q - prev(qthr)) 2^64), exact in one fma: the
            // difference is either <= 0 or at least one ulp of qthr.
            const unsigned long long kk = f2u(__saturatef(fmaf(x0, 0x1p64f, nthr)),
                                              __saturatef(fmaf(x1, 0x1p64f, nthr)));
            cnt2 = add2(cnt2, kk);
            if (QF == kQImg16 || QF == kQImg32) {
              const unsigned long long xk = mul2(f2u(x0, x1), kk);
              x0 = lo32(xk);
              x1 = hi32(xk);
            }
            qv[2 * j] = x0;
            qv[2 * j + 1] = x1;
          }
        } else {
#pragma unroll
          for (int j = 0; j < 32; ++j) qv[j] = 0.f;
        }
        if (q_rows(QF)) {
          if (live) {
            const int k0 = kbase + cc * 32;
            float *dst = (float *)p.q + row * p.ldq + k0;
            if (k0 + 32 <= p.K) {
#pragma unroll
              for (int j = 0; j < 32; j += 4)
                *(float4 *)(dst + j) = make_float4(qv[j], qv[j + 1], qv[j + 2], qv[j + 3]);
            } else {
#pragma unroll
              for (int j = 0; j < 32; ++j)
                if (k0 + j < p.K) dst[j] = qv[j];
            }
          }
        }
        if (q_image(QF)) {
          if (q_rows(QF)) {
            // Combined formats: the rows above keep every posterior; the image
            // keeps those >= qthr (the same flag as in the loop above).
#pragma unroll
            for (int j = 0; j < 32; ++j) qv[j] *= __saturatef(fmaf(qv[j], 0x1p64f, nthr));
          }
          // The hi part goes to the staging as it is formed; the lo part
          // waits in registers for the next buffer.
          uint4 wl[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            uint4 wh;
            if (!q_image32(QF)) {
              wh.x = pack2<true>(qv[8 * j + 0] * kPack, qv[8 * j + 1] * kPack);
              wh.y = pack2<true>(qv[8 * j + 2] * kPack, qv[8 * j + 3] * kPack);
              wh.z = pack2<true>(qv[8 * j + 4] * kPack, qv[8 * j + 5] * kPack);
              wh.w = pack2<true>(qv[8 * j + 6] * kPack, qv[8 * j + 7] * kPack);
            } else {
              split2<true>(qv[8 * j + 0] * kPack, qv[8 * j + 1] * kPack, wh.x, wl[j].x);
              split2<true>(qv[8 * j + 2] * kPack, qv[8 * j + 3] * kPack, wh.y, wl[j].y);
              split2<true>(qv[8 * j + 4] * kPack, qv[8 * j + 5] * kPack, wh.z, wl[j].z);
              split2<true>(qv[8 * j + 6] * kPack, qv[8 * j + 7] * kPack, wh.w, wl[j].w);
            }
            stage_put(j, wh);
          }
          stage_out(cc, 0);
          if (q_image32(QF)) {
#pragma unroll
            for (int j = 0; j < 4; ++j) stage_put(j, wl[j]);
            stage_out(cc, (size_t)p.qpart);
          }
        }
      }
      tc_fence_before();
      mbar_arrive(&acce[buf]);
      if (valid && p.rowcnt) {
        const unsigned cnt = (unsigned)(lo32(cnt2) + hi32(cnt2));
        if (CL) atomicAdd(&p.rowcnt[row], cnt);  // zeroed by the launcher
        else p.rowcnt[row] = cnt;
      }
      // Per-warp log-likelihood partial (fixed shuffle order): 4 per tile.
      double ll = valid ? ((double)mt + log2((double)st)) * kLn2 : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) ll += __shfl_xor_sync(0xffffffffu, ll, o);
      if (lane == 0 && p.ll_part && crank == 0) p.ll_part[tile * 4 + ew] = ll;
    }
    // The image blocks' copies complete before the block exits.
    if (q_image(QF) && lane == 0) bulk_wait_all();
  } else if (warp == 12 && lane == 0) {
    // ---------------------------------------------------------- MMA
    const uint32_t idesc = idesc_f16(128, p.Kp, false, false);
    const uint32_t w_hi = smem_u32(sW), w_lo = w_hi + wbytes;
    int it = 0, tt = 0;
    bool ok = true;
    for (i64 tile = tile0; tile < p.ntiles && ok; tile += tstep, ++tt) {
      const int buf = tt & 1;
      if (!mbar_wait(&acce[buf], ((tt >> 1) & 1) ^ 1, s_abort, p.err, 3)) break;
      tc_fence_after();
      const uint32_t d = tmem + (uint32_t)(buf * 256);
      for (int c = 0; c < NKA; ++c) {
        const int stage = it % p.nst;
        if (!mbar_wait(&full[stage], (it / p.nst) & 1, s_abort, p.err, 4) ||
            (SW && !mbar_wait(&wfull[stage], (it / p.nst) & 1, s_abort, p.err, 20))) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t a_hi = smem_u32(sA + (size_t)stage * stageBytes);
        const uint32_t b_hi = SW ? a_hi + L::kStage : w_hi + c * wpart;
        const uint32_t b_lo = SW ? a_hi + L::kStage + wpart : w_lo + c * wpart;
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
          const uint64_t ah = sdesc(a_hi + ks * 32, 16, 512, kSw64);
          const uint64_t al = sdesc(a_hi + 8192 + ks * 32, 16, 512, kSw64);
          const uint64_t bh = sdesc(b_hi + ks * 32, 16, 512, kSw64);
          const uint64_t bl = sdesc(b_lo + ks * 32, 16, 512, kSw64);
          mma_bf16(d, ah, bh, idesc, (c > 0 || ks > 0) ? 1u : 0u);
          mma_bf16(d, ah, bl, idesc, 1u);
          mma_bf16(d, al, bh, idesc, 1u);
        }
        mma_commit(&empty[stage]);
        ++it;
      }
      if (ok) mma_commit(&accf[buf]);
    }
  } else if (SW && warp == 13 && lane == 0) {
    // ------------------------------------------------------- loader
    // Chunk j of this CTA (tile tile0 + (j / NKA) tstep, chunk j % NKA): its
    // box of descriptor rows goes to ring slot j % nxs, up to nxs chunks
    // ahead of the operand stages, and its k-atom of W (hi and lo parts) to
    // stage j % nst once the MMAs have released the stage.
    const i64 ntl = tile0 < p.ntiles ? (p.ntiles - tile0 + tstep - 1) / tstep : 0;
    const i64 nchunks = ntl * NKA;
    i64 jx = 0, jw = 0;  // boxes and W atoms issued
    bool ok = true;
    for (; jw < nchunks && ok; ++jw) {
      for (; jx < nchunks && jx < jw + p.nxs; ++jx) {
        const int xs = (int)(jx % p.nxs);
        if (!mbar_wait(&xempty[xs], (uint32_t)((jx / p.nxs) & 1) ^ 1u, s_abort, p.err, 10)) {
          ok = false;
          break;
        }
        mbar_arrive_expect_tx(&xfull[xs], L::kXBox);
        tma_load_2d(smem_u32(sX + (size_t)xs * L::kXBox), &p.xmap, 16 * (int)(jx % NKA),
                    (int)((tile0 + (jx / NKA) * tstep) * 128), &xfull[xs]);
      }
      if (!ok) break;
      const int stage = (int)(jw % p.nst);
      if (!mbar_wait(&empty[stage], (uint32_t)((jw / p.nst) & 1) ^ 1u, s_abort, p.err, 17)) break;
      const uint32_t a_hi = smem_u32(sA + (size_t)stage * stageBytes);
      const uint8_t *w = (const uint8_t *)p.wimg + (size_t)(jw % NKA) * p.Kg * 64 + (size_t)kbase * 64;
      mbar_arrive_expect_tx(&wfull[stage], 2 * wpart);
      bulk_g2s(a_hi + L::kStage, w, wpart, &wfull[stage]);
      bulk_g2s(a_hi + L::kStage + wpart, w + wbytesG, wpart, &wfull[stage]);
    }
    // After an abort, copies still in flight land before the block exits:
    // wait (bounded, whatever the abort flag says) for the last box of each
    // ring slot and the last W atom of each stage.
    volatile int never = 0;
    for (i64 j = jx - 1; j >= 0 && j >= jx - p.nxs; --j)
      mbar_wait(&xfull[j % p.nxs], (uint32_t)((j / p.nxs) & 1), &never, p.err, 18);
    for (i64 j = jw - 1; j >= 0 && j >= jw - p.nst; --j)
      mbar_wait(&wfull[j % p.nst], (uint32_t)((j / p.nst) & 1), &never, p.err, 19);
  }
  tc_fence_before();
  __syncthreads();
  // No CTA leaves while another may still read its exchange slots (every
  // role's waits are bounded, so every CTA arrives here).
  if (CL) cg::this_cluster().sync();
  if (warp == 12) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// ========================================================== statistics
struct SItem {
  i64 row0, row1;  // absolute rows of X
  int slot, pad;
};

struct SParams {
  CUtensorMap qmap;     // the image as {256 (one atom, u16), groups, 32-component blocks, parts}
  const float *X;
  const uint8_t *qimg;  // q^T operand image written by the E-step
  i64 qpart;            // bytes of one image part
  i64 qbase;            // row of X that the image's first row corresponds to
  int K, Kp, Kq, nst;
  const float *ctr;
  const float *scale;  // per-dimension scale of x' (fp16 operands), or null
  const SItem *items;
  const int *order;     // item indices, grouped per CTA
  const int *cta_beg;   // gridDim.x + 1 offsets into order
  float *partial;       // [slot][Kp][NST]
  int *err;
};

// Operands are fp16: q 2^14 from the E-step's image and x'' = x' * scale.
// SPLIT 2: both split hi/lo, products hi.hi + hi.lo + lo.hi (fp16x3).
// SPLIT 1: q single fp16, x'' split hi/lo.
template <int DIM, int MT, int SPLIT>
struct SLayout {
  static constexpr int NST = 2 * DIM + 16;            // x', x'^2, [1, 0 x 15]
  static constexpr int NB = (NST + 63) / 64;           // 64-feature MN blocks
  static constexpr int NCH = (NST + 255) / 256;        // MMA N chunks
  static constexpr int NPA = SPLIT == 2 ? 2 : 1;       // q^T parts
  static constexpr int NPB = 2;                        // [x'', x''^2, 1] parts
  static constexpr int A_PART = MT * 4 * 4 * 512;      // [mnblk 4MT][kgroup 4][512 B atom]
  static constexpr int B_PART = NB * 4 * 1024;         // [kgroup 4][nblk NB][1 KB]
  static constexpr int XST = (32 * DIM * 4 + 1023) / 1024 * 1024;  // staged x rows
  static constexpr int kStage = NPA * A_PART + NPB * B_PART + XST;
  static constexpr size_t fixed = 1024 /*ctr*/ + 1024 /*scale*/ + 1024 /*bars*/ + 1024;
  static int max_stages() { return (int)((kSmemLimit - fixed) / kStage); }
  static size_t bytes(int nst) { return fixed + (size_t)nst * kStage; }
  static_assert(MT * NST <= 512, "accumulators exceed TMEM");
};

// Statistics block: converter warps 0-3 and 10-13, epilogue warps 4-7, MMA
// warp 8, loader warp 9.
constexpr int kStatsThreads = 448;
constexpr int kStatsConv = 256;  // converter threads

// Statistics over work items (runs of rows of one image): for each 32-row
// chunk, the loader warp bulk-copies the chunk's q^T operand (four 8-row
// groups of the E-step's image) straight into the operand stage and the
// chunk's x rows into a staging buffer; converter warps build the x-side
// operand [x'', x''^2, 1] (zero rows outside the item); one thread issues the
// MMAs; the epilogue drains the item's accumulators to its partial.
template <int DIM, int MT, int SPLIT>
__global__ void __launch_bounds__(kStatsThreads, 1) k_tc_stats(const __grid_constant__ SParams p) {
  using L = SLayout<DIM, MT, SPLIT>;
  constexpr int NST = L::NST, NB = L::NB, NPA = L::NPA;
  constexpr bool F16 = true;  // fp16 operands: the q image and x'' = x' scale
  constexpr int NF4 = DIM / 4;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *base = align1024(smem_raw);
  uint8_t *sS = base;
  float *s_ctr = (float *)(sS + (size_t)p.nst * L::kStage);
  float *s_scl = s_ctr + 256;
  uint64_t *bars = (uint64_t *)(s_scl + 256);
  uint64_t *full = bars, *empty = bars + 16, *xfull = bars + 32, *accf = bars + 48, *acce = bars + 49;
  uint32_t *s_tmem = (uint32_t *)(bars + 56);
  volatile int *s_abort = (volatile int *)(s_tmem + 1);

  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int comp0 = blockIdx.y * MT * 128;  // first component of this CTA's M tiles
  if (tid == 0) {
    for (int s = 0; s < p.nst; ++s) {
      mbar_init(&full[s], kStatsConv);
      mbar_init(&empty[s], 1);
      mbar_init(&xfull[s], 1);
    }
    mbar_init(accf, 1);
    mbar_init(acce, 128);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 8) {
    tmem_alloc(s_tmem, 512);
    tmem_relinquish();
  }
  for (int d = tid; d < DIM; d += kStatsThreads) {
    s_ctr[d] = p.ctr[d];
    s_scl[d] = p.scale ? p.scale[d] : 1.f;
  }
  // Zero the operand stages once: groups a chunk does not copy keep finite
  // stale values, and their x-side rows are zero.
  for (int s = 0; s < p.nst; ++s) {
    uint4 *st = (uint4 *)(sS + (size_t)s * L::kStage);
    for (int i = tid; i < (NPA * L::A_PART + L::NPB * L::B_PART) / 16; i += kStatsThreads) st[i] = make_uint4(0, 0, 0, 0);
  }
  fence_proxy_async_smem();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const int ib = p.cta_beg[blockIdx.x], ie = p.cta_beg[blockIdx.x + 1];

  if (warp == 9) {
    // ------------------------------------------------------- loader
    if (lane == 0) {
      int it = 0;
      bool ok = true;
      for (int ii = ib; ii < ie && ok; ++ii) {
        const SItem item = p.items[p.order[ii]];
        for (i64 cb = p.qbase + ((item.row0 - p.qbase) & ~(i64)7); cb < item.row1; cb += 32) {
          const int stage = it % p.nst;
          if (!mbar_wait(&empty[stage], ((it / p.nst) & 1) ^ 1, s_abort, p.err, 15)) {
            ok = false;
            break;
          }
          const uint32_t sa = smem_u32(sS + (size_t)stage * L::kStage);
          const uint32_t sx = sa + NPA * L::A_PART + L::NPB * L::B_PART;
          const int nx = (int)min((i64)32, item.row1 - cb);
          mbar_arrive_expect_tx(&xfull[stage], (uint32_t)(NPA * L::A_PART) + (uint32_t)nx * DIM * 4);
          // q^T for the chunk: groups (cb - qbase) / 8 .. +3 of this CTA's
          // 4 MT blocks, all parts, as one box laid out [part][block][group]
          // (groups past the image read as zero; groups past the item are
          // finite and meet zero x-side rows).
          tma_load_4d(sa, &p.qmap, 0, (int)((cb - p.qbase) >> 3), comp0 / 32, 0, &xfull[stage]);
          bulk_g2s(sx, p.X + cb * DIM, (uint32_t)nx * DIM * 4, &xfull[stage]);
          ++it;
        }
      }
    }
  } else if (warp < 4 || warp >= 10) {
    // ---------------------------------------------------- converters
    const int ctid = (warp < 4 ? warp : warp - 6) * 32 + lane;
    int it = 0;
    bool ok = true;
    for (int ii = ib; ii < ie && ok; ++ii) {
      const SItem item = p.items[p.order[ii]];
      for (i64 cb = p.qbase + ((item.row0 - p.qbase) & ~(i64)7); cb < item.row1; cb += 32) {
        const int stage = it % p.nst;
        if (!mbar_wait(&xfull[stage], (it / p.nst) & 1, s_abort, p.err, 11)) {
          ok = false;
          break;
        }
        const uint32_t sa = smem_u32(sS + (size_t)stage * L::kStage);
        const uint32_t sb = sa + NPA * L::A_PART;
        const float *xs = (const float *)(sS + (size_t)stage * L::kStage + NPA * L::A_PART + L::NPB * L::B_PART);
#pragma unroll
        for (int j = 0; j < (32 * NF4 + kStatsConv - 1) / kStatsConv; ++j) {
          const int i = ctid + kStatsConv * j;
          if (i >= 32 * NF4) break;
          const int rs = i / NF4, pp = i % NF4;
          const i64 row = cb + rs;
          const bool in = row >= item.row0 && row < item.row1;
          const int d0 = 4 * pp;
          float v0 = 0.f, v1 = 0.f, v2 = 0.f, v3 = 0.f;
          if (in) {
            const float4 x = *(const float4 *)(xs + rs * DIM + d0);
            v0 = (x.x - s_ctr[d0]) * s_scl[d0];
            v1 = (x.y - s_ctr[d0 + 1]) * s_scl[d0 + 1];
            v2 = (x.z - s_ctr[d0 + 2]) * s_scl[d0 + 2];
            v3 = (x.w - s_ctr[d0 + 3]) * s_scl[d0 + 3];
          }
          const int kr = rs & 7, kg = rs >> 3;
          uint32_t h0, l0, h1, l1;
          {
            split2<F16>(clamp_f16(v0), clamp_f16(v1), h0, l0);
            split2<F16>(clamp_f16(v2), clamp_f16(v3), h1, l1);
            const int f = d0;
            const uint32_t off = kg * (NB * 1024) + (f >> 6) * 1024 + mnmajor_sw128_off(kr, (f & 63) >> 3) + ((f >> 2) & 1) * 8;
            st_shared_v2(sb + off, h0, h1);
            st_shared_v2(sb + L::B_PART + off, l0, l1);
          }
          {
            split2<F16>(clamp_f16(v0 * v0), clamp_f16(v1 * v1), h0, l0);
            split2<F16>(clamp_f16(v2 * v2), clamp_f16(v3 * v3), h1, l1);
            const int f = DIM + d0;
            const uint32_t off = kg * (NB * 1024) + (f >> 6) * 1024 + mnmajor_sw128_off(kr, (f & 63) >> 3) + ((f >> 2) & 1) * 8;
            st_shared_v2(sb + off, h0, h1);
            st_shared_v2(sb + L::B_PART + off, l0, l1);
          }
          if (pp == 0) {  // ones column: counts the posterior mass of in-item rows
            const int f = 2 * DIM;
            const uint32_t off = kg * (NB * 1024) + (f >> 6) * 1024 + mnmajor_sw128_off(kr, (f & 63) >> 3);
            const uint16_t one = F16 ? (uint16_t)0x3C00 : (uint16_t)0x3F80;
            asm volatile("st.shared.u16 [%0], %1;" ::"r"(sb + off), "h"(in ? one : (uint16_t)0) : "memory");
          }
        }
        fence_proxy_async_smem();
        mbar_arrive(&full[stage]);
        ++it;
      }
    }
  } else if (warp < 8) {
    // ----------------------------------------------------- epilogue
    const int ew = warp - 4;
    int n = 0;
    for (int ii = ib; ii < ie; ++ii, ++n) {
      const SItem item = p.items[p.order[ii]];
      if (!mbar_wait(accf, n & 1, s_abort, p.err, 12)) break;
      tc_fence_after();
#pragma unroll 1
      for (int mt = 0; mt < MT; ++mt) {
        const int comp = comp0 + mt * 128 + ew * 32 + lane;
        float *dst = p.partial + ((size_t)item.slot * p.Kp + comp) * NST;
        const uint32_t tb = tmem + ((uint32_t)(ew * 32) << 16) + (uint32_t)(mt * NST);
#pragma unroll 1
        for (int cc = 0; cc < (NST + 31) / 32; ++cc) {
          uint32_t v[32];
          tmem_ld32(tb + cc * 32, v);
          tmem_wait_ld();
          if (comp < p.Kp) {
            if (cc * 32 + 32 <= NST) {
#pragma unroll
              for (int j = 0; j < 32; j += 4)
                *(float4 *)(dst + cc * 32 + j) = make_float4(__uint_as_float(v[j]), __uint_as_float(v[j + 1]),
                                                              __uint_as_float(v[j + 2]), __uint_as_float(v[j + 3]));
            } else {
#pragma unroll
              for (int j = 0; j < 32; ++j)
                if (cc * 32 + j < NST) dst[cc * 32 + j] = __uint_as_float(v[j]);
            }
          }
        }
      }
      tc_fence_before();
      mbar_arrive(acce);
    }
  } else if (warp == 8 && lane == 0) {
    // ---------------------------------------------------------- MMA
    int it = 0, n = 0;
    bool ok = true;
    for (int ii = ib; ii < ie && ok; ++ii, ++n) {
      const SItem item = p.items[p.order[ii]];
      if (!mbar_wait(acce, (n & 1) ^ 1, s_abort, p.err, 13)) break;
      tc_fence_after();
      int chunk = 0;
      for (i64 cb = p.qbase + ((item.row0 - p.qbase) & ~(i64)7); cb < item.row1; cb += 32, ++chunk) {
        const int stage = it % p.nst;
        if (!mbar_wait(&full[stage], (it / p.nst) & 1, s_abort, p.err, 14) ||
            !mbar_wait(&xfull[stage], (it / p.nst) & 1, s_abort, p.err, 16)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t sa = smem_u32(sS + (size_t)stage * L::kStage);
        const uint32_t sb = sa + NPA * L::A_PART;
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
#pragma unroll
          for (int mt = 0; mt < MT; ++mt) {
            // q^T: MN-major 64-byte-swizzled atoms, 32-component blocks 2 KB
            // apart (LBO), 8-row groups 512 B apart (SBO).
            const uint32_t a0 = sa + mt * 4 * 2048 + ks * 2 * 512;
            const uint64_t ah = sdesc(a0, 2048, 512, kSw64);
#pragma unroll
            for (int nc = 0; nc < L::NCH; ++nc) {
              const int nn = (NST - nc * 256) < 256 ? (NST - nc * 256) : 256;
              const uint32_t idesc = F16 ? idesc_f16(128, nn, true, true) : idesc_bf16(128, nn, true, true);
              const uint32_t b0 = sb + ks * 2 * (NB * 1024) + nc * 4 * 1024;
              const uint64_t bh = sdesc(b0, 1024, NB * 1024, kSw128);
              const uint64_t bl = sdesc(b0 + L::B_PART, 1024, NB * 1024, kSw128);
              const uint32_t d = tmem + (uint32_t)(mt * NST + nc * 256);
              mma_bf16(d, ah, bh, idesc, (chunk > 0 || ks > 0) ? 1u : 0u);
              mma_bf16(d, ah, bl, idesc, 1u);
              if (NPA == 2) mma_bf16(d, sdesc(a0 + L::A_PART, 2048, 512, kSw64), bh, idesc, 1u);
            }
          }
        }
        mma_commit(&empty[stage]);
        ++it;
      }
      if (ok) mma_commit(accf);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 8) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// ======================================================= finalize (FV)
// Per-component constants of the Fisher finalisation, computed once per call:
// mu' = mu - m, 1/sigma2, 1/sigma (K x D) and the prefactors 1/sqrt(pi),
// 1/sqrt(2 pi) (0 for components skipped by vl/fisher.c:436).
__global__ void k_tc_fv_consts(const float *__restrict__ means, const float *__restrict__ covs,
                               const float *__restrict__ priors, const float *__restrict__ ctr, int K,
                               int D, double *__restrict__ cmu, double *__restrict__ cis2,
                               double *__restrict__ cisd, double *__restrict__ cup,
                               double *__restrict__ cvp) {
  const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < (i64)K * D) {
    const int d = (int)(e % D);
    const double s2 = (double)covs[e];
    cmu[e] = (double)means[e] - (double)ctr[d];
    cis2[e] = 1.0 / s2;
    cisd[e] = 1.0 / sqrt(s2);
  }
  if (e < K) {
    const double pk = (double)priors[e];
    cup[e] = pk >= 1e-6 ? 1.0 / sqrt(pk) : 0.0;
    cvp[e] = pk >= 1e-6 ? 1.0 / sqrt(2.0 * pk) : 0.0;
  }
}

// Per image: reduce the item partials in double and form the Fisher vector
// (vl/fisher.c:419-485) from S0 = sum q, S1 = sum q x', S2 = sum q x'^2:
//   u = (S1 - mu' S0) / sigma,  v = (S2 - 2 mu' S1 + mu'^2 S0) / sigma2 - S0,
// scaled by 1/(N sqrt pi) and 1/(N sqrt(2 pi)); signed sqrt; L2.
// One cluster of kFinCluster CTAs per image: CTA r forms the outputs of
// components [r K/C, (r+1) K/C) in shared memory (2 (K/C) DIM floats), the
// CTAs exchange their partial L2 norms and term counts through distributed
// shared memory (summed in rank order on every CTA, so every CTA scales by
// the same bits), and each writes its normalised part once, coalesced.
constexpr int kFinThreads = 256;
constexpr int kFinCluster = 4;  // divides K (a multiple of 8 on this path)

// DIM: the dimension the statistics were taken in; Dr <= DIM: the model's own
// dimension (dimensions past it are zero padding, left out of the vector).
template <int DIM>
__global__ void __cluster_dims__(kFinCluster, 1, 1) __launch_bounds__(kFinThreads) k_tc_fv_finalize(
    int K, int Kp, int Dr, const float *__restrict__ partial, const int *__restrict__ imgSlot0,
    const i64 *__restrict__ imgRow0, const double *__restrict__ cmu, const double *__restrict__ cis2,
    const double *__restrict__ cisd, const double *__restrict__ cup, const double *__restrict__ cvp,
    const float *__restrict__ scale, const unsigned *__restrict__ rowcnt, i64 rowcntBase, int flags,
    i64 imgBase, float *__restrict__ enc, unsigned long long *__restrict__ nterms) {
  constexpr int NST = 2 * DIM + 16;
  constexpr int NW = kFinThreads / 32;
  extern __shared__ float s_fv[];  // 2 E: this CTA's u values, then its v values
  __shared__ double s_sq[NW];
  __shared__ unsigned long long s_nt[NW];
  __shared__ double s_is[DIM];  // 1 / scale_d (exact: scale_d is a power of two)
  __shared__ double s_part, s_tot;
  __shared__ unsigned long long s_partn;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int img = blockIdx.x / kFinCluster;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int Kc = K / kFinCluster, k0 = rank * Kc;
  const int E = Kc * Dr, KD = K * Dr, eBase = k0 * Dr;
  const int s0 = imgSlot0[img], s1 = imgSlot0[img + 1];
  const i64 r0 = imgRow0[img], r1 = imgRow0[img + 1];
  const i64 n = r1 - r0;
  const double in = n > 0 ? 1.0 / (double)n : 0.0;
  const size_t slotStride = (size_t)Kp * NST;
  for (int d = tid; d < DIM; d += kFinThreads) s_is[d] = scale ? 1.0 / (double)scale[d] : 1.0;
  const double iq = 1.0 / (double)kQScale;
  __syncthreads();
  // Element (component kl, dimension d) is el = kl Dr + d.  Warp w takes the
  // components w, w + NW, ...; lane l the dimensions l, l + 32, ... below Dr,
  // so no element index is divided and a component's S0 is one broadcast load.
  constexpr int DPL = (DIM + 31) / 32;
  double sq = 0;
#pragma unroll 2
  for (int kl = warp; kl < Kc; kl += NW) {
    const int k = k0 + kl;
    double S0 = 0, S1[DPL], S2[DPL];
#pragma unroll
    for (int j = 0; j < DPL; ++j) S1[j] = S2[j] = 0;
    const float *pp = partial + ((size_t)s0 * Kp + k) * NST;
    for (int s = s0; s < s1; ++s, pp += slotStride) {
      S0 += (double)pp[2 * DIM];
#pragma unroll
      for (int j = 0; j < DPL; ++j) {
        const int d = lane + 32 * j;
        if (d < Dr) {
          S1[j] += (double)pp[d];
          S2[j] += (double)pp[DIM + d];
        }
      }
    }
    // Statistics were taken on q 2^14 and x'' = x' * scale.
    S0 *= iq;
    const double cu = cup[k] * in, cv = cvp[k] * in;
#pragma unroll
    for (int j = 0; j < DPL; ++j) {
      const int d = lane + 32 * j;
      if (d >= Dr) continue;
      const int el = kl * Dr + d, e = eBase + el;
      const double is = s_is[d];
      const double s1 = S1[j] * (is * iq), s2 = S2[j] * (is * is * iq);
      const double mup = cmu[e];
      const double u = cisd[e] * (s1 - mup * S0) * cu;
      const double v = ((s2 - 2.0 * mup * s1 + mup * mup * S0) * cis2[e] - S0) * cv;
      float uf = (float)u, vf = (float)v;
      if (flags & 1) {
        uf = uf >= 0.f ? sqrtf(uf) : -sqrtf(-uf);
        vf = vf >= 0.f ? sqrtf(vf) : -sqrtf(-vf);
      }
      s_fv[el] = uf;
      s_fv[E + el] = vf;
      sq += (double)uf * uf + (double)vf * vf;
    }
  }
  // Term counts: the image's rows are split over the cluster's CTAs.
  unsigned long long nt = 0;
  if (rowcnt)
#pragma unroll 4
    for (i64 r = r0 + rank * kFinThreads + tid; r < r1; r += kFinThreads * kFinCluster)
      nt += rowcnt[r - rowcntBase];
  sq = warp_sum(sq);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) nt += __shfl_xor_sync(0xffffffffu, nt, o);
  if (lane == 0) {
    s_sq[warp] = sq;
    s_nt[warp] = nt;
  }
  __syncthreads();
  if (tid == 0) {
    double t = 0;
    unsigned long long c = 0;
    for (int w = 0; w < NW; ++w) {
      t += s_sq[w];
      c += s_nt[w];
    }
    s_part = t;
    s_partn = c;
  }
  cluster.sync();  // every CTA's partials are written
  if (tid == 0) {
    double t = 0;
    unsigned long long c = 0;
    for (int q = 0; q < kFinCluster; ++q) {
      t += *cluster.map_shared_rank(&s_part, q);
      c += *cluster.map_shared_rank(&s_partn, q);
    }
    s_tot = t;
    if (rank == 0 && nterms) nterms[imgBase + img] = c;
  }
  __syncthreads();
  float *out = enc + (imgBase + img) * 2 * (i64)KD + eBase;
  const bool nrmz = (flags & 2) != 0;
  float nf = 1.f;
  if (nrmz) {
    double nrm = sqrt(s_tot);
    if (nrm < 1e-12) nrm = 1e-12;
    nf = (float)nrm;
  }
  // Both halves in 16-byte pieces where E and the output allow it.
  if (E % 4 == 0 && (((uintptr_t)out | (uintptr_t)(out + KD)) & 15) == 0) {
    for (int el = 4 * tid; el < E; el += 4 * kFinThreads) {
      float4 a = *(const float4 *)(s_fv + el), b = *(const float4 *)(s_fv + E + el);
      if (nrmz) {
        a = make_float4(a.x / nf, a.y / nf, a.z / nf, a.w / nf);
        b = make_float4(b.x / nf, b.y / nf, b.z / nf, b.w / nf);
      }
      *(float4 *)(out + el) = a;
      *(float4 *)(out + KD + el) = b;
    }
  } else {
    for (int el = tid; el < E; el += kFinThreads) {
      out[el] = nrmz ? s_fv[el] / nf : s_fv[el];
      out[KD + el] = nrmz ? s_fv[E + el] / nf : s_fv[E + el];
    }
  }
  cluster.sync();  // the partials stay readable until every CTA has read them
}

// ============================================================ M-step
// M-step (vl/gmm.c:1169-1194) from the statistics of the tensor-core kernel:
// per item S0 = sum q, S1 = sum q x'', S2 = sum q x''^2 with x'' = (x - c)
// scale over the rows whose posterior passed the skip q >= 1e-2/K
// (vl/gmm.c:1099).  Items are summed in f64 in index order; the reference's
// sums follow exactly: sum q x = S1 + c S0, sum q (x - mu_old)^2 =
// S2 - 2 a S1 + a^2 S0 with a = mu_old - c.  Then the reference's update:
// mean, variance about the new mean, the variance floor, and the mass as
// the unnormalised prior.
// Sums of the item partials in f64, item order: S0[k] = sum q, S1[k][d] =
// sum q x'', S2[k][d] = sum q x''^2, with the q 2^14 and x'' = x' scale
// factors (powers of two, so exact) taken out.
__global__ void k_tc_mstep_sums(int nitems, int K, int Kp, int D, const float *__restrict__ partial,
                                const float *__restrict__ scale, double *__restrict__ S0,
                                double *__restrict__ S1, double *__restrict__ S2) {
  const i64 idx = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (i64)K * D) return;
  const int k = (int)(idx / D), d = (int)(idx % D);
  const int NST = 2 * D + 16;
  double s0 = 0, s1 = 0, s2 = 0;
  for (int it = 0; it < nitems; ++it) {
    const float *pp = partial + ((size_t)it * Kp + k) * NST;
    s0 += (double)pp[2 * D];
    s1 += (double)pp[d];
    s2 += (double)pp[D + d];
  }
  const double is = scale ? 1.0 / (double)scale[d] : 1.0, iq = 1.0 / (double)kQScale;
  if (d == 0) S0[k] = s0 * iq;
  S1[idx] = s1 * (is * iq);
  S2[idx] = s2 * (is * is * iq);
}

// The M-step from those sums: the reference's mean and variance about the
// new mean (sum q x = S1 + c S0, sum q (x - mu_old)^2 = S2 - 2 a S1 + a^2 S0
// with a = mu_old - c), the variance floor, the mass as the unnormalised prior.
__global__ void k_tc_mstep_apply(int K, int D, const double *__restrict__ S0, const double *__restrict__ S1,
                                 const double *__restrict__ S2, const float *__restrict__ ctr,
                                 const double *__restrict__ lb, float *__restrict__ means,
                                 float *__restrict__ covs, float *__restrict__ priors) {
  const i64 idx = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (i64)K * D) return;
  const int k = (int)(idx / D), d = (int)(idx % D);
  const double s0 = S0[k], s1 = S1[idx], s2 = S2[idx];
  const double c = (double)ctr[d], oldmu = (double)means[idx], a = oldmu - c;
  const double mass = s0;
  double mu = s1 + c * s0, v = s2 - 2.0 * a * s1 + a * a * s0;
  if (mass >= 1e-6 / (double)K) {
    mu /= mass;
    v /= mass;
    const double df = mu - oldmu;
    v -= df * df;
  }
  float vt = (float)v;
  if ((double)vt < lb[d]) vt = (float)lb[d];
  means[idx] = (float)mu;
  covs[idx] = vt;
  if (d == 0) priors[k] = (float)mass;
}

// Row-major fp32 posteriors -> fp16 q^T operand image, times 2^14 (the layout the
// E-step writes), with VLFeat's q < 1e-6 skip, the optional FAST one-hot of
// the row's arg-max (vl/fisher.c:398-417) and per-row term counts.  One warp
// per row; rows past n (tile padding) are written as zeros.
__global__ void k_rows_to_image16(const float *__restrict__ q, i64 n, int K, int Kq, float thr,
                                  __half *__restrict__ img, unsigned *__restrict__ rowcnt,
                                  i64 rowsPad, bool fast) {
  const i64 row = (i64)blockIdx.x * 8 + threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (row >= rowsPad) return;
  const bool valid = row < n;
  int am = 0;
  if (fast && valid) {
    float bv = -1.f;
    int bi = 0x7fffffff;
    for (int k = lane; k < K; k += 32) {
      const float v = q[row * K + k];
      if (v > bv || (v == bv && k < bi)) { bv = v; bi = k; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
    }
    am = bi;
  }
  unsigned cnt = 0;
  for (int g = lane; g < Kq / 8; g += 32) {
    float v[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      const int k = g * 8 + t;
      float x = (valid && k < K) ? q[row * K + k] : 0.f;
      if (fast) x = (valid && k == am) ? 1.f : 0.f;
      cnt += (x >= 1e-6f) ? 1u : 0u;
      v[t] = x < thr ? 0.f : x;
    }
    uint4 w;
    w.x = pack2<true>(v[0] * kQScale, v[1] * kQScale);
    w.y = pack2<true>(v[2] * kQScale, v[3] * kQScale);
    w.z = pack2<true>(v[4] * kQScale, v[5] * kQScale);
    w.w = pack2<true>(v[6] * kQScale, v[7] * kQScale);
    *(uint4 *)((uint8_t *)img + qimg_off(rowsPad / 8, row, (uint32_t)g)) = w;
  }
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if (lane == 0 && valid && rowcnt) rowcnt[row] = cnt;
}

// ============================================================ padding
// Dimensions the kernels are built for take the data as it is; any other
// dimension up to 128 runs zero-padded to the next of them: each row gets
// zero columns, each component mean 0 and variance 1 there, which adds 0 to
// every (x - mu)^2 / sigma^2 and to every sum of log sigma^2, so the
// posteriors and the Fisher statistics of the real dimensions are unchanged
// (the log-likelihood's D/2 log(2 pi) term is corrected for the padding).
__global__ void k_pad_rows(const float *__restrict__ X, i64 N, int D, int Dp, float *__restrict__ Xp) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N * Dp) return;
  const i64 r = i / Dp;
  const int d = (int)(i - r * Dp);
  Xp[i] = d < D ? X[r * D + d] : 0.f;
}
__global__ void k_pad_model(const float *__restrict__ means, const float *__restrict__ covs, int K, int D, int Dp,
                            float *__restrict__ mp, float *__restrict__ cp) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (i64)K * Dp) return;
  const i64 k = i / Dp;
  const int d = (int)(i - k * Dp);
  mp[i] = d < D ? means[k * D + d] : 0.f;
  cp[i] = d < D ? covs[k * D + d] : 1.f;
}

// ================================================================ host
struct TcPrep {
  int K = 0, Kp = 0, D = 0;
  float *ctr = nullptr, *cst2 = nullptr, *scale = nullptr, *wsc = nullptr, *wbar = nullptr;
  double *cbar = nullptr;
  __half *wimg = nullptr;
};

// Components of the tensor-core path, padded: a multiple of 32 up to 256; above
// that nb = ceil(K / 256) CTAs of a cluster take Kb components each (Kb a
// multiple of 32, at most 256) and K is padded to nb Kb.
int padK(i64 K) {
  const int k32 = (int)((K + 31) / 32 * 32);
  if (k32 <= 256) return k32;
  const int nb = (k32 + 255) / 256;
  const int kb = ((k32 + nb - 1) / nb + 31) / 32 * 32;
  return nb * kb;
}
int kblocks(int Kp) { return (Kp + 255) / 256; }

// Model-derived operands of the tensor-core path: the centre, the
// per-dimension scales, the fp16 W image with its scale, and the constants.
void tc_prepare(const DevModel<float> &m, TcPrep &tp, bool want_scale, Scratch &sc, cudaStream_t s) {
  (void)want_scale;  // the E-step's operands are always scaled
  tp.K = (int)m.K;
  tp.Kp = padK(m.K);
  tp.D = (int)m.D;
  const int KD2 = 2 * tp.D;
  tp.ctr = sc.slot[0].get<float>(256);
  tp.cst2 = sc.slot[1].get<float>(std::max(256, tp.Kp));
  tp.wimg = sc.slot[2].get<__half>((size_t)2 * tp.Kp * KD2);
  tp.scale = sc.slot[12].get<float>(256);
  float *wm = sc.slot[19].get<float>(2);
  tp.wsc = wm + 1;
  tp.wbar = sc.slot[20].get<float>(256);
  double *c64 = sc.slot[21].get<double>((size_t)std::max(256, tp.Kp) + 1);
  tp.cbar = c64 + std::max(256, tp.Kp);
  VLB_LAUNCH("tc_center", s, k_tc_center<<<(tp.D + 7) / 8, 256, 0, s>>>(m.means, tp.K, tp.D, tp.ctr));
  VLB_LAUNCH("tc_scale", s,
             k_tc_scale<<<(tp.D + 7) / 8, 256, 0, s>>>(m.means, m.covs, tp.ctr, tp.K, tp.D, tp.scale));
  VLB_LAUNCH("tc_wbar", s, k_tc_wbar<<<(tp.D + 7) / 8, 256, 0, s>>>(m.covs, tp.scale, tp.K, tp.D, tp.wbar));
  VLB_CUDA(cudaMemsetAsync(wm, 0, sizeof(float), s));
  const i64 nw = (i64)tp.K * KD2;
  VLB_LAUNCH("tc_wmax", s,
             k_tc_wmax<<<(unsigned)((nw + 255) / 256), 256, 0, s>>>(m.means, m.covs, tp.ctr, tp.scale, tp.wbar,
                                                                    tp.K, tp.D, wm));
  const i64 n = (i64)tp.Kp * KD2;
  VLB_LAUNCH("tc_wimage", s,
             k_tc_wimg<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(m.means, m.covs, tp.ctr, tp.scale, tp.wbar,
                                                                  wm, tp.K, tp.Kp, tp.D, tp.wimg, tp.wsc));
  VLB_LAUNCH("tc_constants", s,
             k_tc_cst<<<(tp.Kp + 7) / 8, 256, 0, s>>>(m.priors, m.means, m.covs, tp.ctr, tp.K,
                                                          tp.Kp, tp.D, c64));
  VLB_LAUNCH("tc_constants_center", s, k_tc_cst_center<<<1, 32, 0, s>>>(c64, tp.Kp, tp.cst2, tp.cbar));
}

int padQ(int Kp) { return (Kp + 127) / 128 * 128; }

// Smallest float >= t: the kernels keep q >= qthr (float compare), which then
// equals the reference's "skip p < t" with t a double constant.
float float_at_least(double t) {
  float f = (float)t;
  if ((double)f < t) f = std::nextafter(f, INFINITY);
  return f;
}

// Extra outputs of the combined formats: the image and its threshold.
struct EOut {
  void *qimg = nullptr;
  double qthr = 1e-6;  // vl/fisher.c:440 (the Fisher skip)
};

template <int DIM, int QF, bool SW, bool CL>
i64 launch_estep_impl(const float *X, i64 N, const TcPrep &tp, void *q, int ldq, bool fast,
                      unsigned *rowcnt, double *ll_part, int *err, int nst_req, cudaStream_t s,
                      const EOut &eo) {
  using L = ELayout<DIM, SW, CL>;
  const i64 ntiles = (N + 127) / 128;
  if (ntiles == 0) return 0;
  const int nb = CL ? kblocks(tp.Kp) : 1, Kb = tp.Kp / nb;
  VLB_CHECK(((uintptr_t)X & 15) == 0, VL_ERR_BAD_ARG, "tensor-core E-step: the data must start 16-byte aligned");
  // Row-major posteriors are stored 16 bytes at a time.
  VLB_CHECK(!q_rows(QF) || (((uintptr_t)q & 15) == 0 && ldq % 4 == 0), VL_ERR_BAD_ARG,
            "tensor-core E-step: the posteriors must start 16-byte aligned");
  // W streamed: 3 operand stages unless requested, beside a ring of up to 8
  // (at least 2) boxes of descriptor rows.  W resident: up to 8 stages.
  int nst, nxs = 0;
  if constexpr (SW) {
    nst = std::min(nst_req > 0 ? nst_req : 3, L::max_stages(Kb, 2));
    if (nst >= 2) nxs = std::min<int>(kMaxXs, (int)((kSmemLimit - L::bytes(Kb, nst)) / L::kXBox));
  } else {
    nst = std::min(nst_req > 0 ? nst_req : 8, L::max_stages(Kb));
  }
  VLB_CHECK(nst >= 2 && (!SW || nxs >= 2), VL_ERR_BAD_ARG, "tensor-core E-step: operands exceed shared memory");
  const size_t smem = L::bytes(Kb, nst, nxs);
  auto kern = k_tc_estep<DIM, QF, false, SW, CL>;
  if constexpr (!q_rows(QF) || QF == kQRow) {
    if (fast) kern = k_tc_estep<DIM, QF, true, SW, CL>;
  } else {
    VLB_CHECK(!fast, VL_ERR_BAD_ARG, "tensor-core E-step: the combined formats have no FAST variant");
  }
  VLB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  EParams p;
  p.X = X; p.N = N; p.K = tp.K; p.Kp = Kb; p.Kg = tp.Kp; p.Kq = padQ(tp.Kp); p.nst = nst; p.nxs = nxs;
  if constexpr (SW) {
    // Boxes of 16 dimensions (64 bytes, 16-byte aligned) x 128 rows; the row
    // coordinate is a 32-bit TMA coordinate.
    VLB_CHECK(ntiles * 128 <= (i64)INT32_MAX, VL_ERR_BAD_ARG, "tensor-core E-step: at most 2^31 - 128 rows per launch");
    tc::tma_map_2d(&p.xmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, X, N, DIM, 16, 128, CU_TENSOR_MAP_SWIZZLE_NONE);
  } else {
    std::memset(&p.xmap, 0, sizeof p.xmap);
  }
  p.qpart = ntiles * 128 * (i64)p.Kq * 2;
  p.wimg = (const uint4 *)tp.wimg; p.cst2 = tp.cst2; p.ctr = tp.ctr; p.scl = tp.scale; p.wsc = tp.wsc;
  p.wbar = tp.wbar; p.cbar = tp.cbar;
  p.q = q; p.qimg = eo.qimg; p.ldq = ldq; p.fast = fast ? 1 : 0; p.qthr = float_at_least(eo.qthr);
  p.rowcnt = rowcnt; p.ll_part = ll_part;
  p.err = err; p.ntiles = ntiles;
  if constexpr (!CL) {
    const int grid = (int)std::min<i64>(ntiles, num_sms());
    VLB_LAUNCH("tc_estep_f16x3", s, kern<<<grid, tc_threads(SW), smem, s>>>(p));
  } else {
    // One cluster of nb CTAs per tile, as many clusters as fit at once
    // (persistent: each cluster strides over the tiles).
    if (rowcnt) VLB_CUDA(cudaMemsetAsync(rowcnt, 0, sizeof(unsigned) * (size_t)N, s));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)nb;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(tc_threads(SW));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3((unsigned)(nb * std::max(1, num_sms() / nb)));
    int maxc = 0;
    VLB_CUDA(cudaOccupancyMaxActiveClusters(&maxc, kern, &cfg));
    VLB_CHECK(maxc >= 1, VL_ERR_BAD_ARG, "tensor-core E-step: the CTA cluster does not fit on the device");
    cfg.gridDim = dim3((unsigned)(nb * std::min<i64>(ntiles, maxc)));
    VLB_LAUNCH("tc_estep_f16x3", s, VLB_CUDA(cudaLaunchKernelEx(&cfg, kern, p)));
  }
  return ll_part ? ntiles * 8 : ntiles * 4;  // LL partials written: epilogue's, then the common parts
}

// Up to 256 components W is streamed through the operand stages (it costs
// L2 reads only) and the freed shared memory stages the descriptor rows by
// TMA.  Above 256 components the E-step runs as clusters of CTAs, with W
// resident when two operand stages fit beside it (else streamed).
template <int DIM, int QF>
i64 launch_estep(const float *X, i64 N, const TcPrep &tp, void *q, int ldq, bool fast,
                 unsigned *rowcnt, double *ll_part, int *err, int nst_req, cudaStream_t s,
                 const EOut &eo) {
  if (tp.Kp > 256) {
    const int Kb = tp.Kp / kblocks(tp.Kp);
    if constexpr (DIM == 128) {
      if (ELayout<DIM, false, true>::max_stages(Kb) < 2)
        return launch_estep_impl<DIM, QF, true, true>(X, N, tp, q, ldq, fast, rowcnt, ll_part, err, nst_req, s, eo);
    }
    return launch_estep_impl<DIM, QF, false, true>(X, N, tp, q, ldq, fast, rowcnt, ll_part, err, nst_req, s, eo);
  }
  return launch_estep_impl<DIM, QF, true, false>(X, N, tp, q, ldq, fast, rowcnt, ll_part, err, nst_req, s, eo);
}

template <int DIM, int MT, int SPLIT>
void launch_stats(const SParams &p0, int grid_x, int grid_y, int nst_req, cudaStream_t s) {
  using L = SLayout<DIM, MT, SPLIT>;
  SParams p = p0;
  p.nst = std::min(nst_req > 0 ? nst_req : 8, L::max_stages());
  VLB_CHECK(p.nst >= 2, VL_ERR_BAD_ARG, "tensor-core statistics: operands exceed shared memory");
  const size_t smem = L::bytes(p.nst);
  auto kern = k_tc_stats<DIM, MT, SPLIT>;
  VLB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  {
    // The image (parts of ngroups 8-row groups per 32-component block) for
    // boxes of 4 groups x this CTA's 4 MT blocks x all parts.
    const i64 ngroups = p.qpart / ((i64)p.Kq * 16);
    VLB_CHECK(ngroups <= (i64)INT32_MAX, VL_ERR_BAD_ARG, "tensor-core statistics: image too large for one launch");
    const unsigned long long dims[4] = {256, (unsigned long long)ngroups, (unsigned long long)(p.Kq / 32),
                                        (unsigned long long)L::NPA};
    const unsigned long long strides[3] = {512, (unsigned long long)ngroups * 512, (unsigned long long)p.qpart};
    const unsigned box[4] = {256, 4, 4 * MT, L::NPA};
    tc::tma_map(&p.qmap, CU_TENSOR_MAP_DATA_TYPE_UINT16, 4, p.qimg, dims, strides, box, CU_TENSOR_MAP_SWIZZLE_NONE);
  }
  VLB_LAUNCH(SPLIT == 2 ? "tc_stats_f16x3" : "tc_stats_f16x2", s,
             kern<<<dim3(grid_x, grid_y), kStatsThreads, smem, s>>>(p));
}

template <int DIM>
struct Tc {
  static constexpr bool kTwo = 2 * (2 * DIM + 16) <= 512;  // two M tiles fit in TMEM
  static i64 estep(int qf, const float *X, i64 N, const TcPrep &tp, void *q, int ldq, bool fast,
                   unsigned *rowcnt, double *ll, int *err, int nst, cudaStream_t s, const EOut &eo) {
    switch (qf) {
      case kQImg16: return launch_estep<DIM, kQImg16>(X, N, tp, q, ldq, fast, rowcnt, ll, err, nst, s, eo);
      case kQImg32: return launch_estep<DIM, kQImg32>(X, N, tp, q, ldq, fast, rowcnt, ll, err, nst, s, eo);
      case kQRowImg16: return launch_estep<DIM, kQRowImg16>(X, N, tp, q, ldq, fast, rowcnt, ll, err, nst, s, eo);
      case kQRowImg32: return launch_estep<DIM, kQRowImg32>(X, N, tp, q, ldq, fast, rowcnt, ll, err, nst, s, eo);
      default: return launch_estep<DIM, kQRow>(X, N, tp, q, ldq, fast, rowcnt, ll, err, nst, s, eo);
    }
  }
  // split 2: fp16x3 statistics (q image in two fp16 parts); split 1: one q part.
  // mt: 128-component M tiles per CTA (0: two when they fit in TMEM).
  static void stats(int split, const SParams &p, int grid_x, int mt, int nst, cudaStream_t s) {
    const int mtiles = p.Kq / 128;
    if (kTwo && mtiles % 2 == 0 && mt != 1) {
      if (split == 1) launch_stats<DIM, (kTwo ? 2 : 1), 1>(p, grid_x, mtiles / 2, nst, s);
      else launch_stats<DIM, (kTwo ? 2 : 1), 2>(p, grid_x, mtiles / 2, nst, s);
    } else {
      if (split == 1) launch_stats<DIM, 1, 1>(p, grid_x, mtiles, nst, s);
      else launch_stats<DIM, 1, 2>(p, grid_x, mtiles, nst, s);
    }
  }
};

i64 estep_dispatch(int D, int qf, const float *X, i64 N, const TcPrep &tp, void *q, int ldq, bool fast,
                   unsigned *rowcnt, double *ll, int *err, int nst, cudaStream_t s,
                   const EOut &eo = EOut()) {
  switch (D) {
    case 64: return Tc<64>::estep(qf, X, N, tp, q, ldq, fast, rowcnt, ll, err, nst, s, eo);
    case 80: return Tc<80>::estep(qf, X, N, tp, q, ldq, fast, rowcnt, ll, err, nst, s, eo);
    case 128: return Tc<128>::estep(qf, X, N, tp, q, ldq, fast, rowcnt, ll, err, nst, s, eo);
    default: throw Error(VL_ERR_BAD_ARG, "tensor-core path: unsupported dimension");
  }
}

void stats_dispatch(int D, int split, const SParams &p, int grid_x, int mt, int nst, cudaStream_t s) {
  switch (D) {
    case 64: Tc<64>::stats(split, p, grid_x, mt, nst, s); break;
    case 80: Tc<80>::stats(split, p, grid_x, mt, nst, s); break;
    case 128: Tc<128>::stats(split, p, grid_x, mt, nst, s); break;
    default: throw Error(VL_ERR_BAD_ARG, "tensor-core path: unsupported dimension");
  }
}

void check_err(int *derr, cudaStream_t s) {
  int h = 0;
  VLB_CUDA(cudaMemcpyAsync(&h, derr, sizeof(int), cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaStreamSynchronize(s));
  if (h) throw Error(VL_ERR_BAD_ARG, "tensor-core kernel gave up waiting (code " + std::to_string(h) + ")");
}

// Longest-processing-time assignment of work items to persistent CTAs:
// returns per-CTA item lists as (order, begin offsets).
void lpt_assign(const std::vector<SItem> &items, int gx, std::vector<int> &order, std::vector<int> &beg) {
  const int nitems = (int)items.size();
  std::vector<int> idx(nitems);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
    return items[a].row1 - items[a].row0 > items[b].row1 - items[b].row0;
  });
  std::vector<std::vector<int>> per(gx);
  std::vector<i64> load(gx, 0);
  for (int i : idx) {
    const int best = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    per[best].push_back(i);
    load[best] += items[i].row1 - items[i].row0;
  }
  order.clear();
  beg.assign(gx + 1, 0);
  for (int c = 0; c < gx; ++c) {
    beg[c] = (int)order.size();
    order.insert(order.end(), per[c].begin(), per[c].end());
  }
  beg[gx] = (int)order.size();
}

// Self-test of the bounded waits of the tcgen05 kernels (mbar_wait): one CTA,
// an mbarrier that nothing arrives on.  Thread 0 waits with `limit_ns`, gives
// up, records code 99 in *err and raises the abort flag, as any role of the
// kernels above does when its producer or consumer never comes; warp 1 waits
// on the same barrier with the kernels' own limit and leaves on the flag.
// Every wait is bounded, so the kernel returns in either case.
__global__ void k_wait_selftest(unsigned long long limit_ns, int *err) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_wait(&bar, 0, (volatile int *)&abort_flag, err, 99, limit_ns);
  else if (threadIdx.x == 32) mbar_wait(&bar, 0, (volatile int *)&abort_flag, err, 98);
  __syncthreads();
}

}  // namespace

void wait_selftest(double limit_ms, cudaStream_t s) {
  VLB_CHECK(limit_ms > 0 && limit_ms <= 1000, VL_ERR_BAD_ARG, "wait self-test: limit must be in (0, 1000] ms");
  Scratch &sc = thread_scratch(kArenaTc);
  int *err = sc.slot[3].get<int>(1);
  VLB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
  VLB_LAUNCH("wait_selftest", s, k_wait_selftest<<<1, 64, 0, s>>>((unsigned long long)(limit_ms * 1e6), err));
  check_err(err, s);
}

bool tc_supported(i64 K, i64 D) {
  if (!(D == 64 || D == 80 || D == 128)) return false;
  if (K < 8 || K > 2048 || K % 8) return false;
  // Per CTA: W streamed through two operand stages beside a ring of two boxes
  // of descriptor rows (up to 256 components), or, in clusters of up to 8
  // CTAs above 256, resident beside two stages (D=128: streamed); TMEM holds
  // two accumulators of the CTA's components.
  const int Kp = padK(K), nb = kblocks(Kp), Kb = Kp / nb;
  if (nb > 8) return false;
  if (nb == 1) {
    if (D == 128) return ELayout<128, true>::max_stages(Kb, 2) >= 2;
    return D == 64 ? ELayout<64, true>::max_stages(Kb, 2) >= 2 : ELayout<80, true>::max_stages(Kb, 2) >= 2;
  }
  if (D == 128) return ELayout<128, true, true>::max_stages(Kb, 2) >= 2;
  return D == 64 ? ELayout<64, false, true>::max_stages(Kb) >= 2 : ELayout<80, false, true>::max_stages(Kb) >= 2;
}

int tc_pad_dim(i64 D) { return D <= 64 ? 64 : D <= 80 ? 80 : D <= 128 ? 128 : 0; }

bool tc_supported_padded(i64 K, i64 D) { return tc_pad_dim(D) > 0 && tc_supported(K, tc_pad_dim(D)); }

bool tc_fv_supported_padded(i64 K, i64 D) {
  const int Dp = tc_pad_dim(D);
  return Dp > 0 && tc_supported(K, Dp) && K % kFinCluster == 0 &&
         sizeof(float) * 2 * (size_t)(K / kFinCluster) * D <= (size_t)kSmemLimit;
}

// Zero-padded copies of rows and model in `sc` (slots 22-24).
struct Padded {
  DevModel<float> m;
  const float *X = nullptr;
};
Padded pad_inputs(const float *X, i64 N, const DevModel<float> &m, Scratch &sc, cudaStream_t s) {
  Padded P;
  const int Dp = tc_pad_dim(m.D), D = (int)m.D;
  float *xp = sc.slot[22].get<float>((size_t)std::max<i64>(1, N) * Dp);
  float *mp = sc.slot[23].get<float>((size_t)m.K * Dp), *cp = sc.slot[24].get<float>((size_t)m.K * Dp);
  if (N > 0)
    VLB_LAUNCH("pad_rows", s, k_pad_rows<<<(unsigned)((N * Dp + 255) / 256), 256, 0, s>>>(X, N, D, Dp, xp));
  VLB_LAUNCH("pad_model", s,
             k_pad_model<<<(unsigned)((m.K * Dp + 255) / 256), 256, 0, s>>>(m.means, m.covs, (int)m.K, D, Dp, mp, cp));
  P.X = xp;
  P.m = m;
  P.m.means = mp;
  P.m.covs = cp;
  P.m.D = Dp;
  return P;
}

bool tc_fv_supported(i64 K, i64 D) {
  // The finalize keeps 2 (K / kFinCluster) D floats per CTA in shared memory.
  return tc_supported(K, D) && K % kFinCluster == 0 &&
         sizeof(float) * 2 * (size_t)(K / kFinCluster) * D <= (size_t)kSmemLimit;
}

i64 tc_estep(const float *X, i64 N, const DevModel<float> &m, float *q, double *ll_part, bool fast,
             int precision, cudaStream_t s, Scratch *arena) {
  (void)precision;
  Scratch &sc = arena ? *arena : thread_scratch(kArenaTc);
  if (!tc_supported(m.K, m.D)) {
    // Zero-padded dimension: the same posteriors; the log-likelihood's
    // -D/2 log(2 pi) per row was taken with the padded D, so one more
    // partial adds (Dp - D)/2 log(2 pi) for each row back.
    const Padded P = pad_inputs(X, N, m, sc, s);
    const i64 n = tc_estep(P.X, N, P.m, q, ll_part, fast, precision, s, &sc);
    if (!ll_part) return n;
    const double fix = 0.5 * (double)(P.m.D - m.D) * log(2.0 * 3.141592653589793) * (double)N;
    VLB_CUDA(cudaMemcpyAsync(ll_part + n, &fix, sizeof(double), cudaMemcpyHostToDevice, s));
    VLB_CUDA(cudaStreamSynchronize(s));
    return n + 1;
  }
  TcPrep tp;
  tc_prepare(m, tp, false, sc, s);
  int *err = sc.slot[3].get<int>(1);
  VLB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
  const i64 n = estep_dispatch(tp.D, kQRow, X, N, tp, (void *)q, (int)m.K, fast, nullptr, ll_part, err, 0, s);
  check_err(err, s);
  return n;
}

// ------------------------------------------------- EM, tensor-core M-step
// Host table -> a scratch buffer (stream-ordered; the host copy is staged).
template <typename T>
T *upload(DevBuf &b, const std::vector<T> &v, cudaStream_t s) {
  T *d = b.get<T>(std::max<size_t>(1, v.size()));
  if (!v.empty()) VLB_CUDA(cudaMemcpyAsync(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
  return d;
}

i64 tc_estep_em(const float *X, i64 N, const DevModel<float> &m, float *q, double *ll_part,
                int precision, cudaStream_t s) {
  Scratch &sc = thread_scratch(kArenaTc);
  const bool fp32 = (precision == VLB200_PREC_FP32);
  TcPrep tp;
  tc_prepare(m, tp, !fp32, sc, s);
  const int Kq = padQ(tp.Kp);
  const i64 ntiles = (N + 127) / 128;
  EOut eo;
  eo.qimg = sc.slot[4].get<char>((size_t)std::max<i64>(1, ntiles) * 128 * Kq * (fp32 ? 4 : 2));
  eo.qthr = 1e-2 / (double)m.K;  // vl/gmm.c:1099
  int *err = sc.slot[3].get<int>(1);
  VLB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
  const i64 n = estep_dispatch(tp.D, fp32 ? kQRowImg32 : kQRowImg16, X, N, tp, (void *)q, (int)m.K, false,
                               nullptr, ll_part, err, 0, s, eo);
  check_err(err, s);
  return n;
}

constexpr i64 kEmItemRows = 8192;  // rows per statistics work item in EM

void tc_mstep(const float *X, i64 N, float *means, float *covs, float *priors, i64 K, i64 D,
              const double *lb, int precision, cudaStream_t s) {
  Scratch &sc = thread_scratch(kArenaTc);
  const bool fp32 = (precision == VLB200_PREC_FP32);
  const int Kp = padK(K), Kq = padQ(Kp), NST = (int)(2 * D + 16);
  const i64 ntiles = (N + 127) / 128;
  constexpr i64 kItemRows = 8192;
  std::vector<SItem> items;
  for (i64 r = 0; r < N; r += kItemRows) items.push_back({r, std::min(N, r + kItemRows), (int)items.size(), 0});
  const int nitems = (int)items.size();
  const int gx = std::max(1, std::min(nitems, num_sms()));
  std::vector<int> order, beg;
  lpt_assign(items, gx, order, beg);
  SItem *ditems = upload(sc.slot[7], items, s);
  int *dorder = upload(sc.slot[8], order, s);
  int *dbeg = upload(sc.slot[9], beg, s);
  float *partial = sc.slot[6].get<float>((size_t)std::max(1, nitems) * Kp * NST);
  int *err = sc.slot[3].get<int>(1);
  VLB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
  if (nitems > 0) {
    SParams sp;
    sp.X = X; sp.qimg = (const uint8_t *)sc.slot[4].p; sp.qpart = ntiles * 128 * (i64)Kq * 2; sp.qbase = 0;
    sp.K = (int)K; sp.Kp = Kp; sp.Kq = Kq; sp.nst = 0;
    sp.ctr = (const float *)sc.slot[0].p; sp.scale = (const float *)sc.slot[12].p;
    sp.items = ditems; sp.order = dorder; sp.cta_beg = dbeg; sp.partial = partial; sp.err = err;
    stats_dispatch((int)D, fp32 ? 2 : 1, sp, gx, 0, 0, s);
  }
  tc_em_finalize(nitems, partial, means, covs, priors, K, D, lb, s);
  check_err(err, s);
}

// ------------------------------------------------- streaming EM pieces
// EM over data too large for resident N x K posteriors runs chunk by chunk:
// each chunk's q image lives in this arena's slot 4, its statistics go to
// the caller's item partials (items never straddle chunks), and one
// finalize reduces all items of the pass in f64, in item order.

void tc_em_image_from_rows(const float *qrows, i64 n, const DevModel<float> &m, cudaStream_t s) {
  Scratch &sc = thread_scratch(kArenaTc);
  TcPrep tp;
  tc_prepare(m, tp, true, sc, s);
  const int Kq = padQ(tp.Kp);
  const i64 ntiles = (n + 127) / 128, rowsPad = ntiles * 128;
  __half *img = sc.slot[4].get<__half>((size_t)std::max<i64>(1, ntiles) * 128 * Kq);
  if (rowsPad > 0)
    VLB_LAUNCH("tc_rows_to_image", s,
               k_rows_to_image16<<<(unsigned)((rowsPad + 7) / 8), 256, 0, s>>>(
                   qrows, n, (int)m.K, Kq, float_at_least(1e-2 / (double)m.K), img, nullptr, rowsPad, false));
}

i64 tc_em_items(i64 n) { return (n + kEmItemRows - 1) / kEmItemRows; }

void tc_em_stats(const float *X, i64 row0, i64 n, i64 K, i64 D, int split, float *partial, int item0,
                 cudaStream_t s) {
  if (n <= 0) return;
  Scratch &sc = thread_scratch(kArenaTc);
  const int Kp = padK(K), Kq = padQ(Kp);
  const i64 ntiles = (n + 127) / 128;
  std::vector<SItem> items;
  for (i64 r = 0; r < n; r += kEmItemRows)
    items.push_back({row0 + r, row0 + std::min(n, r + kEmItemRows), item0 + (int)items.size(), 0});
  const int nitems = (int)items.size();
  const int gx = std::max(1, std::min(nitems, num_sms()));
  std::vector<int> order, beg;
  lpt_assign(items, gx, order, beg);
  SItem *ditems = upload(sc.slot[7], items, s);
  int *dorder = upload(sc.slot[8], order, s);
  int *dbeg = upload(sc.slot[9], beg, s);
  int *err = sc.slot[3].get<int>(1);
  VLB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
  SParams sp;
  sp.X = X; sp.qimg = (const uint8_t *)sc.slot[4].p; sp.qpart = ntiles * 128 * (i64)Kq * 2; sp.qbase = row0;
  sp.K = (int)K; sp.Kp = Kp; sp.Kq = Kq; sp.nst = 0;
  sp.ctr = (const float *)sc.slot[0].p; sp.scale = (const float *)sc.slot[12].p;
  sp.items = ditems; sp.order = dorder; sp.cta_beg = dbeg; sp.partial = partial; sp.err = err;
  stats_dispatch((int)D, split, sp, gx, 0, 0, s);
  check_err(err, s);
}

void tc_em_sums(int nitems, const float *partial, i64 K, i64 D, double *S0, double *S1, double *S2,
                cudaStream_t s) {
  Scratch &sc = thread_scratch(kArenaTc);
  VLB_LAUNCH("tc_mstep_sums", s,
             k_tc_mstep_sums<<<(unsigned)((K * D + 255) / 256), 256, 0, s>>>(
                 nitems, (int)K, padK(K), (int)D, partial, (const float *)sc.slot[12].p, S0, S1, S2));
}

void tc_em_apply(const double *S0, const double *S1, const double *S2, float *means, float *covs, float *priors,
                 i64 K, i64 D, const double *lb, cudaStream_t s) {
  Scratch &sc = thread_scratch(kArenaTc);
  VLB_LAUNCH("tc_mstep_apply", s,
             k_tc_mstep_apply<<<(unsigned)((K * D + 255) / 256), 256, 0, s>>>(
                 (int)K, (int)D, S0, S1, S2, (const float *)sc.slot[0].p, lb, means, covs, priors));
  normalize_priors<float>(priors, K, s);
}

void tc_em_finalize(int nitems, const float *partial, float *means, float *covs, float *priors, i64 K, i64 D,
                    const double *lb, cudaStream_t s) {
  Scratch &sc = thread_scratch(kArenaTc);
  double *S = sc.slot[25].get<double>((size_t)(2 * D + 1) * K);
  tc_em_sums(nitems, partial, K, D, S, S + K, S + K + K * D, s);
  tc_em_apply(S, S + K, S + K + K * D, means, covs, priors, K, D, lb, s);
}

size_t tc_em_partial_floats(i64 K, i64 D) { return (size_t)padK(K) * (size_t)(2 * D + 16); }

// ------------------------------------------------- batched Fisher encoding
namespace {

// Host-side layout of one batch of images: chunks of whole images (one
// E-step launch each, at most rowBudget rows unless one image is larger),
// work items (runs of at most itemRows rows of one image; images without rows
// get none and encode to zeros) assigned to the persistent statistics CTAs by
// LPT, and the per-image slot and row tables of the finalize kernel.  The
// tables of all chunks are concatenated; each chunk records its offsets.
struct FvChunk {
  i64 img0 = 0, nimg = 0, row0 = 0, nrows = 0;
  int nitems = 0, gx = 1;
  size_t items = 0, beg = 0, img = 0;  // offsets into items/order, beg, slot0/row0
};

struct FvLayout {
  std::vector<FvChunk> chunks;
  std::vector<SItem> items;
  std::vector<int> order, beg, slot0;
  std::vector<i64> row0;
  i64 maxRows = 0, maxTiles = 0;
  int maxItems = 0;
};

i64 default_row_budget(int Kp, bool fp32) {
  const i64 qsz = fp32 ? 4 : 2;  // bytes per q element over the image parts
  return std::max<i64>(1 << 16, (i64)(4ull << 30) / (Kp * qsz));
}

void fv_layout(const i64 *off, i64 numImages, i64 rowBudget, i64 itemRows, int nsm, FvLayout &L) {
  L = FvLayout();
  i64 img = 0;
  while (img < numImages) {
    FvChunk c;
    c.img0 = img;
    c.row0 = off[img];
    while (img < numImages && (img == c.img0 || off[img + 1] - c.row0 <= rowBudget)) ++img;
    c.nimg = img - c.img0;
    c.nrows = off[img] - c.row0;
    c.items = L.items.size();
    c.img = L.slot0.size();
    std::vector<SItem> items;
    for (i64 j = 0; j < c.nimg; ++j) {
      const i64 a = off[c.img0 + j], b = off[c.img0 + j + 1];
      L.slot0.push_back((int)items.size());
      L.row0.push_back(a);
      for (i64 r = a; r < b; r += itemRows) items.push_back({r, std::min(b, r + itemRows), (int)items.size(), 0});
    }
    L.slot0.push_back((int)items.size());
    L.row0.push_back(off[img]);
    c.nitems = (int)items.size();
    c.gx = std::max(1, std::min(c.nitems, nsm));
    std::vector<int> order, beg;
    lpt_assign(items, c.gx, order, beg);
    c.beg = L.beg.size();
    L.items.insert(L.items.end(), items.begin(), items.end());
    L.order.insert(L.order.end(), order.begin(), order.end());
    L.beg.insert(L.beg.end(), beg.begin(), beg.end());
    L.maxRows = std::max(L.maxRows, c.nrows);
    L.maxTiles = std::max(L.maxTiles, (c.nrows + 127) / 128);
    L.maxItems = std::max(L.maxItems, c.nitems);
    L.chunks.push_back(c);
  }
}

// Scratch slots of the batched encoder (each encoder owns its arena):
// 0-2, 12 model prep; 3 error word; 4 q image; 5 row counts; 6 item
// partials; 7-11 layout tables; 13-17 Fisher constants; 18 router posteriors.

void fv_upload(const FvLayout &L, int Kp, int Kq, int NST, bool fp32, Scratch &sc, cudaStream_t s) {
  const size_t qsz = fp32 ? 4 : 2;
  sc.slot[4].get<char>((size_t)std::max<i64>(1, L.maxTiles) * 128 * Kq * qsz);
  sc.slot[5].get<unsigned>(std::max<i64>(1, L.maxRows));
  sc.slot[6].get<float>((size_t)std::max(1, L.maxItems) * Kp * NST);
  upload(sc.slot[7], L.items, s);
  upload(sc.slot[8], L.order, s);
  upload(sc.slot[9], L.beg, s);
  upload(sc.slot[10], L.slot0, s);
  upload(sc.slot[11], L.row0, s);
}

// Called with a chunk's index before its launches and after its finalize.
using ChunkHook = std::function<void(size_t)>;

// All launches of one batched encode; no host copies, no synchronisation and,
// once the scratch is sized by fv_upload and one earlier run, no allocation.
// m: the model the kernels run on; mreal (or null): the caller's model when m
// is its zero-padded copy (tc_pad_dim), whose dimension the vectors take.
void fv_run(const FvLayout &L, Scratch &sc, const float *X, const DevModel<float> &m, float *enc,
            unsigned long long *nterms, int flags, int precision, const TcFvConfig &cfg, cudaStream_t s,
            const ChunkHook &before = nullptr, const ChunkHook &after = nullptr,
            const DevModel<float> *mreal = nullptr) {
  const bool fp32 = (precision == VLB200_PREC_FP32);
  TcPrep tp;
  tc_prepare(m, tp, !fp32, sc, s);
  const int qf = fp32 ? kQImg32 : kQImg16;
  const int split = fp32 ? 2 : 1;
  const int Kq = padQ(tp.Kp);
  const i64 K = m.K, D = m.D;
  int *err = sc.slot[3].get<int>(1);
  VLB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
  double *cmu = sc.slot[13].get<double>(K * D), *cis2 = sc.slot[14].get<double>(K * D);
  double *cisd = sc.slot[15].get<double>(K * D), *cup = sc.slot[16].get<double>(K);
  double *cvp = sc.slot[17].get<double>(K);
  const DevModel<float> &mr = mreal ? *mreal : m;
  const i64 Dr = mr.D;
  VLB_LAUNCH("tc_fv_consts", s,
             k_tc_fv_consts<<<(unsigned)((K * Dr + 255) / 256), 256, 0, s>>>(
                 mr.means, mr.covs, mr.priors, tp.ctr, (int)K, (int)Dr, cmu, cis2, cisd, cup, cvp));
  void *q = sc.slot[4].p;
  unsigned *rowcnt = (unsigned *)sc.slot[5].p;
  float *partial = (float *)sc.slot[6].p;
  const SItem *ditems = (const SItem *)sc.slot[7].p;
  const int *dorder = (const int *)sc.slot[8].p, *dbeg = (const int *)sc.slot[9].p;
  const int *dslot0 = (const int *)sc.slot[10].p;
  const i64 *drow0 = (const i64 *)sc.slot[11].p;
  auto fin = D == 64 ? k_tc_fv_finalize<64> : D == 80 ? k_tc_fv_finalize<80> : k_tc_fv_finalize<128>;
  const size_t finSmem = sizeof(float) * 2 * (K / kFinCluster) * Dr;
  VLB_CUDA(cudaFuncSetAttribute(fin, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)finSmem));
  for (size_t ci = 0; ci < L.chunks.size(); ++ci) {
    const FvChunk &c = L.chunks[ci];
    if (before) before(ci);
    const i64 ntiles = (c.nrows + 127) / 128;
    if (c.nrows > 0) {
      if (precision == VLB200_PREC_BF16_ROUTER) {
        // Router posteriors (row-major) -> fp16 operand image + row counts.
        float *qrows = sc.slot[18].get<float>((size_t)L.maxRows * K);
        router_default_posteriors(X + c.row0 * D, c.nrows, m, qrows, s);
        const i64 rowsPad = ntiles * 128;
        VLB_LAUNCH("tc_rows_to_image", s,
                   k_rows_to_image16<<<(unsigned)((rowsPad + 7) / 8), 256, 0, s>>>(
                       qrows, c.nrows, (int)K, Kq, 1e-6f, (__half *)q, rowcnt, rowsPad, (flags & 4) != 0));
      } else {
        estep_dispatch(tp.D, qf, X + c.row0 * D, c.nrows, tp, q, (int)K, (flags & 4) != 0, rowcnt, nullptr,
                       err, cfg.estepStages, s);
      }
      SParams sp;
      sp.X = X; sp.qimg = (const uint8_t *)q; sp.qpart = ntiles * 128 * (i64)Kq * 2; sp.qbase = c.row0;
      sp.K = (int)K; sp.Kp = tp.Kp; sp.Kq = Kq; sp.nst = 0;
      sp.ctr = tp.ctr; sp.scale = tp.scale;
      sp.items = ditems + c.items; sp.order = dorder + c.items; sp.cta_beg = dbeg + c.beg;
      sp.partial = partial; sp.err = err;
      stats_dispatch(tp.D, split, sp, c.gx, cfg.statsMT, cfg.statsStages, s);
    }
    VLB_LAUNCH("tc_fv_finalize", s,
               fin<<<(unsigned)(c.nimg * kFinCluster), kFinThreads, finSmem, s>>>(
                   (int)K, tp.Kp, (int)Dr, partial, dslot0 + c.img, drow0 + c.img, cmu, cis2, cisd, cup, cvp,
                   tp.scale, c.nrows > 0 ? rowcnt : nullptr, c.row0, flags, c.img0, enc,
                   nterms));
    if (after) after(ci);
  }
}

}  // namespace

void tc_fisher_batch(const float *X, const i64 *h_offsets, i64 numImages, const DevModel<float> &m,
                     float *enc, unsigned long long *nterms, int flags, int precision, cudaStream_t s) {
  Scratch &sc = thread_scratch(kArenaTc);
  const bool fp32 = (precision == VLB200_PREC_FP32);
  const int Kp = padK(m.K);
  TcFvConfig cfg;
  FvLayout L;
  fv_layout(h_offsets, numImages, default_row_budget(Kp, fp32), cfg.itemRows, num_sms(), L);
  if (!tc_fv_supported(m.K, m.D)) {
    const i64 N = h_offsets[numImages] - h_offsets[0];
    const Padded P = pad_inputs(X + h_offsets[0] * m.D, N, m, sc, s);
    std::vector<i64> offs(h_offsets, h_offsets + numImages + 1);
    for (auto &o : offs) o -= h_offsets[0];
    fv_layout(offs.data(), numImages, default_row_budget(Kp, fp32), cfg.itemRows, num_sms(), L);
    fv_upload(L, Kp, padQ(Kp), (int)(2 * P.m.D + 16), fp32, sc, s);
    fv_run(L, sc, P.X, P.m, enc, nterms, flags, precision, cfg, s, nullptr, nullptr, &m);
    check_err((int *)sc.slot[3].p, s);
    return;
  }
  fv_upload(L, Kp, padQ(Kp), (int)(2 * m.D + 16), fp32, sc, s);
  fv_run(L, sc, X, m, enc, nterms, flags, precision, cfg, s);
  check_err((int *)sc.slot[3].p, s);
}

// A batch encoder bound to one batch layout: it owns its scratch arena and
// device tables, so that run() only launches kernels and can be captured.
struct TcFvPlan {
  i64 D = 0, K = 0, numImages = 0;
  int flags = 0, precision = 0, Kp = 0;
  std::vector<i64> offsets;
  TcFvConfig cfg;
  FvLayout layout;
  Scratch sc;
  // Host-buffer execution: a layout of about kPipeChunks chunks whose
  // host -> device copies, encodes and device -> host copies overlap.
  static constexpr int kPipeChunks = 16;
  bool pipeBuilt = false;
  FvLayout pipe;
  Scratch scPipe;
  DevBuf xdev, encdev, ntdev;
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaEvent_t evStart = nullptr, evEnd = nullptr;
  std::vector<cudaEvent_t> evIn, evOut;

  void drop_pipe() {
    for (cudaEvent_t e : evIn) cudaEventDestroy(e);
    for (cudaEvent_t e : evOut) cudaEventDestroy(e);
    evIn.clear();
    evOut.clear();
    pipeBuilt = false;
  }
  ~TcFvPlan() {
    cudaDeviceSynchronize();
    drop_pipe();
    if (evStart) cudaEventDestroy(evStart);
    if (evEnd) cudaEventDestroy(evEnd);
    if (h2d) cudaStreamDestroy(h2d);
    if (d2h) cudaStreamDestroy(d2h);
  }
};

namespace {
void plan_build(TcFvPlan &p, cudaStream_t s) {
  const bool fp32 = (p.precision == VLB200_PREC_FP32);
  const i64 budget = p.cfg.rowBudget > 0 ? p.cfg.rowBudget : default_row_budget(p.Kp, fp32);
  fv_layout(p.offsets.data(), p.numImages, budget, p.cfg.itemRows, num_sms(), p.layout);
  fv_upload(p.layout, p.Kp, padQ(p.Kp), (int)(2 * p.D + 16), fp32, p.sc, s);
  VLB_CUDA(cudaStreamSynchronize(s));
}
}  // namespace

TcFvPlan *tc_fv_plan_new(i64 D, i64 K, const i64 *offsets, i64 numImages, int flags, int precision,
                         cudaStream_t s) {
  VLB_CHECK(tc_fv_supported(K, D), VL_ERR_BAD_ARG, "batched Fisher plan: unsupported (numClusters, dimension)");
  VLB_CHECK(precision == VLB200_PREC_FP32 || precision == VLB200_PREC_BF16 ||
                precision == VLB200_PREC_BF16_ROUTER,
            VL_ERR_BAD_ARG, "batched Fisher plan: precision must be FP32, BF16 or BF16_ROUTER");
  VLB_CHECK(numImages >= 0 && offsets != nullptr, VL_ERR_BAD_ARG, "batched Fisher plan: bad offsets");
  for (i64 j = 0; j < numImages; ++j)
    VLB_CHECK(offsets[j + 1] >= offsets[j], VL_ERR_BAD_ARG, "batched Fisher plan: offsets must not decrease");
  auto p = std::make_unique<TcFvPlan>();
  p->D = D; p->K = K; p->numImages = numImages; p->flags = flags; p->precision = precision;
  p->Kp = padK(K);
  p->offsets.assign(offsets, offsets + numImages + 1);
  plan_build(*p, s);
  return p.release();
}

void tc_fv_plan_delete(TcFvPlan *p) { delete p; }

TcFvConfig tc_fv_plan_config(const TcFvPlan *p) { return p->cfg; }

void tc_fv_plan_set_config(TcFvPlan *p, const TcFvConfig &c, cudaStream_t s) {
  VLB_CHECK(c.itemRows >= 128 && c.itemRows % 128 == 0, VL_ERR_BAD_ARG, "plan config: itemRows must be a positive multiple of 128");
  VLB_CHECK(c.statsMT >= 0 && c.statsMT <= 2, VL_ERR_BAD_ARG, "plan config: statsMT must be 0, 1 or 2");
  VLB_CHECK(c.statsStages >= 0 && c.estepStages >= 0 && c.rowBudget >= 0, VL_ERR_BAD_ARG, "plan config: negative value");
  VLB_CHECK(c.statsStages != 1 && c.estepStages != 1, VL_ERR_BAD_ARG, "plan config: at least two operand stages");
  VLB_CUDA(cudaStreamSynchronize(s));  // earlier runs may still read the tables
  p->cfg = c;
  p->drop_pipe();
  plan_build(*p, s);
}

void tc_fv_plan_run(TcFvPlan *p, const DevModel<float> &m, const float *X, float *enc,
                    unsigned long long *nterms, cudaStream_t s) {
  VLB_CHECK(m.K == p->K && m.D == p->D, VL_ERR_BAD_ARG, "batched Fisher plan: model shape differs from the plan");
  fv_run(p->layout, p->sc, X, m, enc, nterms, p->flags, p->precision, p->cfg, s);
}

// Host buffers in and out: the chunks' host -> device copies (stream h2d),
// encodes (stream s) and device -> host copies (stream d2h) overlap, ordered
// by per-chunk events.  Overlap needs page-locked host buffers; the call
// returns when the encodings are on the host.
void tc_fv_plan_run_host(TcFvPlan *p, const DevModel<float> &m, const float *Xh, float *ench,
                         unsigned long long *nth, cudaStream_t s) {
  VLB_CHECK(m.K == p->K && m.D == p->D, VL_ERR_BAD_ARG, "batched Fisher plan: model shape differs from the plan");
  const bool fp32 = (p->precision == VLB200_PREC_FP32);
  const i64 row0 = p->offsets.front(), total = p->offsets.back() - row0;
  const i64 D = p->D, FV = 2 * p->K * p->D;
  if (!p->pipeBuilt) {
    const i64 budget = std::max<i64>(1, (total + TcFvPlan::kPipeChunks - 1) / TcFvPlan::kPipeChunks);
    fv_layout(p->offsets.data(), p->numImages, budget, p->cfg.itemRows, num_sms(), p->pipe);
    fv_upload(p->pipe, p->Kp, padQ(p->Kp), (int)(2 * p->D + 16), fp32, p->scPipe, s);
    if (!p->h2d) VLB_CUDA(cudaStreamCreateWithFlags(&p->h2d, cudaStreamNonBlocking));
    if (!p->d2h) VLB_CUDA(cudaStreamCreateWithFlags(&p->d2h, cudaStreamNonBlocking));
    if (!p->evStart) VLB_CUDA(cudaEventCreateWithFlags(&p->evStart, cudaEventDisableTiming));
    if (!p->evEnd) VLB_CUDA(cudaEventCreateWithFlags(&p->evEnd, cudaEventDisableTiming));
    p->evIn.resize(p->pipe.chunks.size(), nullptr);
    p->evOut.resize(p->pipe.chunks.size(), nullptr);
    for (auto *v : {&p->evIn, &p->evOut})
      for (cudaEvent_t &e : *v) VLB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    VLB_CUDA(cudaStreamSynchronize(s));
    p->pipeBuilt = true;
  }
  // Device images of the batch: rows row0.. of X, all images of enc.
  float *Xd = p->xdev.get<float>((size_t)std::max<i64>(1, total) * D) - row0 * D;
  float *encd = p->encdev.get<float>((size_t)std::max<i64>(1, p->numImages) * FV);
  unsigned long long *ntd = p->ntdev.get<unsigned long long>(std::max<i64>(1, p->numImages));
  // This call's copies start after the work already queued on s (an earlier
  // call's encode still reading these device buffers).
  VLB_CUDA(cudaEventRecord(p->evStart, s));
  VLB_CUDA(cudaStreamWaitEvent(p->h2d, p->evStart, 0));
  VLB_CUDA(cudaStreamWaitEvent(p->d2h, p->evStart, 0));
  const std::vector<FvChunk> &ch = p->pipe.chunks;
  for (size_t ci = 0; ci < ch.size(); ++ci) {
    if (ch[ci].nrows > 0)
      VLB_CUDA(cudaMemcpyAsync(Xd + ch[ci].row0 * D, Xh + (ch[ci].row0 - row0) * D,
                               sizeof(float) * ch[ci].nrows * D, cudaMemcpyHostToDevice, p->h2d));
    VLB_CUDA(cudaEventRecord(p->evIn[ci], p->h2d));
  }
  fv_run(p->pipe, p->scPipe, Xd, m, encd, ntd, p->flags, p->precision, p->cfg, s,
         [&](size_t ci) { VLB_CUDA(cudaStreamWaitEvent(s, p->evIn[ci], 0)); },
         [&](size_t ci) {
           const FvChunk &c = ch[ci];
           VLB_CUDA(cudaEventRecord(p->evOut[ci], s));
           VLB_CUDA(cudaStreamWaitEvent(p->d2h, p->evOut[ci], 0));
           VLB_CUDA(cudaMemcpyAsync(ench + c.img0 * FV, encd + c.img0 * FV, sizeof(float) * c.nimg * FV,
                                    cudaMemcpyDeviceToHost, p->d2h));
           if (nth)
             VLB_CUDA(cudaMemcpyAsync(nth + c.img0, ntd + c.img0, sizeof(unsigned long long) * c.nimg,
                                      cudaMemcpyDeviceToHost, p->d2h));
         });
  VLB_CUDA(cudaEventRecord(p->evEnd, p->d2h));
  VLB_CUDA(cudaStreamWaitEvent(s, p->evEnd, 0));
  VLB_CUDA(cudaStreamSynchronize(s));
  VLB_CHECK(tc_fv_plan_error(p, s) == 0, VL_ERR_BAD_ARG, "tensor-core kernel gave up waiting");
}

int tc_fv_plan_error(TcFvPlan *p, cudaStream_t s) {
  int h[2] = {0, 0};
  if (p->sc.slot[3].p)
    VLB_CUDA(cudaMemcpyAsync(&h[0], p->sc.slot[3].p, sizeof(int), cudaMemcpyDeviceToHost, s));
  if (p->scPipe.slot[3].p)
    VLB_CUDA(cudaMemcpyAsync(&h[1], p->scPipe.slot[3].p, sizeof(int), cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaStreamSynchronize(s));
  return h[0] ? h[0] : h[1];
}

// Times each candidate configuration on the plan's own batch (one warm-up
// run, then the median of three runs timed with CUDA events on the stream)
// and keeps the fastest.  Candidates: statistics item rows, statistics
// M tiles per CTA, operand stages of both kernels and the chunk row budget.
TcFvConfig tc_fv_plan_autotune(TcFvPlan *p, const DevModel<float> &m, const float *X, float *enc,
                               unsigned long long *nterms, cudaStream_t s, double *best_ms) {
  const bool fp32 = (p->precision == VLB200_PREC_FP32);
  const i64 total = p->offsets.back() - p->offsets.front();
  std::vector<TcFvConfig> cands;
  const i64 whole = std::max<i64>(total, 1);
  const i64 qsz = fp32 ? 4 : 2;
  // A single chunk when its q image fits in 16 GB; else the default budget.
  const i64 big = std::min<i64>(whole, (i64)(16ull << 30) / (p->Kp * qsz));
  for (int itemRows : {4096, 8192, 16384})
    for (int mt : {0, 1})
      for (int est : {0, 2})
        for (i64 budget : {(i64)0, big}) {
          TcFvConfig c;
          c.itemRows = itemRows; c.statsMT = mt; c.estepStages = est; c.rowBudget = budget;
          cands.push_back(c);
        }
  cudaEvent_t e0, e1;
  VLB_CUDA(cudaEventCreate(&e0));
  VLB_CUDA(cudaEventCreate(&e1));
  TcFvConfig best = p->cfg;
  double bms = 1e300;
  try {
    for (const TcFvConfig &c : cands) {
      tc_fv_plan_set_config(p, c, s);
      tc_fv_plan_run(p, m, X, enc, nterms, s);  // warm-up (sizes every buffer)
      float t[3];
      for (float &ti : t) {
        VLB_CUDA(cudaEventRecord(e0, s));
        tc_fv_plan_run(p, m, X, enc, nterms, s);
        VLB_CUDA(cudaEventRecord(e1, s));
        VLB_CUDA(cudaEventSynchronize(e1));
        VLB_CUDA(cudaEventElapsedTime(&ti, e0, e1));
      }
      std::sort(t, t + 3);
      VLB_CHECK(tc_fv_plan_error(p, s) == 0, VL_ERR_BAD_ARG, "autotune: a candidate kernel gave up waiting");
      if (t[1] < bms) {
        bms = t[1];
        best = c;
      }
    }
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  tc_fv_plan_set_config(p, best, s);
  if (best_ms) *best_ms = bms;
  return best;
}

}  // namespace vlb
