// The recognition app's descriptor prologue on the GPU.
//
// Encoding (apps/recognition/encodeImage.m:91-103): for each descriptor x of
// an image,
//   y = P (x - c)                                 (P: m x D0, c: D0)
//   y = y * (1 / max(1e-12, |y|_2))               (if renormalise)
//   y = [y; (fx - w/2) / w; (fy - h/2) / h]       ('xy' geometric extension,
//                                                  extendDescriptorsWithGeometry.m:19-21)
// with (fx, fy) the descriptor's frame position and (w, h) its image's size.
// Learning (apps/recognition/trainEncoder.m:150-171): c = mean of the sample,
// C = (X - c)^T (X - c) / N, eigenvectors sorted by decreasing eigenvalue,
// d += whiteningRegul * max(d), P = rows of the first m eigenvectors, scaled by
// 1/sqrt(d) when whitening.
//
// The projection runs in fp32 (fused multiply-adds in ascending input
// dimension); mean and covariance are accumulated in fp64 with fixed-order
// reductions; the symmetric eigenproblem (D0 <= 128) is solved on the host by
// cyclic Jacobi rotations in fp64.
#include <algorithm>
#include <cmath>
#include <vector>

#include "engine.h"
#include "tc_common.cuh"

extern "C" {
#include "vlb200.h"
}

namespace vlb {
namespace {

int sm_count() {
  int dev = 0, n = 0;
  VLB_CUDA(cudaGetDevice(&dev));
  VLB_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  return n;
}

constexpr int kPcaRows = 128;  // descriptors per tile
constexpr int kPcaMaxIn = 128, kPcaMaxOut = 128;

// Shared-memory strides (floats): the tile xs[row][ldx] and P^T pt[d][ldp] are
// read as float4; ldx = din rounded up to 4, plus 4, so that the rows one
// thread reads (16 apart) fall on distinct banks.
__host__ __device__ inline int pca_ldx(int din) { return (din + 3) / 4 * 4 + 4; }
__host__ __device__ inline int pca_ldp(int dout) { return (dout + 15) / 16 * 16 + 4; }  // 8 NC + 4

struct PcaParams {
  float *out;
  int ldo, din, dout, renorm;
  i64 N, nimg;
  const float *X, *P, *c, *frames, *sizes;
  const i64 *offs;
  int *err;
};

// Persistent CTAs over tiles of 128 descriptors, 16 x NC threads, two CTAs
// per SM (one loads or finishes a tile while the other multiplies).  Thread
// (rg, cg) forms descriptors rg + 16a (a < 8) x outputs 8 cg .. 8 cg + 7 with
// fp32 fused multiply-adds in ascending input dimension: per 4 dimensions, 8
// float4 loads of the centred tile and 8 of P^T feed 256 FMAs.  BULK (rows of
// 16-byte multiples): thread 0 copies the tile's rows into shared memory with
// bulk asynchronous copies on an mbarrier; otherwise the warps load it.  Then
// the tile is centred in place, the products formed, the outputs staged in
// the same buffer, and a warp per descriptor renormalises, appends the
// geometric extension and stores the row.
template <int NC, bool BULK>  // NC: output groups of 8, even
__global__ void __launch_bounds__(16 * NC, 2) k_pca_project(const PcaParams p) {
  static_assert(NC % 2 == 0, "whole warps only");
  constexpr int kThreads = 16 * NC, kWarps = kThreads / 32;
  extern __shared__ __align__(128) unsigned char pca_raw[];
  uint64_t *full = (uint64_t *)pca_raw;
  volatile int *s_abort = (volatile int *)(full + 1);
  const int din = p.din, dout = p.dout;
  const int ldx = pca_ldx(din), ldp = pca_ldp(dout), ldy = dout + 1;
  const int dinp = (din + 3) / 4 * 4;
  float *pt = (float *)(pca_raw + 128);  // [dinp][ldp], zero past din and dout
  float *sc = pt + dinp * ldp;           // the centre, [ldx], zero past din
  float *xs = sc + ldx;                  // [128][ldx]; then the outputs [128][ldy]
  float *ys = xs;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const i64 ntiles = (p.N + kPcaRows - 1) / kPcaRows;
  if (tid == 0) {
    tc::mbar_init(full, 1);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int d = 0; d < dinp; ++d)
    for (int j = tid; j < ldp; j += kThreads) pt[d * ldp + j] = (j < dout && d < din) ? p.P[(i64)j * din + d] : 0.f;
  for (int d = tid; d < ldx; d += kThreads) sc[d] = d < din ? p.c[d] : 0.f;
  __syncthreads();
  const int rg = tid % 16, cg = tid / 16;
  int k = 0;
  for (i64 t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
    const i64 r0 = t * kPcaRows;
    const int nr = (int)(p.N - r0 < kPcaRows ? p.N - r0 : kPcaRows);
    if (BULK) {
      if (tid == 0) {
        tc::fence_proxy_async_smem();  // the previous tile's generic writes precede the copy's
        tc::mbar_arrive_expect_tx(full, (uint32_t)(nr * din * 4));
        for (int r = 0; r < nr; ++r)
          tc::bulk_g2s(tc::smem_u32(xs + r * ldx), p.X + (r0 + r) * din, (uint32_t)(din * 4), full);
      }
      const bool ok = tc::mbar_wait(full, (uint32_t)(k & 1), s_abort, p.err, 1);
      if (!__syncthreads_and(ok)) break;
    } else {
      for (int r = warp; r < nr; r += kWarps)
        for (int d = lane; d < din; d += 32) xs[r * ldx + d] = p.X[(r0 + r) * din + d];
      __syncthreads();
    }
    // Centre in place; rows past N and the row padding become zeros.
    for (int r = warp; r < kPcaRows; r += kWarps)
      for (int d = lane; d < ldx; d += 32)
        xs[r * ldx + d] = (r < nr && d < din) ? __fsub_rn(xs[r * ldx + d], sc[d]) : 0.f;
    __syncthreads();
    float acc[8][8];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
      for (int b = 0; b < 8; ++b) acc[a][b] = 0.f;
#pragma unroll 2
    for (int d = 0; d < din; d += 4) {
      float4 xv[8];
#pragma unroll
      for (int a = 0; a < 8; ++a) xv[a] = *(const float4 *)(xs + (rg + 16 * a) * ldx + d);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float4 p0 = *(const float4 *)(pt + (d + q) * ldp + 8 * cg);
        const float4 p1 = *(const float4 *)(pt + (d + q) * ldp + 8 * cg + 4);
        const float pv[8] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
#pragma unroll
        for (int a = 0; a < 8; ++a) {
          const float x = q == 0 ? xv[a].x : q == 1 ? xv[a].y : q == 2 ? xv[a].z : xv[a].w;
#pragma unroll
          for (int b = 0; b < 8; ++b) acc[a][b] = __fmaf_rn(pv[b], x, acc[a][b]);
        }
      }
    }
    __syncthreads();  // every thread is done with the tile: stage outputs there
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        const int j = 8 * cg + b;
        if (j < dout) ys[(rg + 16 * a) * ldy + j] = acc[a][b];
      }
    __syncthreads();
    // A warp per descriptor, rows in increasing order per warp, so the image
    // of the frame is found once per warp and then walked forward.
    i64 img = 0, next = INT64_MAX;  // next: first row of image img + 1
    if (p.frames && warp < nr) {
      i64 lo = 0, hi = p.nimg;  // the last image whose first row is <= r0 + warp
      while (hi - lo > 1) {
        const i64 mid = (lo + hi) / 2;
        if (p.offs[mid] <= r0 + warp) lo = mid;
        else hi = mid;
      }
      img = lo;
      next = img + 1 < p.nimg ? p.offs[img + 1] : INT64_MAX;
    }
    for (int r = warp; r < nr; r += kWarps) {
      const i64 row = r0 + r;
      float inv = 1.f;
      if (p.renorm) {
        float ss = 0.f;
        for (int j = lane; j < dout; j += 32) ss = __fmaf_rn(ys[r * ldy + j], ys[r * ldy + j], ss);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
        inv = 1.f / fmaxf(1e-12f, sqrtf(ss));
      }
      float *o = p.out + row * p.ldo;
      for (int j = lane; j < dout; j += 32) o[j] = ys[r * ldy + j] * inv;
      if (p.frames) {
        while (next <= row) {
          ++img;
          next = img + 1 < p.nimg ? p.offs[img + 1] : INT64_MAX;
        }
        if (lane < 2) {
          const float sz = p.sizes[2 * img + lane];
          o[dout + lane] = (p.frames[2 * row + lane] - sz * 0.5f) * (1.f / sz);
        }
      }
    }
    __syncthreads();  // the buffer is free for the next tile
  }
  // A CTA that stopped early lets its copy in flight land before exiting.
  if (BULK && tid == 0 && *s_abort) {
    const unsigned long long t0 = tc::global_ns();
    while (!tc::mbar_try_wait(full, (uint32_t)(k & 1)) && tc::global_ns() - t0 < tc::kWaitNs) {
    }
  }
}

// ------------------------------------------------ tensor-core projection
// The projection as a tcgen05 GEMM per tile of 128 descriptors, in scaled
// fp16x3 (two fp16 parts per operand, products hi.hi + hi.lo + lo.hi with fp32
// accumulation in TMEM):
//  - x' = x - c per descriptor is scaled by 2^s (s per row: max |x'| into
//    [2^14, 2^15)), P by 2^g (one g: max |P| into [2^14, 2^15)); the epilogue
//    undoes both exactly, so fp16's range holds any input and each operand
//    keeps 22 significant bits;
//  - roles: warps 0-7 producers (16 rows each; a lane converts 4 dimensions of
//    a row: coalesced 512-byte row loads, a warp max for the row's scale, the
//    hi/lo split, stores into the K-major 64-byte-swizzled A tile), warps 8-11
//    epilogue (one row per thread: TMEM -> scale -> renormalisation -> 'xy'
//    -> store), warp 12 TMEM allocation and the MMA issue;
//  - two A stages and two TMEM accumulators of np columns; P's image stays in
//    shared memory for the CTA's life.
constexpr int kPtThreads = 416;

struct PcaTcParams {
  float *out;
  int ldo, din, dout, renorm, nka, np, vec_out;  // vec_out: 4, 2 or 1 floats per store
  int vec_xy;                                    // frames and xy outputs as float2
  i64 N, nimg, ntiles;
  const float *X, *P, *c, *frames, *sizes;
  const i64 *offs;
  int *err;
};

// Dynamic shared memory from a 1024-aligned base: A stages (2 x nka x 16 KB:
// hi atoms then lo atoms), P image (hi nka x np x 64 B, then lo), control
// block (barriers, flags, row exponents, the image of each stage's first row).
__host__ __device__ inline size_t pt_a_bytes(int nka) { return (size_t)2 * nka * 16384; }
__host__ __device__ inline size_t pt_p_bytes(int nka, int np) { return (size_t)nka * np * 128; }
constexpr size_t kPtCtl = 128 + 2 * 128 * sizeof(int) + 16;
__host__ inline size_t pt_smem(int nka, int np) { return 1024 + pt_a_bytes(nka) + pt_p_bytes(nka, np) + kPtCtl; }

__device__ __forceinline__ float pow2f(int e) {  // 2^e for e in [-126, 127]
  return __int_as_float((e + 127) << 23);
}

__global__ void __launch_bounds__(kPtThreads, 1) k_pca_tc(const PcaTcParams p) {
  using namespace tc;
  extern __shared__ __align__(16) unsigned char pt_raw[];
  const uint32_t raw_s = smem_u32(pt_raw);
  const uint32_t base_s = (raw_s + 1023u) & ~1023u;
  unsigned char *base = pt_raw + (base_s - raw_s);
  const int nka = p.nka, np = p.np;
  const uint32_t a_s = base_s;                         // stage st: hi at a_s + st*nka*16K, lo + nka*8K
  const uint32_t p_s = base_s + (uint32_t)pt_a_bytes(nka);  // P hi; lo at + nka*np*64
  unsigned char *ctl = base + pt_a_bytes(nka) + pt_p_bytes(nka, np);
  uint64_t *full = (uint64_t *)ctl;       // [2], producers' arrivals
  uint64_t *accf = full + 2;              // [2], MMA commit
  uint64_t *acce = full + 4;              // [2], epilogue arrivals
  volatile int *s_abort = (volatile int *)(full + 6);
  uint32_t *s_tmem = (uint32_t *)(full + 7);
  int *s_g = (int *)(full + 8);
  float *s_red = (float *)(full + 9);     // 13 warp maxima (up to full + 16)
  int *sexp = (int *)(ctl + 128);         // [2][128] row exponents
  i64 *timg = (i64 *)(ctl + 128 + 2 * 128 * sizeof(int));  // [2] image of each stage's first row
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  if (tid == 0) {
    mbar_init(&full[0], 256);
    mbar_init(&full[1], 256);
    mbar_init(&accf[0], 1);
    mbar_init(&accf[1], 1);
    mbar_init(&acce[0], 128);
    mbar_init(&acce[1], 128);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // P's scale: g with max |P| 2^g in [2^14, 2^15).
  float mx = 0.f;
  const int nP = p.dout * p.din;
  for (int e = tid; e < nP; e += kPtThreads) mx = fmaxf(mx, fabsf(__ldg(p.P + e)));
  mx = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(mx)));
  if (lane == 0) s_red[warp] = mx;
  if (warp == 12) tmem_alloc(s_tmem, 256);
  if (warp == 12) tmem_relinquish();
  __syncthreads();
  if (tid == 0) {
    float m = 0.f;
    for (int w = 0; w < kPtThreads / 32; ++w) m = fmaxf(m, s_red[w]);
    int e = 0;
    if (m > 0.f) frexpf(m, &e);
    *s_g = m > 0.f ? max(-126, min(126, 15 - e)) : 0;
  }
  __syncthreads();
  const int g = *s_g;
  {
    // P image: row n (output), element k (input dimension), zero padded.
    const float sg = pow2f(g);
    const int kmax = nka * 32;
    for (int e = tid; e < np * kmax; e += kPtThreads) {
      const int n = e / kmax, k = e - n * kmax;
      const float v = (n < p.dout && k < p.din) ? __ldg(p.P + (i64)n * p.din + k) * sg : 0.f;
      const __half hi = __float2half_rn(v);
      const __half lo = __float2half_rn(v - __half2float(hi));
      const uint32_t off = (uint32_t)(k >> 5) * (uint32_t)np * 64u + kmajor_sw64_off((uint32_t)n, (uint32_t)((k & 31) >> 3)) +
                           (uint32_t)(k & 7) * 2u;
      *(__half *)(base + pt_a_bytes(nka) + off) = hi;
      *(__half *)(base + pt_a_bytes(nka) + (size_t)nka * np * 64 + off) = lo;
    }
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  if (warp < 8) {
    // ------------------------------------------------------- producers
    const int k0 = 4 * lane;
    const bool in = k0 < p.din, pad = k0 < nka * 32;
    float4 cv = make_float4(0.f, 0.f, 0.f, 0.f);
    if (in) cv = __ldg((const float4 *)(p.c + k0));
    const uint32_t aoff = (uint32_t)(lane >> 3) * 8192u;  // atom of this lane's 4 dimensions
    const uint32_t chunk = (uint32_t)((lane & 7) >> 1), half8 = (uint32_t)(lane & 1) * 8u;
    int tt = 0;
    // The rows of the next tile are loaded as soon as the current tile's are
    // converted, before waiting for a free stage, so their latency overlaps
    // that wait.
    float4 xv[16];
    auto load = [&](i64 t) {
      const i64 r0 = t * 128 + 16 * warp;
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        const i64 row = r0 + u;
        xv[u] = (in && t < p.ntiles && row < p.N) ? __ldg((const float4 *)(p.X + row * p.din + k0))
                                                  : make_float4(0.f, 0.f, 0.f, 0.f);
      }
    };
    load(blockIdx.x);
    i64 pimg = 0;  // image of the previous tile's first row (rows only increase)
    for (i64 t = blockIdx.x; t < p.ntiles; t += gridDim.x, ++tt) {
      const int st = tt & 1;
      if (tt >= 2 && !mbar_wait(&acce[st], ((tt >> 1) & 1) ^ 1, s_abort, p.err, 11)) break;
      if (p.frames && tid == 0) {
        // The last image whose first row is <= the tile's first row: gallop
        // forward from the previous tile's, then bisect (offs[nimg] = N).
        const i64 f0 = t * 128;
        i64 lo = pimg, hi = lo + 1, step = 1;
        while (hi < p.nimg && __ldg(p.offs + hi) <= f0) {
          lo = hi;
          step *= 2;
          hi = min(p.nimg, lo + step);
        }
        while (hi - lo > 1) {
          const i64 mid = (lo + hi) / 2;
          if (__ldg(p.offs + mid) <= f0) lo = mid;
          else hi = mid;
        }
        timg[st] = pimg = lo;
      }
      const i64 r0 = t * 128 + 16 * warp;
      const uint32_t ahi = a_s + (uint32_t)st * (uint32_t)nka * 16384u, alo = ahi + (uint32_t)nka * 8192u;
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        const bool live = in && r0 + u < p.N;
        const float v0 = live ? __fsub_rn(xv[u].x, cv.x) : 0.f, v1 = live ? __fsub_rn(xv[u].y, cv.y) : 0.f;
        const float v2 = live ? __fsub_rn(xv[u].z, cv.z) : 0.f, v3 = live ? __fsub_rn(xv[u].w, cv.w) : 0.f;
        const float m = fmaxf(fmaxf(fabsf(v0), fabsf(v1)), fmaxf(fabsf(v2), fabsf(v3)));
        const float rm = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(m)));
        int e = 0;
        if (rm > 0.f) frexpf(rm, &e);
        const int sx = rm > 0.f ? max(-126, min(126, 15 - e)) : 0;
        const float f = pow2f(sx);
        uint32_t h0, l0, h1, l1;
        split2<true>(v0 * f, v1 * f, h0, l0);
        split2<true>(v2 * f, v3 * f, h1, l1);
        const uint32_t rl = (uint32_t)(16 * warp + u);
        if (pad) {
          const uint32_t off = aoff + kmajor_sw64_off(rl, chunk) + half8;
          st_shared_v2(ahi + off, h0, h1);
          st_shared_v2(alo + off, l0, l1);
        }
        if (lane == 0) sexp[st * 128 + rl] = sx;
      }
      fence_proxy_async_smem();
      mbar_arrive(&full[st]);
      load(t + gridDim.x);
    }
  } else if (warp < 12) {
    // -------------------------------------------------------- epilogue
    const int ew = warp - 8, rl = 32 * ew + lane;
    const int nch = (np + 31) / 32;
    int tt = 0;
    for (i64 t = blockIdx.x; t < p.ntiles; t += gridDim.x, ++tt) {
      const int buf = tt & 1;
      if (!mbar_wait(&accf[buf], (tt >> 1) & 1, s_abort, p.err, 12)) break;
      tc_fence_after();
      const i64 row = t * 128 + rl;
      const bool valid = row < p.N;
      const int sx = sexp[buf * 128 + rl];
      const i64 img0 = p.frames ? timg[buf] : 0;  // read before the stage is released below
      // acc 2^-(s + g).  The combined exponent e is applied as 2^e1 2^(e - e1)
      // with e1 the part within a float's normal range: the second factor is 1
      // unless |e| > 126, and the first product cannot overflow (or leave the
      // normal range) when the final value is finite and normal, whatever the
      // signs of s and g.
      const int e = -(sx + g), e1 = e > 126 ? 126 : (e < -126 ? -126 : e);
      const float f1 = pow2f(e1), f2 = pow2f(e - e1);
      const uint32_t taddr = tmem + (uint32_t)(buf * 128) + ((uint32_t)(32 * ew) << 16);
      float inv = 1.f;
      if (p.renorm) {
        float ss = 0.f;
        for (int ch = 0; ch < nch; ++ch) {
          uint32_t v[32];
          tmem_ld32(taddr + (uint32_t)(ch * 32), v);
          tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const float y = __uint_as_float(v[j]) * f1 * f2;
            if (ch * 32 + j < p.dout) ss = __fmaf_rn(y, y, ss);
          }
        }
        inv = 1.f / fmaxf(1e-12f, sqrtf(ss));
      }
      float *o = p.out + row * p.ldo;
      for (int ch = 0; ch < nch; ++ch) {
        uint32_t v[32];
        tmem_ld32(taddr + (uint32_t)(ch * 32), v);
        tmem_wait_ld();
        if (!valid) continue;
        const int j0 = ch * 32;
        if (p.vec_out == 4) {
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            if (j0 + 4 * q < p.dout) {
              float4 w;
              w.x = __uint_as_float(v[4 * q]) * f1 * f2 * inv;
              w.y = __uint_as_float(v[4 * q + 1]) * f1 * f2 * inv;
              w.z = __uint_as_float(v[4 * q + 2]) * f1 * f2 * inv;
              w.w = __uint_as_float(v[4 * q + 3]) * f1 * f2 * inv;
              *(float4 *)(o + j0 + 4 * q) = w;
            }
          }
        } else if (p.vec_out == 2) {
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            if (j0 + 2 * q < p.dout) {
              float2 w;
              w.x = __uint_as_float(v[2 * q]) * f1 * f2 * inv;
              w.y = __uint_as_float(v[2 * q + 1]) * f1 * f2 * inv;
              *(float2 *)(o + j0 + 2 * q) = w;
            }
          }
        } else {
#pragma unroll
          for (int j = 0; j < 32; ++j)
            if (j0 + j < p.dout) o[j0 + j] = __uint_as_float(v[j]) * f1 * f2 * inv;
        }
      }
      tc_fence_before();
      mbar_arrive(&acce[buf]);
      if (p.frames && valid) {
        // Forward from the image of the tile's first row.
        i64 img = img0;
        while (img + 1 < p.nimg && __ldg(p.offs + img + 1) <= row) ++img;
        if (p.vec_xy) {
          const float2 fr = __ldg((const float2 *)(p.frames + 2 * row));
          const float2 sz = __ldg((const float2 *)(p.sizes + 2 * img));
          *(float2 *)(o + p.dout) = make_float2((fr.x - sz.x * 0.5f) * (1.f / sz.x), (fr.y - sz.y * 0.5f) * (1.f / sz.y));
        } else {
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const float sz = __ldg(p.sizes + 2 * img + i);
            o[p.dout + i] = (__ldg(p.frames + 2 * row + i) - sz * 0.5f) * (1.f / sz);
          }
        }
      }
    }
  } else if (lane == 0) {
    // ------------------------------------------------------------- MMA
    const uint32_t idesc = idesc_f16(128, np, false, false);
    const uint32_t phi = p_s, plo = p_s + (uint32_t)nka * (uint32_t)np * 64u;
    int tt = 0;
    for (i64 t = blockIdx.x; t < p.ntiles; t += gridDim.x, ++tt) {
      const int buf = tt & 1;
      if (!mbar_wait(&acce[buf], ((tt >> 1) & 1) ^ 1, s_abort, p.err, 13)) break;
      if (!mbar_wait(&full[buf], (tt >> 1) & 1, s_abort, p.err, 14)) break;
      tc_fence_after();
      const uint32_t d = tmem + (uint32_t)(buf * 128);
      const uint32_t ahi = a_s + (uint32_t)buf * (uint32_t)nka * 16384u, alo = ahi + (uint32_t)nka * 8192u;
      for (int a = 0; a < nka; ++a) {
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
          const uint64_t ah = sdesc(ahi + (uint32_t)a * 8192u + ks * 32, 16, 512, kSw64);
          const uint64_t al = sdesc(alo + (uint32_t)a * 8192u + ks * 32, 16, 512, kSw64);
          const uint64_t bh = sdesc(phi + (uint32_t)a * (uint32_t)np * 64u + ks * 32, 16, 512, kSw64);
          const uint64_t bl = sdesc(plo + (uint32_t)a * (uint32_t)np * 64u + ks * 32, 16, 512, kSw64);
          mma_bf16(d, ah, bh, idesc, (a > 0 || ks > 0) ? 1u : 0u);
          mma_bf16(d, ah, bl, idesc, 1u);
          mma_bf16(d, al, bh, idesc, 1u);
        }
      }
      mma_commit(&accf[buf]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 12) {
    tc_fence_after();
    tmem_dealloc(tmem, 256);
  }
}

// Per-dimension sums (fp64) of a slab of rows: slab b writes sums[b][d].
__global__ void k_pca_colsum(const float *__restrict__ X, int din, i64 N, i64 slab, double *__restrict__ sums) {
  const int d = threadIdx.x;
  if (d >= din) return;
  const i64 r0 = (i64)blockIdx.x * slab, r1 = min(N, r0 + slab);
  double s = 0.0;
  for (i64 r = r0; r < r1; ++r) s += (double)X[r * din + d];
  sums[(i64)blockIdx.x * din + d] = s;
}

// Partial covariance of a slab: part[b][a][e] = sum_r (x_ra - c_a)(x_re - c_e)
// in fp64; one CTA per slab, thread (ty, tx) owns entries (16p + ty, 16q + tx)
// of every 16 x 16 tile (p, q), rows staged 32 at a time.
constexpr int kCovRows = 32;

__global__ void __launch_bounds__(256) k_pca_cov(const float *__restrict__ X, int din, i64 N, i64 slab,
                                                 const double *__restrict__ mean, double *__restrict__ part) {
  __shared__ double xs[kCovRows][kPcaMaxIn + 1];
  const i64 r0 = (i64)blockIdx.x * slab, r1 = min(N, r0 + slab);
  const int ntile = (din + 15) / 16;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  constexpr int kMaxT = kPcaMaxIn / 16;
  double acc[kMaxT][kMaxT];
#pragma unroll
  for (int p = 0; p < kMaxT; ++p)
#pragma unroll
    for (int q = 0; q < kMaxT; ++q) acc[p][q] = 0.0;
  for (i64 rb = r0; rb < r1; rb += kCovRows) {
    __syncthreads();
    for (int i = threadIdx.x; i < kCovRows * din; i += 256) {
      const int r = i / din, d = i % din;
      const i64 row = rb + r;
      xs[r][d] = row < r1 ? (double)X[row * din + d] - mean[d] : 0.0;
    }
    __syncthreads();
    const int nr = r1 - rb < (i64)kCovRows ? (int)(r1 - rb) : kCovRows;
    for (int r = 0; r < nr; ++r) {
#pragma unroll
      for (int p = 0; p < kMaxT; ++p) {
        if (p < ntile) {
          const int a = 16 * p + ty;
          const double va = a < din ? xs[r][a] : 0.0;
#pragma unroll
          for (int q = 0; q < kMaxT; ++q) {
            if (q < ntile) {
              const int e = 16 * q + tx;
              acc[p][q] = fma(va, e < din ? xs[r][e] : 0.0, acc[p][q]);
            }
          }
        }
      }
    }
  }
#pragma unroll
  for (int p = 0; p < kMaxT; ++p)
#pragma unroll
    for (int q = 0; q < kMaxT; ++q) {
      const int a = 16 * p + ty, e = 16 * q + tx;
      if (a < din && e < din) part[((i64)blockIdx.x * din + a) * din + e] = acc[p][q];
    }
}

// Fixed-order sum of the slab partials: out[i] = sum_b part[b][i].
__global__ void k_pca_reduce(const double *__restrict__ part, i64 nslab, i64 n, double *__restrict__ out) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (i64 b = 0; b < nslab; ++b) s += part[b * n + i];
  out[i] = s;
}

// Cyclic Jacobi eigen-decomposition of a symmetric n x n matrix (row-major,
// destroyed): eigenvalues in w, eigenvectors in the columns of V.
void jacobi_eig(std::vector<double> &A, int n, std::vector<double> &w, std::vector<double> &V) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) (i == j ? diag : off) += A[(size_t)i * n + j] * A[(size_t)i * n + j];
    if (off <= 1e-30 * std::max(diag, 1e-300)) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = A[(size_t)p * n + q];
        if (apq == 0.0) continue;
        const double app = A[(size_t)p * n + p], aqq = A[(size_t)q * n + q];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double cs = 1.0 / std::sqrt(t * t + 1.0), sn = t * cs;
        for (int k = 0; k < n; ++k) {  // A = A J (columns p, q)
          const double akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
          A[(size_t)k * n + p] = cs * akp - sn * akq;
          A[(size_t)k * n + q] = sn * akp + cs * akq;
        }
        for (int k = 0; k < n; ++k) {  // A = J^T A (rows p, q)
          const double apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
          A[(size_t)p * n + k] = cs * apk - sn * aqk;
          A[(size_t)q * n + k] = sn * apk + cs * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = V[(size_t)k * n + p], vkq = V[(size_t)k * n + q];
          V[(size_t)k * n + p] = cs * vkp - sn * vkq;
          V[(size_t)k * n + q] = sn * vkp + cs * vkq;
        }
      }
  }
  w.resize(n);
  for (int i = 0; i < n; ++i) w[i] = A[(size_t)i * n + i];
}

}  // namespace

void pca_project(float *out, i64 ldo, const float *X, i64 din, i64 N, i64 dout, const float *P, const float *c,
                 bool renorm, const float *frames, const i64 *h_offsets, const float *sizes, i64 nimg,
                 cudaStream_t s) {
  VLB_CHECK(din >= 1 && din <= kPcaMaxIn && dout >= 1 && dout <= kPcaMaxOut, VL_ERR_BAD_ARG,
            "PCA projection: dimensions must be in [1, 128]");
  if (N <= 0) return;
  Scratch &sc = thread_scratch(kArenaVlad);
  const i64 *doffs = nullptr;
  if (frames) {
    VLB_CHECK(h_offsets && sizes && nimg >= 1, VL_ERR_BAD_ARG, "PCA projection: frames need image offsets and sizes");
    i64 *d = sc.slot[10].get<i64>(nimg + 1);
    VLB_CUDA(cudaMemcpyAsync(d, h_offsets, sizeof(i64) * (nimg + 1), cudaMemcpyHostToDevice, s));
    doffs = d;
  }
  int *derr = sc.slot[15].get<int>(1);
  VLB_CUDA(cudaMemsetAsync(derr, 0, sizeof(int), s));
  PcaParams p;
  p.out = out; p.ldo = (int)ldo; p.din = (int)din; p.dout = (int)dout; p.renorm = renorm ? 1 : 0;
  p.N = N; p.nimg = nimg; p.X = X; p.P = P; p.c = c; p.frames = frames; p.sizes = sizes; p.offs = doffs;
  p.err = derr;
  if (din % 4 == 0 && (uintptr_t)X % 16 == 0 && (uintptr_t)c % 16 == 0) {
    // Tensor-core path: fp16x3 tcgen05 GEMM with the fused epilogue.
    PcaTcParams q;
    q.out = out; q.ldo = (int)ldo; q.din = (int)din; q.dout = (int)dout; q.renorm = renorm ? 1 : 0;
    q.nka = (int)((din + 31) / 32);
    q.np = (int)((dout + 15) / 16 * 16);
    q.vec_out = (ldo % 4 == 0 && dout % 4 == 0 && (uintptr_t)out % 16 == 0)  ? 4
                : (ldo % 2 == 0 && dout % 2 == 0 && (uintptr_t)out % 8 == 0) ? 2
                                                                               : 1;
    q.N = N; q.nimg = frames ? nimg : 0; q.ntiles = (N + 127) / 128;
    q.vec_xy = (frames && (uintptr_t)frames % 8 == 0 && (uintptr_t)sizes % 8 == 0 && ldo % 2 == 0 &&
                dout % 2 == 0 && (uintptr_t)out % 8 == 0) ? 1 : 0;
    q.X = X; q.P = P; q.c = c; q.frames = frames; q.sizes = sizes; q.offs = doffs; q.err = derr;
    const size_t smem = pt_smem(q.nka, q.np);
    const int grid = (int)std::min<i64>(q.ntiles, (i64)sm_count());
    VLB_CUDA(cudaFuncSetAttribute(k_pca_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    VLB_LAUNCH("pca_project_tc", s, k_pca_tc<<<grid, kPtThreads, smem, s>>>(q));
    int herr = 0;
    VLB_CUDA(cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, s));
    VLB_CUDA(cudaStreamSynchronize(s));
    VLB_CHECK(herr == 0, VL_ERR_ALLOC, "PCA projection: a pipeline wait timed out on the device");
    return;
  }
  const bool bulk = (din % 4) == 0 && ((uintptr_t)X % 16) == 0;
  const size_t tile = sizeof(float) * (size_t)kPcaRows * pca_ldx((int)din);
  const size_t smem = 128 + sizeof(float) * ((size_t)((din + 3) / 4 * 4) * pca_ldp((int)dout) + pca_ldx((int)din)) +
                      std::max<size_t>(tile, sizeof(float) * (size_t)kPcaRows * (size_t)(dout + 1));
  const i64 ntiles = (N + kPcaRows - 1) / kPcaRows;
  const int grid = (int)std::min<i64>(ntiles, (i64)sm_count() * 2);
  auto run = [&](auto kern, int threads) {
    VLB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    VLB_LAUNCH("pca_project", s, kern<<<grid, threads, smem, s>>>(p));
  };
  // Output groups of 8, rounded up to even so that every warp is whole (the
  // renormalisation shuffles use full masks); padded outputs are zeros.
  const int nc = (int)(((dout + 7) / 8 + 1) & ~1);
#define VLB_PCA_CASE(n)                                  \
  case n:                                                \
    if (bulk) run(k_pca_project<n, true>, 16 * n);       \
    else run(k_pca_project<n, false>, 16 * n);           \
    break;
  switch (nc) {
    VLB_PCA_CASE(2) VLB_PCA_CASE(4) VLB_PCA_CASE(6) VLB_PCA_CASE(8) VLB_PCA_CASE(10) VLB_PCA_CASE(12)
    VLB_PCA_CASE(14) default: VLB_PCA_CASE(16)
  }
#undef VLB_PCA_CASE
  int herr = 0;
  VLB_CUDA(cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, s));
  // The offsets and error buffers are reused by the next call on this thread.
  VLB_CUDA(cudaStreamSynchronize(s));
  VLB_CHECK(herr == 0, VL_ERR_ALLOC, "PCA projection: a copy wait timed out on the device");
}

void pca_learn(float *P, float *center, i64 m, const float *X, i64 din, i64 N, bool whitening, double regul,
               double *eigenvalues, cudaStream_t s) {
  VLB_CHECK(din >= 1 && din <= kPcaMaxIn, VL_ERR_BAD_ARG, "PCA learning: dimension must be in [1, 128]");
  VLB_CHECK(m >= 1 && m <= din, VL_ERR_BAD_ARG, "PCA learning: numPcaDimensions must be in [1, dimension]");
  VLB_CHECK(N >= 1, VL_ERR_BAD_ARG, "PCA learning: no data");
  Scratch &sc = thread_scratch(kArenaVlad);
  const i64 nslab = std::min<i64>(N, (i64)sm_count() * 2);
  const i64 slab = (N + nslab - 1) / nslab;
  double *sums = sc.slot[11].get<double>((size_t)nslab * din);
  double *mean = sc.slot[12].get<double>(din);
  VLB_LAUNCH("pca_colsum", s, k_pca_colsum<<<(unsigned)nslab, 128, 0, s>>>(X, (int)din, N, slab, sums));
  VLB_LAUNCH("pca_reduce", s,
             k_pca_reduce<<<(unsigned)((din + 127) / 128), 128, 0, s>>>(sums, nslab, din, mean));
  std::vector<double> hmean(din);
  VLB_CUDA(cudaMemcpyAsync(hmean.data(), mean, sizeof(double) * din, cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaStreamSynchronize(s));
  for (auto &v : hmean) v /= (double)N;
  VLB_CUDA(cudaMemcpyAsync(mean, hmean.data(), sizeof(double) * din, cudaMemcpyHostToDevice, s));
  double *part = sc.slot[13].get<double>((size_t)nslab * din * din);
  double *cov = sc.slot[14].get<double>((size_t)din * din);
  VLB_LAUNCH("pca_cov", s, k_pca_cov<<<(unsigned)nslab, 256, 0, s>>>(X, (int)din, N, slab, mean, part));
  VLB_LAUNCH("pca_reduce", s,
             k_pca_reduce<<<(unsigned)((din * din + 255) / 256), 256, 0, s>>>(part, nslab, din * din, cov));
  std::vector<double> A((size_t)din * din);
  VLB_CUDA(cudaMemcpyAsync(A.data(), cov, sizeof(double) * din * din, cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaStreamSynchronize(s));
  // Symmetrise (the two triangles were summed separately) and scale by 1/N.
  for (i64 a = 0; a < din; ++a)
    for (i64 e = a; e < din; ++e) {
      const double v = 0.5 * (A[a * din + e] + A[e * din + a]) / (double)N;
      A[a * din + e] = A[e * din + a] = v;
    }
  std::vector<double> w, V;
  jacobi_eig(A, (int)din, w, V);
  std::vector<int> perm(din);
  for (int i = 0; i < (int)din; ++i) perm[i] = i;
  std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return w[a] > w[b]; });
  const double dmax = w[perm[0]];
  std::vector<float> hP((size_t)m * din);
  for (i64 j = 0; j < m; ++j) {
    const int col = perm[j];
    const double dj = w[col] + regul * dmax;
    // Sign convention: the entry of largest magnitude is positive.
    i64 am = 0;
    for (i64 d = 1; d < din; ++d)
      if (std::fabs(V[d * din + col]) > std::fabs(V[am * din + col])) am = d;
    const double sg = V[am * din + col] < 0 ? -1.0 : 1.0;
    const double scale = whitening ? 1.0 / std::sqrt(dj) : 1.0;
    for (i64 d = 0; d < din; ++d) hP[(size_t)j * din + d] = (float)(sg * scale * V[d * din + col]);
    if (eigenvalues) eigenvalues[j] = dj;
  }
  std::vector<float> hc(din);
  for (i64 d = 0; d < din; ++d) hc[d] = (float)hmean[d];
  VLB_CUDA(cudaMemcpyAsync(P, hP.data(), sizeof(float) * hP.size(), cudaMemcpyHostToDevice, s));
  VLB_CUDA(cudaMemcpyAsync(center, hc.data(), sizeof(float) * din, cudaMemcpyHostToDevice, s));
  VLB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace vlb

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
}  // namespace

extern "C" {

int vlb200_pca_project_device(float *out, vl_size dimOut, float const *data, vl_size dimIn, vl_size numData,
                              float const *projection, float const *center, int renormalize,
                              float const *frames, vl_int64 const *offsets, float const *imageSizes,
                              vl_size numImages, void *stream) {
  return guarded([&] {
    const vl_size ldo = dimOut + (frames ? 2 : 0);
    vlb::pca_project(out, (vlb::i64)ldo, data, (vlb::i64)dimIn, (vlb::i64)numData, (vlb::i64)dimOut, projection,
                     center, renormalize != 0, frames, (const vlb::i64 *)offsets, imageSizes,
                     (vlb::i64)numImages, vlb::pick_stream(stream));
  });
}

int vlb200_pca_learn_device(float *projection, float *center, vl_size numPcaDimensions, float const *data,
                            vl_size dimIn, vl_size numData, int whitening, double whiteningRegul,
                            double *eigenvalues, void *stream) {
  return guarded([&] {
    vlb::pca_learn(projection, center, (vlb::i64)numPcaDimensions, data, (vlb::i64)dimIn, (vlb::i64)numData,
                   whitening != 0, whiteningRegul, eigenvalues, vlb::pick_stream(stream));
  });
}

}  // extern "C"
