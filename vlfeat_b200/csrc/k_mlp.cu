// Dense layers of the learned router on the tensor cores.
//
// One persistent tcgen05 kernel computes C = act(A . B^T + bias) for a layer:
// A (M x Ka) the activations and B (N x Ka) the weights, both bf16 and
// row-major (K-major), fp32 accumulation in TMEM, the bias and ReLU applied
// in the epilogue, C stored as bf16 (hidden layers, the next layer's A) or
// fp32 (logits).  Operand tiles are staged by TMA (cp.async.bulk.tensor.2d,
// 128-byte swizzle, zero fill past the matrix edges) into a ring of shared
// memory stages:
//   warp 0     TMA producer (one thread),
//   warp 1     TMEM allocation and, from one lane, tcgen05.mma issue,
//   warps 2-9  epilogue: TMEM -> registers -> bias, ReLU -> global; two
//              warps per TMEM lane quarter, each taking half of the tile's
//              columns, the bias staged in shared memory.
// Tiles are 128 rows x BN columns (BN = N rounded up to 16, at most 256),
// 64-element k-blocks (4 MMAs of K = 16 each), two TMEM accumulators so that
// one tile's epilogue overlaps the next tile's MMAs.  Every mbarrier wait is
// bounded (tc_common.cuh); an expired wait records its code in the error word.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "engine.h"
#include "tc_common.cuh"

namespace vlb {
namespace {

using namespace tc;

constexpr int kMlpThreads = 320;
constexpr int kMlpEpiThreads = 256;
constexpr int kMlpMaxN = 4096;  // bias entries staged in shared memory
constexpr int kBM = 128, kBK = 64;
constexpr int kMlpSmemLimit = 232448;

constexpr int kSelList = 16;  // the selecting epilogue keeps each row's 16 largest logits

struct MlpParams {
  CUtensorMap ta, tb;  // A: {Ka, M}, box {64, 128};  B: {Ka, N}, box {64, BN}
  const float *bias;
  void *c;
  int M, N, Ka, BN, nst, relu, out_f32;
  // Selecting epilogue (sel = 1): instead of writing C, keep each row's m
  // largest logits (ties: lowest index) and their softmax mass.
  int sel, m;
  int *cand;
  float *cmass;
  int *err;
};

// The j-th tile of this CTA as (mt, nt); false past the last one.  With the
// selecting epilogue a CTA takes whole rows of tiles (every n-tile of an
// m-tile, in order), so each row's logits pass through one thread pair.
__device__ __forceinline__ bool tile_at(const MlpParams &p, int mtiles, int ntiles, int j, int &mt, int &nt) {
  if (p.sel) {
    mt = (int)blockIdx.x + (j / ntiles) * (int)gridDim.x;
    nt = j % ntiles;
    return mt < mtiles;
  }
  const long long t = (long long)blockIdx.x + (long long)j * gridDim.x;
  mt = (int)(t / ntiles);
  nt = (int)(t % ntiles);
  return t < (long long)mtiles * ntiles;
}



__global__ void __launch_bounds__(kMlpThreads, 1) k_tc_dense(const __grid_constant__ MlpParams p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *base = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t aBytes = kBM * kBK * 2, bBytes = (uint32_t)p.BN * kBK * 2, stageBytes = aBytes + bBytes;
  uint64_t *bars = (uint64_t *)(base + (size_t)p.nst * stageBytes);
  uint64_t *full = bars, *empty = bars + 8, *accf = bars + 16, *acce = bars + 18;
  uint32_t *s_tmem = (uint32_t *)(bars + 20);
  volatile int *s_abort = (volatile int *)(s_tmem + 1);
  uint64_t *xbar = bars + 24;  // selecting epilogue: one per TMEM lane quarter (64 arrivals)
  float *s_bias = (float *)(bars + 32);  // N floats
  // Selecting epilogue's exchange: per TMEM lane quarter and lane, the second
  // half's list (values, indices) and its (max, sum).
  float *s_xv = s_bias + ((p.N + 3) & ~3);
  int *s_xi = (int *)(s_xv + 4 * 32 * kSelList);
  float *s_xm = (float *)(s_xi + 4 * 32 * kSelList);
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int mtiles = (p.M + kBM - 1) / kBM, ntiles = (p.N + p.BN - 1) / p.BN;
  const int nkb = (p.Ka + kBK - 1) / kBK;
  if (threadIdx.x == 0) {
    for (int s = 0; s < p.nst; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], kMlpEpiThreads);
    }
    for (int b = 0; b < 4; ++b) mbar_init(&xbar[b], 64);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    tmem_alloc(s_tmem, 512);
    tmem_relinquish();
  }
  for (int n = threadIdx.x; n < p.N; n += kMlpThreads) s_bias[n] = p.bias[n];
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;

  if (warp == 0 && lane == 0) {
    // ---------------------------------------------------------- producer
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&p.ta)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&p.tb)) : "memory");
    int it = 0, mt, nt;
    for (int j = 0; tile_at(p, mtiles, ntiles, j, mt, nt); ++j) {
      bool ok = true;
      for (int kb = 0; kb < nkb; ++kb, ++it) {
        const int st = it % p.nst;
        if (!mbar_wait(&empty[st], ((it / p.nst) & 1) ^ 1, s_abort, p.err, 31)) {
          ok = false;
          break;
        }
        const uint32_t sa = smem_u32(base + (size_t)st * stageBytes);
        mbar_arrive_expect_tx(&full[st], stageBytes);
        tma_load_2d(sa, &p.ta, kb * kBK, mt * kBM, &full[st]);
        tma_load_2d(sa + aBytes, &p.tb, kb * kBK, nt * p.BN, &full[st]);
      }
      if (!ok) break;
    }
  } else if (warp == 1 && lane == 0) {
    // --------------------------------------------------------------- MMA
    const uint32_t idesc = idesc_bf16(kBM, p.BN, false, false);
    int it = 0, tt = 0, mt, nt;
    bool ok = true;
    for (; ok && tile_at(p, mtiles, ntiles, tt, mt, nt); ++tt) {
      const int buf = tt & 1;
      if (!mbar_wait(&acce[buf], ((tt >> 1) & 1) ^ 1, s_abort, p.err, 32)) break;
      tc_fence_after();
      const uint32_t d = tmem + (uint32_t)(buf * 256);
      for (int kb = 0; kb < nkb; ++kb, ++it) {
        const int st = it % p.nst;
        if (!mbar_wait(&full[st], (it / p.nst) & 1, s_abort, p.err, 33)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t sa = smem_u32(base + (size_t)st * stageBytes), sb = sa + aBytes;
#pragma unroll
        for (int ks = 0; ks < kBK / 16; ++ks) {
          const uint64_t ad = sdesc(sa + ks * 32, 16, 1024, kSw128);
          const uint64_t bd = sdesc(sb + ks * 32, 16, 1024, kSw128);
          mma_bf16(d, ad, bd, idesc, (kb > 0 || ks > 0) ? 1u : 0u);
        }
        mma_commit(&empty[st]);
      }
      if (ok) mma_commit(&accf[buf]);
    }
  } else if (warp >= 2) {
    // ---------------------------------------------------------- epilogue
    const int q = warp & 3;  // TMEM lane quarter this warp may access
    const int half = (warp - 2) >> 2;  // which half of the tile's 32-column chunks
    const int r = q * 32 + lane;
    const int nch = (p.BN + 31) / 32, ch0 = half ? (nch + 1) / 2 : 0, ch1 = half ? nch : (nch + 1) / 2;
    int tt = 0, mt, nt;
    // Selecting epilogue state of this thread's row and half: the 16 largest
    // logits seen (descending; ties keep the lower index first, as columns
    // arrive in increasing order) and the online softmax (max, sum).
    float lv[kSelList], smx = -INFINITY, ssum = 0.f;
    int li[kSelList];
    int xph = 0;  // uses of this quarter's exchange barrier so far
    for (; tile_at(p, mtiles, ntiles, tt, mt, nt); ++tt) {
      const int buf = tt & 1;
      if (!mbar_wait(&accf[buf], (tt >> 1) & 1, s_abort, p.err, 34)) break;
      tc_fence_after();
      const long long row = (long long)mt * kBM + r;
      const bool valid = row < p.M;
      const uint32_t tb = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * 256);
      if (p.sel && nt == 0) {
#pragma unroll
        for (int i = 0; i < kSelList; ++i) {
          lv[i] = -INFINITY;
          li[i] = half * kSelList + i;  // distinct valid indices (N >= 32) if nothing beats -inf
        }
        smx = -INFINITY;
        ssum = 0.f;
      }
      for (int c0 = 32 * ch0; c0 < 32 * ch1; c0 += 32) {
        uint32_t v[32];
        tmem_ld32(tb + (uint32_t)c0, v);
        tmem_wait_ld();
        const int n0 = nt * p.BN + c0;
        if (!valid) continue;
        if (p.sel) {
          float cm = -INFINITY;
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const float a = __uint_as_float(v[j]) + (n0 + j < p.N ? s_bias[n0 + j] : 0.f);
            v[j] = __float_as_uint(n0 + j < p.N ? a : -INFINITY);
            cm = fmaxf(cm, __uint_as_float(v[j]));
          }
          if (cm > smx) {
            ssum = smx == -INFINITY ? 0.f : ssum * __expf(smx - cm);
            smx = cm;
          }
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            float cv = __uint_as_float(v[j]);
            ssum += cv == -INFINITY ? 0.f : __expf(cv - smx);
            if (cv > lv[kSelList - 1]) {
              int ci = n0 + j;
#pragma unroll
              for (int i = 0; i < kSelList; ++i)
                if (cv > lv[i]) {
                  const float tv = lv[i];
                  const int ti = li[i];
                  lv[i] = cv;
                  li[i] = ci;
                  cv = tv;
                  ci = ti;
                }
            }
          }
          continue;
        }
#pragma unroll
        for (int g = 0; g < 4; ++g) {
          const int n = n0 + 8 * g;
          if (n >= p.N) break;  // N is a multiple of 8: a group is wholly in or out
          float y[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            float a = __uint_as_float(v[8 * g + j]) + s_bias[n + j];
            y[j] = (p.relu && !(a > 0.f)) ? 0.f : a;
          }
          if (p.out_f32) {
            float4 *dst = (float4 *)((float *)p.c + row * p.N + n);
            dst[0] = make_float4(y[0], y[1], y[2], y[3]);
            dst[1] = make_float4(y[4], y[5], y[6], y[7]);
          } else {
            uint4 w;
            w.x = pack2<false>(y[0], y[1]);
            w.y = pack2<false>(y[2], y[3]);
            w.z = pack2<false>(y[4], y[5]);
            w.w = pack2<false>(y[6], y[7]);
            *(uint4 *)((__nv_bfloat16 *)p.c + row * p.N + n) = w;
          }
        }
      }
      tc_fence_before();
      mbar_arrive(&acce[buf]);
      if (p.sel && nt == ntiles - 1) {
        // Merge the two halves of each row (the warps of a lane quarter pair
        // up through shared memory), then write the row's m candidates and
        // their softmax mass.
        const int slot = q * 32 + lane;
        if (half == 1) {
#pragma unroll
          for (int i = 0; i < kSelList; ++i) {
            s_xv[slot * kSelList + i] = lv[i];
            s_xi[slot * kSelList + i] = li[i];
          }
          s_xm[2 * slot] = smx;
          s_xm[2 * slot + 1] = ssum;
        }
        // Bounded waits: a partner that left on an abort cannot strand this warp.
        mbar_arrive(&xbar[q]);
        if (!mbar_wait(&xbar[q], xph & 1, s_abort, p.err, 35)) break;
        ++xph;
        if (half == 0 && valid) {
          const float omx = s_xm[2 * slot], osum = s_xm[2 * slot + 1];
          const float MX = fmaxf(smx, omx);
          const float S = (smx == -INFINITY ? 0.f : ssum * __expf(smx - MX)) +
                          (omx == -INFINITY ? 0.f : osum * __expf(omx - MX));
          int a = 0, b = 0;
          float mass = 0.f;
          for (int i = 0; i < p.m; ++i) {
            const float bv = b < kSelList ? s_xv[slot * kSelList + b] : -INFINITY;
            const int bi = b < kSelList ? s_xi[slot * kSelList + b] : 0x7fffffff;
            // First list wins ties unless the other's index is lower.
            const bool takeA = a < kSelList && (b >= kSelList || lv[0] > bv || (lv[0] == bv && li[0] < bi));
            float val;
            int idx;
            if (takeA) {
              val = lv[0];
              idx = li[0];
              ++a;
#pragma unroll
              for (int k = 0; k < kSelList - 1; ++k) {
                lv[k] = lv[k + 1];
                li[k] = li[k + 1];
              }
              lv[kSelList - 1] = -INFINITY;
            } else {
              val = bv;
              idx = bi;
              ++b;
            }
            p.cand[row * p.m + i] = idx;
            mass += __expf(val - MX);
          }
          p.cmass[row] = mass / S;
        }
        mbar_arrive(&xbar[q]);
        if (!mbar_wait(&xbar[q], xph & 1, s_abort, p.err, 36)) break;
        ++xph;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// x (n x D, fp32) -> bf16 features (x - centre) * scale, rows padded with
// zeros to Ka columns.
__global__ void k_features_bf16(const float *__restrict__ X, long long n, int D, int Ka,
                                const float *__restrict__ ctr, const float *__restrict__ scl,
                                __nv_bfloat16 *__restrict__ Z) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * Ka) return;
  const long long row = i / Ka;
  const int d = (int)(i % Ka);
  Z[i] = __float2bfloat16_rn(d < D ? (X[row * D + d] - ctr[d]) * scl[d] : 0.f);
}

// fp32 weights (out x in) -> bf16 (out x inPad), zero padding columns.
__global__ void k_weights_bf16(const float *__restrict__ W, int out, int in, int inPad,
                               __nv_bfloat16 *__restrict__ Wb) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)out * inPad) return;
  const int o = (int)(i / inPad), k = (int)(i % inPad);
  Wb[i] = __float2bfloat16_rn(k < in ? W[(long long)o * in + k] : 0.f);
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  });
  VLB_CHECK(fn != nullptr, VL_ERR_BAD_ARG, "cuTensorMapEncodeTiled is not available from the driver");
  return fn;
}

// 2-D bf16 row-major matrix (rows x cols, cols contiguous) for TMA boxes of
// 64 columns x boxRows rows with the 128-byte swizzle.
void make_map(CUtensorMap *m, const void *ptr, long long rows, int cols, int boxRows) {
  tc::tma_map_2d(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, ptr, rows, cols, kBK, boxRows, CU_TENSOR_MAP_SWIZZLE_128B);
}

}  // namespace

namespace tc {
void tma_map(CUtensorMap *m, CUtensorMapDataType type, int rank, const void *ptr, const unsigned long long *dims,
             const unsigned long long *strides, const unsigned *box, CUtensorMapSwizzle swizzle) {
  VLB_CHECK(rank >= 1 && rank <= 5 && ((uintptr_t)ptr & 15) == 0, VL_ERR_BAD_ARG,
            "tensor map: the tensor must start 16-byte aligned");
  cuuint64_t d[5], st[4];
  cuuint32_t bx[5], estr[5];
  for (int i = 0; i < rank; ++i) {
    d[i] = (cuuint64_t)dims[i];
    bx[i] = (cuuint32_t)box[i];
    estr[i] = 1;
    if (i + 1 < rank) {
      VLB_CHECK(strides[i] % 16 == 0, VL_ERR_BAD_ARG, "tensor map: strides must be multiples of 16 bytes");
      st[i] = (cuuint64_t)strides[i];
    }
  }
  const CUresult r = encode_fn()(m, type, (cuuint32_t)rank, const_cast<void *>(ptr), d, st, bx, estr,
                                 CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  VLB_CHECK(r == CUDA_SUCCESS, VL_ERR_BAD_ARG, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
}

void tma_map_2d(CUtensorMap *m, CUtensorMapDataType type, int esize, const void *ptr, long long rows, int cols,
                int boxCols, int boxRows, CUtensorMapSwizzle swizzle) {
  const unsigned long long dims[2] = {(unsigned long long)cols, (unsigned long long)rows};
  const unsigned long long strides[1] = {(unsigned long long)cols * (unsigned long long)esize};
  const unsigned box[2] = {(unsigned)boxCols, (unsigned)boxRows};
  tma_map(m, type, 2, ptr, dims, strides, box, swizzle);
}
}  // namespace tc

bool tc_dense_supported(int N, int Ka) {
  return N >= 8 && N % 8 == 0 && N <= kMlpMaxN && Ka >= 8 && Ka % 8 == 0;
}

void tc_dense(const __nv_bfloat16 *A, long long M, int Ka, const __nv_bfloat16 *W, int N, const float *bias,
              bool relu, bool outF32, void *C, int *err, cudaStream_t s, int selM, int *cand, float *cmass) {
  if (M <= 0) return;
  VLB_CHECK(tc_dense_supported(N, Ka), VL_ERR_BAD_ARG, "dense layer: widths must be multiples of 8, N <= 4096");
  VLB_CHECK(selM == 0 || (selM >= 1 && selM <= kSelList && N >= 32 && cand && cmass), VL_ERR_BAD_ARG,
            "dense layer: selection of 1..16 candidates from at least 32 outputs");
  MlpParams p;
  const int BN = std::min(256, (N + 15) / 16 * 16);
  make_map(&p.ta, A, M, Ka, kBM);
  make_map(&p.tb, W, N, Ka, BN);
  p.bias = bias;
  p.c = C;
  p.M = (int)M;
  p.N = N;
  p.Ka = Ka;
  p.BN = BN;
  p.relu = relu ? 1 : 0;
  p.out_f32 = outF32 ? 1 : 0;
  p.sel = selM > 0 ? 1 : 0;
  p.m = selM;
  p.cand = cand;
  p.cmass = cmass;
  p.err = err;
  const size_t stageBytes = (size_t)(kBM + BN) * kBK * 2;
  const size_t fixed = 1024 /*alignment*/ + 256 /*barriers, TMEM base, abort flag*/ +
                       4 * (size_t)((N + 3) & ~3) /*bias*/ + (size_t)(2 * 4 * 32 * kSelList + 256) * 4 /*exchange*/;
  p.nst = (int)std::min<size_t>(8, (kMlpSmemLimit - fixed) / stageBytes);
  VLB_CHECK(p.nst >= 2, VL_ERR_BAD_ARG, "dense layer: operand stages exceed shared memory");
  const size_t smem = fixed + (size_t)p.nst * stageBytes;
  VLB_CUDA(cudaFuncSetAttribute(k_tc_dense, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long tiles = p.sel ? (M + kBM - 1) / kBM : ((M + kBM - 1) / kBM) * ((N + BN - 1) / BN);
  int nsm = 0, dev = 0;
  VLB_CUDA(cudaGetDevice(&dev));
  VLB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int grid = (int)std::min<long long>(tiles, nsm);
  VLB_LAUNCH("router_dense_tc", s, k_tc_dense<<<grid, kMlpThreads, smem, s>>>(p));
}

void features_bf16(const float *X, long long n, int D, int Ka, const float *ctr, const float *scl,
                   __nv_bfloat16 *Z, cudaStream_t s) {
  const long long total = n * Ka;
  if (total <= 0) return;
  VLB_LAUNCH("router_features_bf16", s,
             k_features_bf16<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(X, n, D, Ka, ctr, scl, Z));
}

void weights_bf16(const float *W, int out, int in, int inPad, __nv_bfloat16 *Wb, cudaStream_t s) {
  const long long total = (long long)out * inPad;
  VLB_LAUNCH("router_weights_bf16", s,
             k_weights_bf16<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(W, out, in, inPad, Wb));
}

}  // namespace vlb
