// Learned candidate router for the E-step.
//
// A small MLP  x -> [Linear, ReLU]* -> Linear -> K logits  predicts, for each
// descriptor, which mixture components carry its posterior mass.  Inference
// keeps the top-m components, evaluates the exact posterior on those only
// (the reference's arithmetic, vl/gmm.c:762-790, restricted to the
// candidates), and falls back to the full E-step for descriptors whose
// predicted candidate mass (router softmax summed over the top-m) is below a
// threshold (0.99 by default).  The router is trained here, on the GPU, by
// the kernels of this file: forward, backward (data and weight gradients),
// top-8 cross-entropy against posteriors produced by the full E-step, and
// Adam.  Weights are held in fp32 and used in the forward and backward passes
// rounded to bf16 (BF16 weights, fp32 accumulation).
//
// All reductions run in a fixed order, so training and inference are
// bitwise reproducible for a given seed.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <vector>

#include "engine.h"

extern "C" {
#include "vlb200.h"
}

using vlb::i64;

namespace vlb {
namespace {

constexpr int kT = 256;
inline unsigned gridn(i64 n, int b) { return (unsigned)((n + b - 1) / b); }

__device__ __forceinline__ float bf16_round(float x) {
  return __bfloat162float(__float2bfloat16_rn(x));
}

// C(m, n) = sum_k A(m, k) B(n, k) (+ bias[n]) (ReLU), with A(m,k) = A[m*sam + k*sak],
// B(n,k) = B[n*sbn + k*sbk].  64 x 64 tiles, 16-deep k slices, 4 x 4 outputs
// per thread, fp32 accumulation; every output is summed over k in order.
template <bool RELU, bool BIAS>
__global__ void __launch_bounds__(kT) k_gemm(const float *__restrict__ A, i64 sam, i64 sak,
                                            const float *__restrict__ B, i64 sbn, i64 sbk,
                                            const float *__restrict__ bias, float *__restrict__ C,
                                            i64 ldc, int M, int N, int Kd) {
  __shared__ float sa[16][64 + 4];
  __shared__ float sb[16][64 + 4];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < Kd; k0 += 16) {
    for (int e = threadIdx.x; e < 16 * 64; e += kT) {
      const int kk = e / 64, mm = e % 64;
      const int m = m0 + mm, k = k0 + kk;
      sa[kk][mm] = (m < M && k < Kd) ? A[(i64)m * sam + (i64)k * sak] : 0.f;
      const int n = n0 + mm;
      sb[kk][mm] = (n < N && k < Kd) ? B[(i64)n * sbn + (i64)k * sbk] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        a[i] = sa[kk][ty * 4 + i];
        b[i] = sb[kk][tx * 4 + i];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * b[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty * 4 + i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx * 4 + j;
      if (n >= N) continue;
      float v = acc[i][j] + (BIAS ? bias[n] : 0.f);
      if (RELU) v = v > 0.f ? v : 0.f;
      C[(i64)m * ldc + n] = v;
    }
  }
}

// Input features: z = (x - centre) * scale.
__global__ void k_features(const float *__restrict__ X, i64 n, int D, const float *__restrict__ ctr,
                           const float *__restrict__ scl, float *__restrict__ Z) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * D) return;
  const int d = (int)(i % D);
  Z[i] = (X[i] - ctr[d]) * scl[d];
}

__global__ void k_round_bf16(const float *__restrict__ w, float *__restrict__ wq, i64 n) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) wq[i] = bf16_round(w[i]);
}

// dH *= (H > 0): ReLU derivative applied to an upstream gradient.
__global__ void k_relu_mask(float *__restrict__ g, const float *__restrict__ h, i64 n) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && !(h[i] > 0.f)) g[i] = 0.f;
}

// Column sums db[n] = sum_m G[m, n] (fixed order over m).
__global__ void k_colsum(const float *__restrict__ G, int M, int N, float *__restrict__ db) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int m = 0; m < M; ++m) s += G[(i64)m * N + n];
  db[n] = s;
}

// Top-T targets of each row of the posteriors: indices and weights
// renormalised over the T entries.  One warp per row, T rounds of arg-max.
template <int T>
__global__ void k_topk_targets(const float *__restrict__ q, i64 n, int K, int *__restrict__ idx,
                               float *__restrict__ w) {
  const i64 row = (i64)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (row >= n) return;
  const float *r = q + row * K;
  int taken[T];
  float tv[T];
  float tot = 0.f;
  for (int t = 0; t < T; ++t) {
    float bv = -1.f;
    int bi = 0x7fffffff;
    for (int k = lane; k < K; k += 32) {
      bool used = false;
      for (int u = 0; u < t; ++u) used |= (taken[u] == k);
      const float v = r[k];
      if (!used && (v > bv || (v == bv && k < bi))) { bv = v; bi = k; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
    }
    taken[t] = bi;
    tv[t] = bv > 0.f ? bv : 0.f;
    tot += tv[t];
  }
  if (lane < T) {
    idx[row * T + lane] = taken[lane];
    w[row * T + lane] = tot > 0.f ? tv[lane] / tot : 1.f / T;
  }
}

// Softmax cross-entropy against sparse top-T target distributions:
// loss_row = -sum_t w_t log softmax(z)_{idx_t};  dZ = (softmax(z) - target) / B.
template <int T>
__global__ void k_xent(const float *__restrict__ Zl, int B, int K, const int *__restrict__ idx,
                       const float *__restrict__ w, float *__restrict__ dZ,
                       double *__restrict__ rowloss) {
  const int row = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (row >= B) return;
  const float *z = Zl + (i64)row * K;
  float mx = -INFINITY;
  for (int k = lane; k < K; k += 32) mx = fmaxf(mx, z[k]);
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  float s = 0.f;
  for (int k = lane; k < K; k += 32) s += expf(z[k] - mx);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  const float lse = mx + logf(s);
  const float invB = 1.f / (float)B;
  for (int k = lane; k < K; k += 32) {
    float t = 0.f;
#pragma unroll
    for (int u = 0; u < T; ++u)
      if (idx[(i64)row * T + u] == k) t += w[(i64)row * T + u];
    dZ[(i64)row * K + k] = (expf(z[k] - lse) - t) * invB;
  }
  if (lane == 0) {
    double l = 0;
    for (int u = 0; u < T; ++u) l -= (double)w[(i64)row * T + u] * ((double)z[idx[(i64)row * T + u]] - lse);
    rowloss[row] = l;
  }
}

__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, i64 n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Candidates: top-m logits of each row and the router's softmax mass on them.
// One warp per row; lane l holds logits l, l + 32, ... in registers (KPL of
// them, K <= 32 KPL).  Each of the m rounds takes the largest logit not yet
// taken (ties: lowest index), found by a lane scan and a warp arg-max; the
// owner lane marks it taken in a bit mask.
template <int KPL>
__global__ void k_select(const float *__restrict__ Zl, i64 n, int K, int m, int *__restrict__ cand,
                         float *__restrict__ cmass) {
  const i64 row = (i64)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (row >= n) return;
  const float *z = Zl + row * K;
  float zv[KPL];
  float mx = -INFINITY;
#pragma unroll
  for (int i = 0; i < KPL; ++i) {
    const int k = lane + 32 * i;
    zv[i] = k < K ? z[k] : -INFINITY;
    if (k < K) mx = fmaxf(mx, zv[i]);
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  float s = 0.f;
#pragma unroll
  for (int i = 0; i < KPL; ++i)
    if (lane + 32 * i < K) s += expf(zv[i] - mx);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  uint32_t taken = 0;
  int mine = 0;
  float sel = 0.f;
  for (int t = 0; t < m; ++t) {
    float bv = -INFINITY;
    int bi = 0x7fffffff;
#pragma unroll
    for (int i = 0; i < KPL; ++i) {
      const int k = lane + 32 * i;
      if (k < K && !((taken >> i) & 1u) && (zv[i] > bv || (zv[i] == bv && k < bi))) {
        bv = zv[i];
        bi = k;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
    }
    if (bi == 0x7fffffff) {
      // No remaining logit compares above -inf (NaN or -inf logits): take the
      // lowest untaken index, so that every candidate is a valid component.
      int li = 0x7fffffff;
#pragma unroll
      for (int i = 0; i < KPL; ++i) {
        const int k = lane + 32 * i;
        if (k < K && !((taken >> i) & 1u) && k < li) li = k;
      }
      for (int o = 16; o > 0; o >>= 1) li = min(li, __shfl_xor_sync(0xffffffffu, li, o));
      bi = li;  // < K: m <= K components are taken in all
      bv = -INFINITY;
    }
    if (lane == (bi & 31)) taken |= 1u << (bi >> 5);
    if (lane == t) mine = bi;
    sel += expf(bv - mx);
  }
  if (lane < m) cand[row * m + lane] = mine;
  if (lane == 0) cmass[row] = sel / s;
}

// Exact posteriors on the candidates (vl/gmm.c:762-790 restricted to them),
// or on all K components for fallback rows.  One warp per row; the dimension
// is spread over the lanes.  Writes a dense row of q (zeros off the
// candidates), the row's log-likelihood share and whether it fell back.
__global__ void k_candidate_estep(const float *__restrict__ X, i64 n, int D, int K,
                                  const float *__restrict__ means, const float *__restrict__ inv,
                                  const double *__restrict__ cst, const int *__restrict__ cand,
                                  const float *__restrict__ cmass, int m, float thr,
                                  float *__restrict__ q, unsigned char *__restrict__ fell,
                                  double *__restrict__ llrow, bool deferFallback) {
  const i64 row = (i64)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (row >= n) return;
  const float *x = X + row * D;
  float *qr = q + row * K;
  const bool fb = !(cmass[row] >= thr);  // a NaN mass (NaN logits) falls back too
  if (fb && deferFallback) {
    // The row goes to the tensor-core E-step with the other fallback rows.
    if (lane == 0) {
      fell[row] = 1;
      if (llrow) llrow[row] = 0.0;
    }
    return;
  }
  const int nc = fb ? K : m;
  for (int k = lane; k < K; k += 32) qr[k] = 0.f;
  __syncwarp();
  // Pass 1: log-densities (stored temporarily in q) and their maximum.  Four
  // candidates at a time, so that their loads and shuffle reductions overlap.
  float mx = -INFINITY;
  for (int c0 = 0; c0 < nc; c0 += 4) {
    int kk[4];
    float acc[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int c = min(c0 + u, nc - 1);  // a partial group repeats the last candidate
      kk[u] = fb ? c : cand[row * m + c];
      acc[u] = 0.f;
    }
    for (int d = lane; d < D; d += 32) {
      const float xd = x[d];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const float df = xd - means[(i64)kk[u] * D + d];
        acc[u] += df * df * inv[(i64)kk[u] * D + d];
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int u = 0; u < 4; ++u) acc[u] += __shfl_xor_sync(0xffffffffu, acc[u], o);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (c0 + u >= nc) break;
      const float p = (float)(cst[kk[u]] - 0.5 * (double)acc[u]);
      if (lane == 0) qr[kk[u]] = p;
      mx = fmaxf(mx, p);
    }
  }
  __syncwarp();
  float s = 0.f;
  for (int c = lane; c < nc; c += 32) {
    const int k = fb ? c : cand[row * m + c];
    s += expf(qr[k] - mx);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __syncwarp();
  for (int c = lane; c < nc; c += 32) {
    const int k = fb ? c : cand[row * m + c];
    qr[k] = expf(qr[k] - mx) / s;
  }
  if (lane == 0) fell[row] = fb ? 1 : 0;
  // The row's log-likelihood over the components evaluated (all of them on
  // fallback rows): the E-step's log-sum-exp restricted to the candidates.
  if (lane == 0 && llrow) llrow[row] = (double)mx + log((double)s);
}

// Stable list of the rows that fell back (their order kept): per-block
// counts, one exclusive scan, then each block writes its rows' indices.
__global__ void k_fb_count(const unsigned char *__restrict__ fell, i64 n, int *__restrict__ counts) {
  const i64 row = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  const int c = __syncthreads_count(row < n && fell[row]);
  if (threadIdx.x == 0) counts[blockIdx.x] = c;
}
__global__ void k_fb_scan(int *__restrict__ counts, int nb, int *__restrict__ total) {
  if (threadIdx.x != 0) return;
  int acc = 0;
  for (int b = 0; b < nb; ++b) {
    const int c = counts[b];
    counts[b] = acc;
    acc += c;
  }
  *total = acc;
}
__global__ void k_fb_scatter(const unsigned char *__restrict__ fell, i64 n, const int *__restrict__ offs,
                             int *__restrict__ idx) {
  __shared__ int warpBase[32];
  const i64 row = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
  const bool f = row < n && fell[row];
  const unsigned bal = __ballot_sync(0xffffffffu, f);
  if (lane == 0) warpBase[warp] = __popc(bal);
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) {
      const int c = warpBase[w];
      warpBase[w] = acc;
      acc += c;
    }
  }
  __syncthreads();
  if (f) idx[offs[blockIdx.x] + warpBase[warp] + __popc(bal & ((1u << lane) - 1u))] = (int)row;
}
// Rows idx[j] of src (width w floats) -> row j of dst, or back (scatter).
__global__ void k_rows_gather(const float *__restrict__ src, const int *__restrict__ idx, int cnt, int w,
                              float *__restrict__ dst, bool scatter) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (i64)cnt * w) return;
  const i64 j = i / w;
  const int c = (int)(i - j * w);
  const i64 r = idx[j];
  if (scatter) dst[r * w + c] = src[i];
  else dst[i] = src[r * w + c];
}

// Missed posterior mass of each row: sum of the full-E-step posteriors that
// the candidate rows set to zero.
__global__ void k_missed(const float *__restrict__ qfull, const float *__restrict__ qc, i64 n, int K,
                         double *__restrict__ out) {
  const i64 row = (i64)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x % 32;
  if (row >= n) return;
  float s = 0.f;
  for (int k = lane; k < K; k += 32)
    if (qc[row * K + k] == 0.f) s += qfull[row * K + k];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) out[row] = s;
}

}  // namespace
}  // namespace vlb

// ====================================================================== host
namespace vlb {
double tc_fallback(const float *X, i64 B, const DevModel<float> &m, const unsigned char *fell, float *q,
                   unsigned long long *nfb, cudaStream_t s);
}

struct _VlB200Router {
  int D = 0, K = 0;
  std::vector<int> sizes;  // D, hidden..., K
  // Parameters (device): per layer W (out x in), b (out); Adam moments.
  std::vector<vlb::DevBuf *> W, b, Wq, mW, vW, mb, vb, gW, gb;
  // bf16 weights for the tensor-core inference (layer l: out x in8(in), the
  // input width rounded up to a multiple of 8 with zero columns).
  std::vector<vlb::DevBuf *> Wb;
  bool tcInfer = true;  // inference on the tensor cores when the widths allow
  vlb::DevBuf ctr, scl;
  long step = 0;
  ~_VlB200Router() {
    for (auto *v : {&W, &b, &Wq, &mW, &vW, &mb, &vb, &gW, &gb, &Wb})
      for (auto *p : *v) delete p;
  }
};

namespace {

using vlb::DevBuf;

template <typename F>
int guarded(F &&f) {
  try {
    f();
    return 0;
  } catch (const vlb::Error &e) {
    return vl_set_last_error(e.code, "%s", e.what());
  } catch (const std::exception &e) {
    return vl_set_last_error(VL_ERR_BAD_ARG, "%s", e.what());
  }
}

int nlayers(const VlB200Router *r) { return (int)r->sizes.size() - 1; }

void gemm(bool relu, bool bias, const float *A, i64 sam, i64 sak, const float *B, i64 sbn, i64 sbk,
          const float *bvec, float *C, i64 ldc, int M, int N, int Kd, cudaStream_t s) {
  dim3 g(vlb::gridn(N, 64), vlb::gridn(M, 64));
  if (relu && bias)
    VLB_LAUNCH("router_gemm", s, (vlb::k_gemm<true, true><<<g, vlb::kT, 0, s>>>(A, sam, sak, B, sbn, sbk, bvec, C, ldc, M, N, Kd)));
  else if (bias)
    VLB_LAUNCH("router_gemm", s, (vlb::k_gemm<false, true><<<g, vlb::kT, 0, s>>>(A, sam, sak, B, sbn, sbk, bvec, C, ldc, M, N, Kd)));
  else
    VLB_LAUNCH("router_gemm", s, (vlb::k_gemm<false, false><<<g, vlb::kT, 0, s>>>(A, sam, sak, B, sbn, sbk, bvec, C, ldc, M, N, Kd)));
}

int in8(int n) { return (n + 7) / 8 * 8; }

void refresh_bf16(VlB200Router *r, cudaStream_t s) {
  for (int l = 0; l < nlayers(r); ++l) {
    const i64 n = (i64)r->sizes[l + 1] * r->sizes[l];
    VLB_LAUNCH("router_round", s,
               vlb::k_round_bf16<<<vlb::gridn(n, 256), 256, 0, s>>>((float *)r->W[l]->p, (float *)r->Wq[l]->p, n));
    const int in = r->sizes[l], out = r->sizes[l + 1];
    while ((int)r->Wb.size() <= l) r->Wb.push_back(new DevBuf());
    vlb::weights_bf16((const float *)r->W[l]->p, out, in, in8(in),
                      r->Wb[l]->get<__nv_bfloat16>((size_t)out * in8(in)), s);
  }
}

// Inference on the tensor cores: every layer's output width a multiple of 8.
bool tc_infer_ok(const VlB200Router *r) {
  if (!r->tcInfer || nlayers(r) > 6) return false;
  for (size_t l = 1; l < r->sizes.size(); ++l)
    if (!vlb::tc_dense_supported(r->sizes[l], in8(r->sizes[l - 1]))) return false;
  return true;
}

i64 infer_chunk(const VlB200Router *r) { return tc_infer_ok(r) ? (1 << 20) : (1 << 17); }

void forward(VlB200Router *r, const float *X, i64 B, std::vector<float *> &act, cudaStream_t s);

// Rows per inference chunk and the forward's buffers for it: the tensor-core
// path needs only the logits (its activations are bf16, in slots 7 and 8),
// so it takes 2^20 rows at a time; the CUDA-core path 2^17 with every layer's
// fp32 activations.
i64 infer_chunk(const VlB200Router *r);
std::vector<float *> infer_buffers(VlB200Router *r, vlb::Scratch &sc, i64 chunk) {
  const int L = nlayers(r);
  std::vector<float *> act(L + 1, nullptr);
  const bool tc = infer_chunk(r) == (1 << 20);
  for (int l = 0; l <= L; ++l)
    if (!tc || l == L) act[l] = sc.slot[l].get<float>((size_t)chunk * r->sizes[l]);
  return act;
}

// Logits (B x K, fp32) of a batch for inference: on the tensor cores (bf16
// features and activations, bf16 weights, fp32 accumulation; tcgen05 dense
// layers), else the training forward on the CUDA cores.  act: the forward's
// buffers (act[L] receives the logits).
// With selM > 0 (and at most 16 of at least 32 outputs) the last layer's
// epilogue selects each row's candidates itself (cand, cmass) instead of
// writing the logits; returns whether it did.
bool forward_infer(VlB200Router *r, const float *X, i64 B, std::vector<float *> &act, vlb::Scratch &sc,
                   cudaStream_t s, int selM = 0, int *cand = nullptr, float *cmass = nullptr) {
  if (!tc_infer_ok(r)) {
    forward(r, X, B, act, s);
    return false;
  }
  const bool sel = selM >= 1 && selM <= 16 && r->K >= 32;
  const int L = nlayers(r);
  int *err = sc.slot[9].get<int>(1);
  VLB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
  // Ping-pong bf16 activation buffers (slots 7 and 8; slots 0 .. L hold the
  // fp32 activations, so L <= 6).
  int wmax = 0;
  for (int l = 0; l < L; ++l) wmax = std::max(wmax, in8(r->sizes[l]));
  __nv_bfloat16 *buf[2] = {sc.slot[7].get<__nv_bfloat16>((size_t)B * wmax),
                           sc.slot[8].get<__nv_bfloat16>((size_t)B * wmax)};
  vlb::features_bf16(X, B, r->D, in8(r->D), (const float *)r->ctr.p, (const float *)r->scl.p, buf[0], s);
  for (int l = 0; l < L; ++l) {
    const int out = r->sizes[l + 1];
    const bool last = l + 1 == L;
    vlb::tc_dense(buf[l & 1], B, in8(r->sizes[l]), (const __nv_bfloat16 *)r->Wb[l]->p, out,
                  (const float *)r->b[l]->p, !last, last, last ? (void *)act[L] : (void *)buf[(l + 1) & 1], err, s,
                  last && sel ? selM : 0, cand, cmass);
  }
  int h = 0;
  VLB_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaStreamSynchronize(s));
  if (h) throw vlb::Error(VL_ERR_BAD_ARG, "router dense layer gave up waiting (code " + std::to_string(h) + ")");
  return sel;
}

// Activations of a batch: act[0] = features, act[l+1] = layer l output.
void forward(VlB200Router *r, const float *X, i64 B, std::vector<float *> &act, cudaStream_t s) {
  const int L = nlayers(r);
  VLB_LAUNCH("router_features", s,
             vlb::k_features<<<vlb::gridn(B * r->D, 256), 256, 0, s>>>(X, B, r->D, (float *)r->ctr.p,
                                                                     (float *)r->scl.p, act[0]));
  for (int l = 0; l < L; ++l) {
    const int in = r->sizes[l], out = r->sizes[l + 1];
    gemm(l + 1 < L, true, act[l], in, 1, (float *)r->Wq[l]->p, in, 1, (float *)r->b[l]->p, act[l + 1],
         out, (int)B, out, in, s);
  }
}

}  // namespace

extern "C" {

VlB200Router *vlb200_router_new(vl_size dimension, vl_size numClusters, vl_size const *hidden,
                                vl_size numHidden, vl_uint32 seed) {
  VlB200Router *r = nullptr;
  int rc = guarded([&] {
    VLB_CHECK(dimension >= 1 && numClusters >= 2, VL_ERR_BAD_ARG, "router: bad sizes");
    r = new VlB200Router();
    r->D = (int)dimension;
    r->K = (int)numClusters;
    r->sizes.push_back((int)dimension);
    for (vl_size i = 0; i < numHidden; ++i) r->sizes.push_back((int)hidden[i]);
    r->sizes.push_back((int)numClusters);
    std::mt19937_64 gen(seed);
    cudaStream_t s = vlb::thread_stream();
    for (int l = 0; l < nlayers(r); ++l) {
      const int in = r->sizes[l], out = r->sizes[l + 1];
      std::vector<float> w((size_t)in * out), bb(out, 0.f);
      std::normal_distribution<float> nd(0.f, std::sqrt(2.f / (float)in));  // He initialisation
      for (auto &v : w) v = nd(gen);
      for (auto *vec : {&r->W, &r->Wq, &r->mW, &r->vW, &r->gW}) vec->push_back(new DevBuf());
      for (auto *vec : {&r->b, &r->mb, &r->vb, &r->gb}) vec->push_back(new DevBuf());
      float *dW = r->W[l]->get<float>(w.size());
      r->Wq[l]->get<float>(w.size());
      r->gW[l]->get<float>(w.size());
      VLB_CUDA(cudaMemsetAsync(r->mW[l]->get<float>(w.size()), 0, w.size() * 4, s));
      VLB_CUDA(cudaMemsetAsync(r->vW[l]->get<float>(w.size()), 0, w.size() * 4, s));
      VLB_CUDA(cudaMemsetAsync(r->mb[l]->get<float>(out), 0, out * 4, s));
      VLB_CUDA(cudaMemsetAsync(r->vb[l]->get<float>(out), 0, out * 4, s));
      r->gb[l]->get<float>(out);
      VLB_CUDA(cudaMemcpyAsync(dW, w.data(), w.size() * 4, cudaMemcpyHostToDevice, s));
      VLB_CUDA(cudaMemcpyAsync(r->b[l]->get<float>(out), bb.data(), out * 4, cudaMemcpyHostToDevice, s));
    }
    std::vector<float> one((size_t)dimension, 1.f), zero((size_t)dimension, 0.f);
    VLB_CUDA(cudaMemcpyAsync(r->ctr.get<float>(dimension), zero.data(), dimension * 4, cudaMemcpyHostToDevice, s));
    VLB_CUDA(cudaMemcpyAsync(r->scl.get<float>(dimension), one.data(), dimension * 4, cudaMemcpyHostToDevice, s));
    refresh_bf16(r, s);
    VLB_CUDA(cudaStreamSynchronize(s));
  });
  if (rc) {
    delete r;
    return nullptr;
  }
  return r;
}

void vlb200_router_delete(VlB200Router *r) { delete r; }

vl_size vlb200_router_num_params(VlB200Router const *r) {
  vl_size n = 0;
  for (size_t l = 0; l + 1 < r->sizes.size(); ++l) n += (vl_size)r->sizes[l + 1] * (r->sizes[l] + 1);
  return n;
}

// Parameters as one host vector: for each layer W (out x in, row-major) then b.
int vlb200_router_get_params(VlB200Router const *r, float *out) {
  return guarded([&] {
    cudaStream_t s = vlb::thread_stream();
    size_t o = 0;
    for (int l = 0; l < nlayers(r); ++l) {
      const size_t nw = (size_t)r->sizes[l + 1] * r->sizes[l], nb = r->sizes[l + 1];
      VLB_CUDA(cudaMemcpyAsync(out + o, r->W[l]->p, nw * 4, cudaMemcpyDeviceToHost, s));
      o += nw;
      VLB_CUDA(cudaMemcpyAsync(out + o, r->b[l]->p, nb * 4, cudaMemcpyDeviceToHost, s));
      o += nb;
    }
    VLB_CUDA(cudaStreamSynchronize(s));
  });
}

int vlb200_router_set_params(VlB200Router *r, float const *in) {
  return guarded([&] {
    cudaStream_t s = vlb::thread_stream();
    size_t o = 0;
    for (int l = 0; l < nlayers(r); ++l) {
      const size_t nw = (size_t)r->sizes[l + 1] * r->sizes[l], nb = r->sizes[l + 1];
      VLB_CUDA(cudaMemcpyAsync(r->W[l]->p, in + o, nw * 4, cudaMemcpyHostToDevice, s));
      o += nw;
      VLB_CUDA(cudaMemcpyAsync(r->b[l]->p, in + o, nb * 4, cudaMemcpyHostToDevice, s));
      o += nb;
    }
    refresh_bf16(r, s);
    VLB_CUDA(cudaStreamSynchronize(s));
  });
}

// Feature normalisation z = (x - centre) * scale (host arrays of D).
int vlb200_router_set_input_transform(VlB200Router *r, float const *centre, float const *scale) {
  return guarded([&] {
    cudaStream_t s = vlb::thread_stream();
    VLB_CUDA(cudaMemcpyAsync(r->ctr.p, centre, r->D * 4, cudaMemcpyHostToDevice, s));
    VLB_CUDA(cudaMemcpyAsync(r->scl.p, scale, r->D * 4, cudaMemcpyHostToDevice, s));
    VLB_CUDA(cudaStreamSynchronize(s));
  });
}

// Loss and gradients of one batch against top-8 targets (device arrays
// tidx, tw: B x 8).  grads: host vector in the get_params layout, or NULL.
// Used by training and by the gradient check against the CPU oracle.
int vlb200_router_loss_grad(VlB200Router *r, float const *X, vl_size B, int const *tidx,
                            float const *tw, double *loss, float *grads) {
  return guarded([&] {
    cudaStream_t s = vlb::thread_stream();
    vlb::Scratch &sc = vlb::thread_scratch(vlb::kArenaRouter);
    const int L = nlayers(r);
    std::vector<float *> act(L + 1), gact(L + 1);
    for (int l = 0; l <= L; ++l) act[l] = sc.slot[l].get<float>((size_t)B * r->sizes[l]);
    for (int l = 1; l <= L; ++l) gact[l] = sc.slot[10 + l].get<float>((size_t)B * r->sizes[l]);
    double *rl = sc.slot[20].get<double>(B);
    double *tot = sc.slot[21].get<double>(1);
    forward(r, X, (i64)B, act, s);
    VLB_LAUNCH("router_xent", s,
               vlb::k_xent<8><<<vlb::gridn(B, 8), 256, 0, s>>>(act[L], (int)B, r->K, tidx, tw, gact[L], rl));
    for (int l = L - 1; l >= 0; --l) {
      const int in = r->sizes[l], out = r->sizes[l + 1];
      // dW = dY^T X  (out x in), summed over the batch in order.
      gemm(false, false, gact[l + 1], 1, out, act[l], 1, in, nullptr, (float *)r->gW[l]->p, in, out, in,
           (int)B, s);
      VLB_LAUNCH("router_colsum", s,
                 vlb::k_colsum<<<vlb::gridn(out, 256), 256, 0, s>>>(gact[l + 1], (int)B, out, (float *)r->gb[l]->p));
      if (l > 0) {
        // dX = dY W (B x in), then the ReLU mask of layer l's output.
        gemm(false, false, gact[l + 1], out, 1, (float *)r->Wq[l]->p, 1, in, nullptr, gact[l], in, (int)B,
             in, out, s);
        VLB_LAUNCH("router_relu_mask", s,
                   vlb::k_relu_mask<<<vlb::gridn((i64)B * in, 256), 256, 0, s>>>(gact[l], act[l], (i64)B * in));
      }
    }
    vlb::sum_doubles(rl, (i64)B, tot, s);
    double h = 0;
    VLB_CUDA(cudaMemcpyAsync(&h, tot, sizeof(double), cudaMemcpyDeviceToHost, s));
    if (grads) {
      size_t o = 0;
      for (int l = 0; l < L; ++l) {
        const size_t nw = (size_t)r->sizes[l + 1] * r->sizes[l], nb = r->sizes[l + 1];
        VLB_CUDA(cudaMemcpyAsync(grads + o, r->gW[l]->p, nw * 4, cudaMemcpyDeviceToHost, s));
        o += nw;
        VLB_CUDA(cudaMemcpyAsync(grads + o, r->gb[l]->p, nb * 4, cudaMemcpyDeviceToHost, s));
        o += nb;
      }
    }
    VLB_CUDA(cudaStreamSynchronize(s));
    if (loss) *loss = h / (double)B;
  });
}

// Top-8 targets (indices, renormalised weights) of N posterior rows (device).
int vlb200_router_targets(float const *posteriors, vl_size N, vl_size K, int *tidx, float *tw) {
  return guarded([&] {
    cudaStream_t s = vlb::thread_stream();
    VLB_LAUNCH("router_targets", s,
               vlb::k_topk_targets<8><<<vlb::gridn(N, 8), 256, 0, s>>>(posteriors, (i64)N, (int)K, tidx, tw));
    VLB_CUDA(cudaStreamSynchronize(s));
  });
}

// Trains the router with Adam on descriptors X (device, N x D) and top-8
// targets (device, N x 8) for `epochs` passes in batches of `batch` rows (in
// order; the caller shuffles).  *loss: mean loss of the last epoch.
int vlb200_router_train(VlB200Router *r, float const *X, vl_size N, int const *tidx, float const *tw,
                        vl_size epochs, vl_size batch, float lr, double *loss) {
  return guarded([&] {
    cudaStream_t s = vlb::thread_stream();
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    double last = 0;
    for (vl_size ep = 0; ep < epochs; ++ep) {
      double acc = 0;
      vl_size nb = 0;
      for (vl_size i0 = 0; i0 + batch <= N; i0 += batch, ++nb) {
        double l = 0;
        if (vlb200_router_loss_grad(r, X + i0 * r->D, batch, tidx + i0 * 8, tw + i0 * 8, &l, nullptr))
          throw vlb::Error(vl_get_last_error(), vl_get_last_error_message());
        acc += l;
        r->step++;
        const float c1 = 1.f - std::pow(b1, (float)r->step), c2 = 1.f - std::pow(b2, (float)r->step);
        for (int l2 = 0; l2 < nlayers(r); ++l2) {
          const i64 nw = (i64)r->sizes[l2 + 1] * r->sizes[l2], nbb = r->sizes[l2 + 1];
          VLB_LAUNCH("router_adam", s,
                     vlb::k_adam<<<vlb::gridn(nw, 256), 256, 0, s>>>((float *)r->W[l2]->p, (float *)r->gW[l2]->p,
                                                                    (float *)r->mW[l2]->p, (float *)r->vW[l2]->p,
                                                                    nw, lr, b1, b2, eps, c1, c2));
          VLB_LAUNCH("router_adam", s,
                     vlb::k_adam<<<vlb::gridn(nbb, 256), 256, 0, s>>>((float *)r->b[l2]->p, (float *)r->gb[l2]->p,
                                                                     (float *)r->mb[l2]->p, (float *)r->vb[l2]->p,
                                                                     nbb, lr, b1, b2, eps, c1, c2));
        }
        refresh_bf16(r, s);
      }
      last = nb ? acc / (double)nb : 0.0;
    }
    VLB_CUDA(cudaStreamSynchronize(s));
    if (loss) *loss = last;
  });
}

// Router E-step: posteriors (device, N x K, dense with zeros off the
// candidates) from the exact evaluation of the top-m candidates, with the
// full E-step for rows whose predicted candidate mass is below `threshold`.
// fallbackRows (host, may be NULL) receives the number of fallback rows.
int vlb200_router_posteriors(VlB200Router *r, float *posteriors, float const *priors,
                             float const *means, float const *covariances, float const *X,
                             vl_size N, vl_size m, float threshold, vl_uint64 *fallbackRows,
                             void *stream) {
  return guarded([&] {
    VLB_CHECK(m >= 1 && m <= 32 && (int)m <= r->K, VL_ERR_BAD_ARG, "router: m must be in [1, 32]");
    VLB_CHECK(r->K <= 1024, VL_ERR_BAD_ARG, "router: at most 1024 components");
    cudaStream_t s = vlb::pick_stream(stream);
    vlb::Scratch &sc = vlb::thread_scratch(vlb::kArenaRouter);
    const int L = nlayers(r), K = r->K, D = r->D;
    vlb::DevModel<float> md;
    md.means = means; md.covs = covariances; md.priors = priors; md.K = K; md.D = D;
    vlb::DevDerived<float> der;
    der.inv = sc.slot[22].get<float>((size_t)K * D);
    der.sis = sc.slot[23].get<float>((size_t)K * D);
    der.cst = sc.slot[24].get<double>(K);
    vlb::exact_prepare(md, der, s);
    const i64 chunk = infer_chunk(r);
    unsigned long long nfb = 0;
    for (i64 i0 = 0; i0 < (i64)N; i0 += chunk) {
      const i64 B = std::min<i64>(chunk, (i64)N - i0);
      std::vector<float *> act = infer_buffers(r, sc, chunk);
      int *cand = sc.slot[25].get<int>((size_t)chunk * m);
      float *cm = sc.slot[26].get<float>(chunk);
      unsigned char *fell = sc.slot[27].get<unsigned char>(chunk);
      if (!forward_infer(r, X + i0 * D, B, act, sc, s, (int)m, cand, cm)) {
        if (K <= 256)
          VLB_LAUNCH("router_select", s,
                     vlb::k_select<8><<<vlb::gridn(B, 8), 256, 0, s>>>(act[L], B, K, (int)m, cand, cm));
        else if (K <= 512)
          VLB_LAUNCH("router_select", s,
                     vlb::k_select<16><<<vlb::gridn(B, 8), 256, 0, s>>>(act[L], B, K, (int)m, cand, cm));
        else
          VLB_LAUNCH("router_select", s,
                     vlb::k_select<32><<<vlb::gridn(B, 8), 256, 0, s>>>(act[L], B, K, (int)m, cand, cm));
      }
      const bool tcfb = vlb::tc_supported_padded(K, D);
      VLB_LAUNCH("router_candidate_estep", s,
                 vlb::k_candidate_estep<<<vlb::gridn(B, 8), 256, 0, s>>>(
                     X + i0 * D, B, D, K, means, der.inv, der.cst, cand, cm, (int)m, threshold,
                     posteriors + i0 * K, fell, nullptr, tcfb));
      if (tcfb) {
        vlb::tc_fallback(X + i0 * D, B, md, fell, posteriors + i0 * K, &nfb, s);
      } else if (fallbackRows) {
        std::vector<unsigned char> h(B);
        VLB_CUDA(cudaMemcpyAsync(h.data(), fell, B, cudaMemcpyDeviceToHost, s));
        VLB_CUDA(cudaStreamSynchronize(s));
        for (auto v : h) nfb += v;
      }
    }
    if (fallbackRows) *fallbackRows = nfb;
  });
}

// Inference engine of the router: 1 = tcgen05 dense layers (default, when
// every width allows), 0 = the training forward on the CUDA cores.
int vlb200_router_set_tensor_core_inference(VlB200Router *r, int on) {
  return guarded([&] { r->tcInfer = on != 0; });
}

// Top-m candidates (N x m int) and their predicted softmax mass (N float) of
// rows X, all device arrays.  fused: selected in the last dense layer's
// epilogue when that applies, else by the selection kernel on the logits.
int vlb200_router_candidates(VlB200Router *r, float const *X, vl_size N, vl_size m, int *cand, float *cmass,
                             int fused, void *stream) {
  return guarded([&] {
    VLB_CHECK(m >= 1 && m <= 32 && (int)m <= r->K, VL_ERR_BAD_ARG, "router: m must be in [1, 32]");
    VLB_CHECK(r->K <= 1024, VL_ERR_BAD_ARG, "router: at most 1024 components");
    cudaStream_t s = vlb::pick_stream(stream);
    vlb::Scratch &sc = vlb::thread_scratch(vlb::kArenaRouter);
    const int L = nlayers(r), K = r->K;
    const i64 chunk = infer_chunk(r);
    for (i64 i0 = 0; i0 < (i64)N; i0 += chunk) {
      const i64 B = std::min<i64>(chunk, (i64)N - i0);
      std::vector<float *> act = infer_buffers(r, sc, chunk);
      int *c = cand + i0 * m;
      float *cm = cmass + i0;
      if (!forward_infer(r, X + i0 * r->D, B, act, sc, s, fused ? (int)m : 0, c, cm)) {
        if (K <= 256)
          VLB_LAUNCH("router_select", s, vlb::k_select<8><<<vlb::gridn(B, 8), 256, 0, s>>>(act[L], B, K, (int)m, c, cm));
        else if (K <= 512)
          VLB_LAUNCH("router_select", s, vlb::k_select<16><<<vlb::gridn(B, 8), 256, 0, s>>>(act[L], B, K, (int)m, c, cm));
        else
          VLB_LAUNCH("router_select", s, vlb::k_select<32><<<vlb::gridn(B, 8), 256, 0, s>>>(act[L], B, K, (int)m, c, cm));
      }
    }
    VLB_CUDA(cudaStreamSynchronize(s));
  });
}

// Inference logits (N x K, fp32, device) of the rows X (N x D, device).
int vlb200_router_logits(VlB200Router *r, float const *X, vl_size N, float *logits, void *stream) {
  return guarded([&] {
    cudaStream_t s = vlb::pick_stream(stream);
    vlb::Scratch &sc = vlb::thread_scratch(vlb::kArenaRouter);
    const int L = nlayers(r);
    const i64 chunk = 1 << 17;
    for (i64 i0 = 0; i0 < (i64)N; i0 += chunk) {
      const i64 B = std::min<i64>(chunk, (i64)N - i0);
      std::vector<float *> act(L + 1);
      for (int l = 0; l < L; ++l) act[l] = sc.slot[l].get<float>((size_t)chunk * r->sizes[l]);
      act[L] = logits + i0 * r->K;
      forward_infer(r, X + i0 * r->D, B, act, sc, s);
    }
    VLB_CUDA(cudaStreamSynchronize(s));
  });
}

// Mean missed posterior mass of candidate posteriors qc against the full
// E-step posteriors qfull (both device, N x K).
int vlb200_router_missed_mass(float const *qfull, float const *qc, vl_size N, vl_size K, double *mean) {
  return guarded([&] {
    cudaStream_t s = vlb::thread_stream();
    vlb::Scratch &sc = vlb::thread_scratch(vlb::kArenaRouter);
    double *rows = sc.slot[28].get<double>(N), *tot = sc.slot[29].get<double>(1);
    VLB_LAUNCH("router_missed", s,
               vlb::k_missed<<<vlb::gridn(N, 8), 256, 0, s>>>(qfull, qc, (i64)N, (int)K, rows));
    vlb::sum_doubles(rows, (i64)N, tot, s);
    double h = 0;
    VLB_CUDA(cudaMemcpyAsync(&h, tot, sizeof(double), cudaMemcpyDeviceToHost, s));
    VLB_CUDA(cudaStreamSynchronize(s));
    *mean = N ? h / (double)N : 0.0;
  });
}

}  // extern "C"

// ------------------------------------------------------ default router
namespace {
std::mutex g_default_mu;
VlB200Router *g_default = nullptr;
vl_size g_default_m = 8;
float g_default_thr = 0.99f;
}  // namespace

extern "C" int vlb200_router_set_default(VlB200Router *router, vl_size m, float threshold) {
  if (router && (m < 1 || m > 32))
    return vl_set_last_error(VL_ERR_BAD_ARG, "vlb200_router_set_default: m must be in [1, 32]");
  std::lock_guard<std::mutex> lk(g_default_mu);
  g_default = router;
  g_default_m = m;
  g_default_thr = threshold;
  return 0;
}

namespace vlb {
// The rows that fell back (fell[i] = 1) go through the tensor-core E-step
// together: their indices listed in row order, the rows gathered into one
// block, their posteriors computed there (fp16x3 split, FP32-grade, every
// component), and scattered back into q.  Returns their log-likelihood and
// adds their count to *nfb.
double tc_fallback(const float *X, i64 B, const DevModel<float> &m, const unsigned char *fell, float *q,
                   unsigned long long *nfb, cudaStream_t s) {
  Scratch &sc = thread_scratch(kArenaRouterTc);
  const int K = (int)m.K, D = (int)m.D;
  const int nb = (int)((B + 1023) / 1024);
  int *counts = sc.slot[25].get<int>((size_t)nb + 1);
  int *idx = sc.slot[26].get<int>((size_t)B);
  VLB_LAUNCH("router_fallback_list", s, k_fb_count<<<nb, 1024, 0, s>>>(fell, B, counts));
  VLB_LAUNCH("router_fallback_list", s, k_fb_scan<<<1, 32, 0, s>>>(counts, nb, counts + nb));
  VLB_LAUNCH("router_fallback_list", s, k_fb_scatter<<<nb, 1024, 0, s>>>(fell, B, counts, idx));
  int cnt = 0;
  VLB_CUDA(cudaMemcpyAsync(&cnt, counts + nb, sizeof(int), cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaStreamSynchronize(s));
  if (nfb) *nfb += (unsigned long long)cnt;
  if (cnt == 0) return 0.0;
  float *xg = sc.slot[27].get<float>((size_t)cnt * D);
  float *qg = sc.slot[28].get<float>((size_t)cnt * K);
  double *llp = sc.slot[29].get<double>(estep_ll_parts(cnt));
  double *tot = sc.slot[30].get<double>(1);
  VLB_LAUNCH("router_fallback_gather", s,
             k_rows_gather<<<gridn((i64)cnt * D, 256), 256, 0, s>>>(X, idx, cnt, D, xg, false));
  const i64 np = tc_estep(xg, cnt, m, qg, llp, false, VLB200_PREC_FP32, s, &sc);
  sum_doubles(llp, np, tot, s);
  VLB_LAUNCH("router_fallback_scatter", s,
             k_rows_gather<<<gridn((i64)cnt * K, 256), 256, 0, s>>>(qg, idx, cnt, K, q, true));
  double h = 0;
  VLB_CUDA(cudaMemcpyAsync(&h, tot, sizeof(double), cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaStreamSynchronize(s));
  return h;
}

// Router E-step of n rows for streamed EM: posteriors q (n x K, zeros off the
// candidates), the rows' log-likelihood over the evaluated components
// (returned), and the number of rows that fell back to the full E-step.
double router_estep(VlB200Router *r, const float *X, i64 n, const DevModel<float> &m, float *q,
                    size_t mcand, float thr, unsigned long long *fallback, cudaStream_t s) {
  VLB_CHECK(r->K == m.K && r->D == m.D, VL_ERR_BAD_ARG, "router does not match the model's K and D");
  VLB_CHECK(mcand >= 1 && mcand <= 32 && (int)mcand <= r->K, VL_ERR_BAD_ARG, "router: m must be in [1, 32]");
  VLB_CHECK(r->K <= 1024, VL_ERR_BAD_ARG, "router: at most 1024 components");
  Scratch &sc = thread_scratch(kArenaRouter);
  const int L = nlayers(r), K = r->K, D = r->D;
  DevDerived<float> der;
  der.inv = sc.slot[22].get<float>((size_t)K * D);
  der.sis = sc.slot[23].get<float>((size_t)K * D);
  der.cst = sc.slot[24].get<double>(K);
  exact_prepare(m, der, s);
  const i64 chunk = infer_chunk(r);
  double ll = 0;
  unsigned long long nfb = 0;
  for (i64 i0 = 0; i0 < n; i0 += chunk) {
    const i64 B = std::min<i64>(chunk, n - i0);
    std::vector<float *> act = infer_buffers(r, sc, chunk);
    int *cand = sc.slot[25].get<int>((size_t)chunk * mcand);
    float *cm = sc.slot[26].get<float>(chunk);
    unsigned char *fell = sc.slot[27].get<unsigned char>(chunk);
    double *llrow = sc.slot[28].get<double>(chunk);
    double *llsum = sc.slot[29].get<double>(1);
    if (!forward_infer(r, X + i0 * D, B, act, sc, s, (int)mcand, cand, cm)) {
      if (K <= 256)
        VLB_LAUNCH("router_select", s, k_select<8><<<gridn(B, 8), 256, 0, s>>>(act[L], B, K, (int)mcand, cand, cm));
      else if (K <= 512)
        VLB_LAUNCH("router_select", s, k_select<16><<<gridn(B, 8), 256, 0, s>>>(act[L], B, K, (int)mcand, cand, cm));
      else
        VLB_LAUNCH("router_select", s, k_select<32><<<gridn(B, 8), 256, 0, s>>>(act[L], B, K, (int)mcand, cand, cm));
    }
    const bool tcfb = tc_supported_padded(K, D);
    VLB_LAUNCH("router_candidate_estep", s,
               k_candidate_estep<<<gridn(B, 8), 256, 0, s>>>(X + i0 * D, B, D, K, m.means, der.inv, der.cst, cand,
                                                             cm, (int)mcand, thr, q + i0 * K, fell, llrow, tcfb));
    sum_doubles(llrow, B, llsum, s);
    double h = 0;
    VLB_CUDA(cudaMemcpyAsync(&h, llsum, sizeof(double), cudaMemcpyDeviceToHost, s));
    VLB_CUDA(cudaStreamSynchronize(s));
    ll += h;
    if (tcfb) {
      ll += tc_fallback(X + i0 * D, B, m, fell, q + i0 * K, &nfb, s);
    } else {
      std::vector<unsigned char> hf(B);
      VLB_CUDA(cudaMemcpyAsync(hf.data(), fell, B, cudaMemcpyDeviceToHost, s));
      VLB_CUDA(cudaStreamSynchronize(s));
      for (auto v : hf) nfb += v;
    }
  }
  if (fallback) *fallback += nfb;
  return ll;
}

// Sum over n rows of the posterior mass of qfull that qc leaves out.
double router_missed_sum(const float *qfull, const float *qc, i64 n, i64 K, cudaStream_t s) {
  if (n <= 0) return 0.0;
  Scratch &sc = thread_scratch(kArenaRouter);
  double *rows = sc.slot[30].get<double>(n), *tot = sc.slot[31].get<double>(1);
  VLB_LAUNCH("router_missed", s, k_missed<<<gridn(n, 8), 256, 0, s>>>(qfull, qc, n, (int)K, rows));
  sum_doubles(rows, n, tot, s);
  double h = 0;
  VLB_CUDA(cudaMemcpyAsync(&h, tot, sizeof(double), cudaMemcpyDeviceToHost, s));
  VLB_CUDA(cudaStreamSynchronize(s));
  return h;
}

// Top-8 targets of full-E-step posteriors q (n x K) and `epochs` epochs of
// training on them (batch 1024, Adam).
void router_fit(VlB200Router *r, const float *X, i64 n, const float *q, int epochs, float lr, cudaStream_t s) {
  if (n <= 0 || epochs <= 0) return;
  DevBuf ti, tw;
  int *tidx = ti.get<int>((size_t)n * 8);
  float *twt = tw.get<float>((size_t)n * 8);
  VLB_CUDA(cudaStreamSynchronize(s));
  if (vlb200_router_targets(q, (vl_size)n, (vl_size)r->K, tidx, twt))
    throw Error(vl_get_last_error(), vl_get_last_error_message());
  double loss = 0;
  if (vlb200_router_train(r, X, (vl_size)n, tidx, twt, (vl_size)epochs, 1024, lr, &loss))
    throw Error(vl_get_last_error(), vl_get_last_error_message());
}

void router_default_posteriors(const float *X, i64 N, const DevModel<float> &m, float *q,
                               cudaStream_t s) {
  VlB200Router *r;
  vl_size mm;
  float thr;
  {
    std::lock_guard<std::mutex> lk(g_default_mu);
    r = g_default;
    mm = g_default_m;
    thr = g_default_thr;
  }
  VLB_CHECK(r != nullptr, VL_ERR_BAD_ARG,
            "VLB200_PREC_BF16_ROUTER: no router set (vlb200_router_set_default)");
  VLB_CHECK(r->K == m.K && r->D == m.D, VL_ERR_BAD_ARG, "router does not match the model's K and D");
  if (vlb200_router_posteriors(r, q, m.priors, m.means, m.covs, X, (vl_size)N, mm, thr, nullptr, s))
    throw Error(vl_get_last_error(), vl_get_last_error_message());
}
}  // namespace vlb
