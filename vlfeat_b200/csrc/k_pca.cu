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
