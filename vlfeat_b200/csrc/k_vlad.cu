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
#include <vector>

#include "engine.h"

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
  const int img = blockIdx.x, k0 = blockIdx.y * kVladKT, tid = threadIdx.x;
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
  T *out = enc + (img0 + img) * (i64)K * D;
  for (int c = 0; c < nk; ++c) {
    for (int d = tid; d < D; d += kVladThreads) {
      T z = zs[c * D + d];
      if (flags & VL_VLAD_FLAG_NORMALIZE_COMPONENTS) z = div_t(z, s_norm[c]);
      out[(i64)(k0 + c) * D + d] = z;
    }
  }
}

// Global L2 of each image's KD values, summed in element order by one thread
// per image (vl/vlad.c:226-237).
template <typename T>
__global__ void k_vlad_global_norm(const T *__restrict__ enc, i64 KD, i64 nimg, T *__restrict__ norm) {
  const i64 img = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (img >= nimg) return;
  const T *e = enc + img * KD;
  T n = (T)0;
  for (i64 i = 0; i < KD; ++i) n = add_t(n, mul_t(e[i], e[i]));
  n = sqrt_t(n);
  norm[img] = (T)fmax((double)n, 1e-12);
}

template <typename T>
__global__ void k_vlad_scale(T *__restrict__ enc, i64 KD, i64 nimg, const T *__restrict__ norm) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= KD * nimg) return;
  enc[i] = div_t(enc[i], norm[i / KD]);
}

template <typename T, int JD>
void launch_accum(T *enc, const T *means, int D, int K, const T *X, const T *A, const i64 *doffs, i64 nimg,
                  int flags, cudaStream_t s) {
  const size_t smem = sizeof(T) * kVladKT * D;
  auto kern = k_vlad_accum<T, JD>;
  VLB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid((unsigned)nimg, (unsigned)((K + kVladKT - 1) / kVladKT));
  VLB_LAUNCH("vlad_accum", s, kern<<<grid, kVladThreads, smem, s>>>(enc, means, D, K, X, A, doffs, 0, flags));
}

}  // namespace

template <typename T>
void vlad_batch(T *enc, const T *means, i64 D, i64 K, const T *X, const T *A, const i64 *h_offsets, i64 nimg,
                int flags, cudaStream_t s) {
  VLB_CHECK(D >= 1 && K >= 1, VL_ERR_BAD_ARG, "VLAD: dimension and numClusters must be >= 1");
  VLB_CHECK(D <= 8 * kVladThreads, VL_ERR_BAD_ARG, "VLAD: dimension above 1024 is not supported");
  if (nimg <= 0) return;
  Scratch &sc = thread_scratch(kArenaVlad);
  std::vector<i64> rel(nimg + 1);
  for (i64 j = 0; j <= nimg; ++j) rel[j] = h_offsets[j];
  i64 *doffs = sc.slot[0].get<i64>(nimg + 1);
  VLB_CUDA(cudaMemcpyAsync(doffs, rel.data(), sizeof(i64) * (nimg + 1), cudaMemcpyHostToDevice, s));
  const int jd = (int)((D + kVladThreads - 1) / kVladThreads);
  if (jd <= 1) launch_accum<T, 1>(enc, means, (int)D, (int)K, X, A, doffs, nimg, flags, s);
  else if (jd <= 2) launch_accum<T, 2>(enc, means, (int)D, (int)K, X, A, doffs, nimg, flags, s);
  else if (jd <= 4) launch_accum<T, 4>(enc, means, (int)D, (int)K, X, A, doffs, nimg, flags, s);
  else launch_accum<T, 8>(enc, means, (int)D, (int)K, X, A, doffs, nimg, flags, s);
  if (!(flags & VL_VLAD_FLAG_UNNORMALIZED)) {
    T *norm = sc.slot[1].get<T>(nimg);
    const i64 KD = K * D;
    VLB_LAUNCH("vlad_global_norm", s,
               k_vlad_global_norm<T><<<(unsigned)((nimg + 127) / 128), 128, 0, s>>>(enc, KD, nimg, norm));
    VLB_LAUNCH("vlad_scale", s,
               k_vlad_scale<T><<<(unsigned)((KD * nimg + 255) / 256), 256, 0, s>>>(enc, KD, nimg, norm));
  }
  // The scratch above is reused by the next call on this thread, which may
  // use another stream: finish before returning.
  VLB_CUDA(cudaStreamSynchronize(s));
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
