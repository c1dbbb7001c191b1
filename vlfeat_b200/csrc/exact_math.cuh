// Explicitly rounded arithmetic for the kernels that reproduce the reference's
// CPU arithmetic bit for bit (Rand and k-means initialisation).  Every sum runs
// in the data type and in the reference's order; multiplies and adds stay
// separate (these intrinsics never contract into a fused multiply-add), so the
// results are the reference's bits.
#pragma once
#include <cuda_runtime.h>

namespace vlb {

__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }

// Squared L2 distance in the order of the reference's kernel for VlDistanceL2
// (vl/mathop.c:472-513): L lanes accumulate (a - b)^2 over consecutive groups
// of L elements (lane l takes elements l, l + L, ...), the lanes are reduced
// in the fixed pattern of the SIMD horizontal sum, and the D mod L remaining
// elements are added in order.  L = 8 (AVX, float), 4 (AVX double or SSE2
// float: ((v0 + v2) + (v1 + v3))), 2 (SSE2 double), 1 (scalar).  Element i of
// a is a[i * as] (as = 1 for a contiguous row; a column of a transposed tile
// in shared memory otherwise).
template <typename T, int L>
__device__ __forceinline__ T l2_ordered_s(const T *__restrict__ a, int as, const T *__restrict__ b, int D) {
  T v[L];
#pragma unroll
  for (int l = 0; l < L; ++l) v[l] = (T)0;
  int i = 0;
  for (; i + L <= D; i += L) {
#pragma unroll
    for (int l = 0; l < L; ++l) {
      const T dl = sub_rn(a[(i + l) * as], b[i + l]);
      v[l] = add_rn(v[l], mul_rn(dl, dl));
    }
  }
  T acc;
  if constexpr (L == 8) {
    acc = add_rn(add_rn(add_rn(v[0], v[1]), add_rn(v[4], v[5])), add_rn(add_rn(v[2], v[3]), add_rn(v[6], v[7])));
  } else if constexpr (L == 4) {
    acc = add_rn(add_rn(v[0], v[2]), add_rn(v[1], v[3]));
  } else if constexpr (L == 2) {
    acc = add_rn(v[0], v[1]);
  } else {
    acc = v[0];
  }
  for (; i < D; ++i) {
    const T dl = sub_rn(a[i * as], b[i]);
    acc = add_rn(acc, mul_rn(dl, dl));
  }
  return acc;
}

template <typename T, int L>
__device__ __forceinline__ T l2_ordered(const T *__restrict__ a, const T *__restrict__ b, int D) {
  return l2_ordered_s<T, L>(a, 1, b, D);
}

}  // namespace vlb
