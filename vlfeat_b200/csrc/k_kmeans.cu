// VLFeat's KMeans initialisation of a GMM (VlGMMKMeans, vl/gmm.c:1315-1370):
// the k-means object the GMM creates for it runs random-selection seeding
// (vl/kmeans.c:528-582), ANN refinement over a one-tree kd-forest
// (vl/kmeans.c:1003-1150, vl/kdtree.c) and the exact final quantisation
// (vl/kmeans.c:656-702).  All data-sized work runs here on the GPU; the host
// keeps what is sequential by definition and K-sized:
//
//  - random draws come from the calling thread's MT19937 in the reference's
//    order: the seeding shuffle, then per refinement iteration the kd-tree's
//    draws, then one draw per empty centre;
//  - the kd-tree over the K centres is built on the host exactly as
//    vl/kdtree.c:165-325 and 491-576 build it (its shape decides the draws);
//  - each row's assignment: when the comparison budget covers every centre,
//    an exact brute-force screen settles every row whose nearest centre is
//    clear of the second by more than the distances' rounding (the search
//    must return that centre); the other rows, and every row when the budget
//    is smaller, get the reference's best-bin-first search (vl/kdtree.c:
//    583-725, 774-840) by one warp each, with the same heap discipline
//    (vl/heap-def.h), comparison budget and tie rules;
//  - distances use the summation order of the reference's SIMD kernel;
//  - a centre is the sum of its points in data order (a stable counting sort
//    by centre, then one block per centre adding its rows in order), divided
//    by its mass rounded to the data type (vl/kmeans.c:1078-1098).
//
// The energy (sum of the point distances, in double) is summed in a fixed
// parallel order instead of the reference's data order; it only steers the
// stopping tests and the choice between repetitions, and differs by rounding.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>

#include "engine.h"
#include "exact_math.cuh"
#include "tc_common.cuh"

extern "C" {
#include "vl/random.h"
}

namespace vlb {
namespace {

constexpr int kKmThreads = 256;
constexpr int kKmChunk = 4096;       // rows per chunk of the stable counting sort
constexpr int kKmEnergyBlocks = 592; // fixed: the energy's summation order
constexpr i64 kKdSampleCap = 1024;   // VL_KDTREE_VARIANCE_EST_NUM_SAMPLES, vl/kdtree.h:21
constexpr size_t kHeapBudget = size_t(1) << 30;  // bytes of search heaps on the device

int num_sms() {
  int dev = 0, n = 0;
  VLB_CUDA(cudaGetDevice(&dev));
  VLB_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  return n > 0 ? n : 1;
}

int blocks_for(i64 n, int t) { return (int)std::max<i64>(1, std::min<i64>((n + t - 1) / t, 1 << 30)); }

// ---------------------------------------------------------------- kd-tree
// Index entry of a node's range, laid out as VlKDTreeDataIndexEntry
// (vl/kdtree.h:46-50) so that the C library's qsort sees the same array and
// comparison results as in the reference and orders equal values alike.
struct KdEntry {
  i64 index;
  double value;
};

struct KdNode {
  i64 lowerChild = 0, upperChild = 0;  // < 0: leaf over entries [-lower-1, -upper-1)
  unsigned splitDimension = 0;
  double splitThreshold = 0, lowerBound = 0, upperBound = 0;
};

int kd_compare(const void *a, const void *b) {  // vl/kdtree.c:143-152
  const double delta = ((const KdEntry *)a)->value - ((const KdEntry *)b)->value;
  if (delta < 0) return -1;
  if (delta > 0) return +1;
  return 0;
}

// One tree of a forest with numTrees = 1 (so the split heap keeps a single
// dimension, vl/kdtree.c:349) and median thresholds (vl/kmeans.c:725).
template <typename T>
struct KdBuilder {
  const T *data;
  i64 D;
  VlRand *rand;
  std::vector<KdNode> nodes;
  std::vector<KdEntry> entries;

  i64 new_node() {
    nodes.emplace_back();
    return (i64)nodes.size() - 1;
  }

  // vl/kdtree.c:165-325.
  void build(i64 n, i64 begin, i64 end) {
    if (end - begin <= 1) {
      nodes[n].lowerChild = -begin - 1;
      nodes[n].upperChild = -end - 1;
      return;
    }
    bool have = false;
    unsigned bestDim = 0;
    double bestVar = 0;
    for (i64 d = 0; d < D; ++d) {
      double mean = 0, second = 0;
      i64 ns = kKdSampleCap;
      bool all = false;
      if (end - begin <= kKdSampleCap) {
        all = true;
        ns = end - begin;
      }
      for (i64 i = 0; i < ns; ++i) {
        vl_uint32 si = all ? (vl_uint32)i : (vl_rand_uint32(rand) % (vl_uint32)kKdSampleCap);
        const i64 di = entries[(size_t)(si + begin)].index;
        const double datum = (double)data[di * D + d];
        mean += datum;
        second += datum * datum;
      }
      mean /= (double)ns;
      second /= (double)ns;
      const double var = second - mean * mean;
      if (var <= 0) continue;
      if (!have || bestVar < var) {
        have = true;
        bestDim = (unsigned)d;
        bestVar = var;
      }
    }
    if (!have) {  // every sampled dimension constant: one leaf for the range
      nodes[n].lowerChild = -begin - 1;
      nodes[n].upperChild = -end - 1;
      return;
    }
    (void)vl_rand_uint32(rand);  // the dice among the kept dimensions (one: % 1)
    nodes[n].splitDimension = bestDim;
    for (i64 i = begin; i < end; ++i)
      entries[(size_t)i].value = (double)data[entries[(size_t)i].index * D + bestDim];
    qsort(entries.data() + begin, (size_t)(end - begin), sizeof(KdEntry), kd_compare);
    const i64 median = (begin + end - 1) / 2;
    nodes[n].splitThreshold = entries[(size_t)median].value;
    const i64 lc = new_node();
    nodes[n].lowerChild = lc;
    build(lc, begin, median + 1);
    const i64 uc = new_node();
    nodes[n].upperChild = uc;
    build(uc, median + 1, end);
  }

  // vl/kdtree.c:491-513.
  void bounds(i64 n, std::vector<double> &sb) {
    const unsigned i = nodes[n].splitDimension;
    const double t = nodes[n].splitThreshold;
    nodes[n].lowerBound = sb[2 * i + 0];
    nodes[n].upperBound = sb[2 * i + 1];
    if (nodes[n].lowerChild > 0) {
      sb[2 * i + 1] = t;
      bounds(nodes[n].lowerChild, sb);
      sb[2 * i + 1] = nodes[n].upperBound;
    }
    if (nodes[n].upperChild > 0) {
      sb[2 * i + 0] = t;
      bounds(nodes[n].upperChild, sb);
      sb[2 * i + 0] = nodes[n].lowerBound;
    }
  }
};

// The tree on the device: node arrays and the centre index of each entry.
struct KdDev {
  const double *thr, *lb, *ub;
  const int *lower, *upper, *dim, *ent;
  int numNodes;
};

// ---------------------------------------------------------------- kernels
// Loads rows [base, base + TB) of X into the block's transposed tile
// sq[d * (TB + 1) + r] (row r's element d): each thread reads its row with
// stride TB + 1, and both the warp's reads and the tile's stores hit
// distinct banks.
template <typename T>
__device__ __forceinline__ void load_rows(const T *__restrict__ X, i64 N, int D, i64 base, T *sq) {
  const int TB = blockDim.x;
  const i64 rows = min((i64)TB, N - base);
  const T *src = X + base * D;
  for (i64 e = threadIdx.x; e < rows * D; e += TB) {
    const i64 r = e / D;
    const int d = (int)(e - r * D);
    sq[(i64)d * (TB + 1) + r] = src[e];
  }
}

__host__ __device__ constexpr size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

template <typename T, int L>
__device__ __forceinline__ T lane_sum(const T *v) {  // the SIMD horizontal sum of l2_ordered_s
  if constexpr (L == 8) {
    return add_rn(add_rn(add_rn(v[0], v[1]), add_rn(v[4], v[5])), add_rn(add_rn(v[2], v[3]), add_rn(v[6], v[7])));
  } else if constexpr (L == 4) {
    return add_rn(add_rn(v[0], v[2]), add_rn(v[1], v[3]));
  } else if constexpr (L == 2) {
    return add_rn(v[0], v[1]);
  } else {
    return v[0];
  }
}

enum : int { kNearestQuantize = 0, kNearestScreen = 1 };

// Every distance of a row to the K centres, each in the reference's order
// (l2_ordered_s), with a register tile of TC centres sharing each lane group
// of the query.
//
// kNearestQuantize: exact quantisation, vl/kmeans.c:656-702: the first centre
// of least distance (strict <, from +inf; rows whose distances are all NaN
// keep centre 0, where the reference leaves the assignment unset).
//
// kNearestScreen: the ANN assignment (vl/kmeans.c:708-771) when the search
// budget covers every centre (K <= maxNumComparisons, one tree): the search
// is then exhaustive up to pruning by exact lower bounds, so when the least
// distance is below every other by more than the distances' rounding
// (margin, relative) the search returns that centre; such rows are assigned
// here (with the update rule: keep the previous centre unless strictly
// farther).  Rows with a near tie, a NaN or an infinite distance go to the
// row list for the kd-tree search itself.
template <typename T, int L, bool VEC, int TC>
__global__ void k_km_nearest(const T *__restrict__ X, i64 N, int D, const T *__restrict__ C, int K, int KC,
                             int mode, int update, uint32_t *__restrict__ assign, T *__restrict__ dist, T margin,
                             uint32_t *__restrict__ list, unsigned long long *__restrict__ count) {
  extern __shared__ __align__(16) unsigned char km_smem[];
  const int TB = blockDim.x;
  const int QS = TB + 1;
  T *sq = (T *)km_smem;
  T *sc = (T *)(km_smem + align16(sizeof(T) * (size_t)QS * D));  // KC centre rows
  const i64 G = (i64)gridDim.x * TB;
  for (i64 base = (i64)blockIdx.x * TB; base < N; base += G) {
    __syncthreads();
    load_rows(X, N, D, base, sq);
    const i64 x = base + threadIdx.x;
    const bool active = x < N;
    const T *q = sq + threadIdx.x;
    const uint32_t pa = (active && mode == kNearestScreen && update) ? assign[x] : 0xffffffffu;
    T best = (T)INFINITY, second = (T)INFINITY, prevd = (T)0;
    uint32_t bi = 0;
    bool nan = false;
    for (int k0 = 0; k0 < K; k0 += KC) {
      // The next KC centres into shared memory (every thread reads the same
      // centre element at a time: broadcast loads).
      const int kn = min(KC, K - k0);
      __syncthreads();
      if constexpr (VEC) {
        const float4 *src = reinterpret_cast<const float4 *>(C + (i64)k0 * D);
        float4 *dst = reinterpret_cast<float4 *>(sc);
        const int n4 = (int)((size_t)kn * D * sizeof(T) / 16);
        for (int e = threadIdx.x; e < n4; e += TB) dst[e] = __ldg(src + e);
      } else {
        for (int e = threadIdx.x; e < kn * D; e += TB) sc[e] = __ldg(C + (i64)k0 * D + e);
      }
      __syncthreads();
      if (!active) continue;
      for (int c0 = 0; c0 < kn; c0 += TC) {
        T acc[TC][L];
#pragma unroll
        for (int t = 0; t < TC; ++t)
#pragma unroll
          for (int l = 0; l < L; ++l) acc[t][l] = (T)0;
        int i = 0;
        if constexpr (sizeof(T) == 4 && L % 2 == 0) {
          // Packed fp32x2: lanes l and l + 1 of the lane sums in one
          // instruction each for the difference, the square and the sum,
          // every half rounded exactly as the scalar operation.
          constexpr unsigned long long kNeg = 0x8000000080000000ull;
          unsigned long long ap[TC][L / 2];
#pragma unroll
          for (int t = 0; t < TC; ++t)
#pragma unroll
            for (int l = 0; l < L / 2; ++l) ap[t][l] = 0ull;
          for (; i + L <= D; i += L) {
            unsigned long long qn[L / 2];  // -q, pairs
#pragma unroll
            for (int l = 0; l < L / 2; ++l) qn[l] = tc::f2u(q[(i + 2 * l) * QS], q[(i + 2 * l + 1) * QS]) ^ kNeg;
#pragma unroll
            for (int t = 0; t < TC; ++t) {
              const float *cr = (const float *)sc + (size_t)min(c0 + t, kn - 1) * D + i;
              unsigned long long cp[L / 2];
              if constexpr (VEC && L % 4 == 0) {
#pragma unroll
                for (int u = 0; u < L / 4; ++u) {
                  const ulonglong2 w = reinterpret_cast<const ulonglong2 *>(cr)[u];
                  cp[2 * u] = w.x;
                  cp[2 * u + 1] = w.y;
                }
              } else {
#pragma unroll
                for (int l = 0; l < L / 2; ++l) cp[l] = tc::f2u(cr[2 * l], cr[2 * l + 1]);
              }
#pragma unroll
              for (int l = 0; l < L / 2; ++l) {
                const unsigned long long dl = tc::add2(cp[l], qn[l]);  // c - q: squared alike
                ap[t][l] = tc::add2(ap[t][l], tc::mul2(dl, dl));
              }
            }
          }
#pragma unroll
          for (int t = 0; t < TC; ++t)
#pragma unroll
            for (int l = 0; l < L / 2; ++l) {
              acc[t][2 * l] = (T)tc::lo32(ap[t][l]);
              acc[t][2 * l + 1] = (T)tc::hi32(ap[t][l]);
            }
        } else {
          for (; i + L <= D; i += L) {
            T qv[L];
#pragma unroll
            for (int l = 0; l < L; ++l) qv[l] = q[(i + l) * QS];
#pragma unroll
            for (int t = 0; t < TC; ++t) {
              const T *cr = sc + (size_t)min(c0 + t, kn - 1) * D + i;  // a partial tile repeats the last row
              T cg[L];
              if constexpr (VEC && (L * sizeof(T)) % 16 == 0) {
                constexpr int V = 16 / sizeof(T);
#pragma unroll
                for (int u = 0; u < L / V; ++u) {
                  const float4 w = reinterpret_cast<const float4 *>(cr)[u];
                  const T *wp = reinterpret_cast<const T *>(&w);
#pragma unroll
                  for (int e = 0; e < V; ++e) cg[u * V + e] = wp[e];
                }
              } else {
#pragma unroll
                for (int l = 0; l < L; ++l) cg[l] = cr[l];
              }
#pragma unroll
              for (int l = 0; l < L; ++l) {
                const T dl = sub_rn(qv[l], cg[l]);
                acc[t][l] = add_rn(acc[t][l], mul_rn(dl, dl));
              }
            }
          }
        }
#pragma unroll
        for (int t = 0; t < TC; ++t) {
          const int cl = c0 + t;
          if (cl >= kn) break;
          const int c = k0 + cl;
          T d = lane_sum<T, L>(acc[t]);
          for (int j = i; j < D; ++j) {
            const T dl = sub_rn(q[j * QS], sc[(size_t)cl * D + j]);
            d = add_rn(d, mul_rn(dl, dl));
          }
          nan |= d != d;
          if ((uint32_t)c == pa) prevd = d;
          if (d < best) {
            second = best;
            best = d;
            bi = (uint32_t)c;
          } else if (d < second) {
            second = d;
          }
        }
      }
    }
    if (!active) continue;
    if (mode == kNearestQuantize) {
      assign[x] = bi;
      continue;
    }
    const bool clear = !nan && best != (T)INFINITY && (K == 1 || second - best > margin * second);
    if (!clear) {
      list[atomicAdd(count, 1ull)] = (uint32_t)x;
      continue;
    }
    if (!update || prevd > best) {
      dist[x] = best;
      assign[x] = bi;
    } else {
      dist[x] = prevd;
    }
  }
}

// Distance of query row q (shared memory) to centre row c in the reference's
// order, by one warp: lane l < L adds (q_i - c_i)^2 for i = l, l + L, ... in
// order (a warp load reads L consecutive elements), the L lane sums are
// gathered into every lane and reduced in the SIMD horizontal-sum pattern, and
// every lane adds the D mod L remaining elements in order.  Every lane returns
// the same value.
template <typename T, int L>
__device__ __forceinline__ T warp_row_dist(const T *q, const T *__restrict__ c, int D, int lane) {
  T a = (T)0;
  const int full = D / L * L;
  if (lane < L)
    for (int i = lane; i < full; i += L) {
      const T dl = sub_rn(q[i], __ldg(c + i));
      a = add_rn(a, mul_rn(dl, dl));
    }
  T v[L];
#pragma unroll
  for (int l = 0; l < L; ++l) v[l] = __shfl_sync(0xffffffffu, a, l);
  T d = lane_sum<T, L>(v);
  for (int i = full; i < D; ++i) {
    const T dl = sub_rn(q[i], __ldg(c + i));
    d = add_rn(d, mul_rn(dl, dl));
  }
  return d;
}

// One query of the forest by one warp, vl/kdtree.c:774-840 with numNeighbors
// = 1 and the recursion of vl/kdtree.c:583-725 unrolled into a loop.  Every
// lane follows the same path (the decisions depend only on values all lanes
// hold); lane 0 alone keeps the search heap (hk, hn: capacity cap = the
// tree's node count, which bounds the pushes of one query, each node being
// pushed at most once) and hands each popped entry to the warp.  Heap moves
// follow vl/heap-def.h: push sifts towards the root while strictly smaller,
// pop moves the last entry to the root and sifts it towards the smaller
// child (the right one on ties) while strictly larger.
template <typename T, int L>
__device__ int kd_query_warp(const T *q, const T *__restrict__ C, int D, const KdDev &tr, i64 maxComp,
                             double *__restrict__ hk, int *__restrict__ hn, int cap, double &bestOut,
                             int *__restrict__ err, int lane) {
  const bool exact = maxComp == 0;
  i64 comps = 0;
  int nh = 1;
  if (lane == 0) {
    hk[0] = 0.0;
    hn[0] = 0;
  }
  bool have = false;
  double best = 0.0;
  int bestIdx = 0;
  while (exact || comps < maxComp) {
    if (nh == 0) break;
    nh -= 1;
    double pk = 0.0;
    int pn = 0;
    if (lane == 0) {
      pk = hk[0];
      pn = hn[0];
      if (nh > 0) {
        const double lk = hk[nh];
        const int ln = hn[nh];
        int i = 0;
        if (nh > 1) {
          while (true) {
            const int l = 2 * i + 1, r = l + 1;
            if (l >= nh) break;
            const int c = (r >= nh) ? l : (hk[l] < hk[r] ? l : r);
            const double ck = hk[c];
            if (lk > ck) {
              hk[i] = ck;
              hn[i] = hn[c];
              i = c;
              if (r >= nh) break;  // a lone left child is the last entry: stop
            } else {
              break;
            }
          }
        }
        hk[i] = lk;
        hn[i] = ln;
      }
    }
    pk = __shfl_sync(0xffffffffu, pk, 0);
    pn = __shfl_sync(0xffffffffu, pn, 0);
    if (have && best < pk) break;  // no better neighbour can remain
    const double dist = pk;
    int n = pn;
    while (true) {
      const int lc = __ldg(tr.lower + n);
      if (lc < 0) {  // leaf
        const int b = -lc - 1, e = -__ldg(tr.upper + n) - 1;
        for (int it = b; it < e && (exact || comps < maxComp); ++it) {
          const int di = __ldg(tr.ent + it);
          const double dd = (double)warp_row_dist<T, L>(q, C + (i64)di * D, D, lane);
          ++comps;
          if (!have) {
            have = true;
            best = dd;
            bestIdx = di;
          } else if (best > dd) {
            best = dd;
            bestIdx = di;
          }
        }
        break;
      }
      const int up = __ldg(tr.upper + n);
      const double xv = (double)q[__ldg(tr.dim + n)];
      const double x1 = __ldg(tr.lb + n), x2 = __ldg(tr.thr + n), x3 = __ldg(tr.ub + n);
      double delta = __dsub_rn(xv, x2);
      double save = __dadd_rn(dist, __dmul_rn(delta, delta));
      int next, sv;
      if (xv <= x2) {
        next = lc;
        sv = up;
        if (xv <= x1) {
          delta = __dsub_rn(xv, x1);
          save = __dsub_rn(save, __dmul_rn(delta, delta));
        }
      } else {
        next = up;
        sv = lc;
        if (xv > x3) {
          delta = __dsub_rn(xv, x3);
          save = __dsub_rn(save, __dmul_rn(delta, delta));
        }
      }
      if (!have || best > save) {
        if (nh >= cap) {
          if (lane == 0) atomicOr(err, 1);  // cannot happen: pushes per query <= nodes
        } else {
          if (lane == 0) {
            int i = nh;
            while (i > 0) {
              const int p = (i - 1) / 2;
              const double pkk = hk[p];
              if (save < pkk) {
                hk[i] = pkk;
                hn[i] = hn[p];
                i = p;
              } else {
                break;
              }
            }
            hk[i] = save;
            hn[i] = sv;
          }
          ++nh;
        }
      }
      n = next;
    }
  }
  bestOut = best;
  return bestIdx;
}

// ANN assignment, vl/kmeans.c:708-771: the forest's nearest centre of each
// row; after the first iteration (update) the previous assignment is kept
// unless the new centre is strictly closer.  One warp per row, WPB warps per
// block; with a row list only rows list[0 .. count) are served.  SH: each
// warp's query row and search heap live in shared memory, else the heap is
// the warp's slice of hkey / hnode.
template <typename T, int L, bool SH>
__global__ void k_km_ann(const T *__restrict__ X, i64 N, int D, const T *__restrict__ C, KdDev tr, i64 maxComp,
                         int update, uint32_t *__restrict__ assign, T *__restrict__ dist,
                         double *__restrict__ hkey, int *__restrict__ hnode, int cap, int *__restrict__ err,
                         const uint32_t *__restrict__ list, i64 count) {
  extern __shared__ __align__(16) unsigned char km_smem[];
  const int WPB = blockDim.x / 32, warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  // Each warp's region (query row, then heap keys and nodes) starts 16-byte aligned.
  const size_t per = align16(align16(sizeof(T) * (size_t)D) + (SH ? (size_t)cap * (sizeof(double) + sizeof(int)) : 0));
  unsigned char *mine = km_smem + per * warp;
  T *q = (T *)mine;
  const i64 gw = (i64)blockIdx.x * WPB + warp, GW = (i64)gridDim.x * WPB;
  double *hk;
  int *hn;
  if constexpr (SH) {
    hk = (double *)(mine + align16(sizeof(T) * (size_t)D));
    hn = (int *)(hk + cap);
  } else {
    hk = hkey + gw * cap;
    hn = hnode + gw * cap;
  }
  const i64 M = list ? count : N;
  for (i64 pidx = gw; pidx < M; pidx += GW) {
    const i64 x = list ? (i64)list[pidx] : pidx;
    __syncwarp();
    for (int d = lane; d < D; d += 32) q[d] = X[x * D + d];
    __syncwarp();
    double nd;
    const int ni = kd_query_warp<T, L>(q, C, D, tr, maxComp, hk, hn, cap, nd, err, lane);
    const T ndt = (T)nd;  // exact: the distance was computed in T
    if (!update) {
      if (lane == 0) {
        dist[x] = ndt;
        assign[x] = (uint32_t)ni;
      }
    } else {
      const T prev = warp_row_dist<T, L>(q, C + (i64)assign[x] * D, D, lane);
      if (lane == 0) {
        if (prev > ndt) {
          dist[x] = ndt;
          assign[x] = (uint32_t)ni;
        } else {
          dist[x] = prev;
        }
      }
    }
  }
}

// out[i] = X[rows[i]] for i < M.
template <typename T>
__global__ void k_km_gather(const T *__restrict__ X, int D, const i64 *__restrict__ rows, i64 M, T *__restrict__ out) {
  const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= M * D) return;
  const i64 i = e / D;
  const int d = (int)(e - i * D);
  out[e] = X[rows[i] * D + d];
}

// Duplicate test of the seeding (vl/kmeans.c:560-571): candidate i (row i of
// Cd) against every earlier pool row j < a + i, the pool being the a
// accepted centres A followed by the candidates.  Row j is a duplicate when
// its distance is 0, i.e. when every (x_d - y_d)^2 rounds to 0 (a sum of
// non-negative terms is 0 only then; NaN never is).  Bit j of bits[i * words
// + j / 32]; any[i] != 0 when row i has a duplicate.
template <typename T>
__global__ void k_km_dups(const T *__restrict__ A, i64 a, const T *__restrict__ Cd, i64 M, int D, int words,
                          uint32_t *__restrict__ bits, int *__restrict__ any) {
  const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= M * words) return;
  const i64 i = e / words;
  const int w = (int)(e - i * words);
  const T *xi = Cd + i * D;
  uint32_t mask = 0;
  for (int jj = 0; jj < 32; ++jj) {
    const i64 j = (i64)w * 32 + jj;
    if (j >= a + i) break;
    const T *y = j < a ? A + j * D : Cd + (j - a) * D;
    bool dup = true;
    for (int d = 0; d < D; ++d) {
      const T df = sub_rn(xi[d], y[d]);
      if (mul_rn(df, df) != (T)0) {
        dup = false;
        break;
      }
    }
    if (dup) mask |= 1u << jj;
  }
  bits[e] = mask;
  if (mask) atomicOr(any + i, 1);
}

// Energy partials: block b sums the distances of its grid-stride share in
// double, then a fixed tree; the order depends only on N.
template <typename T>
__global__ void k_km_energy(const T *__restrict__ dist, i64 N, double *__restrict__ part) {
  __shared__ double red[kKmThreads];
  double acc = 0;
  for (i64 x = (i64)blockIdx.x * kKmThreads + threadIdx.x; x < N; x += (i64)gridDim.x * kKmThreads)
    acc += (double)dist[x];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = kKmThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// Stable counting sort of the rows by centre.  (1) per chunk of kKmChunk rows
// the rows per centre, H[c * nb + b].
__global__ void k_km_hist(const uint32_t *__restrict__ assign, i64 N, int K, int nb, uint32_t *__restrict__ H) {
  extern __shared__ uint32_t km_hist[];
  for (int c = threadIdx.x; c < K; c += blockDim.x) km_hist[c] = 0;
  __syncthreads();
  const i64 beg = (i64)blockIdx.x * kKmChunk, end = min(N, beg + kKmChunk);
  for (i64 i = beg + threadIdx.x; i < end; i += blockDim.x) atomicAdd(&km_hist[assign[i]], 1u);
  __syncthreads();
  for (int c = threadIdx.x; c < K; c += blockDim.x) H[(i64)c * nb + blockIdx.x] = km_hist[c];
}

// (2) per centre: H becomes the exclusive prefix over chunks; count[c] the total.
__global__ void k_km_scan(uint32_t *__restrict__ H, int K, int nb, uint32_t *__restrict__ count) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= K) return;
  uint32_t run = 0;
  for (int b = 0; b < nb; ++b) {
    const uint32_t v = H[(i64)c * nb + b];
    H[(i64)c * nb + b] = run;
    run += v;
  }
  count[c] = run;
}

// (3) one warp per chunk walks its rows in order, 32 at a time: a row's slot
// is its centre's running base plus its rank among the earlier lanes with
// the same centre.  order[off[c] ...] lists centre c's rows increasing.
__global__ void k_km_scatter(const uint32_t *__restrict__ assign, i64 N, int K, int nb,
                             const uint32_t *__restrict__ H, const i64 *__restrict__ off,
                             uint32_t *__restrict__ order) {
  extern __shared__ i64 km_base[];
  const int lane = threadIdx.x;
  for (int c = lane; c < K; c += 32) km_base[c] = off[c] + (i64)H[(i64)c * nb + blockIdx.x];
  __syncwarp();
  const i64 beg = (i64)blockIdx.x * kKmChunk, end = min(N, beg + kKmChunk);
  for (i64 i0 = beg; i0 < end; i0 += 32) {
    const i64 i = i0 + lane;
    const bool ok = i < end;
    const uint32_t a = ok ? assign[i] : 0xffffffffu;
    const unsigned peers = __match_any_sync(0xffffffffu, a);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    i64 slot = 0;
    if (ok) slot = km_base[a] + rank;
    __syncwarp();
    if (ok) {
      order[slot] = (uint32_t)i;
      if (lane == 31 - __clz(peers)) km_base[a] += __popc(peers);
    }
    __syncwarp();
  }
}

// New centres, vl/kmeans.c:1078-1098: block c adds centre c's rows in data
// order from 0, thread t owning dimensions t, t + blockDim, ... (up to
// kSumDims per thread), then divides by the mass rounded to T.  The rows come
// through a shared-memory tile of R rows: the loads of the next tile (into
// registers) overlap the ordered additions of the current one.  Empty
// centres are left for the host's restarts.
constexpr int kSumThreads = 256;
constexpr int kSumDims = 4;          // D <= kSumThreads * kSumDims
constexpr int kSumTileElems = 2048;  // R * D <= this
constexpr int kSumPer = kSumTileElems / kSumThreads;

template <typename T>
__global__ void __launch_bounds__(kSumThreads) k_km_sums(const T *__restrict__ X, int D, int R,
                                                         const i64 *__restrict__ off,
                                                         const uint32_t *__restrict__ order, T *__restrict__ C) {
  __shared__ T tile[kSumTileElems];
  const int c = blockIdx.x;
  const i64 b = off[c], n = off[c + 1] - off[c];
  if (n == 0) return;
  const int t = threadIdx.x;
  T acc[kSumDims];
#pragma unroll
  for (int u = 0; u < kSumDims; ++u) acc[u] = (T)0;
  const int te = R * D;
  T nxt[kSumPer];
  auto fetch = [&](i64 j) {  // tile starting at segment position j, into registers
#pragma unroll
    for (int u = 0; u < kSumPer; ++u) {
      const int e = t + u * kSumThreads;
      const int r = e / D;
      nxt[u] = (e < te && j + r < n) ? __ldg(X + (i64)__ldg(order + b + j + r) * D + (e - r * D)) : (T)0;
    }
  };
  fetch(0);
  for (i64 j = 0; j < n; j += R) {
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kSumPer; ++u) {
      const int e = t + u * kSumThreads;
      if (e < te) tile[e] = nxt[u];
    }
    __syncthreads();
    if (j + R < n) fetch(j + R);
    const int rows = (int)min((i64)R, n - j);
#pragma unroll
    for (int u = 0; u < kSumDims; ++u) {
      const int d = t + u * kSumThreads;
      if (d < D)
        for (int r = 0; r < rows; ++r) acc[u] = add_rn(acc[u], tile[r * D + d]);
    }
  }
  const T m = (T)(unsigned long long)n;
#pragma unroll
  for (int u = 0; u < kSumDims; ++u) {
    const int d = t + u * kSumThreads;
    if (d < D) C[(i64)c * D + d] = div_rn(acc[u], m);
  }
}

template <typename T>
__global__ void k_km_onehot(const uint32_t *__restrict__ assign, i64 N, i64 K, T *__restrict__ q) {
  const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= N * K) return;
  const i64 x = e / K;
  q[e] = (T)((e - x * K) == (i64)assign[x] ? 1 : 0);
}

// ---------------------------------------------------------------- host side
template <typename T>
struct KMeansRun {
  const T *X;
  i64 N, D, K;
  int lanes;
  cudaStream_t s;
  Scratch &sc;
  VlRand *rand;

  // Rows per block of the row-tile kernels: the transposed tile of TB rows
  // must fit the shared memory this kernel may use.
  int tile_rows() const {
    for (int tb : {128, 64, 32})
      if ((size_t)(tb + 1) * D * sizeof(T) <= (size_t)96 * 1024) return tb;
    VLB_CHECK((size_t)33 * D * sizeof(T) <= (size_t)200 * 1024, VL_ERR_BAD_ARG,
              "k-means initialisation: dimension too large");
    return 32;
  }

  // Centre rows can be read in 16-byte vectors: every row start 16-byte
  // aligned and each lane group whole vectors.
  bool vec(int L) const { return (D * sizeof(T)) % 16 == 0 && (L * sizeof(T)) % 16 == 0; }

  template <template <typename, int> class Launch, typename... A>
  void by_lanes(A &&...a) {
    switch (lanes) {
      case 8: Launch<T, 8>::run(a...); break;
      case 4: Launch<T, 4>::run(a...); break;
      case 2: Launch<T, 2>::run(a...); break;
      default: Launch<T, 1>::run(a...); break;
    }
  }

  // Random selection of K distinct rows, vl/kmeans.c:528-582.
  void seed(T *centers) {
    std::vector<i64> perm((size_t)N);
    std::iota(perm.begin(), perm.end(), (i64)0);
    for (i64 n = N; n > 1;) {  // vl/shuffle-def.h:82-91
      const i64 k = (i64)vl_rand_uindex(rand, (vl_uindex)n);
      --n;
      std::swap(perm[(size_t)n], perm[(size_t)k]);
    }
    i64 k = 0, i = 0;
    while (k < K) {
      VLB_CHECK(i < N, VL_ERR_BAD_ARG, "k-means seeding ran out of rows");
      const i64 need = K - k;
      const i64 M = std::min<i64>(N - i, need + need / 8 + 32);
      const i64 a = k;
      const int words = (int)((a + M + 31) / 32);
      i64 *rows = sc.slot[0].get<i64>(M);
      T *cand = sc.slot[1].get<T>(M * D);
      uint32_t *bits = sc.slot[2].get<uint32_t>(M * words);
      int *any = sc.slot[3].get<int>(M);
      VLB_CUDA(cudaMemcpyAsync(rows, perm.data() + i, sizeof(i64) * M, cudaMemcpyHostToDevice, s));
      VLB_LAUNCH("km_gather", s, k_km_gather<T><<<blocks_for(M * D, kKmThreads), kKmThreads, 0, s>>>(
                                     X, (int)D, rows, M, cand));
      VLB_CUDA(cudaMemsetAsync(any, 0, sizeof(int) * M, s));
      VLB_LAUNCH("km_dups", s, k_km_dups<T><<<blocks_for(M * words, kKmThreads), kKmThreads, 0, s>>>(
                                   centers, a, cand, M, (int)D, words, bits, any));
      std::vector<int> hany((size_t)M);
      VLB_CUDA(cudaMemcpyAsync(hany.data(), any, sizeof(int) * M, cudaMemcpyDeviceToHost, s));
      VLB_CUDA(cudaStreamSynchronize(s));
      std::vector<uint32_t> hbits;
      if (std::any_of(hany.begin(), hany.end(), [](int v) { return v != 0; })) {
        hbits.resize((size_t)(M * words));
        VLB_CUDA(cudaMemcpyAsync(hbits.data(), bits, sizeof(uint32_t) * M * words, cudaMemcpyDeviceToHost, s));
        VLB_CUDA(cudaStreamSynchronize(s));
      }
      auto bit = [&](i64 t, i64 j) { return (hbits[(size_t)(t * words + j / 32)] >> (j % 32)) & 1u; };
      std::vector<i64> acc;  // accepted positions of this batch
      i64 t = 0;
      for (; t < M && k < K; ++t) {
        const i64 pos = i + t;
        if (K - k < N - pos && hany[(size_t)t]) {  // enough rows left to be choosy
          bool dup = false;
          for (i64 j = 0; j < a && !dup; ++j) dup = bit(t, j) != 0;
          for (size_t u = 0; u < acc.size() && !dup; ++u) dup = bit(t, a + acc[u]) != 0;
          if (dup) continue;
        }
        acc.push_back(t);
        ++k;
      }
      std::vector<i64> sel(acc.size());
      for (size_t u = 0; u < acc.size(); ++u) sel[u] = perm[(size_t)(i + acc[u])];
      if (!sel.empty()) {
        VLB_CUDA(cudaMemcpyAsync(rows, sel.data(), sizeof(i64) * sel.size(), cudaMemcpyHostToDevice, s));
        const i64 m = (i64)sel.size();
        VLB_LAUNCH("km_gather", s, k_km_gather<T><<<blocks_for(m * D, kKmThreads), kKmThreads, 0, s>>>(
                                       X, (int)D, rows, m, centers + a * D));
      }
      VLB_CUDA(cudaStreamSynchronize(s));  // rows and sel are reused next batch
      i += t;
    }
  }

  // Builds the tree over the current centres (reading them back), uploads
  // it and returns its device view.
  KdDev tree(const T *centers) {
    std::vector<T> hc((size_t)(K * D));
    VLB_CUDA(cudaMemcpyAsync(hc.data(), centers, sizeof(T) * K * D, cudaMemcpyDeviceToHost, s));
    VLB_CUDA(cudaStreamSynchronize(s));
    KdBuilder<T> b{hc.data(), D, rand, {}, {}};
    b.nodes.reserve((size_t)(2 * K));
    b.entries.resize((size_t)K);
    for (i64 k = 0; k < K; ++k) b.entries[(size_t)k] = KdEntry{k, 0.0};
    b.build(b.new_node(), 0, K);
    std::vector<double> sb((size_t)(2 * D));
    for (i64 d = 0; d < D; ++d) {
      sb[(size_t)(2 * d)] = -(double)INFINITY;
      sb[(size_t)(2 * d + 1)] = (double)INFINITY;
    }
    b.bounds(0, sb);
    const i64 nn = (i64)b.nodes.size();
    const size_t dbytes = sizeof(double) * 3 * nn;
    const size_t ibytes = sizeof(int) * (3 * nn + K);
    std::vector<unsigned char> pack(dbytes + ibytes);
    double *pd = (double *)pack.data();
    int *pi = (int *)(pack.data() + dbytes);
    for (i64 n = 0; n < nn; ++n) {
      pd[n] = b.nodes[(size_t)n].splitThreshold;
      pd[nn + n] = b.nodes[(size_t)n].lowerBound;
      pd[2 * nn + n] = b.nodes[(size_t)n].upperBound;
      pi[n] = (int)b.nodes[(size_t)n].lowerChild;
      pi[nn + n] = (int)b.nodes[(size_t)n].upperChild;
      pi[2 * nn + n] = (int)b.nodes[(size_t)n].splitDimension;
    }
    for (i64 k = 0; k < K; ++k) pi[3 * nn + k] = (int)b.entries[(size_t)k].index;
    unsigned char *dev = sc.slot[4].get<unsigned char>(pack.size());
    VLB_CUDA(cudaMemcpyAsync(dev, pack.data(), pack.size(), cudaMemcpyHostToDevice, s));
    VLB_CUDA(cudaStreamSynchronize(s));  // pack is a local
    const double *dd = (const double *)dev;
    const int *di = (const int *)(dev + dbytes);
    return KdDev{dd, dd + nn, dd + 2 * nn, di, di + nn, di + 2 * nn, di + 3 * nn, (int)nn};
  }

  double energy(const T *dist) {
    double *part = sc.slot[8].get<double>(kKmEnergyBlocks + 1);
    VLB_LAUNCH("km_energy", s, k_km_energy<T><<<kKmEnergyBlocks, kKmThreads, 0, s>>>(dist, N, part));
    sum_doubles(part, kKmEnergyBlocks, part + kKmEnergyBlocks, s);
    double e = 0;
    VLB_CUDA(cudaMemcpyAsync(&e, part + kKmEnergyBlocks, sizeof(double), cudaMemcpyDeviceToHost, s));
    VLB_CUDA(cudaStreamSynchronize(s));
    return e;
  }

  template <typename TT, int L>
  struct AnnLaunch {
    static void run(KMeansRun &r, const TT *centers, const KdDev &tr, i64 maxComp, int update, uint32_t *assign,
                    TT *dist, int *err, const uint32_t *list, i64 count) {
      const int cap = tr.numNodes;
      const size_t heap = (size_t)cap * (sizeof(double) + sizeof(int));
      const size_t rowB = align16(sizeof(TT) * (size_t)r.D);
      const i64 M = list ? count : r.N;
      // Up to 8 warps (rows) per block, as many as fit 200 KB with their query
      // rows and, when possible, their heaps.
      const size_t budget = (size_t)200 * 1024;
      const size_t perW = align16(rowB + heap);
      int wpb = (int)std::min<size_t>(8, budget / perW);
      if (wpb >= 1) {
        const i64 blocks = std::max<i64>(1, std::min<i64>((M + wpb - 1) / wpb, (i64)num_sms() * 8));
        const size_t smem = perW * wpb;
        auto kern = k_km_ann<TT, L, true>;
        VLB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        VLB_LAUNCH("km_ann", r.s, (kern<<<(int)blocks, 32 * wpb, smem, r.s>>>(
                                      r.X, r.N, (int)r.D, centers, tr, maxComp, update, assign, dist,
                                      (double *)nullptr, (int *)nullptr, cap, err, list, count)));
        return;
      }
      wpb = 8;
      i64 blocks = std::min<i64>((M + wpb - 1) / wpb, (i64)num_sms() * 8);
      blocks = std::max<i64>(1, std::min<i64>(blocks, (i64)(kHeapBudget / (heap * wpb))));
      const i64 GW = blocks * wpb;
      double *hk = r.sc.slot[5].template get<double>(GW * cap);
      int *hn = r.sc.slot[6].template get<int>(GW * cap);
      const size_t smem = rowB * wpb;
      auto kern = k_km_ann<TT, L, false>;
      VLB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      VLB_LAUNCH("km_ann", r.s, (kern<<<(int)blocks, 32 * wpb, smem, r.s>>>(r.X, r.N, (int)r.D, centers, tr, maxComp,
                                                                             update, assign, dist, hk, hn, cap, err,
                                                                             list, count)));
    }
  };

  template <typename TT, int L>
  struct NearestLaunch {
    static void run(KMeansRun &r, const TT *centers, int mode, int update, uint32_t *assign, TT *dist,
                    uint32_t *list, unsigned long long *count) {
      const int TB = r.tile_rows();
      const i64 blocks = std::min<i64>((r.N + TB - 1) / TB, (i64)num_sms() * 16);
      constexpr int TC = sizeof(TT) == 4 ? 8 : 4;
      // Centre rows staged per chunk of KC (a multiple of TC, about 16 KB).
      const size_t rowBytes = sizeof(TT) * (size_t)r.D;
      int KC = (int)std::max<size_t>(1, (size_t)16384 / rowBytes) / TC * TC;
      KC = std::max(TC, std::min(KC, 64));
      const size_t smem = align16(rowBytes * (TB + 1)) + rowBytes * KC;
      // The distances' rounding: a difference, a square and at most D - 1
      // additions per distance, each rounded once (unit roundoff u), bound
      // the error of a distance d by (D + 6) u d; a relative gap above
      // 2 (D + 8) u between the least and the second least distance keeps
      // the least one's exact value below every other's and below the
      // search's lower bounds for the other centres.
      const TT margin = (TT)((double)(r.D + 8) * (sizeof(TT) == 4 ? 0x1p-23 : 0x1p-52));
      auto go = [&](auto kern) {
        VLB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        VLB_LAUNCH(mode == kNearestQuantize ? "km_quantize" : "km_screen", r.s,
                   (kern<<<(int)blocks, TB, smem, r.s>>>(r.X, r.N, (int)r.D, centers, (int)r.K, KC, mode, update,
                                                         assign, dist, margin, list, count)));
      };
      if (r.vec(L)) go(k_km_nearest<TT, L, true, TC>);
      else go(k_km_nearest<TT, L, false, TC>);
    }
  };

  // New centres from the assignment, restarts of the empty ones
  // (vl/kmeans.c:1072-1100).
  void update_centres(const uint32_t *assign, T *centers) {
    const int nb = (int)((N + kKmChunk - 1) / kKmChunk);
    uint32_t *H = sc.slot[9].get<uint32_t>((i64)K * nb);
    uint32_t *cnt = sc.slot[10].get<uint32_t>(K);
    i64 *off = sc.slot[11].get<i64>(K + 1);
    uint32_t *order = sc.slot[12].get<uint32_t>(N);
    const size_t hsm = sizeof(uint32_t) * (size_t)K;
    VLB_CUDA(cudaFuncSetAttribute(k_km_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsm));
    VLB_LAUNCH("km_hist", s, k_km_hist<<<nb, kKmThreads, hsm, s>>>(assign, N, (int)K, nb, H));
    VLB_LAUNCH("km_scan", s, k_km_scan<<<blocks_for(K, 128), 128, 0, s>>>(H, (int)K, nb, cnt));
    std::vector<uint32_t> hc((size_t)K);
    VLB_CUDA(cudaMemcpyAsync(hc.data(), cnt, sizeof(uint32_t) * K, cudaMemcpyDeviceToHost, s));
    VLB_CUDA(cudaStreamSynchronize(s));
    std::vector<i64> ho((size_t)(K + 1));
    ho[0] = 0;
    for (i64 c = 0; c < K; ++c) ho[(size_t)(c + 1)] = ho[(size_t)c] + (i64)hc[(size_t)c];
    VLB_CUDA(cudaMemcpyAsync(off, ho.data(), sizeof(i64) * (K + 1), cudaMemcpyHostToDevice, s));
    const size_t bsm = sizeof(i64) * (size_t)K;
    VLB_CUDA(cudaFuncSetAttribute(k_km_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsm));
    VLB_LAUNCH("km_scatter", s, k_km_scatter<<<nb, 32, bsm, s>>>(assign, N, (int)K, nb, H, off, order));
    const int R = (int)std::max<i64>(1, std::min<i64>(64, kSumTileElems / D));
    VLB_LAUNCH("km_sums", s, k_km_sums<T><<<(int)K, kSumThreads, 0, s>>>(X, (int)D, R, off, order, centers));
    for (i64 c = 0; c < K; ++c) {
      if (hc[(size_t)c] != 0) continue;
      const i64 x = (i64)vl_rand_uindex(rand, (vl_uindex)N);
      VLB_CUDA(cudaMemcpyAsync(centers + c * D, X + x * D, sizeof(T) * D, cudaMemcpyDeviceToDevice, s));
    }
    VLB_CUDA(cudaStreamSynchronize(s));  // ho is a local
  }

  // ANN refinement, vl/kmeans.c:1003-1150 (L2 distance).
  double refine(const KMeansSettings &cfg, T *centers, uint32_t *assign) {
    T *dist = sc.slot[7].get<T>(N);
    int *err = sc.slot[13].get<int>(1);
    // With a budget of at least K comparisons (one tree) the search is exact
    // up to ties: screen every row by brute force, search the near ties.
    const bool screen = K <= cfg.maxNumComparisons;
    uint32_t *list = sc.slot[15].get<uint32_t>(N);
    unsigned long long *cnt = sc.slot[16].get<unsigned long long>(1);
    VLB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    double energy = INFINITY, prev = INFINITY, initial = INFINITY;
    for (i64 it = 0;; ++it) {
      const KdDev tr = tree(centers);
      const int update = it > 0 ? 1 : 0;
      if (screen) {
        VLB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s));
        by_lanes<NearestLaunch>(*this, (const T *)centers, (int)kNearestScreen, update, assign, dist, list, cnt);
        unsigned long long hc = 0;
        VLB_CUDA(cudaMemcpyAsync(&hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, s));
        VLB_CUDA(cudaStreamSynchronize(s));
        if (hc > 0)
          by_lanes<AnnLaunch>(*this, (const T *)centers, tr, (i64)cfg.maxNumComparisons, update, assign, dist, err,
                              (const uint32_t *)list, (i64)hc);
      } else {
        by_lanes<AnnLaunch>(*this, (const T *)centers, tr, (i64)cfg.maxNumComparisons, update, assign, dist, err,
                            (const uint32_t *)nullptr, (i64)0);
      }
      energy = this->energy(dist);
      if (it >= cfg.maxNumIterations) break;
      if (energy == prev) break;
      if (it == 0) {
        initial = energy;
      } else {
        const double eps = (prev - energy) / (initial - energy);
        if (eps < cfg.minEnergyVariation) break;
      }
      prev = energy;
      update_centres(assign, centers);
    }
    int herr = 0;
    VLB_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    VLB_CUDA(cudaStreamSynchronize(s));
    VLB_CHECK(herr == 0, VL_ERR_BAD_ARG, "k-means: kd-tree search heap overflow");
    return energy;
  }
};

}  // namespace

template <typename T>
double kmeans_ann(const T *X, i64 N, i64 D, i64 K, const KMeansSettings &cfg, int lanes, T *centers,
                  uint32_t *assign, cudaStream_t s) {
  VLB_CHECK(N >= 1 && D >= 1 && K >= 1, VL_ERR_BAD_ARG, "k-means: empty data or no centres");
  VLB_CHECK(D <= (i64)kSumThreads * kSumDims, VL_ERR_BAD_ARG, "k-means initialisation: dimension above 1024");
  VLB_CHECK(N >= K, VL_ERR_BAD_ARG, "k-means: fewer data points than centres");
  VLB_CHECK(N < ((i64)1 << 32) && K <= 16384, VL_ERR_BAD_ARG, "k-means: too many data points or centres");
  VLB_CHECK(cfg.numRepetitions >= 1, VL_ERR_BAD_ARG, "k-means: at least one repetition");
  KMeansRun<T> r{X, N, D, K, lanes, s, thread_scratch(kArenaKMeans), vl_get_rand()};
  T *work = cfg.numRepetitions > 1 ? r.sc.slot[14].template get<T>(K * D) : centers;
  double bestEnergy = INFINITY;
  for (i64 rep = 0; rep < cfg.numRepetitions; ++rep) {  // vl/kmeans.c:2034-2088
    r.seed(work);
    const double e = r.refine(cfg, work, assign);
    if (e < bestEnergy || rep == 0) {
      bestEnergy = e;
      if (work != centers)
        VLB_CUDA(cudaMemcpyAsync(centers, work, sizeof(T) * K * D, cudaMemcpyDeviceToDevice, s));
    }
  }
  r.template by_lanes<KMeansRun<T>::template NearestLaunch>(r, (const T *)centers, (int)kNearestQuantize, 0, assign,
                                                             (T *)nullptr, (uint32_t *)nullptr,
                                                             (unsigned long long *)nullptr);
  return bestEnergy;
}

template <typename T>
void onehot_posteriors(const uint32_t *assign, i64 N, i64 K, T *q, cudaStream_t s) {
  VLB_LAUNCH("km_onehot", s, k_km_onehot<T><<<blocks_for(N * K, kKmThreads), kKmThreads, 0, s>>>(assign, N, K, q));
}

template double kmeans_ann<float>(const float *, i64, i64, i64, const KMeansSettings &, int, float *, uint32_t *,
                                  cudaStream_t);
template double kmeans_ann<double>(const double *, i64, i64, i64, const KMeansSettings &, int, double *, uint32_t *,
                                   cudaStream_t);
template void onehot_posteriors<float>(const uint32_t *, i64, i64, float *, cudaStream_t);
template void onehot_posteriors<double>(const uint32_t *, i64, i64, double *, cudaStream_t);

}  // namespace vlb
