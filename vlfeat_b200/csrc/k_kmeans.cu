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
//  - each data point's query is one GPU thread running the reference's
//    best-bin-first search (vl/kdtree.c:583-725, 774-840) with the same heap
//    discipline (vl/heap-def.h), comparison budget and tie rules;
//  - distances use the summation order of the reference's SIMD kernel;
//  - a centre is the sum of its points in data order (a stable counting sort
//    by centre, then one thread per centre and dimension adding in order),
//    divided by its mass rounded to the data type (vl/kmeans.c:1078-1098).
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
// sq[d * TB + r] (row r's element d), so that each thread reads its row with
// stride TB and a warp's reads hit distinct banks.
template <typename T>
__device__ __forceinline__ void load_rows(const T *__restrict__ X, i64 N, int D, i64 base, T *sq) {
  const int TB = blockDim.x;
  const i64 rows = min((i64)TB, N - base);
  const T *src = X + base * D;
  for (i64 e = threadIdx.x; e < rows * D; e += TB) {
    const i64 r = e / D;
    const int d = (int)(e - r * D);
    sq[(i64)d * TB + r] = src[e];
  }
}

// Distance of the query (stride qs) to centre row c; VEC reads the row in
// 16-byte vectors (row starts 16-byte aligned, whole vectors per lane group).
template <typename T, int L, bool VEC>
__device__ __forceinline__ T row_dist(const T *q, int qs, const T *__restrict__ c, int D) {
  if constexpr (VEC && (L * sizeof(T)) % 16 == 0) {
    return l2_ordered_sv<T, L>(q, qs, c, D);
  } else {
    return l2_ordered_s<T, L>(q, qs, c, D);
  }
}

// One query of the forest, vl/kdtree.c:774-840 with numNeighbors = 1, the
// recursion of vl/kdtree.c:583-725 unrolled into a loop.  The search heap of
// this thread lives at hk[e * G], hn[e * G] (entry e), capacity cap = the
// tree's node count, which bounds the pushes of one query (each node is
// pushed at most once).  Heap moves follow vl/heap-def.h: push sifts towards
// the root while strictly smaller, pop moves the last entry to the root and
// sifts it down towards the smaller child (the right one on ties) while it
// is strictly larger.
template <typename T, int L, bool VEC>
__device__ __forceinline__ int kd_query(const T *q, int qs, const T *__restrict__ C, int D, const KdDev &tr,
                                        i64 maxComp, double *__restrict__ hk, int *__restrict__ hn, i64 G,
                                        int cap, double &bestOut, int *__restrict__ err) {
  const bool exact = maxComp == 0;
  i64 comps = 0;
  int nh = 1;
  hk[0] = 0.0;
  hn[0] = 0;
  bool have = false;
  double best = 0.0;
  int bestIdx = 0;
  while (exact || comps < maxComp) {
    if (nh == 0) break;
    // Pop (vl/heap-def.h pop + up).
    nh -= 1;
    const double pk = hk[0];
    const int pn = hn[0];
    if (nh > 0) {
      const double lk = hk[(i64)nh * G];
      const int ln = hn[(i64)nh * G];
      int i = 0;
      if (nh > 1) {
        while (true) {
          const int l = 2 * i + 1, r = l + 1;
          if (l >= nh) break;
          int c;
          if (r >= nh) {
            c = l;
          } else {
            c = hk[(i64)l * G] < hk[(i64)r * G] ? l : r;
          }
          const double ck = hk[(i64)c * G];
          if (lk > ck) {
            hk[(i64)i * G] = ck;
            hn[(i64)i * G] = hn[(i64)c * G];
            i = c;
            if (r >= nh) break;  // a lone left child is the last entry: stop
          } else {
            break;
          }
        }
      }
      hk[(i64)i * G] = lk;
      hn[(i64)i * G] = ln;
    }
    if (have && best < pk) break;  // no better neighbour can remain
    double dist = pk;
    int n = pn;
    while (true) {
      const int lc = tr.lower[n];
      if (lc < 0) {  // leaf
        const int b = -lc - 1, e = -tr.upper[n] - 1;
        for (int it = b; it < e && (exact || comps < maxComp); ++it) {
          const int di = tr.ent[it];
          const double dd = (double)row_dist<T, L, VEC>(q, qs, C + (i64)di * D, D);
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
      const double xv = (double)q[(i64)tr.dim[n] * qs];
      const double x1 = tr.lb[n], x2 = tr.thr[n], x3 = tr.ub[n];
      double delta = __dsub_rn(xv, x2);
      double save = __dadd_rn(dist, __dmul_rn(delta, delta));
      int next, sv;
      if (xv <= x2) {
        next = lc;
        sv = tr.upper[n];
        if (xv <= x1) {
          delta = __dsub_rn(xv, x1);
          save = __dsub_rn(save, __dmul_rn(delta, delta));
        }
      } else {
        next = tr.upper[n];
        sv = lc;
        if (xv > x3) {
          delta = __dsub_rn(xv, x3);
          save = __dsub_rn(save, __dmul_rn(delta, delta));
        }
      }
      if (!have || best > save) {
        if (nh >= cap) {
          atomicOr(err, 1);  // cannot happen: pushes per query <= nodes
        } else {
          int i = nh++;
          while (i > 0) {
            const int p = (i - 1) / 2;
            const double pkk = hk[(i64)p * G];
            if (save < pkk) {
              hk[(i64)i * G] = pkk;
              hn[(i64)i * G] = hn[(i64)p * G];
              i = p;
            } else {
              break;
            }
          }
          hk[(i64)i * G] = save;
          hn[(i64)i * G] = sv;
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
// unless the new centre is strictly closer.  Persistent blocks of TB rows.
template <typename T, int L, bool VEC>
__global__ void k_km_ann(const T *__restrict__ X, i64 N, int D, const T *__restrict__ C, KdDev tr, i64 maxComp,
                         int update, uint32_t *__restrict__ assign, T *__restrict__ dist,
                         double *__restrict__ hkey, int *__restrict__ hnode, int cap, int *__restrict__ err) {
  extern __shared__ __align__(16) unsigned char km_smem[];
  T *sq = (T *)km_smem;
  const int TB = blockDim.x;
  const i64 G = (i64)gridDim.x * TB;
  const i64 g = (i64)blockIdx.x * TB + threadIdx.x;
  for (i64 base = (i64)blockIdx.x * TB; base < N; base += G) {
    __syncthreads();
    load_rows(X, N, D, base, sq);
    __syncthreads();
    const i64 x = base + threadIdx.x;
    if (x >= N) continue;
    const T *q = sq + threadIdx.x;
    double nd;
    const int ni = kd_query<T, L, VEC>(q, TB, C, D, tr, maxComp, hkey + g, hnode + g, G, cap, nd, err);
    const T ndt = (T)nd;  // exact: the distance was computed in T
    if (!update) {
      dist[x] = ndt;
      assign[x] = (uint32_t)ni;
    } else {
      const T prev = row_dist<T, L, VEC>(q, TB, C + (i64)assign[x] * D, D);
      if (prev > ndt) {
        dist[x] = ndt;
        assign[x] = (uint32_t)ni;
      } else {
        dist[x] = prev;
      }
    }
  }
}

// Exact quantisation, vl/kmeans.c:656-702: the first centre of least
// distance (strict <, starting from +inf; rows whose distances are all NaN
// keep centre 0, where the reference leaves the assignment unset).
template <typename T, int L, bool VEC>
__global__ void k_km_quantize(const T *__restrict__ X, i64 N, int D, const T *__restrict__ C, int K,
                              uint32_t *__restrict__ assign) {
  extern __shared__ __align__(16) unsigned char km_smem[];
  T *sq = (T *)km_smem;
  const int TB = blockDim.x;
  const i64 G = (i64)gridDim.x * TB;
  for (i64 base = (i64)blockIdx.x * TB; base < N; base += G) {
    __syncthreads();
    load_rows(X, N, D, base, sq);
    __syncthreads();
    const i64 x = base + threadIdx.x;
    if (x >= N) continue;
    const T *q = sq + threadIdx.x;
    T best = (T)INFINITY;
    uint32_t bi = 0;
    for (int k = 0; k < K; ++k) {
      const T dd = row_dist<T, L, VEC>(q, TB, C + (i64)k * D, D);
      if (dd < best) {
        best = dd;
        bi = (uint32_t)k;
      }
    }
    assign[x] = bi;
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

// New centres, vl/kmeans.c:1078-1098: one thread per (centre, dimension) adds
// the centre's rows in data order from 0, then divides by the mass rounded to
// T.  Empty centres are left for the host's restarts.
template <typename T>
__global__ void k_km_sums(const T *__restrict__ X, int D, int K, const i64 *__restrict__ off,
                          const uint32_t *__restrict__ order, T *__restrict__ C) {
  const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (i64)K * D) return;
  const int c = (int)(e / D);
  const int d = (int)(e - (i64)c * D);
  const i64 b = off[c], n = off[c + 1] - off[c];
  if (n == 0) return;
  T acc = (T)0;
  i64 j = 0;
  for (; j + 8 <= n; j += 8) {
    uint32_t idx[8];
    T v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) idx[u] = order[b + j + u];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = X[(i64)idx[u] * D + d];
#pragma unroll
    for (int u = 0; u < 8; ++u) acc = add_rn(acc, v[u]);
  }
  for (; j < n; ++j) acc = add_rn(acc, X[(i64)order[b + j] * D + d]);
  C[e] = div_rn(acc, (T)(unsigned long long)n);
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
      if ((size_t)tb * D * sizeof(T) <= (size_t)96 * 1024) return tb;
    VLB_CHECK((size_t)32 * D * sizeof(T) <= (size_t)200 * 1024, VL_ERR_BAD_ARG,
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
                    TT *dist, int *err) {
      const int TB = r.tile_rows();
      const int cap = tr.numNodes;
      const i64 perThread = (i64)cap * (sizeof(double) + sizeof(int));
      i64 blocks = std::min<i64>((r.N + TB - 1) / TB, (i64)num_sms() * 12);
      blocks = std::max<i64>(1, std::min<i64>(blocks, (i64)(kHeapBudget / (size_t)(perThread * TB))));
      const i64 G = blocks * TB;
      double *hk = r.sc.slot[5].template get<double>(G * cap);
      int *hn = r.sc.slot[6].template get<int>(G * cap);
      const size_t smem = sizeof(TT) * (size_t)TB * (size_t)r.D;
      auto go = [&](auto kern) {
        VLB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        VLB_LAUNCH("km_ann", r.s, (kern<<<(int)blocks, TB, smem, r.s>>>(r.X, r.N, (int)r.D, centers, tr, maxComp,
                                                                         update, assign, dist, hk, hn, cap, err)));
      };
      if (r.vec(L)) go(k_km_ann<TT, L, true>);
      else go(k_km_ann<TT, L, false>);
    }
  };

  template <typename TT, int L>
  struct QuantLaunch {
    static void run(KMeansRun &r, const TT *centers, uint32_t *assign) {
      const int TB = r.tile_rows();
      const i64 blocks = std::min<i64>((r.N + TB - 1) / TB, (i64)num_sms() * 16);
      const size_t smem = sizeof(TT) * (size_t)TB * (size_t)r.D;
      auto go = [&](auto kern) {
        VLB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        VLB_LAUNCH("km_quantize", r.s, (kern<<<(int)blocks, TB, smem, r.s>>>(r.X, r.N, (int)r.D, centers,
                                                                              (int)r.K, assign)));
      };
      if (r.vec(L)) go(k_km_quantize<TT, L, true>);
      else go(k_km_quantize<TT, L, false>);
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
    VLB_LAUNCH("km_sums", s, k_km_sums<T><<<blocks_for(K * D, kKmThreads), kKmThreads, 0, s>>>(
                                 X, (int)D, (int)K, off, order, centers));
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
    VLB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    double energy = INFINITY, prev = INFINITY, initial = INFINITY;
    for (i64 it = 0;; ++it) {
      const KdDev tr = tree(centers);
      by_lanes<AnnLaunch>(*this, (const T *)centers, tr, (i64)cfg.maxNumComparisons, it > 0 ? 1 : 0, assign, dist,
                          err);
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
  r.template by_lanes<KMeansRun<T>::template QuantLaunch>(r, (const T *)centers, assign);
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
