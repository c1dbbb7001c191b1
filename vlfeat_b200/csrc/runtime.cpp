// Runtime services: the vl_* runtime symbols that programs written against
// VLFeat link (vl/generic.h), plus the library's stream, scratch, launch
// accounting and event-timing plumbing.
#include <atomic>
#include <chrono>
#include <cstdarg>
#include <cstdlib>
#include <cpuid.h>
#include <cstring>
#include <ctime>
#include <map>
#include <mutex>

#include <nvtx3/nvToolsExt.h>

#include "common.h"

extern "C" {
#include "vlb200.h"
}

// ---------------------------------------------------------------- errors
namespace {
thread_local int g_last_error = VL_ERR_OK;
thread_local char g_last_msg[1024] = "";
std::atomic<vl_size> g_num_threads{1};
std::atomic<int> g_simd{1};
// The process-wide mode starts as EXACT, VLFeat's own float arithmetic, so a
// program relinked against this library gets the reference's float results;
// the environment variable VLB200_PRECISION (exact, fp32, bf16) selects
// another mode without a code change.
int initial_precision() {
  const char *e = getenv("VLB200_PRECISION");
  if (!e) return VLB200_PREC_EXACT;
  if (!strcmp(e, "fp32") || !strcmp(e, "FP32")) return VLB200_PREC_FP32;
  if (!strcmp(e, "bf16") || !strcmp(e, "BF16")) return VLB200_PREC_BF16;
  return VLB200_PREC_EXACT;
}
std::atomic<int> g_precision{initial_precision()};
printf_func_t g_printf = (printf_func_t)&printf;

int silent_printf(char const *, ...) { return 0; }
}  // namespace

extern "C" {

int vl_get_last_error(void) { return g_last_error; }
char const *vl_get_last_error_message(void) { return g_last_msg; }

int vl_set_last_error(int error, char const *errorMessage, ...) {
  g_last_error = error;
  if (errorMessage) {
    va_list ap;
    va_start(ap, errorMessage);
    vsnprintf(g_last_msg, sizeof(g_last_msg), errorMessage, ap);
    va_end(ap);
  } else {
    g_last_msg[0] = 0;
  }
  return error;
}

// ------------------------------------------------------------ info/state
char const *vl_get_version_string(void) { return "0.9.21-b200"; }
char const *vlb200_version(void) { return "vlfeat-b200 0.1 (sm_100a)"; }
void vl_set_simd_enabled(vl_bool x) { g_simd = x ? 1 : 0; }
vl_bool vl_get_simd_enabled(void) { return g_simd.load(); }

// cpuid leaf 1: SSE2 = EDX bit 26, SSE3 = ECX bit 0, AVX = ECX bit 28.
static unsigned cpuid1(int reg) {
  unsigned a = 0, b = 0, c = 0, d = 0;
  if (!__get_cpuid(1, &a, &b, &c, &d)) return 0;
  return reg == 2 ? c : d;
}
vl_bool vl_cpu_has_avx(void) { return (cpuid1(2) >> 28) & 1u; }
vl_bool vl_cpu_has_sse3(void) { return cpuid1(2) & 1u; }
vl_bool vl_cpu_has_sse2(void) { return (cpuid1(3) >> 26) & 1u; }

// ------------------------------------------------------------------- RNG
// MT19937 (Matsumoto and Nishimura; the 2002 initialisation), the generator
// of vl/random.c: 624 words of state and an index; index 625 marks a
// generator that was never seeded and is seeded with 5489 on first use.
static constexpr int kMtN = 624, kMtM = 397;

void vl_rand_init(VlRand *self) {
  memset(self->mt, 0, sizeof(self->mt));
  self->mti = kMtN + 1;
}

void vl_rand_seed(VlRand *self, vl_uint32 s) {
  vl_uint32 *mt = self->mt;
  mt[0] = s;
  for (vl_uint32 i = 1; i < (vl_uint32)kMtN; ++i) mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + i;
  self->mti = kMtN;
}

void vl_rand_seed_by_array(VlRand *self, vl_uint32 const key[], vl_size keySize) {
  vl_rand_seed(self, 19650218u);
  vl_uint32 *mt = self->mt;
  int i = 1;
  vl_size j = 0;
  for (vl_size k = keySize > (vl_size)kMtN ? keySize : (vl_size)kMtN; k; --k) {
    mt[i] = (mt[i] ^ ((mt[i - 1] ^ (mt[i - 1] >> 30)) * 1664525u)) + key[j] + (vl_uint32)j;
    if (++i >= kMtN) {
      mt[0] = mt[kMtN - 1];
      i = 1;
    }
    if (++j >= keySize) j = 0;
  }
  for (int k = kMtN - 1; k; --k) {
    mt[i] = (mt[i] ^ ((mt[i - 1] ^ (mt[i - 1] >> 30)) * 1566083941u)) - (vl_uint32)i;
    if (++i >= kMtN) {
      mt[0] = mt[kMtN - 1];
      i = 1;
    }
  }
  mt[0] = 0x80000000u;  // non-zero state
}

vl_uint32 vl_rand_uint32(VlRand *self) {
  vl_uint32 *mt = self->mt;
  if (self->mti >= (vl_uint32)kMtN) {
    if (self->mti == (vl_uint32)kMtN + 1) vl_rand_seed(self, 5489u);
    // Regenerate all words; indices wrap, so later words use the new values
    // of earlier ones as the recurrence requires.
    for (int k = 0; k < kMtN; ++k) {
      const vl_uint32 y = (mt[k] & 0x80000000u) | (mt[(k + 1) % kMtN] & 0x7fffffffu);
      mt[k] = mt[(k + kMtM) % kMtN] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
    }
    self->mti = 0;
  }
  vl_uint32 y = mt[self->mti++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

void vl_rand_permute_indexes(VlRand *self, vl_index *array, vl_size size) {
  for (vl_index i = (vl_index)size - 1; i > 0; --i) {
    const vl_index j = (vl_index)vl_rand_uindex(self, (vl_uindex)i + 1);
    const vl_index t = array[i];
    array[i] = array[j];
    array[j] = t;
  }
}

VlRand *vl_get_rand(void) {
  struct ThreadRand {
    VlRand r;
    ThreadRand() { vl_rand_init(&r); }
  };
  static thread_local ThreadRand t;
  return &t.r;
}
vl_size vl_get_max_threads(void) { return g_num_threads.load(); }
void vl_set_num_threads(vl_size n) { g_num_threads = n ? n : 1; }
vl_size vl_get_thread_limit(void) { return 1; }

int vlb200_set_precision(int p) {
  if (p < VLB200_PREC_EXACT || p > VLB200_PREC_BF16_ROUTER) {
    return vl_set_last_error(VL_ERR_BAD_ARG, "vlb200_set_precision: unknown mode %d", p);
  }
  g_precision = p;
  return 0;
}
int vlb200_get_precision(void) { return g_precision.load(); }

int vlb200_device_ok(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n > 0;
}

// ---------------------------------------------------------------- memory
void *vl_malloc(size_t n) { return malloc(n); }
void *vl_realloc(void *ptr, size_t n) { return realloc(ptr, n); }
void *vl_calloc(size_t n, size_t size) { return calloc(n, size); }
void *vl_memalign(size_t n, size_t size) {
  void *p = nullptr;
  if (posix_memalign(&p, n < sizeof(void *) ? sizeof(void *) : n, size)) return nullptr;
  return p;
}
void vl_free(void *ptr) { free(ptr); }

// ---------------------------------------------------------------- printf
void vl_set_printf_func(printf_func_t f) { g_printf = f ? f : (printf_func_t)&silent_printf; }
printf_func_t vl_get_printf_func(void) { return g_printf; }

// ---------------------------------------------------------------- timing
static thread_local std::chrono::steady_clock::time_point g_tic;
void vl_tic(void) { g_tic = std::chrono::steady_clock::now(); }
double vl_toc(void) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - g_tic).count();
}
double vl_get_cpu_time(void) { return (double)clock() / (double)CLOCKS_PER_SEC; }

}  // extern "C"

// ------------------------------------------------------------ plumbing
namespace vlb {

void throw_cuda(cudaError_t e, const char *what, const char *file, int line) {
  cudaGetLastError();
  char buf[512];
  snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e),
           what, file, line);
  throw Error(e == cudaErrorMemoryAllocation ? VL_ERR_ALLOC : VL_ERR_BAD_ARG, buf);
}

namespace {
struct StreamHolder {
  cudaStream_t s = nullptr;
  ~StreamHolder() {
    // Streams die with the context at process exit; destroying them from a
    // thread_local destructor after the runtime has shut down is unsafe.
  }
};
thread_local StreamHolder g_stream;
thread_local Scratch *g_scratch[kNumArenas] = {};
thread_local DevBuf *g_pinned_dummy = nullptr;
thread_local void *g_pinned = nullptr;
thread_local size_t g_pinned_cap = 0;

std::atomic<uint64_t> g_launches{0};
std::atomic<int> g_profile{0};

struct ProfRec {
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
  double ms = 0;
  uint64_t launches = 0;
};
std::mutex g_prof_mu;
std::map<std::string, ProfRec> g_prof;
thread_local cudaEvent_t g_open_event = nullptr;
}  // namespace

cudaStream_t thread_stream() {
  if (!g_stream.s) VLB_CUDA(cudaStreamCreateWithFlags(&g_stream.s, cudaStreamNonBlocking));
  return g_stream.s;
}

Scratch &thread_scratch(int arena) {
  if (arena < 0 || arena >= kNumArenas) arena = kArenaApi;
  if (!g_scratch[arena]) g_scratch[arena] = new Scratch();  // lives until process exit
  return *g_scratch[arena];
}

void *pinned_host(size_t bytes) {
  (void)g_pinned_dummy;
  if (bytes > g_pinned_cap) {
    if (g_pinned) cudaFreeHost(g_pinned);
    g_pinned = nullptr;
    g_pinned_cap = 0;
    size_t want = bytes + bytes / 8;
    VLB_CUDA(cudaMallocHost(&g_pinned, want));
    g_pinned_cap = want;
  }
  return g_pinned;
}

int default_precision() { return g_precision.load(); }

thread_local int t_last_precision = 0;
void note_precision(int used) { t_last_precision = used; }

std::atomic<long long> g_fail_allocs{0};
bool take_injected_alloc_failure() {
  if (g_fail_allocs.load() <= 0) return false;
  return g_fail_allocs.fetch_sub(1) > 0;
}

int resolve_precision(int p, bool is_double) {
  if (is_double) return VLB200_PREC_EXACT;
  if (p == VLB200_PREC_DEFAULT) p = g_precision.load();
  VLB_CHECK(p >= VLB200_PREC_EXACT && p <= VLB200_PREC_BF16_ROUTER, VL_ERR_BAD_ARG,
            "unknown precision mode");
  return p;
}

// Each launch is also an NVTX range named after its kernel, so a timeline
// tool shows the library's kernels by name (a no-op without one attached).
void launch_begin(const char *name, cudaStream_t s) {
  nvtxRangePushA(name);
  if (g_profile.load()) {
    VLB_CUDA(cudaEventCreate(&g_open_event));
    VLB_CUDA(cudaEventRecord(g_open_event, s));
  }
}

void count_launch() { g_launches.fetch_add(1); }
void count_launches(unsigned long long n) { g_launches.fetch_add(n); }
bool profile_swap(bool on) { return g_profile.exchange(on ? 1 : 0) != 0; }

void launch_end(const char *name, cudaStream_t s) {
  nvtxRangePop();
  g_launches.fetch_add(1);
  if (g_profile.load() && g_open_event) {
    cudaEvent_t e1;
    VLB_CUDA(cudaEventCreate(&e1));
    VLB_CUDA(cudaEventRecord(e1, s));
    std::lock_guard<std::mutex> lk(g_prof_mu);
    auto &r = g_prof[name];
    r.pending.emplace_back(g_open_event, e1);
    r.launches++;
    g_open_event = nullptr;
  }
}

}  // namespace vlb

extern "C" {

int vlb200_last_precision(void) { return vlb::t_last_precision; }

void vlb200_debug_fail_allocations(vl_size n) { vlb::g_fail_allocs.store((long long)n); }

vl_uint64 vlb200_launch_count(void) { return vlb::g_launches.load(); }

void vlb200_profile_enable(int on) { vlb::g_profile = on ? 1 : 0; }

void vlb200_profile_reset(void) {
  std::lock_guard<std::mutex> lk(vlb::g_prof_mu);
  for (auto &kv : vlb::g_prof)
    for (auto &pe : kv.second.pending) {
      cudaEventDestroy(pe.first);
      cudaEventDestroy(pe.second);
    }
  vlb::g_prof.clear();
}

int vlb200_profile_read(char *names, vl_size nameStride, double *ms, vl_uint64 *launches,
                        vl_size maxEntries) {
  std::lock_guard<std::mutex> lk(vlb::g_prof_mu);
  vl_size i = 0;
  for (auto &kv : vlb::g_prof) {
    auto &r = kv.second;
    for (auto &pe : r.pending) {
      float t = 0;
      if (cudaEventSynchronize(pe.second) == cudaSuccess &&
          cudaEventElapsedTime(&t, pe.first, pe.second) == cudaSuccess)
        r.ms += t;
      cudaEventDestroy(pe.first);
      cudaEventDestroy(pe.second);
    }
    r.pending.clear();
    if (i < maxEntries) {
      if (names && nameStride) {
        strncpy(names + i * nameStride, kv.first.c_str(), nameStride - 1);
        names[i * nameStride + nameStride - 1] = 0;
      }
      if (ms) ms[i] = r.ms;
      if (launches) launches[i] = r.launches;
    }
    ++i;
  }
  return (int)i;
}

}  // extern "C"
