// Internal plumbing shared by the host-side API files and the kernel files:
// CUDA error handling, per-thread streams, grow-only device scratch, launch
// accounting and optional per-kernel event timing.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

extern "C" {
#include "vl/generic.h"
}

namespace vlb {

// An error that the C boundary turns into vl_set_last_error + a sentinel.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void throw_cuda(cudaError_t e, const char *what, const char *file, int line);

#define VLB_CUDA(x)                                                   \
  do {                                                                \
    cudaError_t e_ = (x);                                             \
    if (e_ != cudaSuccess) ::vlb::throw_cuda(e_, #x, __FILE__, __LINE__); \
  } while (0)

#define VLB_CHECK(cond, code, msg)                     \
  do {                                                 \
    if (!(cond)) throw ::vlb::Error((code), (msg));   \
  } while (0)

// The calling thread's library stream (non-blocking, created on first use).
cudaStream_t thread_stream();
inline cudaStream_t pick_stream(void *s) { return s ? (cudaStream_t)s : thread_stream(); }

// Launch accounting: every kernel launch of the library goes through
// launch_begin/launch_end (the LAUNCH macro below).
void launch_begin(const char *name, cudaStream_t s);
void launch_end(const char *name, cudaStream_t s);

#define VLB_LAUNCH(name, stream, ...)           \
  do {                                          \
    ::vlb::launch_begin((name), (stream));      \
    __VA_ARGS__;                                \
    VLB_CUDA(cudaGetLastError());               \
    ::vlb::launch_end((name), (stream));        \
  } while (0)

// Launch without the optional event timing (which creates CUDA events): used
// by the entry point that must not allocate.  The launch is still counted.
void count_launch();
// Adds n launches (the kernels of a replayed CUDA graph) to the count.
void count_launches(unsigned long long n);
// Sets the per-launch event timing on or off; returns the previous setting.
bool profile_swap(bool on);
#define VLB_LAUNCH_PLAIN(stream, ...)  \
  do {                                 \
    __VA_ARGS__;                       \
    VLB_CUDA(cudaGetLastError());      \
    ::vlb::count_launch();             \
  } while (0)

// Host-side fault injection (vlb200_debug_fail_allocations): the next n
// device allocations of the library's buffers fail as cudaMalloc failures
// do.  Returns true when this allocation is to fail.
bool take_injected_alloc_failure();

// Grow-only device buffer.  Contents are not preserved across growth.
struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }
  void release() {
    // Kernels still queued may read the old buffer: drain the device first.
    if (p) {
      cudaDeviceSynchronize();
      cudaFree(p);
    }
    p = nullptr;
    cap = 0;
  }
  template <typename T>
  T *get(size_t count) {
    size_t bytes = count * sizeof(T);
    if (bytes == 0) bytes = 16;
    if (bytes > cap) {
      release();
      size_t want = bytes + bytes / 8;
      cudaError_t e = take_injected_alloc_failure() ? cudaErrorMemoryAllocation : cudaMalloc(&p, want);
      if (e != cudaSuccess) {
        p = nullptr;
        cudaGetLastError();
        throw Error(VL_ERR_ALLOC, std::string("cudaMalloc of ") + std::to_string(want) +
                                      " bytes failed: " + cudaGetErrorString(e));
      }
      cap = want;
    }
    return static_cast<T *>(p);
  }
};

// Per-thread scratch arenas of device buffers reused across calls on one
// thread.  Each module owns an arena so slot numbers never collide.
struct Scratch {
  DevBuf slot[32];
};
enum ScratchArena {
  kArenaApi = 0,
  kArenaExact = 1,
  kArenaTc = 2,
  kArenaRouter = 3,
  kArenaVlad = 4,
  kArenaKMeans = 5,
  kArenaRouterTc = 6,  // the router's fallback rows on the tensor-core E-step
  kNumArenas = 7
};
Scratch &thread_scratch(int arena = kArenaApi);

// Pinned host staging buffer (per thread), for host-pointer API calls.
void *pinned_host(size_t bytes);

// Process-wide precision default (VLB200_PREC_*).
int default_precision();
int resolve_precision(int precision, bool is_double);
// Records the arithmetic a call actually used (VLB200_PREC_*), per thread:
// a request for a tensor-core mode on a shape the tensor-core kernels do not
// take runs EXACT, and vlb200_last_precision() reports that.
void note_precision(int used);

// Host-side printf through the VLFeat hook.
#define VLB_PRINTF(...) ((*vl_get_printf_func())(__VA_ARGS__))

}  // namespace vlb
