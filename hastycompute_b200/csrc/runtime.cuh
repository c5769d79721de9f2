// Host-side runtime shared by the library's translation units: error reporting
// (hb_last_error), launch accounting and profiling (hb_launch_count, hb_profile_*),
// device guard and the workspace bump allocator.  The state is held in C++17 inline
// variables, so every translation unit of the library sees one instance.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/hasty_b200.h"

namespace hb {

// Image size and device of a Toeplitz plan (defined with struct hb_plan), and its team
// twiddle tables of nz, ny, nx back to back (device).
void plan_geometry(const ::hb_plan* plan, int* N, int* device);
const float2* plan_image_tables(const ::hb_plan* plan);

// psf(d) = prod(M)^-1 * sum_j w_j exp(+i c_j . d) (w_j = 1 when weights is null) on an
// M0 x M1 x M2 grid in circulant layout
// (offset d = n for n < M/2, n - M otherwise), through a type-1 NUFFT at tolerance tol;
// out: [M0][M1][M2] complex64.  Synchronises st.
int nufft_psf_circulant(const int* M, const float* coords, int64_t nsamples, double tol, const float* weights,
                        int device, float2* out, cudaStream_t st);

// Message of the last failure on this thread (hb_last_error).
inline thread_local std::string g_err;

inline int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define HB_CUDA(call)                                                                 \
  do {                                                                                \
    cudaError_t _e = (call);                                                          \
    if (_e != cudaSuccess)                                                            \
      return fail(HB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e));   \
  } while (0)

#define HB_CHECK_LAUNCH()                                                             \
  do {                                                                                \
    cudaError_t _e = cudaGetLastError();                                              \
    if (_e != cudaSuccess)                                                            \
      return fail(HB_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(_e)); \
  } while (0)


struct DeviceGuard {
  int prev = -1;
  bool ok = true;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) { ok = false; return; }
    if (prev != dev && cudaSetDevice(dev) != cudaSuccess) ok = false;
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// ------------------------------------------------------------ launch accounting ----
inline std::atomic<uint64_t> g_launches{0};
struct ProfRec {
  int kind;
  cudaEvent_t a, b;
};
inline std::mutex g_prof_mu;
inline std::atomic<bool> g_prof_on{false};
inline std::vector<ProfRec> g_prof;
inline std::vector<cudaEvent_t> g_ev_pool;

inline cudaEvent_t take_event() {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (!g_ev_pool.empty()) {
    cudaEvent_t e = g_ev_pool.back();
    g_ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}

// Counts one kernel launch; while profiling, brackets it with an event pair on `st`.
struct LaunchScope {
  int kind;
  cudaStream_t st;
  cudaEvent_t a = nullptr, b = nullptr;
  LaunchScope(int k, cudaStream_t s) : kind(k), st(s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) return;  // graph replays count
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (g_prof_on.load(std::memory_order_relaxed)) {
      a = take_event();
      b = take_event();
      if (a && b) cudaEventRecord(a, st);
    }
  }
  ~LaunchScope() {
    if (a && b) {
      cudaEventRecord(b, st);
      std::lock_guard<std::mutex> lk(g_prof_mu);
      g_prof.push_back({kind, a, b});
    }
  }
};

// Bump allocator over a caller workspace (dry run when base == nullptr).
struct Arena {
  char* base;
  size_t off = 0;
  explicit Arena(void* b) : base((char*)b) {}
  template <typename T>
  T* take(size_t n) {
    off = (off + 255) & ~size_t(255);
    T* p = base ? (T*)(base + off) : nullptr;
    off += n * sizeof(T);
    return p;
  }
};

}  // namespace hb
