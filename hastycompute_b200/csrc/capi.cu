// C ABI of the B200 Toeplitz SENSE normal operator and batched CG (include/hasty_b200.h).
#include <cuda_runtime.h>

#include <atomic>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/hasty_b200.h"
#include "cg_kernels.cuh"
#include "diag_kernels.cuh"
#include "toeplitz_kernels.cuh"

using namespace hb;

struct hb_plan {
  int N0, N1, N2;
  int device;
  float2* tables;  // device twiddle tables (table_offsets layout)
  TableOffsets to;
};

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
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

// Supported axis lengths and their row in the launcher tables.
int axis_index(int64_t n) {
  switch (n) {
    case 8: return 0;
    case 16: return 1;
    case 32: return 2;
    case 64: return 3;
    case 128: return 4;
    case 96: return 5;
    case 160: return 6;
    default: return -1;
  }
}
bool is_pow2_axis(int64_t n) { int i = axis_index(n); return i >= 0 && i <= 4; }
int ilog2(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}

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
std::atomic<uint64_t> g_launches{0};
struct ProfRec {
  int kind;
  cudaEvent_t a, b;
};
std::mutex g_prof_mu;
std::atomic<bool> g_prof_on{false};
std::vector<ProfRec> g_prof;
std::vector<cudaEvent_t> g_ev_pool;

cudaEvent_t take_event() {
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

template <typename K>
cudaError_t ensure_smem(K kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// ---------------------------------------------------------------- pass launchers ----
using PassLauncher = cudaError_t (*)(const PassArgs&, int, cudaStream_t);

template <int N2, int YT>
cudaError_t launch_a(const PassArgs& a, int nslots, cudaStream_t st) {
  using C = XPassCfg<N2, YT>;
  const size_t smem = C::SMEM_F2 * sizeof(float2);
  cudaError_t e = ensure_smem(expand_fwd_x_kernel<N2, YT>, smem);
  if (e != cudaSuccess) return e;
  dim3 grid(a.N1 / YT, a.N0, nslots);
  LaunchScope ls(HB_KERNEL_EXPAND_FWD_X, st);
  expand_fwd_x_kernel<N2, YT><<<grid, C::THREADS, smem, st>>>(a);
  return cudaGetLastError();
}

template <int N2, int YT>
cudaError_t launch_c(const PassArgs& a, int nsys, cudaStream_t st) {
  using C = XPassCfg<N2, YT>;
  const size_t smem = C::SMEM_F2_C * sizeof(float2);
  cudaError_t e = ensure_smem(inv_x_combine_kernel<N2, YT>, smem);
  if (e != cudaSuccess) return e;
  dim3 grid(a.N1 / YT, a.N0, nsys);
  LaunchScope ls(HB_KERNEL_INV_X_COMBINE, st);
  inv_x_combine_kernel<N2, YT><<<grid, C::THREADS, smem, st>>>(a);
  return cudaGetLastError();
}

template <int N0, int N1, int Q, int THREADS>
cudaError_t launch_b(const PassArgs& a, int nslots, cudaStream_t st) {
  using C = PlaneCfg<N0, N1, Q, THREADS>;
  const size_t smem = C::SMEM_F2 * sizeof(float2);
  cudaError_t e = ensure_smem(plane_yz_kernel<N0, N1, Q, THREADS>, smem);
  if (e != cudaSuccess) return e;
  dim3 grid(2 * Q, nslots, 2 * a.N2);
  PassArgs b = a;
  // one wave of clusters ahead: co-resident clusters = SMs * (CTAs per SM) / (2Q)
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  const int per_sm = (int)((227 * 1024) / (smem + 1024));
  b.prefetch_ahead = getenv("HB_NO_L2_PREFETCH") ? 0 : sms * (per_sm < 1 ? 1 : per_sm) / (2 * Q);
  LaunchScope ls(HB_KERNEL_PLANE_YZ, st);
  plane_yz_kernel<N0, N1, Q, THREADS><<<grid, THREADS, smem, st>>>(b);
  return cudaGetLastError();
}

// Plane-pass variants for the large planes (selected by HB_PLANE_VARIANT for tuning)
struct PlaneVariant {
  const char* name;
  PassLauncher fn;
};
const PlaneVariant kPlane128[] = {
    {"q1t512", &launch_b<128, 128, 1, 512>}, {"q2t256", &launch_b<128, 128, 2, 256>},
    {"q2t128", &launch_b<128, 128, 2, 128>}, {"q4t256", &launch_b<128, 128, 4, 256>},
    {"q4t128", &launch_b<128, 128, 4, 128>},
};
const PlaneVariant kPlane64[] = {
    {"q1t256", &launch_b<64, 64, 1, 256>}, {"q2t128", &launch_b<64, 64, 2, 128>},
    {"q1t128", &launch_b<64, 64, 1, 128>}, {"q2t256", &launch_b<64, 64, 2, 256>},
};

int plane_variant_index(int nvariants) {
  const char* env = getenv("HB_PLANE_VARIANT");
  if (!env) return 0;
  int v = atoi(env);
  return (v >= 0 && v < nvariants) ? v : 0;
}

// [log2(N2)-3][log2(YT)-3]
#define HB_XROW(N2, F) {&F<N2, 8>, &F<N2, 16>}
const PassLauncher kLaunchA[7][2] = {HB_XROW(8, launch_a),   HB_XROW(16, launch_a), HB_XROW(32, launch_a),
                                     HB_XROW(64, launch_a),  HB_XROW(128, launch_a), HB_XROW(96, launch_a),
                                     HB_XROW(160, launch_a)};
const PassLauncher kLaunchC[7][2] = {HB_XROW(8, launch_c),   HB_XROW(16, launch_c), HB_XROW(32, launch_c),
                                     HB_XROW(64, launch_c),  HB_XROW(128, launch_c), HB_XROW(96, launch_c),
                                     HB_XROW(160, launch_c)};
#define HB_BROW(N0)                                                                                    \
  {&launch_b<N0, 8, 1, 128>, &launch_b<N0, 16, 1, 128>, &launch_b<N0, 32, 1, 128>, &launch_b<N0, 64, 1, 256>, \
   &launch_b<N0, 128, 1, 512>}
const PassLauncher kLaunchB[5][5] = {HB_BROW(8), HB_BROW(16), HB_BROW(32), HB_BROW(64), HB_BROW(128)};

PassLauncher plane_launcher(int N0, int N1) {
  if (N0 == 128 && N1 == 128) return kPlane128[plane_variant_index(5)].fn;
  if (N0 == 64 && N1 == 64) return kPlane64[plane_variant_index(4)].fn;
  if (N0 == 96 && N1 == 96) return &launch_b<96, 96, 1, 256>;
  if (N0 == 160 && N1 == 160) return &launch_b<160, 160, 2, 128>;
  return kLaunchB[ilog2(N0) - 3][ilog2(N1) - 3];
}

int yt_for(int N1) { return N1 < 16 ? N1 : 16; }

// Runs passes A, B, C for `nsys` systems described by `a`.
int run_normal(const hb_plan* p, PassArgs a, cudaStream_t st) {
  const int yt = yt_for(p->N1);
  const int ia = axis_index(p->N2), iy = ilog2(yt) - 3;
  const int nslots = a.nsys * a.ncoil;
  if (nslots > 65535) return fail(HB_ERR_INVALID, "too many system x coil slots in one launch (max 65535)");
  cudaError_t e = kLaunchA[ia][iy](a, nslots, st);
  if (e != cudaSuccess) return fail(HB_ERR_CUDA, std::string("pass A: ") + cudaGetErrorString(e));
  e = plane_launcher(p->N0, p->N1)(a, nslots, st);
  if (e != cudaSuccess) return fail(HB_ERR_CUDA, std::string("pass B: ") + cudaGetErrorString(e));
  e = kLaunchC[ia][iy](a, a.nsys, st);
  if (e != cudaSuccess) return fail(HB_ERR_CUDA, std::string("pass C: ") + cudaGetErrorString(e));
  return HB_OK;
}

long long image_elems(const hb_plan* p) { return (long long)p->N0 * p->N1 * p->N2; }
long long spill_elems_per_slot(const hb_plan* p) { return 2LL * image_elems(p); }
int npap_blocks(const hb_plan* p) { return (p->N1 / yt_for(p->N1)) * p->N0; }
int nrr_blocks(const hb_plan* p) {
  long long b = (image_elems(p) + 1023) / 1024;
  return (int)(b < 128 ? (b < 1 ? 1 : b) : 128);
}

struct NormalWs {
  float2* spill;
  int* coils;
  int* diag;
};
NormalWs carve_normal(Arena& ar, const hb_plan* p, int64_t nsys, int64_t ncoil) {
  NormalWs w;
  w.spill = ar.take<float2>((size_t)(nsys * ncoil) * spill_elems_per_slot(p));
  w.coils = ar.take<int>((size_t)ncoil);
  w.diag = ar.take<int>((size_t)nsys);
  return w;
}

struct CgWs {
  NormalWs n;
  float2 *r, *pv, *ap;
  double *rz, *pap, *rr;
  int *status, *active, *iters_done;
};
CgWs carve_cg(Arena& ar, const hb_plan* p, int64_t nsys, int64_t ncoil, int iters) {
  CgWs w;
  w.n = carve_normal(ar, p, nsys, ncoil);
  const size_t nv = (size_t)image_elems(p);
  w.r = ar.take<float2>(nsys * nv);
  w.pv = ar.take<float2>(nsys * nv);
  w.ap = ar.take<float2>(nsys * nv);
  w.rz = ar.take<double>(nsys * (size_t)(iters + 1));
  w.pap = ar.take<double>(nsys * (size_t)npap_blocks(p));
  w.rr = ar.take<double>(nsys * (size_t)nrr_blocks(p));
  w.status = ar.take<int>(nsys);
  w.active = ar.take<int>(nsys);
  w.iters_done = ar.take<int>(nsys);
  return w;
}

int check_plan(const hb_plan* p) {
  if (!p) return fail(HB_ERR_INVALID, "plan is NULL");
  return HB_OK;
}

int upload_indices(const int64_t* coils, int64_t ncoil, const int64_t* diag_index, int64_t s0, int64_t g,
                   int* dcoils, int* ddiag, cudaStream_t st, std::vector<int>& hc, std::vector<int>& hd) {
  hc.resize(ncoil);
  for (int64_t i = 0; i < ncoil; ++i) hc[i] = (int)coils[i];
  hd.resize(g);
  for (int64_t i = 0; i < g; ++i) hd[i] = diag_index ? (int)diag_index[s0 + i] : 0;
  HB_CUDA(cudaMemcpyAsync(dcoils, hc.data(), ncoil * sizeof(int), cudaMemcpyHostToDevice, st));
  HB_CUDA(cudaMemcpyAsync(ddiag, hd.data(), g * sizeof(int), cudaMemcpyHostToDevice, st));
  // the host vectors must outlive the copies
  HB_CUDA(cudaStreamSynchronize(st));
  return HB_OK;
}

// Twiddle tables (table_offsets layout), computed in FP64 on the host and rounded.
void fill_tables(float2* h, int N0, int N1, int N2) {
  const TableOffsets to = table_offsets(N0, N1, N2);
  auto team_table = [&](int off, int L) {
    int E = 0, S = 0;
    switch (L) {
      case 8: E = 4; S = 2; break;
      case 16: E = 4; S = 4; break;
      case 32: E = 8; S = 4; break;
      case 64: E = 8; S = 8; break;
      case 128: E = 16; S = 8; break;
      case 256: E = 16; S = 16; break;
      case 96: E = 24; S = 4; break;
      case 160: E = 40; S = 4; break;
      case 192: E = 24; S = 8; break;
      case 320: E = 40; S = 8; break;
    }
    for (int k1 = 0; k1 < E; ++k1)
      for (int t = 0; t < S; ++t) {
        const double a = -2.0 * M_PI * (double)(t * k1) / (double)L;
        h[off + k1 * S + t] = make_float2((float)std::cos(a), (float)std::sin(a));
      }
  };
  team_table(to.x, 2 * N2);
  team_table(to.row, N1);
  team_table(to.z, 2 * N0);
  for (int y = 0; y < N1; ++y) {
    const double a = -2.0 * M_PI * (double)y / (double)(2 * N1);
    h[to.par + y] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
}

// ------------------------------------------------ allocation-free Toeplitz apply ----
// The spill and the twiddle tables of hb_toeplitz_apply_noalloc live in these arrays;
// host code reaches them only through cudaGetSymbolAddress (per device).
constexpr int kNoAllocMaxTables = 2 * 160 + 160 + 2 * 160 + 160;
static __device__ __align__(256) unsigned char g_noalloc_scratch[HB_NOALLOC_SCRATCH_BYTES];
static __device__ __align__(256) float2 g_noalloc_tables[kNoAllocMaxTables];

constexpr int kNoAllocMaxDevices = 64;
struct NoAllocDevice {
  bool ready = false;
  void* scratch = nullptr;
  float2* tables = nullptr;
  int dims[3] = {0, 0, 0};  // size the device's tables currently hold
};
NoAllocDevice g_noalloc[kNoAllocMaxDevices];
std::mutex g_noalloc_mu;

}  // namespace

extern "C" {

int hb_version(void) { return 100; }

const char* hb_last_error(void) { return g_err.c_str(); }

int hb_size_supported(int64_t nz, int64_t ny, int64_t nx) {
  if (axis_index(nz) < 0 || axis_index(ny) < 0 || axis_index(nx) < 0) return 0;
  const bool plane_ok = (is_pow2_axis(nz) && is_pow2_axis(ny)) || (nz == 96 && ny == 96) || (nz == 160 && ny == 160);
  return plane_ok ? 1 : 0;
}

int hb_plan_create(hb_plan** out, int64_t nz, int64_t ny, int64_t nx, int device) {
  if (!out) return fail(HB_ERR_INVALID, "plan output pointer is NULL");
  *out = nullptr;
  if (!hb_size_supported(nz, ny, nx))
    return fail(HB_ERR_UNSUPPORTED, "image size " + std::to_string(nz) + "x" + std::to_string(ny) + "x" +
                                        std::to_string(nx) +
                                        " not supported (axes in {8,16,32,64,128}, or nz = ny in {96, 160}; nx in "
                                        "{8,16,32,64,96,128,160})");
  DeviceGuard dg(device);
  if (!dg.ok) return fail(HB_ERR_CUDA, "cannot select device " + std::to_string(device));
  hb_plan* p = new hb_plan();
  p->N0 = (int)nz;
  p->N1 = (int)ny;
  p->N2 = (int)nx;
  p->device = device;
  p->to = table_offsets(p->N0, p->N1, p->N2);
  // twiddle tables in FP64 on the host, rounded to float
  std::vector<float2> h(p->to.total);
  fill_tables(h.data(), p->N0, p->N1, p->N2);
  cudaError_t e = cudaMalloc(&p->tables, h.size() * sizeof(float2));
  if (e == cudaSuccess) e = cudaMemcpy(p->tables, h.data(), h.size() * sizeof(float2), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    if (p->tables) cudaFree(p->tables);
    delete p;
    return fail(HB_ERR_CUDA, std::string("plan tables: ") + cudaGetErrorString(e));
  }
  *out = p;
  return HB_OK;
}

int hb_plan_destroy(hb_plan* p) {
  if (!p) return HB_OK;
  DeviceGuard dg(p->device);
  if (p->tables) cudaFree(p->tables);
  delete p;
  return HB_OK;
}

int64_t hb_diag_packed_floats(const hb_plan* p) { return p ? 8LL * image_elems(p) : 0; }

int hb_diag_pack(const hb_plan* p, const void* T_complex, float* packed, void* stream) {
  if (int r = check_plan(p)) return r;
  if (!T_complex || !packed) return fail(HB_ERR_INVALID, "hb_diag_pack: NULL pointer");
  DeviceGuard dg(p->device);
  const int M0 = 2 * p->N0, M1 = 2 * p->N1, M2 = 2 * p->N2;
  const long long n = (long long)M0 * M1 * M2;
  const double scale = 1.0 / (double)n;  // inverse-FFT normalisation
  LaunchScope ls(HB_KERNEL_DIAG, (cudaStream_t)stream);
  diag_pack_kernel<float2><<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      (const float2*)T_complex, M0, M1, M2, scale, packed);
  HB_CHECK_LAUNCH();
  return HB_OK;
}

static int64_t diag_chunk(const hb_plan* p, int64_t nsamples) {
  int64_t c = 8192;
  return nsamples < c ? (nsamples < 1 ? 1 : nsamples) : c;
}

size_t hb_diag_build_workspace_bytes(const hb_plan* p, int64_t nsamples) {
  if (!p) return 0;
  Arena ar(nullptr);
  const int64_t kc = diag_chunk(p, nsamples);
  ar.take<double2>((size_t)8 * image_elems(p));
  ar.take<double2>((size_t)kc * 2 * p->N0);
  ar.take<double2>((size_t)kc * 2 * p->N1);
  ar.take<double2>((size_t)kc * 2 * p->N2);
  return ar.off + 256;
}

int hb_diag_build(const hb_plan* p, const float* coords, int64_t nsamples, float* packed, void* T_complex,
                  void* ws, size_t ws_bytes, void* stream) {
  if (int r = check_plan(p)) return r;
  if (!coords || nsamples < 1) return fail(HB_ERR_INVALID, "hb_diag_build: coords empty");
  if (!packed && !T_complex) return fail(HB_ERR_INVALID, "hb_diag_build: no output requested");
  if (!ws || ws_bytes < hb_diag_build_workspace_bytes(p, nsamples))
    return fail(HB_ERR_WORKSPACE, "hb_diag_build: workspace too small");
  DeviceGuard dg(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int M0 = 2 * p->N0, M1 = 2 * p->N1, M2 = 2 * p->N2;
  const long long n = (long long)M0 * M1 * M2;
  const int64_t kc = diag_chunk(p, nsamples);
  Arena ar(ws);
  double2* acc = ar.take<double2>((size_t)n);
  double2* Dz = ar.take<double2>((size_t)kc * M0);
  double2* Dy = ar.take<double2>((size_t)kc * M1);
  double2* Dx = ar.take<double2>((size_t)kc * M2);
  HB_CUDA(cudaMemsetAsync(acc, 0, (size_t)n * sizeof(double2), st));
  for (int64_t j0 = 0; j0 < nsamples; j0 += kc) {
    const int nj = (int)((nsamples - j0) < kc ? (nsamples - j0) : kc);
    const double2* tabs[3] = {Dz, Dy, Dx};
    const int Ms[3] = {M0, M1, M2};
    for (int ax = 0; ax < 3; ++ax) {
      const long long cnt = (long long)nj * Ms[ax];
      LaunchScope ls(HB_KERNEL_DIAG, st);
      dirichlet_table_kernel<<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(coords + ax * nsamples, j0, nj, Ms[ax],
                                                                             (double2*)tabs[ax]);
      HB_CHECK_LAUNCH();
    }
    LaunchScope ls(HB_KERNEL_DIAG, st);
    if (T_complex) {
      dim3 grid((M2 + kDiagTileX - 1) / kDiagTileX, (M1 + 63) / 64, M0);
      diag_accumulate_kernel<true, 4><<<grid, 256, 0, st>>>(Dz, Dy, Dx, nj, M0, M1, M2, acc);
    } else {
      dim3 grid((M2 + kDiagTileX - 1) / kDiagTileX, (M1 + 127) / 128, M0);
      diag_accumulate_kernel<false, 8><<<grid, 256, 0, st>>>(Dz, Dy, Dx, nj, M0, M1, M2, acc);
    }
    HB_CHECK_LAUNCH();
  }
  const double psf_scale = 1.0 / (double)n;
  if (T_complex) {
    LaunchScope ls(HB_KERNEL_DIAG, st);
    diag_to_complex_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(acc, n, psf_scale, (float2*)T_complex);
    HB_CHECK_LAUNCH();
  }
  if (packed) {
    LaunchScope ls(HB_KERNEL_DIAG, st);
    diag_pack_kernel<double2><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(acc, M0, M1, M2, psf_scale / (double)n,
                                                                          packed);
    HB_CHECK_LAUNCH();
  }
  return HB_OK;
}

size_t hb_normal_workspace_bytes(const hb_plan* p, int64_t nsys, int64_t ncoil) {
  if (!p || nsys < 1 || ncoil < 1) return 0;
  Arena ar(nullptr);
  carve_normal(ar, p, nsys, ncoil);
  return ar.off + 256;
}

int hb_toeplitz_apply(const hb_plan* p, const void* in, void* out, int64_t out_ldz, int64_t out_ldy, const void* mul,
                      int accumulate, const float* packed_diag, void* ws, size_t ws_bytes, void* stream) {
  if (int r = check_plan(p)) return r;
  if (!in || !out || !packed_diag) return fail(HB_ERR_INVALID, "hb_toeplitz_apply: NULL pointer");
  if (!ws || ws_bytes < hb_normal_workspace_bytes(p, 1, 1))
    return fail(HB_ERR_WORKSPACE, "hb_toeplitz_apply: workspace too small");
  DeviceGuard dg(p->device);
  Arena ar(ws);
  NormalWs w = carve_normal(ar, p, 1, 1);
  PassArgs a{};
  a.N0 = p->N0; a.N1 = p->N1; a.N2 = p->N2;
  a.nsys = 1; a.ncoil = 1;
  a.coils = nullptr; a.diag_of_sys = nullptr; a.active = nullptr;
  a.x = (const float2*)in;
  a.smaps = nullptr;
  a.mul = (const float2*)mul;
  a.spill = w.spill;
  a.diag = packed_diag;
  a.tables = p->tables;
  a.out = (float2*)out;
  a.out_sys_stride = 0;
  a.out_ldz = out_ldz;
  a.out_ldy = out_ldy;
  a.accumulate = accumulate ? 1 : 0;
  a.lambda = 0.f;
  a.dot_partials = nullptr;
  return run_normal(p, a, (cudaStream_t)stream);
}

int hb_sense_normal_apply(const hb_plan* p, int64_t nsys, const void* x, void* out, const void* smaps,
                          const int64_t* coils, int64_t ncoil, const float* packed_diags, const int64_t* diag_index,
                          float lambda, void* ws, size_t ws_bytes, void* stream) {
  if (int r = check_plan(p)) return r;
  if (nsys < 1 || ncoil < 1) return fail(HB_ERR_INVALID, "hb_sense_normal_apply: nsys and ncoil must be >= 1");
  if (!x || !out || !smaps || !coils || !packed_diags) return fail(HB_ERR_INVALID, "hb_sense_normal_apply: NULL pointer");
  const size_t one = hb_normal_workspace_bytes(p, 1, ncoil);
  if (!ws || ws_bytes < one) return fail(HB_ERR_WORKSPACE, "hb_sense_normal_apply: workspace too small");
  DeviceGuard dg(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  int64_t g = nsys;
  while (g > 1 && hb_normal_workspace_bytes(p, g, ncoil) > ws_bytes) g = (g + 1) / 2;
  while (g * ncoil > 65535) g = (g + 1) / 2;
  const long long nv = image_elems(p);
  std::vector<int> hc, hd;
  for (int64_t s0 = 0; s0 < nsys; s0 += g) {
    const int64_t gg = (nsys - s0) < g ? (nsys - s0) : g;
    Arena ar(ws);
    NormalWs w = carve_normal(ar, p, gg, ncoil);
    if (int r = upload_indices(coils, ncoil, diag_index, s0, gg, w.coils, w.diag, st, hc, hd)) return r;
    PassArgs a{};
    a.N0 = p->N0; a.N1 = p->N1; a.N2 = p->N2;
    a.nsys = (int)gg; a.ncoil = (int)ncoil;
    a.coils = w.coils; a.diag_of_sys = w.diag; a.active = nullptr;
    a.x = (const float2*)x + s0 * nv;
    a.smaps = (const float2*)smaps;
    a.mul = nullptr;
    a.spill = w.spill;
    a.diag = packed_diags;
    a.tables = p->tables;
    a.out = (float2*)out + s0 * nv;
    a.out_sys_stride = nv;
    a.out_ldz = (long long)p->N1 * p->N2;
    a.out_ldy = p->N2;
    a.accumulate = 0;
    a.lambda = lambda;
    a.dot_partials = nullptr;
    if (int r = run_normal(p, a, st)) return r;
  }
  return HB_OK;
}

size_t hb_cg_workspace_bytes(const hb_plan* p, int64_t nsys, int64_t ncoil, int iters) {
  if (!p || nsys < 1 || ncoil < 1 || iters < 0) return 0;
  Arena ar(nullptr);
  carve_cg(ar, p, nsys, ncoil, iters);
  return ar.off + 256;
}

int hb_cg_run(const hb_plan* p, int64_t nsys, void* x, const void* b, const void* smaps, const int64_t* coils,
              int64_t ncoil, const float* packed_diags, const int64_t* diag_index, float lambda, int iters, double tol,
              int32_t* status_host, int32_t* iters_done_host, void* ws, size_t ws_bytes, void* stream) {
  if (int r = check_plan(p)) return r;
  if (nsys < 1 || ncoil < 1) return fail(HB_ERR_INVALID, "hb_cg_run: nsys and ncoil must be >= 1");
  if (!x || !b || !smaps || !coils || !packed_diags) return fail(HB_ERR_INVALID, "hb_cg_run: NULL pointer");
  if (iters < 1) {
    for (int64_t s = 0; s < nsys; ++s) {
      if (status_host) status_host[s] = HB_CG_RUNNING;
      if (iters_done_host) iters_done_host[s] = 0;
    }
    return HB_OK;  // ConjugateGradient::run returns immediately for iter < 1
  }
  if (!ws || ws_bytes < hb_cg_workspace_bytes(p, 1, ncoil, iters))
    return fail(HB_ERR_WORKSPACE, "hb_cg_run: workspace too small");
  DeviceGuard dg(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  int64_t g = nsys;
  while (g > 1 && hb_cg_workspace_bytes(p, g, ncoil, iters) > ws_bytes) g = (g + 1) / 2;
  while (g * ncoil > 65535) g = (g + 1) / 2;
  const long long nv = image_elems(p);
  const int nrr = nrr_blocks(p);
  std::vector<int> hc, hd;
  std::vector<int> stat_all(nsys), done_all(nsys);
  for (int64_t s0 = 0; s0 < nsys; s0 += g) {
    const int64_t gg = (nsys - s0) < g ? (nsys - s0) : g;
    Arena ar(ws);
    CgWs w = carve_cg(ar, p, gg, ncoil, iters);
    if (int r = upload_indices(coils, ncoil, diag_index, s0, gg, w.n.coils, w.n.diag, st, hc, hd)) return r;
    PassArgs a{};
    a.N0 = p->N0; a.N1 = p->N1; a.N2 = p->N2;
    a.nsys = (int)gg; a.ncoil = (int)ncoil;
    a.coils = w.n.coils; a.diag_of_sys = w.n.diag; a.active = nullptr;
    a.x = (const float2*)x + s0 * nv;
    a.smaps = (const float2*)smaps;
    a.mul = nullptr;
    a.spill = w.n.spill;
    a.diag = packed_diags;
    a.tables = p->tables;
    a.out = w.ap;
    a.out_sys_stride = nv;
    a.out_ldz = (long long)p->N1 * p->N2;
    a.out_ldy = p->N2;
    a.accumulate = 0;
    a.lambda = lambda;
    a.dot_partials = nullptr;
    // r = b - (A + lambda I) x
    if (int r = run_normal(p, a, st)) return r;
    CgState s{};
    s.nsys = (int)gg;
    s.nv = nv;
    s.x = (float2*)x + s0 * nv;
    s.b = (const float2*)b + s0 * nv;
    s.r = w.r; s.p = w.pv; s.ap = w.ap;
    s.rz = w.rz; s.rz_ld = iters + 1;
    s.status = w.status; s.active = w.active; s.iters_done = w.iters_done;
    s.pap_part = w.pap; s.npap = npap_blocks(p);
    s.rr_part = w.rr;
    s.tol = tol;
    dim3 ugrid(nrr, (unsigned)gg);
    {
      LaunchScope ls(HB_KERNEL_CG_UPDATE, st);
      cg_init_kernel<<<ugrid, 256, 0, st>>>(s);
    }
    HB_CHECK_LAUNCH();
    {
      LaunchScope ls(HB_KERNEL_CG_UPDATE, st);
      cg_init_finish_kernel<<<(unsigned)gg, 256, 0, st>>>(s, nrr);
    }
    HB_CHECK_LAUNCH();
    a.x = w.pv;
    a.active = w.active;
    a.dot_partials = w.pap;
    for (int it = 0; it < iters; ++it) {
      if (int r = run_normal(p, a, st)) return r;
      {
        LaunchScope ls(HB_KERNEL_CG_UPDATE, st);
        cg_step_xr_kernel<<<ugrid, 256, 0, st>>>(s, it);
      }
      HB_CHECK_LAUNCH();
      {
        LaunchScope ls(HB_KERNEL_CG_UPDATE, st);
        cg_step_p_kernel<<<ugrid, 256, 0, st>>>(s, it);
      }
      HB_CHECK_LAUNCH();
    }
    HB_CUDA(cudaMemcpyAsync(stat_all.data() + s0, w.status, gg * sizeof(int), cudaMemcpyDeviceToHost, st));
    HB_CUDA(cudaMemcpyAsync(done_all.data() + s0, w.iters_done, gg * sizeof(int), cudaMemcpyDeviceToHost, st));
  }
  HB_CUDA(cudaStreamSynchronize(st));
  bool notpd = false;
  for (int64_t s = 0; s < nsys; ++s) {
    if (status_host) status_host[s] = stat_all[s];
    if (iters_done_host) iters_done_host[s] = done_all[s];
    if (stat_all[s] == kCgNotPD) notpd = true;
  }
  if (notpd) return fail(HB_ERR_NOT_PD, "A was not positive definite");
  return HB_OK;
}

int hb_toeplitz_apply_noalloc(int64_t nz, int64_t ny, int64_t nx, const void* in, void* out, int64_t out_ldz,
                              int64_t out_ldy, const void* mul, int accumulate, const float* packed_diag,
                              void* stream) {
  if (!hb_size_supported(nz, ny, nx))
    return fail(HB_ERR_UNSUPPORTED, "hb_toeplitz_apply_noalloc: image size not supported");
  if (!in || !out || !packed_diag) return fail(HB_ERR_INVALID, "hb_toeplitz_apply_noalloc: NULL pointer");
  const unsigned long long need = 16ull * (unsigned long long)(nz * ny * nx);
  if (need > HB_NOALLOC_SCRATCH_BYTES)
    return fail(HB_ERR_WORKSPACE, "hb_toeplitz_apply_noalloc: " + std::to_string(nz) + "x" + std::to_string(ny) + "x" +
                                      std::to_string(nx) + " needs " + std::to_string(need) +
                                      " bytes of scratch, more than the built-in " +
                                      std::to_string((unsigned long long)HB_NOALLOC_SCRATCH_BYTES) +
                                      " (use hb_toeplitz_apply with a caller workspace)");
  int dev = 0;
  HB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(HB_ERR_INVALID, "hb_toeplitz_apply_noalloc: device index");
  cudaStream_t st = (cudaStream_t)stream;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  NoAllocDevice& d = g_noalloc[dev];
  if (!d.ready) {  // once per device, with that device current
    HB_CUDA(cudaGetSymbolAddress(&d.scratch, g_noalloc_scratch));
    HB_CUDA(cudaGetSymbolAddress((void**)&d.tables, g_noalloc_tables));
    d.ready = true;
  }
  if (d.dims[0] != nz || d.dims[1] != ny || d.dims[2] != nx) {
    float2 h[kNoAllocMaxTables];  // host stack, no heap
    fill_tables(h, (int)nz, (int)ny, (int)nx);
    const int n = table_offsets((int)nz, (int)ny, (int)nx).total;
    HB_CUDA(cudaMemcpyAsync(d.tables, h, n * sizeof(float2), cudaMemcpyHostToDevice, st));
    HB_CUDA(cudaStreamSynchronize(st));  // the host array leaves scope
    d.dims[0] = (int)nz;
    d.dims[1] = (int)ny;
    d.dims[2] = (int)nx;
  }
  hb_plan p;
  p.N0 = (int)nz;
  p.N1 = (int)ny;
  p.N2 = (int)nx;
  p.device = dev;
  p.tables = d.tables;
  p.to = table_offsets(p.N0, p.N1, p.N2);
  PassArgs a{};
  a.N0 = p.N0; a.N1 = p.N1; a.N2 = p.N2;
  a.nsys = 1; a.ncoil = 1;
  a.coils = nullptr; a.diag_of_sys = nullptr; a.active = nullptr;
  a.x = (const float2*)in;
  a.smaps = nullptr;
  a.mul = (const float2*)mul;
  a.spill = (float2*)d.scratch;
  a.diag = packed_diag;
  a.tables = d.tables;
  a.out = (float2*)out;
  a.out_sys_stride = 0;
  a.out_ldz = out_ldz;
  a.out_ldy = out_ldy;
  a.accumulate = accumulate ? 1 : 0;
  a.lambda = 0.f;
  a.dot_partials = nullptr;
  return run_normal(&p, a, st);
}

uint64_t hb_launch_count(void) { return g_launches.load(); }

int hb_profile_start(void) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  for (auto& r : g_prof) {
    g_ev_pool.push_back(r.a);
    g_ev_pool.push_back(r.b);
  }
  g_prof.clear();
  g_prof_on.store(true);
  return HB_OK;
}

int hb_profile_stop(double* ms, int64_t* launches, int nkinds) {
  g_prof_on.store(false);
  std::vector<ProfRec> recs;
  {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    recs.swap(g_prof);
  }
  for (int k = 0; k < nkinds; ++k) {
    if (ms) ms[k] = 0.0;
    if (launches) launches[k] = 0;
  }
  int rc = HB_OK;
  for (auto& r : recs) {
    float t = 0.f;
    cudaError_t e = cudaEventSynchronize(r.b);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, r.a, r.b);
    if (e != cudaSuccess) rc = fail(HB_ERR_CUDA, std::string("profile events: ") + cudaGetErrorString(e));
    if (r.kind >= 0 && r.kind < nkinds) {
      if (ms) ms[r.kind] += t;
      if (launches) launches[r.kind] += 1;
    }
  }
  std::lock_guard<std::mutex> lk(g_prof_mu);
  for (auto& r : recs) {
    g_ev_pool.push_back(r.a);
    g_ev_pool.push_back(r.b);
  }
  return rc;
}

}  // extern "C"
