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
#include "fft3_launch.cuh"
#include "runtime.cuh"
#include "tc_kernels.cuh"
#include "toeplitz_kernels.cuh"

using namespace hb;

struct hb_plan {
  int N0, N1, N2;
  int device;
  float2* tables;  // device twiddle tables (table_offsets layout)
  TableOffsets to;
  int plane_variant = -1;  // plane-pass schedule chosen by hb_plan_autotune (-1: default)
  int precision = HB_PRECISION_FP32;
  unsigned char* tc_ftab = nullptr;  // tensor-core pass A: DFT rows in operand layout
  int* tc_wait_error = nullptr;      // device address of g_tc_wait_error
  int tc_stall_chunk = -1;           // fault injection for tests (hb_plan_inject_tc_stall)
  int x_stall_coil = -1;             // fault injection for tests (hb_plan_inject_x_stall)
};

namespace hb {
void plan_geometry(const ::hb_plan* p, int* N, int* device) {
  N[0] = p->N0;
  N[1] = p->N1;
  N[2] = p->N2;
  *device = p->device;
}
const float2* plan_image_tables(const ::hb_plan* p) { return p->tables + p->to.total; }
}  // namespace hb

namespace {

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


// Opt-in to large dynamic shared memory, once per kernel and device (the first call of
// a kernel on a device happens outside any stream capture).
template <auto kernel>
cudaError_t ensure_smem(size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  static std::atomic<uint64_t> done{0};  // one flag set per kernel, one bit per device
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = 1ull << (dev & 63);
  if (done.load() & bit) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) done.fetch_or(bit);
  return e;
}

// ---------------------------------------------------------------- pass launchers ----
using PassLauncher = cudaError_t (*)(const PassArgs&, int, cudaStream_t);

// Set by the tensor-core pass when an mbarrier wait gave up (read and cleared by
// hb_wait_status).
__device__ int g_tc_wait_error;

// Reads and clears g_tc_wait_error on the current device (synchronous; outside captures):
// HB_ERR_CUDA with a message if a tensor-core pass gave up waiting.
int tc_wait_check() {
  int flag = 0;
  const int zero = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&flag, g_tc_wait_error, sizeof(int));
  if (e == cudaSuccess && flag) e = cudaMemcpyToSymbol(g_tc_wait_error, &zero, sizeof(int));
  if (e != cudaSuccess) return fail(HB_ERR_CUDA, std::string("tensor-core wait flag: ") + cudaGetErrorString(e));
  if (flag)
    return fail(HB_ERR_CUDA, "a pass gave up waiting for a bulk copy, its operands or its contractions (about 1 s); "
                             "its output is incomplete");
  return HB_OK;
}

cudaError_t launch_a_tc(const hb_plan* p, const PassArgs& a, cudaStream_t st) {
  cudaError_t e = ensure_smem<expand_fwd_x_tc_kernel<128>>(tc::kSmemBytes);
  if (e != cudaSuccess) return e;
  dim3 grid(a.N0, a.nslots);
  LaunchScope ls(HB_KERNEL_EXPAND_FWD_X, st);
  expand_fwd_x_tc_kernel<128><<<grid, tc::kThreadsAll, tc::kSmemBytes, st>>>(a, p->tc_ftab, p->tc_wait_error,
                                                                             p->tc_stall_chunk);
  return cudaGetLastError();
}

uint16_t bf16_bits_rn(float f) {  // round to nearest even (finite inputs)
  uint32_t u;
  memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}
double bf16_value(uint16_t b) {
  const uint32_t u = (uint32_t)b << 16;
  float f;
  memcpy(&f, &u, 4);
  return (double)f;
}

// Forward DFT rows F[kx][x] = exp(-2 pi i kx x / M2) (kx < M2, x < N2) in the tensor-core
// pass's operand layout: [16-sample chunk][re_hi, re_lo, im_hi, im_lo] blocks of
// tc::kArrF bytes, element (kx, x) at tc::operand_offset(kx, x % 16); hi = bf16(v),
// lo = bf16(v - hi), v in FP64.
std::vector<uint16_t> tc_dft_table(int N2) {
  const int M2 = 2 * N2, nch = N2 / tc::kKc;
  const size_t arr = tc::kArrF / 2;  // uint16 per array
  std::vector<uint16_t> t((size_t)nch * 4 * arr);
  for (int kx = 0; kx < M2; ++kx)
    for (int x = 0; x < N2; ++x) {
      const long long m = ((long long)kx * x) % M2;
      const double ang = -2.0 * M_PI * (double)m / (double)M2;
      const double v[2] = {std::cos(ang), std::sin(ang)};
      const size_t blk = (size_t)(x / tc::kKc);
      const size_t off = (size_t)tc::operand_offset(kx, x % tc::kKc) / 2;
      for (int c = 0; c < 2; ++c) {
        const uint16_t hi = bf16_bits_rn((float)v[c]);
        const uint16_t lo = bf16_bits_rn((float)(v[c] - bf16_value(hi)));
        t[(blk * 4 + 2 * c) * arr + off] = hi;
        t[(blk * 4 + 2 * c + 1) * arr + off] = lo;
      }
    }
  return t;
}

template <int N2, int YT>
cudaError_t launch_a(const PassArgs& a, int nsys, cudaStream_t st) {
  using C = XPassCfg<N2, YT>;
  const size_t smem = C::SMEM_F2 * sizeof(float2);
  cudaError_t e = ensure_smem<expand_fwd_x_kernel<N2, YT>>(smem);
  if (e != cudaSuccess) return e;
  dim3 grid(a.N1 / YT, a.N0, nsys);
  LaunchScope ls(HB_KERNEL_EXPAND_FWD_X, st);
  expand_fwd_x_kernel<N2, YT><<<grid, C::THREADS, smem, st>>>(a);
  return cudaGetLastError();
}

template <int N2, int YT>
cudaError_t launch_c(const PassArgs& a, int nsys, cudaStream_t st) {
  using C = XPassCfg<N2, YT>;
  const size_t smem = C::SMEM_F2_C * sizeof(float2);
  cudaError_t e = ensure_smem<inv_x_combine_kernel<N2, YT>>(smem);
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
  cudaError_t e = ensure_smem<plane_yz_kernel<N0, N1, Q, THREADS>>(smem);
  if (e != cudaSuccess) return e;
  // persistent: as many clusters as can be co-resident (cached per kernel and device)
  static std::atomic<int> cached[64];
  int dev = 0;
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int ncl = cached[dev & 63].load();
  if (ncl <= 0) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * Q, 1, 1);
    cfg.blockDim = dim3(THREADS, 1, 1);
    cfg.dynamicSmemBytes = smem;
    e = cudaOccupancyMaxActiveClusters(&ncl, plane_yz_kernel<N0, N1, Q, THREADS>, &cfg);
    if (e != cudaSuccess) return e;
    if (ncl < 1) ncl = 1;
    cached[dev & 63].store(ncl);
  }
  const long long nitems = (long long)nslots * 2 * a.N2;
  if (ncl > nitems) ncl = (int)nitems;
  if (ncl > 65535) ncl = 65535;
  dim3 grid(2 * Q, ncl, 1);
  const PassArgs& b = a;
  LaunchScope ls(HB_KERNEL_PLANE_YZ, st);
  plane_yz_kernel<N0, N1, Q, THREADS><<<grid, THREADS, smem, st>>>(b);
  return cudaGetLastError();
}

template <int N0, int N1, int K, int THREADS>
cudaError_t launch_bmod(const PassArgs& a, int nslots, cudaStream_t st) {
  using C = PlaneModCfg<N0, N1, K, THREADS>;
  const size_t smem = C::SMEM_F2 * sizeof(float2);
  cudaError_t e = ensure_smem<plane_mod_kernel<N0, N1, K, THREADS>>(smem);
  if (e != cudaSuccess) return e;
  dim3 grid(K, nslots, 2 * a.N2);
  // one wave of clusters ahead: as many clusters as can be co-resident
  static std::atomic<int> ahead[64];
  int dev = 0;
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int pa = ahead[dev & 63].load();
  if (pa <= 0) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(K, 1, 1);
    cfg.blockDim = dim3(THREADS, 1, 1);
    cfg.dynamicSmemBytes = smem;
    int ncl = 0;
    e = cudaOccupancyMaxActiveClusters(&ncl, plane_mod_kernel<N0, N1, K, THREADS>, &cfg);
    if (e != cudaSuccess) return e;
    pa = ncl < 1 ? 1 : ncl;
    ahead[dev & 63].store(pa);
  }
  PassArgs b = a;
  b.prefetch_ahead = getenv("HB_NO_L2_PREFETCH") ? 0 : pa;
  LaunchScope ls(HB_KERNEL_PLANE_YZ, st);
  plane_mod_kernel<N0, N1, K, THREADS><<<grid, THREADS, smem, st>>>(b);
  return cudaGetLastError();
}

// Plane-pass schedules (cluster split Q x CTA size) per plane size; hb_plan_autotune
// times them, HB_PLANE_VARIANT overrides, index 0 is the default.
struct PlaneVariant {
  const char* name;
  PassLauncher fn;
};
const PlaneVariant kPlane128[] = {
    {"mod4t256", &launch_bmod<128, 128, 4, 256>}, {"q1t512", &launch_b<128, 128, 1, 512>},
    {"q2t256", &launch_b<128, 128, 2, 256>},      {"q2t128", &launch_b<128, 128, 2, 128>},
    {"q4t256", &launch_b<128, 128, 4, 256>},      {"q4t128", &launch_b<128, 128, 4, 128>},
    {"mod4t512", &launch_bmod<128, 128, 4, 512>}, {"mod4t128", &launch_bmod<128, 128, 4, 128>},
    {"mod8t256", &launch_bmod<128, 128, 8, 256>}, {"mod8t128", &launch_bmod<128, 128, 8, 128>},
};
const PlaneVariant kPlane64[] = {
    {"q1t256", &launch_b<64, 64, 1, 256>}, {"q2t128", &launch_b<64, 64, 2, 128>},
    {"q1t128", &launch_b<64, 64, 1, 128>}, {"q2t256", &launch_b<64, 64, 2, 256>},
    {"mod4t256", &launch_bmod<64, 64, 4, 256>}, {"mod4t128", &launch_bmod<64, 64, 4, 128>},
    {"mod8t128", &launch_bmod<64, 64, 8, 128>},
};
const PlaneVariant kPlane96[] = {
    {"q1t256", &launch_b<96, 96, 1, 256>}, {"q2t128", &launch_b<96, 96, 2, 128>},
    {"q2t256", &launch_b<96, 96, 2, 256>},
};
const PlaneVariant kPlane160[] = {
    {"q2t128", &launch_b<160, 160, 2, 128>}, {"q4t128", &launch_b<160, 160, 4, 128>},
};

const PlaneVariant* plane_variants(int N0, int N1, int* n) {
  *n = 0;
  if (N0 == 128 && N1 == 128) { *n = 10; return kPlane128; }
  if (N0 == 64 && N1 == 64) { *n = 7; return kPlane64; }
  if (N0 == 96 && N1 == 96) { *n = 3; return kPlane96; }
  if (N0 == 160 && N1 == 160) { *n = 2; return kPlane160; }
  return nullptr;
}

int plane_variant_index(int nvariants, int chosen) {
  const char* env = getenv("HB_PLANE_VARIANT");
  if (env) {
    int v = atoi(env);
    return (v >= 0 && v < nvariants) ? v : 0;
  }
  return (chosen >= 0 && chosen < nvariants) ? chosen : 0;
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

PassLauncher plane_launcher(const hb_plan* p) {
  int n = 0;
  const PlaneVariant* v = plane_variants(p->N0, p->N1, &n);
  if (v) return v[plane_variant_index(n, p->plane_variant)].fn;
  return kLaunchB[ilog2(p->N0) - 3][ilog2(p->N1) - 3];
}

int yt_for(int N1) { return N1 < 16 ? N1 : 16; }

// Runs passes A, B, C for `nsys` systems described by `a`.
int run_normal(const hb_plan* p, PassArgs a, cudaStream_t st) {
  const int yt = yt_for(p->N1);
  const int ia = axis_index(p->N2), iy = ilog2(yt) - 3;
  const int nslots = a.nslots;
  if (nslots > 65535) return fail(HB_ERR_INVALID, "too many system x coil slots in one launch (max 65535)");
  cudaError_t e = p->precision == HB_PRECISION_BF16X3 ? launch_a_tc(p, a, st) : kLaunchA[ia][iy](a, a.nsys, st);
  if (e != cudaSuccess) return fail(HB_ERR_CUDA, std::string("pass A: ") + cudaGetErrorString(e));
  e = plane_launcher(p)(a, nslots, st);
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

int check_plan(const hb_plan* p) {
  if (!p) return fail(HB_ERR_INVALID, "plan is NULL");
  return HB_OK;
}

// ------------------------------------------------------------- system tables ----
// Per-group descriptor tables live in one block of the workspace and are uploaded with
// a single copy.  Layout (byte offsets within the block) is computed identically on
// the host.
struct TableLayout {
  size_t sys_x_init, sys_x_iter, sys_out, sys_smaps, sys_diag, cg_x, cg_b;  // pointer arrays
  size_t sys_pdiag;                                                           // pointer array
  size_t sys_lambda;                                                          // float array
  size_t slot_sys, slot_coil, sys_slot0, sys_nslot;                           // int arrays
  size_t bytes;
};
TableLayout table_layout(int64_t g, int64_t slots) {
  TableLayout L;
  size_t o = 0;
  auto take = [&](size_t n) {
    o = (o + 15) & ~size_t(15);
    size_t r = o;
    o += n;
    return r;
  };
  L.sys_x_init = take(8 * g);
  L.sys_x_iter = take(8 * g);
  L.sys_out = take(8 * g);
  L.sys_smaps = take(8 * g);
  L.sys_diag = take(8 * g);
  L.cg_x = take(8 * g);
  L.cg_b = take(8 * g);
  L.sys_pdiag = take(8 * g);
  L.sys_lambda = take(4 * g);
  L.slot_sys = take(4 * slots);
  L.slot_coil = take(4 * slots);
  L.sys_slot0 = take(4 * g);
  L.sys_nslot = take(4 * g);
  L.bytes = (o + 255) & ~size_t(255);
  return L;
}

struct GroupWs {
  float2* spill;
  char* tables;
  TableLayout L;
  // CG state (null when not a CG group)
  float2 *r, *pv, *ap, *z;
  double *rz, *pap, *rr;
  int *status, *active, *iters_done, *iter;
};

GroupWs carve_group(Arena& ar, const hb_plan* p, int64_t g, int64_t slots, int iters, bool cg) {
  GroupWs w{};
  w.spill = ar.take<float2>((size_t)slots * spill_elems_per_slot(p));
  w.L = table_layout(g, slots);
  w.tables = ar.take<char>(w.L.bytes);
  if (cg) {
    const size_t nv = (size_t)image_elems(p);
    w.r = ar.take<float2>(g * nv);
    w.pv = ar.take<float2>(g * nv);
    w.ap = ar.take<float2>(g * nv);
    w.z = ar.take<float2>(g * nv);
    w.rz = ar.take<double>(g * (size_t)(iters + 1));
    w.pap = ar.take<double>(g * (size_t)npap_blocks(p));
    w.rr = ar.take<double>(g * (size_t)nrr_blocks(p));
    w.status = ar.take<int>(g);
    w.active = ar.take<int>(g);
    w.iters_done = ar.take<int>(g);
    w.iter = ar.take<int>(1);
  }
  return w;
}

size_t group_bytes(const hb_plan* p, int64_t g, int64_t slots, int iters, bool cg) {
  Arena ar(nullptr);
  carve_group(ar, p, g, slots, iters, cg);
  return ar.off + 256;
}

// Fills the host image of the tables of systems [s0, s0 + g) (h has L.bytes bytes).
void fill_group_tables(char* h, const hb_plan* p, const GroupWs& w, const hb_system* sys, int64_t s0, int64_t g,
                       bool cg) {
  const TableLayout& L = w.L;
  std::memset(h, 0, L.bytes);
  auto put_ptr = [&](size_t off, int64_t i, const void* v) { std::memcpy(h + off + 8 * i, &v, 8); };
  auto put_int = [&](size_t off, int64_t i, int v) { std::memcpy(h + off + 4 * i, &v, 4); };
  const size_t nv = (size_t)image_elems(p);
  int slot = 0;
  for (int64_t i = 0; i < g; ++i) {
    const hb_system& q = sys[s0 + i];
    if (cg) {
      put_ptr(L.sys_x_init, i, q.x);
      put_ptr(L.sys_x_iter, i, w.pv + i * nv);
      put_ptr(L.sys_out, i, w.ap + i * nv);
      put_ptr(L.cg_x, i, q.x);
      put_ptr(L.cg_b, i, q.b);
    } else {
      put_ptr(L.sys_x_init, i, q.x);
      put_ptr(L.sys_x_iter, i, q.x);
      put_ptr(L.sys_out, i, q.out);
    }
    put_ptr(L.sys_smaps, i, q.smaps);
    put_ptr(L.sys_pdiag, i, cg ? q.precond : nullptr);
    put_ptr(L.sys_diag, i, q.packed_diag);
    float lam = q.lambda;
    std::memcpy(h + L.sys_lambda + 4 * i, &lam, 4);
    put_int(L.sys_slot0, i, slot);
    put_int(L.sys_nslot, i, (int)q.ncoil);
    for (int64_t c = 0; c < q.ncoil; ++c, ++slot) {
      put_int(L.slot_sys, slot, (int)i);
      put_int(L.slot_coil, slot, (int)q.coils[c]);
    }
  }
}

// Fills and uploads the tables.  Synchronises `st` (the host image is local).
int upload_tables(const hb_plan* p, const GroupWs& w, const hb_system* sys, int64_t s0, int64_t g, bool cg,
                  cudaStream_t st) {
  std::vector<char> h(w.L.bytes);
  fill_group_tables(h.data(), p, w, sys, s0, g, cg);
  HB_CUDA(cudaMemcpyAsync(w.tables, h.data(), w.L.bytes, cudaMemcpyHostToDevice, st));
  HB_CUDA(cudaStreamSynchronize(st));
  return HB_OK;
}

PassArgs group_pass_args(const hb_plan* p, const GroupWs& w, int64_t g, int64_t slots, bool iter_inputs) {
  PassArgs a{};
  a.N0 = p->N0; a.N1 = p->N1; a.N2 = p->N2;
  a.nsys = (int)g;
  a.nslots = (int)slots;
  const char* t = w.tables;
  a.slot_sys = (const int*)(t + w.L.slot_sys);
  a.slot_coil = (const int*)(t + w.L.slot_coil);
  a.sys_slot0 = (const int*)(t + w.L.sys_slot0);
  a.sys_nslot = (const int*)(t + w.L.sys_nslot);
  a.active = nullptr;
  a.sys_x = (const float2* const*)(t + (iter_inputs ? w.L.sys_x_iter : w.L.sys_x_init));
  a.sys_out = (float2* const*)(t + w.L.sys_out);
  a.sys_smaps = (const float2* const*)(t + w.L.sys_smaps);
  a.sys_diag = (const float* const*)(t + w.L.sys_diag);
  a.sys_lambda = (const float*)(t + w.L.sys_lambda);
  a.mul = nullptr;
  a.spill = w.spill;
  a.tables = p->tables;
  a.out_ldz = (long long)p->N1 * p->N2;
  a.out_ldy = p->N2;
  a.accumulate = 0;
  a.dot_partials = nullptr;
  a.wait_error = p->tc_wait_error;
  a.inject_stall = p->x_stall_coil + 1;
  return a;
}

// The plane pass reads each packed z column with 16-byte vector loads.
bool diag_aligned(const float* d) { return ((uintptr_t)d & 15u) == 0; }
// Passes A and C move spill tiles with bulk copies, which need 16-byte aligned addresses;
// the workspace is carved at 256-byte offsets from its start.
bool ws_aligned(const void* w) { return ((uintptr_t)w & 15u) == 0; }

int validate_systems(const hb_plan* p, int64_t nsys, const hb_system* sys, bool cg) {
  if (nsys < 1 || !sys) return fail(HB_ERR_INVALID, "no systems");
  for (int64_t i = 0; i < nsys; ++i) {
    const hb_system& q = sys[i];
    if (!q.x || !q.smaps || !q.packed_diag || (q.ncoil > 0 && !q.coils))
      return fail(HB_ERR_INVALID, "system " + std::to_string(i) + ": NULL pointer");
    if (!diag_aligned(q.packed_diag))
      return fail(HB_ERR_INVALID, "system " + std::to_string(i) + ": packed diagonal not 16-byte aligned");
    if (cg ? !q.b : !q.out) return fail(HB_ERR_INVALID, "system " + std::to_string(i) + ": NULL pointer");
    if (q.ncoil < 1 || q.ncoil > 65535) return fail(HB_ERR_INVALID, "system " + std::to_string(i) + ": ncoil");
    for (int64_t c = 0; c < q.ncoil; ++c)
      if (q.coils[c] < 0) return fail(HB_ERR_INVALID, "system " + std::to_string(i) + ": negative coil index");
  }
  (void)p;
  return HB_OK;
}

// Consecutive systems [s0, s0 + g) whose workspace fits ws_bytes (at least one system).
int64_t next_group(const hb_plan* p, const hb_system* sys, int64_t s0, int64_t nsys, int iters, bool cg,
                   size_t ws_bytes, int64_t* slots_out) {
  int64_t g = 0, slots = 0;
  while (s0 + g < nsys) {
    const int64_t ns = slots + sys[s0 + g].ncoil;
    if (ns > 65535 || (g > 0 && group_bytes(p, g + 1, ns, iters, cg) > ws_bytes)) break;
    slots = ns;
    ++g;
  }
  *slots_out = slots;
  return g;
}

// ----------------------------------------------------------- graph replay state ----
struct GraphStream {
  bool ready = false;
  cudaStream_t s = nullptr;
  cudaEvent_t e1 = nullptr, e2 = nullptr;
};
GraphStream g_graph_streams[64];
std::mutex g_graph_mu;         // serialises use of the side streams
std::mutex g_graph_create_mu;  // guards their creation

int graph_stream(int dev, GraphStream** out) {
  std::lock_guard<std::mutex> lk(g_graph_create_mu);
  if (dev < 0 || dev >= 64) return fail(HB_ERR_INVALID, "device index");
  GraphStream& gs = g_graph_streams[dev];
  if (!gs.ready) {
    HB_CUDA(cudaStreamCreateWithFlags(&gs.s, cudaStreamNonBlocking));
    HB_CUDA(cudaEventCreateWithFlags(&gs.e1, cudaEventDisableTiming));
    HB_CUDA(cudaEventCreateWithFlags(&gs.e2, cudaEventDisableTiming));
    gs.ready = true;
  }
  *out = &gs;
  return HB_OK;
}

int launch_cg_update(int kind, void (*fn)(CgState), dim3 grid, const CgState& s, cudaStream_t st) {
  LaunchScope ls(kind, st);
  fn<<<grid, 256, 0, st>>>(s);
  HB_CHECK_LAUNCH();
  return HB_OK;
}

// z = P r for every system of the group (circulant preconditioner, identity for systems
// without one): forward FFT, x diagonal / nv, inverse FFT, then the Re<r, z> partials
// (and p = z at initialisation).
int cg_precondition(const hb_plan* p, const CgState& s, dim3 ugrid, int init, cudaStream_t st) {
  HB_CUDA(cudaMemcpyAsync(s.z, s.r, (size_t)s.nsys * s.nv * sizeof(float2), cudaMemcpyDeviceToDevice, st));
  const float2* tw = p->tables + p->to.total;
  HB_CUDA(fftl::fft3_grid<-1>(p->N0, p->N1, p->N2, tw, s.z, s.nsys, st, HB_KERNEL_CG_UPDATE));
  if (int r = launch_cg_update(HB_KERNEL_CG_UPDATE, cg_precond_scale_kernel, ugrid, s, st)) return r;
  HB_CUDA(fftl::fft3_grid<1>(p->N0, p->N1, p->N2, tw, s.z, s.nsys, st, HB_KERNEL_CG_UPDATE));
  {
    LaunchScope ls(HB_KERNEL_CG_UPDATE, st);
    cg_rz_kernel<<<ugrid, 256, 0, st>>>(s, init);
  }
  HB_CHECK_LAUNCH();
  return HB_OK;
}
constexpr int kKernelsPerPrecondition = 8;  // 2 x 3 FFT passes, scale, partials

// One CG iteration for a group: normal op with partials, x/r update, [z = P r], p update,
// advance.
int cg_iteration(const hb_plan* p, const PassArgs& a, const CgState& s, dim3 ugrid, int* iter, cudaStream_t st) {
  if (int r = run_normal(p, a, st)) return r;
  if (int r = launch_cg_update(HB_KERNEL_CG_UPDATE, cg_step_xr_kernel, ugrid, s, st)) return r;
  if (s.z)
    if (int r = cg_precondition(p, s, ugrid, 0, st)) return r;
  if (int r = launch_cg_update(HB_KERNEL_CG_UPDATE, cg_step_p_kernel, ugrid, s, st)) return r;
  {
    LaunchScope ls(HB_KERNEL_CG_UPDATE, st);
    cg_advance_kernel<<<1, 1, 0, st>>>(iter);
  }
  HB_CHECK_LAUNCH();
  return HB_OK;
}
constexpr int kKernelsPerCgIteration = 6;

int cg_systems_impl(const hb_plan* p, int64_t nsys, const hb_system* sys, int iters, double tol, int flags,
                    int32_t* status_host, int32_t* iters_done_host, void* ws, size_t ws_bytes, cudaStream_t st) {
  if (int r = validate_systems(p, nsys, sys, true)) return r;
  if (iters < 1) {
    for (int64_t i = 0; i < nsys; ++i) {
      if (status_host) status_host[i] = HB_CG_RUNNING;
      if (iters_done_host) iters_done_host[i] = 0;
    }
    return HB_OK;  // ConjugateGradient::run returns immediately for iter < 1
  }
  const int64_t nv = image_elems(p);
  const int nrr = nrr_blocks(p);
  std::vector<int> stat_all(nsys), done_all(nsys);
  const bool use_graph = (flags & HB_CG_GRAPH) && !g_prof_on.load();
  for (int64_t s0 = 0; s0 < nsys;) {
    int64_t slots = 0;
    const int64_t g = next_group(p, sys, s0, nsys, iters, true, ws_bytes, &slots);
    if (!ws || group_bytes(p, g, slots, iters, true) > ws_bytes)
      return fail(HB_ERR_WORKSPACE, "hb_cg_run: workspace too small for one system");
    if (!ws_aligned(ws)) return fail(HB_ERR_INVALID, "hb_cg_run: workspace not 16-byte aligned");
    Arena ar(ws);
    GroupWs w = carve_group(ar, p, g, slots, iters, true);
    if (int r = upload_tables(p, w, sys, s0, g, true, st)) return r;
    PassArgs a = group_pass_args(p, w, g, slots, false);
    // r = b - (A + lambda I) x
    if (int r = run_normal(p, a, st)) return r;
    CgState s{};
    s.nsys = (int)g;
    s.nv = nv;
    s.sys_x = (float2* const*)(w.tables + w.L.cg_x);
    s.sys_b = (const float2* const*)(w.tables + w.L.cg_b);
    s.iter = w.iter;
    s.r = w.r; s.p = w.pv; s.ap = w.ap;
    s.rz = w.rz; s.rz_ld = iters + 1;
    s.status = w.status; s.active = w.active; s.iters_done = w.iters_done;
    s.pap_part = w.pap; s.npap = npap_blocks(p);
    s.rr_part = w.rr;
    s.tol = tol;
    bool precond = false;
    for (int64_t i = 0; i < g; ++i) precond = precond || sys[s0 + i].precond != nullptr;
    s.z = precond ? w.z : nullptr;
    s.sys_pdiag = (const float* const*)(w.tables + w.L.sys_pdiag);
    dim3 ugrid(nrr, (unsigned)g);
    if (int r = launch_cg_update(HB_KERNEL_CG_UPDATE, cg_init_kernel, ugrid, s, st)) return r;
    if (precond)
      if (int r = cg_precondition(p, s, ugrid, 1, st)) return r;
    {
      LaunchScope ls(HB_KERNEL_CG_UPDATE, st);
      cg_init_finish_kernel<<<(unsigned)g, 256, 0, st>>>(s, nrr);
    }
    HB_CHECK_LAUNCH();
    PassArgs ai = group_pass_args(p, w, g, slots, true);
    ai.active = w.active;
    ai.dot_partials = w.pap;
    if (!use_graph) {
      for (int it = 0; it < iters; ++it)
        if (int r = cg_iteration(p, ai, s, ugrid, w.iter, st)) return r;
    } else {
      // capture one iteration and replay it `iters` times: on the caller's stream, or,
      // for the legacy default streams (which cannot be captured), on a per-device side
      // stream ordered against the caller's stream by events
      const bool own = st != nullptr && st != cudaStreamLegacy && st != cudaStreamPerThread;
      std::unique_lock<std::mutex> side_lock(g_graph_mu, std::defer_lock);
      cudaStream_t cs = st;
      GraphStream* gs = nullptr;
      if (!own) {
        int dev = 0;
        HB_CUDA(cudaGetDevice(&dev));
        if (int r = graph_stream(dev, &gs)) return r;
        side_lock.lock();
        cs = gs->s;
        HB_CUDA(cudaEventRecord(gs->e1, st));
        HB_CUDA(cudaStreamWaitEvent(cs, gs->e1, 0));
      }
      cudaGraph_t graph = nullptr;
      HB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
      int rc = cg_iteration(p, ai, s, ugrid, w.iter, cs);
      cudaError_t ce = cudaStreamEndCapture(cs, &graph);
      if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      if (ce != cudaSuccess) return fail(HB_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
      cudaGraphExec_t exec = nullptr;
      ce = cudaGraphInstantiate(&exec, graph, 0);
      if (ce != cudaSuccess) {
        cudaGraphDestroy(graph);
        return fail(HB_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
      }
      for (int it = 0; it < iters && ce == cudaSuccess; ++it) ce = cudaGraphLaunch(exec, cs);
      g_launches.fetch_add((uint64_t)(kKernelsPerCgIteration + (precond ? kKernelsPerPrecondition : 0)) * iters,
                           std::memory_order_relaxed);
      cudaError_t ce2 = cudaSuccess;
      if (!own) {
        ce2 = cudaEventRecord(gs->e2, cs);
        if (ce2 == cudaSuccess) ce2 = cudaStreamWaitEvent(st, gs->e2, 0);
      }
      cudaGraphExecDestroy(exec);
      cudaGraphDestroy(graph);
      if (ce != cudaSuccess) return fail(HB_ERR_CUDA, std::string("graph launch: ") + cudaGetErrorString(ce));
      if (ce2 != cudaSuccess) return fail(HB_ERR_CUDA, std::string("graph join: ") + cudaGetErrorString(ce2));
    }
    HB_CUDA(cudaMemcpyAsync(stat_all.data() + s0, w.status, g * sizeof(int), cudaMemcpyDeviceToHost, st));
    HB_CUDA(cudaMemcpyAsync(done_all.data() + s0, w.iters_done, g * sizeof(int), cudaMemcpyDeviceToHost, st));
    HB_CUDA(cudaStreamSynchronize(st));  // the next group reuses the workspace tables
    s0 += g;
  }
  HB_CUDA(cudaStreamSynchronize(st));
  // a pass that gave up waiting for a copy (or, on tensor-core plans, a contraction) left
  // its output incomplete, which invalidates every solve
  if (int r = tc_wait_check()) return r;
  bool notpd = false;
  for (int64_t i = 0; i < nsys; ++i) {
    if (status_host) status_host[i] = stat_all[i];
    if (iters_done_host) iters_done_host[i] = done_all[i];
    if (stat_all[i] == kCgNotPD) notpd = true;
  }
  if (notpd) return fail(HB_ERR_NOT_PD, "A was not positive definite");
  return HB_OK;
}

// ------------------------------------------------------- running batch of CG solves ----
// Layout of the per-member arrays that follow the pass tables in the batch's table block.
struct BatchLayout {
  size_t x, b, r, p, ap, rz, phase, it, tol, bytes;
};
BatchLayout batch_layout(size_t off, int64_t k) {
  BatchLayout B;
  size_t o = off;
  auto take = [&](size_t n) {
    o = (o + 15) & ~size_t(15);
    size_t r = o;
    o += n;
    return r;
  };
  B.x = take(8 * k);
  B.b = take(8 * k);
  B.r = take(8 * k);
  B.p = take(8 * k);
  B.ap = take(8 * k);
  B.rz = take(8 * k);
  B.phase = take(4 * k);
  B.it = take(4 * k);
  B.tol = take(8 * k);
  B.bytes = (o + 255) & ~size_t(255);
  return B;
}

struct BatchCarve {
  float2* spill;
  char* tables;
  TableLayout L;   // pass tables for the full capacity (a smaller member set uses a prefix layout)
  BatchLayout B;   // member arrays, after the pass tables
  float2 *r, *p, *ap;
  double *rz, *pap, *rr;
  int* status;
};
BatchCarve carve_batch(Arena& ar, const hb_plan* p, int64_t K, int64_t S) {
  BatchCarve c{};
  const size_t nv = (size_t)image_elems(p);
  c.spill = ar.take<float2>((size_t)S * spill_elems_per_slot(p));
  c.L = table_layout(K, S);
  c.B = batch_layout(c.L.bytes, K);
  c.tables = ar.take<char>(c.B.bytes);
  c.r = ar.take<float2>(K * nv);
  c.p = ar.take<float2>(K * nv);
  c.ap = ar.take<float2>(K * nv);
  c.rz = ar.take<double>(2 * K);
  c.pap = ar.take<double>(K * (size_t)npap_blocks(p));
  c.rr = ar.take<double>(K * (size_t)nrr_blocks(p));
  c.status = ar.take<int>(K);
  return c;
}

}  // namespace

struct hb_cg_batch {
  struct Member {
    bool used = false;
    int64_t handle = -1;
    hb_system sys{};
    std::vector<int64_t> coils;
    int iters = 0;      // iteration budget
    double tol = 0.0;
    int phase = 0;      // 1: initialise at the next step, 2: iterating
    int it = 0;         // iterations completed
  };
  const hb_plan* plan = nullptr;
  int64_t max_sys = 0, max_slots = 0;
  BatchCarve c{};
  std::vector<Member> m;
  int64_t next_handle = 0;
  int64_t coils_in_use = 0;
  std::vector<int64_t> fin_handle;
  std::vector<int32_t> fin_status, fin_iters;
};

namespace {

int normal_systems_impl(const hb_plan* p, int64_t nsys, const hb_system* sys, void* ws, size_t ws_bytes,
                        cudaStream_t st) {
  if (int r = validate_systems(p, nsys, sys, false)) return r;
  for (int64_t s0 = 0; s0 < nsys;) {
    int64_t slots = 0;
    const int64_t g = next_group(p, sys, s0, nsys, 0, false, ws_bytes, &slots);
    if (!ws || group_bytes(p, g, slots, 0, false) > ws_bytes)
      return fail(HB_ERR_WORKSPACE, "hb_sense_normal_apply: workspace too small for one system");
    if (!ws_aligned(ws)) return fail(HB_ERR_INVALID, "hb_sense_normal_apply: workspace not 16-byte aligned");
    Arena ar(ws);
    GroupWs w = carve_group(ar, p, g, slots, 0, false);
    if (int r = upload_tables(p, w, sys, s0, g, false, st)) return r;
    PassArgs a = group_pass_args(p, w, g, slots, false);
    if (int r = run_normal(p, a, st)) return r;
    s0 += g;
  }
  return HB_OK;
}

// Builds hb_system descriptors for the contiguous-array entry points.
std::vector<hb_system> contiguous_systems(const hb_plan* p, int64_t nsys, const void* x, void* out, const void* b,
                                          const void* smaps, const int64_t* coils, int64_t ncoil,
                                          const float* packed_diags, const int64_t* diag_index, float lambda) {
  const long long nv = image_elems(p);
  const long long pk = 8LL * nv;
  std::vector<hb_system> v(nsys);
  for (int64_t i = 0; i < nsys; ++i) {
    hb_system& q = v[i];
    q.x = const_cast<float2*>((const float2*)x + i * nv);
    q.out = out ? (void*)((float2*)out + i * nv) : nullptr;
    q.b = b ? (const void*)((const float2*)b + i * nv) : nullptr;
    q.smaps = smaps;
    q.coils = coils;
    q.ncoil = ncoil;
    q.packed_diag = packed_diags + (diag_index ? diag_index[i] : 0) * pk;
    q.lambda = lambda;
  }
  return v;
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
  if ((N1 & (N1 - 1)) == 0 && N1 >= 16) team_table(to.row2, N1 / 2);
  else
    for (int i = 0; i < N1 / 2; ++i) h[to.row2 + i] = make_float2(1.f, 0.f);
  if ((N1 & (N1 - 1)) == 0 && N1 >= 32) team_table(to.row4, N1 / 4);
  else
    for (int i = 0; i < N1 / 4; ++i) h[to.row4 + i] = make_float2(1.f, 0.f);
  for (int k = 0; k < 2 * N1; ++k) {
    const double a = -2.0 * M_PI * (double)k / (double)(2 * N1);
    h[to.circ + k] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
}

// ------------------------------------------------ allocation-free Toeplitz apply ----
// The spill and the twiddle tables of hb_toeplitz_apply_noalloc live in these arrays;
// host code reaches them only through cudaGetSymbolAddress (per device).
// Sized for table_offsets(160, 160, 160).total, the largest supported axes; each call
// checks its own size against it.
constexpr int kNoAllocMaxTables = 2 * 160 + 160 + 2 * 160 + 160 + 80 + 40 + 2 * 160;
static __device__ __align__(256) unsigned char g_noalloc_scratch[HB_NOALLOC_SCRATCH_BYTES];
static __device__ __align__(256) float2 g_noalloc_tables[kNoAllocMaxTables];
constexpr int kNoAllocDescBytes = 512;  // descriptor tables of one system
static __device__ __align__(256) unsigned char g_noalloc_desc[kNoAllocDescBytes];

constexpr int kNoAllocMaxDevices = 64;
struct NoAllocDevice {
  bool ready = false;
  void* scratch = nullptr;
  float2* tables = nullptr;
  void* desc = nullptr;
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
  // + the team tables of nz, ny, nx (image-grid FFTs of the preconditioner)
  const int nimg[3] = {p->N0, p->N1, p->N2};
  const std::vector<float2> himg = fftl::team_tables(nimg);
  h.insert(h.end(), himg.begin(), himg.end());
  cudaError_t e = cudaMalloc(&p->tables, h.size() * sizeof(float2));
  if (e == cudaSuccess) e = cudaMemcpy(p->tables, h.data(), h.size() * sizeof(float2), cudaMemcpyHostToDevice);
  // the device's flag for a pass that gave up waiting (bulk copies, tensor-core operands)
  if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&p->tc_wait_error, g_tc_wait_error);
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
  if (p->tc_ftab) cudaFree(p->tc_ftab);
  delete p;
  return HB_OK;
}

int hb_plan_set_precision(hb_plan* p, int precision) {
  if (int r = check_plan(p)) return r;
  if (precision == HB_PRECISION_FP32) {
    p->precision = precision;
    return HB_OK;
  }
  if (precision != HB_PRECISION_BF16X3) return fail(HB_ERR_INVALID, "hb_plan_set_precision: unknown precision");
  if (p->N1 != 128 || p->N2 != 128)
    return fail(HB_ERR_UNSUPPORTED, "HB_PRECISION_BF16X3 needs ny = nx = 128 (tensor-core x pass), got ny = " +
                                        std::to_string(p->N1) + ", nx = " + std::to_string(p->N2));
  DeviceGuard dg(p->device);
  if (!p->tc_ftab) {
    const std::vector<uint16_t> t = tc_dft_table(p->N2);
    cudaError_t e = cudaMalloc(&p->tc_ftab, t.size() * sizeof(uint16_t));
    if (e == cudaSuccess) e = cudaMemcpy(p->tc_ftab, t.data(), t.size() * sizeof(uint16_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      if (p->tc_ftab) cudaFree(p->tc_ftab);
      p->tc_ftab = nullptr;
      return fail(HB_ERR_CUDA, std::string("tensor-core tables: ") + cudaGetErrorString(e));
    }
  }
  p->precision = precision;
  return HB_OK;
}

int hb_plan_precision(const hb_plan* p) { return p ? p->precision : -1; }

int hb_plan_inject_tc_stall(hb_plan* p, int chunk) {
  if (int r = check_plan(p)) return r;
  if (chunk < -1 || chunk >= p->N2 / tc::kKc)
    return fail(HB_ERR_INVALID, "hb_plan_inject_tc_stall: chunk must be -1 or in [0, nx / 16)");
  p->tc_stall_chunk = chunk;
  return HB_OK;
}

int hb_plan_inject_x_stall(hb_plan* p, int coil) {
  if (int r = check_plan(p)) return r;
  if (coil < -1) return fail(HB_ERR_INVALID, "hb_plan_inject_x_stall: coil must be -1 or >= 0");
  p->x_stall_coil = coil;
  return HB_OK;
}

int hb_wait_status(int device) {
  DeviceGuard dg(device);
  if (!dg.ok) return fail(HB_ERR_CUDA, "cannot select device " + std::to_string(device));
  return tc_wait_check();
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
  return group_bytes(p, nsys, nsys * ncoil, 0, false);
}

size_t hb_systems_workspace_bytes(const hb_plan* p, int64_t nsys, int64_t total_coils, int iters) {
  if (!p || nsys < 1 || total_coils < 1) return 0;
  return group_bytes(p, nsys, total_coils, iters < 0 ? 0 : iters, iters >= 0);
}

int hb_toeplitz_apply(const hb_plan* p, const void* in, void* out, int64_t out_ldz, int64_t out_ldy, const void* mul,
                      int accumulate, const float* packed_diag, void* ws, size_t ws_bytes, void* stream) {
  if (int r = check_plan(p)) return r;
  if (!in || !out || !packed_diag) return fail(HB_ERR_INVALID, "hb_toeplitz_apply: NULL pointer");
  if (!diag_aligned(packed_diag)) return fail(HB_ERR_INVALID, "hb_toeplitz_apply: packed diagonal not 16-byte aligned");
  if (!ws || ws_bytes < hb_normal_workspace_bytes(p, 1, 1))
    return fail(HB_ERR_WORKSPACE, "hb_toeplitz_apply: workspace too small");
  if (!ws_aligned(ws)) return fail(HB_ERR_INVALID, "hb_toeplitz_apply: workspace not 16-byte aligned");
  DeviceGuard dg(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t coil0 = 0;
  hb_system q{};
  q.x = const_cast<void*>(in);
  q.out = out;
  q.smaps = nullptr;
  q.coils = &coil0;
  q.ncoil = 1;
  q.packed_diag = packed_diag;
  q.lambda = 0.f;
  Arena ar(ws);
  GroupWs w = carve_group(ar, p, 1, 1, 0, false);
  if (int r = upload_tables(p, w, &q, 0, 1, false, st)) return r;
  PassArgs a = group_pass_args(p, w, 1, 1, false);
  a.mul = (const float2*)mul;
  a.out_ldz = out_ldz;
  a.out_ldy = out_ldy;
  a.accumulate = accumulate ? 1 : 0;
  return run_normal(p, a, st);
}

int hb_sense_normal_apply(const hb_plan* p, int64_t nsys, const void* x, void* out, const void* smaps,
                          const int64_t* coils, int64_t ncoil, const float* packed_diags, const int64_t* diag_index,
                          float lambda, void* ws, size_t ws_bytes, void* stream) {
  if (int r = check_plan(p)) return r;
  if (nsys < 1 || ncoil < 1) return fail(HB_ERR_INVALID, "hb_sense_normal_apply: nsys and ncoil must be >= 1");
  if (!x || !out || !smaps || !coils || !packed_diags) return fail(HB_ERR_INVALID, "hb_sense_normal_apply: NULL pointer");
  DeviceGuard dg(p->device);
  std::vector<hb_system> v =
      contiguous_systems(p, nsys, x, out, nullptr, smaps, coils, ncoil, packed_diags, diag_index, lambda);
  return normal_systems_impl(p, nsys, v.data(), ws, ws_bytes, (cudaStream_t)stream);
}

int hb_sense_normal_apply_systems(const hb_plan* p, int64_t nsys, const hb_system* systems, void* ws,
                                  size_t ws_bytes, void* stream) {
  if (int r = check_plan(p)) return r;
  DeviceGuard dg(p->device);
  return normal_systems_impl(p, nsys, systems, ws, ws_bytes, (cudaStream_t)stream);
}

size_t hb_cg_workspace_bytes(const hb_plan* p, int64_t nsys, int64_t ncoil, int iters) {
  if (!p || nsys < 1 || ncoil < 1 || iters < 0) return 0;
  return group_bytes(p, nsys, nsys * ncoil, iters, true);
}

int hb_cg_run(const hb_plan* p, int64_t nsys, void* x, const void* b, const void* smaps, const int64_t* coils,
              int64_t ncoil, const float* packed_diags, const int64_t* diag_index, float lambda, int iters, double tol,
              int32_t* status_host, int32_t* iters_done_host, void* ws, size_t ws_bytes, void* stream) {
  if (int r = check_plan(p)) return r;
  if (nsys < 1 || ncoil < 1) return fail(HB_ERR_INVALID, "hb_cg_run: nsys and ncoil must be >= 1");
  if (!x || !b || !smaps || !coils || !packed_diags) return fail(HB_ERR_INVALID, "hb_cg_run: NULL pointer");
  DeviceGuard dg(p->device);
  std::vector<hb_system> v =
      contiguous_systems(p, nsys, x, nullptr, b, smaps, coils, ncoil, packed_diags, diag_index, lambda);
  return cg_systems_impl(p, nsys, v.data(), iters, tol, 0, status_host, iters_done_host, ws, ws_bytes,
                         (cudaStream_t)stream);
}

int hb_cg_run_systems(const hb_plan* p, int64_t nsys, const hb_system* systems, int iters, double tol, int flags,
                      int32_t* status_host, int32_t* iters_done_host, void* ws, size_t ws_bytes, void* stream) {
  if (int r = check_plan(p)) return r;
  DeviceGuard dg(p->device);
  return cg_systems_impl(p, nsys, systems, iters, tol, flags, status_host, iters_done_host, ws, ws_bytes,
                         (cudaStream_t)stream);
}

size_t hb_cg_batch_workspace_bytes(const hb_plan* p, int64_t max_systems, int64_t max_coil_slots) {
  if (!p || max_systems < 1 || max_coil_slots < 1) return 0;
  Arena ar(nullptr);
  carve_batch(ar, p, max_systems, max_coil_slots);
  return ar.off + 256;
}

int hb_cg_batch_create(hb_cg_batch** out, const hb_plan* p, int64_t max_systems, int64_t max_coil_slots, void* ws,
                       size_t ws_bytes) {
  if (!out) return fail(HB_ERR_INVALID, "hb_cg_batch_create: output pointer is NULL");
  *out = nullptr;
  if (int r = check_plan(p)) return r;
  if (max_systems < 1 || max_coil_slots < 1 || max_systems > 65535 || max_coil_slots > 65535)
    return fail(HB_ERR_INVALID, "hb_cg_batch_create: capacity out of range");
  if (!ws || ws_bytes < hb_cg_batch_workspace_bytes(p, max_systems, max_coil_slots))
    return fail(HB_ERR_WORKSPACE, "hb_cg_batch_create: workspace too small");
  if (!ws_aligned(ws)) return fail(HB_ERR_INVALID, "hb_cg_batch_create: workspace not 16-byte aligned");
  hb_cg_batch* e = new hb_cg_batch();
  e->plan = p;
  e->max_sys = max_systems;
  e->max_slots = max_coil_slots;
  Arena ar(ws);
  e->c = carve_batch(ar, p, max_systems, max_coil_slots);
  e->m.resize((size_t)max_systems);
  *out = e;
  return HB_OK;
}

int hb_cg_batch_destroy(hb_cg_batch* e) {
  delete e;
  return HB_OK;
}

int hb_cg_batch_add(hb_cg_batch* e, const hb_system* sys, int iters, double tol, int64_t* handle) {
  if (!e || !sys || !handle) return fail(HB_ERR_INVALID, "hb_cg_batch_add: NULL pointer");
  if (int r = validate_systems(e->plan, 1, sys, true)) return r;
  if (sys->precond) return fail(HB_ERR_UNSUPPORTED, "hb_cg_batch_add: preconditioned systems run in hb_cg_run_systems");
  if (iters < 1) return fail(HB_ERR_INVALID, "hb_cg_batch_add: iters must be >= 1");
  int64_t k = -1;
  for (int64_t i = 0; i < e->max_sys && k < 0; ++i)
    if (!e->m[i].used) k = i;
  if (k < 0 || e->coils_in_use + sys->ncoil > e->max_slots)
    return fail(HB_ERR_WORKSPACE, "hb_cg_batch_add: the batch is full (retire finished systems first)");
  hb_cg_batch::Member& q = e->m[k];
  q = hb_cg_batch::Member();
  q.used = true;
  q.handle = e->next_handle++;
  q.sys = *sys;
  q.coils.assign(sys->coils, sys->coils + sys->ncoil);
  q.sys.coils = q.coils.data();
  q.iters = iters;
  q.tol = tol;
  q.phase = 1;
  e->coils_in_use += sys->ncoil;
  *handle = q.handle;
  return HB_OK;
}

int hb_cg_batch_step(hb_cg_batch* e, void* stream, int64_t* in_batch) {
  if (!e) return fail(HB_ERR_INVALID, "hb_cg_batch_step: NULL batch");
  const hb_plan* p = e->plan;
  DeviceGuard dg(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<int64_t> mem;  // capacity slots of the members, in slot order
  int64_t slots = 0;
  for (int64_t k = 0; k < e->max_sys; ++k)
    if (e->m[k].used) {
      mem.push_back(k);
      slots += e->m[k].sys.ncoil;
    }
  const int64_t g = (int64_t)mem.size();
  if (in_batch) *in_batch = g;
  if (g == 0) return HB_OK;
  const size_t nv = (size_t)image_elems(p);
  // pass tables of the member set (normal-op input: x when initialising, p otherwise;
  // output: Ap), then the member arrays
  GroupWs w{};
  w.spill = e->c.spill;
  w.tables = e->c.tables;
  w.L = table_layout(g, slots);
  std::vector<hb_system> q(g);
  for (int64_t i = 0; i < g; ++i) {
    const hb_cg_batch::Member& mm = e->m[mem[i]];
    q[i] = mm.sys;
    q[i].x = mm.phase == 1 ? mm.sys.x : (void*)(e->c.p + mem[i] * nv);
    q[i].out = e->c.ap + mem[i] * nv;
  }
  std::vector<char> h(e->c.B.bytes);
  fill_group_tables(h.data(), p, w, q.data(), 0, g, false);
  const BatchLayout& B = e->c.B;
  for (int64_t i = 0; i < g; ++i) {
    const int64_t k = mem[i];
    const hb_cg_batch::Member& mm = e->m[k];
    auto put = [&](size_t off, size_t sz, const void* v) { std::memcpy(h.data() + off + sz * i, v, sz); };
    void* xp = mm.sys.x;
    const void* bp = mm.sys.b;
    void* rp = e->c.r + k * nv;
    void* pp = e->c.p + k * nv;
    void* app = e->c.ap + k * nv;
    void* rzp = e->c.rz + 2 * k;
    const int ph = mm.phase, it = mm.it;
    const double tl = mm.tol;
    put(B.x, 8, &xp);
    put(B.b, 8, &bp);
    put(B.r, 8, &rp);
    put(B.p, 8, &pp);
    put(B.ap, 8, &app);
    put(B.rz, 8, &rzp);
    put(B.phase, 4, &ph);
    put(B.it, 4, &it);
    put(B.tol, 8, &tl);
  }
  HB_CUDA(cudaMemcpyAsync(e->c.tables, h.data(), B.bytes, cudaMemcpyHostToDevice, st));
  PassArgs a = group_pass_args(p, w, g, slots, false);
  a.dot_partials = e->c.pap;  // Re<p, Ap> partials, per member
  if (int r = run_normal(p, a, st)) return r;
  CgBatchState s{};
  s.nmem = (int)g;
  s.nv = (long long)nv;
  const char* t = e->c.tables;
  s.x = (float2* const*)(t + B.x);
  s.b = (const float2* const*)(t + B.b);
  s.r = (float2* const*)(t + B.r);
  s.p = (float2* const*)(t + B.p);
  s.ap = (const float2* const*)(t + B.ap);
  s.rz = (double* const*)(t + B.rz);
  s.phase = (const int*)(t + B.phase);
  s.it = (const int*)(t + B.it);
  s.tol = (const double*)(t + B.tol);
  s.status = e->c.status;
  s.pap_part = e->c.pap;
  s.npap = npap_blocks(p);
  s.rr_part = e->c.rr;
  const dim3 ugrid(nrr_blocks(p), (unsigned)g);
  {
    LaunchScope ls(HB_KERNEL_CG_UPDATE, st);
    cg_batch_xr_kernel<<<ugrid, 256, 0, st>>>(s);
  }
  HB_CHECK_LAUNCH();
  {
    LaunchScope ls(HB_KERNEL_CG_UPDATE, st);
    cg_batch_p_kernel<<<ugrid, 256, 0, st>>>(s);
  }
  HB_CHECK_LAUNCH();
  std::vector<int> stat(g);
  HB_CUDA(cudaMemcpyAsync(stat.data(), e->c.status, g * sizeof(int), cudaMemcpyDeviceToHost, st));
  HB_CUDA(cudaStreamSynchronize(st));  // the host image of the tables is reused next step
  if (int r = tc_wait_check()) return r;
  // advance every member; finished ones leave the batch
  int64_t left = 0;
  for (int64_t i = 0; i < g; ++i) {
    hb_cg_batch::Member& mm = e->m[mem[i]];
    int done_status = -1;
    if (mm.phase == 1) {
      if (stat[i] == kCgConverged) done_status = HB_CG_CONVERGED;
      mm.phase = 2;
      mm.it = 0;
    } else if (stat[i] == kCgNotPD) {
      done_status = HB_CG_NOT_PD;
    } else {
      mm.it += 1;
      if (stat[i] == kCgConverged) done_status = HB_CG_CONVERGED;
      else if (mm.it >= mm.iters) done_status = HB_CG_RUNNING;
    }
    if (done_status >= 0) {
      e->fin_handle.push_back(mm.handle);
      e->fin_status.push_back(done_status);
      e->fin_iters.push_back(mm.it);
      e->coils_in_use -= mm.sys.ncoil;
      mm = hb_cg_batch::Member();
    } else {
      ++left;
    }
  }
  if (in_batch) *in_batch = left;
  return HB_OK;
}

int hb_cg_batch_retire(hb_cg_batch* e, int64_t* handles, int32_t* status, int32_t* iters, int64_t cap,
                       int64_t* n_out) {
  if (!e || !n_out) return fail(HB_ERR_INVALID, "hb_cg_batch_retire: NULL pointer");
  const int64_t n = std::min<int64_t>(cap, (int64_t)e->fin_handle.size());
  for (int64_t i = 0; i < n; ++i) {
    if (handles) handles[i] = e->fin_handle[i];
    if (status) status[i] = e->fin_status[i];
    if (iters) iters[i] = e->fin_iters[i];
  }
  e->fin_handle.erase(e->fin_handle.begin(), e->fin_handle.begin() + n);
  e->fin_status.erase(e->fin_status.begin(), e->fin_status.begin() + n);
  e->fin_iters.erase(e->fin_iters.begin(), e->fin_iters.begin() + n);
  *n_out = n;
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
  if (!diag_aligned(packed_diag))
    return fail(HB_ERR_INVALID, "hb_toeplitz_apply_noalloc: packed diagonal not 16-byte aligned");
  // the built-in twiddle-table array holds the tables of axes up to 160; a size whose
  // tables would not fit is refused before anything is written
  if (table_offsets((int)nz, (int)ny, (int)nx).total > kNoAllocMaxTables)
    return fail(HB_ERR_UNSUPPORTED, "hb_toeplitz_apply_noalloc: twiddle tables of " + std::to_string(nz) + "x" +
                                        std::to_string(ny) + "x" + std::to_string(nx) + " exceed the built-in " +
                                        std::to_string(kNoAllocMaxTables) + " entries");
  int dev = 0;
  HB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(HB_ERR_INVALID, "hb_toeplitz_apply_noalloc: device index");
  cudaStream_t st = (cudaStream_t)stream;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  NoAllocDevice& d = g_noalloc[dev];
  if (!d.ready) {  // once per device, with that device current
    HB_CUDA(cudaGetSymbolAddress(&d.scratch, g_noalloc_scratch));
    HB_CUDA(cudaGetSymbolAddress((void**)&d.tables, g_noalloc_tables));
    HB_CUDA(cudaGetSymbolAddress(&d.desc, g_noalloc_desc));
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
  // one system, one unit coil: its descriptor tables go to the built-in table block
  const int64_t coil0 = 0;
  hb_system q{};
  q.x = const_cast<void*>(in);
  q.out = out;
  q.smaps = nullptr;
  q.coils = &coil0;
  q.ncoil = 1;
  q.packed_diag = packed_diag;
  q.lambda = 0.f;
  GroupWs w{};
  w.spill = (float2*)d.scratch;
  w.L = table_layout(1, 1);
  w.tables = (char*)d.desc;
  char h[kNoAllocDescBytes];  // host stack, no heap
  fill_group_tables(h, &p, w, &q, 0, 1, false);
  HB_CUDA(cudaMemcpyAsync(w.tables, h, w.L.bytes, cudaMemcpyHostToDevice, st));
  HB_CUDA(cudaStreamSynchronize(st));
  PassArgs a = group_pass_args(&p, w, 1, 1, false);
  a.mul = (const float2*)mul;
  a.out_ldz = out_ldz;
  a.out_ldy = out_ldy;
  a.accumulate = accumulate ? 1 : 0;
  return run_normal(&p, a, st);
}

const char* hb_plan_plane_schedule(const hb_plan* p) {
  if (!p) return "";
  int n = 0;
  const PlaneVariant* v = plane_variants(p->N0, p->N1, &n);
  if (!v) return "plane_yz:q1";
  return v[plane_variant_index(n, p->plane_variant)].name;
}

size_t hb_autotune_workspace_bytes(const hb_plan* p, int64_t nslots) {
  if (!p || nslots < 1) return 0;
  Arena ar(nullptr);
  carve_group(ar, p, 1, nslots, 0, false);
  ar.take<float>((size_t)hb_diag_packed_floats(p));
  return ar.off + 256;
}

int hb_plan_autotune(hb_plan* p, int64_t nslots, void* ws, size_t ws_bytes, void* stream, int* chosen,
                     double* best_ms) {
  if (int r = check_plan(p)) return r;
  if (nslots < 1 || nslots > 65535) return fail(HB_ERR_INVALID, "hb_plan_autotune: nslots");
  if (!ws || ws_bytes < hb_autotune_workspace_bytes(p, nslots))
    return fail(HB_ERR_WORKSPACE, "hb_plan_autotune: workspace too small");
  if (!ws_aligned(ws)) return fail(HB_ERR_INVALID, "hb_plan_autotune: workspace not 16-byte aligned");
  DeviceGuard dg(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  int nvar = 0;
  const PlaneVariant* vars = plane_variants(p->N0, p->N1, &nvar);
  if (!vars) {  // a single schedule: nothing to choose
    p->plane_variant = 0;
    if (chosen) *chosen = 0;
    if (best_ms) *best_ms = 0.0;
    return HB_OK;
  }
  Arena ar(ws);
  GroupWs w = carve_group(ar, p, 1, nslots, 0, false);
  float* diag = ar.take<float>((size_t)hb_diag_packed_floats(p));
  // one system whose nslots coils all use a unit map; only the plane pass runs, on
  // zeroed data (its timing does not depend on the values)
  std::vector<int64_t> coils(nslots, 0);
  hb_system q{};
  q.x = w.spill;
  q.out = w.spill;
  q.smaps = nullptr;
  q.coils = coils.data();
  q.ncoil = nslots;
  q.packed_diag = diag;
  if (int r = upload_tables(p, w, &q, 0, 1, false, st)) return r;
  HB_CUDA(cudaMemsetAsync(w.spill, 0, (size_t)nslots * spill_elems_per_slot(p) * sizeof(float2), st));
  HB_CUDA(cudaMemsetAsync(diag, 0, (size_t)hb_diag_packed_floats(p) * sizeof(float), st));
  PassArgs a = group_pass_args(p, w, 1, nslots, false);
  cudaEvent_t e0, e1;
  HB_CUDA(cudaEventCreate(&e0));
  HB_CUDA(cudaEventCreate(&e1));
  int best = 0;
  double best_t = 1e300;
  cudaError_t err = cudaSuccess;
  for (int v = 0; v < nvar && err == cudaSuccess; ++v) {
    err = vars[v].fn(a, (int)nslots, st);  // warm-up (and shared-memory opt-in)
    if (err != cudaSuccess) break;
    err = cudaEventRecord(e0, st);
    for (int k = 0; k < 3 && err == cudaSuccess; ++k) err = vars[v].fn(a, (int)nslots, st);
    if (err == cudaSuccess) err = cudaEventRecord(e1, st);
    if (err == cudaSuccess) err = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    if (err == cudaSuccess && ms / 3.0 < best_t) {
      best_t = ms / 3.0;
      best = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess) return fail(HB_ERR_CUDA, std::string("hb_plan_autotune: ") + cudaGetErrorString(err));
  p->plane_variant = best;
  if (chosen) *chosen = best;
  if (best_ms) *best_ms = best_t;
  return HB_OK;
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
