// C ABI of the NUFFT (types 1 and 2) and the SENSE forward/adjoint around it
// (include/hasty_b200.h, section "Non-uniform FFT").  Replaces the cufinufft plans of
// hasty::fft::CUDANufft (lib/fft/nufft.cpp:540-767, declared nufft.ixx:108-160), the
// coil loops of the SENSE operators that use them (lib/mri/sense.ixx:426-497) and the
// NUFFT construction of the Toeplitz diagonal (build_diagonal_base, nufft.cpp:932-971).
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/hasty_b200.h"
#include "fft3_launch.cuh"
#include "nufft_kernels.cuh"
#include "runtime.cuh"

using namespace hb;
using hb::fftl::fft3_grid;
using hb::fftl::team_length;
using hb::fftl::team_tables;

struct hb_nufft {
  int device;
  NufftGeom g;
  int maxbatch;
  float* coords = nullptr;  // [3][K] (a copy)
  int* perm = nullptr;      // [K] samples in bin order
  float* corr = nullptr;    // [N0 | N1 | N2] 1 / phi_hat
  float2* tw = nullptr;     // team twiddle tables of n0, n1, n2 (offsets 0, n0, n0 + n1)
  float2* grid = nullptr;   // [maxbatch][n0][n1][n2]
  float2* modes = nullptr;  // [maxbatch][N0][N1][N2] (SENSE temporaries)
  float2* kbuf = nullptr;   // [maxbatch][K] (SENSE normal temporaries)
};

namespace {

template <int DIR>
cudaError_t fft3(const hb_nufft* p, float2* grid, int nt, cudaStream_t st) {
  return fft3_grid<DIR>(p->g.n[0], p->g.n[1], p->g.n[2], p->tw, grid, nt, st);
}

// Kernel width for a requested tolerance (upsampling 2): w = ceil(log10(1/tol)) + 1.
int width_for_tol(double tol) {
  int w = (int)std::ceil(std::log10(1.0 / tol)) + 1;
  return w < 2 ? 2 : (w > 16 ? 16 : w);
}

// Gauss-Legendre nodes and weights on [-1, 1] (Newton iteration on the Legendre
// polynomial, the textbook method), computed once.
constexpr int kGaussNodes = 64;
struct GaussLegendre {
  double x[kGaussNodes], w[kGaussNodes];
  GaussLegendre() {
    const int n = kGaussNodes;
    for (int i = 0; i < n; ++i) {
      double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
      for (int it = 0; it < 100; ++it) {
        double p0 = 1.0, p1 = z;  // P_0, P_1
        for (int k = 2; k <= n; ++k) {
          const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
          p0 = p1;
          p1 = p2;
        }
        dp = n * (z * p1 - p0) / (z * z - 1.0);  // P_n'(z)
        const double dz = p1 / dp;
        z -= dz;
        if (std::fabs(dz) < 1e-16) break;
      }
      x[i] = z;
      w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
  }
};

// phi_hat(k) = integral over |z| < w/2 of phi(z) cos(2 pi k z / n), by 64-point
// Gauss-Legendre quadrature on [0, w/2] (the integrand is even); relative error below
// 1e-11 for the widths of tolerances <= 1e-4.
double phi_hat(int k, int n, int w, double beta) {
  static const GaussLegendre gl;
  const double hw = 0.5 * w;
  double acc = 0.0;
  for (int i = 0; i < kGaussNodes; ++i) {
    const double z = 0.5 * hw * (gl.x[i] + 1.0);
    const double t = z / hw, s = 1.0 - t * t;
    const double phi = s > 0.0 ? std::exp(beta * (std::sqrt(s) - 1.0)) : 0.0;
    acc += gl.w[i] * phi * std::cos(2.0 * M_PI * k * z / n);
  }
  return 2.0 * 0.5 * hw * acc;
}

template <int W>
cudaError_t spread_w(const hb_nufft* p, const float2* c, long long c_ld, int nb, cudaStream_t st) {
  dim3 grid((unsigned)((p->g.K + 255) / 256), nb);
  LaunchScope ls(HB_KERNEL_NUFFT, st);
  if (p->g.dim == 3) nufft_spread_kernel<W, 3><<<grid, 256, 0, st>>>(p->g, p->coords, p->perm, c, c_ld, p->grid);
  else if (p->g.dim == 2) nufft_spread_kernel<W, 2><<<grid, 256, 0, st>>>(p->g, p->coords, p->perm, c, c_ld, p->grid);
  else nufft_spread_kernel<W, 1><<<grid, 256, 0, st>>>(p->g, p->coords, p->perm, c, c_ld, p->grid);
  return cudaGetLastError();
}
template <int W>
cudaError_t interp_w(const hb_nufft* p, float2* c, long long c_ld, int nb, cudaStream_t st) {
  dim3 grid((unsigned)((p->g.K + 255) / 256), nb);
  LaunchScope ls(HB_KERNEL_NUFFT, st);
  if (p->g.dim == 3) nufft_interp_kernel<W, 3><<<grid, 256, 0, st>>>(p->g, p->coords, p->perm, p->grid, c, c_ld);
  else if (p->g.dim == 2) nufft_interp_kernel<W, 2><<<grid, 256, 0, st>>>(p->g, p->coords, p->perm, p->grid, c, c_ld);
  else nufft_interp_kernel<W, 1><<<grid, 256, 0, st>>>(p->g, p->coords, p->perm, p->grid, c, c_ld);
  return cudaGetLastError();
}

#define HB_W_DISPATCH(FN, ...)                                                                      \
  switch (p->g.w) {                                                                                 \
    case 2: return FN<2>(__VA_ARGS__);   case 3: return FN<3>(__VA_ARGS__);                          \
    case 4: return FN<4>(__VA_ARGS__);   case 5: return FN<5>(__VA_ARGS__);                          \
    case 6: return FN<6>(__VA_ARGS__);   case 7: return FN<7>(__VA_ARGS__);                          \
    case 8: return FN<8>(__VA_ARGS__);   case 9: return FN<9>(__VA_ARGS__);                          \
    case 10: return FN<10>(__VA_ARGS__); case 11: return FN<11>(__VA_ARGS__);                        \
    case 12: return FN<12>(__VA_ARGS__); case 13: return FN<13>(__VA_ARGS__);                        \
    case 14: return FN<14>(__VA_ARGS__); case 15: return FN<15>(__VA_ARGS__);                        \
    case 16: return FN<16>(__VA_ARGS__);                                                             \
    default: return cudaErrorInvalidValue;                                                           \
  }

cudaError_t spread(const hb_nufft* p, const float2* c, long long c_ld, int nb, cudaStream_t st) {
  HB_W_DISPATCH(spread_w, p, c, c_ld, nb, st)
}
cudaError_t interp(const hb_nufft* p, float2* c, long long c_ld, int nb, cudaStream_t st) {
  HB_W_DISPATCH(interp_w, p, c, c_ld, nb, st)
}

long long nmodes(const hb_nufft* p) { return (long long)p->g.N[0] * p->g.N[1] * p->g.N[2]; }
long long nfine(const hb_nufft* p) { return (long long)p->g.n[0] * p->g.n[1] * p->g.n[2]; }

// nb <= maxbatch transforms: c [nb][K] (row pitch c_ld) -> f [nb][modes] (row pitch f_ld)
int type1_batch(const hb_nufft* p, const float2* c, long long c_ld, float2* f, long long f_ld, int nb, int isign,
                cudaStream_t st) {
  HB_CUDA(cudaMemsetAsync(p->grid, 0, (size_t)nb * nfine(p) * sizeof(float2), st));
  HB_CUDA(spread(p, c, c_ld, nb, st));
  HB_CUDA(isign > 0 ? fft3<1>(p, p->grid, nb, st) : fft3<-1>(p, p->grid, nb, st));
  dim3 grid((unsigned)((nmodes(p) + 255) / 256), nb);
  {
    LaunchScope ls(HB_KERNEL_NUFFT, st);
    nufft_deconv_kernel<<<grid, 256, 0, st>>>(p->g, p->grid, p->corr, f, f_ld);
  }
  HB_CHECK_LAUNCH();
  return HB_OK;
}

// nb <= maxbatch transforms: f [nb][modes] -> c [nb][K]
int type2_batch(const hb_nufft* p, const float2* f, long long f_ld, float2* c, long long c_ld, int nb, int isign,
                cudaStream_t st) {
  HB_CUDA(cudaMemsetAsync(p->grid, 0, (size_t)nb * nfine(p) * sizeof(float2), st));
  dim3 grid((unsigned)((nmodes(p) + 255) / 256), nb);
  {
    LaunchScope ls(HB_KERNEL_NUFFT, st);
    nufft_precorrect_kernel<<<grid, 256, 0, st>>>(p->g, f, f_ld, p->corr, p->grid);
  }
  HB_CHECK_LAUNCH();
  HB_CUDA(isign > 0 ? fft3<1>(p, p->grid, nb, st) : fft3<-1>(p, p->grid, nb, st));
  HB_CUDA(interp(p, c, c_ld, nb, st));
  return HB_OK;
}

void free_plan(hb_nufft* p) {
  if (!p) return;
  cudaFree(p->coords);
  cudaFree(p->perm);
  cudaFree(p->corr);
  cudaFree(p->tw);
  cudaFree(p->grid);
  cudaFree(p->modes);
  cudaFree(p->kbuf);
  delete p;
}

}  // namespace

namespace hb {

int nufft_psf_circulant(const int* M, const float* coords, int64_t nsamples, double tol, const float* weights,
                        int device, float2* out, cudaStream_t st) {
  const long long vol = (long long)M[0] * M[1] * M[2];
  hb_nufft* np = nullptr;
  // type 1 over the grid's modes: sum_j exp(+i c_j . d), d in [-M/2, M/2)
  if (int r = hb_nufft_create(&np, M[0], M[1], M[2], coords, nsamples, tol, 1, device, st)) return r;
  float2* ones = nullptr;
  int rc = HB_OK;
  cudaError_t e = cudaMalloc(&ones, nsamples * sizeof(float2));
  if (e == cudaSuccess) {
    {
      LaunchScope ls(HB_KERNEL_DIAG, st);
      fill_c64_kernel<<<(unsigned)((nsamples + 255) / 256), 256, 0, st>>>(ones, nsamples, make_float2(1.f, 0.f),
                                                                          weights);
    }
    rc = type1_batch(np, ones, nsamples, np->modes, vol, 1, +1, st);
    if (rc == HB_OK) {
      LaunchScope ls(HB_KERNEL_DIAG, st);
      ifftshift3_scale_kernel<<<(unsigned)((vol + 255) / 256), 256, 0, st>>>(np->modes, M[0], M[1], M[2],
                                                                             (float)(1.0 / (double)vol), out);
    }
    if (rc == HB_OK && (e = cudaGetLastError()) != cudaSuccess)
      rc = fail(HB_ERR_CUDA, std::string("psf: ") + cudaGetErrorString(e));
    if (rc == HB_OK && (e = cudaStreamSynchronize(st)) != cudaSuccess)
      rc = fail(HB_ERR_CUDA, std::string("psf: ") + cudaGetErrorString(e));
  } else {
    rc = fail(HB_ERR_CUDA, std::string("psf: ") + cudaGetErrorString(e));
  }
  if (rc != HB_OK) cudaStreamSynchronize(st);
  cudaFree(ones);
  hb_nufft_destroy(np);
  return rc;
}

}  // namespace hb

extern "C" {

int hb_nufft_create(hb_nufft** out, int64_t nz, int64_t ny, int64_t nx, const float* coords, int64_t nsamples,
                    double tol, int maxbatch, int device, void* stream) {
  if (!out) return fail(HB_ERR_INVALID, "hb_nufft_create: null output");
  *out = nullptr;
  if (!coords || nsamples < 1 || nsamples > (int64_t)0x7fffffff)
    return fail(HB_ERR_INVALID, "hb_nufft_create: need coords and 1 <= nsamples < 2^31");
  if (!(tol > 0.0 && tol < 1.0)) return fail(HB_ERR_INVALID, "hb_nufft_create: tol must be in (0, 1)");
  if (maxbatch < 1 || maxbatch > kNufftMaxBatch)
    return fail(HB_ERR_INVALID, "hb_nufft_create: maxbatch must be in [1, " + std::to_string(kNufftMaxBatch) + "]");
  const int64_t Nv[3] = {nz, ny, nx};
  NufftGeom g{};
  g.w = width_for_tol(tol);
  g.beta = (float)(2.30 * g.w);
  g.K = nsamples;
  // nz = 1: a 2-D plan over (ny, nx); nz = ny = 1: a 1-D plan over nx (coords [dim][K])
  g.dim = nz != 1 ? 3 : (ny != 1 ? 2 : 1);
  for (int a = 0; a < 3; ++a) {
    if (a < 3 - g.dim) {  // degenerate leading axis
      g.N[a] = g.n[a] = g.nb[a] = 1;
      continue;
    }
    int E = 0, S = 0;
    const int64_t n = 2 * Nv[a];
    if (Nv[a] < 1 || n > 512 || !team_length((int)n, &E, &S) || n < 2 * g.w)
      return fail(HB_ERR_UNSUPPORTED, "hb_nufft_create: mode count " + std::to_string(Nv[a]) +
                                          " unsupported (2N must be one of 8,16,32,64,128,256,512,96,160,192,320 "
                                          "and >= 2w)");
    g.N[a] = (int)Nv[a];
    g.n[a] = (int)n;
    g.nb[a] = (g.n[a] + kNufftBin - 1) / kNufftBin;
  }
  DeviceGuard dg(device);
  if (!dg.ok) return fail(HB_ERR_CUDA, "hb_nufft_create: cannot select device");
  cudaStream_t st = (cudaStream_t)stream;
  hb_nufft* p = new hb_nufft();
  p->device = device;
  p->g = g;
  p->maxbatch = maxbatch;
  const long long nbins = (long long)g.nb[0] * g.nb[1] * g.nb[2];
  const long long vol = (long long)g.n[0] * g.n[1] * g.n[2];
  const long long nm = (long long)g.N[0] * g.N[1] * g.N[2];
  int* bin_of = nullptr;
  int* counts = nullptr;
  auto bail = [&](cudaError_t e, const char* what) {
    cudaFree(bin_of);
    cudaFree(counts);
    free_plan(p);
    return fail(HB_ERR_CUDA, std::string("hb_nufft_create: ") + what + ": " + cudaGetErrorString(e));
  };
  cudaError_t e;
  if ((e = cudaMalloc(&p->coords, 3 * nsamples * sizeof(float))) != cudaSuccess) return bail(e, "coords");
  if ((e = cudaMalloc(&p->perm, nsamples * sizeof(int))) != cudaSuccess) return bail(e, "perm");
  if ((e = cudaMalloc(&p->corr, (g.N[0] + g.N[1] + g.N[2]) * sizeof(float))) != cudaSuccess) return bail(e, "corr");
  if ((e = cudaMalloc(&p->tw, (g.n[0] + g.n[1] + g.n[2]) * sizeof(float2))) != cudaSuccess) return bail(e, "tables");
  if ((e = cudaMalloc(&p->grid, (size_t)maxbatch * vol * sizeof(float2))) != cudaSuccess) return bail(e, "fine grid");
  if ((e = cudaMalloc(&p->modes, (size_t)maxbatch * nm * sizeof(float2))) != cudaSuccess) return bail(e, "modes");
  if ((e = cudaMalloc(&p->kbuf, (size_t)maxbatch * nsamples * sizeof(float2))) != cudaSuccess) return bail(e, "kbuf");
  if ((e = cudaMalloc(&bin_of, nsamples * sizeof(int))) != cudaSuccess) return bail(e, "bins");
  if ((e = cudaMalloc(&counts, 2 * nbins * sizeof(int))) != cudaSuccess) return bail(e, "bins");

  // host tables: 1/phi_hat per axis and the team twiddles of each fine-grid length
  std::vector<float> corr;
  for (int a = 0; a < 3; ++a)
    for (int i = 0; i < g.N[a]; ++i)
      corr.push_back(a < 3 - g.dim ? 1.f : (float)(1.0 / phi_hat(i - g.N[a] / 2, g.n[a], g.w, 2.30 * g.w)));
  const std::vector<float2> tw = team_tables(g.n);
  if ((e = cudaMemcpyAsync(p->corr, corr.data(), corr.size() * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return bail(e, "upload");
  if ((e = cudaMemcpyAsync(p->tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return bail(e, "upload");
  // the caller's [dim][K] rows become the trailing rows of [3][K]; degenerate rows are 0
  const int lead = 3 - g.dim;
  if (lead > 0 && (e = cudaMemsetAsync(p->coords, 0, lead * nsamples * sizeof(float), st)) != cudaSuccess)
    return bail(e, "coords copy");
  if ((e = cudaMemcpyAsync(p->coords + lead * nsamples, coords, g.dim * nsamples * sizeof(float),
                           cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
    return bail(e, "coords copy");
  // counting sort of the samples by bin
  if ((e = cudaMemsetAsync(counts, 0, nbins * sizeof(int), st)) != cudaSuccess) return bail(e, "memset");
  const unsigned blocks = (unsigned)((nsamples + 255) / 256);
  {
    LaunchScope ls(HB_KERNEL_NUFFT, st);
    nufft_bin_count_kernel<<<blocks, 256, 0, st>>>(g, p->coords, bin_of, counts);
  }
  {
    LaunchScope ls(HB_KERNEL_NUFFT, st);
    nufft_scan_kernel<<<1, 1024, 0, st>>>(counts, counts + nbins, (int)nbins);
  }
  {
    LaunchScope ls(HB_KERNEL_NUFFT, st);
    nufft_bin_scatter_kernel<<<blocks, 256, 0, st>>>(nsamples, bin_of, counts + nbins, p->perm);
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return bail(e, "binning");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return bail(e, "binning");
  cudaFree(bin_of);
  cudaFree(counts);
  *out = p;
  return HB_OK;
}

int hb_nufft_destroy(hb_nufft* plan) {
  if (!plan) return HB_OK;
  DeviceGuard dg(plan->device);
  free_plan(plan);
  return HB_OK;
}

int hb_nufft_width(const hb_nufft* plan) { return plan ? plan->g.w : -1; }

int hb_nufft_type1(const hb_nufft* plan, const void* c, void* f, int64_t ntransf, int isign, void* stream) {
  if (!plan || !c || !f || ntransf < 0 || (isign != 1 && isign != -1))
    return fail(HB_ERR_INVALID, "hb_nufft_type1: null argument, negative ntransf or isign not +-1");
  DeviceGuard dg(plan->device);
  const long long K = plan->g.K, nm = nmodes(plan);
  for (int64_t t0 = 0; t0 < ntransf; t0 += plan->maxbatch) {
    const int nb = (int)((ntransf - t0) < plan->maxbatch ? (ntransf - t0) : plan->maxbatch);
    if (int r = type1_batch(plan, (const float2*)c + t0 * K, K, (float2*)f + t0 * nm, nm, nb, isign,
                            (cudaStream_t)stream))
      return r;
  }
  return HB_OK;
}

int hb_nufft_type2(const hb_nufft* plan, const void* f, void* c, int64_t ntransf, int isign, void* stream) {
  if (!plan || !c || !f || ntransf < 0 || (isign != 1 && isign != -1))
    return fail(HB_ERR_INVALID, "hb_nufft_type2: null argument, negative ntransf or isign not +-1");
  DeviceGuard dg(plan->device);
  const long long K = plan->g.K, nm = nmodes(plan);
  for (int64_t t0 = 0; t0 < ntransf; t0 += plan->maxbatch) {
    const int nb = (int)((ntransf - t0) < plan->maxbatch ? (ntransf - t0) : plan->maxbatch);
    if (int r = type2_batch(plan, (const float2*)f + t0 * nm, nm, (float2*)c + t0 * K, K, nb, isign,
                            (cudaStream_t)stream))
      return r;
  }
  return HB_OK;
}

int hb_sense_adjoint_nufft(const hb_nufft* plan, const void* kdata, const void* smaps, const int64_t* coils,
                           int64_t ncoil, const float* weights, void* out, int accumulate, void* stream) {
  if (!plan || !kdata || !smaps || !out || ncoil < 0 || (ncoil > 0 && !coils))
    return fail(HB_ERR_INVALID, "hb_sense_adjoint_nufft: null argument or negative ncoil");
  for (int64_t b = 0; b < ncoil; ++b)
    if (coils[b] < 0) return fail(HB_ERR_INVALID, "hb_sense_adjoint_nufft: negative coil index");
  DeviceGuard dg(plan->device);
  cudaStream_t st = (cudaStream_t)stream;
  const long long K = plan->g.K, nm = nmodes(plan);
  const unsigned vb = (unsigned)((nm + 255) / 256), kb = (unsigned)((K + 255) / 256);
  if (ncoil == 0 && !accumulate) HB_CUDA(cudaMemsetAsync(out, 0, nm * sizeof(float2), st));
  for (int64_t b0 = 0; b0 < ncoil; b0 += plan->maxbatch) {
    const int nb = (int)((ncoil - b0) < plan->maxbatch ? (ncoil - b0) : plan->maxbatch);
    const float2* src = (const float2*)kdata + b0 * K;
    if (weights) {  // w * kdata rows into the plan's k-space temporaries
      KdataPtrs ys{};
      for (int b = 0; b < nb; ++b) ys.y[b] = src + b * K;
      {
        LaunchScope ls(HB_KERNEL_NUFFT, st);
        sense_kspace_weight_kernel<<<kb, 256, 0, st>>>(plan->kbuf, nb, K, ys, weights);
      }
      HB_CHECK_LAUNCH();
      src = plan->kbuf;
    }
    if (int r = type1_batch(plan, src, K, plan->modes, nm, nb, +1, st)) return r;
    CoilMaps maps{};
    for (int b = 0; b < nb; ++b) maps.s[b] = (const float2*)smaps + coils[b0 + b] * nm;
    {
      LaunchScope ls(HB_KERNEL_NUFFT, st);
      sense_coil_combine_kernel<<<vb, 256, 0, st>>>(plan->modes, nb, nm, maps, (float2*)out,
                                                    (b0 > 0 || accumulate) ? 1 : 0);
    }
    HB_CHECK_LAUNCH();
  }
  return HB_OK;
}

int hb_sense_forward_nufft(const hb_nufft* plan, const void* x, const void* smaps, const int64_t* coils,
                           int64_t ncoil, void* kdata, void* stream) {
  if (!plan || !x || !smaps || !kdata || ncoil < 0 || (ncoil > 0 && !coils))
    return fail(HB_ERR_INVALID, "hb_sense_forward_nufft: null argument or negative ncoil");
  for (int64_t b = 0; b < ncoil; ++b)
    if (coils[b] < 0) return fail(HB_ERR_INVALID, "hb_sense_forward_nufft: negative coil index");
  DeviceGuard dg(plan->device);
  cudaStream_t st = (cudaStream_t)stream;
  const long long K = plan->g.K, nm = nmodes(plan);
  const unsigned vb = (unsigned)((nm + 255) / 256);
  for (int64_t b0 = 0; b0 < ncoil; b0 += plan->maxbatch) {
    const int nb = (int)((ncoil - b0) < plan->maxbatch ? (ncoil - b0) : plan->maxbatch);
    CoilMaps maps{};
    for (int b = 0; b < nb; ++b) maps.s[b] = (const float2*)smaps + coils[b0 + b] * nm;
    {
      LaunchScope ls(HB_KERNEL_NUFFT, st);
      sense_coil_expand_kernel<<<vb, 256, 0, st>>>((const float2*)x, nb, nm, maps, plan->modes);
    }
    HB_CHECK_LAUNCH();
    if (int r = type2_batch(plan, plan->modes, nm, (float2*)kdata + b0 * K, K, nb, -1, st)) return r;
  }
  return HB_OK;
}

int hb_sense_normal_nufft(const hb_nufft* plan, const void* x, const void* smaps, const int64_t* coils, int64_t ncoil,
                          const void* kdata, const float* weights, void* out, int accumulate, void* stream) {
  if (!plan || !x || !smaps || !out || ncoil < 0 || (ncoil > 0 && !coils))
    return fail(HB_ERR_INVALID, "hb_sense_normal_nufft: null argument or negative ncoil");
  for (int64_t b = 0; b < ncoil; ++b)
    if (coils[b] < 0) return fail(HB_ERR_INVALID, "hb_sense_normal_nufft: negative coil index");
  DeviceGuard dg(plan->device);
  cudaStream_t st = (cudaStream_t)stream;
  const long long K = plan->g.K, nm = nmodes(plan);
  const unsigned vb = (unsigned)((nm + 255) / 256), kb = (unsigned)((K + 255) / 256);
  if (ncoil == 0 && !accumulate) HB_CUDA(cudaMemsetAsync(out, 0, nm * sizeof(float2), st));
  for (int64_t b0 = 0; b0 < ncoil; b0 += plan->maxbatch) {
    const int nb = (int)((ncoil - b0) < plan->maxbatch ? (ncoil - b0) : plan->maxbatch);
    CoilMaps maps{};
    KdataPtrs ys{};
    for (int b = 0; b < nb; ++b) {
      maps.s[b] = (const float2*)smaps + coils[b0 + b] * nm;
      ys.y[b] = kdata ? (const float2*)kdata + coils[b0 + b] * K : nullptr;
    }
    {
      LaunchScope ls(HB_KERNEL_NUFFT, st);
      sense_coil_expand_kernel<<<vb, 256, 0, st>>>((const float2*)x, nb, nm, maps, plan->modes);
    }
    HB_CHECK_LAUNCH();
    if (int r = type2_batch(plan, plan->modes, nm, plan->kbuf, K, nb, -1, st)) return r;
    if (kdata || weights) {
      LaunchScope ls(HB_KERNEL_NUFFT, st);
      sense_kspace_mid_kernel<<<kb, 256, 0, st>>>(plan->kbuf, nb, K, ys, weights);
    }
    HB_CHECK_LAUNCH();
    if (int r = type1_batch(plan, plan->kbuf, K, plan->modes, nm, nb, +1, st)) return r;
    {
      LaunchScope ls(HB_KERNEL_NUFFT, st);
      sense_coil_combine_kernel<<<vb, 256, 0, st>>>(plan->modes, nb, nm, maps, (float2*)out,
                                                    (b0 > 0 || accumulate) ? 1 : 0);
    }
    HB_CHECK_LAUNCH();
  }
  return HB_OK;
}

int hb_diag_build_nufft(const hb_plan* plan, const float* coords, int64_t nsamples, double tol, const float* weights,
                        float* packed, void* T_complex, void* stream) {
  if (!plan || !coords || nsamples < 1) return fail(HB_ERR_INVALID, "hb_diag_build_nufft: null plan or no samples");
  if (!packed && !T_complex) return fail(HB_ERR_INVALID, "hb_diag_build_nufft: no output requested");
  int N[3], dev = 0;
  plan_geometry(plan, N, &dev);
  DeviceGuard dg(dev);
  cudaStream_t st = (cudaStream_t)stream;
  const int M[3] = {2 * N[0], 2 * N[1], 2 * N[2]};
  const long long vol = (long long)M[0] * M[1] * M[2];
  float2* T = nullptr;
  float2* tw = nullptr;
  int rc = HB_OK;
  auto cuda_fail = [&](cudaError_t e, const char* what) {
    rc = fail(HB_ERR_CUDA, std::string("hb_diag_build_nufft: ") + what + ": " + cudaGetErrorString(e));
  };
  do {
    cudaError_t e;
    if ((e = cudaMalloc(&T, vol * sizeof(float2))) != cudaSuccess) { cuda_fail(e, "alloc"); break; }
    const std::vector<float2> tables = team_tables(M);
    if ((e = cudaMalloc(&tw, tables.size() * sizeof(float2))) != cudaSuccess) { cuda_fail(e, "alloc"); break; }
    if ((e = cudaMemcpyAsync(tw, tables.data(), tables.size() * sizeof(float2), cudaMemcpyHostToDevice, st)) !=
        cudaSuccess) {
      cuda_fail(e, "upload");
      break;
    }
    // PSF in circulant layout on the 2x grid, then T = FFT(PSF)
    if ((rc = nufft_psf_circulant(M, coords, nsamples, tol, weights, dev, T, st)) != HB_OK) break;
    if ((e = fft3_grid<-1>(M[0], M[1], M[2], tw, T, 1, st)) != cudaSuccess) { cuda_fail(e, "fft"); break; }
    if (packed && (rc = hb_diag_pack(plan, T, packed, stream)) != HB_OK) break;
    if (T_complex &&
        (e = cudaMemcpyAsync(T_complex, T, vol * sizeof(float2), cudaMemcpyDeviceToDevice, st)) != cudaSuccess) {
      cuda_fail(e, "copy");
      break;
    }
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) cuda_fail(e, "sync");
  } while (false);
  if (rc != HB_OK) cudaStreamSynchronize(st);
  cudaFree(T);
  cudaFree(tw);
  return rc;
}

}  // extern "C"
