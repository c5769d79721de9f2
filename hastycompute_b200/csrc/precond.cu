// Circulant preconditioner of the SENSE normal operator (include/hasty_b200.h, section
// "Circulant preconditioner").  Replaces hasty::mri::CirculantPreconditionerOp
// (lib/mri/precond.cpp:17-60: apply; :65-117: build_diagonal) and its Python twin
// circulant_precond (python/python/hastypy/base/torch_precond.py:60-105), both "based on
// sigpy".
//
// For B = sum_c S_c^H Toep S_c (+ lambda I) the best circulant approximation in the
// unitary Fourier basis of the N grid has the diagonal
//   d[k] = (F B F^H)[k, k] = prod(N)^-1 sum_delta psf(delta) R(delta) e^{-2 pi i k.delta / N} + lambda,
//   R(delta) = sum_c sum_m conj(S_c[m + delta]) S_c[m]        (coil-map autocorrelations),
// where psf is the Toeplitz operator's kernel on the 2x grid.  It is evaluated as in
// sigpy: R = IFFT_2N(sum_c |FFT_2N(pad(conj S_c))|^2), d = FFT_2N(psf * R)[2k] / prod(N)
// + lambda, and P = IFFT_N diag(1 / d) FFT_N.  The diagonal is stored in FFT (uncentred)
// order; the reference's centred form ifftc(diag * fftc(x)) is the same operator with the
// diagonal fftshifted.  The two reference builders disagree on centring and scaling (the
// C++ one also accumulates into a [nsamples] tensor), so the construction follows the
// definition they both port.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/hasty_b200.h"
#include "fft3_launch.cuh"
#include "runtime.cuh"

using namespace hb;

namespace {

constexpr int kMaxMaps = 8;  // coil maps transformed per batch
struct MapBatch {
  const float2* s[kMaxMaps];
};

// G[b] = pad_2N(conj(S_b)) (zero outside the N grid)
__global__ void precond_pad_conj_kernel(MapBatch maps, int N0, int N1, int N2, float2* G) {
  const int M0 = 2 * N0, M1 = 2 * N1, M2 = 2 * N2;
  const long long vol = (long long)M0 * M1 * M2;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= vol) return;
  const int x = (int)(i % M2), y = (int)((i / M2) % M1), z = (int)(i / ((long long)M1 * M2));
  float2 v = make_float2(0.f, 0.f);
  if (x < N2 && y < N1 && z < N0) v = cconj(maps.s[blockIdx.y][((long long)z * N1 + y) * N2 + x]);
  G[(long long)blockIdx.y * vol + i] = v;
}

// Q (+)= sum_b |G[b]|^2
__global__ void precond_abs2_kernel(const float2* G, int nb, long long vol, float* Q, int first) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= vol) return;
  float acc = first ? 0.f : Q[i];
  for (int b = 0; b < nb; ++b) {
    const float2 v = G[b * vol + i];
    acc = fmaf(v.x, v.x, fmaf(v.y, v.y, acc));
  }
  Q[i] = acc;
}

__global__ void precond_real_to_complex_kernel(const float* Q, long long vol, float2* G) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < vol) G[i] = make_float2(Q[i], 0.f);
}

// G = G * psf * s
__global__ void precond_mul_psf_kernel(float2* G, const float2* psf, long long vol, float s) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < vol) G[i] = cscale(cmul(G[i], psf[i]), s);
}

// out[k] = 1 / (Re G[2k] / prod(N) + lambda), or 1 where that is not positive
__global__ void precond_finish_kernel(const float2* G, int N0, int N1, int N2, float inv_n, float lambda, float* out) {
  const long long nv = (long long)N0 * N1 * N2;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  const int x = (int)(i % N2), y = (int)((i / N2) % N1), z = (int)(i / ((long long)N1 * N2));
  const long long j = ((long long)(2 * z) * (2 * N1) + 2 * y) * (2 * N2) + 2 * x;
  const float d = G[j].x * inv_n + lambda;
  out[i] = d > 0.f ? 1.f / d : 1.f;
}

// z *= d / nv
__global__ void precond_scale_kernel(float2* z, const float* d, long long nv) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nv) z[i] = cscale(z[i], d[i] / (float)nv);
}

unsigned blocks_for(long long n) { return (unsigned)((n + 255) / 256); }

}  // namespace

extern "C" {

int hb_precond_build(const hb_plan* plan, const float* coords, int64_t nsamples, double tol, const void* smaps,
                     const int64_t* coils, int64_t ncoil, float lambda, float* precond, void* stream) {
  if (!plan || !coords || nsamples < 1 || !smaps || !precond || ncoil < 1 || !coils)
    return fail(HB_ERR_INVALID, "hb_precond_build: null argument, no samples or no coils");
  for (int64_t c = 0; c < ncoil; ++c)
    if (coils[c] < 0) return fail(HB_ERR_INVALID, "hb_precond_build: negative coil index");
  int N[3], dev = 0;
  plan_geometry(plan, N, &dev);
  DeviceGuard dg(dev);
  cudaStream_t st = (cudaStream_t)stream;
  const int M[3] = {2 * N[0], 2 * N[1], 2 * N[2]};
  const long long vol = (long long)M[0] * M[1] * M[2];
  const long long nv = (long long)N[0] * N[1] * N[2];
  const int nb = (int)(ncoil < kMaxMaps ? ncoil : kMaxMaps);
  float2* psf = nullptr;
  float2* G = nullptr;
  float* Q = nullptr;
  float2* tw = nullptr;
  int rc = HB_OK;
  auto cuda_fail = [&](cudaError_t e, const char* what) {
    rc = fail(HB_ERR_CUDA, std::string("hb_precond_build: ") + what + ": " + cudaGetErrorString(e));
  };
  do {
    cudaError_t e;
    if ((e = cudaMalloc(&psf, vol * sizeof(float2))) != cudaSuccess) { cuda_fail(e, "alloc"); break; }
    if ((rc = nufft_psf_circulant(M, coords, nsamples, tol, nullptr, dev, psf, st)) != HB_OK) break;
    if ((e = cudaMalloc(&G, (size_t)nb * vol * sizeof(float2))) != cudaSuccess) { cuda_fail(e, "alloc"); break; }
    if ((e = cudaMalloc(&Q, vol * sizeof(float))) != cudaSuccess) { cuda_fail(e, "alloc"); break; }
    const std::vector<float2> tables = fftl::team_tables(M);
    if ((e = cudaMalloc(&tw, tables.size() * sizeof(float2))) != cudaSuccess) { cuda_fail(e, "alloc"); break; }
    if ((e = cudaMemcpyAsync(tw, tables.data(), tables.size() * sizeof(float2), cudaMemcpyHostToDevice, st)) !=
        cudaSuccess) {
      cuda_fail(e, "upload");
      break;
    }
    // sum_c |FFT_2N(pad(conj S_c))|^2, nb maps at a time
    for (int64_t c0 = 0; c0 < ncoil && rc == HB_OK; c0 += nb) {
      const int n = (int)((ncoil - c0) < nb ? (ncoil - c0) : nb);
      MapBatch maps{};
      for (int b = 0; b < n; ++b) maps.s[b] = (const float2*)smaps + coils[c0 + b] * nv;
      {
        LaunchScope ls(HB_KERNEL_DIAG, st);
        precond_pad_conj_kernel<<<dim3(blocks_for(vol), n), 256, 0, st>>>(maps, N[0], N[1], N[2], G);
      }
      if ((e = cudaGetLastError()) != cudaSuccess) { cuda_fail(e, "kernel launch"); break; }
      if ((e = fftl::fft3_grid<-1>(M[0], M[1], M[2], tw, G, n, st, HB_KERNEL_DIAG)) != cudaSuccess) {
        cuda_fail(e, "fft");
        break;
      }
      {
        LaunchScope ls(HB_KERNEL_DIAG, st);
        precond_abs2_kernel<<<blocks_for(vol), 256, 0, st>>>(G, n, vol, Q, c0 == 0 ? 1 : 0);
      }
      if ((e = cudaGetLastError()) != cudaSuccess) cuda_fail(e, "kernel launch");
    }
    if (rc != HB_OK) break;
    // R = IFFT(Q) (normalised), x psf, FFT, every other sample
    {
      LaunchScope ls(HB_KERNEL_DIAG, st);
      precond_real_to_complex_kernel<<<blocks_for(vol), 256, 0, st>>>(Q, vol, G);
    }
    if ((e = fftl::fft3_grid<1>(M[0], M[1], M[2], tw, G, 1, st, HB_KERNEL_DIAG)) != cudaSuccess) {
      cuda_fail(e, "fft");
      break;
    }
    {
      LaunchScope ls(HB_KERNEL_DIAG, st);
      precond_mul_psf_kernel<<<blocks_for(vol), 256, 0, st>>>(G, psf, vol, (float)(1.0 / (double)vol));
    }
    if ((e = fftl::fft3_grid<-1>(M[0], M[1], M[2], tw, G, 1, st, HB_KERNEL_DIAG)) != cudaSuccess) {
      cuda_fail(e, "fft");
      break;
    }
    {
      LaunchScope ls(HB_KERNEL_DIAG, st);
      precond_finish_kernel<<<blocks_for(nv), 256, 0, st>>>(G, N[0], N[1], N[2], (float)(1.0 / (double)nv), lambda,
                                                            precond);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) { cuda_fail(e, "kernel launch"); break; }
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) cuda_fail(e, "sync");
  } while (false);
  if (rc != HB_OK) cudaStreamSynchronize(st);
  cudaFree(psf);
  cudaFree(G);
  cudaFree(Q);
  cudaFree(tw);
  return rc;
}

int hb_precond_apply(const hb_plan* plan, const float* precond, const void* in, void* out, void* stream) {
  if (!plan || !precond || !in || !out) return fail(HB_ERR_INVALID, "hb_precond_apply: null argument");
  int N[3], dev = 0;
  plan_geometry(plan, N, &dev);
  DeviceGuard dg(dev);
  cudaStream_t st = (cudaStream_t)stream;
  const long long nv = (long long)N[0] * N[1] * N[2];
  const float2* tw = plan_image_tables(plan);
  if (in != out) HB_CUDA(cudaMemcpyAsync(out, in, nv * sizeof(float2), cudaMemcpyDeviceToDevice, st));
  HB_CUDA(fftl::fft3_grid<-1>(N[0], N[1], N[2], tw, (float2*)out, 1, st, HB_KERNEL_CG_UPDATE));
  {
    LaunchScope ls(HB_KERNEL_CG_UPDATE, st);
    precond_scale_kernel<<<blocks_for(nv), 256, 0, st>>>((float2*)out, precond, nv);
  }
  HB_CHECK_LAUNCH();
  HB_CUDA(fftl::fft3_grid<1>(N[0], N[1], N[2], tw, (float2*)out, 1, st, HB_KERNEL_CG_UPDATE));
  return HB_OK;
}

}  // extern "C"
