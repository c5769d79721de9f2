// Toeplitz diagonal (the 2x-grid transfer function T) construction and packing.
//
// The reference builds T as fftn(ifftshift(NUFFT1(NUFFT2(delta)))) on the 2x grid
// (lib/fft/nufft.cpp:932-971); the two NUFFTs of a centred impulse reduce to the direct
// NUDFT  psf(d) = prod(M)^-1 sum_j exp(+i c_j . d),  d in [-N, N)^3.  Taking the FFT of
// that sum analytically gives, per axis, a Dirichlet kernel:
//   T[k] = prod(M)^-1 sum_j prod_a D_{N_a}(c_{j,a} - 2*pi*k_a/M_a),
//   D_N(phi) = sum_{d=-N}^{N-1} exp(i d phi) = exp(-i phi/2) sin(N phi) / sin(phi/2).
// So T is a sum over samples of separable rank-1 terms: the kernels below tabulate D
// per axis for a chunk of samples (FP64) and accumulate the triple product into an FP64
// grid with a register-tiled contraction.  No FFT and no NUFFT tolerance are involved.
#pragma once

#include "common.cuh"
#include "fft.cuh"

namespace hb {

// D[j][k] for one axis: coords c (float, [K] with stride), k in [0, M), N = M/2.
__global__ void dirichlet_table_kernel(const float* __restrict__ c, long long j0, int nj, int M,
                                       double2* __restrict__ D) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)nj * M) return;
  const int jl = (int)(idx / M), k = (int)(idx % M);
  const int N = M / 2;
  const double phi = (double)c[j0 + jl] - 2.0 * 3.14159265358979323846 * (double)k / (double)M;
  double re, im;
  const double s2 = sin(0.5 * phi);
  if (fabs(s2) > 1e-8) {
    const double amp = sin((double)N * phi) / s2;
    double sh, ch;
    sincos(-0.5 * phi, &sh, &ch);
    re = amp * ch;
    im = amp * sh;
  } else {
    re = 0.0;
    im = 0.0;
    for (int d = -N; d < N; ++d) {
      double sd, cd;
      sincos((double)d * phi, &sd, &cd);
      re += cd;
      im += sd;
    }
  }
  D[idx] = make_double2(re, im);
}

// acc[kz][ky][kx] += sum_j Dz[j][kz] * Dy[j][ky] * Dx[j][kx]   (FP64)
// CPLX: the full complex sum; otherwise only its real part (half the FMAs), which is all
// the normal operator reads.  grid: (ceil(M2/64), ceil(M1/(16*TI)), M0), block 16 x 16
// lanes, each lane a TI x 4 (ky, kx) register tile.
constexpr int kDiagTileX = 64;
constexpr int kDiagJB = 16;

template <bool CPLX, int TI>
__global__ void __launch_bounds__(256)
diag_accumulate_kernel(const double2* __restrict__ Dz, const double2* __restrict__ Dy,
                       const double2* __restrict__ Dx, int nj, int M0, int M1, int M2,
                       double2* __restrict__ acc) {
  constexpr int TY = 16 * TI;
  __shared__ double2 As[kDiagJB][TY];
  __shared__ double2 Bs[kDiagJB][kDiagTileX];
  const int kx0 = blockIdx.x * kDiagTileX, ky0 = blockIdx.y * TY, kz = blockIdx.z;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  double2 r[TI][4];
#pragma unroll
  for (int i = 0; i < TI; ++i)
#pragma unroll
    for (int m = 0; m < 4; ++m) r[i][m] = make_double2(0.0, 0.0);

  for (int jb = 0; jb < nj; jb += kDiagJB) {
    __syncthreads();
    for (int i = threadIdx.x; i < kDiagJB * TY; i += 256) {
      const int jl = i / TY, q = i % TY;
      const int j = jb + jl;
      double2 a = make_double2(0.0, 0.0);
      const int ky = ky0 + q;
      if (j < nj && ky < M1) {
        const double2 dz = Dz[(long long)j * M0 + kz];
        const double2 dy = Dy[(long long)j * M1 + ky];
        a = make_double2(dz.x * dy.x - dz.y * dy.y, dz.x * dy.y + dz.y * dy.x);
      }
      As[jl][q] = a;
    }
    for (int i = threadIdx.x; i < kDiagJB * kDiagTileX; i += 256) {
      const int jl = i / kDiagTileX, q = i % kDiagTileX;
      const int j = jb + jl, kx = kx0 + q;
      Bs[jl][q] = (j < nj && kx < M2) ? Dx[(long long)j * M2 + kx] : make_double2(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll 4
    for (int jl = 0; jl < kDiagJB; ++jl) {
      double2 av[TI], bv[4];
#pragma unroll
      for (int i = 0; i < TI; ++i) av[i] = As[jl][ty + 16 * i];
#pragma unroll
      for (int m = 0; m < 4; ++m) bv[m] = Bs[jl][tx + 16 * m];
#pragma unroll
      for (int i = 0; i < TI; ++i)
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          r[i][m].x = fma(av[i].x, bv[m].x, fma(-av[i].y, bv[m].y, r[i][m].x));
          if (CPLX) r[i][m].y = fma(av[i].x, bv[m].y, fma(av[i].y, bv[m].x, r[i][m].y));
        }
    }
  }
#pragma unroll
  for (int i = 0; i < TI; ++i) {
    const int ky = ky0 + ty + 16 * i;
    if (ky >= M1) continue;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int kx = kx0 + tx + 16 * m;
      if (kx >= M2) continue;
      double2* p = acc + ((long long)kz * M1 + ky) * M2 + kx;
      double2 v = *p;
      v.x += r[i][m].x;
      if (CPLX) v.y += r[i][m].y;
      *p = v;
    }
  }
}

// FP64 accumulator (unscaled sum over samples) -> complex64 T in the reference layout
// [M0][M1][M2], scaled by 1/prod(M) (the psf normalisation).
__global__ void diag_to_complex_kernel(const double2* __restrict__ acc, long long n, double scale,
                                       float2* __restrict__ T) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  T[i] = make_float2((float)(acc[i].x * scale), (float)(acc[i].y * scale));
}

// Pack Re(T) into the layout pass B reads: packed[kx][h][ky'][p] (ky = 2*ky' + h), one
// M0-long column per (kx, ky) in the order the z transform's lanes consume it: position
// p = t*E + r holds kz = dout_index<M0>(t, r) (lane t's E values are contiguous, so a lane
// fetches them with 16-byte loads).  Scaled by `scale` (the inverse-FFT factor 1/prod(M),
// plus any psf scaling).  Source is either a float2 reference-layout T or a double2
// accumulator.
template <typename Src>
__global__ void diag_pack_kernel(const Src* __restrict__ T, int M0, int M1, int M2, double scale,
                                 float* __restrict__ packed) {
  const long long n = (long long)M0 * M1 * M2;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // i enumerates the packed layout
  const int kz = column_kz(M0, (int)(i % M0));
  long long r = i / M0;
  const int N1 = M1 / 2;
  const int kyh = (int)(r % N1);
  r /= N1;
  const int h = (int)(r % 2);
  const int kx = (int)(r / 2);
  const int ky = 2 * kyh + h;
  const double re = (double)T[((long long)kz * M1 + ky) * M2 + kx].x;
  packed[i] = (float)(re * scale);
}

}  // namespace hb
