// Host launchers of the batched 3D FFT (fft3_kernels.cuh) on [nt][n0][n1][n2] complex64
// grids, in place, for every team length the library compiles; shared by the NUFFT and
// the circulant preconditioner.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "fft3_kernels.cuh"
#include "runtime.cuh"

namespace hb {
namespace fftl {

inline bool team_length(int L, int* E, int* S) {
  switch (L) {
    case 8: *E = 4; *S = 2; return true;
    case 16: *E = 4; *S = 4; return true;
    case 32: *E = 8; *S = 4; return true;
    case 64: *E = 8; *S = 8; return true;
    case 128: *E = 16; *S = 8; return true;
    case 256: *E = 16; *S = 16; return true;
    case 96: *E = 24; *S = 4; return true;
    case 160: *E = 40; *S = 4; return true;
    case 192: *E = 24; *S = 8; return true;
    case 320: *E = 40; *S = 8; return true;
    case 512: *E = 32; *S = 16; return true;
    default: return false;
  }
}

// ---- 3D FFT of nt grids [n0][n1][n2], in place ----
template <auto kernel>
inline cudaError_t allow_smem(size_t bytes) {
  static bool done[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || done[dev & 63] || bytes <= 48 * 1024) return e;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) done[dev & 63] = true;
  return e;
}

template <int L, int DIR>
cudaError_t lines_contig(float2* d, long long nlines, const float2* tw, cudaStream_t st, int kind) {
  using C = LineCfg<L>;
  const size_t smem = C::SMEM_C * sizeof(float2);
  cudaError_t e = allow_smem<fft_lines_contig_kernel<L, DIR>>(smem);
  if (e != cudaSuccess) return e;
  long long blocks = (nlines + C::NTEAMS_C - 1) / C::NTEAMS_C;
  if (blocks > 148 * 16) blocks = 148 * 16;
  LaunchScope ls(kind, st);
  fft_lines_contig_kernel<L, DIR><<<(unsigned)blocks, C::THREADS_C, smem, st>>>(d, nlines, tw);
  return cudaGetLastError();
}

template <int L, int DIR>
cudaError_t lines_strided(float2* d, long long row_stride, int ncols, int ny, long long oy, int nz, long long oz,
                          const float2* tw, cudaStream_t st, int kind) {
  using C = LineCfg<L>;
  const size_t smem = C::SMEM_S * sizeof(float2);
  cudaError_t e = allow_smem<fft_lines_strided_kernel<L, DIR>>(smem);
  if (e != cudaSuccess) return e;
  dim3 grid((ncols + C::XT - 1) / C::XT, ny, nz);
  LaunchScope ls(kind, st);
  fft_lines_strided_kernel<L, DIR><<<grid, C::THREADS_S, smem, st>>>(d, row_stride, ncols, oy, oz, tw);
  return cudaGetLastError();
}

template <int DIR>
cudaError_t contig_any(int L, float2* d, long long nlines, const float2* tw, cudaStream_t st, int kind) {
  switch (L) {
    case 8: return lines_contig<8, DIR>(d, nlines, tw, st, kind);
    case 16: return lines_contig<16, DIR>(d, nlines, tw, st, kind);
    case 32: return lines_contig<32, DIR>(d, nlines, tw, st, kind);
    case 64: return lines_contig<64, DIR>(d, nlines, tw, st, kind);
    case 128: return lines_contig<128, DIR>(d, nlines, tw, st, kind);
    case 256: return lines_contig<256, DIR>(d, nlines, tw, st, kind);
    case 96: return lines_contig<96, DIR>(d, nlines, tw, st, kind);
    case 160: return lines_contig<160, DIR>(d, nlines, tw, st, kind);
    case 192: return lines_contig<192, DIR>(d, nlines, tw, st, kind);
    case 320: return lines_contig<320, DIR>(d, nlines, tw, st, kind);
    case 512: return lines_contig<512, DIR>(d, nlines, tw, st, kind);
    default: return cudaErrorInvalidValue;
  }
}

template <int DIR>
cudaError_t strided_any(int L, float2* d, long long rs, int ncols, int ny, long long oy, int nz, long long oz,
                        const float2* tw, cudaStream_t st, int kind) {
  switch (L) {
    case 8: return lines_strided<8, DIR>(d, rs, ncols, ny, oy, nz, oz, tw, st, kind);
    case 16: return lines_strided<16, DIR>(d, rs, ncols, ny, oy, nz, oz, tw, st, kind);
    case 32: return lines_strided<32, DIR>(d, rs, ncols, ny, oy, nz, oz, tw, st, kind);
    case 64: return lines_strided<64, DIR>(d, rs, ncols, ny, oy, nz, oz, tw, st, kind);
    case 128: return lines_strided<128, DIR>(d, rs, ncols, ny, oy, nz, oz, tw, st, kind);
    case 256: return lines_strided<256, DIR>(d, rs, ncols, ny, oy, nz, oz, tw, st, kind);
    case 96: return lines_strided<96, DIR>(d, rs, ncols, ny, oy, nz, oz, tw, st, kind);
    case 160: return lines_strided<160, DIR>(d, rs, ncols, ny, oy, nz, oz, tw, st, kind);
    case 192: return lines_strided<192, DIR>(d, rs, ncols, ny, oy, nz, oz, tw, st, kind);
    case 320: return lines_strided<320, DIR>(d, rs, ncols, ny, oy, nz, oz, tw, st, kind);
    case 512: return lines_strided<512, DIR>(d, rs, ncols, ny, oy, nz, oz, tw, st, kind);
    default: return cudaErrorInvalidValue;
  }
}

// nt grids [n0][n1][n2] in place; tw: team tables of n0, n1, n2 back to back
template <int DIR>
cudaError_t fft3_grid(int n0, int n1, int n2, const float2* tw, float2* grid, int nt, cudaStream_t st,
                      int kind = HB_KERNEL_NUFFT) {
  const long long vol = (long long)n0 * n1 * n2;
  cudaError_t e = contig_any<DIR>(n2, grid, (long long)nt * n0 * n1, tw + n0 + n1, st, kind);
  if (e != cudaSuccess) return e;
  if (n1 > 1) {  // a length-1 axis (the leading axes of a 1-D or 2-D plan) needs no transform
    e = strided_any<DIR>(n1, grid, n2, n2, n0, (long long)n1 * n2, nt, vol, tw + n0, st, kind);
    if (e != cudaSuccess) return e;
  }
  if (n0 == 1) return cudaSuccess;
  return strided_any<DIR>(n0, grid, (long long)n1 * n2, n2, n1, n2, nt, vol, tw, st, kind);
}

// Team twiddle tables of the three lengths, back to back (forward sign, FP64 rounded); a
// length-1 axis holds the single entry 1.
inline std::vector<float2> team_tables(const int* n) {
  std::vector<float2> tw;
  for (int a = 0; a < 3; ++a) {
    if (n[a] == 1) {
      tw.push_back(make_float2(1.f, 0.f));
      continue;
    }
    int E = 0, S = 0;
    team_length(n[a], &E, &S);
    for (int k1 = 0; k1 < E; ++k1)
      for (int t = 0; t < S; ++t) {
        const double ang = -2.0 * M_PI * (double)(t * k1) / (double)n[a];
        tw.push_back(make_float2((float)std::cos(ang), (float)std::sin(ang)));
      }
  }
  return tw;
}

}  // namespace fftl
}  // namespace hb
