// Batched in-place 3D FFT building blocks on [nt][n0][n1][n2] complex64 grids: one
// kernel per axis, built on the team engine of fft.cuh (unnormalised, DIR = -1 forward,
// +1 inverse).  Used by the NUFFT's fine grid.
//
//   fft_lines_contig   : lines along the contiguous axis (n2); a team of S lanes loads
//                        its line directly (S consecutive values per load).
//   fft_lines_strided  : lines along a strided axis (n1 or n0); a CTA stages a tile of
//                        L rows x XT consecutive columns in shared memory (rows of XT
//                        values are contiguous in global memory), each team transforms
//                        one column, the tile is written back.
#pragma once

#include "common.cuh"
#include "fft.cuh"

namespace hb {

template <int L>
struct LineCfg {
  static constexpr int E = TeamCfg<L>::E, S = TeamCfg<L>::S;
  static constexpr int TBUF = team_buf_stride<L>();
  // contiguous kernel: 256 threads
  static constexpr int THREADS_C = 256;
  static constexpr int NTEAMS_C = THREADS_C / S;
  static constexpr int SMEM_C = NTEAMS_C * TBUF + L;  // float2 slots
  // strided kernel: one team per tile column
  static constexpr int XT = 16;
  static constexpr int THREADS_S = XT * S;
  static constexpr int TILE_LD = XT + 1;
  static constexpr int SMEM_S = L * TILE_LD + XT * TBUF + L;  // float2 slots
};

// nlines lines of length L, line i at data + i * L.  The loop runs the same number of
// rounds in every team, so teams sharing a warp stay converged for the warp-level
// exchanges; a team without a line of its own transforms (and discards) a copy.
template <int L, int DIR>
__global__ void __launch_bounds__(LineCfg<L>::THREADS_C) fft_lines_contig_kernel(float2* data, long long nlines,
                                                                                 const float2* tw) {
  using C = LineCfg<L>;
  constexpr int E = C::E, S = C::S;
  extern __shared__ float2 smem[];
  float2* xbuf = smem;
  float2* tws = xbuf + C::NTEAMS_C * C::TBUF;
  for (int i = threadIdx.x; i < L; i += C::THREADS_C) tws[i] = tw[i];
  __syncthreads();
  const int team = threadIdx.x / S, t = threadIdx.x % S;
  float2* buf = xbuf + team * C::TBUF;
  for (long long base = (long long)blockIdx.x * C::NTEAMS_C; base < nlines; base += (long long)gridDim.x * C::NTEAMS_C) {
    const long long line = base + team;
    const bool ok = line < nlines;
    const float2* src = data + (ok ? line : nlines - 1) * L;
    float2 v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = src[din_index<L>(t, e)];
    team_fft_din_to_dout<L, DIR, false>(v, t, buf, tws);
    if (ok) {
      float2* dst = data + line * L;
#pragma unroll
      for (int r = 0; r < E; ++r) dst[dout_index<L>(t, r)] = v[r];
    }
  }
}

// Lines of length L along an axis with element stride `row_stride`; the CTA at
// (blockIdx.x, blockIdx.y, blockIdx.z) covers columns [XT*blockIdx.x, +XT) (of ncols,
// contiguous) of the lines starting at data + blockIdx.y * oy_stride + blockIdx.z * oz_stride.
template <int L, int DIR>
__global__ void __launch_bounds__(LineCfg<L>::THREADS_S) fft_lines_strided_kernel(float2* data, long long row_stride,
                                                                                  int ncols, long long oy_stride,
                                                                                  long long oz_stride, const float2* tw) {
  using C = LineCfg<L>;
  constexpr int E = C::E, S = C::S, XT = C::XT, LD = C::TILE_LD;
  extern __shared__ float2 smem[];
  float2* tile = smem;                 // [L][LD]
  float2* xbuf = tile + L * LD;        // [XT][TBUF]
  float2* tws = xbuf + XT * C::TBUF;   // [L]
  const int x0 = blockIdx.x * XT;
  float2* base = data + (long long)blockIdx.y * oy_stride + (long long)blockIdx.z * oz_stride + x0;
  const int nc = (ncols - x0) < XT ? (ncols - x0) : XT;
  for (int i = threadIdx.x; i < L; i += C::THREADS_S) tws[i] = tw[i];
  // the tile arrives by asynchronous copies, all in flight at once
  for (int i = threadIdx.x; i < L * XT; i += C::THREADS_S) {
    const int r = i / XT, c = i % XT;
    if (c < nc) cp_async8(&tile[r * LD + c], base + (long long)r * row_stride + c);
    else tile[r * LD + c] = make_float2(0.f, 0.f);
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  const int team = threadIdx.x / S, t = threadIdx.x % S;  // team = tile column
  {
    float2 v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = tile[din_index<L>(t, e) * LD + team];
    team_fft_din_to_dout<L, DIR, false>(v, t, xbuf + team * C::TBUF, tws);
#pragma unroll
    for (int r = 0; r < E; ++r) tile[dout_index<L>(t, r) * LD + team] = v[r];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < L * XT; i += C::THREADS_S) {
    const int r = i / XT, c = i % XT;
    if (c < nc) base[(long long)r * row_stride + c] = tile[r * LD + c];
  }
}

}  // namespace hb
