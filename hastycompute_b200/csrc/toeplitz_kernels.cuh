// The three fused passes of the Toeplitz-embedded SENSE normal operator.
//
//   out = sum_c conj(S_c) * crop( IFFT_M( T * FFT_M( pad( S_c * x ) ) ) )     (M = 2N)
//
// Pass A  expand_fwd_x : per (slot, z, y-tile): S_c * x, zero-pad along x, M2-point FFT,
//                        written transposed to the spill  spill[slot][kx][z][y].
// Pass B  plane_yz     : per (slot, kx) a 2-CTA cluster owns one N0 x N1 (z, y) plane of
//                        the spill.  CTA h takes the ky-parity-h half of the 2x y-grid
//                        (ky = 2*ky' + h): pre-twiddle, N1-point FFT along y, then per ky'
//                        column an M0-point FFT along z (upper half zero), x T, inverse
//                        M0-point FFT keeping z < N0, inverse N1-point FFT along y and
//                        post-twiddle.  The two halves are summed through distributed
//                        shared memory and written back in place.
// Pass C  inv_x_combine: per (system, z, y-tile), looping over the coils: inverse
//                        M2-point FFT along x keeping x < N2, x conj(S_c), accumulate;
//                        epilogue adds lambda*x_in, optionally the previous output, and
//                        emits an FP64 partial of Re<x_in, out> for the CG.
//
// The inverse-FFT scale 1/(M0*M1*M2) is folded into the packed diagonal.
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"
#include "fft.cuh"

namespace hb {

// ---------------------------------------------------------------- launch geometry ----
// Pass A / C: a CTA covers YT consecutive y lines of one z plane; every team of S lanes
// transforms LPT of them.
template <int N2, int YT>
struct XPassCfg {
  static constexpr int M2 = 2 * N2;
  static constexpr int E = TeamCfg<M2>::E;
  static constexpr int S = TeamCfg<M2>::S;
  static constexpr int LPT = (YT * S > 256) ? (YT * S / 256) : 1;
  static constexpr int THREADS = YT * S / LPT;
  static constexpr int NTEAMS = THREADS / S;
  static constexpr int TILE_LD = YT + 1;  // padded row of the [kx][y] staging tile
  static constexpr int TBUF = team_buf_stride<M2>();
  // float2 slots of dynamic shared memory
  static constexpr int SMEM_F2 = M2 * TILE_LD + NTEAMS * TBUF + M2;
  static_assert(THREADS % 32 == 0, "x-pass CTA must be whole warps");
};

// Pass B: a CTA of THREADS lanes owns an N0 x N1 plane (one ky-parity half).
template <int N0, int N1>
struct PlaneCfg {
  static constexpr int M0 = 2 * N0;
  static constexpr int THREADS = (N0 * N1 >= 4096) ? 512 : 128;
  static constexpr int SR = TeamCfg<N1>::S, ER = TeamCfg<N1>::E;
  static constexpr int SZ = TeamCfg<M0>::S, EZ = TeamCfg<M0>::E;
  static constexpr int NTEAMS_R = THREADS / SR;
  static constexpr int NTEAMS_Z = THREADS / SZ;
  static constexpr int LD = N1 + 1;  // padded plane row
  static constexpr int TBUF_R = team_buf_stride<N1>();
  static constexpr int TBUF_Z = team_buf_stride<M0>();
  static constexpr int XBUF = (NTEAMS_R * TBUF_R > NTEAMS_Z * TBUF_Z) ? NTEAMS_R * TBUF_R : NTEAMS_Z * TBUF_Z;
  // plane + exchange buffers + tables (rows: N1, z: M0, parity twiddle: N1)
  static constexpr int SMEM_F2 = N0 * LD + XBUF + N1 + M0 + N1;
};

// Table layout inside one device buffer (float2 entries):
//   [0, M2)                team table for L = M2
//   [M2, M2+N1)            team table for L = N1
//   [M2+N1, M2+N1+M0)      team table for L = M0
//   [.., +N1)              parity twiddle exp(-2*pi*i*y/M1), y < N1
struct TableOffsets {
  int x, row, z, par, total;
};
__host__ __device__ inline TableOffsets table_offsets(int N0, int N1, int N2) {
  TableOffsets o;
  o.x = 0;
  o.row = 2 * N2;
  o.z = o.row + N1;
  o.par = o.z + 2 * N0;
  o.total = o.par + N1;
  return o;
}

// Problem descriptor shared by the passes.
struct PassArgs {
  int N0, N1, N2;
  int nsys, ncoil;              // slots = nsys * ncoil
  const int* coils;             // [ncoil] coil index into smaps (device)
  const int* diag_of_sys;       // [nsys] diagonal index per system (device)
  const int* active;            // [nsys] nonzero = process this system (device, nullable)
  const float2* x;              // [nsys][N0][N1][N2]
  const float2* smaps;          // [*][N0][N1][N2] (nullable -> S = 1)
  const float2* mul;            // [N0][N1][N2] unconjugated multiplier (nullable)
  float2* spill;                // [nsys*ncoil][M2][N0][N1]
  const float* diag;            // packed diagonals [ndiag][M2][2][N1][M0]
  const float2* tables;         // twiddle tables, see table_offsets
  float2* out;                  // output base
  long long out_sys_stride, out_ldz, out_ldy;  // element strides of out
  int accumulate;               // 1: out += result, 0: out = result
  float lambda;                 // adds lambda * x
  double* dot_partials;         // [nsys][nblocks_c] Re<x, out> partials (nullable)
};

// ------------------------------------------------------------------------ pass A ----
template <int N2, int YT>
__global__ void __launch_bounds__(XPassCfg<N2, YT>::THREADS)
expand_fwd_x_kernel(PassArgs a) {
  using C = XPassCfg<N2, YT>;
  constexpr int M2 = C::M2, E = C::E, S = C::S;
  extern __shared__ float2 smem[];
  float2* tile = smem;                          // [M2][TILE_LD]
  float2* xbuf = tile + M2 * C::TILE_LD;        // teams' exchange buffers
  float2* tw = xbuf + C::NTEAMS * C::TBUF;      // [M2]

  const int slot = blockIdx.z;
  const int sys = slot / a.ncoil;
  if (a.active && !a.active[sys]) return;
  const int coil = a.coils ? a.coils[slot % a.ncoil] : 0;
  const int z = blockIdx.y;
  const int y0 = blockIdx.x * YT;
  const int N0 = a.N0, N1 = a.N1;

  for (int i = threadIdx.x; i < M2; i += C::THREADS) tw[i] = a.tables[i];
  __syncthreads();

  const int team = threadIdx.x / S, t = threadIdx.x % S;
  float2* buf = xbuf + team * C::TBUF;
  const long long plane = (long long)N1 * N2;
  const float2* xs = a.x + (long long)sys * N0 * plane + (long long)z * plane;
  const float2* ss = a.smaps ? a.smaps + (long long)coil * N0 * plane + (long long)z * plane : nullptr;

#pragma unroll 1
  for (int it = 0; it < C::LPT; ++it) {
    const int line = team + it * C::NTEAMS;
    const long long row = (long long)(y0 + line) * N2;
    float2 v[E];
#pragma unroll
    for (int e = 0; e < E / 2; ++e) {
      const int xi = din_index<M2>(t, e);
      float2 val = xs[row + xi];
      if (ss) val = cmul(val, ss[row + xi]);
      v[e] = val;
    }
    team_fft_din_to_dout<M2, -1, true>(v, t, buf, tw);
#pragma unroll
    for (int r = 0; r < E; ++r) tile[dout_index<M2>(t, r) * C::TILE_LD + line] = v[r];
  }
  __syncthreads();

  float2* dst = a.spill + (long long)slot * M2 * N0 * N1 + (long long)z * N1 + y0;
  for (int i = threadIdx.x; i < M2 * YT; i += C::THREADS) {
    const int kx = i / YT, j = i % YT;
    dst[(long long)kx * N0 * N1 + j] = tile[kx * C::TILE_LD + j];
  }
}

// ------------------------------------------------------------------------ pass B ----
template <int N0, int N1>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(PlaneCfg<N0, N1>::THREADS)
plane_yz_kernel(PassArgs a) {
  namespace cg = cooperative_groups;
  using C = PlaneCfg<N0, N1>;
  constexpr int M0 = C::M0, LD = C::LD;
  constexpr int SR = C::SR, ER = C::ER, SZ = C::SZ, EZ = C::EZ;
  extern __shared__ float2 smem[];
  float2* blk = smem;                 // [N0][LD]
  float2* xbuf = blk + N0 * LD;
  float2* tw_r = xbuf + C::XBUF;      // [N1]
  float2* tw_z = tw_r + N1;           // [M0]
  float2* par = tw_z + M0;            // [N1]

  cg::cluster_group cluster = cg::this_cluster();
  const int h = (int)cluster.block_rank();  // ky parity handled by this CTA
  const int slot = blockIdx.y;
  const int kx = blockIdx.z;
  const int sys = slot / a.ncoil;
  if (a.active && !a.active[sys]) return;  // uniform for both CTAs of the cluster
  const int M2 = 2 * a.N2;

  const TableOffsets to = table_offsets(N0, N1, a.N2);
  for (int i = threadIdx.x; i < N1; i += C::THREADS) {
    tw_r[i] = a.tables[to.row + i];
    par[i] = a.tables[to.par + i];
  }
  for (int i = threadIdx.x; i < M0; i += C::THREADS) tw_z[i] = a.tables[to.z + i];
  __syncthreads();

  float2* g = a.spill + ((long long)slot * M2 + kx) * N0 * N1;
  const float* T = a.diag + ((((long long)(a.diag_of_sys ? a.diag_of_sys[sys] : 0) * M2 + kx) * 2 + h) * N1) * M0;

  // stage 1: rows, forward N1-point FFT of the parity-h half
  {
    const int team = threadIdx.x / SR, t = threadIdx.x % SR;
    float2* buf = xbuf + team * C::TBUF_R;
#pragma unroll 1
    for (int z0 = 0; z0 < N0; z0 += C::NTEAMS_R) {
      const int z = z0 + team;
      const bool ok = z < N0;
      float2 v[ER];
#pragma unroll
      for (int e = 0; e < ER; ++e) {
        const int y = din_index<N1>(t, e);
        float2 val = ok ? g[(long long)z * N1 + y] : make_float2(0.f, 0.f);
        if (h) val = cmul(val, par[y]);
        v[e] = val;
      }
      team_fft_din_to_dout<N1, -1, false>(v, t, buf, tw_r);
      if (ok) {
#pragma unroll
        for (int r = 0; r < ER; ++r) blk[z * LD + dout_index<N1>(t, r)] = v[r];
      }
    }
  }
  __syncthreads();

  // stage 2: columns, M0-point FFT along z (upper half zero), x T, inverse, crop
  {
    const int team = threadIdx.x / SZ, t = threadIdx.x % SZ;
    float2* buf = xbuf + team * C::TBUF_Z;
#pragma unroll 1
    for (int c0 = 0; c0 < N1; c0 += C::NTEAMS_Z) {
      const int ky = c0 + team;
      const bool ok = ky < N1;
      const int kyc = ok ? ky : 0;
      float2 v[EZ];
#pragma unroll
      for (int e = 0; e < EZ / 2; ++e) v[e] = ok ? blk[din_index<M0>(t, e) * LD + kyc] : make_float2(0.f, 0.f);
      team_fft_din_to_dout<M0, -1, true>(v, t, buf, tw_z);
      const float* Tc = T + (long long)kyc * M0;
#pragma unroll
      for (int r = 0; r < EZ; ++r) v[r] = cscale(v[r], Tc[dout_index<M0>(t, r)]);
      team_fft_dout_to_din<M0, 1, true>(v, t, buf, tw_z);
      if (ok) {
#pragma unroll
        for (int e = 0; e < EZ / 2; ++e) blk[din_index<M0>(t, e) * LD + ky] = v[e];
      }
    }
  }
  __syncthreads();

  // stage 3: rows, inverse N1-point FFT, post-twiddle
  {
    const int team = threadIdx.x / SR, t = threadIdx.x % SR;
    float2* buf = xbuf + team * C::TBUF_R;
#pragma unroll 1
    for (int z0 = 0; z0 < N0; z0 += C::NTEAMS_R) {
      const int z = z0 + team;
      const bool ok = z < N0;
      const int zc = ok ? z : 0;
      float2 v[ER];
#pragma unroll
      for (int r = 0; r < ER; ++r) v[r] = blk[zc * LD + dout_index<N1>(t, r)];
      team_fft_dout_to_din<N1, 1, false>(v, t, buf, tw_r);
      if (ok) {
#pragma unroll
        for (int e = 0; e < ER; ++e) {
          const int y = din_index<N1>(t, e);
          blk[z * LD + y] = h ? cmulc(v[e], par[y]) : v[e];
        }
      }
    }
  }
  // both halves complete (and all global reads of the plane done) in both CTAs
  cluster.sync();

  // stage 4: sum the two halves, CTA h writes rows [h*N0/2, (h+1)*N0/2)
  {
    const float2* other = cluster.map_shared_rank(blk, h ^ 1);
    constexpr int HALF = N0 / 2;
    for (int i = threadIdx.x; i < HALF * N1; i += C::THREADS) {
      const int z = h * HALF + i / N1, y = i % N1;
      g[(long long)z * N1 + y] = cadd(blk[z * LD + y], other[z * LD + y]);
    }
  }
  // keep this CTA's shared memory alive until the partner has read it
  cluster.sync();
}

// ------------------------------------------------------------------------ pass C ----
template <int N2, int YT>
__global__ void __launch_bounds__(XPassCfg<N2, YT>::THREADS)
inv_x_combine_kernel(PassArgs a) {
  using C = XPassCfg<N2, YT>;
  constexpr int M2 = C::M2, E = C::E, S = C::S, LPT = C::LPT;
  extern __shared__ float2 smem[];
  float2* tile = smem;
  float2* xbuf = tile + M2 * C::TILE_LD;
  float2* tw = xbuf + C::NTEAMS * C::TBUF;
  __shared__ double red[32];

  const int sys = blockIdx.z;
  if (a.active && !a.active[sys]) return;
  const int z = blockIdx.y;
  const int y0 = blockIdx.x * YT;
  const int N0 = a.N0, N1 = a.N1;

  for (int i = threadIdx.x; i < M2; i += C::THREADS) tw[i] = a.tables[i];

  const int team = threadIdx.x / S, t = threadIdx.x % S;
  float2* buf = xbuf + team * C::TBUF;
  const long long plane = (long long)N1 * N2;

  float2 acc[LPT][E / 2];
#pragma unroll
  for (int l = 0; l < LPT; ++l)
#pragma unroll
    for (int e = 0; e < E / 2; ++e) acc[l][e] = make_float2(0.f, 0.f);

#pragma unroll 1
  for (int ci = 0; ci < a.ncoil; ++ci) {
    const int slot = sys * a.ncoil + ci;
    const int coil = a.coils ? a.coils[ci] : 0;
    __syncthreads();  // previous coil's tile fully consumed (and the table loaded)
    const float2* src = a.spill + (long long)slot * M2 * N0 * N1 + (long long)z * N1 + y0;
    for (int i = threadIdx.x; i < M2 * YT; i += C::THREADS) {
      const int kx = i / YT, j = i % YT;
      tile[kx * C::TILE_LD + j] = src[(long long)kx * N0 * N1 + j];
    }
    __syncthreads();
    const float2* ss = a.smaps ? a.smaps + (long long)coil * N0 * plane + (long long)z * plane : nullptr;
#pragma unroll
    for (int l = 0; l < LPT; ++l) {
      const int line = team + l * C::NTEAMS;
      float2 v[E];
#pragma unroll
      for (int r = 0; r < E; ++r) v[r] = tile[dout_index<M2>(t, r) * C::TILE_LD + line];
      team_fft_dout_to_din<M2, 1, true>(v, t, buf, tw);
      const long long row = (long long)(y0 + line) * N2;
#pragma unroll
      for (int e = 0; e < E / 2; ++e) {
        const int xi = din_index<M2>(t, e);
        float2 val = v[e];
        if (ss) val = cmulc(val, ss[row + xi]);
        else if (a.mul) val = cmul(val, a.mul[(long long)z * plane + row + xi]);
        acc[l][e] = cadd(acc[l][e], val);
      }
    }
  }

  // epilogue
  double dot = 0.0;
  const float2* xs = a.x + (long long)sys * N0 * plane + (long long)z * plane;
#pragma unroll
  for (int l = 0; l < LPT; ++l) {
    const int y = y0 + team + l * C::NTEAMS;
#pragma unroll
    for (int e = 0; e < E / 2; ++e) {
      const int xi = din_index<M2>(t, e);
      float2 val = acc[l][e];
      const float2 xv = xs[(long long)y * N2 + xi];
      if (a.lambda != 0.f) val = make_float2(fmaf(a.lambda, xv.x, val.x), fmaf(a.lambda, xv.y, val.y));
      float2* o = a.out + sys * a.out_sys_stride + z * a.out_ldz + y * a.out_ldy + xi;
      if (a.accumulate) val = cadd(*o, val);
      *o = val;
      dot += (double)xv.x * (double)val.x + (double)xv.y * (double)val.y;
    }
  }
  if (a.dot_partials) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) dot += __shfl_down_sync(0xffffffffu, dot, off);
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (lane == 0) red[warp] = dot;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < C::THREADS / 32; ++w) s += red[w];
      const int nblk = gridDim.x * gridDim.y;
      a.dot_partials[(long long)sys * nblk + blockIdx.y * gridDim.x + blockIdx.x] = s;
    }
  }
}

}  // namespace hb
