// The three fused passes of the Toeplitz-embedded SENSE normal operator.
//
//   out = sum_c conj(S_c) * crop( IFFT_M( T * FFT_M( pad( S_c * x ) ) ) )     (M = 2N)
//
// Pass A  expand_fwd_x : per (slot, z, y-tile): S_c * x, zero-pad along x, M2-point FFT,
//                        written transposed to the spill  spill[slot][z][kx][y].
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

#include "bulk.cuh"
#include "common.cuh"
#include "fft.cuh"

namespace hb {

// ------------------------------------------------------------------- spill layout ----
// The spill holds, per (system, coil) slot, the image after the forward x transform:
// [slot][z][yt][kx][yy'] with yt = y / YT, yy' = pos(y % YT) ^ (kx % YT), YT = spill_yt(N1),
// pos(u) = 2 * (u % (YT/2)) + u / (YT/2).
// * The (slot, z, yt) tile that passes A and C move is one contiguous M2 x YT block, so it
//   travels as one bulk copy and lies in shared memory exactly as in global memory.
// * The XOR puts the YT values of one kx row in an order that depends on kx, so a tile
//   column (one y, consecutive kx: what one FFT team writes or reads) falls on distinct
//   shared-memory banks without padding.
// * pos interleaves the two halves of a kx row: y and y + YT/2 sit side by side (in either
//   order after the XOR) in one aligned 16-byte pair, which is what a lane of an
//   (YT/2)-lane FFT team of pass B needs for two of its registers.
// * Row z of the (slot, kx) plane that pass B transforms is N1 / YT chunks of YT values
//   (128 bytes for YT = 16), M2 * YT apart, rows M2 * N1 apart.
__host__ __device__ constexpr int spill_yt(int N1) { return N1 < 16 ? N1 : 16; }
__host__ __device__ inline long long spill_tile_offset(int slot, int z, int yt, int N0, int N1, int M2) {
  const int YT = spill_yt(N1);
  return (((long long)slot * N0 + z) * (N1 / YT) + yt) * (long long)(M2 * YT);
}
__host__ __device__ constexpr int spill_pos(int yy, int YT) {
  return YT < 2 ? yy : 2 * (yy % (YT / 2)) + yy / (YT / 2);
}
__host__ __device__ constexpr int spill_in_tile(int kx, int yy, int YT) {
  return kx * YT + (spill_pos(yy, YT) ^ (kx & (YT - 1)));
}
__host__ __device__ inline long long spill_index(int slot, int z, int kx, int y, int N0, int N1, int M2) {
  const int YT = spill_yt(N1);
  return spill_tile_offset(slot, z, y / YT, N0, N1, M2) + spill_in_tile(kx, y % YT, YT);
}

// Rows of one (slot, kx) plane of the spill, for pass B (N1 a compile-time constant).
template <int N1>
struct SpillPlane {
  static constexpr int YT = spill_yt(N1);
  float2* base;    // element (z, y) at base + z * rs + (y / YT) * cs + ((y % YT) ^ sw)
  long long rs;    // z pitch: M2 * N1
  long long cs;    // y-chunk pitch: M2 * YT
  int sw;          // kx % YT
  __device__ __forceinline__ SpillPlane(float2* spill, int slot, int kx, int N0, int M2) {
    base = spill + spill_tile_offset(slot, 0, 0, N0, N1, M2) + (long long)kx * YT;
    rs = (long long)M2 * N1;
    cs = (long long)M2 * YT;
    sw = kx & (YT - 1);
  }
  // Offsets within one plane fit in 32 bits: N0 * M2 * N1 <= 160 * 320 * 160 elements for
  // every supported size (32-bit index arithmetic is the cheaper form).
  __device__ __forceinline__ int off(int z, int y) const {
    return z * (int)rs + (y / YT) * (int)cs + (spill_pos(y % YT, YT) ^ sw);
  }
  __device__ __forceinline__ float2& at(int z, int y) const { return base[off(z, y)]; }
  // lo = at(z, y), hi = at(z, y + YT/2) for y % YT < YT/2, as one 16-byte load (YT >= 4;
  // base is 16-byte aligned: kx * YT elements past a tile start)
  __device__ __forceinline__ void pair(int z, int y, float2& lo, float2& hi) const {
    const float4 w = *reinterpret_cast<const float4*>(
        base + (z * (int)rs + (y / YT) * (int)cs + ((2 * (y % (YT / 2))) ^ (sw & ~1))));
    const bool swap = sw & 1;  // the XOR's low bit exchanges the two
    lo = swap ? make_float2(w.z, w.w) : make_float2(w.x, w.y);
    hi = swap ? make_float2(w.x, w.y) : make_float2(w.z, w.w);
  }
};

// ---------------------------------------------------------------- launch geometry ----
// Pass A / C: a CTA covers YT consecutive y lines (one spill y-tile) of one z plane of one
// system and loops over the system's coils; every team of S lanes transforms LPT lines.
template <int N2, int YT>
struct XPassCfg {
  static constexpr int M2 = 2 * N2;
  static constexpr int E = TeamCfg<M2>::E;
  static constexpr int S = TeamCfg<M2>::S;
  static constexpr int LPT = (YT * S > 256) ? (YT * S / 256) : 1;
  static constexpr int THREADS = YT * S / LPT;
  static constexpr int NTEAMS = THREADS / S;
  static constexpr int TBUF = team_buf_stride<M2>();
  static constexpr int TILE_ELEMS = M2 * YT;           // one spill tile, dense (swizzled)
  static constexpr unsigned TILE_BYTES = TILE_ELEMS * 8u;
  // pass A: the tile; the same space serves as the teams' FFT exchange buffers
  static constexpr int TILE = (TILE_ELEMS > NTEAMS * TBUF) ? TILE_ELEMS : NTEAMS * TBUF;
  static constexpr int SMT = YT * N2;     // one coil's map rows [y][x]
  // float2 slots of dynamic shared memory: pass A = one tile (also the exchange buffers)
  // + two coil-map stages; pass C = two tiles + the exchange buffers; each + the M2-entry
  // twiddle table
  static constexpr int SMEM_F2 = TILE + 2 * SMT + M2;
  // pass C: a team of S = 16 lanes with one line (LPT = 1) exchanges inside its share of
  // the tile it has just read (no separate exchange buffers)
  static constexpr bool C_IN_TILE = S == 16 && LPT == 1 && NTEAMS * M2 == TILE_ELEMS;
  static constexpr int SMEM_F2_C = 2 * TILE_ELEMS + (C_IN_TILE ? 0 : NTEAMS * TBUF) + M2;
  static_assert(THREADS % 32 == 0, "x-pass CTA must be whole warps");
  static_assert((YT & (YT - 1)) == 0, "the tile swizzle needs a power-of-two tile height");
  static_assert(TILE_BYTES % 16 == 0 && (SMT * 8) % 16 == 0, "bulk copies move whole 16-byte units");
};

// Row handled by team j of a row stage: the teams sharing a half-warp take rows S apart,
// so their (odd-pitch) plane rows start on disjoint shared-memory banks.
template <int S, int NTEAMS, int ROWS>
__device__ __forceinline__ int row_of_team(int j) {
  constexpr int TPH = S < 16 ? 16 / S : 1;
  if constexpr (TPH > 1 && NTEAMS % 16 == 0 && ROWS % 16 == 0) {
    return (j / 16) * 16 + (j % TPH) * S + (j / TPH) % S;
  } else {
    return j;
  }
}

// Pass B: a cluster of 2*Q CTAs owns one N0 x N1 (z, y) plane.  CTA rank r = h*Q + q
// handles ky parity h; for the z-FFTs it owns the ky' columns [q*H, (q+1)*H) (H = N1/Q),
// for the y-FFTs the rows [q*ZR, (q+1)*ZR) (ZR = N0/Q).  Rows and columns meet through
// distributed shared memory.
template <int N0, int N1, int Q, int THREADS_>
struct PlaneCfg {
  static constexpr int M0 = 2 * N0;
  static constexpr int THREADS = THREADS_;
  static constexpr int SR = TeamCfg<N1>::S, ER = TeamCfg<N1>::E;
  static constexpr int SZ = TeamCfg<M0>::S, EZ = TeamCfg<M0>::E;
  static constexpr int H = N1 / Q;    // owned columns (z stage)
  static constexpr int ZR = N0 / Q;   // owned rows (y stages)
  static constexpr int NTEAMS_R = THREADS / SR;
  static constexpr int NTEAMS_Z = THREADS / SZ;
  static constexpr int LPT_R = (ZR + NTEAMS_R - 1) / NTEAMS_R;  // rows per team
  static constexpr int LDP = H + 1;   // column-stage row pitch
  // Row z of the column stage sits at buffer row pos(z) = Q*(z % ZR) + z / ZR, so the Q
  // rows that every CTA of the cluster consumes in one round of the inverse row stage
  // are adjacent; output row zl then overwrites exactly those Q*LDP >= N1 + 1 slots.
  static constexpr int PBUF = N0 * LDP;
  static constexpr int GROW = Q * LDP;  // output-row pitch
  static constexpr int TBUF_R = team_buf_stride<N1>();
  static constexpr int TBUF_Z = team_buf_stride<M0>();
  static constexpr int XBUF = (NTEAMS_R * TBUF_R > NTEAMS_Z * TBUF_Z) ? NTEAMS_R * TBUF_R : NTEAMS_Z * TBUF_Z;
  // plane + exchange buffers + tables (rows: N1, z: M0, parity twiddle: N1)
  static constexpr int SMEM_F2 = PBUF + XBUF + N1 + M0 + N1;
  static_assert(N1 % Q == 0 && N0 % (2 * Q) == 0, "plane split must divide the plane");
  static_assert(GROW >= N1, "an output row must fit in the rows it replaces");
  static_assert(THREADS % 32 == 0 && THREADS % SR == 0 && THREADS % SZ == 0, "teams must tile the CTA");
};

// Table layout inside one device buffer (float2 entries):
//   [0, M2)                team table for L = M2
//   [M2, M2+N1)            team table for L = N1
//   [M2+N1, M2+N1+M0)      team table for L = M0
//   [.., +N1)              parity twiddle exp(-2*pi*i*y/M1), y < N1
//   [.., +N1/2)            team table for L = N1/2 (power-of-two N1 only)
//   [.., +N1/4)            team table for L = N1/4 (power-of-two N1 only)
//   [.., +2*N1)            full circle exp(-2*pi*i*k/M1), k < M1
struct TableOffsets {
  int x, row, z, par, row2, row4, circ, total;
};
__host__ __device__ inline TableOffsets table_offsets(int N0, int N1, int N2) {
  TableOffsets o;
  o.x = 0;
  o.row = 2 * N2;
  o.z = o.row + N1;
  o.par = o.z + 2 * N0;
  o.row2 = o.par + N1;
  o.row4 = o.row2 + N1 / 2;
  o.circ = o.row4 + N1 / 4;
  o.total = o.circ + 2 * N1;
  return o;
}

// Problem descriptor shared by the passes.  Systems are described by per-system tables
// so that one launch sequence can carry systems of different jobs (own buffers, coil
// maps, coil counts, diagonals, lambda).  A slot is one (system, coil) pair; the slots
// of a system are consecutive.
struct PassArgs {
  int N0, N1, N2;
  int nsys, nslots;
  const int* slot_sys;             // [nslots] system of the slot
  const int* slot_coil;            // [nslots] coil index into that system's coil maps
  const int* sys_slot0;            // [nsys] first slot of the system
  const int* sys_nslot;            // [nsys] number of coils of the system
  const int* active;               // [nsys] nonzero = process this system (nullable)
  const float2* const* sys_x;      // [nsys] input image [N0][N1][N2]
  float2* const* sys_out;          // [nsys] output image (strides out_ldz, out_ldy, 1)
  const float2* const* sys_smaps;  // [nsys] coil maps [*][N0][N1][N2]; a null entry = unit map
  const float* const* sys_diag;    // [nsys] packed diagonal [M2][2][N1][M0]
  const float* sys_lambda;         // [nsys] adds lambda * x (nullable = 0)
  const float2* mul;               // [N0][N1][N2] unconjugated multiplier (single system, nullable)
  float2* spill;                   // [nslots][N0][N1/YT][M2][YT], see spill_index
  int* wait_error;                 // set to 1 when a pass gave up waiting for a bulk copy
  const float2* tables;            // twiddle tables, see table_offsets
  long long out_ldz, out_ldy;      // element strides of every output image
  int accumulate;                  // 1: out += result, 0: out = result
  double* dot_partials;            // [nsys][nblocks_c] Re<x, out> partials (nullable)
  int prefetch_ahead;              // mod-4 plane pass: L2-prefetch distance in clusters (0 = off)
  int inject_stall;                // tests only: pass C omits the tile copy of coil index
                                   // inject_stall - 1 of every system (0 = off)
};


// ------------------------------------------------------------------------ pass A ----
// Per (system, z, y-tile): the x lines stay in registers while the coils stream by; coil
// c + 1's map rows are copied asynchronously while coil c is transformed and stored.
template <int N2, int YT>
__global__ void __launch_bounds__(XPassCfg<N2, YT>::THREADS)
expand_fwd_x_kernel(PassArgs a) {
  using C = XPassCfg<N2, YT>;
  constexpr int M2 = C::M2, E = C::E, S = C::S, LPT = C::LPT;
  extern __shared__ __align__(128) float2 smem[];
  float2* tile = smem;                // spill tile [M2][YT] (swizzled) / exchange buffers
  float2* smt = tile + C::TILE;       // 2 x [YT][N2] coil-map stages
  float2* tw = smt + 2 * C::SMT;      // [M2]

  const int sys = blockIdx.z;
  if (a.active && !a.active[sys]) return;
  const int z = blockIdx.y;
  const int y0 = blockIdx.x * YT;
  const int N0 = a.N0, N1 = a.N1;

  for (int i = threadIdx.x; i < M2; i += C::THREADS) tw[i] = a.tables[i];

  const int team = threadIdx.x / S, t = threadIdx.x % S;
  float2* buf = tile + team * C::TBUF;
  const long long plane = (long long)N1 * N2;
  const float2* sm = a.sys_smaps[sys];
  const int slot0 = a.sys_slot0[sys], ncoil = a.sys_nslot[sys];
  // Coil ci's map rows [y0, y0 + YT) of plane z are one contiguous block: one bulk copy
  // into smt[ci & 1], landing on bar[ci & 1] (phase ci >> 1), when the maps are 16-byte
  // aligned; per-thread 8-byte asynchronous copies otherwise.
  __shared__ __align__(8) uint64_t bar[3];  // [0], [1]: map stages; [2]: the image rows
  __shared__ int abort_sh;
  const bool bulk_maps = sm && (((uintptr_t)sm) & 15u) == 0;
  const float2* xs = a.sys_x[sys] + (long long)z * plane + (long long)y0 * N2;  // rows [y0, y0 + YT)
  const bool bulk_x = (((uintptr_t)xs) & 15u) == 0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < 3; ++i) mbar_init(smem_u32(&bar[i]), 1);
    fence_mbar_init();
    abort_sh = 0;
  }
  __syncthreads();
  // the image rows of this tile, once: one bulk copy into the second map stage, which the
  // first map copy into it (coil 1) waits for below
  if (bulk_x && threadIdx.x == 0) {
    mbar_expect_tx(smem_u32(&bar[2]), C::SMT * 8u);
    bulk_copy_g2s(smem_u32(smt + C::SMT), xs, C::SMT * 8u, smem_u32(&bar[2]));
  }
  int issued = 0, landed = 0;  // map copies issued (thread 0) / waited for
  auto prefetch = [&](int ci) {
    const float2* src = sm + ((long long)a.slot_coil[slot0 + ci] * N0 + z) * plane + (long long)y0 * N2;
    float2* dst = smt + (ci & 1) * C::SMT;
    if (bulk_maps) {
      if (threadIdx.x == 0) {
        const uint32_t b = smem_u32(&bar[ci & 1]);
        mbar_expect_tx(b, C::SMT * 8u);
        bulk_copy_g2s(smem_u32(dst), src, C::SMT * 8u, b);
        issued = ci + 1;
      }
    } else {
      for (int i = threadIdx.x; i < C::SMT; i += C::THREADS) cp_async8(dst + i, src + i);
      cp_async_commit();
    }
  };
  if (sm && ncoil > 0) prefetch(0);

  // the x lines stay in registers while the coils stream by
  float2 xv[LPT][E / 2];
  bool x_ok = true;
  if (bulk_x) x_ok = mbar_wait(smem_u32(&bar[2]), 0, &abort_sh);
  {
    const float2* xsrc = bulk_x ? smt + C::SMT : xs;
#pragma unroll
    for (int l = 0; l < LPT; ++l)
#pragma unroll
      for (int e = 0; e < E / 2; ++e) xv[l][e] = xsrc[(team + l * C::NTEAMS) * N2 + din_index<M2>(t, e)];
  }
  if (!x_ok) abort_sh = 1;
  __syncthreads();  // every thread has its x lines: the second map stage may be refilled
  if (abort_sh && bulk_x && threadIdx.x == 0) {
    const long long t0 = clock64();  // drain the image copy (bounded) before anything else
    while (!mbar_try_wait(smem_u32(&bar[2]), 0) && clock64() - t0 < kWaitCycles) {
    }
  }

#pragma unroll 1
  for (int ci = 0; ci < ncoil; ++ci) {
    if (sm) {
      if (ci + 1 < ncoil) prefetch(ci + 1);
      if (bulk_maps) {
        if (!mbar_wait(smem_u32(&bar[ci & 1]), (ci >> 1) & 1, &abort_sh)) abort_sh = 1;
      } else if (ci + 1 < ncoil) {
        cp_async_wait<1>();  // coil ci's rows have landed
      } else {
        cp_async_wait<0>();
      }
    }
    // the previous coil's tile has been read out by its bulk store: the space may take
    // this coil's exchanges
    if (threadIdx.x == 0 && ci > 0) bulk_wait_read0();
    __syncthreads();  // coil ci's rows are visible; the tile space is free
    if (abort_sh) break;  // read after the barrier: the same decision in every thread
    landed = ci + 1;
    const float2* mt = smt + (ci & 1) * C::SMT;
    float2 v[LPT][E];
#pragma unroll
    for (int l = 0; l < LPT; ++l) {
      const int line = team + l * C::NTEAMS;
#pragma unroll
      for (int e = 0; e < E / 2; ++e)
        v[l][e] = sm ? cmul(xv[l][e], mt[line * N2 + din_index<M2>(t, e)]) : xv[l][e];
      team_fft_din_to_dout<M2, -1, true>(v[l], t, buf, tw);
    }
    __syncthreads();  // every exchange is done: the space becomes the output tile
#pragma unroll
    for (int l = 0; l < LPT; ++l) {
      const int line = team + l * C::NTEAMS;
#pragma unroll
      for (int r = 0; r < E; ++r) tile[spill_in_tile(dout_index<M2>(t, r), line, YT)] = v[l][r];
    }
    fence_proxy_async_smem();  // the tile's writes become visible to the bulk copy
    __syncthreads();
    if (threadIdx.x == 0) {
      bulk_copy_s2g(a.spill + spill_tile_offset(slot0 + ci, z, blockIdx.x, N0, N1, M2), smem_u32(tile),
                    C::TILE_BYTES);
      bulk_commit();
    }
  }
  if (threadIdx.x == 0) {
    bulk_wait0();  // the tiles are in global memory before the CTA ends
    if (abort_sh) {
      // a map copy did not land in time: wait (bounded, one by one) for the copies still
      // in flight so none writes into shared memory after the CTA ends, and report
      for (int j = landed; j < issued; ++j) {
        const long long t0 = clock64();
        while (!mbar_try_wait(smem_u32(&bar[j & 1]), (j >> 1) & 1) && clock64() - t0 < kWaitCycles) {
        }
      }
      if (a.wait_error) atomicExch(a.wait_error, 1);
    }
  }
}

// Lane t's EZ diagonal values of one z column (team of SZ lanes): the packed column holds
// registers 4j..4j+3 of lane t at (j*SZ + t)*4 (diag_pack_kernel), so the team's j-th
// 16-byte loads cover SZ*16 contiguous bytes.
template <int EZ, int SZ>
__device__ __forceinline__ void load_tcol(float* dst, const float* col, int t) {
  static_assert(EZ % 4 == 0, "whole 16-byte vectors");
  const float4* src = reinterpret_cast<const float4*>(col) + t;
#pragma unroll
  for (int j = 0; j < EZ / 4; ++j) {
    const float4 v = __ldg(src + j * SZ);
    dst[4 * j] = v.x;
    dst[4 * j + 1] = v.y;
    dst[4 * j + 2] = v.z;
    dst[4 * j + 3] = v.w;
  }
}

// L2 prefetch (a hint) of rows [r0, r0 + nrows) of a spill plane: each row is N1 / YT
// chunks of YT values (YT * 8 bytes, at least 64), one prefetch per chunk, spread over the
// CTA's threads
template <int THREADS, int N1>
__device__ __forceinline__ void prefetch_plane_rows_l2(const SpillPlane<N1>& pl, int r0, int nrows) {
  constexpr int YT = SpillPlane<N1>::YT, CH = N1 / YT;
  for (int i = threadIdx.x; i < nrows * CH; i += THREADS) {
    const float2* p = pl.base + (r0 + i / CH) * pl.rs + (long long)(i % CH) * pl.cs;
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
  }
}

// ------------------------------------------------------------------------ pass B ----
template <int N0, int N1, int Q, int THREADS_>
__global__ void __cluster_dims__(2 * Q, 1, 1) __launch_bounds__(THREADS_)
plane_yz_kernel(PassArgs a) {
  namespace cg = cooperative_groups;
  using C = PlaneCfg<N0, N1, Q, THREADS_>;
  constexpr int M0 = C::M0, H = C::H, ZR = C::ZR, LDP = C::LDP, GROW = C::GROW;
  auto pos = [](int z) { return Q * (z % ZR) + z / ZR; };
  constexpr int SR = C::SR, ER = C::ER, SZ = C::SZ, EZ = C::EZ, LPT = C::LPT_R;
  extern __shared__ float2 smem[];
  float2* P = smem;                   // [N0][LDP] columns, later [ZR][LDG] output rows
  float2* xbuf = P + C::PBUF;
  float2* tw_r = xbuf + C::XBUF;      // [N1]
  float2* tw_z = tw_r + N1;           // [M0]
  float2* par = tw_z + M0;            // [N1]

  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int h = rank / Q;  // ky parity
  const int q = rank % Q;  // owned column / row block
  const int M2 = 2 * a.N2;

  const TableOffsets to = table_offsets(N0, N1, a.N2);
  for (int i = threadIdx.x; i < N1; i += C::THREADS) {
    tw_r[i] = a.tables[to.row + i];
    par[i] = a.tables[to.par + i];
  }
  for (int i = threadIdx.x; i < M0; i += C::THREADS) tw_z[i] = a.tables[to.z + i];
  __syncthreads();

  float2* Pr[Q];  // column blocks of this parity, one per cluster rank h*Q + q'
#pragma unroll
  for (int qq = 0; qq < Q; ++qq) Pr[qq] = cluster.map_shared_rank(P, h * Q + qq);

  // Persistent: cluster c of gridDim.y takes work items c, c + gridDim.y, ...; item i is
  // (slot = i % nslots, kx = i / nslots), so co-resident clusters share kx (and the
  // diagonal's kx plane in L2).
  const long long nitems = (long long)a.nslots * M2;
  const int ncl = gridDim.y;
#pragma unroll 1
  for (long long item = blockIdx.y; item < nitems; item += ncl) {
    const int slot = (int)(item % a.nslots);
    const int kx = (int)(item / a.nslots);
    const int sys = a.slot_sys[slot];
    if (a.active && !a.active[sys]) continue;  // uniform for the whole cluster
    const SpillPlane<N1> g(a.spill, slot, kx, N0, M2);  // element (z, y) at g.at(z, y)
    const float* T = a.sys_diag[sys] + (((long long)kx * 2 + h) * N1) * M0;

    // Q == 1: the plane lands in the (row-major, padded) column buffer in row groups of
    // NTEAMS_R rows (one asynchronous copy group each); the row FFTs of the first group
    // start while the later groups are still arriving.
    constexpr int RG = C::NTEAMS_R;
    constexpr int NGRP = (ZR + RG - 1) / RG;
    if constexpr (Q == 1) {
#pragma unroll 1
      for (int grp = 0; grp < NGRP; ++grp) {
        const int r0 = grp * RG, nr = (N0 - r0) < RG ? (N0 - r0) : RG;
        for (int i = threadIdx.x; i < nr * N1; i += C::THREADS)
          cp_async8(&P[(r0 + i / N1) * LDP + (i % N1)], &g.at(r0 + i / N1, i % N1));
        cp_async_commit();
      }
    }
    // warm L2 with this cluster's next plane (a hint only)
    if (item + ncl < nitems) {
      const long long nx = item + ncl;
      const SpillPlane<N1> nxt(a.spill, (int)(nx % a.nslots), (int)(nx / a.nslots), N0, M2);
      prefetch_plane_rows_l2<C::THREADS>(nxt, rank * (N0 / (2 * Q)), N0 / (2 * Q));
    }
    // stage 1: owned rows, forward N1-point FFT of the parity-h half; each output column
    // goes to the CTA that owns it
    {
      const int team = threadIdx.x / SR, t = threadIdx.x % SR;
      const int tr = row_of_team<SR, C::NTEAMS_R, ZR>(team);
      float2* buf = xbuf + team * C::TBUF_R;
  #pragma unroll 1
      for (int it = 0; it < LPT; ++it) {
        if constexpr (Q == 1) {
          cp_async_wait_dyn(NGRP - 1 - it);  // group `it` (rows it*RG ...) has landed
          __syncthreads();
        }
        const int zl = tr + it * C::NTEAMS_R;
        const int z = q * ZR + (zl < ZR ? zl : 0);
        float2 v[ER];
  #pragma unroll
        for (int e = 0; e < ER; ++e) {
          const int y = din_index<N1>(t, e);
          float2 val = Q == 1 ? P[z * LDP + y] : g.at(z, y);
          if (h) val = cmul(val, par[y]);
          v[e] = val;
        }
        team_fft_din_to_dout<N1, -1, false>(v, t, buf, tw_r);
        if (zl < ZR) {
  #pragma unroll
          for (int r = 0; r < ER; ++r) {
            const int ky = dout_index<N1>(t, r);
            Pr[ky / H][pos(z) * LDP + ky % H] = v[r];
          }
        }
      }
    }
    cluster.sync();

    // stage 2: owned columns, M0-point FFT along z (upper half zero), x T, inverse, crop
    {
      const int team = threadIdx.x / SZ, t = threadIdx.x % SZ;
      float2* buf = xbuf + team * C::TBUF_Z;
      // this lane's z twiddles, reused by every column (registers when they are few)
      constexpr bool kRegTw = EZ <= 16;
      float2 twz[kRegTw ? EZ : 1];
      if constexpr (kRegTw) load_lane_twiddles<M0>(twz, tw_z, t);
      // the diagonal's columns are fetched one iteration ahead of their use
      float tnext[EZ];
      {
        const int col = team < H ? team : 0;
        load_tcol<EZ, SZ>(tnext, T + (long long)(q * H + col) * M0, t);
      }
  #pragma unroll 1
      for (int c0 = 0; c0 < H; c0 += C::NTEAMS_Z) {
        const int col = c0 + team;
        const bool ok = col < H;
        const int colc = ok ? col : 0;
        float tv[EZ];
  #pragma unroll
        for (int r = 0; r < EZ; ++r) tv[r] = tnext[r];
        if (c0 + C::NTEAMS_Z < H) {
          const int cn = c0 + C::NTEAMS_Z + team;
          load_tcol<EZ, SZ>(tnext, T + (long long)(q * H + (cn < H ? cn : 0)) * M0, t);
        }
        float2 v[EZ];
  #pragma unroll
        for (int e = 0; e < EZ / 2; ++e) v[e] = P[pos(din_index<M0>(t, e)) * LDP + colc];
        if constexpr (kRegTw) team_fft_din_to_dout_r<M0, -1, true>(v, t, buf, twz);
        else team_fft_din_to_dout<M0, -1, true>(v, t, buf, tw_z);
  #pragma unroll
        for (int r = 0; r < EZ; ++r) v[r] = cscale(v[r], tv[r]);
        if constexpr (kRegTw) team_fft_dout_to_din_r<M0, 1, true>(v, t, buf, twz);
        else team_fft_dout_to_din<M0, 1, true>(v, t, buf, tw_z);
        if (ok) {
  #pragma unroll
          for (int e = 0; e < EZ / 2; ++e) P[pos(din_index<M0>(t, e)) * LDP + col] = v[e];
        }
      }
    }
    cluster.sync();

    // stage 3: owned rows gathered from the column owners, inverse N1-point FFT along y,
    // post-twiddle.  Output row zl replaces the Q buffer rows consumed in the same round.
    {
      const int team = threadIdx.x / SR, t = threadIdx.x % SR;
      const int tr = row_of_team<SR, C::NTEAMS_R, ZR>(team);
      float2* buf = xbuf + team * C::TBUF_R;
  #pragma unroll 1
      for (int it = 0; it < LPT; ++it) {
        const int zl = tr + it * C::NTEAMS_R;
        const int z = q * ZR + (zl < ZR ? zl : 0);
        float2 v[ER];
  #pragma unroll
        for (int r = 0; r < ER; ++r) {
          const int ky = dout_index<N1>(t, r);
          v[r] = Pr[ky / H][pos(z) * LDP + ky % H];
        }
        if constexpr (Q > 1) cluster.sync();  // every CTA has read this round's rows
        team_fft_dout_to_din<N1, 1, false>(v, t, buf, tw_r);
        if (zl < ZR) {
  #pragma unroll
          for (int e = 0; e < ER; ++e) {
            const int y = din_index<N1>(t, e);
            P[zl * GROW + y] = h ? cmulc(v[e], par[y]) : v[e];
          }
        }
      }
    }
    cluster.sync();

    // stage 4: sum the two parities; CTA (h, q) writes the h-th half of rows block q
    {
      const float2* other = cluster.map_shared_rank(P, (1 - h) * Q + q);
      constexpr int HALF = ZR / 2;
      for (int i = threadIdx.x; i < HALF * N1; i += C::THREADS) {
        const int zl = h * HALF + i / N1, y = i % N1;
        g.at(q * ZR + zl, y) = cadd(P[zl * GROW + y], other[zl * GROW + y]);
      }
    }

    // the partners have read this CTA's buffer before the next item overwrites it
    cluster.sync();
  }
}

// ---------------------------------------------------------------- pass B (mod K) ----
// Plane pass split K ways (K = 4 or 8): a cluster of K CTAs owns one (z, y) plane and
// CTA q takes the 2x y-grid frequencies ky = K*k + q (k < L = 2*N1/K).  With
// y = y' + L*m (m < K/2) the row transform is
//   X_q[k] = FFT_L( w_M1^(y'*q) * sum_m a[y' + L*m] * e^(-2*pi*i*m*q/K) )[k],
// the z stage runs on the CTA's L columns, and the inverse rows give R_q = IFFT_L.  The
// only cross-CTA step is the final sum (distributed shared memory): with
// u_q = w_M1^(-y'*q) R_q[y'],  out[y' + L*m] = sum_q e^(+2*pi*i*m*q/K) u_q  (m < K/2),
// a K-point inverse DFT of which half the outputs are kept.  A CTA holds only
// N0 x L of the plane, so several CTAs share an SM and one CTA's memory phases
// overlap another's arithmetic.
template <int N0, int N1, int K, int THREADS_>
struct PlaneModCfg {
  static constexpr int M0 = 2 * N0, M1 = 2 * N1, L = M1 / K;
  static constexpr int THREADS = THREADS_;
  static constexpr int SR = TeamCfg<L>::S, ER = TeamCfg<L>::E;
  static constexpr int SZ = TeamCfg<M0>::S, EZ = TeamCfg<M0>::E;
  static constexpr int NTEAMS_R = THREADS / SR, NTEAMS_Z = THREADS / SZ;
  static constexpr int LPT = (N0 + NTEAMS_R - 1) / NTEAMS_R;
  static constexpr int LDP = L + 1;
  static constexpr int PBUF = N0 * LDP;
  static constexpr int TBUF_R = team_buf_stride<L>(), TBUF_Z = team_buf_stride<M0>();
  static constexpr int XBUF = (NTEAMS_R * TBUF_R > NTEAMS_Z * TBUF_Z) ? NTEAMS_R * TBUF_R : NTEAMS_Z * TBUF_Z;
  static constexpr int SMEM_F2 = PBUF + XBUF + L + M0 + M1;  // + tables: row (L), z (M0), circle (M1)
  static_assert((K == 4 || K == 8) && N0 % K == 0 && L >= 8, "K-way plane split");
  static_assert(THREADS % SR == 0 && THREADS % SZ == 0, "teams must tile the CTA");
};

template <int V>
struct IntC {
  static constexpr int value = V;
};
// f(IntC<r>{}) for the run-time r in [0, K): one instantiation of f per value
template <int K, int I = 0, class F>
__device__ __forceinline__ void with_rank(int r, F&& f) {
  if constexpr (I < K) {
    if (r == I) f(IntC<I>{});
    else with_rank<K, I + 1>(r, f);
  }
}

// v * exp(DIR * 2*pi*i * p / K) for a runtime p (K = 4 or 8): rotations and one
// multiply by sqrt(1/2) at most
template <int K, int DIR>
HB_DEV float2 rootK(float2 v, int p) {
  p &= K - 1;
  if constexpr (K == 8) {
    if (p & 1) {
      const float2 r = make_float2(kC8 * (v.x - DIR * v.y), kC8 * (v.y + DIR * v.x));  // v * e^(DIR i pi/4)
      v = r;
    }
    p >>= 1;
  }
  switch (p & 3) {
    case 1: return rot90<DIR>(v);
    case 2: return make_float2(-v.x, -v.y);
    case 3: return rot90<-DIR>(v);
    default: return v;
  }
}

template <int N0, int N1, int K, int THREADS_>
__global__ void __cluster_dims__(K, 1, 1) __launch_bounds__(THREADS_)
plane_mod_kernel(PassArgs a) {
  namespace cg = cooperative_groups;
  using C = PlaneModCfg<N0, N1, K, THREADS_>;
  constexpr int M0 = C::M0, M1 = C::M1, L = C::L, LDP = C::LDP;
  constexpr int SR = C::SR, ER = C::ER, SZ = C::SZ, EZ = C::EZ;
  constexpr int NM = K / 2;  // fold terms per output
  extern __shared__ float2 smem[];
  float2* P = smem;                 // [N0][LDP]: this CTA's share of the plane
  float2* xbuf = P + C::PBUF;
  float2* tw_r = xbuf + C::XBUF;    // [L]
  float2* tw_z = tw_r + L;          // [M0]
  float2* circ = tw_z + M0;         // [M1] exp(-2*pi*i*k/M1)

  cg::cluster_group cluster = cg::this_cluster();
  const int q = (int)cluster.block_rank();  // ky mod K
  const int slot = blockIdx.y;
  const int kx = blockIdx.z;
  const int sys = a.slot_sys[slot];
  if (a.active && !a.active[sys]) return;  // uniform for the whole cluster
  const int M2 = 2 * a.N2;

  const TableOffsets to = table_offsets(N0, N1, a.N2);
  const int trow = K == 4 ? to.row2 : to.row4;
  for (int i = threadIdx.x; i < L; i += C::THREADS) tw_r[i] = a.tables[trow + i];
  for (int i = threadIdx.x; i < M0; i += C::THREADS) tw_z[i] = a.tables[to.z + i];
  for (int i = threadIdx.x; i < M1; i += C::THREADS) circ[i] = a.tables[to.circ + i];
  __syncthreads();

  const SpillPlane<N1> g(a.spill, slot, kx, N0, M2);  // element (z, y) at g.at(z, y)
  {
    // warm L2 with the plane of the cluster a.prefetch_ahead clusters later (a hint only)
    const long long cl = (long long)blockIdx.z * gridDim.y + blockIdx.y + a.prefetch_ahead;
    if (a.prefetch_ahead > 0 && cl < (long long)gridDim.y * gridDim.z) {
      const SpillPlane<N1> nxt(a.spill, (int)(cl % gridDim.y), (int)(cl / gridDim.y), N0, M2);
      prefetch_plane_rows_l2<C::THREADS>(nxt, q * (N0 / K), N0 / K);
    }
  }
  // T column of ky = K*k + q: packed index h = q & 1, ky' = (K/2)*k + (q >> 1)
  const float* T = a.sys_diag[sys] + (((long long)kx * 2 + (q & 1)) * N1) * M0;

  // stage 1: rows.  Lane t of a row team loads y' + L*m for y' = t + SR*e, folds with
  // the K-th roots of unity, twiddles once by w_M1^(y'*q), then an L-point FFT.  Lane t
  // uses the same row-FFT twiddles (tw_r[k1*SR + t]) and fold twiddles w_M1^(y'*q) for
  // every row: they are read from shared memory once, into registers (stage 3 likewise).
  // The rank is a compile-time constant inside (one copy of the stage per rank), so the
  // fold's roots of unity and the rank-0 case cost no run-time selects.
  with_rank<K>(q, [&](auto rank) {
    constexpr int q = decltype(rank)::value;
    const int team = threadIdx.x / SR, t = threadIdx.x % SR;
    const int tr = row_of_team<SR, C::NTEAMS_R, N0>(team);
    float2* buf = xbuf + team * C::TBUF_R;
    float2 twr[ER];
    load_lane_twiddles<L>(twr, tw_r, t);
    float2 cw[ER];
#pragma unroll
    for (int e = 0; e < ER; ++e) cw[e] = circ[(din_index<L>(t, e) * q) % M1];
    float2 nv[NM][ER];  // the next row's values, loaded while the current one is transformed
    // With YT = 2*SR, y = t + SR*e and y + SR (registers e, e + 1 for even e) are one
    // aligned 16-byte pair of the spill row: a team of SR lanes reads 16*SR contiguous bytes.
    constexpr int YT = SpillPlane<N1>::YT;
    constexpr bool kPair = YT == 2 * SR && L % YT == 0 && ER % 2 == 0;
    auto load_row = [&](int zz) {
#pragma unroll
      for (int m = 0; m < NM; ++m) {
        if constexpr (kPair) {
#pragma unroll
          for (int e = 0; e < ER; e += 2) g.pair(zz, din_index<L>(t, e) + L * m, nv[m][e], nv[m][e + 1]);
        } else {
#pragma unroll
          for (int e = 0; e < ER; ++e) nv[m][e] = g.at(zz, din_index<L>(t, e) + L * m);
        }
      }
    };
    load_row(tr < N0 ? tr : 0);
#pragma unroll 2
    for (int it = 0; it < C::LPT; ++it) {
      const int z = tr + it * C::NTEAMS_R;
      float2 v[ER];
#pragma unroll
      for (int e = 0; e < ER; ++e) {
        float2 acc = nv[0][e];
#pragma unroll
        for (int m = 1; m < NM; ++m) acc = cadd(acc, rootK<K, -1>(nv[m][e], m * q));
        v[e] = q == 0 ? acc : cmul(acc, cw[e]);
      }
      if (it + 1 < C::LPT) load_row(z + C::NTEAMS_R < N0 ? z + C::NTEAMS_R : 0);
      team_fft_din_to_dout_r<L, -1, false>(v, t, buf, twr);
      if (z < N0) {
#pragma unroll
        for (int r = 0; r < ER; ++r) P[z * LDP + dout_index<L>(t, r)] = v[r];
      }
    }
  });
  __syncthreads();

  // stage 2: the CTA's L columns, M0-point FFT along z (upper half zero), x T,
  // inverse, crop
  {
    const int team = threadIdx.x / SZ, t = threadIdx.x % SZ;
    float2* buf = xbuf + team * C::TBUF_Z;
    constexpr bool kRegTw = EZ <= 16;
    float2 twz[kRegTw ? EZ : 1];
    if constexpr (kRegTw) load_lane_twiddles<M0>(twz, tw_z, t);
    auto tcol = [&](int col) { return T + (long long)((K / 2) * col + (q >> 1)) * M0; };
    float tnext[EZ];
    load_tcol<EZ, SZ>(tnext, tcol(team < L ? team : 0), t);
#pragma unroll
    for (int c0 = 0; c0 < L; c0 += C::NTEAMS_Z) {
      const int col = c0 + team;
      // team < NTEAMS_Z, so with L a multiple of NTEAMS_Z every column exists
      constexpr bool kFull = L % C::NTEAMS_Z == 0;
      const bool ok = kFull || col < L;
      const int colc = ok ? col : 0;
      float tv[EZ];
#pragma unroll
      for (int r = 0; r < EZ; ++r) tv[r] = tnext[r];
      float2 v[EZ];
#pragma unroll
      for (int e = 0; e < EZ / 2; ++e) v[e] = P[din_index<M0>(t, e) * LDP + colc];
      if constexpr (kRegTw) team_fft_din_to_dout_r<M0, -1, true>(v, t, buf, twz);
      else team_fft_din_to_dout<M0, -1, true>(v, t, buf, tw_z);
#pragma unroll
      for (int r = 0; r < EZ; ++r) v[r] = cscale(v[r], tv[r]);
      if (c0 + C::NTEAMS_Z < L) {
        const int cn = c0 + C::NTEAMS_Z + team;
        load_tcol<EZ, SZ>(tnext, tcol(kFull || cn < L ? cn : 0), t);
      }
      if constexpr (kRegTw) team_fft_dout_to_din_r<M0, 1, true>(v, t, buf, twz);
      else team_fft_dout_to_din<M0, 1, true>(v, t, buf, tw_z);
      if (ok) {
#pragma unroll
        for (int e = 0; e < EZ / 2; ++e) P[din_index<M0>(t, e) * LDP + col] = v[e];
      }
    }
  }
  __syncthreads();

  // stage 3: rows, L-point inverse FFT in place: P[z][y'] = R_q[z][y']
  {
    const int team = threadIdx.x / SR, t = threadIdx.x % SR;
    const int tr = row_of_team<SR, C::NTEAMS_R, N0>(team);
    float2* buf = xbuf + team * C::TBUF_R;
    float2 twr[ER];
    load_lane_twiddles<L>(twr, tw_r, t);
#pragma unroll 2
    for (int it = 0; it < C::LPT; ++it) {
      const int z = tr + it * C::NTEAMS_R;
      const int zc = z < N0 ? z : 0;
      float2 v[ER];
#pragma unroll
      for (int r = 0; r < ER; ++r) v[r] = P[zc * LDP + dout_index<L>(t, r)];
      team_fft_dout_to_din_r<L, 1, false>(v, t, buf, twr);
      if (z < N0) {
#pragma unroll
        for (int e = 0; e < ER; ++e) P[z * LDP + din_index<L>(t, e)] = v[e];
      }
    }
  }
  cluster.sync();  // every R_q is complete

  // stage 4: CTA q writes rows [q*N0/K, (q+1)*N0/K): u_q = w_M1^(-y'*q) R_q[y'],
  // out[y' + L*m] = sum_q e^(2*pi*i*m*q/K) u_q for m < K/2 (a K-point inverse DFT)
  {
    const float2* R[K];
#pragma unroll
    for (int qq = 0; qq < K; ++qq) R[qq] = cluster.map_shared_rank(P, qq);
    constexpr int ROWS = N0 / K;
    static_assert(C::THREADS % L == 0, "a thread keeps its y through the stage-4 loop");
    const int y = threadIdx.x % L;  // the same for every item of this thread
    float2 cy[K];                   // w_M1^(y*qq), from registers
#pragma unroll
    for (int qq = 1; qq < K; ++qq) cy[qq] = circ[(y * qq) % M1];
    static_assert((ROWS * L) % C::THREADS == 0, "stage-4 items per thread");
#pragma unroll
    for (int j = 0; j < ROWS * L / C::THREADS; ++j) {
      const int i = threadIdx.x + j * C::THREADS;
      const int z = q * ROWS + i / L;
      float2 u[K];
      u[0] = R[0][z * LDP + y];
#pragma unroll
      for (int qq = 1; qq < K; ++qq) u[qq] = cmulc(R[qq][z * LDP + y], cy[qq]);
      Dft<K, 1>::run(u);
#pragma unroll
      for (int m = 0; m < NM; ++m) g.at(z, y + L * m) = u[m];
    }
  }
  // Keep this CTA's shared memory alive until the partners have read it.  Every value a
  // thread read from a partner was consumed by the stores above, so those reads have been
  // performed; the arrive needs no release ordering (which would also wait for this CTA's
  // global stores to complete), hence the relaxed form.
  asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.aligned;\n" ::: "memory");
}

// ------------------------------------------------------------------------ pass C ----
template <int N2, int YT>
__global__ void __launch_bounds__(XPassCfg<N2, YT>::THREADS, XPassCfg<N2, YT>::C_IN_TILE ? 3 : 1)
inv_x_combine_kernel(PassArgs a) {
  using C = XPassCfg<N2, YT>;
  constexpr int M2 = C::M2, E = C::E, S = C::S, LPT = C::LPT;
  extern __shared__ __align__(128) float2 smem[];
  float2* tiles = smem;                          // 2 x spill tile [M2][YT] (swizzled)
  float2* xbuf = tiles + 2 * C::TILE_ELEMS;      // teams' exchange buffers (unless in the tile)
  float2* tw = xbuf + (C::C_IN_TILE ? 0 : C::NTEAMS * C::TBUF);
  __shared__ double red[32];
  __shared__ __align__(8) uint64_t bar[2];       // tile ci landed: bar[ci & 1], phase ci >> 1
  __shared__ int abort_sh;

  const int sys = blockIdx.z;
  if (a.active && !a.active[sys]) return;
  const int z = blockIdx.y;
  const int y0 = blockIdx.x * YT;
  const int N0 = a.N0, N1 = a.N1;

  if (threadIdx.x == 0) {
    mbar_init(smem_u32(&bar[0]), 1);
    mbar_init(smem_u32(&bar[1]), 1);
    fence_mbar_init();
    abort_sh = 0;
  }
  for (int i = threadIdx.x; i < M2; i += C::THREADS) tw[i] = a.tables[i];
  __syncthreads();

  const int team = threadIdx.x / S, t = threadIdx.x % S;
  float2* buf = xbuf + team * C::TBUF;
  const long long plane = (long long)N1 * N2;

  const int slot0 = a.sys_slot0[sys], ncoil = a.sys_nslot[sys];
  // one bulk copy of coil ci's spill tile into tiles[ci & 1] (thread 0)
  auto issue = [&](int ci) {
    if (a.inject_stall == ci + 1) return;  // a wait that nothing completes (fault injection)
    const uint32_t b = smem_u32(&bar[ci & 1]);
    mbar_expect_tx(b, C::TILE_BYTES);
    bulk_copy_g2s(smem_u32(tiles + (ci & 1) * C::TILE_ELEMS),
                  a.spill + spill_tile_offset(slot0 + ci, z, blockIdx.x, N0, N1, M2), C::TILE_BYTES, b);
  };

  float2 acc[LPT][E / 2];
#pragma unroll
  for (int l = 0; l < LPT; ++l)
#pragma unroll
    for (int e = 0; e < E / 2; ++e) acc[l][e] = make_float2(0.f, 0.f);

  const float2* sm = a.sys_smaps[sys];
  if (threadIdx.x == 0 && ncoil > 0) issue(0);
  int issued = ncoil > 0 ? 1 : 0;  // thread 0's count of copies issued
  int landed = 0;                  // copies whose wait completed
#pragma unroll 1
  for (int ci = 0; ci < ncoil; ++ci) {
    // the buffer of coil ci + 1 was released by the barrier at the end of coil ci - 1
    if (threadIdx.x == 0 && ci + 1 < ncoil) {
      issue(ci + 1);
      issued = ci + 2;
    }
    if (!mbar_wait(smem_u32(&bar[ci & 1]), (ci >> 1) & 1, &abort_sh)) abort_sh = 1;
    __syncthreads();
    if (abort_sh) break;  // read after the barrier: the same decision in every thread
    landed = ci + 1;
    const int coil = a.slot_coil[slot0 + ci];
    const float2* ss = sm ? sm + (long long)coil * N0 * plane + (long long)z * plane : nullptr;
    float2* tile = tiles + (ci & 1) * C::TILE_ELEMS;
#pragma unroll
    for (int l = 0; l < LPT; ++l) {
      const int line = team + l * C::NTEAMS;
      const long long row = (long long)(y0 + line) * N2;
      // coil-map (or multiplier) values first: their latency hides behind the FFT
      float2 m[E / 2];
#pragma unroll
      for (int e = 0; e < E / 2; ++e) {
        const int xi = din_index<M2>(t, e);
        m[e] = ss ? ss[row + xi] : (a.mul ? a.mul[(long long)z * plane + row + xi] : make_float2(1.f, 0.f));
      }
      float2 v[E];
#pragma unroll
      for (int r = 0; r < E; ++r) v[r] = tile[spill_in_tile(dout_index<M2>(t, r), line, YT)];
      if constexpr (C::C_IN_TILE) {
        __syncthreads();  // every team has its values: the tile becomes the exchange space
        team_fft_dout_to_din_xor<M2, 1>(v, t, tile + team * M2, tw);
        fence_proxy_async_smem();  // these writes precede the bulk copy that refills the tile
      } else {
        team_fft_dout_to_din<M2, 1, true>(v, t, buf, tw);
      }
#pragma unroll
      for (int e = 0; e < E / 2; ++e) {
        const float2 val = ss ? cmulc(v[e], m[e]) : cmul(v[e], m[e]);
        acc[l][e] = cadd(acc[l][e], val);
      }
    }
    __syncthreads();  // this tile buffer is refilled two coils later
  }
  if (abort_sh) {
    // a copy did not land in time: wait (bounded, one by one) for the copies still in
    // flight so none writes into shared memory after the CTA ends, report, write nothing
    if (threadIdx.x == 0) {
      for (int j = landed; j < issued; ++j) {
        const long long t0 = clock64();
        while (!mbar_try_wait(smem_u32(&bar[j & 1]), (j >> 1) & 1) && clock64() - t0 < kWaitCycles) {
        }
      }
      if (a.wait_error) atomicExch(a.wait_error, 1);
    }
    return;
  }

  // epilogue
  double dot = 0.0;
  const float2* xs = a.sys_x[sys] + (long long)z * plane;
  float2* outp = a.sys_out[sys];
  const float lambda = a.sys_lambda ? a.sys_lambda[sys] : 0.f;
#pragma unroll
  for (int l = 0; l < LPT; ++l) {
    const int y = y0 + team + l * C::NTEAMS;
#pragma unroll
    for (int e = 0; e < E / 2; ++e) {
      const int xi = din_index<M2>(t, e);
      float2 val = acc[l][e];
      const float2 xv = xs[(long long)y * N2 + xi];
      if (lambda != 0.f) val = make_float2(fmaf(lambda, xv.x, val.x), fmaf(lambda, xv.y, val.y));
      float2* o = outp + z * a.out_ldz + y * a.out_ldy + xi;
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
