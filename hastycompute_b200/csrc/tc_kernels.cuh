// Pass A on the 5th-generation tensor cores (tcgen05): the zero-padded 2nx-point DFT along
// x as a dense contraction, for nx = ny = 128.
//
//   spill(slot, z, kx, y) = sum_{x < nx} F[kx][x] * (S_c * x)[z][y][x],  F[kx][x] = e^{-2 pi i kx x / 2nx}
// (stored at spill_index, the tiled layout passes B and C read)
//
// One CTA per (slot, z): D^T[y][kx] = A[y][x] . F[kx][x]^T with A = S_c * x (M = 128
// lines y, N = 256 frequencies kx, K = 128 samples x), so every sample is loaded and split
// once.  Complex products are four real products (the F_im terms of the real part through
// the instruction's negate-A bit).  Both operands are split into BF16 hi + lo parts and
// three products are kept per real product (hi*hi + hi*lo + lo*hi); the accumulators D_re
// and D_im are FP32 in tensor memory (all 512 columns: one CTA per SM).
//
// K runs in chunks of 16 samples (one instruction deep).  Warps 0-7 split chunk kc of A
// into the canonical K-major layout (ring of kStagesA slots; the samples of chunk kc + 1
// are loaded meanwhile) and arrive on the slot's "ready" mbarrier, while the tensor core
// contracts chunk kc - 1.  One lane of warp 8 streams the constant F table (already in
// that layout, hi/lo split on the host) by bulk copies (not multicast), kFAhead chunks
// early into a ring of kStagesF slots with a "full" mbarrier each, waits for "ready" and
// "full", issues the chunk's contractions and commits them to the chunk's "done"
// mbarrier, which frees both slots.  Every wait on an mbarrier gives up after about a
// second of SM clocks (or once another thread of the CTA has given up): the CTA then
// drains its own copies and contractions, releases its tensor memory, sets the caller's
// error word and returns without writing its output.
//
// No counterpart in the reference, which runs this transform through cuFFT
// (lib/fft/nufft.cpp:1163-1197, fftn with s = 2N); the arithmetic is the transform's
// definition restricted to the nonzero half of the padded input.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include "toeplitz_kernels.cuh"

namespace hb {
namespace tc {

constexpr int kRows = 128;                 // MMA M: y lines of one (slot, z) plane
constexpr int kCols = 256;                 // MMA N: kx frequencies (all of them)
constexpr int kKc = 16;                    // MMA K: x samples per chunk
constexpr int kArr = kRows * kKc * 2;      // bytes of one BF16 A array [128][16]
constexpr int kArrF = kCols * kKc * 2;     // bytes of one BF16 F array [256][16]
constexpr int kStageA = 4 * kArr;          // A: re_hi, re_lo, im_hi, im_lo
constexpr int kStageF = 4 * kArrF;         // F: re_hi, re_lo, im_hi, im_lo
constexpr int kStagesA = 2;                // A slot of chunk kc is refilled by chunk kc + 2
constexpr int kStagesF = 4;                // F slot of chunk kc is refilled by chunk kc + 4
constexpr int kFAhead = 2;                 // F copies run this many chunks ahead
constexpr int kDone = kStagesF;            // "done" mbarrier of chunk kc: kc % kDone
constexpr int kThreads = 256;             // operand warps 0-7 (preparation, epilogue)
constexpr int kThreadsAll = kThreads + 32;  // + warp 8: bulk copies and contractions
constexpr int kTmemCols = 2 * kCols;       // D_re [0, 256), D_im [256, 512)
constexpr int kSmemBytes = kStagesA * kStageA + kStagesF * kStageF;  // 160 KB
static_assert(kFAhead + kStagesA <= kStagesF, "the F slot refilled at chunk kc was freed by chunk kc - kStagesA");

// Byte offset of element (row r, k) in a [rows][16] K-major operand array without swizzle:
// core matrices of 8 rows x 16 bytes; the two 8-element K halves of an 8-row group are
// adjacent (kLbo = 128 bytes apart, the descriptor's leading offset) and 8-row groups are
// kSbo = 256 bytes apart (its stride offset).  With these two strides every address the
// tensor core can form from the descriptor stays inside the array (4 KB for A, 8 KB for F)
// whichever of the two offsets it applies to which direction.
constexpr int kLbo = 128;
constexpr int kSbo = 256;
__host__ __device__ constexpr int operand_offset(int r, int k) {
  return (r / 8) * kSbo + (k / 8) * kLbo + (r % 8) * 16 + (k % 8) * 2;
}
static_assert(15 * kSbo + kLbo + 127 < kArr && 15 * kLbo + kSbo + 127 < kArr, "descriptor reach inside A");
static_assert(31 * kSbo + kLbo + 127 < kArrF && 31 * kLbo + kSbo + 127 < kArrF, "descriptor reach inside F");

// Instruction descriptor of tcgen05.mma kind::f16: FP32 accumulator (bits 4-5 = 1), BF16
// A and B (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24; bit 13
// negates A.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kCols >> 3) << 17) |
                            ((uint32_t)(kRows >> 4) << 24);
constexpr uint32_t kIdescNegA = kIdesc | (1u << 13);

// Shared-memory matrix descriptor: start address, leading (K) and stride (8-row) byte
// offsets in 16-byte units, version 1 (bits 46-47), no swizzle (bits 61-63 = 0).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((kLbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((kSbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

__device__ __forceinline__ void st_shared_b32(uint32_t addr, uint32_t v) {
  asm volatile("st.shared.b32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// one warp: allocate ncols tensor-memory columns, address written to shared memory
__device__ __forceinline__ void tmem_alloc(uint32_t dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// D (+)= A . B^T on the tensor core (issued by one thread)
__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// arrive on the mbarrier once every tensor-core operation issued so far by this thread is done
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
// 16 consecutive columns of this warp's 32 lanes, one lane per thread
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// hi = bf16(v), lo = bf16(v - hi) for 2 values, packed in K order (v[0] in the low half)
__device__ __forceinline__ void split_bf16x2(const float* v, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 p = __floats2bfloat162_rn(v[0], v[1]);
  const float2 pf = __bfloat1622float2(p);
  const __nv_bfloat162 q = __floats2bfloat162_rn(v[0] - pf.x, v[1] - pf.y);
  hi = *reinterpret_cast<const uint32_t*>(&p);
  lo = *reinterpret_cast<const uint32_t*>(&q);
}

}  // namespace tc

// ftab: the forward DFT rows in operand layout, [chunk][re_hi, re_lo, im_hi,
// im_lo][operand_offset] BF16 (kStageF bytes per chunk); wait_error: set to 1 when an
// mbarrier wait gave up; stall_chunk: fault injection for tests, -1 in normal use (the
// DFT-table copy of that chunk is not issued, so the wait for it runs out).
template <int N2>
__global__ void __launch_bounds__(tc::kThreadsAll, 1) expand_fwd_x_tc_kernel(PassArgs a, const unsigned char* ftab,
                                                                             int* wait_error, int stall_chunk) {
  using namespace tc;
  static_assert(N2 == 128, "tensor-core x pass: nx = 128");
  constexpr int M2 = 2 * N2, NCH = N2 / kKc;
  static_assert(M2 == kCols, "one contraction covers every frequency kx");
  extern __shared__ float2 smem[];  // A ring, then F ring (16-byte aligned, checked below)
  __shared__ __align__(8) uint64_t bar_full[kStagesF];   // F slot landed (bulk copy)
  __shared__ __align__(8) uint64_t bar_ready[kStagesA];  // A slot written (kThreads arrivals)
  __shared__ __align__(8) uint64_t bar_done[kDone];      // chunk contracted (tcgen05.commit)
  __shared__ uint32_t tmem_sh;
  __shared__ int abort_sh;
  volatile int* abort = &abort_sh;

  const int z = blockIdx.x, slot = blockIdx.y;
  const int sys = a.slot_sys[slot];
  if (a.active && !a.active[sys]) return;  // uniform for the CTA, before any allocation
  const int N0 = a.N0, N1 = a.N1;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const uint32_t sbase = smem_u32(smem);
  if (sbase & 15u) {  // descriptors address 16-byte units
    if (tid == 0) atomicExch(wait_error, 1);
    return;
  }
  const uint32_t sF = sbase + kStagesA * kStageA;

  if (warp == 0) tmem_alloc(smem_u32(&tmem_sh), kTmemCols);
  if (tid == 0) {
    for (int s = 0; s < kStagesF; ++s) mbar_init(smem_u32(&bar_full[s]), 1);
    for (int s = 0; s < kStagesA; ++s) mbar_init(smem_u32(&bar_ready[s]), kThreads);
    for (int s = 0; s < kDone; ++s) mbar_init(smem_u32(&bar_done[s]), 1);
    fence_mbar_init();
    abort_sh = 0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_sh;
  auto done_wait = [&](int c) { return mbar_wait(smem_u32(&bar_done[c % kDone]), (c / kDone) & 1, abort); };

  if (warp == kThreads / 32) {
    if (lane == 0) {
      // ---- issuer: F table copies and the contractions ----
      static_assert(NCH <= 32, "one bit per chunk");
      uint32_t inflight = 0;  // chunks whose F copy was issued and not yet seen complete
      auto issue_f = [&](int c) {
        if (c == stall_chunk) return;
        const int fs = c % kStagesF;
        mbar_expect_tx(smem_u32(&bar_full[fs]), kStageF);
        bulk_copy_g2s(sF + fs * kStageF, ftab + (size_t)c * kStageF, kStageF, smem_u32(&bar_full[fs]));
        inflight |= 1u << c;
      };
      int committed = -1;
      bool ok = true;
      for (int c = 0; c < kFAhead && c < NCH; ++c) issue_f(c);
#pragma unroll 1
      for (int kc = 0; kc < NCH && ok; ++kc) {
        if (kc + kFAhead < NCH) {
          const int prev = kc + kFAhead - kStagesF;  // last user of that F slot
          if (prev >= 0 && !done_wait(prev)) { ok = false; break; }
          issue_f(kc + kFAhead);
        }
        if (!mbar_wait(smem_u32(&bar_ready[kc % kStagesA]), (kc / kStagesA) & 1, abort) ||
            !mbar_wait(smem_u32(&bar_full[kc % kStagesF]), (kc / kStagesF) & 1, abort)) {
          ok = false;
          break;
        }
        inflight &= ~(1u << kc);
        tc_fence_after();
        const uint32_t sa = sbase + (kc % kStagesA) * kStageA, sf = sF + (kc % kStagesF) * kStageF;
        const uint64_t A0 = smem_desc(sa), A1 = smem_desc(sa + kArr), A2 = smem_desc(sa + 2 * kArr),
                       A3 = smem_desc(sa + 3 * kArr);
        const uint64_t F0 = smem_desc(sf), F1 = smem_desc(sf + kArrF), F2 = smem_desc(sf + 2 * kArrF),
                       F3 = smem_desc(sf + 3 * kArrF);
        const uint32_t dre = tmem, dim = tmem + kCols;
        const uint32_t acc = kc > 0 ? 1u : 0u;
        // D_re += A_re F_re - A_im F_im
        mma_bf16(dre, A0, F0, kIdesc, acc);
        mma_bf16(dre, A0, F1, kIdesc, 1u);
        mma_bf16(dre, A1, F0, kIdesc, 1u);
        mma_bf16(dre, A2, F2, kIdescNegA, 1u);
        mma_bf16(dre, A2, F3, kIdescNegA, 1u);
        mma_bf16(dre, A3, F2, kIdescNegA, 1u);
        // D_im += A_re F_im + A_im F_re
        mma_bf16(dim, A0, F2, kIdesc, acc);
        mma_bf16(dim, A0, F3, kIdesc, 1u);
        mma_bf16(dim, A1, F2, kIdesc, 1u);
        mma_bf16(dim, A2, F0, kIdesc, 1u);
        mma_bf16(dim, A2, F1, kIdesc, 1u);
        mma_bf16(dim, A3, F0, kIdesc, 1u);
        mma_commit(smem_u32(&bar_done[kc % kDone]));
        committed = kc;
      }
      if (!ok) abort_sh = 1;
      // before the shared memory is released: every commit's arrival and every copy in
      // flight has landed (waits bounded one by one, ignoring the abort flag)
      for (int c = committed; c >= 0 && c > committed - kDone; --c) {
        const long long t0 = clock64();
        while (!mbar_try_wait(smem_u32(&bar_done[c % kDone]), (c / kDone) & 1) && clock64() - t0 < kWaitCycles) {
        }
      }
      for (int c = 0; c < NCH; ++c) {
        if (!(inflight & (1u << c))) continue;
        const long long t0 = clock64();
        while (!mbar_try_wait(smem_u32(&bar_full[c % kStagesF]), (c / kStagesF) & 1) && clock64() - t0 < kWaitCycles) {
        }
      }
    }
  } else {
    // ---- operand warps: task j (< 4) of a thread is row r = 32 j + 4 warp + lane / 8 and
    // the sample pair pp = lane % 8 of the chunk, so that one load instruction of a warp
    // reads four 128-byte row segments; 16-byte loads when the image and the coil maps are
    // 16-byte aligned, else 8-byte loads (complex64 alignment); the next chunk's samples
    // are loaded while the current one is split ----
    const long long plane = (long long)N1 * N2;
    const float2* xs = a.sys_x[sys] + (long long)z * plane;
    const float2* sm = a.sys_smaps[sys];
    const float2* ss = sm ? sm + ((long long)a.slot_coil[slot] * N0 + z) * plane : nullptr;
    const int pp = lane % 8, rbase = 4 * warp + lane / 8;
    const bool vec = ((reinterpret_cast<uintptr_t>(xs) | reinterpret_cast<uintptr_t>(ss)) & 15u) == 0;
    float4 nx[4], ns[4];
    auto ld2 = [&](const float2* q) {
      if (vec) return __ldg(reinterpret_cast<const float4*>(q));
      const float2 u = __ldg(q), v = __ldg(q + 1);
      return make_float4(u.x, u.y, v.x, v.y);
    };
    auto load_chunk = [&](int kc) {
      const int x0 = kc * kKc + 2 * pp;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const long long o = (long long)(rbase + 32 * j) * N2 + x0;
        nx[j] = ld2(xs + o);
        if (ss) ns[j] = ld2(ss + o);
      }
    };
    load_chunk(0);
    bool ok = true;
#pragma unroll 1
    for (int kc = 0; kc < NCH; ++kc) {
      // the contraction of chunk kc - kStagesA, which read this A slot, has finished
      if (kc >= kStagesA && !done_wait(kc - kStagesA)) {
        ok = false;
        break;
      }
      const uint32_t sa = sbase + (kc % kStagesA) * kStageA;
      float re[4][2], im[4][2];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        float2 u = make_float2(nx[j].x, nx[j].y), v = make_float2(nx[j].z, nx[j].w);
        if (ss) {
          u = cmul(u, make_float2(ns[j].x, ns[j].y));
          v = cmul(v, make_float2(ns[j].z, ns[j].w));
        }
        re[j][0] = u.x;
        re[j][1] = v.x;
        im[j][0] = u.y;
        im[j][1] = v.y;
      }
      if (kc + 1 < NCH) load_chunk(kc + 1);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        uint32_t rh, rl, ih, il;
        split_bf16x2(re[j], rh, rl);
        split_bf16x2(im[j], ih, il);
        const uint32_t off = sa + (uint32_t)operand_offset(rbase + 32 * j, 2 * pp);
        st_shared_b32(off + 0 * kArr, rh);
        st_shared_b32(off + 1 * kArr, rl);
        st_shared_b32(off + 2 * kArr, ih);
        st_shared_b32(off + 3 * kArr, il);
      }
      fence_proxy_async_smem();  // the generic-proxy stores become visible to the tensor core
      mbar_arrive(smem_u32(&bar_ready[kc % kStagesA]));
    }
    if (ok) ok = done_wait(NCH - 1);  // the last commit covers every contraction
    if (!ok) {
      abort_sh = 1;
    } else {
      tc_fence_after();
      // epilogue: warp w reads TMEM lanes [32 (w % 4), +32) = lines y, columns (kx) of half w / 4
      const int q = warp % 4, ch = warp / 4;
      const int y = q * 32 + lane;
      constexpr int YT = spill_yt(kRows);
      float2* dst = a.spill + spill_tile_offset(slot, z, y / YT, N0, N1, M2);  // y's spill tile
#pragma unroll 1
      for (int cb = 0; cb < kCols / 32; ++cb) {
        const int c0 = ch * (kCols / 2) + cb * 16;
        uint32_t re[16], im[16];
        tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, re);
        tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(kCols + c0), im);
        tmem_ld_wait();
#pragma unroll
        for (int j = 0; j < 16; ++j)
          dst[spill_in_tile(c0 + j, y % YT, YT)] = make_float2(__uint_as_float(re[j]), __uint_as_float(im[j]));
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (tid == 0 && abort_sh) atomicExch(wait_error, 1);
  if (warp == 0) tmem_dealloc(tmem, kTmemCols);
}

}  // namespace hb
