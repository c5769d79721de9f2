// Pass A on the 5th-generation tensor cores (tcgen05): the zero-padded 2nx-point DFT along
// x as a dense contraction, for nx = ny = 128.
//
//   spill[slot][z][kx][y] = sum_{x < nx} F[kx][x] * (S_c * x)[z][y][x],  F[kx][x] = e^{-2 pi i kx x / 2nx}
//
// One CTA per (slot, z, kx half): D^T[y][kx] = A[y][x] . F[kx][x]^T with A = S_c * x
// (M = 128 lines y, N = 128 frequencies kx, K = 128 samples x).  Complex products are four
// real products (the F_im terms of the real part through the instruction's negate-A bit).
// Both operands are split into BF16 hi + lo parts and three products are kept per real
// product (hi*hi + hi*lo + lo*hi); the accumulators D_re and D_im are FP32 in tensor
// memory, 256 columns per CTA, so two CTAs share an SM and one CTA's epilogue overlaps the
// other's contraction.
//
// K runs in chunks of 16 samples (one instruction deep) through a ring of kStages stages:
// the threads split their chunk of A into the canonical K-major layout while the tensor
// core contracts the previous chunk; the matching 16 KB of the constant F table (already
// in that layout, hi/lo split on the host) arrives by one bulk copy (not multicast) that
// completes on the stage's "full" mbarrier, and tcgen05.commit signals the stage's "done"
// mbarrier when the contraction that read it has finished.  Every wait on an mbarrier
// gives up after about a second of SM clocks, sets the caller's error word and lets the
// CTA release its tensor memory and return.
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
constexpr int kCols = 128;                 // MMA N: kx frequencies of one half
constexpr int kKc = 16;                    // MMA K: x samples per chunk
constexpr int kArr = kRows * kKc * 2;      // bytes of one BF16 operand array [128][16]
constexpr int kStageA = 4 * kArr;          // A: re_hi, re_lo, im_hi, im_lo
constexpr int kStageF = 4 * kArr;          // F: re_hi, re_lo, im_hi, im_lo
constexpr int kStage = kStageA + kStageF;  // 32 KB
constexpr int kStages = 3;
constexpr int kThreads = 256;
constexpr int kTmemCols = 2 * kCols;       // D_re [0, 128), D_im [128, 256)
constexpr int kSmemBytes = kStages * kStage;
constexpr long long kWaitCycles = 2000000000LL;  // about one second of SM clocks

// Byte offset of element (row r, k) in a [128][16] K-major operand array without swizzle:
// core matrices of 8 rows x 16 bytes; the two 8-element K halves of an 8-row group are
// adjacent (kLbo = 128 bytes apart, the descriptor's leading offset) and 8-row groups are
// kSbo = 256 bytes apart (its stride offset).  With these two strides every address the
// tensor core can form from the descriptor stays inside the 4 KB array whichever of the
// two offsets it applies to which direction.
constexpr int kLbo = 128;
constexpr int kSbo = 256;
__host__ __device__ constexpr int operand_offset(int r, int k) {
  return (r / 8) * kSbo + (k / 8) * kLbo + (r % 8) * 16 + (k % 8) * 2;
}
static_assert(15 * kSbo + kLbo + 127 < kArr && 15 * kLbo + kSbo + 127 < kArr, "descriptor reach inside the array");

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

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase of the given parity to complete; false after kWaitCycles.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > kWaitCycles) return false;
  return true;
}
__device__ __forceinline__ void bulk_copy_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint4 v) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
               : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
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
// 32 consecutive columns of this warp's 32 lanes, one lane per thread
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// hi = bf16(v), lo = bf16(v - hi) for 8 values, packed in K order (element 2i in the low half)
__device__ __forceinline__ void split_bf16x8(const float* v, uint4& hi, uint4& lo) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const __nv_bfloat162 p = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    const float2 pf = __bfloat1622float2(p);
    const __nv_bfloat162 q = __floats2bfloat162_rn(v[2 * i] - pf.x, v[2 * i + 1] - pf.y);
    h[i] = *reinterpret_cast<const uint32_t*>(&p);
    l[i] = *reinterpret_cast<const uint32_t*>(&q);
  }
  hi = make_uint4(h[0], h[1], h[2], h[3]);
  lo = make_uint4(l[0], l[1], l[2], l[3]);
}

}  // namespace tc

// ftab: the forward DFT rows in operand layout, [kx half][chunk][re_hi, re_lo, im_hi,
// im_lo][operand_offset] BF16 (kStageF bytes per (half, chunk)); wait_error: set to 1 when
// an mbarrier wait gave up.
template <int N2>
__global__ void __launch_bounds__(tc::kThreads, 2) expand_fwd_x_tc_kernel(PassArgs a, const unsigned char* ftab,
                                                                          int* wait_error) {
  using namespace tc;
  static_assert(N2 == 128, "tensor-core x pass: nx = 128");
  constexpr int M2 = 2 * N2, NCH = N2 / kKc;
  extern __shared__ float2 smem[];  // operand stages (16-byte aligned, checked below)
  __shared__ __align__(8) uint64_t bar_full[kStages];
  __shared__ __align__(8) uint64_t bar_done[kStages];
  __shared__ uint32_t tmem_sh;
  __shared__ int abort_sh;

  const int h = blockIdx.x, z = blockIdx.y, slot = blockIdx.z;
  const int sys = a.slot_sys[slot];
  if (a.active && !a.active[sys]) return;  // uniform for the CTA, before any allocation
  const int N0 = a.N0, N1 = a.N1;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const uint32_t sbase = smem_u32(smem);
  if (sbase & 15u) {  // descriptors address 16-byte units
    if (tid == 0) atomicExch(wait_error, 1);
    return;
  }

  if (warp == 0) tmem_alloc(smem_u32(&tmem_sh), kTmemCols);
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(smem_u32(&bar_full[s]), 1);
      mbar_init(smem_u32(&bar_done[s]), 1);
    }
    fence_mbar_init();
    abort_sh = 0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_sh;

  const long long plane = (long long)N1 * N2;
  const float2* xs = a.sys_x[sys] + (long long)z * plane;
  const float2* sm = a.sys_smaps[sys];
  const float2* ss = sm ? sm + ((long long)a.slot_coil[slot] * N0 + z) * plane : nullptr;
  // operand preparation: thread -> row y = pr, 8-sample K half pg of each chunk
  const int pr = tid % kRows, pg = tid / kRows;
  const uint32_t poff = (uint32_t)operand_offset(pr, 8 * pg);

  int committed = -1;  // last chunk whose contraction was committed (thread 0)
  int pending = -1;    // chunk whose F copy was issued and not yet seen complete (thread 0)
#pragma unroll 1
  for (int kc = 0; kc < NCH; ++kc) {
    const int s = kc % kStages, use = kc / kStages;
    const uint32_t st = sbase + s * kStage;
    if (tid == 0) {
      // the contraction that last read stage s has finished
      if (kc >= kStages && !mbar_wait(smem_u32(&bar_done[s]), (use - 1) & 1)) abort_sh = 1;
      if (!abort_sh) {
        mbar_expect_tx(smem_u32(&bar_full[s]), kStageF);
        bulk_copy_g2s(st + kStageA, ftab + (size_t)(h * NCH + kc) * kStageF, kStageF, smem_u32(&bar_full[s]));
        pending = kc;
      }
    }
    __syncthreads();
    if (abort_sh) break;
    {
      // 8-byte loads: a system's image and coil maps need only complex64 alignment
      const int x0 = kc * kKc + 8 * pg;
      const float2* xp = xs + (long long)pr * N2 + x0;
      float re[8], im[8];
      float2 xv[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) xv[i] = __ldg(xp + i);
      if (ss) {
        const float2* sp = ss + (long long)pr * N2 + x0;
#pragma unroll
        for (int i = 0; i < 8; ++i) xv[i] = cmul(xv[i], __ldg(sp + i));
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        re[i] = xv[i].x;
        im[i] = xv[i].y;
      }
      uint4 rh, rl, ih, il;
      split_bf16x8(re, rh, rl);
      split_bf16x8(im, ih, il);
      st_shared_v4(st + 0 * kArr + poff, rh);
      st_shared_v4(st + 1 * kArr + poff, rl);
      st_shared_v4(st + 2 * kArr + poff, ih);
      st_shared_v4(st + 3 * kArr + poff, il);
    }
    fence_proxy_async_smem();  // the generic-proxy stores become visible to the tensor core
    __syncthreads();
    if (tid == 0) {
      if (!mbar_wait(smem_u32(&bar_full[s]), use & 1)) {
        abort_sh = 1;
      } else {
        pending = -1;
        tc_fence_after();
        const uint32_t fb = st + kStageA;
        const uint64_t A0 = smem_desc(st), A1 = smem_desc(st + kArr), A2 = smem_desc(st + 2 * kArr),
                       A3 = smem_desc(st + 3 * kArr);
        const uint64_t F0 = smem_desc(fb), F1 = smem_desc(fb + kArr), F2 = smem_desc(fb + 2 * kArr),
                       F3 = smem_desc(fb + 3 * kArr);
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
        mma_commit(smem_u32(&bar_done[s]));
        committed = kc;
      }
    }
  }
  if (tid == 0) {
    // the last commit covers every contraction issued before it; the earlier commits'
    // arrivals are awaited too, so that none lands after the CTA's shared memory is released
    for (int c = committed; c >= 0 && c > committed - kStages; --c)
      if (!mbar_wait(smem_u32(&bar_done[c % kStages]), (c / kStages) & 1)) abort_sh = 1;
    // on an abort, a copy still in flight must land before the CTA's shared memory is released
    if (pending >= 0) mbar_wait(smem_u32(&bar_full[pending % kStages]), (pending / kStages) & 1);
  }
  __syncthreads();
  if (!abort_sh) {
    tc_fence_after();
    // epilogue: warp w reads TMEM lanes [32 (w % 4), +32) = lines y, columns (kx) of half w / 4
    const int q = warp % 4, ch = warp / 4;
    const int y = q * 32 + lane;
    float2* dst = a.spill + spill_offset(slot, z, h * kCols, N0, N1, M2) + y;
#pragma unroll 1
    for (int cb = 0; cb < 2; ++cb) {
      const int c0 = ch * 64 + cb * 32;
      uint32_t re[32], im[32];
      tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, re);
      tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(kCols + c0), im);
      tmem_ld_wait();
#pragma unroll
      for (int j = 0; j < 32; ++j)
        dst[(long long)(c0 + j) * N1] = make_float2(__uint_as_float(re[j]), __uint_as_float(im[j]));
    }
  } else if (tid == 0) {
    atomicExch(wait_error, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kTmemCols);
}

}  // namespace hb
