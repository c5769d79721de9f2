// Block singular-value thresholding (the locally-low-rank proximal step): restates
// hasty::svt::svt_soft / svt_hard on extracted blocks (lib/op/svt.cpp:60-168, block
// extraction :11-58 and insertion :170-240, the block loops of Random3DBlocksSVT and
// Normal3DBlocksSVT :268-490).
//
// x is [d0][d1][S0][S1][S2] complex64.  A block with corner (c0, c1, c2) and shape
// b0 x b1 x b2 is the matrix M [R = d1*b0*b1*b2][d0] (row = (d1 index, voxel in the block,
// row-major), column = d0 index), as extract_block(..., flatten_split 0, transpose) forms
// it.  With M = U S V^H: soft f(s) = max(s - thresh, 0), hard keeps the `rank` largest s,
// and the block is replaced by U f(S) V^H = M W,  W = V diag(f(s)/s) V^H  (0 where s = 0).
// One CTA per block:
//   1. G = M^H M in FP64 (rows staged through shared memory in chunks);
//   2. one warp diagonalises G by cyclic complex Jacobi rotations (FP64, shared memory):
//      G = V diag(lambda) V^H, s = sqrt(lambda);
//   3. W, then every row is replaced by (row) W in FP32, in place.
// Blocks of one launch must not overlap (the host launches overlapping sets in waves).
#pragma once

#include "common.cuh"

namespace hb {

constexpr int kSvtMaxCols = 32;  // d0 <= 32
constexpr int kSvtThreads = 128;
constexpr int kSvtChunk = 32;    // rows staged per Gram step (the same space later holds W)
constexpr int kSvtMaxSweeps = 15;

struct SvtArgs {
  float2* x;
  int d0, d1, S0, S1, S2;
  int b0, b1, b2;
  const int* corners;  // [nblocks][3]
  int soft;            // 1: soft threshold, 0: hard (keep `rank`)
  float thresh;
  int rank;
};

struct dcomplex {
  double x, y;
};

__device__ __forceinline__ long long svt_row_offset(const SvtArgs& a, int c0, int c1, int c2, int r) {
  const int nbv = a.b0 * a.b1 * a.b2;
  const int d1i = r / nbv, v = r % nbv;
  const int i0 = v / (a.b1 * a.b2), i1 = (v / a.b2) % a.b1, i2 = v % a.b2;
  return (((long long)d1i * a.S0 + (c0 + i0)) * a.S1 + (c1 + i1)) * a.S2 + (c2 + i2);
}

__global__ void __launch_bounds__(kSvtThreads) svt_blocks_kernel(SvtArgs a) {
  static_assert(kSvtChunk == kSvtMaxCols, "the row chunk and W share their shared memory");
  __shared__ float2 chunk[kSvtChunk][kSvtMaxCols + 1];  // Gram: staged rows; afterwards W
  __shared__ dcomplex A[kSvtMaxCols][kSvtMaxCols + 1];
  __shared__ dcomplex V[kSvtMaxCols][kSvtMaxCols + 1];
  __shared__ double wdiag[kSvtMaxCols];
  float2(*W)[kSvtMaxCols + 1] = chunk;
  const int n = a.d0;
  const int c0 = a.corners[3 * blockIdx.x], c1 = a.corners[3 * blockIdx.x + 1], c2 = a.corners[3 * blockIdx.x + 2];
  // a block that does not fit inside the image is left untouched (the host validates corners)
  if (c0 < 0 || c1 < 0 || c2 < 0 || c0 + a.b0 > a.S0 || c1 + a.b1 > a.S1 || c2 + a.b2 > a.S2) return;
  const int R = a.d1 * a.b0 * a.b1 * a.b2;
  const long long col_stride = (long long)a.d1 * a.S0 * a.S1 * a.S2;

  // 1. Gram matrix, FP64: thread t accumulates the pairs (p, q), p <= q, numbered t, t + T, ...
  const int npairs = n * (n + 1) / 2;
  constexpr int kMaxPairsPerThread = (kSvtMaxCols * (kSvtMaxCols + 1) / 2 + kSvtThreads - 1) / kSvtThreads;
  dcomplex acc[kMaxPairsPerThread];
  int pp[kMaxPairsPerThread], pq[kMaxPairsPerThread];
#pragma unroll
  for (int k = 0; k < kMaxPairsPerThread; ++k) {
    acc[k] = {0.0, 0.0};
    int idx = threadIdx.x + k * kSvtThreads, p = 0;
    while (idx >= n - p && p < n) {  // pair number -> (p, q)
      idx -= n - p;
      ++p;
    }
    pp[k] = p;
    pq[k] = p + idx;
  }
  for (int r0 = 0; r0 < R; r0 += kSvtChunk) {
    const int nr = (R - r0) < kSvtChunk ? (R - r0) : kSvtChunk;
    __syncthreads();
    for (int i = threadIdx.x; i < nr * n; i += kSvtThreads) {
      const int r = i % nr, c = i / nr;  // consecutive threads: consecutive rows of one column
      chunk[r][c] = a.x[c * col_stride + svt_row_offset(a, c0, c1, c2, r0 + r)];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kMaxPairsPerThread; ++k) {
      if (threadIdx.x + k * kSvtThreads >= npairs) continue;
      const int p = pp[k], q = pq[k];
      double sx = 0.0, sy = 0.0;
      for (int r = 0; r < nr; ++r) {
        const float2 u = chunk[r][p], v = chunk[r][q];  // conj(u) * v
        sx += (double)u.x * v.x + (double)u.y * v.y;
        sy += (double)u.x * v.y - (double)u.y * v.x;
      }
      acc[k].x += sx;
      acc[k].y += sy;
    }
  }
#pragma unroll
  for (int k = 0; k < kMaxPairsPerThread; ++k) {
    if (threadIdx.x + k * kSvtThreads >= npairs) continue;
    const int p = pp[k], q = pq[k];
    A[p][q] = acc[k];
    A[q][p] = {acc[k].x, -acc[k].y};
  }
  for (int i = threadIdx.x; i < n * n; i += kSvtThreads) V[i / n][i % n] = {i / n == i % n ? 1.0 : 0.0, 0.0};
  __syncthreads();

  // 2. cyclic complex Jacobi by warp 0; lane k owns row / column k of the updates
  if (threadIdx.x < 32) {
    const int k = threadIdx.x;
    double fro = 0.0;
    for (int j = 0; j < n; ++j)
      if (k < n) fro += A[k][j].x * A[k][j].x + A[k][j].y * A[k][j].y;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) fro += __shfl_xor_sync(0xffffffffu, fro, off);
    for (int sweep = 0; sweep < kSvtMaxSweeps; ++sweep) {
      double offd = 0.0;
      for (int j = 0; j < n; ++j)
        if (k < n && j != k) offd += A[k][j].x * A[k][j].x + A[k][j].y * A[k][j].y;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) offd += __shfl_xor_sync(0xffffffffu, offd, off);
      if (!(offd > 1e-30 * fro)) break;  // uniform across the warp
      for (int p = 0; p < n - 1; ++p) {
        for (int q = p + 1; q < n; ++q) {
          const dcomplex apq = A[p][q];
          const double mag = sqrt(apq.x * apq.x + apq.y * apq.y);
          if (!(mag > 1e-300)) continue;
          const double tau = (A[q][q].x - A[p][p].x) / (2.0 * mag);
          const double t = tau == 0.0 ? 1.0 : (tau > 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
          const double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
          const double ex = apq.x / mag, ey = apq.y / mag;  // e = apq / |apq|
          __syncwarp();
          if (k < n) {  // columns p, q of A and V: new_p = c col_p - s conj(e) col_q, new_q = s e col_p + c col_q
            const dcomplex ap = A[k][p], aq = A[k][q];
            A[k][p] = {c * ap.x - s * (ex * aq.x + ey * aq.y), c * ap.y - s * (ex * aq.y - ey * aq.x)};
            A[k][q] = {s * (ex * ap.x - ey * ap.y) + c * aq.x, s * (ex * ap.y + ey * ap.x) + c * aq.y};
            const dcomplex vp = V[k][p], vq = V[k][q];
            V[k][p] = {c * vp.x - s * (ex * vq.x + ey * vq.y), c * vp.y - s * (ex * vq.y - ey * vq.x)};
            V[k][q] = {s * (ex * vp.x - ey * vp.y) + c * vq.x, s * (ex * vp.y + ey * vp.x) + c * vq.y};
          }
          __syncwarp();
          if (k < n) {  // rows p, q of A: new_p = c row_p - s e row_q, new_q = s conj(e) row_p + c row_q
            const dcomplex rp = A[p][k], rq = A[q][k];
            A[p][k] = {c * rp.x - s * (ex * rq.x - ey * rq.y), c * rp.y - s * (ex * rq.y + ey * rq.x)};
            A[q][k] = {s * (ex * rp.x + ey * rp.y) + c * rq.x, s * (ex * rp.y - ey * rp.x) + c * rq.y};
          }
          __syncwarp();
        }
      }
    }
    // 3a. thresholded weights f(s)/s per eigenvalue
    if (k < n) {
      const double lam = A[k][k].x > 0.0 ? A[k][k].x : 0.0;
      const double sv = sqrt(lam);
      double w = 0.0;
      if (a.soft) {
        w = sv > (double)a.thresh ? (sv - (double)a.thresh) / sv : 0.0;
      } else {
        int larger = 0;  // rank of this eigenvalue (ties broken by index)
        for (int j = 0; j < n; ++j) {
          const double lj = A[j][j].x;
          larger += (lj > A[k][k].x || (lj == A[k][k].x && j < k)) ? 1 : 0;
        }
        w = larger < a.rank ? 1.0 : 0.0;
      }
      wdiag[k] = w;
    }
  }
  __syncthreads();
  // 3b. W = V diag(w) V^H
  for (int i = threadIdx.x; i < n * n; i += kSvtThreads) {
    const int r = i / n, c = i % n;
    double sx = 0.0, sy = 0.0;
    for (int j = 0; j < n; ++j) {
      const dcomplex vr = V[r][j], vc = V[c][j];  // V[r][j] w_j conj(V[c][j])
      sx += wdiag[j] * (vr.x * vc.x + vr.y * vc.y);
      sy += wdiag[j] * (vr.y * vc.x - vr.x * vc.y);
    }
    W[r][c] = make_float2((float)sx, (float)sy);
  }
  __syncthreads();
  // 3c. rows <- rows W, in place
  for (int r = threadIdx.x; r < R; r += kSvtThreads) {
    const long long off = svt_row_offset(a, c0, c1, c2, r);
    float2 m[kSvtMaxCols];
#pragma unroll
    for (int c = 0; c < kSvtMaxCols; ++c)
      if (c < n) m[c] = a.x[c * col_stride + off];
#pragma unroll 1
    for (int c = 0; c < n; ++c) {
      float2 o = make_float2(0.f, 0.f);
#pragma unroll
      for (int j = 0; j < kSvtMaxCols; ++j)
        if (j < n) o = cadd(o, cmul(m[j], W[j][c]));
      a.x[c * col_stride + off] = o;
    }
  }
}

// ADMM vector steps around the CG x-update and the SVT z-update (scaled form, constraint
// x = z; lib/op/opalgs.cpp:103-111, lib/mri/batch_sense.ixx:302-431):
//   stage 0: b = b0 + (rho/2) (z - u)    (right-hand side of (A^H A + rho/2 I) x = b)
//   stage 1: z = x + u                   (input of the proximal step, thresholded in place)
//   stage 2: u = u + x - z               (dual update)
__global__ void admm_vectors_kernel(long long n, int stage, const float2* x, float2* z, float2* u, const float2* b0,
                                    float2* b, float rho) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (stage == 0) {
    b[i] = cadd(b0[i], cscale(csub(z[i], u[i]), 0.5f * rho));
  } else if (stage == 1) {
    z[i] = cadd(x[i], u[i]);
  } else {
    u[i] = cadd(u[i], csub(x[i], z[i]));
  }
}

}  // namespace hb
