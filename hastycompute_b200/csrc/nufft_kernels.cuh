// Non-uniform FFT (types 1 and 2) on sm_100a: the gridding method with the
// "exponential of semicircle" kernel of Barnett, Magland and af Klinteberg (SIAM J. Sci.
// Comput. 41, 2019), the method of the finufft/cufinufft libraries that the reference
// calls (hasty::fft::CUDANufft, lib/fft/nufft.cpp:540-767).
//
// Conventions (those of the reference's plans): coordinates [3][K] float32, row a pairs
// with image axis a (nufft.cpp:192-197), any real value, 2*pi periodic; modes are
// centred, k_a = i_a - floor(N_a/2) for array index i_a < N_a;
//   type 1:  f[k] = sum_j c_j exp(isign * i * k . x_j)
//   type 2:  c_j  = sum_k f[k] exp(isign * i * k . x_j)
// Fine grid n_a = 2 N_a (upsampling 2).  Kernel width w from the tolerance,
// phi(z) = exp(beta * (sqrt(1 - (2z/w)^2) - 1)) for |z| < w/2 (z in fine-grid cells),
// beta = 2.30 w.  Type 1 = spread c_j * phi(g - u_j) onto the fine grid (u_j = x_j n/(2pi)),
// FFT with sign isign, divide by phi_hat(k) and crop; type 2 = the transpose.
//
// Samples are bucketed by fine-grid bin once per plan (counting sort), so that spreading
// (vector reductions into global memory) and interpolation (gathers) walk the grid with
// locality.  The atomics make type 1 bitwise non-deterministic, as the reference's
// cufinufft is.
#pragma once

#include "common.cuh"

namespace hb {

constexpr int kNufftBin = 8;  // fine-grid cells per bin edge
constexpr float kNufftInvTwoPi = 0.159154943091895336f;

// A plan of dimension d < 3 keeps the 3-axis layout with its leading 3 - d axes
// degenerate (N = n = 1, one bin, coordinates 0, no spreading along them, correction 1).
struct NufftGeom {
  int N[3];          // modes per axis
  int n[3];          // fine grid per axis (2 N; 1 on a degenerate axis)
  int nb[3];         // bins per axis
  int w;             // kernel width (cells)
  float beta;        // kernel shape
  long long K;       // samples
  int dim;           // 1, 2 or 3 transformed axes (the trailing ones)
};

__device__ __forceinline__ float nufft_grid_pos(float x, int n) {
  float u = x * kNufftInvTwoPi * (float)n;
  u -= (float)n * floorf(u / (float)n);
  return u < (float)n ? u : 0.f;  // rounding may land exactly on n
}

__device__ __forceinline__ float es_kernel(float z, float beta, float inv_hw) {
  const float t = z * inv_hw;
  const float s = 1.f - t * t;
  return s > 0.f ? expf(beta * (sqrtf(s) - 1.f)) : 0.f;
}

// First cell and the W kernel values of one axis.
template <int W>
__device__ __forceinline__ int nufft_axis_weights(float u, float beta, float* wt) {
  const float hw = 0.5f * (float)W;
  const int i0 = (int)ceilf(u - hw);
  const float inv_hw = 1.f / hw;
#pragma unroll
  for (int m = 0; m < W; ++m) wt[m] = es_kernel((float)(i0 + m) - u, beta, inv_hw);
  return i0;
}

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// *p += v as one vector reduction (no value returned, so the issuing warp does not wait)
__device__ __forceinline__ void red_add(float2* p, float2 v) {
  asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(v.x), "f"(v.y) : "memory");
}

// ---- binning (once per plan) ----
__global__ void nufft_bin_count_kernel(NufftGeom g, const float* coords, int* sample_bin, int* bin_count) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= g.K) return;
  int b[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float u = nufft_grid_pos(coords[a * g.K + j], g.n[a]);
    const int bi = (int)u / kNufftBin;
    b[a] = bi < g.nb[a] ? bi : g.nb[a] - 1;
  }
  const int bin = (b[0] * g.nb[1] + b[1]) * g.nb[2] + b[2];
  sample_bin[j] = bin;
  atomicAdd(&bin_count[bin], 1);
}

// Exclusive prefix sum of n ints by one CTA of 1024 threads (bin counts -> offsets).
__global__ void __launch_bounds__(1024) nufft_scan_kernel(const int* count, int* offset, int n) {
  __shared__ int part[1024];
  const int per = (n + 1023) / 1024;
  const int lo = threadIdx.x * per, hi = (lo + per) < n ? (lo + per) : n;
  int s = 0;
  for (int i = lo; i < hi; ++i) s += count[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {  // inclusive Hillis-Steele scan of the parts
    const int v = threadIdx.x >= d ? part[threadIdx.x - d] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int run = part[threadIdx.x] - s;
  for (int i = lo; i < hi; ++i) {
    offset[i] = run;
    run += count[i];
  }
}

__global__ void nufft_bin_scatter_kernel(long long K, const int* sample_bin, int* cursor, int* perm) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= K) return;
  perm[atomicAdd(&cursor[sample_bin[j]], 1)] = (int)j;
}

// Kernel weights of axis a, or the single weight 1 at cell 0 on a degenerate axis
template <int W, int WA>
__device__ __forceinline__ int nufft_axis(const NufftGeom& g, const float* coords, int a, int j, float* wt) {
  if constexpr (WA == 1) {
    wt[0] = 1.f;
    return 0;
  } else {
    return nufft_axis_weights<W>(nufft_grid_pos(coords[a * g.K + j], g.n[a]), g.beta, wt);
  }
}

// ---- type 1: spread (grid pre-zeroed); grid y = transform within the batch ----
template <int W, int DIM>
__global__ void __launch_bounds__(256) nufft_spread_kernel(NufftGeom g, const float* coords, const int* perm,
                                                           const float2* c, long long c_ld, float2* grid) {
  constexpr int W0 = DIM >= 3 ? W : 1, W1 = DIM >= 2 ? W : 1;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.K) return;
  const int j = perm[i];
  const float2 cj = c[(long long)blockIdx.y * c_ld + j];
  float w0[W0], w1[W1], w2[W];
  const int i0 = nufft_axis<W, W0>(g, coords, 0, j, w0);
  const int i1 = nufft_axis<W, W1>(g, coords, 1, j, w1);
  const int i2 = nufft_axis<W, W>(g, coords, 2, j, w2);
  float2* G = grid + (long long)blockIdx.y * g.n[0] * g.n[1] * g.n[2];
  int x2[W];
#pragma unroll
  for (int m = 0; m < W; ++m) x2[m] = wrap(i2 + m, g.n[2]);
#pragma unroll 1
  for (int a = 0; a < W0; ++a) {
    const float2 ca = cscale(cj, w0[a]);
    float2* Ga = G + (long long)wrap(i0 + a, g.n[0]) * g.n[1] * g.n[2];
#pragma unroll
    for (int b = 0; b < W1; ++b) {
      const float2 cab = cscale(ca, w1[b]);
      float2* Gab = Ga + (long long)wrap(i1 + b, g.n[1]) * g.n[2];
#pragma unroll
      for (int m = 0; m < W; ++m) red_add(Gab + x2[m], cscale(cab, w2[m]));
    }
  }
}

// ---- type 2: interpolate ----
template <int W, int DIM>
__global__ void __launch_bounds__(256) nufft_interp_kernel(NufftGeom g, const float* coords, const int* perm,
                                                           const float2* grid, float2* c, long long c_ld) {
  constexpr int W0 = DIM >= 3 ? W : 1, W1 = DIM >= 2 ? W : 1;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.K) return;
  const int j = perm[i];
  float w0[W0], w1[W1], w2[W];
  const int i0 = nufft_axis<W, W0>(g, coords, 0, j, w0);
  const int i1 = nufft_axis<W, W1>(g, coords, 1, j, w1);
  const int i2 = nufft_axis<W, W>(g, coords, 2, j, w2);
  const float2* G = grid + (long long)blockIdx.y * g.n[0] * g.n[1] * g.n[2];
  int x2[W];
#pragma unroll
  for (int m = 0; m < W; ++m) x2[m] = wrap(i2 + m, g.n[2]);
  float2 acc = make_float2(0.f, 0.f);
#pragma unroll 1
  for (int a = 0; a < W0; ++a) {
    const float2* Ga = G + (long long)wrap(i0 + a, g.n[0]) * g.n[1] * g.n[2];
    float2 sa = make_float2(0.f, 0.f);
#pragma unroll
    for (int b = 0; b < W1; ++b) {
      const float2* Gab = Ga + (long long)wrap(i1 + b, g.n[1]) * g.n[2];
      float2 sb = make_float2(0.f, 0.f);
#pragma unroll
      for (int m = 0; m < W; ++m) {
        const float2 v = Gab[x2[m]];
        sb.x = fmaf(w2[m], v.x, sb.x);
        sb.y = fmaf(w2[m], v.y, sb.y);
      }
      sa.x = fmaf(w1[b], sb.x, sa.x);
      sa.y = fmaf(w1[b], sb.y, sa.y);
    }
    acc.x = fmaf(w0[a], sa.x, acc.x);
    acc.y = fmaf(w0[a], sa.y, acc.y);
  }
  c[(long long)blockIdx.y * c_ld + j] = acc;
}

// ---- mode <-> fine-grid maps with the kernel correction 1/phi_hat (corr: [N0 | N1 | N2]) ----
__device__ __forceinline__ long long nufft_mode_cell(const NufftGeom& g, long long m, float* scale,
                                                     const float* corr) {
  const int i2 = (int)(m % g.N[2]);
  const int i1 = (int)((m / g.N[2]) % g.N[1]);
  const int i0 = (int)(m / ((long long)g.N[2] * g.N[1]));
  const int k0 = i0 - g.N[0] / 2, k1 = i1 - g.N[1] / 2, k2 = i2 - g.N[2] / 2;
  *scale = corr[i0] * corr[g.N[0] + i1] * corr[g.N[0] + g.N[1] + i2];
  const int c0 = k0 < 0 ? k0 + g.n[0] : k0, c1 = k1 < 0 ? k1 + g.n[1] : k1, c2 = k2 < 0 ? k2 + g.n[2] : k2;
  return ((long long)c0 * g.n[1] + c1) * g.n[2] + c2;
}

// type 1: f[t][mode] = grid[t][cell(mode)] / phi_hat(mode)
__global__ void nufft_deconv_kernel(NufftGeom g, const float2* grid, const float* corr, float2* f, long long f_ld) {
  const long long nm = (long long)g.N[0] * g.N[1] * g.N[2];
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nm) return;
  float s;
  const long long cell = nufft_mode_cell(g, m, &s, corr);
  const float2 v = grid[(long long)blockIdx.y * g.n[0] * g.n[1] * g.n[2] + cell];
  f[(long long)blockIdx.y * f_ld + m] = cscale(v, s);
}

// type 2: grid[t][cell(mode)] = f[t][mode] / phi_hat(mode)  (grid pre-zeroed)
__global__ void nufft_precorrect_kernel(NufftGeom g, const float2* f, long long f_ld, const float* corr, float2* grid) {
  const long long nm = (long long)g.N[0] * g.N[1] * g.N[2];
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nm) return;
  float s;
  const long long cell = nufft_mode_cell(g, m, &s, corr);
  grid[(long long)blockIdx.y * g.n[0] * g.n[1] * g.n[2] + cell] = cscale(f[(long long)blockIdx.y * f_ld + m], s);
}

// ---- Toeplitz diagonal through the NUFFT ----
// a[i] = v, times w[i] when w is given
__global__ void fill_c64_kernel(float2* a, long long n, float2 v, const float* w) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = w ? cscale(v, w[i]) : v;
}

// Circulant (ifftshift) layout of a centred [M0][M1][M2] array, scaled:
// out[n] = s * in[(n + M/2) mod M] per axis (offset d = n for n < M/2, n - M otherwise).
__global__ void ifftshift3_scale_kernel(const float2* in, int M0, int M1, int M2, float s, float2* out) {
  const long long nv = (long long)M0 * M1 * M2;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  const int n2 = (int)(i % M2), n1 = (int)((i / M2) % M1), n0 = (int)(i / ((long long)M1 * M2));
  const int c0 = (n0 + M0 / 2) % M0, c1 = (n1 + M1 / 2) % M1, c2 = (n2 + M2 / 2) % M2;
  out[i] = cscale(in[((long long)c0 * M1 + c1) * M2 + c2], s);
}

// ---- SENSE around the NUFFT ----
constexpr int kNufftMaxBatch = 32;  // transforms per batch (coil-map pointers by value)
struct CoilMaps {
  const float2* s[kNufftMaxBatch];
};

// out (+)= sum_b conj(S_b) * f[b]   (f: [nb][nvox]); accumulate = 0 overwrites
__global__ void sense_coil_combine_kernel(const float2* f, int nb, long long nvox, CoilMaps maps, float2* out,
                                          int accumulate) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nvox) return;
  float2 acc = accumulate ? out[v] : make_float2(0.f, 0.f);
  for (int b = 0; b < nb; ++b) acc = cadd(acc, cmulc(f[b * nvox + v], maps.s[b][v]));
  out[v] = acc;
}

// k-space step of the SENSE normal operator (the reference's mid-appliers):
// k[b][j] = (k[b][j] - y_b[j]) * w[j]  (y_b and w nullable)
struct KdataPtrs {
  const float2* y[kNufftMaxBatch];
};
__global__ void sense_kspace_mid_kernel(float2* k, int nb, long long K, KdataPtrs y, const float* w) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= K) return;
  const float wj = w ? w[j] : 1.f;
  for (int b = 0; b < nb; ++b) {
    float2 v = k[b * K + j];
    if (y.y[b]) v = csub(v, y.y[b][j]);
    k[b * K + j] = cscale(v, wj);
  }
}

// k[b][j] = y_b[j] * w[j]  (weighted copy of k-space rows)
__global__ void sense_kspace_weight_kernel(float2* k, int nb, long long K, KdataPtrs y, const float* w) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= K) return;
  const float wj = w[j];
  for (int b = 0; b < nb; ++b) k[b * K + j] = cscale(y.y[b][j], wj);
}

// f[b] = S_b * x
__global__ void sense_coil_expand_kernel(const float2* x, int nb, long long nvox, CoilMaps maps, float2* f) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nvox) return;
  const float2 xv = x[v];
  for (int b = 0; b < nb; ++b) f[b * nvox + v] = cmul(xv, maps.s[b][v]);
}

}  // namespace hb
