// Batched conjugate-gradient vector updates with FP64 reductions, kept on the device.
//
// Restates lib/op/opalgs.cpp:50-96 (ConjugateGradient::run) for many independent
// systems at once.  Per iteration i (rz[i] = Re<r, r> known):
//   normal op:   Ap = (A + lambda I) p, plus per-CTA FP64 partials of Re<p, Ap>
//   step_xr:     pAp = sum(partials); if pAp <= 0 -> status NOT_PD (x untouched);
//                alpha = rz[i] / pAp;  x += alpha p;  r -= alpha Ap;  partials of Re<r,r>
//   step_p:      rz[i+1] = sum(partials); p = r + (rz[i+1] / rz[i]) p;
//                sqrt(rz[i+1]) < tol -> status CONVERGED
// Preconditioned (z != null): between step_xr and step_p the host applies z = P r and
// cg_rz replaces the partials by those of Re<r, z>; step_p then uses z for r, as
// opalgs.cpp:78-88 does (and the tolerance test reads sqrt(Re<r, z>)).
// Every CTA reduces the partial arrays itself in one fixed order, so all CTAs agree
// bit for bit and no host synchronisation is needed.  A system whose status is not
// RUNNING is skipped by every later kernel (active[sys] == 0).
#pragma once

#include "common.cuh"

namespace hb {

enum CgStatus : int { kCgRunning = 0, kCgConverged = 1, kCgNotPD = 2 };

struct CgState {
  int nsys;
  long long nv;               // elements per system
  float2* const* sys_x;       // [nsys] solution of each system (caller buffers)
  const float2* const* sys_b; // [nsys] right-hand side of each system (caller buffers)
  int* iter;                  // current iteration (device counter, advanced by cg_advance)
  float2* r;             // [nsys][nv]
  float2* p;             // [nsys][nv]
  float2* ap;            // [nsys][nv]
  double* rz;            // [nsys][iters+1]
  int rz_ld;             // iters + 1
  int* status;           // [nsys]
  int* active;           // [nsys]
  int* iters_done;       // [nsys]
  const double* pap_part;  // [nsys][npap]
  int npap;
  double* rr_part;       // [nsys][gridDim.x of the update kernels]
  double tol;
  float2* z;             // [nsys][nv] preconditioned residual (null: no preconditioner)
  const float* const* sys_pdiag;  // [nsys] circulant preconditioner diagonals (entries nullable)
};

// Deterministic block-wide sum of n doubles (same order in every CTA).
__device__ double block_sum_fixed(const double* v, int n, double* red) {
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += v[i];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  __syncthreads();
  if (lane == 0) red[warp] = s;
  __syncthreads();
  double tot = 0.0;
  const int nw = blockDim.x / 32;
  for (int w = 0; w < nw; ++w) tot += red[w];
  __syncthreads();
  return tot;
}

__device__ void block_write_partial(double s, double* out, double* red) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  __syncthreads();
  if (lane == 0) red[warp] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x / 32); ++w) tot += red[w];
    *out = tot;
  }
}

// r = b - Ap; p = r; partial Re<r, r>
__global__ void __launch_bounds__(256) cg_init_kernel(CgState s) {
  __shared__ double red[32];
  const int sys = blockIdx.y;
  const long long base = (long long)sys * s.nv;
  double acc = 0.0;
  const float2* b = s.sys_b[sys];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < s.nv; i += (long long)gridDim.x * blockDim.x) {
    const float2 r = csub(b[i], s.ap[base + i]);
    s.r[base + i] = r;
    s.p[base + i] = r;
    acc += (double)r.x * r.x + (double)r.y * r.y;
  }
  block_write_partial(acc, s.rr_part + (long long)sys * gridDim.x + blockIdx.x, red);
}

// rz[0] = sum of partials; status/active from tol.   grid: nsys blocks
__global__ void __launch_bounds__(256) cg_init_finish_kernel(CgState s, int nrr) {
  __shared__ double red[32];
  const int sys = blockIdx.x;
  const double rz = block_sum_fixed(s.rr_part + (long long)sys * nrr, nrr, red);
  if (threadIdx.x == 0) {
    if (sys == 0) *s.iter = 0;
    s.rz[(long long)sys * s.rz_ld] = rz;
    s.iters_done[sys] = 0;
    const bool run = !(sqrt(rz) < s.tol);
    s.status[sys] = run ? kCgRunning : kCgConverged;
    s.active[sys] = run ? 1 : 0;
  }
}

__global__ void __launch_bounds__(256) cg_step_xr_kernel(CgState s) {
  __shared__ double red[32];
  const int sys = blockIdx.y;
  if (!s.active[sys]) return;
  const int it = *s.iter;
  const double pap = block_sum_fixed(s.pap_part + (long long)sys * s.npap, s.npap, red);
  if (!(pap > 0.0)) {  // also catches NaN
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      s.status[sys] = kCgNotPD;
      s.active[sys] = 0;
    }
    return;
  }
  const double alpha = s.rz[(long long)sys * s.rz_ld + it] / pap;
  const float af = (float)alpha;
  const long long base = (long long)sys * s.nv;
  float2* xv = s.sys_x[sys];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < s.nv; i += (long long)gridDim.x * blockDim.x) {
    const float2 p = s.p[base + i];
    const float2 ap = s.ap[base + i];
    float2 x = xv[i];
    float2 r = s.r[base + i];
    x.x = fmaf(af, p.x, x.x);
    x.y = fmaf(af, p.y, x.y);
    r.x = fmaf(-af, ap.x, r.x);
    r.y = fmaf(-af, ap.y, r.y);
    xv[i] = x;
    s.r[base + i] = r;
    acc += (double)r.x * r.x + (double)r.y * r.y;
  }
  block_write_partial(acc, s.rr_part + (long long)sys * gridDim.x + blockIdx.x, red);
}

__global__ void __launch_bounds__(256) cg_step_p_kernel(CgState s) {
  __shared__ double red[32];
  const int sys = blockIdx.y;
  if (!s.active[sys]) return;
  const int it = *s.iter;
  const double rznew = block_sum_fixed(s.rr_part + (long long)sys * gridDim.x, gridDim.x, red);
  const double rzold = s.rz[(long long)sys * s.rz_ld + it];
  const float beta = (float)(rznew / rzold);
  const long long base = (long long)sys * s.nv;
  const float2* zr = s.z ? s.z : s.r;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < s.nv; i += (long long)gridDim.x * blockDim.x) {
    const float2 r = zr[base + i];
    float2 p = s.p[base + i];
    p.x = fmaf(beta, p.x, r.x);
    p.y = fmaf(beta, p.y, r.y);
    s.p[base + i] = p;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    s.rz[(long long)sys * s.rz_ld + it + 1] = rznew;
    s.iters_done[sys] = it + 1;
    if (sqrt(rznew) < s.tol) {
      s.status[sys] = kCgConverged;
      s.active[sys] = 0;
    }
  }
}

// Partials of Re<r, z> (replacing those of Re<r, r>); at initialisation also p = z.
__global__ void __launch_bounds__(256) cg_rz_kernel(CgState s, int init) {
  __shared__ double red[32];
  const int sys = blockIdx.y;
  if (!init && !s.active[sys]) return;
  const long long base = (long long)sys * s.nv;
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < s.nv; i += (long long)gridDim.x * blockDim.x) {
    const float2 r = s.r[base + i];
    const float2 z = s.z[base + i];
    if (init) s.p[base + i] = z;
    acc += (double)r.x * z.x + (double)r.y * z.y;
  }
  block_write_partial(acc, s.rr_part + (long long)sys * gridDim.x + blockIdx.x, red);
}

// Frequency-domain step of z = P r: z[sys] *= pdiag[sys] / nv (identity for a system
// without a preconditioner; 1/nv is the inverse FFT's normalisation).
__global__ void __launch_bounds__(256) cg_precond_scale_kernel(CgState s) {
  const int sys = blockIdx.y;
  const float* d = s.sys_pdiag[sys];
  const float inv = 1.f / (float)s.nv;
  const long long base = (long long)sys * s.nv;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < s.nv; i += (long long)gridDim.x * blockDim.x)
    s.z[base + i] = cscale(s.z[base + i], d ? d[i] * inv : inv);
}

// Ends an iteration: every kernel of the next one reads the advanced counter.
__global__ void cg_advance_kernel(int* iter) { *iter += 1; }

// ------------------------------------------------------------ running batch (engine) ----
// A running batch holds systems at different points of their solves: a member that joined
// at this iteration boundary initialises (phase 1: r = b - A x, p = r, rz = Re<r, r>) while
// the others take one iteration (phase 2), in the same launches.  The host owns each
// member's phase and iteration number and uploads them with the member tables before the
// step; rz of capacity slot k lives in rz[k][0..1], iteration i reading rz[k][i & 1] and
// writing rz[k][(i + 1) & 1], so no kernel reads what another CTA of it writes.  The
// arithmetic of an iteration is that of cg_step_xr_kernel / cg_step_p_kernel (same
// operands, same order), so a member's iterates are bitwise those of hb_cg_run_systems.
struct CgBatchState {
  int nmem;
  long long nv;
  float2* const* x;        // [nmem] solution (caller buffer)
  const float2* const* b;  // [nmem] right-hand side (caller buffer)
  float2* const* r;        // [nmem] capacity-slot vectors
  float2* const* p;
  const float2* const* ap;
  double* const* rz;       // [nmem] -> rz pair of the member's capacity slot
  const int* phase;        // [nmem] 1 = initialise, 2 = iterate
  const int* it;           // [nmem] iteration index (phase 2)
  const double* tol;       // [nmem]
  int* status;             // [nmem] out: kCgRunning / kCgConverged / kCgNotPD
  const double* pap_part;  // [nmem][npap] partials of Re<p, Ap> (pass C)
  int npap;
  double* rr_part;         // [nmem][gridDim.x]
};

// phase 1: r = b - Ap, p = r;  phase 2: the x/r update of cg_step_xr_kernel.  Partials of
// Re<r, r> either way.
__global__ void __launch_bounds__(256) cg_batch_xr_kernel(CgBatchState s) {
  __shared__ double red[32];
  const int m = blockIdx.y;
  float2* r = s.r[m];
  float2* p = s.p[m];
  const float2* ap = s.ap[m];
  double acc = 0.0;
  if (s.phase[m] == 1) {
    if (blockIdx.x == 0 && threadIdx.x == 0) s.status[m] = kCgRunning;
    const float2* b = s.b[m];
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < s.nv;
         i += (long long)gridDim.x * blockDim.x) {
      const float2 v = csub(b[i], ap[i]);
      r[i] = v;
      p[i] = v;
      acc += (double)v.x * v.x + (double)v.y * v.y;
    }
  } else {
    const double pap = block_sum_fixed(s.pap_part + (long long)m * s.npap, s.npap, red);
    if (!(pap > 0.0)) {  // also catches NaN
      if (blockIdx.x == 0 && threadIdx.x == 0) s.status[m] = kCgNotPD;
      return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) s.status[m] = kCgRunning;
    const double alpha = s.rz[m][s.it[m] & 1] / pap;
    const float af = (float)alpha;
    float2* xv = s.x[m];
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < s.nv;
         i += (long long)gridDim.x * blockDim.x) {
      const float2 pv = p[i];
      const float2 apv = ap[i];
      float2 xx = xv[i];
      float2 rr = r[i];
      xx.x = fmaf(af, pv.x, xx.x);
      xx.y = fmaf(af, pv.y, xx.y);
      rr.x = fmaf(-af, apv.x, rr.x);
      rr.y = fmaf(-af, apv.y, rr.y);
      xv[i] = xx;
      r[i] = rr;
      acc += (double)rr.x * rr.x + (double)rr.y * rr.y;
    }
  }
  block_write_partial(acc, s.rr_part + (long long)m * gridDim.x + blockIdx.x, red);
}

// phase 1: rz[0] = Re<r, r>, converged if below tol;  phase 2: the p update of
// cg_step_p_kernel, rz of the next iteration, converged if below tol.
__global__ void __launch_bounds__(256) cg_batch_p_kernel(CgBatchState s) {
  __shared__ double red[32];
  const int m = blockIdx.y;
  if (s.status[m] == kCgNotPD) return;  // written by cg_batch_xr_kernel, complete
  const double rznew = block_sum_fixed(s.rr_part + (long long)m * gridDim.x, gridDim.x, red);
  if (s.phase[m] == 1) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      s.rz[m][0] = rznew;
      if (sqrt(rznew) < s.tol[m]) s.status[m] = kCgConverged;
    }
    return;
  }
  const int it = s.it[m];
  const double rzold = s.rz[m][it & 1];
  const float beta = (float)(rznew / rzold);
  float2* p = s.p[m];
  const float2* r = s.r[m];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < s.nv; i += (long long)gridDim.x * blockDim.x) {
    const float2 rv = r[i];
    float2 pv = p[i];
    pv.x = fmaf(beta, pv.x, rv.x);
    pv.y = fmaf(beta, pv.y, rv.y);
    p[i] = pv;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    s.rz[m][(it + 1) & 1] = rznew;
    if (sqrt(rznew) < s.tol[m]) s.status[m] = kCgConverged;
  }
}

}  // namespace hb
