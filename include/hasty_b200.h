/*
 * hasty_b200.h -- C ABI of the B200 (sm_100a) Toeplitz-embedded SENSE normal operator
 * and its batched conjugate-gradient solver.
 *
 * Plain pointers and sizes only.  Complex arrays are interleaved complex64
 * (float re, float im), C-contiguous, in the reference's axis order: an image is
 * [nz][ny][nx] (x fastest), the 2x Toeplitz grid is [2nz][2ny][2nx].  All data pointers
 * are DEVICE pointers on the plan's device unless a parameter says "host".
 * `stream` is a cudaStream_t (NULL = legacy default stream).  Every call is
 * asynchronous on `stream` unless documented otherwise.
 *
 * Calls that take systems (hb_toeplitz_apply, hb_sense_normal_apply*, hb_cg_run*)
 * synchronise `stream` once per group of systems to upload its descriptor tables.
 *
 * Every function returns HB_OK (0) or an error code; hb_last_error() gives the
 * message of the last failure on the calling thread.  No function aborts the process
 * or traps on the device.
 *
 * Reference interfaces replaced (HastyCompute, paths inside that project):
 *   hb_diag_build / hb_diag_pack   hasty::fft::CUDANormalNufftToeplitz::build_diagonal
 *                                  (lib/fft/nufft.cpp:932-1053, decl nufft.ixx:234-259)
 *                                  and the from-diagonal constructor (nufft.cpp:1133-1161)
 *   hb_toeplitz_apply              CUDANormalNufftToeplitz::apply / apply_add /
 *                                  apply_addcmul / apply_inplace (nufft.cpp:1163-1197)
 *   hb_sense_normal_apply          hasty::mri::sense_normal_apply with the Toeplitz body
 *                                  (lib/mri/sense.ixx:500-578; CUDASenseNormal::apply
 *                                  sense.ixx:274-282) and BatchedSenseNormal::apply over
 *                                  outer batches (lib/mri/batch_sense.cpp:349-450)
 *   hb_cg_run                      hasty::op::ConjugateGradient::run (lib/op/opalgs.cpp:50-96)
 *                                  and BatchedConjugateGradient::run (opalgs.ixx:93-121)
 */
#ifndef HASTY_B200_H
#define HASTY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HB_OK 0
#define HB_ERR_INVALID 1     /* bad argument (null pointer, size, alignment)       */
#define HB_ERR_UNSUPPORTED 2 /* image size not compiled in                          */
#define HB_ERR_CUDA 3        /* CUDA runtime error                                  */
#define HB_ERR_WORKSPACE 4   /* workspace smaller than required                     */
#define HB_ERR_NOT_PD 5      /* CG: p^H A p <= 0 ("A was not positive definite")    */

/* CG per-system status codes (hb_cg_run status_host) */
#define HB_CG_RUNNING 0
#define HB_CG_CONVERGED 1
#define HB_CG_NOT_PD 2

typedef struct hb_plan hb_plan;

/* Library version (major*10000 + minor*100 + patch). */
int hb_version(void);

/* Message of the last error on this thread ("" if none). */
const char* hb_last_error(void);

/* True (1) if an image of nz x ny x nx is supported by the compiled kernels. */
int hb_size_supported(int64_t nz, int64_t ny, int64_t nx);

/* Geometry plan for images nz x ny x nx on `device`: uploads the twiddle tables
 * (allocates a few KB of device memory).  Replaces the geometry part of the
 * CUDANormalNufftToeplitz constructors (nufft.cpp:1055-1161). */
int hb_plan_create(hb_plan** plan, int64_t nz, int64_t ny, int64_t nx, int device);
int hb_plan_destroy(hb_plan* plan);

/* Arithmetic of the normal operator's x-axis pass.  No counterpart in the reference (its
 * transforms are cuFFT in FP32).
 *  HB_PRECISION_FP32   (default) every pass in FP32 on the CUDA cores.
 *  HB_PRECISION_BF16X3 the forward x pass (coil expand, zero-pad, 2nx-point DFT) as a
 *                      dense contraction on the tensor cores (tcgen05): BF16 hi + lo parts
 *                      of both operands, three products per real product, FP32
 *                      accumulation; the other passes stay FP32.  ny = nx = 128 only
 *                      (HB_ERR_UNSUPPORTED otherwise).  Uploads a 256 KB table once.
 * The setting applies to every later call with this plan. */
#define HB_PRECISION_FP32 0
#define HB_PRECISION_BF16X3 1
int hb_plan_set_precision(hb_plan* plan, int precision);
int hb_plan_precision(const hb_plan* plan);

/* Reads and clears the device's flag for a pass that gave up waiting on one of its
 * mbarriers (after about one second): the x passes' bulk copies of spill tiles, or the
 * tensor-core pass's operands and contractions.  HB_ERR_CUDA with a message if it was set
 * (the output of that launch is incomplete), else HB_OK.  Synchronous.  hb_cg_run and
 * hb_cg_run_systems check it themselves; after the asynchronous calls (normal op,
 * Toeplitz apply) the caller checks it.  The flag is one word per device: calls that run
 * concurrently on one device (several streams or threads) share it, so one call's check
 * may report, and clear, another's stall; a caller that needs the attribution runs such
 * calls one after another. */
int hb_wait_status(int device);

/* Fault injection for tests of the path above (no counterpart in the reference): later
 * tensor-core x passes of this plan omit the DFT-table copy of 16-sample chunk `chunk`
 * (0 <= chunk < nx / 16), so each CTA's wait for it runs out after about one second and
 * the CTA returns without writing its output; the device stays usable and hb_wait_status
 * (or the CG's own check) reports it.  chunk = -1 turns it off (the default). */
int hb_plan_inject_tc_stall(hb_plan* plan, int chunk);
/* The same for the FP32 x passes: later inverse x passes (pass C) of this plan omit the
 * bulk copy of the spill tile of coil index `coil` (0-based within each system), so each
 * CTA's wait for it runs out after about one second and the CTA returns without writing
 * its output; reported as above.  coil = -1 turns it off (the default).  Systems with
 * fewer coils are not affected. */
int hb_plan_inject_x_stall(hb_plan* plan, int coil);

/* Number of floats of one packed diagonal (= 8 * nz * ny * nx).  Every packed diagonal
 * passed to the calls below must start on a 16-byte boundary (HB_ERR_INVALID otherwise):
 * the plane pass reads its z columns with 16-byte loads. */
int64_t hb_diag_packed_floats(const hb_plan* plan);

/* Pack a reference-layout diagonal T [2nz][2ny][2nx] complex64 into the internal
 * layout the normal operator reads (real part only; the imaginary part of T only acts
 * on the cropped-away Nyquist offsets).  Replaces taking ownership of `diagonal` in
 * CUDANormalNufftToeplitz(at::Tensor&& diagonal, nmodes) (nufft.cpp:1133-1161). */
int hb_diag_pack(const hb_plan* plan, const void* T_complex, float* packed, void* stream);

/* Workspace bytes for hb_diag_build with `nsamples` sample points. */
size_t hb_diag_build_workspace_bytes(const hb_plan* plan, int64_t nsamples);

/* Build the Toeplitz diagonal of a trajectory (build_diagonal, nufft.cpp:932-1053):
 * coords: float [3][nsamples] device (row a pairs with image axis a: z, y, x; radians
 * in [-pi, pi)).  Writes the packed diagonal (if `packed` != NULL) and/or the
 * reference-layout complex64 T [2nz][2ny][2nx] (if `T_complex` != NULL).  FP64
 * arithmetic throughout. */
int hb_diag_build(const hb_plan* plan, const float* coords, int64_t nsamples, float* packed,
                  void* T_complex, void* workspace, size_t workspace_bytes, void* stream);

/* Workspace bytes of hb_sense_normal_apply for nsys systems of ncoil coils (all in one
 * launch); hb_toeplitz_apply needs hb_normal_workspace_bytes(plan, 1, 1). */
size_t hb_normal_workspace_bytes(const hb_plan* plan, int64_t nsys, int64_t ncoil);

/* Single Toeplitz normal op (no coils), nufft.cpp:1163-1197:
 *   y = crop(IFFT(T * FFT(pad(in))))
 *   out[z*out_ldz + y*out_ldy + x] (=|+=) y * (mul ? mul : 1)
 * accumulate = 0: apply / apply_inplace (out may alias in); 1: apply_add / apply_addcmul. */
int hb_toeplitz_apply(const hb_plan* plan, const void* in, void* out, int64_t out_ldz,
                      int64_t out_ldy, const void* mul, int accumulate, const float* packed_diag,
                      void* workspace, size_t workspace_bytes, void* stream);

/* Toeplitz SENSE normal op over nsys independent systems:
 *   out[s] = sum_{c in coils} conj(S_c) * Top_{d(s)}(S_c * x[s]) + lambda * x[s]
 * x, out: [nsys][nz][ny][nx]; smaps: [ncoil_total][nz][ny][nx];
 * coils: host array [ncoil] of indices into smaps; packed_diags: [ndiag][packed];
 * diag_index: host array [nsys] (NULL = diagonal 0 for every system).
 * out must not alias x.  Systems are processed in groups that fit the workspace. */
int hb_sense_normal_apply(const hb_plan* plan, int64_t nsys, const void* x, void* out,
                          const void* smaps, const int64_t* coils, int64_t ncoil,
                          const float* packed_diags, const int64_t* diag_index, float lambda,
                          void* workspace, size_t workspace_bytes, void* stream);

/* One system of a heterogeneous batch (jobs with their own buffers, coil maps, coil
 * lists, diagonals and lambda).  All pointers are device pointers except `coils` (host).
 *   x      normal op: input image; CG: initial guess in, solution out
 *   out    normal op: output image (must not alias another system's x); CG: unused
 *   b      CG: right-hand side; normal op: unused
 *   smaps  this system's coil maps [*][nz][ny][nx]; coils[0..ncoil) index into them
 *   packed_diag  this system's packed diagonal; lambda adds lambda * x */
typedef struct hb_system {
  void* x;
  void* out;
  const void* b;
  const void* smaps;
  const int64_t* coils;
  int64_t ncoil;
  const float* packed_diag;
  float lambda;
  /* CG only, nullable: circulant preconditioner of this system ([nz][ny][nx] float32 from
   * hb_precond_build); when set, hb_cg_run_systems runs preconditioned CG for it
   * (opalgs.cpp:50-96 with P).  Zero-initialise the struct to leave it unset. */
  const float* precond;
} hb_system;

/* Workspace bytes for nsys systems with total_coils (system, coil) pairs handled in one
 * launch sequence: normal op when iters < 0, CG with `iters` iterations otherwise. */
size_t hb_systems_workspace_bytes(const hb_plan* plan, int64_t nsys, int64_t total_coils, int iters);

/* The Toeplitz SENSE normal op over a heterogeneous batch (BatchedSenseNormal::apply,
 * lib/mri/batch_sense.cpp:349-450, with per-outer-batch coil lists).  Systems are
 * processed in groups that fit the workspace, each group in one launch sequence. */
int hb_sense_normal_apply_systems(const hb_plan* plan, int64_t nsys, const hb_system* systems,
                                  void* workspace, size_t workspace_bytes, void* stream);

/* Capture each CG iteration of a group as a CUDA graph and replay it (hb_cg_run_systems). */
#define HB_CG_GRAPH 1

/* Batched CG over a heterogeneous batch (BatchedConjugateGradient::run,
 * lib/op/opalgs.ixx:93-121); same semantics and return codes as hb_cg_run. */
int hb_cg_run_systems(const hb_plan* plan, int64_t nsys, const hb_system* systems, int iters,
                      double tol, int flags, int32_t* status_host, int32_t* iters_done_host,
                      void* workspace, size_t workspace_bytes, void* stream);

/* ---- Running batch of CG solves (continuous batching) ----
 *
 * Replaces the reference's host-side fan-out of independent CG solves over a thread pool
 * of stream contexts (BatchedConjugateGradient::run, lib/op/opalgs.ixx:93-121, fed by
 * lib/mri/batch_sense.cpp:45-79) by one device-resident batch per image size that
 * systems join and leave at iteration boundaries: every hb_cg_batch_step runs, in one
 * launch sequence over all members, the initialisation of the systems added since the
 * previous step (r = b - (A + lambda I) x, p = r) and one iteration of every other member
 * (opalgs.cpp:50-96).  A member leaves when it converges (sqrt(Re<r, r>) < tol), breaks
 * down (HB_CG_NOT_PD) or has run its own iteration budget.  A member's iterates are bitwise
 * those of hb_cg_run_systems on the same system, whatever else is in the batch.
 *
 * The batch holds up to max_systems systems with up to max_coil_slots (system, coil)
 * pairs in total, in a caller workspace of hb_cg_batch_workspace_bytes.  x (initial guess
 * in, solution out) and b stay caller buffers and must stay alive until the system is
 * retired.  Preconditioned systems (hb_system.precond) are refused (HB_ERR_UNSUPPORTED).
 * hb_cg_batch_step synchronises `stream` (it reads the members' status back). */
typedef struct hb_cg_batch hb_cg_batch;
size_t hb_cg_batch_workspace_bytes(const hb_plan* plan, int64_t max_systems, int64_t max_coil_slots);
int hb_cg_batch_create(hb_cg_batch** batch, const hb_plan* plan, int64_t max_systems, int64_t max_coil_slots,
                       void* workspace, size_t workspace_bytes);
int hb_cg_batch_destroy(hb_cg_batch* batch);
/* Queues one system (copied, coil list included) with its iteration budget (>= 1) and
 * tolerance; *handle identifies it.  HB_ERR_WORKSPACE when no capacity is free. */
int hb_cg_batch_add(hb_cg_batch* batch, const hb_system* system, int iters, double tol, int64_t* handle);
/* One iteration boundary for every member (see above); *in_batch receives the number of
 * members still in the batch afterwards. */
int hb_cg_batch_step(hb_cg_batch* batch, void* stream, int64_t* in_batch);
/* Up to cap systems that left the batch, oldest first: handle, HB_CG_* status and
 * iterations done (host arrays, each nullable); *n_out receives how many. */
int hb_cg_batch_retire(hb_cg_batch* batch, int64_t* handles, int32_t* status, int32_t* iters, int64_t cap,
                       int64_t* n_out);

/* Workspace bytes of hb_cg_run for nsys systems handled at once. */
size_t hb_cg_workspace_bytes(const hb_plan* plan, int64_t nsys, int64_t ncoil, int iters);

/* Batched CG on (A^H A)_toeplitz + lambda I, opalgs.cpp:50-96 per system:
 * x: [nsys][image] initial guess, overwritten with the solution; b: right-hand sides.
 * Runs `iters` iterations (stops a system early when sqrt(r^H r) < tol).
 * status_host / iters_done_host: optional host arrays [nsys], filled on return.
 * This call synchronises `stream` before it returns (the reference reads the CG
 * scalars on the host too).  Returns HB_ERR_NOT_PD if any system hit p^H A p <= 0
 * (that system's x is left at its last valid iterate). */
int hb_cg_run(const hb_plan* plan, int64_t nsys, void* x, const void* b, const void* smaps,
              const int64_t* coils, int64_t ncoil, const float* packed_diags,
              const int64_t* diag_index, float lambda, int iters, double tol,
              int32_t* status_host, int32_t* iters_done_host, void* workspace,
              size_t workspace_bytes, void* stream);

/* Autotuner (no counterpart in the reference, which has one cuFFT call per transform):
 * times every compiled schedule of the plane pass (cluster split x CTA size) for this
 * plan's image size on `nslots` (system, coil) slots and keeps the fastest in the plan.
 * Synchronises `stream`.  chosen / best_ms (nullable) receive the schedule index and its
 * time per launch.  The environment variable HB_PLANE_VARIANT, when set, overrides. */
size_t hb_autotune_workspace_bytes(const hb_plan* plan, int64_t nslots);
/* Name of the plane-pass schedule the plan's next call launches ("mod4t256": the ky-mod-4
 * split plane_mod_kernel, 4-CTA clusters of 256 threads; "q2t128": the parity split
 * plane_yz_kernel, 2x2-CTA clusters of 128 threads; ...), after HB_PLANE_VARIANT and
 * hb_plan_autotune.  A static string owned by the library.  No counterpart in the
 * reference (cuFFT chooses its own plans, nufft.cpp:1184-1186). */
const char* hb_plan_plane_schedule(const hb_plan* plan);
int hb_plan_autotune(hb_plan* plan, int64_t nslots, void* workspace, size_t workspace_bytes,
                     void* stream, int* chosen, double* best_ms);

/* Allocation-free variant of hb_toeplitz_apply.  No counterpart in the reference.
 *
 * For callers that may not allocate device memory themselves, e.g. reconstruction
 * plugins that run inside a host application that owns a fixed device-memory budget,
 * or code under a memory manager that forbids cudaMalloc after start-up.  It needs no
 * plan and no workspace: the scratch (the 2 * nz * ny * nx complex64 spill of the
 * three passes) is a file-scope device array of HB_NOALLOC_SCRATCH_BYTES that every GPU
 * loading this library holds until the process exits, and the twiddle tables live in a
 * second small device array.  The caller still passes the input, the output and the
 * packed diagonal (hb_diag_pack / hb_diag_build write into caller memory).
 *
 * Limits and behaviour:
 *  - 16 * nz * ny * nx must not exceed HB_NOALLOC_SCRATCH_BYTES (16 MiB: up to 2^20
 *    voxels, e.g. 128 x 128 x 64); larger sizes return HB_ERR_WORKSPACE with a message.
 *  - Sizes whose twiddle tables exceed the built-in table array return
 *    HB_ERR_UNSUPPORTED (every size hb_size_supported accepts fits).
 *  - Works on the calling thread's current device.  The first call on a device looks up
 *    the arrays' device addresses.
 *  - Every call copies its descriptor block (and, when the size differs from the
 *    previous call's on this device, the twiddle tables) from host memory with
 *    cudaMemcpyAsync on `stream` and then waits for `stream` with
 *    cudaStreamSynchronize, so the call returns only after the work queued on `stream`
 *    before it has finished; the three passes themselves are then queued on `stream`
 *    without waiting.  hb_toeplitz_apply does the same through its table upload.
 *  - All calls share the arrays, which keep the last call's contents (nothing in them
 *    needs to start at zero).  Calls that overlap on the GPU (several streams or
 *    threads) race on the shared scratch: serialise them.
 *  - Calls no cudaMalloc, cudaFree or other allocating routine. */
#define HB_NOALLOC_SCRATCH_BYTES (16u << 20)
int hb_toeplitz_apply_noalloc(int64_t nz, int64_t ny, int64_t nx, const void* in, void* out,
                              int64_t out_ldz, int64_t out_ldy, const void* mul, int accumulate,
                              const float* packed_diag, void* stream);

/* ---- Non-uniform FFT (types 1 and 2) and the SENSE operators around it ----
 *
 * Replaces hasty::fft::CUDANufft (cufinufft plan + setpts + execute,
 * lib/fft/nufft.cpp:540-767, declared nufft.ixx:108-160) and the coil loops of the SENSE
 * forward/adjoint operators that use it (lib/mri/sense.ixx:426-497).  Same conventions:
 * coords is float32 [3][nsamples] on the device, row a pairing with image axis a
 * (nufft.cpp:192-197), in radians (2*pi periodic); modes are centred,
 * k_a = i_a - floor(N_a / 2) for array index i_a, arrays [nz][ny][nx];
 *   type 1:  f[k] = sum_j c[j] exp(isign * i * k . x_j)      (reference: isign = +1)
 *   type 2:  c[j] = sum_k f[k] exp(isign * i * k . x_j)      (reference: isign = -1)
 * Method: exponential-of-semicircle gridding kernel with upsampling 2 (the published
 * method of finufft); kernel width w = ceil(log10(1/tol)) + 1 fine-grid cells.
 * 2*N_a must be one of 8, 16, 32, 64, 128, 256, 512, 96, 160, 192, 320 and >= 2w.
 * Type 1 accumulates with atomics, so its last bits vary from run to run.
 * Lower dimensions (the reference's 1-D and 2-D plans, nufft.ixx:72-160): nz = 1 makes a
 * 2-D plan over (ny, nx) and nz = ny = 1 a 1-D plan over nx; coords is then [2][nsamples]
 * or [1][nsamples] (rows pairing with the transformed axes in order).
 *
 * hb_nufft_create copies coords, sorts the samples by fine-grid bin and allocates the
 * fine grids of `maxbatch` (1..32) transforms plus as many mode and k-space arrays; it synchronises
 * `stream`.  Transforms run in batches of maxbatch.  c is [ntransf][nsamples], f is
 * [ntransf][nz][ny][nx]. */
typedef struct hb_nufft hb_nufft;
int hb_nufft_create(hb_nufft** plan, int64_t nz, int64_t ny, int64_t nx, const float* coords, int64_t nsamples,
                    double tol, int maxbatch, int device, void* stream);
int hb_nufft_destroy(hb_nufft* plan);
/* Kernel width w (fine-grid cells) the plan uses. */
int hb_nufft_width(const hb_nufft* plan);
int hb_nufft_type1(const hb_nufft* plan, const void* c, void* f, int64_t ntransf, int isign, void* stream);
int hb_nufft_type2(const hb_nufft* plan, const void* f, void* c, int64_t ntransf, int isign, void* stream);

/* SENSE adjoint: out (+)= sum_b conj(S[coils[b]]) * type1(w * kdata[b]) (isign +1), kdata
 * [ncoil][nsamples], smaps [*][nz][ny][nx], coils a HOST array of ncoil map indices,
 * weights float32 [nsamples] (nullable: w = 1); accumulate = 0 overwrites out.  The CG
 * right-hand side of the reference's SENSE reconstructions (reconstruct_util.py:69-87). */
int hb_sense_adjoint_nufft(const hb_nufft* plan, const void* kdata, const void* smaps, const int64_t* coils,
                           int64_t ncoil, const float* weights, void* out, int accumulate, void* stream);
/* SENSE normal operator through the NUFFT with the reference's k-space manipulators
 * (BatchedSenseNormal standard_kdata / standard_weighted / standard_weighted_kdata
 * manipulators, lib/mri/batch_sense.cpp:452-486; the coil loop of sense.ixx:426-497):
 *   out (+)= sum_b conj(S[c_b]) * type1( w * (type2(S[c_b] * x) - kdata[c_b]) ),  c_b = coils[b]
 * kdata [C][nsamples] indexed by coil number (nullable), weights [nsamples] float32
 * (nullable); with both NULL it is the explicit normal operator A^H A.  The plan's mode
 * and k-space arrays are its temporaries. */
int hb_sense_normal_nufft(const hb_nufft* plan, const void* x, const void* smaps, const int64_t* coils, int64_t ncoil,
                          const void* kdata, const float* weights, void* out, int accumulate, void* stream);

/* Toeplitz diagonal through the NUFFT, the reference's own construction
 * (build_diagonal_base, lib/fft/nufft.cpp:932-971, at tolerance `tol`): the PSF is a
 * type-1 NUFFT of the sample weights (nullable float32 [nsamples], 1 when NULL; the
 * density-compensated kernel of reconstruct_util.py:59-66) onto the 2x grid's modes,
 * shifted to circulant layout and
 * scaled by 1/prod(2N), then FFT'd.  Same outputs as hb_diag_build (packed and/or the
 * complex T [2nz][2ny][2nx]) to the NUFFT tolerance instead of FP64-exact, in
 * milliseconds instead of seconds.  Needs 4*N per axis among the NUFFT's fine-grid lengths
 * (image axes of 8..128; HB_ERR_UNSUPPORTED for 96 and 160, use hb_diag_build there).  Allocates its NUFFT plan (a (4nz)(4ny)(4nx)
 * complex64 fine grid) for the duration of the call and synchronises `stream`. */
int hb_diag_build_nufft(const hb_plan* plan, const float* coords, int64_t nsamples, double tol, const float* weights,
                        float* packed, void* T_complex, void* stream);

/* SENSE forward: kdata[b] = type2(S[coils[b]] * x) (isign -1). */
int hb_sense_forward_nufft(const hb_nufft* plan, const void* x, const void* smaps, const int64_t* coils,
                           int64_t ncoil, void* kdata, void* stream);

/* ---- Circulant preconditioner ----
 *
 * Replaces hasty::mri::CirculantPreconditionerOp (build_diagonal and apply,
 * lib/mri/precond.cpp:17-117) and circulant_precond (python/python/hastypy/base/
 * torch_precond.py:60-105).  P = IFFT diag(precond) FFT on the nz x ny x nx grid, the
 * inverse of the best circulant approximation of sum_c S_c^H A^H A S_c + lambda I (the
 * operator hb_cg_run_systems solves): precond[k] = 1 / (d[k] + lambda) with d[k] its
 * Fourier-domain diagonal, evaluated from the trajectory's PSF (a type-1 NUFFT at `tol`)
 * and the coil maps' autocorrelations on the 2x grid.  precond is float32 [nz][ny][nx] in
 * FFT (uncentred) order.  hb_precond_build allocates its temporaries for the duration of
 * the call (a NUFFT fine grid of (4nz)(4ny)(4nx) complex64, then up to nine (2nz)(2ny)(2nx)
 * arrays) and synchronises `stream`.  `coils` is a HOST array of ncoil map indices. */
int hb_precond_build(const hb_plan* plan, const float* coords, int64_t nsamples, double tol, const void* smaps,
                     const int64_t* coils, int64_t ncoil, float lambda, float* precond, void* stream);
/* out = P in (one image; in == out allowed). */
int hb_precond_apply(const hb_plan* plan, const float* precond, const void* in, void* out, void* stream);

/* ---- Locally low rank: block singular-value thresholding and ADMM vector steps ----
 *
 * hb_svt_blocks replaces hasty::svt::svt_soft / svt_hard on extracted blocks and the block
 * loops of Random3DBlocksSVT / Normal3DBlocksSVT (lib/op/svt.cpp:60-490).  x is
 * [d0][d1][S0][S1][S2] complex64 (d0 <= 32: the low-rank axis, e.g. frames; d1 e.g.
 * encodings), thresholded in place.  corners is a DEVICE int32 [nblocks][3] array of block
 * corners in (S0, S1, S2); a block is the matrix [d1*b0*b1*b2][d0] (extract_block with
 * flatten_split 0 and transpose, svt.cpp:11-58).  soft = 1: singular values s -> max(s -
 * thresh, 0); soft = 0: keep the round(thresh) largest.  The blocks of one call must not
 * overlap (they are processed concurrently); a corner whose block does not fit is
 * skipped.  Singular values come from an FP64 eigen-decomposition of the block's Gram
 * matrix (cyclic Jacobi), the block update is in FP32.
 *
 * hb_admm_vectors: the scaled-ADMM vector steps around the CG x-update and the SVT
 * z-update (opalgs.cpp:103-111, batch_sense.ixx:302-431), n complex64 values:
 *   stage 0: b = b0 + (rho/2)(z - u);  stage 1: z = x + u;  stage 2: u = u + x - z. */
int hb_svt_blocks(void* x, int64_t d0, int64_t d1, int64_t S0, int64_t S1, int64_t S2, int64_t b0, int64_t b1,
                  int64_t b2, const int32_t* corners, int64_t nblocks, double thresh, int soft, void* stream);
int hb_admm_vectors(int64_t n, int stage, const void* x, void* z, void* u, const void* b0, void* b, float rho,
                    void* stream);

/* ---- measurement hooks (no counterpart in the reference; used by benchmarks) ----
 * Kernel kinds for the profile counters. */
#define HB_KERNEL_EXPAND_FWD_X 0   /* pass A */
#define HB_KERNEL_PLANE_YZ 1       /* pass B */
#define HB_KERNEL_INV_X_COMBINE 2  /* pass C */
#define HB_KERNEL_CG_UPDATE 3      /* CG vector updates / reductions */
#define HB_KERNEL_DIAG 4           /* diagonal construction / packing */
#define HB_KERNEL_NUFFT 5          /* NUFFT: binning, spreading, fine-grid FFT, interpolation, SENSE */
#define HB_KERNEL_KINDS 6

/* Total number of kernels this library has launched in this process. */
uint64_t hb_launch_count(void);

/* Start recording a CUDA event pair around every kernel launch (on the launching
 * stream).  hb_profile_stop synchronises the recorded events, writes per-kind total
 * device milliseconds and launch counts (arrays of `nkinds`), and stops recording. */
int hb_profile_start(void);
int hb_profile_stop(double* ms, int64_t* launches, int nkinds);

#ifdef __cplusplus
}
#endif

#endif /* HASTY_B200_H */
