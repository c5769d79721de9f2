// C ABI of the block singular-value thresholding step (include/hasty_b200.h, section
// "Locally low rank").  Replaces the block loops of hasty::svt::Random3DBlocksSVT and
// Normal3DBlocksSVT (lib/op/svt.cpp:268-490) with one launch per set of non-overlapping
// blocks.
#include <cuda_runtime.h>

#include <string>

#include "../../include/hasty_b200.h"
#include "runtime.cuh"
#include "svt_kernels.cuh"

using namespace hb;

extern "C" {

int hb_svt_blocks(void* x, int64_t d0, int64_t d1, int64_t S0, int64_t S1, int64_t S2, int64_t b0, int64_t b1,
                  int64_t b2, const int32_t* corners, int64_t nblocks, double thresh, int soft, void* stream) {
  if (!x || (nblocks > 0 && !corners) || nblocks < 0)
    return fail(HB_ERR_INVALID, "hb_svt_blocks: null pointer or negative block count");
  if (d0 < 1 || d0 > kSvtMaxCols) return fail(HB_ERR_UNSUPPORTED, "hb_svt_blocks: d0 must be in [1, 32]");
  if (d1 < 1 || b0 < 1 || b1 < 1 || b2 < 1 || b0 > S0 || b1 > S1 || b2 > S2)
    return fail(HB_ERR_INVALID, "hb_svt_blocks: block shape must be positive and fit the image");
  if (d1 * b0 * b1 * b2 > (int64_t)1 << 30 || d1 * S0 * S1 * S2 * d0 > ((int64_t)1 << 40))
    return fail(HB_ERR_INVALID, "hb_svt_blocks: sizes too large");
  if (!soft && thresh < 0.0) return fail(HB_ERR_INVALID, "hb_svt_blocks: hard thresholding needs rank >= 0");
  if (nblocks == 0) return HB_OK;
  if (nblocks > 0x7fffffff) return fail(HB_ERR_INVALID, "hb_svt_blocks: too many blocks");
  SvtArgs a{};
  a.x = (float2*)x;
  a.d0 = (int)d0; a.d1 = (int)d1;
  a.S0 = (int)S0; a.S1 = (int)S1; a.S2 = (int)S2;
  a.b0 = (int)b0; a.b1 = (int)b1; a.b2 = (int)b2;
  a.corners = corners;
  a.soft = soft ? 1 : 0;
  a.thresh = (float)thresh;
  a.rank = soft ? 0 : (int)(thresh + 0.5);
  cudaStream_t st = (cudaStream_t)stream;
  {
    LaunchScope ls(HB_KERNEL_CG_UPDATE, st);
    svt_blocks_kernel<<<(unsigned)nblocks, kSvtThreads, 0, st>>>(a);
  }
  HB_CHECK_LAUNCH();
  return HB_OK;
}

int hb_admm_vectors(int64_t n, int stage, const void* x, void* z, void* u, const void* b0, void* b, float rho,
                    void* stream) {
  if (n < 0 || stage < 0 || stage > 2 || !x || !z || !u || (stage == 0 && (!b0 || !b)))
    return fail(HB_ERR_INVALID, "hb_admm_vectors: bad stage or null pointer");
  if (n == 0) return HB_OK;
  cudaStream_t st = (cudaStream_t)stream;
  {
    LaunchScope ls(HB_KERNEL_CG_UPDATE, st);
    admm_vectors_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, stage, (const float2*)x, (float2*)z,
                                                                    (float2*)u, (const float2*)b0, (float2*)b, rho);
  }
  HB_CHECK_LAUNCH();
  return HB_OK;
}

}  // extern "C"
