// multiscale.cuh — device-side scale-level changes (multiscale.cu).
#pragma once

#include "aw_common.cuh"

namespace aw {

// device scratch downsample() needs for an input grid din
size_t downsample_scratch_bytes(const Dims &din);
// ImageUtils::gaussianDownsample of in (grid din, spacing sin) to dout
cudaError_t downsample(const float *in, Dims din, Spacing sin, float *out, Dims dout,
                       void *scratch, cudaStream_t s);
// ImageUtils::resampleNew (clamp, linear, origin 0) of in (grid din,
// spacing sin) onto dout with spacing sout: MultiscaleManager's image
// upsampling (Algorithms/Common/MultiscaleManager.cxx:301-323)
cudaError_t resample_image(const float *in, Dims din, Spacing sin, float *out, Dims dout,
                           Spacing sout, cudaStream_t s);
// hToVelocity + resampleNew(CLAMP, rescale) + velocityToH; scratch holds
// 3 * din.n() floats
cudaError_t upsample_hfield(const float *const h[3], Dims din, float *const out[3], Dims dout,
                            int rescale, void *scratch, cudaStream_t s);

}  // namespace aw
