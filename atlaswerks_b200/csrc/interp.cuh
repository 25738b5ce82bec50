// interp.cuh — launchers for the interpolation-family kernels (interp.cu).
#pragma once

#include "aw_common.cuh"

namespace aw {

cudaError_t launch_apply(const float *img, const float *hx, const float *hy, const float *hz,
                         float *out, Dims d, float bg, cudaStream_t s);
cudaError_t launch_gradient(const float *a, float *gx, float *gy, float *gz, Dims d, Spacing sp,
                            int wrap, cudaStream_t s);
// scale multiplies v (device scalar when scale_ptr != nullptr, else scale_val)
cudaError_t launch_compose_hv(const float *const g[3], const float *const v[3], float *const o[3],
                              Dims d, Spacing sp, int dir, int bgs, const float *scale_ptr,
                              float scale_val, cudaStream_t s);
cudaError_t launch_compose_vh(const float *const v[3], const float *const g[3], float *const o[3],
                              Dims d, Spacing sp, int dir, int bgs, const float *scale_ptr,
                              float scale_val, cudaStream_t s);

}  // namespace aw
