// fluid_fast.cuh — launchers of the register-FFT fluid kernels
// (fluid_fast.cu), used when every axis is a power of two in [16, 256] and
// the slab fits in shared memory.
#pragma once

#include "fluid.cuh"

namespace aw {

bool fast_supported(int n);
size_t fast_xy_smem(int nx, int ny);
int fast_z_cols();
size_t fast_z_smem(int nz, int q);
cudaError_t fast_configure(const FluidPlan &p);
template <class Src>
cudaError_t fast_xy_forward(const FluidPlan &p, const Src &src, cudaStream_t s);
template <class Dst>
cudaError_t fast_xy_inverse(const FluidPlan &p, const Dst &dst, cudaStream_t s);
cudaError_t fast_xy_inverse_compose(const FluidPlan &p, const ComposeArgs &a, cudaStream_t s);
cudaError_t fast_z_solve(const FluidPlan &p, int inverse, cudaStream_t s);

}  // namespace aw
