// splat.cuh — deterministic splatting (the adjoint of trilinear
// interpolation), HField3DUtils::forwardApply with normalize = false
// (UtilitiesDataTypes/HField3DUtils.txx:1058-1279).
//
// The reference CPU adds each source voxel's eight weighted corner
// contributions in source (z, y, x) order, in float; the reference GPU path
// uses int32 fixed-point atomics (CUDACommon/src/cudaSplatAtomic.cu:379-448).
// Here the sources are bucketed by the cell their h lands in (counting sort:
// count, exclusive scan, scatter, per-bucket sort by source index), then
// every destination voxel merges the eight buckets that can reach it in
// source-index order and adds the contributions sequentially. No float
// atomics, run-to-run bitwise identical, and with identical inputs bitwise
// equal to the reference CPU.
#pragma once

#include "aw_common.cuh"

namespace aw {

// device scratch of one splat, sized for a grid (extended by one cell per
// axis for sources landing in (-1, 0))
struct SplatWork {
  Dims d;
  long next;        // (nx+1)(ny+1)(nz+1)
  int *offsets;     // next + 1: bucket counts, then exclusive offsets
  int *cursor;      // next: scatter cursors
  int *order;       // n: source indices grouped by bucket
  int *blocksums;   // scan partials
  int nblocks;
  float *wts;       // 8n or null: the corner weights of the source at each sorted position
};

// bytes of device scratch one splat of grid d needs; weights: room for the
// corner weights the sort can precompute (32 bytes per voxel)
size_t splat_scratch_bytes(const Dims &d, bool weights = true);
// lays out a SplatWork inside caller-provided device memory (256-aligned)
void splat_work_bind(SplatWork *w, const Dims &d, void *scratch, bool weights = true);

// out = splat of img by h (three planes), background bg; stream-ordered
cudaError_t splat(const SplatWork &w, const float *img, const float *hx, const float *hy,
                  const float *hz, float *out, float bg, cudaStream_t s);
// the two halves of splat(): the bucket sort of the sources by h, kept in w,
// and the ordered per-destination sums of img, which any number of images
// splatted by the same h can share
cudaError_t splat_sort(const SplatWork &w, const float *hx, const float *hy, const float *hz,
                       cudaStream_t s);
cudaError_t splat_gather(const SplatWork &w, const float *img, const float *hx, const float *hy,
                         const float *hz, float *out, float bg, cudaStream_t s);

}  // namespace aw
