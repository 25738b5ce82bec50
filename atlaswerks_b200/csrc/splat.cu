// splat.cu — deterministic counting-sort splat (see splat.cuh).
#include <climits>

#include "splat.cuh"

namespace aw {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kScanBlock = kScanThreads * kScanItems;

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// bucket of a source: the cell of its h, shifted by one so that
// h in (-1, 0) lands in bucket 0. Returns -1 for sources the reference
// skips: those outside the volume grown by one voxel
// (HField3DUtils.txx:1110-1112).
AW_D long bucket_of(const Dims &d, float px, float py, float pz) {
  if (!(px > -1.0f && px < (float)d.nx && py > -1.0f && py < (float)d.ny && pz > -1.0f &&
        pz < (float)d.nz))
    return -1;
  const int fx = ref_floor_f(px), fy = ref_floor_f(py), fz = ref_floor_f(pz);
  return ((long)(fz + 1) * (d.ny + 1) + (fy + 1)) * (d.nx + 1) + (fx + 1);
}

__global__ void __launch_bounds__(kRowThreads)
    k_count(const float *__restrict__ hx, const float *__restrict__ hy, const float *__restrict__ hz,
            Dims d, int *__restrict__ counts) {
  Voxel v;
  if (!voxel_of(d, v)) return;
  const long b = bucket_of(d, hx[v.i], hy[v.i], hz[v.i]);
  if (b >= 0) atomicAdd(counts + b, 1);
}

// block-local exclusive scan of kScanBlock ints held 4 per thread
AW_D int block_scan(int (&a)[kScanItems], int *wsum) {
  int tsum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const int x = a[k];
    a[k] = tsum;
    tsum += x;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = tsum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = lane < kScanThreads / 32 ? wsum[lane] : 0;
    int wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < kScanThreads / 32) wsum[lane] = wi - w;  // exclusive warp offsets
    if (lane == kScanThreads / 32 - 1) wsum[kScanThreads / 32] = wi;  // block total
  }
  __syncthreads();
  const int base = wsum[warp] + (incl - tsum);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) a[k] += base;
  const int total = wsum[kScanThreads / 32];
  __syncthreads();
  return total;
}

__global__ void __launch_bounds__(kScanThreads)
    k_scan_reduce(const int *__restrict__ x, long n, int *__restrict__ blocksums) {
  const long b0 = (long)blockIdx.x * kScanBlock;
  int s = 0;
  for (int k = 0; k < kScanItems; ++k) {
    const long i = b0 + (long)k * kScanThreads + threadIdx.x;
    if (i < n) s += x[i];
  }
  __shared__ int ws[kScanThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < kScanThreads / 32; ++w) t += ws[w];
    blocksums[blockIdx.x] = t;
  }
}

// one block: exclusive scan of the block sums, chunk by chunk
__global__ void __launch_bounds__(kScanThreads) k_scan_blocksums(int *__restrict__ bs, int nb) {
  __shared__ int wsum[kScanThreads / 32 + 1];
  int carry = 0;
  for (int c0 = 0; c0 < nb; c0 += kScanBlock) {
    int a[kScanItems];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      const int i = c0 + threadIdx.x * kScanItems + k;
      a[k] = i < nb ? bs[i] : 0;
    }
    const int total = block_scan(a, wsum);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      const int i = c0 + threadIdx.x * kScanItems + k;
      if (i < nb) bs[i] = a[k] + carry;
    }
    carry += total;
    __syncthreads();
  }
}

// exclusive scan in place; x[n] receives the total
__global__ void __launch_bounds__(kScanThreads)
    k_scan_apply(int *__restrict__ x, long n, const int *__restrict__ blocksums) {
  __shared__ int wsum[kScanThreads / 32 + 1];
  const long b0 = (long)blockIdx.x * kScanBlock;
  int a[kScanItems];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const long i = b0 + (long)threadIdx.x * kScanItems + k;
    a[k] = i < n ? x[i] : 0;
  }
  const int total = block_scan(a, wsum);
  const int off = blocksums[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const long i = b0 + (long)threadIdx.x * kScanItems + k;
    if (i < n) x[i] = a[k] + off;
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) x[n] = off + total;
}

__global__ void __launch_bounds__(kRowThreads)
    k_scatter(const float *__restrict__ hx, const float *__restrict__ hy,
              const float *__restrict__ hz, Dims d, const int *__restrict__ offsets,
              int *__restrict__ cursor, int *__restrict__ order) {
  Voxel v;
  if (!voxel_of(d, v)) return;
  const long b = bucket_of(d, hx[v.i], hy[v.i], hz[v.i]);
  if (b < 0) return;
  const int pos = offsets[b] + atomicAdd(cursor + b, 1);
  order[pos] = (int)v.i;
}

// weight of corner (cx, cy, cz) of a source at p, rounded to float as
// forwardApply writes it (HField3DUtils.txx:1116-1123): the product runs left
// to right, in double once a (1.0 - r) factor has entered it and in float
// before, so w110 = (rx*ry in float) * (1.0 - rz) and w111 = rx*ry*rz in float.
AW_D float corner_weight(float px, float py, float pz, int cx, int cy, int cz) {
  const int fx = ref_floor_f(px), fy = ref_floor_f(py), fz = ref_floor_f(pz);
  const float rx = fsub(px, __int2float_rn(fx)), ry = fsub(py, __int2float_rn(fy)),
              rz = fsub(pz, __int2float_rn(fz));
  if (cx && cy) {
    const float rxy = fmul(rx, ry);
    return cz ? fmul(rxy, rz) : __double2float_rn(dmul((double)rxy, dsub(1.0, (double)rz)));
  }
  const double ax = cx ? (double)rx : dsub(1.0, (double)rx);
  const double ay = cy ? (double)ry : dsub(1.0, (double)ry);
  const double az = cz ? (double)rz : dsub(1.0, (double)rz);
  return __double2float_rn(dmul(dmul(ax, ay), az));
}

// the eight corner weights (index dx + 2 dy + 4 dz) of the source at sorted
// position i
AW_D void store_weights(const int *__restrict__ order, int i, const float *__restrict__ hx,
                        const float *__restrict__ hy, const float *__restrict__ hz,
                        float *__restrict__ wts) {
  const int m = order[i];
  const float px = __ldg(hx + m), py = __ldg(hy + m), pz = __ldg(hz + m);
  float w[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) w[k] = corner_weight(px, py, pz, k & 1, (k >> 1) & 1, (k >> 2) & 1);
  float4 *o = reinterpret_cast<float4 *>(wts + (long)i * 8);
  o[0] = make_float4(w[0], w[1], w[2], w[3]);
  o[1] = make_float4(w[4], w[5], w[6], w[7]);
}

// Buckets of up to kSmallBucket sources are insertion-sorted by one thread
// (at most k(k-1)/2 moves); longer ones, which only a strongly compressing
// or collapsed map produces, by the whole CTA with a stable radix sort.
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSmallBucket = 64;

struct SortShared {
  int large[kSortThreads];         // block-local indices of the long buckets
  int nlarge;
  int base[256];                   // running digit offsets within the segment
  int wc[kSortWarps][256];         // per-warp digit counts of one 256-key tile
  int red[2][kSortWarps];
};

// Stable LSD radix sort of the distinct source indices order[s, e) by the
// whole CTA, 8 bits a pass over the keys' range, ping-ponging through
// tmp[s, e). Every key's position comes from counts (no atomic order), so
// the result is the ascending order whatever the input order; the work is
// O(k) per pass and at most four passes.
AW_D void block_radix_sort(int *__restrict__ order, int *__restrict__ tmp, int s, int e,
                           SortShared &sh) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int mn = INT_MAX, mx = INT_MIN;
  for (int i = s + tid; i < e; i += kSortThreads) {
    const int k = order[i];
    mn = min(mn, k);
    mx = max(mx, k);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if (lane == 0) {
    sh.red[0][warp] = mn;
    sh.red[1][warp] = mx;
  }
  __syncthreads();
  mn = sh.red[0][0];
  mx = sh.red[1][0];
  for (int w = 1; w < kSortWarps; ++w) {
    mn = min(mn, sh.red[0][w]);
    mx = max(mx, sh.red[1][w]);
  }
  __syncthreads();
  const unsigned range = (unsigned)mx - (unsigned)mn;
  const int passes = range ? (32 - __clz((int)range) + 7) / 8 : 0;
  int *src = order, *dst = tmp;
  const unsigned lt = (1u << lane) - 1u;
  for (int p = 0; p < passes; ++p) {
    const int shift = 8 * p;
    sh.base[tid] = 0;
    __syncthreads();
    for (int i = s + tid; i < e; i += kSortThreads)
      atomicAdd(&sh.base[(((unsigned)src[i] - (unsigned)mn) >> shift) & 255u], 1);
    __syncthreads();
    {  // exclusive scan of the 256 digit counts, one per thread
      const int c = sh.base[tid];
      int incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane == 31) sh.red[0][warp] = incl;
      __syncthreads();
      int off = 0;
      for (int w = 0; w < warp; ++w) off += sh.red[0][w];
      sh.base[tid] = off + incl - c;
      __syncthreads();
    }
    for (int t0 = s; t0 < e; t0 += kSortThreads) {
      const int i = t0 + tid;
      const bool valid = i < e;
      const int key = valid ? src[i] : 0;
      const int dg = valid ? (int)((((unsigned)key - (unsigned)mn) >> shift) & 255u) : 256;
#pragma unroll
      for (int w = 0; w < kSortWarps; ++w) sh.wc[w][tid] = 0;
      __syncthreads();
      const unsigned peers = __match_any_sync(0xffffffffu, dg);
      if (valid && (__ffs(peers) - 1) == lane) sh.wc[warp][dg] = __popc(peers);
      __syncthreads();
      if (valid) {
        int pre = sh.base[dg];
        for (int w = 0; w < warp; ++w) pre += sh.wc[w][dg];
        dst[s + pre + __popc(peers & lt)] = key;
      }
      __syncthreads();
      int add = 0;
#pragma unroll
      for (int w = 0; w < kSortWarps; ++w) add += sh.wc[w][tid];
      sh.base[tid] += add;
      __syncthreads();
    }
    int *t = src;
    src = dst;
    dst = t;
  }
  if (src != order) {
    for (int i = s + tid; i < e; i += kSortThreads) order[i] = src[i];
  }
  __syncthreads();
}

// Sorts every bucket by source index; with wts, then writes the eight corner
// weights of the source at every sorted position, once per sort: the gathers
// of every image splatted by the same h read them instead of the source's h
// and the weight arithmetic. One CTA per 256 buckets; tmp (the scatter's
// cursors, dead by now) holds at least n ints.
__global__ void __launch_bounds__(kSortThreads)
    k_bucket_sort(const int *__restrict__ offsets, int *__restrict__ order, int *__restrict__ tmp,
                  long next, const float *__restrict__ hx, const float *__restrict__ hy,
                  const float *__restrict__ hz, float *__restrict__ wts) {
  __shared__ SortShared sh;
  if (threadIdx.x == 0) sh.nlarge = 0;
  __syncthreads();
  const long b = (long)blockIdx.x * kSortThreads + threadIdx.x;
  if (b < next) {
    const int s = offsets[b], e = offsets[b + 1];
    if (e - s <= kSmallBucket) {
      for (int i = s + 1; i < e; ++i) {
        const int key = order[i];
        int j = i - 1;
        while (j >= s && order[j] > key) {
          order[j + 1] = order[j];
          --j;
        }
        order[j + 1] = key;
      }
      if (wts)
        for (int i = s; i < e; ++i) store_weights(order, i, hx, hy, hz, wts);
    } else {
      sh.large[atomicAdd(&sh.nlarge, 1)] = threadIdx.x;
    }
  }
  __syncthreads();
  const int nl = sh.nlarge;
  for (int q = 0; q < nl; ++q) {
    const long bb = (long)blockIdx.x * kSortThreads + sh.large[q];
    const int s = offsets[bb], e = offsets[bb + 1];
    block_radix_sort(order, tmp, s, e, sh);
    if (wts)
      for (int i = s + threadIdx.x; i < e; i += kSortThreads) store_weights(order, i, hx, hy, hz, wts);
  }
}

// every destination merges its eight candidate buckets in source order (the
// order forwardApply adds them). Buckets (dx = 1, dx = 0) of one (dy, dz) are
// adjacent: three offsets bound both.
//
// Fast path: the bucket of corner (dx, dy, dz) is the cell v - (dx, dy, dz),
// so its sources usually precede those of every corner with a smaller
// dx + 2 dy + 4 dz. The four (dy, dz) ranges are walked in that order
// (dz = 1 first, then dy = 1; dx = 1 before dx = 0 inside each); when every
// source index exceeds the one before it, this walk is the merged order and
// the sum is complete. A source out of order (a folding or strongly
// compressing map) sends the destination to the general eight-way merge,
// which starts the sum again. (Fetching all candidates up front and merging
// them in registers measured slower: the 16-way selection costs more issue
// slots than the dependent loads it saves.)
template <bool PRE>
__global__ void __launch_bounds__(kRowThreads)
    k_gather(const float *__restrict__ img, const float *__restrict__ hx,
             const float *__restrict__ hy, const float *__restrict__ hz, Dims d,
             const int *__restrict__ offsets, const int *__restrict__ order,
             const float *__restrict__ wts, float *__restrict__ out, float bg) {
  Voxel v;
  if (!voxel_of(d, v)) return;
  int pos[8], end[8], cur[8];
  const long sy = d.nx + 1, sz = (long)(d.nx + 1) * (d.ny + 1);
  // bucket k = (dz, dy, dx) bits; source in bucket b contributes corner
  // (dx, dy, dz) to this voxel
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int dy = r & 1, dz = r >> 1;
    const long b1 = (long)(v.z - dz + 1) * sz + (long)(v.y - dy + 1) * sy + v.x;  // dx = 1
    const int o0 = __ldg(offsets + b1), o1 = __ldg(offsets + b1 + 1), o2 = __ldg(offsets + b1 + 2);
    pos[2 * r + 1] = o0;
    end[2 * r + 1] = o1;
    pos[2 * r] = o1;
    end[2 * r] = o2;
  }
  float acc = bg;
  int prev = -1;
  bool ordered = true;
#pragma unroll
  for (int r = 3; r >= 0; --r) {
    const int dy = r & 1, dz = r >> 1;
    for (int p = pos[2 * r + 1]; ordered && p < end[2 * r]; ++p) {
      const int m = __ldg(order + p);
      if (m <= prev) {
        ordered = false;
        break;
      }
      prev = m;
      const int dx = p < end[2 * r + 1] ? 1 : 0;
      const float w = PRE ? __ldg(wts + (long)p * 8 + (dx + 2 * dy + 4 * dz))
                          : corner_weight(hx[m], hy[m], hz[m], dx, dy, dz);
      acc = fadd(acc, fmul(w, img[m]));
    }
  }
  if (ordered) {
    out[v.i] = acc;
    return;
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) cur[k] = pos[k] < end[k] ? order[pos[k]] : INT_MAX;
  acc = bg;
  while (true) {
    int m = INT_MAX, sel = -1;
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (cur[k] < m) {
        m = cur[k];
        sel = k;
      }
    if (sel < 0) break;
    int at = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (k == sel) at = pos[k];
    const float w = PRE ? __ldg(wts + (long)at * 8 + sel)
                        : corner_weight(hx[m], hy[m], hz[m], sel & 1, (sel >> 1) & 1,
                                        (sel >> 2) & 1);
    acc = fadd(acc, fmul(w, img[m]));
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (k == sel) {
        ++pos[k];
        cur[k] = pos[k] < end[k] ? order[pos[k]] : INT_MAX;
      }
    }
  }
  out[v.i] = acc;
}

}  // namespace

size_t splat_scratch_bytes(const Dims &d, bool weights) {
  const long next = (long)(d.nx + 1) * (d.ny + 1) * (d.nz + 1);
  const long nb = (next + kScanBlock - 1) / kScanBlock;
  return align256(sizeof(int) * (next + 1)) + align256(sizeof(int) * next) +
         align256(sizeof(int) * d.n()) + align256(sizeof(int) * nb) +
         (weights ? align256(sizeof(float) * 8 * d.n()) : 0);
}

void splat_work_bind(SplatWork *w, const Dims &d, void *scratch, bool weights) {
  char *p = static_cast<char *>(scratch);
  w->d = d;
  w->next = (long)(d.nx + 1) * (d.ny + 1) * (d.nz + 1);
  w->nblocks = (int)((w->next + kScanBlock - 1) / kScanBlock);
  w->offsets = reinterpret_cast<int *>(p);
  p += align256(sizeof(int) * (w->next + 1));
  w->cursor = reinterpret_cast<int *>(p);
  p += align256(sizeof(int) * w->next);
  w->order = reinterpret_cast<int *>(p);
  p += align256(sizeof(int) * d.n());
  w->blocksums = reinterpret_cast<int *>(p);
  p += align256(sizeof(int) * w->nblocks);
  w->wts = weights ? reinterpret_cast<float *>(p) : nullptr;
}

cudaError_t splat_sort(const SplatWork &w, const float *hx, const float *hy, const float *hz,
                       cudaStream_t s) {
  const Dims d = w.d;
  cudaError_t e;
  if ((e = cudaMemsetAsync(w.offsets, 0, sizeof(int) * (w.next + 1), s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(w.cursor, 0, sizeof(int) * w.next, s)) != cudaSuccess) return e;
  k_count<<<row_grid(d), kRowThreads, 0, s>>>(hx, hy, hz, d, w.offsets);
  k_scan_reduce<<<w.nblocks, kScanThreads, 0, s>>>(w.offsets, w.next, w.blocksums);
  k_scan_blocksums<<<1, kScanThreads, 0, s>>>(w.blocksums, w.nblocks);
  k_scan_apply<<<w.nblocks, kScanThreads, 0, s>>>(w.offsets, w.next, w.blocksums);
  k_scatter<<<row_grid(d), kRowThreads, 0, s>>>(hx, hy, hz, d, w.offsets, w.cursor, w.order);
  k_bucket_sort<<<(int)((w.next + kSortThreads - 1) / kSortThreads), kSortThreads, 0, s>>>(
      w.offsets, w.order, w.cursor, w.next, hx, hy, hz, w.wts);
  return cudaGetLastError();
}

cudaError_t splat_gather(const SplatWork &w, const float *img, const float *hx, const float *hy,
                         const float *hz, float *out, float bg, cudaStream_t s) {
  const Dims d = w.d;
  if (w.wts)
    k_gather<true><<<row_grid(d), kRowThreads, 0, s>>>(img, hx, hy, hz, d, w.offsets, w.order,
                                                       w.wts, out, bg);
  else
    k_gather<false><<<row_grid(d), kRowThreads, 0, s>>>(img, hx, hy, hz, d, w.offsets, w.order,
                                                        nullptr, out, bg);
  return cudaGetLastError();
}

cudaError_t splat(const SplatWork &w, const float *img, const float *hx, const float *hy,
                  const float *hz, float *out, float bg, cudaStream_t s) {
  const cudaError_t e = splat_sort(w, hx, hy, hz, s);
  return e != cudaSuccess ? e : splat_gather(w, img, hx, hy, hz, out, bg, s);
}

}  // namespace aw
