// greedy.cu — one greedy-fluid iteration on the device, GreedyIteratorGPU /
// GreedyIteratorCPU::Iterate (Algorithms/Greedy/GreedyIteratorCPU.cxx:99-138)
// restated as six stream-ordered launches with no host synchronisation:
//
//   1 force_prep     I0(h) and the energy partial sums of (I1 - I0(h))^2
//   2 energy_final   deterministic block-ordered sum -> energy history,
//                    optional AutoStepReduce (GreedyDeformationData.cxx:176-183)
//   3 xy-forward     body force grad(I0(h)) * (I1 - I0(h)) fused into the FFT
//   4 z-solve        L^-1 per wavenumber
//   5 xy-inverse     v = K f
//   6 update         h' = h(x + eps*v/sp) [PARTIAL_ID], optionally
//                    hinv' = hinv - (eps*v)(hinv)/sp [PARTIAL_ZERO]
//
// plus, at a step-size update (iteration 0 of a scale level,
// GreedyWarp.txx:99), a max|v| reduction and eps = MaxPert / max|v| computed
// on the device (GreedyIteratorCPU.cxx:125-131). On the register-FFT path,
// iterations without a step update or an inverse field run 5 and 6 as one
// kernel (k_xy_inv_compose, fluid_fast.cu): five launches.
#include <algorithm>
#include <climits>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "bulk.cuh"
#include "greedy.cuh"
#include "interp.cuh"
#include "tma_host.cuh"

namespace aw {

namespace {

constexpr int kThreads = 256;

// Rows per force-prep block: each block sums the energy of kPrepRows rows, so
// the fixed-order final sum has few partials to read.
constexpr int kPrepRows = 2;

// I0(h) and the energy partials. With AFFINE the subject image lives on its
// own grid di and h is in template voxels: the sample point is the atlas map
// of h (atlas_point, interp.cuh). FAST: the float-tree interpolation.
template <bool AFFINE, bool FAST>
__global__ void __launch_bounds__(kRowThreads)
    k_force_prep(const float *__restrict__ I0, const float *__restrict__ I1,
                 const float *__restrict__ hx, const float *__restrict__ hy,
                 const float *__restrict__ hz, float *__restrict__ idef, double *__restrict__ partials,
                 Dims d, Dims di, AtlasMap am) {
  const int x = blockIdx.x * kRowThreads + threadIdx.x;
  const int z = blockIdx.z;
  double e = 0.0;
  if (x < d.nx) {
    const int y0 = blockIdx.y * kPrepRows;
    const int y1 = min(y0 + kPrepRows, d.ny);
    for (int y = y0; y < y1; ++y) {
      const long i = ((long)z * d.ny + y) * d.nx + x;
      double px = (double)hx[i], py = (double)hy[i], pz = (double)hz[i];
      if (AFFINE) atlas_point(am, px, py, pz);
      const float v = trilerp_scalar<FAST>(I0, AFFINE ? di : d, px, py, pz, 0.0f);
      idef[i] = v;
      const float r = -fsub(v, I1[i]);
      e += (double)r * (double)r;
    }
  }
  __shared__ double ws[kRowThreads / 32];
  e = warp_sum(e);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < kRowThreads / 32 ? ws[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0)
      partials[((long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = t;
  }
}

inline dim3 prep_grid(const Dims &d) {
  return dim3((unsigned)((d.nx + kRowThreads - 1) / kRowThreads),
              (unsigned)((d.ny + kPrepRows - 1) / kPrepRows), (unsigned)d.nz);
}

// Fixed-order reduction of the block partials, so the energy is bitwise
// reproducible run to run: four independent thread-strided sums per thread,
// combined in a fixed order, then the warp and block trees.
constexpr int kFinalThreads = 1024;

__global__ void __launch_bounds__(kFinalThreads)
    k_energy_final(const double *__restrict__ partials, int nparts, double scale,
                   GreedyDevState st, int auto_reduce) {
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  const int step = 4 * kFinalThreads;
  int i = threadIdx.x;
  for (; i + 3 * kFinalThreads < nparts; i += step) {
    a0 += partials[i];
    a1 += partials[i + kFinalThreads];
    a2 += partials[i + 2 * kFinalThreads];
    a3 += partials[i + 3 * kFinalThreads];
  }
  for (; i < nparts; i += kFinalThreads) a0 += partials[i];
  double t = (a0 + a1) + (a2 + a3);
  __shared__ double ws[kFinalThreads / 32];
  t = warp_sum(t);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x < 32) {
    double u = ws[threadIdx.x];
    u = warp_sum(u);
    if (threadIdx.x == 0) {
      const double e = u * scale;
      const int k = *st.count;
      if (auto_reduce && k > 0) {
        const double prev = st.energy[(k - 1) % st.cap];
        if ((float)e - (float)prev > 0.0f) *st.step = *st.step / 2.0f;
      }
      st.energy[k % st.cap] = e;
      *st.count = k + 1;
    }
  }
}

__global__ void __launch_bounds__(kThreads)
    k_max_norm(const float *__restrict__ vx, const float *__restrict__ vy,
               const float *__restrict__ vz, long n, unsigned *__restrict__ maxbits) {
  float m = 0.0f;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float a = vx[i], b = vy[i], c = vz[i];
    const float l = sqrtf(fadd(fadd(fmul(a, a), fmul(b, b)), fmul(c, c)));
    m = fmaxf(m, l);
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) atomicMax(maxbits, __float_as_uint(m));
}

__global__ void k_set_step(const unsigned *__restrict__ maxbits, float max_pert, float *step) {
  *step = fdiv(max_pert, __uint_as_float(*maxbits));
}

// composeHV(h, eps*v, PARTIAL_ID) and, when hinv is given,
// composeVHInv(eps*v, hinv, PARTIAL_ZERO) — GreedyIteratorCPU::updateDeformation
// (GreedyIteratorCPU.cxx:83-95), both from one read of v.
// composeHV(h, eps*v, PARTIAL_ID) and, when hinv is given,
// composeVHInv(eps*v, hinv, PARTIAL_ZERO) — GreedyIteratorCPU::updateDeformation
// (GreedyIteratorCPU.cxx:83-95), both from one read of v. q[] divides by the
// float spacing (a multiply when it is a power of two).
struct UpdateArgs {
  const float *hx, *hy, *hz, *vx, *vy, *vz;
  float *ox, *oy, *oz;
  const float *gx, *gy, *gz;  // hinv (null: no inverse)
  float *qx, *qy, *qz;        // hinv'
  DivF q0, q1, q2;
};

__global__ void __launch_bounds__(kRowThreads)
    k_update(UpdateArgs a, Dims d, const float *__restrict__ step_ptr) {
  Voxel vox;
  if (!voxel_of(d, vox)) return;
  const long i = vox.i;
  const int x = vox.x, y = vox.y, z = vox.z;
  const float eps = *step_ptr;
  const float px = fadd(__int2float_rn(x), fdivq(fmul(a.vx[i], eps), a.q0));
  const float py = fadd(__int2float_rn(y), fdivq(fmul(a.vy[i], eps), a.q1));
  const float pz = fadd(__int2float_rn(z), fdivq(fmul(a.vz[i], eps), a.q2));
  float rx, ry, rz;
  trilerp_vector(a.hx, a.hy, a.hz, d, px, py, pz, BG_PARTIAL_ID, 1.0f, rx, ry, rz);
  a.ox[i] = rx;
  a.oy[i] = ry;
  a.oz[i] = rz;
  if (a.gx) {
    const float g0 = a.gx[i], g1 = a.gy[i], g2 = a.gz[i];
    float b0, b1, b2;
    trilerp_vector(a.vx, a.vy, a.vz, d, g0, g1, g2, BG_PARTIAL_ZERO, eps, b0, b1, b2);
    // b / -s = -(b / s) exactly in round-to-nearest
    a.qx[i] = fadd(-fdivq(b0, a.q0), g0);
    a.qy[i] = fadd(-fdivq(b1, a.q1), g1);
    a.qz[i] = fadd(-fdivq(b2, a.q2), g2);
  }
}

// tuning input: h = identity, v = 0.4 in every component
__global__ void __launch_bounds__(kRowThreads)
    k_fill_identity_shift(float *__restrict__ hx, float *__restrict__ hy, float *__restrict__ hz,
                          float *__restrict__ v, Dims d) {
  Voxel p;
  if (!voxel_of(d, p)) return;
  const long n = d.n();
  hx[p.i] = (float)p.x;
  hy[p.i] = (float)p.y;
  hz[p.i] = (float)p.z;
  v[p.i] = 0.4f;
  v[n + p.i] = 0.4f;
  v[2 * n + p.i] = 0.4f;
}

// The update with h staged in shared memory. The step keeps eps*v/sp within
// MaxPert of a voxel at the iteration that sets it, so the eight corners a
// voxel reads lie within one voxel of it: a CTA owns a 32 x TY x TZ tile and
// the three components of h over the tile plus a one-voxel halo arrive by
// TMA tensor loads (x from x0 - 4, so the box starts on a 16-byte boundary:
// 40 x (TY+2) x (TZ+2) floats each). Corners inside the volume and the box
// are read from shared memory with trilerp_vector's own arithmetic (corner
// order, double weights, lerp tree); any other voxel (a corner outside the
// volume, a larger step) takes trilerp_vector from global memory. No inverse
// field. The tile shape is chosen per grid by timing (tune_update_tile).
constexpr int kUTX = 32, kUBX = 40;
template <int TY, int TZ>
struct UTile {
  static constexpr int BY = TY + 2, BZ = TZ + 2, BOX = kUBX * BY * BZ;
};
// candidate tile shapes (TY, TZ); index 0 is the default
constexpr int kNumTiles = 4;
constexpr int kTileTY[kNumTiles] = {8, 4, 8, 16}, kTileTZ[kNumTiles] = {4, 8, 8, 2};

struct HMaps {
  CUtensorMap m[3];
};

template <int TY, int TZ>
__global__ void __launch_bounds__(kUTX * TY, 1024 / (kUTX * TY))
    k_update_tiled(const __grid_constant__ HMaps maps, UpdateArgs a, Dims d,
                   const float *__restrict__ step_ptr, int *status) {
  using U = UTile<TY, TZ>;
  constexpr int kUTY = TY, kUTZ = TZ, kUBY = U::BY, kUBZ = U::BZ, kUBox = U::BOX;
  __shared__ __align__(128) float sh[3][kUBox];
  __shared__ uint64_t mbar;
  const int tx = (d.nx + kUTX - 1) / kUTX, ty = (d.ny + kUTY - 1) / kUTY;
  int t = blockIdx.x;
  const int x0 = (t % tx) * kUTX;
  t /= tx;
  const int y0 = (t % ty) * kUTY;
  const int z0 = (t / ty) * kUTZ;
  const int bx0 = x0 - 4, by0 = y0 - 1, bz0 = z0 - 1;
  if (threadIdx.x == 0) {
    mbar_init(&mbar, 1);
    mbar_expect_tx(&mbar, (uint32_t)(3 * kUBox * sizeof(float)));
    for (int c = 0; c < 3; ++c) tma_load_3d(sh[c], &maps.m[c], bx0, by0, bz0, &mbar);
  }
  __syncthreads();
  const int x = x0 + (threadIdx.x % kUTX), y = y0 + (threadIdx.x / kUTX);
  const bool col = x < d.nx && y < d.ny;
  // v of the thread's four voxels first: independent of the staged h, so
  // these loads overlap the tile's arrival
  const float eps = *step_ptr;
  float vx4[kUTZ], vy4[kUTZ], vz4[kUTZ];
#pragma unroll
  for (int zz = 0; zz < kUTZ; ++zz) {
    const long i = d.idx(x, y, z0 + zz);
    const bool ok = col && z0 + zz < d.nz;
    vx4[zz] = ok ? __ldg(a.vx + i) : 0.0f;
    vy4[zz] = ok ? __ldg(a.vy + i) : 0.0f;
    vz4[zz] = ok ? __ldg(a.vz + i) : 0.0f;
  }
  const bool staged = mbar_wait(&mbar, 0, status);
  if (!col) return;
#pragma unroll
  for (int zz = 0; zz < kUTZ; ++zz) {
    const int z = z0 + zz;
    if (z >= d.nz) break;
    const long i = d.idx(x, y, z);
    const float px = fadd(__int2float_rn(x), fdivq(fmul(vx4[zz], eps), a.q0));
    const float py = fadd(__int2float_rn(y), fdivq(fmul(vy4[zz], eps), a.q1));
    const float pz = fadd(__int2float_rn(z), fdivq(fmul(vz4[zz], eps), a.q2));
    const int fx = ref_floor_f(px), fy = ref_floor_f(py), fz = ref_floor_f(pz);
    const bool fast = staged && fx >= 0 && fx + 1 < d.nx && fy >= 0 && fy + 1 < d.ny &&
                      fz >= 0 && fz + 1 < d.nz && fx >= bx0 && fx + 1 < bx0 + kUBX &&
                      fy >= by0 && fy + 1 < by0 + kUBY && fz >= bz0 && fz + 1 < bz0 + kUBZ;
    float rx, ry, rz;
    if (fast) {
      const double tt = (double)fsub(px, __int2float_rn(fx));
      const double uu = (double)fsub(py, __int2float_rn(fy));
      const double vv = (double)fsub(pz, __int2float_rn(fz));
      const double omt = dsub(1.0, tt), omu = dsub(1.0, uu), omv = dsub(1.0, vv);
      const int b = ((fz - bz0) * kUBY + (fy - by0)) * kUBX + (fx - bx0);
      constexpr int sy = kUBX, sz = kUBX * kUBY;
      const int off[8] = {b, b + 1, b + sy + 1, b + sy, b + sy + sz, b + sy + sz + 1, b + sz + 1,
                          b + sz};
      float cx[8], cy[8], cz[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        cx[c] = sh[0][off[c]];
        cy[c] = sh[1][off[c]];
        cz[c] = sh[2][off[c]];
      }
      rx = __double2float_rn(lerp_tree(cx, tt, uu, vv, omt, omu, omv));
      ry = __double2float_rn(lerp_tree(cy, tt, uu, vv, omt, omu, omv));
      rz = __double2float_rn(lerp_tree(cz, tt, uu, vv, omt, omu, omv));
    } else {
      trilerp_vector(a.hx, a.hy, a.hz, d, px, py, pz, BG_PARTIAL_ID, 1.0f, rx, ry, rz);
    }
    a.ox[i] = rx;
    a.oy[i] = ry;
    a.oz[i] = rz;
  }
}

// tensor maps of h planes, one per (pointer, grid), encoded on first use
struct HMapCache {
  // (plane, nx, ny, nz, box x, box y, box z) -> map
  std::map<std::tuple<const float *, int, int, int, int, int, int>, CUtensorMap> maps;
};

// tensor map of one float plane of the handle's grid with a bx x by x bz box
bool plane_map(GreedyCtx *g, const float *p, int bx, int by, int bz, CUtensorMap *out) {
  if (!g->hmaps) return false;
  auto *cache = static_cast<HMapCache *>(g->hmaps);
  const Dims d = g->d;
  const auto key = std::make_tuple(p, d.nx, d.ny, d.nz, bx, by, bz);
  auto it = cache->maps.find(key);
  if (it != cache->maps.end()) {
    *out = it->second;
    return true;
  }
  const PFN_cuTensorMapEncodeTiled encode = tensor_map_encoder();
  if (!encode || reinterpret_cast<uintptr_t>(p) % 16 || d.nx % 4 || d.nx < bx || d.ny < by ||
      d.nz < bz)
    return false;
  CUtensorMap m;
  const cuuint64_t dims[3] = {(cuuint64_t)d.nx, (cuuint64_t)d.ny, (cuuint64_t)d.nz};
  const cuuint64_t strides[2] = {(cuuint64_t)d.nx * 4, (cuuint64_t)d.nx * d.ny * 4};
  const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz};
  const cuuint32_t estr[3] = {1, 1, 1};
  if (encode(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(p), dims, strides, box,
             estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  cache->maps[key] = m;
  *out = m;
  return true;
}

bool h_map(GreedyCtx *g, const float *p, int tile, CUtensorMap *out) {
  return plane_map(g, p, kUBX, kTileTY[tile] + 2, kTileTZ[tile] + 2, out);
}

template <int TY, int TZ>
void launch_tiled(const HMaps &maps, const UpdateArgs &a, const Dims &d, const float *step,
                  int *status, cudaStream_t s) {
  const unsigned tiles = (unsigned)(((d.nx + kUTX - 1) / kUTX) * ((d.ny + TY - 1) / TY) *
                                    ((d.nz + TZ - 1) / TZ));
  k_update_tiled<TY, TZ><<<tiles, kUTX * TY, 0, s>>>(maps, a, d, step, status);
}

// the staged update with tile shape `tile`; false when h cannot be staged
// (grid or alignment), so the caller takes the global-gather kernel
bool launch_update_tiled(GreedyCtx *g, int tile, const UpdateArgs &a, const float *const h[3],
                         cudaStream_t s) {
  HMaps maps;
  for (int c = 0; c < 3; ++c)
    if (!h_map(g, h[c], tile, &maps.m[c])) return false;
  const Dims d = g->d;
  int *st = g->plan.status;
  switch (tile) {
    case 0: launch_tiled<8, 4>(maps, a, d, g->st.step, st, s); break;
    case 1: launch_tiled<4, 8>(maps, a, d, g->st.step, st, s); break;
    case 2: launch_tiled<8, 8>(maps, a, d, g->st.step, st, s); break;
    default: launch_tiled<16, 2>(maps, a, d, g->st.step, st, s); break;
  }
  return true;
}

// tuned tile per (grid, device), kept for the process
std::mutex g_tile_mu;
std::map<std::tuple<int, int, int, int>, int> g_tile;

// Times every tile shape on an update of the identity by a field of 0.4
// voxel (all staged reads, the common case), 3 launches after 1 untimed
// each, and keeps the fastest; a grid the staged kernel cannot take keeps 0.
void tune_update_tile(GreedyCtx *g) {
  g->utile = 0;
  const Dims d = g->d;
  const auto key = std::make_tuple(d.nx, d.ny, d.nz, g->plan.device);
  {
    std::lock_guard<std::mutex> lock(g_tile_mu);
    auto it = g_tile.find(key);
    if (it != g_tile.end()) {
      g->utile = it->second;
      return;
    }
  }
  const long n = d.n();
  float *buf = nullptr;
  float *step = nullptr;
  // no room for the tuning scratch: keep the default shape (and clear the
  // allocation error, which is not the handle's)
  if (cudaMalloc(&buf, sizeof(float) * 6 * n) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  if (cudaMalloc(&step, sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(buf);
    return;
  }
  const float one = 1.0f;
  cudaMemcpy(step, &one, sizeof(float), cudaMemcpyHostToDevice);
  float *h[3] = {buf, buf + n, buf + 2 * n}, *o[3] = {buf + 3 * n, buf + 4 * n, buf + 5 * n};
  k_fill_identity_shift<<<row_grid(d), kRowThreads>>>(h[0], h[1], h[2], g->vbuf, d);
  const UpdateArgs a{h[0], h[1], h[2], g->vbuf, g->vbuf + n, g->vbuf + 2 * n, o[0], o[1], o[2],
                     nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                     make_divf((float)g->sp.x), make_divf((float)g->sp.y),
                     make_divf((float)g->sp.z)};
  const float *hc[3] = {h[0], h[1], h[2]};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int pick = 0;
  bool any = false;
  float *saved_step = g->st.step;
  g->st.step = step;
  for (int tile = 0; tile < kNumTiles; ++tile) {
    if (!launch_update_tiled(g, tile, a, hc, 0)) break;
    any = true;
    cudaEventRecord(e0, 0);
    for (int r = 0; r < 3; ++r) launch_update_tiled(g, tile, a, hc, 0);
    cudaEventRecord(e1, 0);
    float ms = 0.f;
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
      break;
    if (ms < best) {
      best = ms;
      pick = tile;
    }
  }
  g->st.step = saved_step;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(step);
  cudaFree(buf);
  // the tensor maps of the scratch planes go with them
  static_cast<HMapCache *>(g->hmaps)->maps.clear();
  if (cudaGetLastError() != cudaSuccess || !any) return;
  g->utile = pick;
  std::lock_guard<std::mutex> lock(g_tile_mu);
  g_tile[key] = pick;
}

#define AW_TRY(x)                         \
  do {                                    \
    cudaError_t _e = (x);                 \
    if (_e != cudaSuccess) return _e;     \
  } while (0)

}  // namespace

int greedy_create(GreedyCtx *g, int nx, int ny, int nz, double spx, double spy, double spz,
                  float alpha, float beta, float gamma, float max_pert, int history_cap) {
  std::memset(g, 0, sizeof(*g));
  const int rc = fluid_plan_create(&g->plan, nx, ny, nz, spx, spy, spz, alpha, beta, gamma);
  if (rc) return rc;
  g->d = g->plan.d;
  g->di = g->d;
  g->sp = g->plan.sp;
  g->max_pert = max_pert;
  const long n = g->d.n();
  {
    const dim3 gr = prep_grid(g->d);
    g->nparts = (int)(gr.x * gr.y * gr.z);
  }
  g->sms = 148;
  cudaDeviceGetAttribute(&g->sms, cudaDevAttrMultiProcessorCount, g->plan.device);
  g->st.cap = history_cap > 0 ? history_cap : 4096;
  if (cudaMalloc(&g->idef, sizeof(float) * n) != cudaSuccess) return 3;
  if (cudaMalloc(&g->vbuf, sizeof(float) * 3 * n) != cudaSuccess) return 3;
  if (cudaMalloc(&g->partials, sizeof(double) * g->nparts) != cudaSuccess) return 3;
  if (cudaMalloc(&g->st.energy, sizeof(double) * g->st.cap) != cudaSuccess) return 3;
  if (cudaMalloc(&g->scalars, 64) != cudaSuccess) return 3;
  cudaMemset(g->scalars, 0, 64);
  g->st.step = reinterpret_cast<float *>(g->scalars);
  g->st.count = reinterpret_cast<int *>(g->scalars + 4);
  g->maxbits = reinterpret_cast<unsigned *>(g->scalars + 8);
  g->hmaps = new HMapCache();
  if (cudaStreamCreateWithFlags(&g->aux, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&g->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&g->ev_join, cudaEventDisableTiming) != cudaSuccess)
    return 4;
  if (cudaGetLastError() != cudaSuccess) return 4;
  tune_update_tile(g);
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

void greedy_destroy(GreedyCtx *g) {
  fluid_plan_destroy(&g->plan);
  if (g->idef) cudaFree(g->idef);
  if (g->vbuf) cudaFree(g->vbuf);
  if (g->partials) cudaFree(g->partials);
  if (g->st.energy) cudaFree(g->st.energy);
  if (g->scalars) cudaFree(g->scalars);
  if (g->aux) cudaStreamDestroy(g->aux);
  if (g->ev_fork) cudaEventDestroy(g->ev_fork);
  if (g->ev_join) cudaEventDestroy(g->ev_join);
  delete static_cast<HMapCache *>(g->hmaps);
  std::memset(g, 0, sizeof(*g));
}

cudaError_t greedy_stage(GreedyCtx *g, int stage, const float *I0, const float *I1,
                         const float *const h[3], float *const h_out[3], const float *const hinv[3],
                         float *const hinv_out[3], int auto_reduce, int solve_inverse,
                         cudaStream_t s) {
  const Dims d = g->d;
  const long n = d.n();
  float *v[3] = {g->vbuf, g->vbuf + n, g->vbuf + 2 * n};
  switch (stage) {
    case kStageForcePrep: {
      // (staging the box of I0 a tile's h points into measured slower here:
      // the h load, the block's range reduction and the box's arrival run
      // one after another, against eight L2-resident gathers per voxel)
      const dim3 pg = prep_grid(d);
      if (g->am.on && g->fast_interp)
        k_force_prep<true, true><<<pg, kRowThreads, 0, s>>>(I0, I1, h[0], h[1], h[2], g->idef,
                                                            g->partials, d, g->di, g->am);
      else if (g->am.on)
        k_force_prep<true, false><<<pg, kRowThreads, 0, s>>>(I0, I1, h[0], h[1], h[2], g->idef,
                                                             g->partials, d, g->di, g->am);
      else if (g->fast_interp)
        k_force_prep<false, true><<<pg, kRowThreads, 0, s>>>(I0, I1, h[0], h[1], h[2], g->idef,
                                                             g->partials, d, d, g->am);
      else
        k_force_prep<false, false><<<pg, kRowThreads, 0, s>>>(I0, I1, h[0], h[1], h[2], g->idef,
                                                              g->partials, d, d, g->am);
      return cudaGetLastError();
    }
    case kStageEnergy: {
      const double spprod = g->sp.x * g->sp.y * g->sp.z;
      k_energy_final<<<1, kFinalThreads, 0, s>>>(g->partials, g->nparts, spprod, g->st,
                                                 auto_reduce);
      return cudaGetLastError();
    }
    case kStageXYForward:
      return fluid_forward_force(g->plan, g->idef, I1, 1, s);
    case kStageZSolve:
      return fluid_solve(g->plan, solve_inverse, s);
    case kStageXYInverse:
      return fluid_inverse_store(g->plan, v[0], v[1], v[2], s);
    case kStageMaxNorm: {
      AW_TRY(cudaMemsetAsync(g->maxbits, 0, sizeof(unsigned), s));
      k_max_norm<<<g->sms * 4, kThreads, 0, s>>>(v[0], v[1], v[2], n, g->maxbits);
      AW_TRY(cudaGetLastError());
      k_set_step<<<1, 1, 0, s>>>(g->maxbits, g->max_pert, g->st.step);
      return cudaGetLastError();
    }
    case kStageUpdate: {
      const bool inv = hinv && hinv[0] && hinv_out && hinv_out[0];
      const UpdateArgs a{h[0], h[1], h[2], v[0], v[1], v[2], h_out[0], h_out[1], h_out[2],
                         inv ? hinv[0] : nullptr, inv ? hinv[1] : nullptr,
                         inv ? hinv[2] : nullptr, inv ? hinv_out[0] : nullptr,
                         inv ? hinv_out[1] : nullptr, inv ? hinv_out[2] : nullptr,
                         make_divf((float)g->sp.x), make_divf((float)g->sp.y),
                         make_divf((float)g->sp.z)};
      if (inv || g->no_staged_update || !launch_update_tiled(g, g->utile, a, h, s))
        k_update<<<row_grid(d), kRowThreads, 0, s>>>(a, d, g->st.step);
      return cudaGetLastError();
    }
    case kStageInvCompose: {
      // grids the fused kernel does not take run the two stages it replaces
      if (!g->plan.fast) {
        AW_TRY(greedy_stage(g, kStageXYInverse, I0, I1, h, h_out, hinv, hinv_out, auto_reduce,
                            solve_inverse, s));
        return greedy_stage(g, kStageUpdate, I0, I1, h, h_out, nullptr, nullptr, auto_reduce,
                            solve_inverse, s);
      }
      const ComposeArgs a{h[0], h[1], h[2], h_out[0], h_out[1], h_out[2], g->st.step,
                          make_divf((float)g->sp.x), make_divf((float)g->sp.y),
                          make_divf((float)g->sp.z), g->fast_interp};
      return fluid_inverse_compose(g->plan, a, s);
    }
  }
  return cudaErrorInvalidValue;
}

// The energy sum runs on a side stream, concurrently with the transforms;
// it joins before the step-size stage and the update, the two readers and
// writers of the step it may reduce (AutoStepReduce).
//
// Without a step-size update or an inverse field, on the register-FFT path,
// the inverse transform and the update are one kernel (kStageInvCompose):
// v = K f stays in shared memory. The step update needs max |v| over the
// whole field before any voxel moves, and the inverse field gathers v at
// h^-1(x) anywhere in the volume, so those iterations store v.
cudaError_t greedy_iterate(GreedyCtx *g, const float *I0, const float *I1, const float *const h[3],
                           float *const h_out[3], const float *const hinv[3],
                           float *const hinv_out[3], int update_step, int auto_reduce,
                           cudaStream_t s) {
  const bool inv = hinv && hinv[0] && hinv_out && hinv_out[0];
  const bool fuse = !update_step && !inv && !g->no_fused_update && g->plan.fast;
  AW_TRY(greedy_stage(g, kStageForcePrep, I0, I1, h, h_out, hinv, hinv_out, auto_reduce, 1, s));
  AW_TRY(cudaEventRecord(g->ev_fork, s));
  AW_TRY(cudaStreamWaitEvent(g->aux, g->ev_fork, 0));
  AW_TRY(greedy_stage(g, kStageEnergy, I0, I1, h, h_out, hinv, hinv_out, auto_reduce, 1, g->aux));
  AW_TRY(cudaEventRecord(g->ev_join, g->aux));
  AW_TRY(greedy_stage(g, kStageXYForward, I0, I1, h, h_out, hinv, hinv_out, auto_reduce, 1, s));
  AW_TRY(greedy_stage(g, kStageZSolve, I0, I1, h, h_out, hinv, hinv_out, auto_reduce, 1, s));
  if (fuse) {
    AW_TRY(cudaStreamWaitEvent(s, g->ev_join, 0));
    return greedy_stage(g, kStageInvCompose, I0, I1, h, h_out, nullptr, nullptr, auto_reduce, 1,
                        s);
  }
  AW_TRY(greedy_stage(g, kStageXYInverse, I0, I1, h, h_out, hinv, hinv_out, auto_reduce, 1, s));
  AW_TRY(cudaStreamWaitEvent(s, g->ev_join, 0));
  if (update_step)
    AW_TRY(greedy_stage(g, kStageMaxNorm, I0, I1, h, h_out, hinv, hinv_out, auto_reduce, 1, s));
  return greedy_stage(g, kStageUpdate, I0, I1, h, h_out, hinv, hinv_out, auto_reduce, 1, s);
}

}  // namespace aw
