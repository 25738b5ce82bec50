// fluid_fast.cu — the fluid-operator kernels for power-of-two axes
// (16..256), with register-resident line FFTs (fft_reg.cuh).
//
// Same three passes as fluid.cu (xy-forward, z-solve, xy-inverse) and the
// same arithmetic definition; the layout of work differs:
//  * xy kernels: one 256-thread CTA per (z-slab, component) holding only the
//    slab's half spectrum in shared memory (66.5 KB at 128 x 128, three
//    CTAs per SM). x-lines are row pairs packed as one complex line; the
//    kx = 0 and kx = nx/2 columns (real after the x-transform) are packed into
//    one complex y-line, so a 128 x 128 slab is exactly 64 x-lines + 64
//    y-lines. Every line's four-step exchange runs in place in the slab slots
//    that line owns, so the CTA needs no scratch. Lines that share a
//    half-warp are placed 8 banks apart, which with the exchange swizzle
//    makes every shared-memory access conflict-free. The finished slab leaves
//    (forward) or arrives (inverse) as one bulk copy.
//  * z kernel: one CTA per 16 consecutive (ky,kx) columns, all three
//    components. The [nz x 16] complex tiles arrive by TMA tensor copies in
//    the 128-byte swizzled layout (one 128-byte row per kz), each z-line
//    transforms in place in its tile column, the 3x3 solve runs in the
//    tiles, and TMA tensor stores write them back.
#include <cooperative_groups.h>
#include <cstdint>

#include "bulk.cuh"
#include "fft_reg.cuh"
#include "fluid.cuh"
#include "fluid_fast.cuh"

namespace aw {

namespace cg = cooperative_groups;

namespace {

constexpr int kXYThreads = 256;
constexpr int kXYWarps = kXYThreads / 32;
// columns per z tile: 16 (one 128-byte row per kz, 128-byte swizzle) or 8
// (64-byte rows, 64-byte swizzle), chosen by timing when a plan is created
constexpr int kZq = 16;

template <int NX, int NY>
struct XYShape {
  static constexpr int NXH = NX / 2 + 1;
  static constexpr int TX = LineCfg<NX>::T, EX = LineCfg<NX>::E;
  static constexpr int TY = LineCfg<NY>::T, EY = LineCfg<NY>::E;
  // the slab, then copies of the x and y twiddle tables
  static constexpr size_t smem() { return sizeof(float2) * ((size_t)NY * NXH + NX + NY); }
  // CTAs that fit one SM's shared memory, at most 3 (85 registers a thread)
  static constexpr int ctas() {
    return (int)((227u * 1024u) / (smem() + 1024u)) >= 3 ? 3
           : (int)((227u * 1024u) / (smem() + 1024u)) >= 2 ? 2 : 1;
  }
};

// Row pair of x-line g. A row pair is 2*NXH = nx + 2 slots long (2 banks mod
// 16), so the 16/T lines of a half-warp take pairs 8/(16/T) apart.
template <int T>
AW_D int xline_pair(int g) {
  constexpr int H = 16 / T;
  const int r = g & 7;
  return (g & ~7) + (r % H) * (8 / H) + r / H;
}

// Column of y-line g (column 0 stands for the packed 0 | nx/2 line). Columns
// are 1 bank apart (NXH = 1 mod 16), so the lines of a half-warp take
// columns BC/(16/T) apart within blocks of BC.
template <int T, int BC>
AW_D int yline_col(int g) {
  constexpr int H = (16 / T) < BC ? (16 / T) : BC;
  const int r = g % BC;
  return g - r + (r % H) * (BC / H) + r / H;
}

// the x and y twiddle tables into shared memory after the slab; the
// caller's next __syncthreads makes them visible
template <int NX, int NY>
AW_D SmemTw copy_twiddles(float2 *sm, const FluidPlan &p) {
  float2 *tw = sm + (size_t)NY * XYShape<NX, NY>::NXH;
  for (int i = threadIdx.x; i < NX; i += blockDim.x) tw[i] = __ldg(p.ax.tw + i);
  for (int i = threadIdx.x; i < NY; i += blockDim.x) tw[NX + i] = __ldg(p.ay.tw + i);
  return SmemTw{tw};
}

template <int NX, int NY, class Src>
__global__ void __launch_bounds__(kXYThreads, (XYShape<NX, NY>::ctas()))
    k_xy_fwd_fast(FluidPlan p, Src src) {
  using S = XYShape<NX, NY>;
  constexpr int NXH = S::NXH, TX = S::TX, EX = S::EX, TY = S::TY, EY = S::EY;
  extern __shared__ __align__(128) float2 sm[];
  float2 *C = sm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const Dims d = p.d;
  const int z = blockIdx.x, comp = blockIdx.y;
  const SmemTw twx = copy_twiddles<NX, NY>(sm, p);
  const SmemTw twy{twx.p + NX};
  __syncthreads();

  // ---- x: row pairs (y0, y0+1) as one complex line, exchanged in place ----
  {
    constexpr int L = 32 / TX, NLINES = NY / 2;
    static_assert(NLINES % 8 == 0 && NLINES % L == 0, "x-lines fill whole warps");
    constexpr int KU = (NXH + TX - 1) / TX;
    const int lw = lane / TX, t = lane % TX;
    for (int base = warp * L; base < NLINES; base += kXYWarps * L) {
      const int y0 = 2 * xline_pair<TX>(base + lw);
      float2 *row = C + y0 * NXH;
      float2 v[EX];
      if constexpr (NX >= 32) {
        // The warp's L row pairs, one at a time, with its 32 lanes on 32
        // consecutive x: every load is one 128-byte line (the line layout,
        // TX lanes of TX-strided x on each of L rows, would touch L lines
        // per load). The pairs go into their own slots, then each line
        // reads its strided elements back. (Unrolling over the pairs, all
        // their loads in flight at once, measured slower: 33.3 -> 35.4 us.)
#pragma unroll 1
        for (int l = 0; l < L; ++l) {
          const int yl = 2 * xline_pair<TX>(base + l);
          float2 u[NX / 32];
          src.template row_pair<NX / 32, 32>(comp, lane, yl, z, d, u);
          float2 *rl = C + yl * NXH;
#pragma unroll
          for (int j = 0; j < NX / 32; ++j) rl[lane + 32 * j] = u[j];
        }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < EX; ++j) v[j] = row[t + TX * j];
      } else {
        src.template row_pair<EX, TX>(comp, t, y0, z, d, v);
      }
      line_fft<NX, -1>(v, t, [row](int m) { return row + m; }, twx);
#pragma unroll
      for (int r = 0; r < EX; ++r) row[line_out_index<NX>(t, r)] = v[r];
      __syncwarp();
      // two real rows from one complex transform:
      // X0[k] = (Z[k] + conj Z[n-k]) / 2,  X1[k] = (Z[k] - conj Z[n-k]) / 2i
      float2 Zk[KU], Zm[KU];
#pragma unroll
      for (int i = 0; i < KU; ++i) {
        const int k = t + TX * i;
        if (k < NXH) {
          Zk[i] = row[k];
          Zm[i] = row[(NX - k) & (NX - 1)];
        }
      }
      __syncwarp();
#pragma unroll
      for (int i = 0; i < KU; ++i) {
        const int k = t + TX * i;
        if (k < NXH) {
          const float2 Z = Zk[i], M = Zm[i];
          row[k] = make_float2(0.5f * (Z.x + M.x), 0.5f * (Z.y - M.y));
          row[NXH + k] = make_float2(0.5f * (Z.y + M.y), -0.5f * (Z.x - M.x));
        }
      }
    }
  }
  __syncthreads();

  // ---- y: columns kx = 1..NX/2-1, plus the packed real columns 0 | NX/2 ---
  {
    constexpr int L = 32 / TY, NLINES = NX / 2, BC = NLINES >= 16 ? 16 : NLINES;
    static_assert(NLINES % L == 0, "y-lines fill whole warps");
    const int lw = lane / TY, t = lane % TY;
    for (int base = warp * L; base < NLINES; base += kXYWarps * L) {
      const int l = yline_col<TY, BC>(base + lw);
      const bool packed = l == 0;
      float2 *col = C + l;
      float2 v[EY];
#pragma unroll
      for (int j = 0; j < EY; ++j) {
        const int y = t + TY * j;
        v[j] = packed ? make_float2(C[y * NXH].x, C[y * NXH + NX / 2].x) : col[y * NXH];
      }
      line_fft<NY, -1>(v, t, [col](int m) { return col + m * NXH; }, twy);
#pragma unroll
      for (int r = 0; r < EY; ++r) col[line_out_index<NY>(t, r) * NXH] = v[r];
      if (packed) {
        // split the packed line into the spectra of columns 0 and NX/2
        const unsigned mask = (TY == 32 ? 0xffffffffu : ((1u << TY) - 1u)) << (lw * TY);
        float2 Zm[EY];
        __syncwarp(mask);
#pragma unroll
        for (int i = 0; i < EY; ++i) {
          const int k = t + TY * i;
          v[i] = C[k * NXH];
          Zm[i] = C[((NY - k) & (NY - 1)) * NXH];
        }
        __syncwarp(mask);
#pragma unroll
        for (int i = 0; i < EY; ++i) {
          const int k = t + TY * i;
          const float2 Z = v[i], M = Zm[i];
          C[k * NXH] = make_float2(0.5f * (Z.x + M.x), 0.5f * (Z.y - M.y));
          C[k * NXH + NX / 2] = make_float2(0.5f * (Z.y + M.y), -0.5f * (Z.x - M.x));
        }
      }
      __syncwarp();
    }
  }

  // ---- store the slab: one bulk copy shared -> HBM -----------------------
  fence_async_smem();
  __syncthreads();
  if (threadIdx.x == 0) {
    bulk_store(p.spec + ((long)comp * d.nz + z) * NY * NXH, C,
               (uint32_t)(sizeof(float2) * NY * NXH));
    bulk_wait_read();
  }
}

// Inverse y-transform of every column of the slab in shared memory, the
// packed real columns 0 | NX/2 included.
template <int NX, int NY>
AW_D void inv_y_pass(float2 *C, const SmemTw &tw, int warp, int lane) {
  using S = XYShape<NX, NY>;
  constexpr int NXH = S::NXH, TY = S::TY, EY = S::EY;
  constexpr int L = 32 / TY, NLINES = NX / 2, BC = NLINES >= 16 ? 16 : NLINES;
  const int lw = lane / TY, t = lane % TY;
  for (int base = warp * L; base < NLINES; base += kXYWarps * L) {
    const int l = yline_col<TY, BC>(base + lw);
    const bool packed = l == 0;
    float2 *col = C + l;
    float2 v[EY];
#pragma unroll
    for (int j = 0; j < EY; ++j) {
      const int y = t + TY * j;
      if (packed) {
        const float2 a = C[y * NXH], b = C[y * NXH + NX / 2];
        v[j] = make_float2(a.x - b.y, a.y + b.x);  // a + i b
      } else {
        v[j] = col[y * NXH];
      }
    }
    line_fft<NY, +1>(v, t, [col](int m) { return col + m * NXH; }, tw);
#pragma unroll
    for (int r = 0; r < EY; ++r) {
      const int y = line_out_index<NY>(t, r);
      if (packed) {
        // real parts of the two columns; c2r ignores their imaginary parts
        C[y * NXH] = make_float2(v[r].x, 0.f);
        C[y * NXH + NX / 2] = make_float2(v[r].y, 0.f);
      } else {
        col[y * NXH] = v[r];
      }
    }
  }
}

// Inverse x-transform (complex to real) of every row pair with Hermitian
// completion; out(x, y, value) receives each real output, from the warp's 32
// lanes on 32 consecutive x of one row at a time (NX >= 32). A row pair's
// lines read and write only that pair's own slots, which hold 2 * NXH >= NX
// + 2 floats per row: the outputs are staged there once the line's
// transform has returned (line_fft ends on a warp barrier), and the warp
// reads them back for its coalesced writes; afterwards row y holds its
// outputs as floats at (float *)(C + y * NXH).
template <int NX, int NY, class Out>
AW_D void inv_x_pass(float2 *C, const SmemTw &tw, int warp, int lane, const Out &out) {
  using S = XYShape<NX, NY>;
  constexpr int NXH = S::NXH, TX = S::TX, EX = S::EX;
  constexpr int L = 32 / TX, NLINES = NY / 2;
  const int lw = lane / TX, t = lane % TX;
  for (int base = warp * L; base < NLINES; base += kXYWarps * L) {
    const int y0 = 2 * xline_pair<TX>(base + lw);
    float2 *row = C + y0 * NXH;
    float2 v[EX];
#pragma unroll
    for (int j = 0; j < EX; ++j) {
      const int k = t + TX * j;
      const bool upper = k > NX / 2;
      const int kk = upper ? NX - k : k;
      float2 X0 = row[kk], X1 = row[NXH + kk];
      if (kk == 0 || kk == NX / 2) { X0.y = 0.f; X1.y = 0.f; }
      if (upper) { X0.y = -X0.y; X1.y = -X1.y; }
      v[j] = make_float2(X0.x - X1.y, X0.y + X1.x);
    }
    line_fft<NX, +1>(v, t, [row](int m) { return row + m; }, tw);
    if constexpr (NX >= 32) {
      // the outputs into the line's own slots as floats, then the warp
      // writes its L row pairs out with its 32 lanes on 32 consecutive x
      // (one 128-byte line per store instead of L)
      float *r0 = reinterpret_cast<float *>(row), *r1 = reinterpret_cast<float *>(row + NXH);
#pragma unroll
      for (int r = 0; r < EX; ++r) {
        const int x = line_out_index<NX>(t, r);
        r0[x] = v[r].x;
        r1[x] = v[r].y;
      }
      __syncwarp();
#pragma unroll 1
      for (int l = 0; l < L; ++l) {
        const int yl = 2 * xline_pair<TX>(base + l);
        const float *q0 = reinterpret_cast<const float *>(C + yl * NXH);
        const float *q1 = reinterpret_cast<const float *>(C + (yl + 1) * NXH);
#pragma unroll
        for (int j = 0; j < NX / 32; ++j) {
          out(lane + 32 * j, yl, q0[lane + 32 * j]);
          out(lane + 32 * j, yl + 1, q1[lane + 32 * j]);
        }
      }
    } else {
#pragma unroll
      for (int r = 0; r < EX; ++r) {
        const int x = line_out_index<NX>(t, r);
        out(x, y0, v[r].x);
        out(x, y0 + 1, v[r].y);
      }
    }
  }
}

// the slab of (z, comp), one bulk copy HBM -> shared; false (status word
// set) when it never lands
template <int NX, int NY>
AW_D bool load_slab(float2 *C, uint64_t *mbar, const FluidPlan &p, int z, int comp) {
  using S = XYShape<NX, NY>;
  if (threadIdx.x == 0) {
    const uint32_t bytes = (uint32_t)(sizeof(float2) * NY * S::NXH);
    mbar_init(mbar, 1);
    mbar_expect_tx(mbar, bytes);
    bulk_load(C, p.spec + ((long)comp * p.d.nz + z) * NY * S::NXH, bytes, mbar);
  }
  __syncthreads();
  return !__syncthreads_or(!mbar_wait(mbar, 0, p.status));
}

template <int NX, int NY, class Dst>
__global__ void __launch_bounds__(kXYThreads, (XYShape<NX, NY>::ctas()))
    k_xy_inv_fast(FluidPlan p, Dst dst) {
  extern __shared__ __align__(128) float2 sm[];
  __shared__ uint64_t mbar;
  float2 *C = sm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const Dims d = p.d;
  const int z = blockIdx.x, comp = blockIdx.y;
  const SmemTw twx = copy_twiddles<NX, NY>(sm, p);
  const SmemTw twy{twx.p + NX};
  // a slab that never lands: the status word says so and the CTA leaves as one
  if (!load_slab<NX, NY>(C, &mbar, p, z, comp)) return;
  inv_y_pass<NX, NY>(C, twy, warp, lane);
  __syncthreads();
  const auto o = dst.bind(comp);
  if constexpr (Dst::kReads && NX >= 32) {
    // a store that reads the old value (the LDMM update): the x pass leaves
    // the plane in shared memory, then each thread reads kBatch old values
    // before it writes any, so their loads overlap instead of each waiting
    // behind the previous store
    inv_x_pass<NX, NY>(C, twx, warp, lane, [](int, int, float) {});
    __syncthreads();
    constexpr int NXH = XYShape<NX, NY>::NXH, PER = NX * NY / kXYThreads;
    constexpr int kBatch = PER < 8 ? PER : 8;
    const float *P = reinterpret_cast<const float *>(C);
#pragma unroll 1
    for (int k0 = 0; k0 < PER; k0 += kBatch) {
      long idx[kBatch];
      float u[kBatch];
#pragma unroll
      for (int j = 0; j < kBatch; ++j) {
        const int e = threadIdx.x + kXYThreads * (k0 + j), y = e / NX, x = e % NX;
        idx[j] = d.idx(x, y, z);
        u[j] = P[y * 2 * NXH + x];
      }
      o.template store_n<kBatch>(idx, u);
    }
  } else {
    inv_x_pass<NX, NY>(C, twx, warp, lane,
                       [&](int x, int y, float v) { o.store(d.idx(x, y, z), v); });
  }
}

// The inverse transform fused with the greedy update h'(x) = h(x + eps v(x)/sp)
// (composeHV with PARTIAL_ID, HField3DUtils.txx:436-455, as k_update in
// greedy.cu computes it). The three CTAs of a cluster hold the three
// components of one z-slab: each transforms its component and keeps v in
// its own shared memory, then each updates a third of the slab's rows,
// reading the three components of v there through distributed shared
// memory, so v never goes to HBM.
template <int NX, int NY, bool FAST>
__global__ void __cluster_dims__(1, 3, 1) __launch_bounds__(kXYThreads, (XYShape<NX, NY>::ctas()))
    k_xy_inv_compose(FluidPlan p, ComposeArgs a) {
  using S = XYShape<NX, NY>;
  constexpr int NXH = S::NXH;
  extern __shared__ __align__(128) float2 sm[];
  __shared__ uint64_t mbar;
  float2 *C = sm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const Dims d = p.d;
  const int z = blockIdx.x, comp = blockIdx.y;
  cg::cluster_group cluster = cg::this_cluster();
  const SmemTw twx = copy_twiddles<NX, NY>(sm, p);
  const SmemTw twy{twx.p + NX};
  // a slab that never lands: the status word says so; the CTA still takes
  // part in both cluster barriers, so its partners never wait for it
  const bool ok = load_slab<NX, NY>(C, &mbar, p, z, comp);
  if (ok) {
    inv_y_pass<NX, NY>(C, twy, warp, lane);
    __syncthreads();
    // v stays in shared memory: row y as floats at (float *)(C + y * NXH)
    // (inv_x_pass leaves it there itself when NX >= 32)
    inv_x_pass<NX, NY>(C, twx, warp, lane, [C](int x, int y, float v) {
      if constexpr (NX < 32) reinterpret_cast<float *>(C + y * NXH)[x] = v;
    });
  }
  cluster.sync();  // all three components of v are in the cluster's shared memory
  if (ok) {
    const float *V0 = reinterpret_cast<const float *>(cluster.map_shared_rank(C, 0));
    const float *V1 = reinterpret_cast<const float *>(cluster.map_shared_rank(C, 1));
    const float *V2 = reinterpret_cast<const float *>(cluster.map_shared_rank(C, 2));
    const float eps = *a.step;
    // CTA `comp` updates a contiguous third of the rows, so the h rows
    // that neighbouring rows' gathers share are read close together in time
    constexpr int RPI = kXYThreads / NX;  // rows per pass
    const int x = threadIdx.x % NX;
    const int y1 = (comp + 1) * NY / 3;
#pragma unroll 2
    for (int y = comp * NY / 3 + threadIdx.x / NX; y < y1; y += RPI) {
      const int e = y * 2 * NXH + x;
      const float vx = V0[e], vy = V1[e], vz = V2[e];
      const float px = fadd(__int2float_rn(x), fdivq(fmul(vx, eps), a.q0));
      const float py = fadd(__int2float_rn(y), fdivq(fmul(vy, eps), a.q1));
      const float pz = fadd(__int2float_rn(z), fdivq(fmul(vz, eps), a.q2));
      float rx, ry, rz;
      trilerp_vector<FAST>(a.hx, a.hy, a.hz, d, px, py, pz, BG_PARTIAL_ID, 1.0f, rx, ry, rz);
      const long i = d.idx(x, y, z);
      a.ox[i] = rx;
      a.oy[i] = ry;
      a.oz[i] = rz;
    }
  }
  cluster.sync();  // no CTA leaves while a partner may still read its v
}

// per-wavenumber solve of one (kx, ky, kz): the three components at b0p,
// b1p, b2p (DiffOper.cxx:1005-1083 for the inverse, 1088-1116 for L)
AW_D void solve_point(const FluidPlan &p, int kx, int ky, int kz, int inverse, float invN,
                      float2 *b0p, float2 *b1p, float2 *b2p) {
  const float *cwx = p.lut, *swx = cwx + p.d.nx, *cwy = swx + p.d.nx, *swy = cwy + p.d.ny,
              *cwz = swy + p.d.ny, *swz = cwz + p.d.nz;
  const float cx = __ldg(cwx + kx), cy = __ldg(cwy + ky), cz = __ldg(cwz + kz);
  const float sx = __ldg(swx + kx), sy = __ldg(swy + ky), sz = __ldg(swz + kz);
  const float lambda = -p.alpha * (cx + cy + cz) + p.gamma;
  const float L00 = lambda - p.beta * cx, L11 = lambda - p.beta * cy, L22 = lambda - p.beta * cz;
  const float L10 = p.beta * sx * sy, L20 = p.beta * sx * sz, L21 = p.beta * sy * sz;
  float2 b0 = *b0p, b1 = *b1p, b2 = *b2p;
  b0.x *= invN; b0.y *= invN; b1.x *= invN; b1.y *= invN; b2.x *= invN; b2.y *= invN;
  float2 o0, o1, o2;
  if (inverse) {
    // Cholesky L = G G^T, then G y = b, G^T x = y (real matrix, complex
    // rhs), dividing by the diagonal through its reciprocals
    const float G00 = sqrtf(L00), i00 = 1.0f / G00;
    const float G10 = L10 * i00, G20 = L20 * i00;
    const float G11 = sqrtf(L11 - G10 * G10), i11 = 1.0f / G11;
    const float G21 = (L21 - G20 * G10) * i11;
    const float G22 = sqrtf(L22 - (G20 * G20 + G21 * G21)), i22 = 1.0f / G22;
    float2 y0, y1, y2;
    y0.x = b0.x * i00;                              y0.y = b0.y * i00;
    y1.x = (b1.x - G10 * y0.x) * i11;               y1.y = (b1.y - G10 * y0.y) * i11;
    y2.x = (b2.x - G20 * y0.x - G21 * y1.x) * i22;  y2.y = (b2.y - G20 * y0.y - G21 * y1.y) * i22;
    o2.x = y2.x * i22;                              o2.y = y2.y * i22;
    o1.x = (y1.x - G21 * o2.x) * i11;               o1.y = (y1.y - G21 * o2.y) * i11;
    o0.x = (y0.x - G10 * o1.x - G20 * o2.x) * i00;  o0.y = (y0.y - G10 * o1.y - G20 * o2.y) * i00;
  } else {
    o0.x = L00 * b0.x + L10 * b1.x + L20 * b2.x;  o0.y = L00 * b0.y + L10 * b1.y + L20 * b2.y;
    o1.x = L10 * b0.x + L11 * b1.x + L21 * b2.x;  o1.y = L10 * b0.y + L11 * b1.y + L21 * b2.y;
    o2.x = L20 * b0.x + L21 * b1.x + L22 * b2.x;  o2.y = L20 * b0.y + L21 * b1.y + L22 * b2.y;
  }
  *b0p = o0;
  *b1p = o1;
  *b2p = o2;
}

// element (kz, q) of a [nz x Q] complex tile in the TMA swizzle of its row
// size: with 128-byte rows (Q = 16) the 16-byte chunk q/2 of row kz sits at
// chunk (q/2) ^ (kz mod 8); with 64-byte rows (Q = 8) at (q/2) ^ ((kz/2) mod 4)
template <int Q>
AW_D int zt(int k, int q) {
  static_assert(Q == 16 || Q == 8, "z tile width");
  return Q == 16 ? k * 16 + (q ^ ((k & 7) << 1)) : k * 8 + (q ^ (((k >> 1) & 3) << 1));
}

template <int NZ, int Q>
constexpr int z_threads() { return 3 * Q * LineCfg<NZ>::T; }

// z-pass over one CTA's 16 columns; tiles TB[c] = [nz x 16] complex. With
// TMA the tiles move by tensor copies (columns past the spectrum's end read
// as zero and are not written back), else by coalesced plain copies.
template <int NZ, int Q, bool TMA>
__global__ void __launch_bounds__(z_threads<NZ, Q>(), (NZ <= 128 ? 48 / Q : 16 / Q))
    k_z_solve_fast(FluidPlan p, const __grid_constant__ CUtensorMap tmap, int inverse) {
  constexpr int T = LineCfg<NZ>::T, E = LineCfg<NZ>::E, TILE = NZ * Q;
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint64_t mbar[3];
  // the swizzle pattern repeats every 1024 bytes: align the tiles to it
  float2 *TB = reinterpret_cast<float2 *>(smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u));
  // the z twiddle table after the three tiles (visible after the first barrier)
  float2 *twz = TB + 3 * TILE;
  for (int i = threadIdx.x; i < NZ; i += blockDim.x) twz[i] = __ldg(p.az.tw + i);
  const SmemTw tw{twz};
  const long ncols = (long)p.d.ny * p.nxh;
  const long j0 = (long)blockIdx.x * Q;
  const int line = threadIdx.x / T, t = threadIdx.x % T;
  const int c = line / Q, q = line % Q;
  float2 *tile = TB + c * TILE;
  bool ok = true;
  if constexpr (TMA) {
    if (threadIdx.x == 0) {
      for (int cc = 0; cc < 3; ++cc) mbar_init(&mbar[cc], 1);
      for (int cc = 0; cc < 3; ++cc) {
        mbar_expect_tx(&mbar[cc], (uint32_t)(TILE * sizeof(float2)));
        tma_load_3d(TB + cc * TILE, &tmap, (int)(2 * j0), 0, cc, &mbar[cc]);
      }
    }
    __syncthreads();
    // each component's lines start as soon as their own tile has landed
    ok = mbar_wait(&mbar[c], 0, p.status);
  } else {
    for (int i = threadIdx.x; i < 3 * TILE; i += blockDim.x) {
      const int qq = i % Q, r = i / Q;  // r = cc*NZ + kz
      const int cc = r / NZ, kz = r - cc * NZ;
      TB[cc * TILE + zt<Q>(kz, qq)] =
          (j0 + qq < ncols) ? p.spec[(long)r * ncols + j0 + qq] : make_float2(0.f, 0.f);
    }
    __syncthreads();
  }

  float2 v[E];
#pragma unroll
  for (int j = 0; j < E; ++j) v[j] = tile[zt<Q>(t + T * j, q)];
  line_fft<NZ, -1>(v, t, [tile, q](int m) { return tile + zt<Q>(m, q); }, tw);
#pragma unroll
  for (int r = 0; r < E; ++r) tile[zt<Q>(line_out_index<NZ>(t, r), q)] = v[r];
  if (__syncthreads_or(!ok)) return;  // a tile never landed: the status word says so

  const float invN = 1.0f / (float)p.d.n();
  const int nxh = p.nxh;
  for (int i = threadIdx.x; i < TILE; i += blockDim.x) {
    const int kz = i / Q, qq = i % Q;
    const long jj = j0 + qq;
    if (jj >= ncols) continue;
    const int ky = (int)(jj / nxh), kx = (int)(jj - (long)ky * nxh);
    const int e = zt<Q>(kz, qq);
    solve_point(p, kx, ky, kz, inverse, invN, TB + e, TB + TILE + e, TB + 2 * TILE + e);
  }
  __syncthreads();

#pragma unroll
  for (int j = 0; j < E; ++j) v[j] = tile[zt<Q>(t + T * j, q)];
  line_fft<NZ, +1>(v, t, [tile, q](int m) { return tile + zt<Q>(m, q); }, tw);
#pragma unroll
  for (int r = 0; r < E; ++r) tile[zt<Q>(line_out_index<NZ>(t, r), q)] = v[r];

  if constexpr (TMA) {
    fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int cc = 0; cc < 3; ++cc) tma_store_3d(&tmap, (int)(2 * j0), 0, cc, TB + cc * TILE);
      bulk_commit();
      bulk_wait_read();
    }
  } else {
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * TILE; i += blockDim.x) {
      const int qq = i % Q, r = i / Q;
      const int cc = r / NZ, kz = r - cc * NZ;
      if (j0 + qq < ncols) p.spec[(long)r * ncols + j0 + qq] = TB[cc * TILE + zt<Q>(kz, qq)];
    }
  }
}

// ---- dispatch over the supported sizes -------------------------------------
template <class F>
bool dispatch_n(int n, F &&f) {
  switch (n) {
    case 16: f(std::integral_constant<int, 16>()); return true;
    case 32: f(std::integral_constant<int, 32>()); return true;
    case 64: f(std::integral_constant<int, 64>()); return true;
    case 128: f(std::integral_constant<int, 128>()); return true;
    case 256: f(std::integral_constant<int, 256>()); return true;
    default: return false;
  }
}

}  // namespace

bool fast_supported(int n) { return n == 16 || n == 32 || n == 64 || n == 128 || n == 256; }

size_t fast_xy_smem(int nx, int ny) {
  size_t r = 0;
  dispatch_n(nx, [&](auto X) {
    dispatch_n(ny, [&](auto Y) { r = XYShape<decltype(X)::value, decltype(Y)::value>::smem(); });
  });
  return r;
}

int fast_z_cols() { return kZq; }

size_t fast_z_smem(int nz, int q) { return sizeof(float2) * (3 * (size_t)nz * q + nz) + 1024; }

cudaError_t fast_configure(const FluidPlan &p) {
  cudaError_t e = cudaSuccess;
  const size_t sxy = fast_xy_smem(p.d.nx, p.d.ny);
  auto set = [&](const void *k, size_t bytes) {
    cudaError_t r = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (r != cudaSuccess) e = r;
  };
  dispatch_n(p.d.nx, [&](auto X) {
    dispatch_n(p.d.ny, [&](auto Y) {
      constexpr int NX = decltype(X)::value, NY = decltype(Y)::value;
      set((const void *)k_xy_fwd_fast<NX, NY, SrcField>, sxy);
      set((const void *)k_xy_fwd_fast<NX, NY, SrcForce>, sxy);
      set((const void *)k_xy_inv_fast<NX, NY, DstField>, sxy);
      set((const void *)k_xy_inv_fast<NX, NY, DstAxpby>, sxy);
      set((const void *)k_xy_inv_fast<NX, NY, DstNeg>, sxy);
      set((const void *)k_xy_inv_compose<NX, NY, false>, sxy);
      set((const void *)k_xy_inv_compose<NX, NY, true>, sxy);
    });
  });
  dispatch_n(p.d.nz, [&](auto Z) {
    constexpr int NZ = decltype(Z)::value;
    set((const void *)k_z_solve_fast<NZ, 16, true>, fast_z_smem(NZ, 16));
    set((const void *)k_z_solve_fast<NZ, 16, false>, fast_z_smem(NZ, 16));
    set((const void *)k_z_solve_fast<NZ, 8, true>, fast_z_smem(NZ, 8));
    set((const void *)k_z_solve_fast<NZ, 8, false>, fast_z_smem(NZ, 8));
  });
  return e;
}

template <class Src>
cudaError_t fast_xy_forward(const FluidPlan &p, const Src &src, cudaStream_t s) {
  dispatch_n(p.d.nx, [&](auto X) {
    dispatch_n(p.d.ny, [&](auto Y) {
      constexpr int NX = decltype(X)::value, NY = decltype(Y)::value;
      k_xy_fwd_fast<NX, NY, Src><<<dim3(p.d.nz, 3), kXYThreads, p.fast_smem_xy, s>>>(p, src);
    });
  });
  return cudaGetLastError();
}

template <class Dst>
cudaError_t fast_xy_inverse(const FluidPlan &p, const Dst &dst, cudaStream_t s) {
  dispatch_n(p.d.nx, [&](auto X) {
    dispatch_n(p.d.ny, [&](auto Y) {
      constexpr int NX = decltype(X)::value, NY = decltype(Y)::value;
      k_xy_inv_fast<NX, NY, Dst><<<dim3(p.d.nz, 3), kXYThreads, p.fast_smem_xy, s>>>(p, dst);
    });
  });
  return cudaGetLastError();
}

cudaError_t fast_xy_inverse_compose(const FluidPlan &p, const ComposeArgs &a, cudaStream_t s) {
  dispatch_n(p.d.nx, [&](auto X) {
    dispatch_n(p.d.ny, [&](auto Y) {
      constexpr int NX = decltype(X)::value, NY = decltype(Y)::value;
      const dim3 grid(p.d.nz, 3);
      if (a.fast)
        k_xy_inv_compose<NX, NY, true><<<grid, kXYThreads, p.fast_smem_xy, s>>>(p, a);
      else
        k_xy_inv_compose<NX, NY, false><<<grid, kXYThreads, p.fast_smem_xy, s>>>(p, a);
    });
  });
  return cudaGetLastError();
}

cudaError_t fast_z_solve(const FluidPlan &p, int inverse, cudaStream_t s) {
  const long ncols = (long)p.d.ny * p.nxh;
  const int q = p.fast_kq == 8 ? 8 : 16;
  const int grid = (int)((ncols + q - 1) / q);
  dispatch_n(p.d.nz, [&](auto Z) {
    constexpr int NZ = decltype(Z)::value;
    const size_t sm = fast_z_smem(NZ, q);
    if (q == 8 && p.fast_tma)
      k_z_solve_fast<NZ, 8, true><<<grid, z_threads<NZ, 8>(), sm, s>>>(p, p.spec_map, inverse);
    else if (q == 8)
      k_z_solve_fast<NZ, 8, false><<<grid, z_threads<NZ, 8>(), sm, s>>>(p, p.spec_map, inverse);
    else if (p.fast_tma)
      k_z_solve_fast<NZ, 16, true><<<grid, z_threads<NZ, 16>(), sm, s>>>(p, p.spec_map, inverse);
    else
      k_z_solve_fast<NZ, 16, false><<<grid, z_threads<NZ, 16>(), sm, s>>>(p, p.spec_map, inverse);
  });
  return cudaGetLastError();
}

template cudaError_t fast_xy_forward<SrcField>(const FluidPlan &, const SrcField &, cudaStream_t);
template cudaError_t fast_xy_forward<SrcForce>(const FluidPlan &, const SrcForce &, cudaStream_t);
template cudaError_t fast_xy_inverse<DstField>(const FluidPlan &, const DstField &, cudaStream_t);
template cudaError_t fast_xy_inverse<DstAxpby>(const FluidPlan &, const DstAxpby &, cudaStream_t);
template cudaError_t fast_xy_inverse<DstNeg>(const FluidPlan &, const DstNeg &, cudaStream_t);

}  // namespace aw
