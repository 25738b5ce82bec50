// nn.cu — the learned warm start's network kernels: 3D convolutions as
// implicit GEMMs on the 5th-generation tensor cores (tcgen05, BF16 x BF16
// -> FP32 in TMEM), forward, data gradient and weight gradient, plus the
// elementwise layers of the encoder-decoder (average pooling, nearest
// upsampling, skip concatenation), the MSE loss and Adam.
//
// Activations are BF16, channels last: [B][D][H][W][C] with C a multiple of
// 16. Weights are BF16 [Cout][taps][Cin] (K = taps * Cin contiguous per
// output channel) with an FP32 master copy; taps is 27 (3x3x3, zero
// padding) or 1.
//
// One GEMM kernel serves the three products. A CTA owns 128 rows of D and
// all N columns (N = the output channels, 16..256): 128 threads gather the
// A and B tiles of one 64-deep K step into shared memory (two stages), one
// thread issues four K=16 MMAs per step into the TMEM accumulator and
// commits them to the stage's mbarrier, and the four warps read their 32
// TMEM lanes back for the fused epilogue.
//   forward  D[voxel][co]  = sum_{tap,ci} X[voxel + off(tap)][ci] W[co][tap][ci]
//   dgrad    D[voxel][ci]  = sum_{tap,co} dY[voxel - off(tap)][co] W[co][tap][ci]
//   wgrad    D[(tap,ci)][co] = sum_voxel X[voxel + off(tap)][ci] dY[voxel][co]
// (wgrad: K = voxels, split over CTAs; both of its operands are read
// MN-major straight from the channels-last tensors).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

#include "tma_host.cuh"
#include "umma.cuh"

namespace aw {

namespace {

constexpr int kGBM = 128;      // rows per CTA
constexpr int kGBK = 64;       // K per stage
constexpr int kGThreads = 128;
constexpr int kAStage = kGBM * kGBK * 2;  // bytes

typedef __nv_bfloat16 bf16;

// n / d for 0 <= n < 2^31 by multiply and shift (round-up method):
// mul = floor(2^32 (2^l - d) / d) + 1, l = ceil(log2 d), q = (hi(n mul) + n) >> l
struct FastDiv {
  uint32_t d, mul, l;
  AW_D uint32_t div(uint32_t n) const { return (__umulhi(n, mul) + n) >> l; }
};
inline FastDiv make_fastdiv(uint32_t d) {
  uint32_t l = 0;
  while ((1ull << l) < d) ++l;
  const uint64_t mul = ((1ull << 32) * ((1ull << l) - d)) / d + 1;
  return FastDiv{d, (uint32_t)mul, l};
}

struct Vol {
  int B, D, H, W;
  FastDiv fw, fh, fd;
  AW_HD long voxels() const { return (long)B * D * H * W; }
};
inline Vol make_vol(int B, int D, int H, int W) {
  return Vol{B, D, H, W, make_fastdiv(W), make_fastdiv(H), make_fastdiv(D)};
}

// tap -> (dz, dy, dx) offsets of a 3x3x3 stencil, packed as 3 x 2 bits (+1)
AW_D void tap_offset(int tap, int ntaps, int &dz, int &dy, int &dx) {
  if (ntaps == 1) {
    dz = dy = dx = 0;
  } else {
    dz = tap / 9 - 1;
    dy = (tap / 3) % 3 - 1;
    dx = tap % 3 - 1;
  }
}

// voxel index m -> (b, z, y, x)
AW_D void voxel_coords(const Vol &v, int m, int &b, int &z, int &y, int &x) {
  const int q1 = (int)v.fw.div((uint32_t)m);
  x = m - q1 * v.W;
  const int q2 = (int)v.fh.div((uint32_t)q1);
  y = q1 - q2 * v.H;
  b = (int)v.fd.div((uint32_t)q2);
  z = q2 - b * v.D;
}

AW_D uint32_t kmajor_off(int r, int j, int R) { return j * (R * 16) + (r >> 3) * 128 + (r & 7) * 16; }
AW_D uint32_t mnmajor_off(int k, int c, int R) { return (k >> 3) * (R * 16) + c * 128 + (k & 7) * 16; }

// ---- operand loaders ----------------------------------------------------------
// Each loader copies this thread's 16-byte chunks of one 64-deep K step
// from global memory straight into the stage's canonical layout with
// cp.async (zero-filled past kend or outside the volume; cached in L1, where
// the 27 taps of neighbouring rows meet); init() computes the per-thread
// context once per CTA.
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gsrc, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(smem_dst)),
               "l"(gsrc), "r"(valid ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// A of forward / dgrad: rows = voxels, K = (tap, channel) of X shifted by
// sign * off(tap); K-major (the 8 channels of a chunk are contiguous).
// Thread t owns row t of the tile; which taps stay inside the volume for
// that voxel is a 27-bit mask, and the voxel-index offset of each tap a
// table in shared memory, both made once per CTA.
struct LoadConvA {
  const bf16 *x;
  Vol v;
  int C, ntaps, sign;
  int M;
  FastDiv fc;
  static constexpr int kMN = 0;
  struct Ctx {
    int m;
    uint32_t vmask;
    const int *toff;
  };
  AW_D Ctx init(long m0) const {
    __shared__ int s_toff[27];
    if (threadIdx.x < ntaps) {
      int dz, dy, dx;
      tap_offset(threadIdx.x, ntaps, dz, dy, dx);
      s_toff[threadIdx.x] = sign * ((dz * v.H + dy) * v.W + dx);
    }
    Ctx c;
    c.m = (int)m0 + threadIdx.x;
    c.toff = s_toff;
    c.vmask = 0;
    if (c.m < M) {
      int b, z, y, xx;
      voxel_coords(v, c.m, b, z, y, xx);
      for (int t = 0; t < ntaps; ++t) {
        int dz, dy, dx;
        tap_offset(t, ntaps, dz, dy, dx);
        const int zz = z + sign * dz, yy = y + sign * dy, xs = xx + sign * dx;
        if (zz >= 0 && zz < v.D && yy >= 0 && yy < v.H && xs >= 0 && xs < v.W) c.vmask |= 1u << t;
      }
    }
    return c;  // the caller synchronises the CTA before the first issue()
  }
  AW_D void issue(const Ctx &c, uint8_t *s, int k0, int kend) const {
    int tap = (int)fc.div((uint32_t)k0);
    int ci = k0 - tap * C;
#pragma unroll
    for (int j = 0; j < kGBK / 8; ++j) {
      const bool ok = ((c.vmask >> tap) & 1u) && (k0 + 8 * j < kend);
      const bf16 *src = ok ? x + (long)(c.m + c.toff[tap]) * C + ci : x;
      cp_async16(s + kmajor_off(threadIdx.x, j, kGBM), src, ok);
      ci += 8;
      if (ci == C) {
        ci = 0;
        ++tap;
      }
    }
  }
};

// B of forward / dgrad: rows = output columns n < N, K contiguous per row.
// Chunk i = tid + 128 q: row i / 8, K chunk i % 8 (8 threads read one
// row's 128 contiguous bytes).
template <int BN>
struct LoadRowsB {
  const bf16 *w;  // [BN][K]
  int K;
  static constexpr int kMN = 0, kChunks = BN * (kGBK / 8) / kGThreads;
  static_assert(BN * (kGBK / 8) % kGThreads == 0, "whole chunks per thread");
  struct Ctx {};
  AW_D Ctx init(long) const { return Ctx{}; }
  AW_D void issue(const Ctx &, uint8_t *s, int k0, int kend) const {
#pragma unroll
    for (int q = 0; q < kChunks; ++q) {
      const int i = threadIdx.x + kGThreads * q;
      const int row = i >> 3, j = i & 7, k = k0 + 8 * j;
      const bool ok = k < kend;
      cp_async16(s + kmajor_off(row, j, BN), ok ? w + (long)row * K + k : w, ok);
    }
  }
};

// A of wgrad: rows = (tap, ci) < ntaps*C, K = voxels; MN-major: the 8
// channels of a chunk are contiguous in X. Thread t owns the channel chunk
// c = (t / 8) % 16 (a fixed (tap, ci0) for the CTA) at voxels
// k0 + t % 8 + 8j, so consecutive threads fill consecutive shared slots.
struct LoadWgradA {
  const bf16 *x;
  Vol v;
  int C, ntaps;
  int Mtot;  // ntaps * C
  FastDiv fc;
  static constexpr int kMN = 1;
  struct Ctx {
    int ok, ci, dz, dy, dx;
  };
  AW_D Ctx init(long m0) const {
    Ctx c;
    const int mn = (int)m0 + 8 * ((threadIdx.x >> 3) & 15);
    c.ok = mn < Mtot;
    const int tap = c.ok ? (int)fc.div((uint32_t)mn) : 0;
    c.ci = mn - tap * C;
    tap_offset(tap, ntaps, c.dz, c.dy, c.dx);
    return c;
  }
  AW_D void issue(const Ctx &c, uint8_t *s, int k0, int kend) const {
    // the voxel of the first chunk decoded once, then stepped by 8 along x
    int k = k0 + (threadIdx.x & 7);
    int b = 0, z = 0, y = 0, xx = 0;
    if (k < kend) voxel_coords(v, k, b, z, y, xx);
#pragma unroll
    for (int j = 0; j < kGBK / 8; ++j) {
      const bf16 *src = x;
      bool ok = false;
      if (c.ok && k < kend) {
        const int zz = z + c.dz, yy = y + c.dy, xs = xx + c.dx;
        if (zz >= 0 && zz < v.D && yy >= 0 && yy < v.H && xs >= 0 && xs < v.W) {
          src = x + (long)(((b * v.D + zz) * v.H + yy) * v.W + xs) * C + c.ci;
          ok = true;
        }
      }
      cp_async16(s + mnmajor_off((threadIdx.x & 7) + 8 * j, (threadIdx.x >> 3) & 15, kGBM), src,
                 ok);
      k += 8;
      xx += 8;
      while (xx >= v.W) {
        xx -= v.W;
        if (++y == v.H) {
          y = 0;
          if (++z == v.D) {
            z = 0;
            ++b;
          }
        }
      }
    }
  }
};

// B of wgrad: rows = co < BN, K = voxels; MN-major (dY's channels
// contiguous). Chunk i = tid + 128 q: voxel i / (BN/8), channel chunk i % (BN/8).
template <int BN>
struct LoadWgradB {
  const bf16 *dy;  // [voxels][BN]
  static constexpr int kMN = 1, kChunks = kGBK * (BN / 8) / kGThreads;
  static_assert(kGBK * (BN / 8) % kGThreads == 0, "whole chunks per thread");
  struct Ctx {};
  AW_D Ctx init(long) const { return Ctx{}; }
  AW_D void issue(const Ctx &, uint8_t *s, int k0, int kend) const {
#pragma unroll
    for (int q = 0; q < kChunks; ++q) {
      const int i = threadIdx.x + kGThreads * q;
      const int kk = i / (BN / 8), c = i % (BN / 8);
      const int k = k0 + kk;
      const bool ok = k < kend;
      cp_async16(s + mnmajor_off(kk, c, BN), ok ? dy + (long)k * BN + 8 * c : dy, ok);
    }
  }
};

// ---- epilogues: row m, 16 columns from n0 ----------------------------------
// forward: + bias, optional ReLU, BF16 out (or FP32 out)
template <int BN>
struct EpiAct {
  const float *bias;
  bf16 *out;
  float *outf;
  int relu;
  long M;
  AW_D void store(long m, int n0, const float (&v)[16]) const {
    if (m >= M) return;
    float r[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      float t = v[i] + (bias ? bias[n0 + i] : 0.0f);
      r[i] = relu ? fmaxf(t, 0.0f) : t;
    }
    if (outf) {
#pragma unroll
      for (int i = 0; i < 16; i += 4)
        *reinterpret_cast<float4 *>(outf + m * BN + n0 + i) = make_float4(r[i], r[i + 1], r[i + 2], r[i + 3]);
    } else {
      __align__(16) bf16 h[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) h[i] = __float2bfloat16_rn(r[i]);
      uint4 *dst = reinterpret_cast<uint4 *>(out + m * BN + n0);
      dst[0] = reinterpret_cast<const uint4 *>(h)[0];
      dst[1] = reinterpret_cast<const uint4 *>(h)[1];
    }
  }
};

// dgrad: the gradient times the ReLU derivative of the layer input (its
// post-activation value > 0), BF16 out
template <int BN>
struct EpiMask {
  const bf16 *mask;  // [M][BN], or null
  bf16 *out;
  long M;
  AW_D void store(long m, int n0, const float (&v)[16]) const {
    if (m >= M) return;
    __align__(16) bf16 h[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const bool on = !mask || __bfloat162float(mask[m * BN + n0 + i]) > 0.0f;
      h[i] = __float2bfloat16_rn(on ? v[i] : 0.0f);
    }
    uint4 *dst = reinterpret_cast<uint4 *>(out + m * BN + n0);
    dst[0] = reinterpret_cast<const uint4 *>(h)[0];
    dst[1] = reinterpret_cast<const uint4 *>(h)[1];
  }
};

// split K of forward / dgrad: FP32 partial of this split, [split][M][BN]
template <int BN>
struct EpiPartial {
  float *part;
  long M;
  AW_D void store(long m, int n0, const float (&v)[16]) const {
    if (m >= M) return;
    float *p = part + ((long)blockIdx.y * M + m) * BN + n0;
#pragma unroll
    for (int i = 0; i < 16; i += 4)
      *reinterpret_cast<float4 *>(p + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
  }
};

// wgrad: FP32 partial of this K split, stored [split][co][(tap,ci)]
template <int BN>
struct EpiWgrad {
  float *part;
  int Mtot;
  AW_D void store(long m, int n0, const float (&v)[16]) const {
    if (m >= Mtot) return;
    float *p = part + (long)blockIdx.y * BN * Mtot;
#pragma unroll
    for (int i = 0; i < 16; ++i) p[(long)(n0 + i) * Mtot + m] = v[i];
  }
};

template <int BN>
constexpr int tmem_cols() {
  return BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
}
// pipeline depth: shared-memory stages of one K step each
template <int BN>
constexpr int gemm_stages() {
  return 3;
}
template <int BN>
constexpr size_t stage_bytes() {
  return (size_t)kAStage + (size_t)BN * kGBK * 2;
}
template <int BN>
constexpr size_t gemm_smem() {
  return 1024 + gemm_stages<BN>() * stage_bytes<BN>();
}

// One CTA: 128 rows x BN columns of D over K in [kbeg, kend). Stage s % S
// of shared memory holds K step s; cp.async keeps S-1 steps in flight while
// one thread issues the MMAs of the oldest, each step's MMAs committed to
// the stage's mbarrier (phase = the step's use count of that stage).
template <int BN, class LA, class LB, class EP>
__global__ void __launch_bounds__(kGThreads)
    k_umma_gemm(LA la, LB lb, EP ep, int K, int k_per_split, int *status) {
  constexpr int S = gemm_stages<BN>();
  extern __shared__ __align__(1024) uint8_t smraw[];
  __shared__ uint64_t mbar[S];
  __shared__ uint32_t tbase;
  uint8_t *base = smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u);
  constexpr int TC = tmem_cols<BN>();
  constexpr uint32_t IDESC = umma_idesc_bf16(kGBM, BN, LA::kMN, LB::kMN);
  const int tid = threadIdx.x, warp = tid >> 5;
  const long m0 = (long)blockIdx.x * kGBM;
  const int kbeg = blockIdx.y * k_per_split;
  const int kend = min(K, kbeg + k_per_split);
  const int nsteps = kend > kbeg ? (kend - kbeg + kGBK - 1) / kGBK : 0;
  auto sA = [&](int st) { return base + st * stage_bytes<BN>(); };
  auto sB = [&](int st) { return base + st * stage_bytes<BN>() + kAStage; };

  if (warp == 0) tmem_alloc(&tbase, TC);
  if (tid == 0)
    for (int i = 0; i < S; ++i) mbar_init(&mbar[i], 1);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tbase;

  const typename LA::Ctx ca = la.init(m0);
  const typename LB::Ctx cb = lb.init(m0);
  __syncthreads();  // per-CTA loader tables
  bool ok = true;
  // steps 0 .. S-2 in flight before the loop; one commit group per step
#pragma unroll
  for (int p = 0; p < S - 1; ++p) {
    if (p < nsteps) {
      la.issue(ca, sA(p), kbeg + p * kGBK, kend);
      lb.issue(cb, sB(p), kbeg + p * kGBK, kend);
    }
    cp_async_commit();
  }
  for (int s = 0; s < nsteps; ++s) {
    const int st = s % S;
    const int nxt = s + S - 1;
    if (nxt < nsteps) {
      // stage nxt % S last held step s - 1: its MMAs must be done
      if (s >= 1) ok = mbar_wait(&mbar[(s - 1) % S], ((s - 1) / S) & 1u, status) && ok;
      la.issue(ca, sA(nxt % S), kbeg + nxt * kGBK, kend);
      lb.issue(cb, sB(nxt % S), kbeg + nxt * kGBK, kend);
    }
    cp_async_commit();
    cp_async_wait<S - 1>();  // this thread's copies of step s have landed
    fence_async_smem();      // and are visible to the tensor core
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a0 = smem_u32(sA(st)), b0 = smem_u32(sB(st));
#pragma unroll
      for (int kk = 0; kk < kGBK / 16; ++kk) {
        const uint64_t da = umma_desc(a0 + kk * 2 * (kGBM * 16), kGBM * 16, 128);
        const uint64_t db = umma_desc(b0 + kk * 2 * (BN * 16), BN * 16, 128);
        umma_bf16(tmem, da, db, IDESC, (s > 0 || kk > 0) ? 1u : 0u);
      }
      umma_commit(&mbar[st]);
    }
  }
  cp_async_wait<0>();
  if (nsteps > 0) {
    const int last = nsteps - 1;
    ok = mbar_wait(&mbar[last % S], (last / S) & 1u, status) && ok;
  }
  tc_fence_after();
  // epilogue: warp w owns TMEM lanes (rows) 32w .. 32w+31
  const long m = m0 + 32 * warp + (tid & 31);
#pragma unroll 1
  for (int c = 0; c < BN / 16; ++c) {
    float v[16];
    tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(16 * c), v);
    if (nsteps == 0 || !ok) {
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = 0.0f;
    }
    ep.store(m, 16 * c, v);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, TC);
}

template <int BN, class LA, class LB, class EP>
cudaError_t launch_gemm(const LA &la, const LB &lb, const EP &ep, long M, int K, int splits,
                        int k_per_split, int *status, cudaStream_t s) {
  const size_t smem = gemm_smem<BN>();
  auto kern = k_umma_gemm<BN, LA, LB, EP>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)((M + kGBM - 1) / kGBM), (unsigned)splits);
  kern<<<grid, kGThreads, smem, s>>>(la, lb, ep, K, k_per_split, status);
  return cudaGetLastError();
}

template <class F>
bool dispatch_bn(int n, F &&f) {
  switch (n) {
    case 16: f(std::integral_constant<int, 16>()); return true;
    case 32: f(std::integral_constant<int, 32>()); return true;
    case 48: f(std::integral_constant<int, 48>()); return true;
    case 64: f(std::integral_constant<int, 64>()); return true;
    case 96: f(std::integral_constant<int, 96>()); return true;
    case 128: f(std::integral_constant<int, 128>()); return true;
    case 192: f(std::integral_constant<int, 192>()); return true;
    default: return false;
  }
}

// ---- elementwise layers ------------------------------------------------------
constexpr int kEw = 256;
inline unsigned ew_grid(long n) { return (unsigned)((n + kEw - 1) / kEw); }

// the sum of split-K partials [splits][M][N] in split order, then the
// forward epilogue (+ bias, ReLU, BF16 or FP32) or the dgrad one (mask)
__global__ void k_splitk_finish(const float *__restrict__ part, int splits, long M, int N,
                                const float *__restrict__ bias, int relu, bf16 *__restrict__ out,
                                float *__restrict__ outf, const bf16 *__restrict__ mask) {
  const long i = (long)blockIdx.x * kEw + threadIdx.x;
  if (i >= M * N) return;
  float t = 0.0f;
  for (int k = 0; k < splits; ++k) t += part[k * M * N + i];
  const int n = (int)(i % N);
  if (bias) t += bias[n];
  if (relu) t = fmaxf(t, 0.0f);
  if (mask && !(__bfloat162float(mask[i]) > 0.0f)) t = 0.0f;
  if (outf)
    outf[i] = t;
  else
    out[i] = __float2bfloat16_rn(t);
}

// 2x2x2 average pooling, channels last; backward spreads dY / 8
__global__ void k_pool_fwd(const bf16 *__restrict__ x, bf16 *__restrict__ y, Vol vo, int C) {
  const long i = (long)blockIdx.x * kEw + threadIdx.x;  // over output voxels * C
  if (i >= vo.voxels() * C) return;
  const int c = (int)(i % C);
  int b, z, yy, xx;
  voxel_coords(vo, (int)(i / C), b, z, yy, xx);
  const int viD = 2 * vo.D, viH = 2 * vo.H, viW = 2 * vo.W;
  float s = 0.0f;
  for (int dz = 0; dz < 2; ++dz)
    for (int dy = 0; dy < 2; ++dy)
      for (int dx = 0; dx < 2; ++dx)
        s += __bfloat162float(
            x[((((long)b * viD + 2 * z + dz) * viH + 2 * yy + dy) * viW + 2 * xx + dx) * C + c]);
  y[i] = __float2bfloat16_rn(0.125f * s);
}
// backward: dx = (dy / 8 + add) where mask > 0 (mask: the pooled
// post-ReLU activation; add, mask may be null)
__global__ void k_pool_bwd(const bf16 *__restrict__ dy, bf16 *__restrict__ dx, Vol vi, int C,
                           const bf16 *__restrict__ add, const bf16 *__restrict__ mask) {
  const long i = (long)blockIdx.x * kEw + threadIdx.x;  // over input voxels * C
  if (i >= vi.voxels() * C) return;
  const int c = (int)(i % C);
  int b, z, y, x;
  voxel_coords(vi, (int)(i / C), b, z, y, x);
  const Vol vo{vi.B, vi.D / 2, vi.H / 2, vi.W / 2};
  float g = 0.125f * __bfloat162float(dy[((((long)b * vo.D + z / 2) * vo.H + y / 2) * vo.W + x / 2) * C + c]);
  if (add) g += __bfloat162float(add[i]);
  if (mask && !(__bfloat162float(mask[i]) > 0.0f)) g = 0.0f;
  dx[i] = __float2bfloat16_rn(g);
}
// nearest x2 upsampling into channels [c0, c0 + C) of a Ct-channel tensor;
// backward sums the 8 children
__global__ void k_up_fwd(const bf16 *__restrict__ x, bf16 *__restrict__ y, Vol vo, int C, int Ct,
                         int c0) {
  const long i = (long)blockIdx.x * kEw + threadIdx.x;  // over output voxels * C
  if (i >= vo.voxels() * C) return;
  const int c = (int)(i % C);
  const long m = i / C;
  int b, z, yy, xx;
  voxel_coords(vo, (int)m, b, z, yy, xx);
  const Vol vi{vo.B, vo.D / 2, vo.H / 2, vo.W / 2};
  y[m * Ct + c0 + c] = x[((((long)b * vi.D + z / 2) * vi.H + yy / 2) * vi.W + xx / 2) * C + c];
}
__global__ void k_up_bwd(const bf16 *__restrict__ dy, bf16 *__restrict__ dx, Vol vi, int C, int Ct,
                         int c0) {
  const long i = (long)blockIdx.x * kEw + threadIdx.x;  // over input (coarse) voxels * C
  if (i >= vi.voxels() * C) return;
  const int c = (int)(i % C);
  int b, z, y, x;
  voxel_coords(vi, (int)(i / C), b, z, y, x);
  const Vol vo{vi.B, 2 * vi.D, 2 * vi.H, 2 * vi.W};
  float s = 0.0f;
  for (int dz = 0; dz < 2; ++dz)
    for (int dyy = 0; dyy < 2; ++dyy)
      for (int dxx = 0; dxx < 2; ++dxx)
        s += __bfloat162float(
            dy[((((long)b * vo.D + 2 * z + dz) * vo.H + 2 * y + dyy) * vo.W + 2 * x + dxx) * Ct + c0 + c]);
  dx[i] = __float2bfloat16_rn(s);
}
// copy C channels into / out of channels [c0, c0 + C) of a Ct-channel tensor
// (the skip half of a concatenation); out += when accumulate
__global__ void k_slice(const bf16 *__restrict__ src, int Cs, int cs0, bf16 *__restrict__ dst,
                        int Cd, int cd0, int C, long voxels, int accumulate) {
  const long i = (long)blockIdx.x * kEw + threadIdx.x;
  if (i >= voxels * C) return;
  const long m = i / C;
  const int c = (int)(i % C);
  float v = __bfloat162float(src[m * Cs + cs0 + c]);
  if (accumulate) v += __bfloat162float(dst[m * Cd + cd0 + c]);
  dst[m * Cd + cd0 + c] = __float2bfloat16_rn(v);
}

// The same three layers eight channels (16 bytes) per thread, for channel
// counts whose 8-channel chunk count is a power of two (lg = its log2) and
// 8-aligned channel offsets: one vector load and store per chunk.
__device__ __forceinline__ void bf8_to_f(const uint4 &u, float (&f)[8]) {
  const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float2 t = __bfloat1622float2(h[k]);
    f[2 * k] = t.x;
    f[2 * k + 1] = t.y;
  }
}
__device__ __forceinline__ uint4 f_to_bf8(const float (&f)[8]) {
  uint4 u;
  __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&u);
#pragma unroll
  for (int k = 0; k < 4; ++k) h[k] = __floats2bfloat162_rn(f[2 * k], f[2 * k + 1]);
  return u;
}
__global__ void k_up_fwd8(const bf16 *__restrict__ x, bf16 *__restrict__ y, Vol vo, int C, int lg,
                          int Ct, int c0) {
  const long i = (long)blockIdx.x * kEw + threadIdx.x;  // over output voxels * C/8
  if (i >= (vo.voxels() << lg)) return;
  const int c = (int)(i & ((1 << lg) - 1)) * 8;
  const long m = i >> lg;
  int b, z, yy, xx;
  voxel_coords(vo, (int)m, b, z, yy, xx);
  const Vol vi{vo.B, vo.D / 2, vo.H / 2, vo.W / 2};
  const uint4 v = __ldg(reinterpret_cast<const uint4 *>(
      x + ((((long)b * vi.D + z / 2) * vi.H + yy / 2) * vi.W + xx / 2) * C + c));
  *reinterpret_cast<uint4 *>(y + m * Ct + c0 + c) = v;
}
__global__ void k_slice8(const bf16 *__restrict__ src, int Cs, int cs0, bf16 *__restrict__ dst,
                         int Cd, int cd0, int lg, long voxels, int accumulate) {
  const long i = (long)blockIdx.x * kEw + threadIdx.x;
  if (i >= (voxels << lg)) return;
  const long m = i >> lg;
  const int c = (int)(i & ((1 << lg) - 1)) * 8;
  uint4 v = __ldg(reinterpret_cast<const uint4 *>(src + m * Cs + cs0 + c));
  uint4 *d = reinterpret_cast<uint4 *>(dst + m * Cd + cd0 + c);
  if (accumulate) {
    float a[8], b[8];
    bf8_to_f(v, a);
    bf8_to_f(*d, b);
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] += b[k];
    v = f_to_bf8(a);
  }
  *d = v;
}
__global__ void k_pool_fwd8(const bf16 *__restrict__ x, bf16 *__restrict__ y, Vol vo, int C, int lg) {
  const long i = (long)blockIdx.x * kEw + threadIdx.x;  // over output voxels * C/8
  if (i >= (vo.voxels() << lg)) return;
  const int c = (int)(i & ((1 << lg) - 1)) * 8;
  const long m = i >> lg;
  int b, z, yy, xx;
  voxel_coords(vo, (int)m, b, z, yy, xx);
  const int viD = 2 * vo.D, viH = 2 * vo.H, viW = 2 * vo.W;
  float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  for (int dz = 0; dz < 2; ++dz)
    for (int dy = 0; dy < 2; ++dy)
      for (int dx = 0; dx < 2; ++dx) {
        float f[8];
        bf8_to_f(__ldg(reinterpret_cast<const uint4 *>(
                     x + ((((long)b * viD + 2 * z + dz) * viH + 2 * yy + dy) * viW + 2 * xx + dx) * C +
                     c)),
                 f);
#pragma unroll
        for (int k = 0; k < 8; ++k) s[k] += f[k];
      }
#pragma unroll
  for (int k = 0; k < 8; ++k) s[k] = 0.125f * s[k];
  *reinterpret_cast<uint4 *>(y + m * C + c) = f_to_bf8(s);
}

inline bool al16(const void *p) { return reinterpret_cast<uintptr_t>(p) % 16 == 0; }

// log2 of C/8 when C is 8 times a power of two, else -1
inline int chunk_lg(int C) {
  if (C <= 0 || C % 8) return -1;
  const int q = C / 8;
  if (q & (q - 1)) return -1;
  int lg = 0;
  while ((1 << lg) < q) ++lg;
  return lg;
}

// (I0, I1) planar float -> channels 0, 1 of a 16-channel BF16 tensor
__global__ void k_pack_pair(const float *__restrict__ a, const float *__restrict__ b,
                            bf16 *__restrict__ x, long voxels) {
  const long m = (long)blockIdx.x * kEw + threadIdx.x;
  if (m >= voxels) return;
  __align__(16) bf16 h[16];
#pragma unroll
  for (int c = 0; c < 16; ++c) h[c] = __float2bfloat16_rn(0.0f);
  h[0] = __float2bfloat16_rn(a[m]);
  h[1] = __float2bfloat16_rn(b[m]);
  uint4 *d = reinterpret_cast<uint4 *>(x + m * 16);
  d[0] = reinterpret_cast<const uint4 *>(h)[0];
  d[1] = reinterpret_cast<const uint4 *>(h)[1];
}

// MSE over the first 3 of 16 prediction channels against a planar target:
// block partial sums of squares and the BF16 gradient 2 (p - t) / (3 V)
__global__ void k_mse(const float *__restrict__ pred, const float *__restrict__ tgt, long voxels,
                      bf16 *__restrict__ grad, double *__restrict__ partials) {
  const long m = (long)blockIdx.x * kEw + threadIdx.x;
  double e = 0.0;
  if (m < voxels) {
    __align__(16) bf16 h[16];
    const float scale = 2.0f / (3.0f * (float)voxels);
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      float g = 0.0f;
      if (c < 3) {
        const float d = pred[m * 16 + c] - tgt[c * voxels + m];
        e += (double)d * d;
        g = scale * d;
      }
      h[c] = __float2bfloat16_rn(g);
    }
    uint4 *dst = reinterpret_cast<uint4 *>(grad + m * 16);
    dst[0] = reinterpret_cast<const uint4 *>(h)[0];
    dst[1] = reinterpret_cast<const uint4 *>(h)[1];
  }
  __shared__ double ws[kEw / 32];
  e = warp_sum(e);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kEw / 32; ++w) t += ws[w];
    partials[blockIdx.x] = t;
  }
}
__global__ void k_sum_partials(const double *__restrict__ p, int n, double scale,
                               float *__restrict__ out) {
  double t = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) t += p[i];
  __shared__ double ws[32];
  t = warp_sum(t);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) s += ws[w];
    *out = (float)(s * scale);
  }
}

// dW = sum over K splits of the partials [split][co][K]
__global__ void k_reduce_splits(const float *__restrict__ part, int splits, long n,
                                float *__restrict__ dw) {
  const long i = (long)blockIdx.x * kEw + threadIdx.x;
  if (i >= n) return;
  float s = 0.0f;
  for (int k = 0; k < splits; ++k) s += part[k * n + i];
  dw[i] = s;
}
// bias gradient: column sums of dY [M][N]; block b sums rows
// [b*kBiasRows, (b+1)*kBiasRows) into part[b][N], then one block adds the
// partials in block order
constexpr int kBiasRows = 512;
__global__ void k_bias_partial(const bf16 *__restrict__ dy, long M, int N, float *__restrict__ part) {
  const int groups = kEw / N;
  const int n = threadIdx.x % N, g = threadIdx.x / N;
  const long r0 = (long)blockIdx.x * kBiasRows, r1 = min(M, r0 + kBiasRows);
  float s = 0.0f;
  if (g < groups)
    for (long m = r0 + g; m < r1; m += groups) s += __bfloat162float(dy[m * N + n]);
  __shared__ float sh[kEw];
  sh[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x < N) {
    float t = 0.0f;
    for (int gg = 0; gg < groups; ++gg) t += sh[gg * N + threadIdx.x];
    part[(long)blockIdx.x * N + threadIdx.x] = t;
  }
}
__global__ void k_bias_final(const float *__restrict__ part, int nb, int N, float *__restrict__ db) {
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    float t = 0.0f;
    for (int b = 0; b < nb; ++b) t += part[(long)b * N + n];
    db[n] = t;
  }
}

// Adam (Kingma & Ba 2015) on the FP32 masters
__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m1,
                       float *__restrict__ m2, long n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  const long i = (long)blockIdx.x * kEw + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float a = b1 * m1[i] + (1.0f - b1) * gi;
  const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = b;
  w[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}
// BF16 weights [co][tap][ci] and the dgrad copy [ci][tap][co]
__global__ void k_weights_bf16(const float *__restrict__ w, int cout, int ntaps, int cin,
                               bf16 *__restrict__ wb, bf16 *__restrict__ wt) {
  const long i = (long)blockIdx.x * kEw + threadIdx.x;
  const long n = (long)cout * ntaps * cin;
  if (i >= n) return;
  const int ci = (int)(i % cin);
  const long r = i / cin;
  const int tap = (int)(r % ntaps), co = (int)(r / ntaps);
  const bf16 v = __float2bfloat16_rn(w[i]);
  wb[i] = v;
  if (wt) wt[((long)ci * ntaps + tap) * cout + co] = v;
}

// h = identity + the first 3 prediction channels (the warm start)
__global__ void k_disp_to_h(const float *__restrict__ pred, Vol v, float *__restrict__ hx,
                            float *__restrict__ hy, float *__restrict__ hz) {
  const long m = (long)blockIdx.x * kEw + threadIdx.x;
  if (m >= v.voxels()) return;
  int b, z, y, x;
  voxel_coords(v, (int)m, b, z, y, x);
  hx[m] = (float)x + pred[m * 16 + 0];
  hy[m] = (float)y + pred[m * 16 + 1];
  hz[m] = (float)z + pred[m * 16 + 2];
}

// ---- direct 3x3x3 convolution from a TMA-staged halo tile ------------------
// For the wide, shallow layers (16-48 channels) the im2col gather of the
// GEMM above costs ten times the tensor and HBM work. Here a CTA owns an
// output tile of 8 (x) x 16 (y) voxels x ZT planes of one batch item; the
// input box it needs — CIN/8 chunks of 8 channels, each [ZT+2][18][10]
// cells of 16 bytes — arrives by TMA tensor loads, zero-filled outside the
// volume. Row r = x + 8y of a 128-row MMA tile is voxel (x, y), so for tap
// (dz, dy, dx) and plane zz the A operand is that box shifted by
// (dx, dy, zz + dz): core matrix i (row group y = i) starts at cell
// (dx, i + dy, zz + dz), 160 bytes apart, its 8 rows (x) 16 bytes apart in
// one contiguous 128-byte run, and the two 8-channel chunks of a K = 16
// step one region apart. One MMA per (plane, tap, 16 input channels), no
// operand copy at all; the weights sit in shared memory in the canonical
// K-major layout; each plane accumulates in its own COUT TMEM columns.
// Small shared footprint, one tile per CTA, several CTAs per SM: the TMA
// loads, MMAs and epilogues of co-resident CTAs overlap. (A persistent
// double-buffered variant measured slower here: with N = 16 the MMAs are
// bound by reading the 4 KB A operand from shared memory, and fewer
// resident CTAs left that bandwidth idle between tiles.)
template <int CIN, int COUT, int ZT>
struct DirectCfg {
  static constexpr int NCH = CIN / 8;
  static constexpr int CELLS = 10 * 18 * (ZT + 2);
  static constexpr int BOX_BYTES = CELLS * 16;
  static constexpr int REGION = (BOX_BYTES + 127) / 128 * 128;
  static constexpr int IN_BYTES = NCH * REGION;
  static constexpr int W_BYTES = 27 * CIN * COUT * 2;  // a multiple of 128
  static constexpr int COLS = ZT * COUT;
  static constexpr int TMEM_COLS = COLS <= 32 ? 32 : COLS <= 64 ? 64 : COLS <= 128 ? 128 : 256;
  static constexpr size_t smem() { return 1024 + (size_t)IN_BYTES + W_BYTES; }
  static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COLS <= 256, "direct conv shape");
};

template <int CIN, int COUT, int ZT>
__global__ void __launch_bounds__(128)
    k_conv_direct(const __grid_constant__ CUtensorMap tmap, const bf16 *__restrict__ w,
                  const float *__restrict__ bias, int relu, bf16 *__restrict__ out,
                  float *__restrict__ outf, int D, int H, int W, int *status) {
  using C = DirectCfg<CIN, COUT, ZT>;
  extern __shared__ __align__(1024) uint8_t smraw[];
  __shared__ uint64_t mbar[2];  // 0: input box landed, 1: MMAs done
  __shared__ uint32_t tbase;
  __shared__ int s_ok;
  uint8_t *base = smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u);
  uint8_t *sW = base, *sIn = base + C::W_BYTES;
  constexpr uint32_t IDESC = umma_idesc_bf16(128, COUT, 0, 0);
  const int tid = threadIdx.x, warp = tid >> 5;
  // tile coordinates: x fastest, then y, z, batch
  const int tx = W / 8, ty = H / 16, tz = D / ZT;
  int t = blockIdx.x;
  const int x0 = (t % tx) * 8;
  t /= tx;
  const int y0 = (t % ty) * 16;
  t /= ty;
  const int z0 = (t % tz) * ZT;
  const int b = t / tz;

  if (warp == 0) tmem_alloc(&tbase, C::TMEM_COLS);
  if (tid == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tbase;
  if (tid == 0) {
    mbar_expect_tx(&mbar[0], (uint32_t)(C::NCH * C::BOX_BYTES));
#pragma unroll 1
    for (int j = 0; j < C::NCH; ++j)
      tma_load_5d(sIn + j * C::REGION, &tmap, 8 * j, x0 - 1, y0 - 1, z0 - 1, b, &mbar[0]);
  }
  // weights [COUT][27][CIN] -> chunk (tap, j, n) at ((tap*NCH + j)*(COUT/8) + n/8)*128 +
  // (n%8)*16 = 16 c for c = (tap*NCH + j)*COUT + n: consecutive threads, consecutive chunks
#pragma unroll 1
  for (int c = tid; c < COUT * 27 * C::NCH; c += 128) {
    const int n = c % COUT, r = c / COUT;
    const int j = r % C::NCH, tap = r / C::NCH;
    const uint4 val = __ldg(reinterpret_cast<const uint4 *>(w + ((long)n * 27 + tap) * CIN + 8 * j));
    *reinterpret_cast<uint4 *>(sW + 16 * c) = val;
  }
  fence_async_smem();
  __syncthreads();
  if (tid == 0) {
    s_ok = mbar_wait(&mbar[0], 0, status) ? 1 : 0;
    if (s_ok) {
      tc_fence_after();
      const uint32_t a0 = smem_u32(sIn), b0 = smem_u32(sW);
#pragma unroll 1
      for (int zz = 0; zz < ZT; ++zz) {
#pragma unroll 1
        for (int tap = 0; tap < 27; ++tap) {
          const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
          const uint32_t cell = (uint32_t)((((zz + dz) * 18 + dy) * 10 + dx) * 16);
#pragma unroll
          for (int jp = 0; jp < C::NCH / 2; ++jp) {
            const uint64_t da = umma_desc(a0 + 2 * jp * C::REGION + cell, C::REGION, 160);
            const uint64_t db =
                umma_desc(b0 + (tap * C::NCH + 2 * jp) * (COUT / 8) * 128, COUT * 16, 128);
            umma_bf16(tmem + (uint32_t)(zz * COUT), da, db, IDESC, (tap | jp) ? 1u : 0u);
          }
        }
      }
      umma_commit(&mbar[1]);
    }
  }
  __syncthreads();
  const bool ok = s_ok && mbar_wait(&mbar[1], 0, status);
  tc_fence_after();
  // epilogue: warp w owns TMEM lanes 32w .. 32w+31 = rows r = x + 8y
  const int r = 32 * warp + (tid & 31);
  const int x = x0 + (r & 7), y = y0 + (r >> 3);
#pragma unroll 1
  for (int zz = 0; zz < ZT; ++zz) {
    const long m = (((long)b * D + z0 + zz) * H + y) * W + x;
#pragma unroll
    for (int g = 0; g < COUT / 16; ++g) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(zz * COUT + 16 * g), v);
      float o[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float tv = ok ? v[i] + (bias ? bias[16 * g + i] : 0.0f) : 0.0f;
        o[i] = relu ? fmaxf(tv, 0.0f) : tv;
      }
      if (outf) {
#pragma unroll
        for (int i = 0; i < 16; i += 4)
          *reinterpret_cast<float4 *>(outf + m * COUT + 16 * g + i) =
              make_float4(o[i], o[i + 1], o[i + 2], o[i + 3]);
      } else {
        __align__(16) bf16 h[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) h[i] = __float2bfloat16_rn(o[i]);
        uint4 *dst = reinterpret_cast<uint4 *>(out + m * COUT + 16 * g);
        dst[0] = reinterpret_cast<const uint4 *>(h)[0];
        dst[1] = reinterpret_cast<const uint4 *>(h)[1];
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, C::TMEM_COLS);
}


template <int CIN, int COUT, int ZT>
cudaError_t launch_direct(const void *x, int B, int D, int H, int W, const void *w,
                          const float *bias, int relu, void *out, float *outf, int *status,
                          cudaStream_t s) {
  using C = DirectCfg<CIN, COUT, ZT>;
  PFN_cuTensorMapEncodeTiled encode = tensor_map_encoder();
  if (!encode) return cudaErrorNotSupported;
  CUtensorMap tmap;
  const cuuint64_t dims[5] = {(cuuint64_t)CIN, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)D,
                              (cuuint64_t)B};
  const cuuint64_t strides[4] = {(cuuint64_t)CIN * 2, (cuuint64_t)W * CIN * 2,
                                 (cuuint64_t)H * W * CIN * 2, (cuuint64_t)D * H * W * CIN * 2};
  const cuuint32_t box[5] = {8, 10, 18, (cuuint32_t)(ZT + 2), 1};
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  if (reinterpret_cast<uintptr_t>(x) % 16 || reinterpret_cast<uintptr_t>(w) % 16 ||
      encode(&tmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void *>(x), dims, strides, box,
             estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return cudaErrorNotSupported;
  auto kern = k_conv_direct<CIN, COUT, ZT>;
  cudaError_t e =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::smem());
  if (e != cudaSuccess) return e;
  const unsigned grid = (unsigned)((long)B * (D / ZT) * (H / 16) * (W / 8));
  kern<<<grid, 128, C::smem(), s>>>(tmap, static_cast<const bf16 *>(w), bias, relu,
                                     static_cast<bf16 *>(out), outf, D, H, W, status);
  return cudaGetLastError();
}

template <int CIN, int COUT>
size_t direct_smem(int zt) {
  return zt == 4 ? DirectCfg<CIN, COUT, 4>::smem()
                 : zt == 2 ? DirectCfg<CIN, COUT, 2>::smem() : DirectCfg<CIN, COUT, 1>::smem();
}

// planes per tile for the direct kernel (0: the GEMM path): the deepest tile
// whose grid still gives two CTAs per SM, else the shallowest (the most
// CTAs), within two CTAs' shared memory per SM
int direct_planes(int cin, int cout, int ntaps, int B, int D, int H, int W, int sms) {
  // the input box (10 x 18 x (planes + 2) voxels) stays within the tensor's extents
  if (ntaps != 27 || W % 8 || H % 16 || W < 16 || H < 32 || B < 1 || D < 3) return 0;
  size_t (*smem)(int) = nullptr;
  if (cin == 16 && cout == 16) smem = direct_smem<16, 16>;
  else if (cin == 48 && cout == 16) smem = direct_smem<48, 16>;
  else if (cin == 16 && cout == 32) smem = direct_smem<16, 32>;
  else if (cin == 32 && cout == 32) smem = direct_smem<32, 32>;
  if (!smem) return 0;
  int shallowest = 0;
  for (int zt : {4, 2, 1}) {
    if (D % zt || D < zt + 2 || smem(zt) > 113u * 1024u) continue;
    shallowest = zt;
    if ((long)B * (D / zt) * (H / 16) * (W / 8) >= 2L * sms) return zt;
  }
  return shallowest;
}

template <int CIN, int COUT>
cudaError_t direct_zt(int zt, const void *x, int B, int D, int H, int W, const void *w,
                      const float *bias, int relu, void *out, float *outf, int *status,
                      cudaStream_t s) {
  if (zt == 4) return launch_direct<CIN, COUT, 4>(x, B, D, H, W, w, bias, relu, out, outf, status, s);
  if (zt == 2) return launch_direct<CIN, COUT, 2>(x, B, D, H, W, w, bias, relu, out, outf, status, s);
  return launch_direct<CIN, COUT, 1>(x, B, D, H, W, w, bias, relu, out, outf, status, s);
}

cudaError_t conv_direct(int zt, const void *x, int B, int D, int H, int W, int cin, const void *w,
                        const float *bias, int cout, int relu, void *out, float *outf,
                        int *status, cudaStream_t s) {
  if (cin == 16 && cout == 16)
    return direct_zt<16, 16>(zt, x, B, D, H, W, w, bias, relu, out, outf, status, s);
  if (cin == 48 && cout == 16)
    return direct_zt<48, 16>(zt, x, B, D, H, W, w, bias, relu, out, outf, status, s);
  if (cin == 16 && cout == 32)
    return direct_zt<16, 32>(zt, x, B, D, H, W, w, bias, relu, out, outf, status, s);
  if (cin == 32 && cout == 32)
    return direct_zt<32, 32>(zt, x, B, D, H, W, w, bias, relu, out, outf, status, s);
  return cudaErrorInvalidValue;
}

}  // namespace

// ---- host entry points (called from capi.cu) ---------------------------------
// 1: every forward convolution on the implicit-GEMM kernel (the direct
// kernel off), for comparing the two paths; process-wide
static int g_gemm_only = 0;
void nn_set_gemm_only(int on) { g_gemm_only = on ? 1 : 0; }

int nn_conv_direct_planes(int B, int D, int H, int W, int cin, int cout, int ntaps) {
  if (g_gemm_only) return 0;
  int sms = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return direct_planes(cin, cout, ntaps, B, D, H, W, sms);
}

bool nn_channels_ok(int c) { return dispatch_bn(c, [](auto) {}); }

// K splits for a GEMM of `mtiles` row tiles and `ksteps` 64-deep steps:
// about four CTAs per SM, at least two steps per split
inline int choose_splits(long mtiles, int ksteps, int sms) {
  const long target = 4L * sms;  // CTAs
  if (mtiles * 2 > target) return 1;
  long want = (target + mtiles - 1) / mtiles;
  long maxs = ksteps / 2;
  long sp = want < maxs ? want : maxs;
  return sp < 1 ? 1 : (int)sp;
}

size_t nn_splitk_floats(long M, int N, int K) {
  const int sp = choose_splits((M + kGBM - 1) / kGBM, (K + kGBK - 1) / kGBK, 148);
  return sp > 1 ? (size_t)sp * M * N : 0;
}

// the conv GEMM of forward (sign +1) or dgrad (-1), split over K when the
// row tiles alone cannot fill the GPU and the scratch allows
template <class EPI_DIRECT>
cudaError_t conv_gemm(const void *a, const Vol &v, int ca, int ntaps, int sign, const void *b,
                      int N, long M, const float *bias, int relu, void *out, float *outf,
                      const void *mask, float *scratch, size_t scratch_floats, int *status,
                      cudaStream_t s) {
  const int K = ntaps * ca;
  int sms = 148;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long mtiles = (M + kGBM - 1) / kGBM;
  const int ksteps = (K + kGBK - 1) / kGBK;
  int splits = choose_splits(mtiles, ksteps, sms);
  const int per = ((ksteps + splits - 1) / splits) * kGBK;
  splits = (K + per - 1) / per;
  if (splits > 1 && (!scratch || scratch_floats < (size_t)splits * M * N)) splits = 1;
  cudaError_t e = cudaErrorInvalidValue;
  dispatch_bn(N, [&](auto BNc) {
    constexpr int BN = decltype(BNc)::value;
    LoadConvA la{static_cast<const bf16 *>(a), v, ca, ntaps, sign, (int)M, make_fastdiv(ca)};
    LoadRowsB<BN> lb{static_cast<const bf16 *>(b), K};
    if (splits > 1) {
      EpiPartial<BN> ep{scratch, M};
      e = launch_gemm<BN>(la, lb, ep, M, K, splits, per, status, s);
      if (e == cudaSuccess) {
        k_splitk_finish<<<ew_grid(M * BN), kEw, 0, s>>>(
            scratch, splits, M, BN, bias, relu, static_cast<bf16 *>(out), outf,
            static_cast<const bf16 *>(mask));
        e = cudaGetLastError();
      }
    } else if (EPI_DIRECT::kForward) {
      EpiAct<BN> ep{bias, static_cast<bf16 *>(out), outf, relu, M};
      e = launch_gemm<BN>(la, lb, ep, M, K, 1, K, status, s);
    } else {
      EpiMask<BN> ep{static_cast<const bf16 *>(mask), static_cast<bf16 *>(out), M};
      e = launch_gemm<BN>(la, lb, ep, M, K, 1, K, status, s);
    }
  });
  return e;
}
struct FwdTag { static constexpr bool kForward = true; };
struct DgradTag { static constexpr bool kForward = false; };

cudaError_t nn_conv_fwd(const void *x, int B, int D, int H, int W, int cin, const void *w,
                        const float *bias, int cout, int ntaps, int relu, void *out,
                        float *outf, float *scratch, size_t scratch_floats, int *status,
                        cudaStream_t s) {
  const long M = (long)B * D * H * W;
  const int zt = nn_conv_direct_planes(B, D, H, W, cin, cout, ntaps);
  if (zt > 0) {
    // cudaErrorNotSupported: no tensor map for this tensor (nothing launched)
    const cudaError_t e =
        conv_direct(zt, x, B, D, H, W, cin, w, bias, cout, relu, out, outf, status, s);
    if (e != cudaErrorNotSupported) return e;
  }
  return conv_gemm<FwdTag>(x, make_vol(B, D, H, W), cin, ntaps, 1, w, cout, M, bias, relu, out,
                           outf, nullptr, scratch, scratch_floats, status, s);
}

cudaError_t nn_conv_dgrad(const void *dy, int B, int D, int H, int W, int cout, const void *wt,
                          int cin, int ntaps, const void *mask, void *dx, float *scratch,
                          size_t scratch_floats, int *status, cudaStream_t s) {
  const long M = (long)B * D * H * W;
  return conv_gemm<DgradTag>(dy, make_vol(B, D, H, W), cout, ntaps, -1, wt, cin, M, nullptr, 0,
                             dx, nullptr, mask, scratch, scratch_floats, status, s);
}

size_t nn_wgrad_part_floats(int cin, int cout, int ntaps, int splits) {
  return (size_t)splits * cout * ntaps * cin;
}

cudaError_t nn_conv_wgrad(const void *x, const void *dy, int B, int D, int H, int W, int cin,
                          int cout, int ntaps, int splits, float *part, float *dw, int *status,
                          cudaStream_t s) {
  const Vol v = make_vol(B, D, H, W);
  const long voxels = (long)B * D * H * W;
  const int Mtot = ntaps * cin;
  long per = (voxels + splits - 1) / splits;
  per = ((per + kGBK - 1) / kGBK) * kGBK;
  splits = (int)((voxels + per - 1) / per);
  cudaError_t e = cudaErrorInvalidValue;
  dispatch_bn(cout, [&](auto BNc) {
    constexpr int BN = decltype(BNc)::value;
    LoadWgradA la{static_cast<const bf16 *>(x), v, cin, ntaps, Mtot, make_fastdiv(cin)};
    LoadWgradB<BN> lb{static_cast<const bf16 *>(dy)};
    EpiWgrad<BN> ep{part, Mtot};
    e = launch_gemm<BN>(la, lb, ep, Mtot, (int)voxels, splits, (int)per, status, s);
  });
  if (e != cudaSuccess) return e;
  const long n = (long)cout * Mtot;
  k_reduce_splits<<<ew_grid(n), kEw, 0, s>>>(part, splits, n, dw);
  return cudaGetLastError();
}

size_t nn_bias_scratch_floats(long M, int N) {
  return (size_t)((M + kBiasRows - 1) / kBiasRows) * N;
}

cudaError_t nn_bias_grad(const void *dy, long M, int N, float *scratch, float *db, cudaStream_t s) {
  const int nb = (int)((M + kBiasRows - 1) / kBiasRows);
  k_bias_partial<<<nb, kEw, 0, s>>>(static_cast<const bf16 *>(dy), M, N, scratch);
  k_bias_final<<<1, 256, 0, s>>>(scratch, nb, N, db);
  return cudaGetLastError();
}

cudaError_t nn_pool(const void *in, int B, int D, int H, int W, int C, void *out, int backward,
                    const void *add, const void *mask, cudaStream_t s) {
  // forward: (D,H,W) is the input grid; backward: the input-gradient grid
  if (!backward) {
    const Vol vo = make_vol(B, D / 2, H / 2, W / 2);
    const int lg = al16(in) && al16(out) ? chunk_lg(C) : -1;
    if (lg >= 0)
      k_pool_fwd8<<<ew_grid(vo.voxels() << lg), kEw, 0, s>>>(static_cast<const bf16 *>(in),
                                                             static_cast<bf16 *>(out), vo, C, lg);
    else
      k_pool_fwd<<<ew_grid(vo.voxels() * C), kEw, 0, s>>>(static_cast<const bf16 *>(in),
                                                          static_cast<bf16 *>(out), vo, C);
  } else {
    const Vol vi = make_vol(B, D, H, W);
    k_pool_bwd<<<ew_grid(vi.voxels() * C), kEw, 0, s>>>(static_cast<const bf16 *>(in),
                                                        static_cast<bf16 *>(out), vi, C,
                                                        static_cast<const bf16 *>(add),
                                                        static_cast<const bf16 *>(mask));
  }
  return cudaGetLastError();
}

cudaError_t nn_upsample(const void *in, int B, int D, int H, int W, int C, void *out, int Ct,
                        int c0, int backward, cudaStream_t s) {
  // (D,H,W) is the coarse grid in both directions
  const Vol vc = make_vol(B, D, H, W);
  const Vol vf = make_vol(B, 2 * D, 2 * H, 2 * W);
  const int lg = al16(in) && al16(out) ? chunk_lg(C) : -1;
  if (!backward && lg >= 0 && Ct % 8 == 0 && c0 % 8 == 0)
    k_up_fwd8<<<ew_grid(vf.voxels() << lg), kEw, 0, s>>>(static_cast<const bf16 *>(in),
                                                         static_cast<bf16 *>(out), vf, C, lg, Ct,
                                                         c0);
  else if (!backward)
    k_up_fwd<<<ew_grid(vf.voxels() * C), kEw, 0, s>>>(static_cast<const bf16 *>(in),
                                                      static_cast<bf16 *>(out), vf, C, Ct, c0);
  else
    k_up_bwd<<<ew_grid(vc.voxels() * C), kEw, 0, s>>>(static_cast<const bf16 *>(in),
                                                      static_cast<bf16 *>(out), vc, C, Ct, c0);
  return cudaGetLastError();
}

cudaError_t nn_slice(const void *src, int Cs, int cs0, void *dst, int Cd, int cd0, int C,
                     long voxels, int accumulate, cudaStream_t s) {
  const int lg = al16(src) && al16(dst) ? chunk_lg(C) : -1;
  if (lg >= 0 && Cs % 8 == 0 && cs0 % 8 == 0 && Cd % 8 == 0 && cd0 % 8 == 0)
    k_slice8<<<ew_grid(voxels << lg), kEw, 0, s>>>(static_cast<const bf16 *>(src), Cs, cs0,
                                                    static_cast<bf16 *>(dst), Cd, cd0, lg, voxels,
                                                    accumulate);
  else
    k_slice<<<ew_grid(voxels * C), kEw, 0, s>>>(static_cast<const bf16 *>(src), Cs, cs0,
                                                 static_cast<bf16 *>(dst), Cd, cd0, C, voxels,
                                                 accumulate);
  return cudaGetLastError();
}

cudaError_t nn_pack_pair(const float *a, const float *b, long voxels, void *x, cudaStream_t s) {
  k_pack_pair<<<ew_grid(voxels), kEw, 0, s>>>(a, b, static_cast<bf16 *>(x), voxels);
  return cudaGetLastError();
}

size_t nn_mse_partials(long voxels) { return ew_grid(voxels); }

cudaError_t nn_mse(const float *pred, const float *tgt, long voxels, void *grad, double *partials,
                   float *loss, cudaStream_t s) {
  const unsigned g = ew_grid(voxels);
  k_mse<<<g, kEw, 0, s>>>(pred, tgt, voxels, static_cast<bf16 *>(grad), partials);
  k_sum_partials<<<1, 1024, 0, s>>>(partials, (int)g, 1.0 / (3.0 * (double)voxels), loss);
  return cudaGetLastError();
}

cudaError_t nn_adam(float *w, const float *g, float *m1, float *m2, long n, float lr, float b1,
                    float b2, float eps, int t, cudaStream_t s) {
  const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
  k_adam<<<ew_grid(n), kEw, 0, s>>>(w, g, m1, m2, n, lr, b1, b2, eps, c1, c2);
  return cudaGetLastError();
}

cudaError_t nn_weights_bf16(const float *w, int cout, int ntaps, int cin, void *wb, void *wt,
                            cudaStream_t s) {
  const long n = (long)cout * ntaps * cin;
  k_weights_bf16<<<ew_grid(n), kEw, 0, s>>>(w, cout, ntaps, cin, static_cast<bf16 *>(wb),
                                            static_cast<bf16 *>(wt));
  return cudaGetLastError();
}

cudaError_t nn_disp_to_h(const float *pred, int D, int H, int W, float *hx, float *hy, float *hz,
                         cudaStream_t s) {
  const Vol v = make_vol(1, D, H, W);
  k_disp_to_h<<<ew_grid(v.voxels()), kEw, 0, s>>>(pred, v, hx, hy, hz);
  return cudaGetLastError();
}

}  // namespace aw
