// fluid_fast.cu — the fluid-operator kernels for power-of-two axes
// (16..256), with register-resident line FFTs (fft_reg.cuh).
//
// Same three passes as fluid.cu (xy-forward, z-solve, xy-inverse) and the
// same arithmetic definition; the layout of work differs:
//  * xy kernels: one 512-thread CTA per (z-slab, component); x-lines are
//    row pairs packed as one complex line; the kx = 0 and kx = nx/2 columns
//    (real after the x-transform) are packed into one complex y-line, so a
//    128 x 128 slab is exactly 64 x-lines + 64 y-lines.
//  * z kernel: one CTA per Kq consecutive (ky,kx) columns, all three
//    components, lines loaded straight from HBM into registers.
#include "fft_reg.cuh"
#include "fluid.cuh"
#include "fluid_fast.cuh"

namespace aw {

namespace {

constexpr int kXYThreads = 512;
constexpr int kXYWarps = kXYThreads / 32;

template <int NX, int NY>
struct XYShape {
  static constexpr int NXH = NX / 2 + 1;
  static constexpr int TX = LineCfg<NX>::T, EX = LineCfg<NX>::E;
  static constexpr int TY = LineCfg<NY>::T, EY = LineCfg<NY>::E;
  static constexpr int LSX = line_scratch<NX>(), LSY = line_scratch<NY>();
  static constexpr int LS = LSX > LSY ? LSX : LSY;
  static constexpr int LPW = 32 / (TX < TY ? TX : TY);  // max lines per warp
  static constexpr size_t smem() {
    return sizeof(float2) * ((size_t)NY * NXH + (size_t)kXYWarps * LPW * LS);
  }
};

template <int NX, int NY, class Src>
__global__ void __launch_bounds__(kXYThreads) k_xy_fwd_fast(FluidPlan p, Src src) {
  using S = XYShape<NX, NY>;
  constexpr int NXH = S::NXH, TX = S::TX, EX = S::EX, TY = S::TY, EY = S::EY;
  extern __shared__ float2 sm[];
  float2 *C = sm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2 *wscr = C + NY * NXH + warp * S::LPW * S::LS;
  const Dims d = p.d;
  const int z = blockIdx.x, comp = blockIdx.y;

  // ---- x: row pairs (y0, y1) as one complex line -------------------------
  {
    constexpr int L = 32 / TX;
    const int lw = lane / TX, t = lane % TX;
    float2 *scr = wscr + lw * S::LS;
    for (int base = warp * L; base < NY / 2; base += kXYWarps * L) {
      const int pr = base + lw;
      const bool act = pr < NY / 2;
      const int y0 = 2 * (act ? pr : 0);
      float2 v[EX];
#pragma unroll
      for (int j = 0; j < EX; ++j) {
        const int x = t + TX * j;
        v[j] = make_float2(src.value(comp, x, y0, z, d), src.value(comp, x, y0 + 1, z, d));
      }
      line_fft<NX, -1>(v, t, scr, p.ax.tw);
#pragma unroll
      for (int r = 0; r < EX; ++r) scr[line_out_index<NX>(t, r)] = v[r];
      __syncwarp();
      if (act) {
        for (int k = t; k < NXH; k += TX) {
          const float2 Z = scr[k], Zm = scr[(NX - k) & (NX - 1)];
          C[y0 * NXH + k] = make_float2(0.5f * (Z.x + Zm.x), 0.5f * (Z.y - Zm.y));
          C[(y0 + 1) * NXH + k] = make_float2(0.5f * (Z.y + Zm.y), -0.5f * (Z.x - Zm.x));
        }
      }
      __syncwarp();
    }
  }
  __syncthreads();

  // ---- y: columns kx = 1..NX/2-1, plus the packed real columns 0 | NX/2 ---
  {
    constexpr int L = 32 / TY;
    const int lw = lane / TY, t = lane % TY;
    float2 *scr = wscr + lw * S::LS;
    constexpr int NL = NXH - 1;  // lines
    for (int base = warp * L; base < NL; base += kXYWarps * L) {
      const int l = base + lw;
      const bool act = l < NL;
      const bool packed = (l == 0);
      const int kx = act ? l : 1;
      float2 v[EY];
#pragma unroll
      for (int j = 0; j < EY; ++j) {
        const int y = t + TY * j;
        v[j] = packed ? make_float2(C[y * NXH].x, C[y * NXH + NX / 2].x) : C[y * NXH + kx];
      }
      line_fft<NY, -1>(v, t, scr, p.ay.tw);
      if (packed) {
#pragma unroll
        for (int r = 0; r < EY; ++r) scr[line_out_index<NY>(t, r)] = v[r];
      }
      __syncwarp();
      if (act && !packed) {
#pragma unroll
        for (int r = 0; r < EY; ++r) C[line_out_index<NY>(t, r) * NXH + kx] = v[r];
      } else if (packed) {
        for (int k = t; k < NY; k += TY) {
          const float2 Z = scr[k], Zm = scr[(NY - k) & (NY - 1)];
          C[k * NXH] = make_float2(0.5f * (Z.x + Zm.x), 0.5f * (Z.y - Zm.y));
          C[k * NXH + NX / 2] = make_float2(0.5f * (Z.y + Zm.y), -0.5f * (Z.x - Zm.x));
        }
      }
      __syncwarp();
    }
  }
  __syncthreads();

  // ---- store the slab: contiguous, 16-byte vectors ------------------------
  const float4 *c4 = reinterpret_cast<const float4 *>(C);
  float4 *o4 = reinterpret_cast<float4 *>(p.spec + ((long)comp * d.nz + z) * NY * NXH);
  for (int i = threadIdx.x; i < NY * NXH / 2; i += kXYThreads) o4[i] = c4[i];
}

template <int NX, int NY, class Dst>
__global__ void __launch_bounds__(kXYThreads) k_xy_inv_fast(FluidPlan p, Dst dst) {
  using S = XYShape<NX, NY>;
  constexpr int NXH = S::NXH, TX = S::TX, EX = S::EX, TY = S::TY, EY = S::EY;
  extern __shared__ float2 sm[];
  float2 *C = sm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2 *wscr = C + NY * NXH + warp * S::LPW * S::LS;
  const Dims d = p.d;
  const int z = blockIdx.x, comp = blockIdx.y;
  {
    float4 *c4 = reinterpret_cast<float4 *>(C);
    const float4 *i4 = reinterpret_cast<const float4 *>(p.spec + ((long)comp * d.nz + z) * NY * NXH);
    for (int i = threadIdx.x; i < NY * NXH / 2; i += kXYThreads) c4[i] = i4[i];
  }
  __syncthreads();

  // ---- inverse y on columns; packed real columns 0 | NX/2 -----------------
  {
    constexpr int L = 32 / TY;
    const int lw = lane / TY, t = lane % TY;
    float2 *scr = wscr + lw * S::LS;
    constexpr int NL = NXH - 1;
    for (int base = warp * L; base < NL; base += kXYWarps * L) {
      const int l = base + lw;
      const bool act = l < NL;
      const bool packed = (l == 0);
      const int kx = act ? l : 1;
      float2 v[EY];
#pragma unroll
      for (int j = 0; j < EY; ++j) {
        const int y = t + TY * j;
        if (packed) {
          const float2 a = C[y * NXH], b = C[y * NXH + NX / 2];
          v[j] = make_float2(a.x - b.y, a.y + b.x);  // a + i b
        } else {
          v[j] = C[y * NXH + kx];
        }
      }
      __syncwarp();
      line_fft<NY, +1>(v, t, scr, p.ay.tw);
      if (act) {
#pragma unroll
        for (int r = 0; r < EY; ++r) {
          const int y = line_out_index<NY>(t, r);
          if (packed) {
            // real parts of the two columns; c2r ignores their imaginary parts
            C[y * NXH] = make_float2(v[r].x, 0.f);
            C[y * NXH + NX / 2] = make_float2(v[r].y, 0.f);
          } else {
            C[y * NXH + kx] = v[r];
          }
        }
      }
      __syncwarp();
    }
  }
  __syncthreads();

  // ---- inverse x: row pairs, Hermitian completion, real output ------------
  {
    constexpr int L = 32 / TX;
    const int lw = lane / TX, t = lane % TX;
    float2 *scr = wscr + lw * S::LS;
    for (int base = warp * L; base < NY / 2; base += kXYWarps * L) {
      const int pr = base + lw;
      const bool act = pr < NY / 2;
      const int y0 = 2 * (act ? pr : 0);
      float2 v[EX];
#pragma unroll
      for (int j = 0; j < EX; ++j) {
        const int k = t + TX * j;
        const bool upper = k > NX / 2;
        const int kk = upper ? NX - k : k;
        float2 X0 = C[y0 * NXH + kk], X1 = C[(y0 + 1) * NXH + kk];
        if (kk == 0 || kk == NX / 2) { X0.y = 0.f; X1.y = 0.f; }
        if (upper) { X0.y = -X0.y; X1.y = -X1.y; }
        v[j] = make_float2(X0.x - X1.y, X0.y + X1.x);
      }
      line_fft<NX, +1>(v, t, scr, p.ax.tw);
      if (act) {
#pragma unroll
        for (int r = 0; r < EX; ++r) {
          const int x = line_out_index<NX>(t, r);
          dst.store(comp, d.idx(x, y0, z), v[r].x);
          dst.store(comp, d.idx(x, y0 + 1, z), v[r].y);
        }
      }
    }
  }
}

template <int NZ>
__global__ void __launch_bounds__(768) k_z_solve_fast(FluidPlan p, int inverse, int Kq) {
  constexpr int T = LineCfg<NZ>::T, E = LineCfg<NZ>::E, LS = line_scratch<NZ>();
  extern __shared__ float2 sm[];
  const int nxh = p.nxh;
  const long ncols = (long)p.d.ny * nxh;
  const long j0 = (long)blockIdx.x * Kq;
  const long plane = ncols;
  const int line = threadIdx.x / T, t = threadIdx.x % T;  // line = c*Kq + q
  const int c = line / Kq, q = line - c * Kq;
  const bool act = (j0 + q) < ncols;
  const long col = act ? j0 + q : j0;
  float2 *S = sm + line * LS;
  float2 v[E];
#pragma unroll
  for (int j = 0; j < E; ++j) v[j] = p.spec[((long)c * NZ + t + T * j) * plane + col];
  line_fft<NZ, -1>(v, t, S, p.az.tw);
#pragma unroll
  for (int r = 0; r < E; ++r) S[line_out_index<NZ>(t, r)] = v[r];
  __syncthreads();
  // per-wavenumber solve (DiffOper.cxx:1005-1083) on all (q, kz) of the tile
  {
    const float *cwx = p.lut, *swx = cwx + p.d.nx, *cwy = swx + p.d.nx, *swy = cwy + p.d.ny,
                *cwz = swy + p.d.ny, *swz = cwz + NZ;
    const float invN = 1.0f / (float)p.d.n();
    for (int i = threadIdx.x; i < Kq * NZ; i += blockDim.x) {
      const int qq = i / NZ, kz = i - qq * NZ;
      const long jj = j0 + qq;
      if (jj >= ncols) continue;
      const int ky = (int)(jj / nxh), kx = (int)(jj - (long)ky * nxh);
      const float cx = __ldg(cwx + kx), cy = __ldg(cwy + ky), cz = __ldg(cwz + kz);
      const float sx = __ldg(swx + kx), sy = __ldg(swy + ky), sz = __ldg(swz + kz);
      const float lambda = -p.alpha * (cx + cy + cz) + p.gamma;
      const float L00 = lambda - p.beta * cx, L11 = lambda - p.beta * cy, L22 = lambda - p.beta * cz;
      const float L10 = p.beta * sx * sy, L20 = p.beta * sx * sz, L21 = p.beta * sy * sz;
      float2 *s0 = sm + (0 * Kq + qq) * LS + kz, *s1 = sm + (1 * Kq + qq) * LS + kz,
             *s2 = sm + (2 * Kq + qq) * LS + kz;
      float2 b0 = *s0, b1 = *s1, b2 = *s2;
      b0.x *= invN; b0.y *= invN; b1.x *= invN; b1.y *= invN; b2.x *= invN; b2.y *= invN;
      float2 o0, o1, o2;
      if (inverse) {
        const float G00 = sqrtf(L00);
        const float G10 = L10 / G00, G20 = L20 / G00;
        const float G11 = sqrtf(L11 - G10 * G10);
        const float G21 = (L21 - G20 * G10) / G11;
        const float G22 = sqrtf(L22 - (G20 * G20 + G21 * G21));
        float2 y0, y1, y2;
        y0.x = b0.x / G00;                              y0.y = b0.y / G00;
        y1.x = (b1.x - G10 * y0.x) / G11;               y1.y = (b1.y - G10 * y0.y) / G11;
        y2.x = (b2.x - G20 * y0.x - G21 * y1.x) / G22;  y2.y = (b2.y - G20 * y0.y - G21 * y1.y) / G22;
        o2.x = y2.x / G22;                              o2.y = y2.y / G22;
        o1.x = (y1.x - G21 * o2.x) / G11;               o1.y = (y1.y - G21 * o2.y) / G11;
        o0.x = (y0.x - G10 * o1.x - G20 * o2.x) / G00;  o0.y = (y0.y - G10 * o1.y - G20 * o2.y) / G00;
      } else {
        o0.x = L00 * b0.x + L10 * b1.x + L20 * b2.x;  o0.y = L00 * b0.y + L10 * b1.y + L20 * b2.y;
        o1.x = L10 * b0.x + L11 * b1.x + L21 * b2.x;  o1.y = L10 * b0.y + L11 * b1.y + L21 * b2.y;
        o2.x = L20 * b0.x + L21 * b1.x + L22 * b2.x;  o2.y = L20 * b0.y + L21 * b1.y + L22 * b2.y;
      }
      *s0 = o0;
      *s1 = o1;
      *s2 = o2;
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < E; ++j) v[j] = S[t + T * j];
  line_fft<NZ, +1>(v, t, S, p.az.tw);
  if (act) {
#pragma unroll
    for (int r = 0; r < E; ++r)
      p.spec[((long)c * NZ + line_out_index<NZ>(t, r)) * plane + col] = v[r];
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

int fast_z_kq(const FluidPlan &p, int sms) {
  // Enough columns per CTA that one wave covers the spectrum, in whole lines
  // per warp, bounded by 768 threads.
  const int T = (p.d.nz == 16 || p.d.nz == 32) ? 4 : (p.d.nz == 256 ? 16 : 8);
  const int lpw = 32 / T;
  const long ncols = (long)p.d.ny * p.nxh;
  long kq = (ncols + 3L * sms - 1) / (3L * sms);
  kq = ((kq + lpw - 1) / lpw) * lpw;
  const long maxkq = (768 / T) / 3 / lpw * lpw;
  if (kq > maxkq) kq = maxkq;
  if (kq < lpw) kq = lpw;
  return (int)kq;
}

size_t fast_z_smem(int nz, int kq) {
  size_t r = 0;
  dispatch_n(nz, [&](auto Z) { r = sizeof(float2) * 3 * (size_t)kq * line_scratch<decltype(Z)::value>(); });
  return r;
}

cudaError_t fast_configure(const FluidPlan &p) {
  cudaError_t e = cudaSuccess;
  const size_t sxy = fast_xy_smem(p.d.nx, p.d.ny);
  dispatch_n(p.d.nx, [&](auto X) {
    dispatch_n(p.d.ny, [&](auto Y) {
      constexpr int NX = decltype(X)::value, NY = decltype(Y)::value;
      auto set = [&](const void *k) {
        cudaError_t r = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sxy);
        if (r != cudaSuccess) e = r;
      };
      set((const void *)k_xy_fwd_fast<NX, NY, SrcField>);
      set((const void *)k_xy_fwd_fast<NX, NY, SrcForce>);
      set((const void *)k_xy_inv_fast<NX, NY, DstField>);
      set((const void *)k_xy_inv_fast<NX, NY, DstAxpby>);
    });
  });
  dispatch_n(p.d.nz, [&](auto Z) {
    constexpr int NZ = decltype(Z)::value;
    cudaError_t r = cudaFuncSetAttribute((const void *)k_z_solve_fast<NZ>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)p.fast_smem_z);
    if (r != cudaSuccess) e = r;
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

cudaError_t fast_z_solve(const FluidPlan &p, int inverse, cudaStream_t s) {
  const long ncols = (long)p.d.ny * p.nxh;
  const int grid = (int)((ncols + p.fast_kq - 1) / p.fast_kq);
  dispatch_n(p.d.nz, [&](auto Z) {
    constexpr int NZ = decltype(Z)::value;
    constexpr int T = LineCfg<NZ>::T;
    k_z_solve_fast<NZ><<<grid, 3 * p.fast_kq * T, p.fast_smem_z, s>>>(p, inverse, p.fast_kq);
  });
  return cudaGetLastError();
}

template cudaError_t fast_xy_forward<SrcField>(const FluidPlan &, const SrcField &, cudaStream_t);
template cudaError_t fast_xy_forward<SrcForce>(const FluidPlan &, const SrcForce &, cudaStream_t);
template cudaError_t fast_xy_inverse<DstField>(const FluidPlan &, const DstField &, cudaStream_t);
template cudaError_t fast_xy_inverse<DstAxpby>(const FluidPlan &, const DstAxpby &, cudaStream_t);

}  // namespace aw
