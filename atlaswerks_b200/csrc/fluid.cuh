// fluid.cuh — the fluid operator L = -alpha*Lap - beta*grad(div) + gamma and
// its inverse, applied in Fourier space by three fused kernels:
//
//   xy-forward  one CTA per (z-slab, component): producer (a field, or the
//               greedy/LDMM body force computed on the fly) -> real-to-complex
//               FFT along x (two real rows packed per complex line) -> FFT
//               along y -> half spectrum to HBM.
//   z-solve     one CTA per tile of K (ky,kx) columns, all three components:
//               FFT along z -> per-wavenumber 3x3 Cholesky solve (or multiply)
//               with 1/N scaling -> inverse FFT along z -> back to HBM.
//   xy-inverse  one CTA per (z-slab, component): inverse FFT along y ->
//               complex-to-real along x -> consumer epilogue (store, or the
//               LDMM velocity update).
//
// The half spectrum (3 x nz x ny x (nx/2+1) complex64) makes two HBM round
// trips instead of the six of a pass-per-axis transform.
#pragma once

#include <cuda.h>

#include "aw_common.cuh"
#include "fft_smem.cuh"

namespace aw {

struct FluidPlan {
  Dims d;
  Spacing sp;
  float alpha, beta, gamma;
  int nxh;
  FFTAxis ax, ay, az;
  float2 *tw;      // device twiddle tables (x | y | z)
  float *lut;      // device LUT: cos x | sin x | cos y | sin y | cos z | sin z
  float2 *spec;    // device half spectrum [3][nz][ny][nxh]
  int pairs_per_batch, cols_per_batch, zcols_per_cta;
  size_t smem_xy, smem_z;
  // slabs whose half spectrum does not fit one CTA's shared memory: the xy
  // transforms run as an x pass and a y pass through the spectrum in HBM
  int split;
  size_t smem_x, smem_y;
  int device;
  // register-FFT path (fluid_fast.cu): power-of-two axes
  int fast;
  int fast_kq;               // (ky,kx) columns per z-pass CTA
  size_t fast_smem_xy, fast_smem_z;
  int *status;               // device status word: bounded waits that timed out
  int fast_tma;              // z-pass tiles moved by TMA tensor copies
  CUtensorMap spec_map;      // spectrum as [3][nz][2*ny*nxh] floats, 128B swizzle
};

// --- producers for the forward pass ----------------------------------------
// plain vector field input
struct SrcField {
  const float *c[3];
  AW_D float value(int comp, int x, int y, int z, const Dims &d) const {
    return __ldg(c[comp] + d.idx(x, y, z));
  }
  // rows y0 and y0+1 of slab z at x = t + TX*j, j < E, as (row y0, row y0+1)
  template <int E, int TX>
  AW_D void row_pair(int comp, int t, int y0, int z, const Dims &d, float2 *v) const {
    const float *r0 = (comp == 0 ? c[0] : comp == 1 ? c[1] : c[2]) + d.idx(t, y0, z);
    const float *r1 = r0 + d.nx;
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = make_float2(__ldg(r0 + TX * j), __ldg(r1 + TX * j));
  }
};

// body force f_c = d/dc(G) * M, with M = A - G (mode 1, greedy: G = I0(h),
// A = I1), M = A (mode 0, LDMM IterateNew: G = J0_{t-1}, A = splatted
// residual) or M = (G - A) * B (mode 2, LDMM IterateOrig: G = I0(h),
// A = JT_t, B = JacDet_t; LDMMIteratorCPU.cxx:447-452). The gradient is
// Array3DUtils::computeGradient with wrap = false (Array3DUtils.txx:783-900):
// central differences / (2 sp), one-sided at the borders, the float
// difference divided in double.
struct SrcForce {
  const float *G;
  const float *A;
  const float *B;
  int mode;
  DivD c2[3], c1[3];  // 2 sp and sp per axis
  // All six divisors are powers of two whose reciprocals are normal floats:
  // the difference times the float reciprocal is then the same float as the
  // double quotient rounded (both are the exact product, rounded once to
  // nearest), so the gradient needs no double arithmetic.
  int fexact;
  float r2[3], r1[3];
  AW_D float grad(float diff, int comp, bool interior) const {
    if (fexact) return fmul(diff, interior ? r2[comp] : r1[comp]);
    return __double2float_rn(ddiv((double)diff, interior ? c2[comp] : c1[comp]));
  }
  // M from preloaded values (b is read only in mode 2)
  AW_D float mismatch_v(float g0, float a, float b) const {
    return mode == 0 ? a : (mode == 1 ? -fsub(g0, a) : fmul(fsub(g0, a), b));
  }
  // One voxel. The neighbours are clamped to the voxel itself at the
  // borders (G[1] - G[0] at the first, G[n-1] - G[n-2] at the last; every
  // axis has n >= 2), so every load is issued before the arithmetic, with
  // no branch between them.
  AW_D float value(int comp, int x, int y, int z, const Dims &d) const {
    const long i = d.idx(x, y, z);
    int pos, n;
    long stride;
    if (comp == 0) { pos = x; n = d.nx; stride = 1; }
    else if (comp == 1) { pos = y; n = d.ny; stride = d.nx; }
    else { pos = z; n = d.nz; stride = (long)d.nx * d.ny; }
    const long ihi = pos < n - 1 ? i + stride : i, ilo = pos > 0 ? i - stride : i;
    const float g0 = __ldg(G + i), gh = __ldg(G + ihi), gl = __ldg(G + ilo), a = __ldg(A + i);
    const float b = mode == 2 ? __ldg(B + i) : 0.f;
    const float g = grad(fsub(gh, gl), comp, pos > 0 && pos < n - 1);
    return fmul(g, mismatch_v(g0, a, b));
  }
  // Rows y0 and y0+1 of slab z at x = t + TX*j, j < E, as (row y0, row
  // y0+1): the same values as value(), from row pointers formed once and one
  // code path per component. Every load of the row pair (G and its
  // neighbours, A, and B in mode 2; of each chunk of it in 256-wide rows) is
  // issued before any arithmetic that depends on one, so the pair costs one
  // round trip to L2, not one per array. Needs nx, ny, nz >= 3, an even ny, TX * E = nx and the TX lanes
  // of a line consecutive within a warp, every lane of the warp calling it
  // (the x neighbours come by shuffles).
  template <int E, int TX>
  AW_D void row_pair(int comp, int t, int y0, int z, const Dims &d, float2 *v) const {
    // the values of each array per lane in flight at once: the whole row
    // pair up to E = 4, chunks of two above (a 256-wide row would spill)
    constexpr int C = E <= 4 ? E : 2;
    const long i0 = d.idx(t, y0, z);
    const int nx = d.nx;
    const float *g0p = G + i0, *g1p = g0p + nx, *a0p = A + i0, *b0p = B + i0;
    float a0[C], a1[C], b0[C], b1[C];
    // A (and B) of chunk j0 .. j0 + C - 1
    auto load_ab = [&](int j0) {
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int o = TX * (j0 + c);
        a0[c] = __ldg(a0p + o);
        a1[c] = __ldg(a0p + o + nx);
      }
      if (mode == 2) {
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const int o = TX * (j0 + c);
          b0[c] = __ldg(b0p + o);
          b1[c] = __ldg(b0p + o + nx);
        }
      } else {
#pragma unroll
        for (int c = 0; c < C; ++c) b0[c] = b1[c] = 0.f;
      }
    };
    if (comp == 0) {
      // the line covers the row (TX * E = nx): x +- 1 is held by the
      // neighbouring lane at the same j, or by the line's first / last lane
      // at j +- 1, so the neighbours come by shuffles instead of loads
      float r0[E], r1[E];
#pragma unroll
      for (int j = 0; j < E; ++j) {
        r0[j] = __ldg(g0p + TX * j);
        r1[j] = __ldg(g1p + TX * j);
      }
      const unsigned full = 0xffffffffu;
      const int up = (t + 1) & (TX - 1), dn = (t - 1) & (TX - 1);
#pragma unroll
      for (int j0 = 0; j0 < E; j0 += C) {
        load_ab(j0);
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const int j = j0 + c;
          const int jn = j + 1 < E ? j + 1 : j, jp = j > 0 ? j - 1 : j;
          const float n0 = __shfl_sync(full, r0[j], up, TX), n1 = __shfl_sync(full, r1[j], up, TX);
          const float w0 = __shfl_sync(full, r0[jn], 0, TX), w1 = __shfl_sync(full, r1[jn], 0, TX);
          const float p0 = __shfl_sync(full, r0[j], dn, TX), p1 = __shfl_sync(full, r1[j], dn, TX);
          const float q0 = __shfl_sync(full, r0[jp], TX - 1, TX),
                      q1 = __shfl_sync(full, r1[jp], TX - 1, TX);
          const int x = t + TX * j;
          const bool first = x == 0, last = x == nx - 1, in = !first && !last;
          // G[x + hi] and G[x + lo], hi = 0 at the last voxel, lo = 0 at the first
          const float h0 = last ? r0[j] : (t == TX - 1 ? w0 : n0);
          const float h1 = last ? r1[j] : (t == TX - 1 ? w1 : n1);
          const float l0 = first ? r0[j] : (t == 0 ? q0 : p0);
          const float l1 = first ? r1[j] : (t == 0 ? q1 : p1);
          v[j] = make_float2(fmul(grad(fsub(h0, l0), 0, in), mismatch_v(r0[j], a0[c], b0[c])),
                             fmul(grad(fsub(h1, l1), 0, in), mismatch_v(r1[j], a1[c], b1[c])));
        }
      }
    } else if (comp == 1) {
      // y0 - 1 (or y0 at the first row) and y0 + 2 (or y0 + 1 at the last)
      const int lo = y0 > 0 ? -nx : 0, hi = y0 + 2 < d.ny ? 2 * nx : nx;
      const bool in0 = y0 > 0, in1 = y0 + 2 < d.ny;
#pragma unroll
      for (int j0 = 0; j0 < E; j0 += C) {
        float g0[C], g1[C], gl[C], gh[C];
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const int o = TX * (j0 + c);
          g0[c] = __ldg(g0p + o);
          g1[c] = __ldg(g1p + o);
          gl[c] = __ldg(g0p + o + lo);
          gh[c] = __ldg(g0p + o + hi);
        }
        load_ab(j0);
#pragma unroll
        for (int c = 0; c < C; ++c) {
          // row y0: G[y0+1] - G[y0-1], or G[1] - G[0] (lo = 0);
          // row y0+1: G[y0+2] - G[y0], or G[ny-1] - G[ny-2] (hi = nx)
          const float d0 = fsub(g1[c], gl[c]);
          const float d1 = fsub(gh[c], g0[c]);
          v[j0 + c] = make_float2(fmul(grad(d0, 1, in0), mismatch_v(g0[c], a0[c], b0[c])),
                                  fmul(grad(d1, 1, in1), mismatch_v(g1[c], a1[c], b1[c])));
        }
      }
    } else {
      const long sl = (long)nx * d.ny;
      const long lo = z > 0 ? -sl : 0, hi = z < d.nz - 1 ? sl : 0;
      const bool in = z > 0 && z < d.nz - 1;
#pragma unroll
      for (int j0 = 0; j0 < E; j0 += C) {
        float g0[C], g1[C], h0[C], l0[C], h1[C], l1[C];
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const int o = TX * (j0 + c);
          g0[c] = __ldg(g0p + o);
          g1[c] = __ldg(g1p + o);
          h0[c] = __ldg(g0p + o + hi);
          l0[c] = __ldg(g0p + o + lo);
          h1[c] = __ldg(g1p + o + hi);
          l1[c] = __ldg(g1p + o + lo);
        }
        load_ab(j0);
#pragma unroll
        for (int c = 0; c < C; ++c) {
          const float d0 = fsub(h0[c], l0[c]);
          const float d1 = fsub(h1[c], l1[c]);
          v[j0 + c] = make_float2(fmul(grad(d0, 2, in), mismatch_v(g0[c], a0[c], b0[c])),
                                  fmul(grad(d1, 2, in), mismatch_v(g1[c], a1[c], b1[c])));
        }
      }
    }
  }
};
inline SrcForce make_force(const float *G, const float *A, int mode, const Spacing &sp,
                           const float *B = nullptr) {
  SrcForce f;
  f.G = G;
  f.A = A;
  f.B = B;
  f.mode = mode;
  const double s[3] = {sp.x, sp.y, sp.z};
  f.fexact = 1;
  for (int c = 0; c < 3; ++c) {
    f.c2[c] = make_div(2.0 * s[c]);
    f.c1[c] = make_div(s[c]);
    f.r2[c] = (float)f.c2[c].r;
    f.r1[c] = (float)f.c1[c].r;
    // a power of two whose reciprocal is a float (well inside the normal range)
    for (const DivD *q : {&f.c2[c], &f.c1[c]})
      if (!q->p2 || !(q->r >= 0x1p-100 && q->r <= 0x1p+100)) f.fexact = 0;
  }
  return f;
}

// --- consumers for the inverse pass ----------------------------------------
// A kernel stores component `comp` through dst.bind(comp): the component's
// pointer picked once (no indexed parameter array) and any per-launch
// factors formed once.
struct DstFieldBound {
  float *c;
  AW_D void store(long i, float v) const { c[i] = v; }
};
struct DstField {
  static constexpr bool kReads = false;
  float *c[3];
  AW_D DstFieldBound bind(int comp) const {
    return DstFieldBound{comp == 0 ? c[0] : comp == 1 ? c[1] : c[2]};
  }
};

// -K f: the shooting velocities (LDMMAdShootingIteratorCPU.cxx:256-261,
// 291-296 scale K f by -1, an exact sign flip)
struct DstNegBound {
  float *c;
  AW_D void store(long i, float v) const { c[i] = -v; }
};
struct DstNeg {
  static constexpr bool kReads = false;
  float *c[3];
  AW_D DstNegBound bind(int comp) const {
    return DstNegBound{comp == 0 ? c[0] : comp == 1 ? c[1] : c[2]};
  }
};

// LDMM velocity update v = vfac * v + ufac * u (LDMMIteratorCPU::updateVelocity,
// LDMM/LDMMIteratorCPU.cxx:177-190) with vfac = 1 - 2*eps and
// ufac = 2*eps / sigma^2 formed from the device-resident step eps, float
// arithmetic in the reference's order (LDMMIteratorCPU.cxx:606-609).
struct DstAxpbyBound {
  float *c;
  float vfac, ufac;
  AW_D void store(long i, float u) const { c[i] = fadd(fmul(vfac, c[i]), fmul(ufac, u)); }
  // n elements: every old value is read before any is written
  template <int N>
  AW_D void store_n(const long (&i)[N], const float (&u)[N]) const {
    float old[N];
#pragma unroll
    for (int j = 0; j < N; ++j) old[j] = c[i[j]];
#pragma unroll
    for (int j = 0; j < N; ++j) c[i[j]] = fadd(fmul(vfac, old[j]), fmul(ufac, u[j]));
  }
};
struct DstAxpby {
  static constexpr bool kReads = true;
  float *c[3];
  const float *step;
  float sigma;
  // the step read once per thread, the two factors formed once
  AW_D DstAxpbyBound bind(int comp) const {
    const float eps = *step;
    const float vfac = fsub(1.0f, fmul(2.0f, eps));
    const float ufac = fdiv(fmul(2.0f, eps), fmul(sigma, sigma));
    return DstAxpbyBound{comp == 0 ? c[0] : comp == 1 ? c[1] : c[2], vfac, ufac};
  }
};

// The greedy update h'(x) = h(x + eps v(x)/sp) the inverse pass can apply
// itself (fluid_inverse_compose): h in, h' out, the device-resident step,
// the spacing divisors.
struct ComposeArgs {
  const float *hx, *hy, *hz;
  float *ox, *oy, *oz;
  const float *step;
  DivF q0, q1, q2;
  int fast;  // 1: float-tree interpolation (trilerp_vector<true>)
};

// host API (fluid.cu)
int fluid_plan_create(FluidPlan *p, int nx, int ny, int nz, double spx, double spy, double spz,
                      float alpha, float beta, float gamma);
void fluid_plan_destroy(FluidPlan *p);

cudaError_t fluid_forward_field(const FluidPlan &p, const float *fx, const float *fy,
                                const float *fz, cudaStream_t s);
cudaError_t fluid_forward_force(const FluidPlan &p, const float *G, const float *A, int diff,
                                cudaStream_t s);
// force (G - A) * B * grad G (mode 2)
cudaError_t fluid_forward_force_jac(const FluidPlan &p, const float *G, const float *A,
                                    const float *B, cudaStream_t s);
cudaError_t fluid_solve(const FluidPlan &p, int inverse, cudaStream_t s);
// shapes of the shared-memory (any-size) path; fluid_get_shapes returns 0 on
// the register path, whose shapes are fixed
int fluid_get_shapes(const FluidPlan &p, int *P, int *Q, int *K);
cudaError_t fluid_set_shapes(FluidPlan *p, int P, int Q, int K);
cudaError_t fluid_autotune(FluidPlan *p, cudaStream_t s);
// the plan's status word: *timed_out = 1 when a transform kernel's bounded
// wait ran out since the last call; the word is cleared (stream-ordered)
cudaError_t fluid_take_status(FluidPlan *p, int *timed_out, cudaStream_t s);
// one CTA whose bounded wait (polls polls) on an mbarrier that nothing
// arrives on runs out and records the timeout in the plan's status word
cudaError_t fluid_wait_selftest(const FluidPlan &p, int polls, cudaStream_t s);
cudaError_t fluid_inverse_store(const FluidPlan &p, float *ox, float *oy, float *oz,
                                cudaStream_t s);
cudaError_t fluid_inverse_store_neg(const FluidPlan &p, float *ox, float *oy, float *oz,
                                    cudaStream_t s);
// v = K f never leaves the chip: h' = h(x + eps v/sp) from the inverse pass
// itself (power-of-two grids: the register-FFT path); cudaErrorNotSupported
// on other grids, where the caller stores v and updates separately
cudaError_t fluid_inverse_compose(const FluidPlan &p, const ComposeArgs &a, cudaStream_t s);
cudaError_t fluid_inverse_axpby(const FluidPlan &p, float *vx, float *vy, float *vz,
                                const float *step, float sigma, cudaStream_t s);

}  // namespace aw
