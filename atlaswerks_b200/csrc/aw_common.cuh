// aw_common.cuh — shared device helpers for the sm_100a registration kernels.
//
// Interpolation arithmetic follows the reference CPU routines operation by
// operation (HField3DUtils::trilerp, Array3DUtils::trilerp,
// HField3DUtils::forwardApply): float positions and data, double weights and
// sums. Every product and sum below is an explicit round-to-nearest
// intrinsic so the compiler cannot contract it into a fused multiply-add;
// with identical inputs the results are bit-identical to the reference.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#define AW_HD __host__ __device__ __forceinline__
#define AW_D __device__ __forceinline__

namespace aw {

// HField3DUtils::VectorBackgroundStrategy (UtilitiesDataTypes/HField3DUtils.h:44-49)
enum BgStrategy { BG_PARTIAL_ID = 0, BG_ID = 1, BG_PARTIAL_ZERO = 2, BG_ZERO = 3, BG_CLAMP = 4, BG_WRAP = 5 };

struct Dims {
  int nx, ny, nz;
  AW_HD long n() const { return (long)nx * ny * nz; }
  AW_HD long idx(int x, int y, int z) const { return ((long)z * ny + y) * nx + x; }
};

struct Spacing {
  double x, y, z;
};

// Elementwise launch shape: 128 threads along x, one grid row per (y, z), so
// a thread finds its voxel without any integer division.
constexpr int kRowThreads = 128;
inline dim3 row_grid(const Dims &d) {
  return dim3((unsigned)((d.nx + kRowThreads - 1) / kRowThreads), (unsigned)d.ny, (unsigned)d.nz);
}
struct Voxel {
  int x, y, z;
  long i;
};
AW_D bool voxel_of(const Dims &d, Voxel &v) {
  v.x = blockIdx.x * kRowThreads + threadIdx.x;
  v.y = blockIdx.y;
  v.z = blockIdx.z;
  v.i = ((long)v.z * d.ny + v.y) * d.nx + v.x;
  return v.x < d.nx;
}

// ---- exact-rounding arithmetic -------------------------------------------
AW_D double dmul(double a, double b) { return __dmul_rn(a, b); }
AW_D double dadd(double a, double b) { return __dadd_rn(a, b); }
AW_D double dsub(double a, double b) { return __dsub_rn(a, b); }
AW_D float fmul(float a, float b) { return __fmul_rn(a, b); }
AW_D float fadd(float a, float b) { return __fadd_rn(a, b); }
AW_D float fsub(float a, float b) { return __fsub_rn(a, b); }
AW_D float fdiv(float a, float b) { return __fdiv_rn(a, b); }

// x / d as the reference divides (IEEE, round to nearest). When d is a power
// of two the quotient is x scaled by an exact power of two, and x * (1/d)
// is the same number: the multiply replaces the division sequence.
struct DivD {
  double d, r;
  int p2;
};
struct DivF {
  float d, r;
  int p2;
};
inline bool host_is_pow2(double d) {
  if (!(d > 0.0)) return false;
  int e = 0;
  const double m = frexp(d, &e);
  return m == 0.5 && e > -1000 && e < 1000;
}
inline DivD make_div(double d) { return DivD{d, 1.0 / d, host_is_pow2(d) ? 1 : 0}; }
inline DivF make_divf(float d) { return DivF{d, 1.0f / d, host_is_pow2((double)d) ? 1 : 0}; }
AW_D double ddiv(double x, const DivD &q) { return q.p2 ? dmul(x, q.r) : __ddiv_rn(x, q.d); }
AW_D float fdivq(float x, const DivF &q) { return q.p2 ? fmul(x, q.r) : fdiv(x, q.d); }

// Atlas subjects on grids of their own: a deformation lives on the template
// grid (n voxels per axis) and points into the subject's grid (m voxels per
// axis) through the map of voxel centres of equal physical extent,
// p -> (p + 0.5) * (m / n) - 0.5, in double. `on` is 0 when m == n, and the
// sample point is then h itself, as in the reference's equal-grid atlas.
struct AtlasMap {
  int on;
  double r[3];  // m / n per axis
};
AW_D void atlas_point(const AtlasMap &a, double &x, double &y, double &z) {
  x = dsub(dmul(dadd(x, 0.5), a.r[0]), 0.5);
  y = dsub(dmul(dadd(y, 0.5), a.r[1]), 0.5);
  z = dsub(dmul(dadd(z, 0.5), a.r[2]), 0.5);
}

// floor as the reference computes it: truncate, then step down for
// negative non-integers (Array3DUtils.txx:70-75)
// Positions are clamped to [-2^30, 2^30] first (NaN to -2^30): the same
// floor for every position a grid can hold, and for huge, infinite or NaN
// positions a cell far outside every grid, so fx + 1 cannot overflow and
// the callers' inside/outside tests never pass an out-of-range corner.
AW_D int ref_floor_d(double x) {
  x = fmin(fmax(x, -0x1p30), 0x1p30);
  int f = __double2int_rz(x);
  if (x < 0.0 && x != (double)f) --f;
  return f;
}
AW_D int ref_floor_f(float x) {
  x = fminf(fmaxf(x, -0x1p30f), 0x1p30f);
  int f = __float2int_rz(x);
  if (x < 0.0f && x != __int2float_rn(f)) --f;
  return f;
}

// ((omt*(omu*(c0*omv + c7*v) + u*(c3*omv + c4*v))) + t*(omu*(c1*omv + c6*v) + u*(c2*omv + c5*v)))
AW_D double lerp_tree(const float c[8], double t, double u, double v, double omt, double omu,
                      double omv) {
  const double a = dmul(omt, dadd(dmul(omu, dadd(dmul((double)c[0], omv), dmul((double)c[7], v))),
                                  dmul(u, dadd(dmul((double)c[3], omv), dmul((double)c[4], v)))));
  const double b = dmul(t, dadd(dmul(omu, dadd(dmul((double)c[1], omv), dmul((double)c[6], v))),
                                dmul(u, dadd(dmul((double)c[2], omv), dmul((double)c[5], v)))));
  return dadd(a, b);
}

// The same tree in float with fused multiply-adds, a + t (b - a) per lerp
// (x first, then y, then z): the fast-interpolation mode. Not bit-identical
// to the double tree; the difference is a few float ulps of the result.
AW_D float lerpf(float a, float b, float t) { return fmaf(t, b - a, a); }
AW_D float lerp_tree_f(const float c[8], float t, float u, float v) {
  const float x00 = lerpf(c[0], c[1], t), x10 = lerpf(c[3], c[2], t);
  const float x01 = lerpf(c[7], c[6], t), x11 = lerpf(c[4], c[5], t);
  return lerpf(lerpf(x00, x10, u), lerpf(x01, x11, u), v);
}

// Scalar trilinear sample, background value per out-of-volume corner
// (Array3DUtils::trilerp<T, BACKGROUND_STRATEGY_VAL>, Array3DUtils.txx:59-232).
// FAST: the float tree (lerp_tree_f) on float fractions.
template <bool FAST = false>
AW_D float trilerp_scalar(const float *__restrict__ a, const Dims d, double x, double y, double z,
                          float bg) {
  const int fx = ref_floor_d(x), fy = ref_floor_d(y), fz = ref_floor_d(z);
  const int cx = fx + 1, cy = fy + 1, cz = fz + 1;
  const double t = dsub(x, (double)fx), u = dsub(y, (double)fy), v = dsub(z, (double)fz);
  const double omt = FAST ? 0.0 : dsub(1.0, t), omu = FAST ? 0.0 : dsub(1.0, u),
               omv = FAST ? 0.0 : dsub(1.0, v);
  float c[8];
  const bool inside = fx >= 0 && cx < d.nx && fy >= 0 && cy < d.ny && fz >= 0 && cz < d.nz;
  if (inside) {
    // 32-bit offsets: every grid here has fewer than 2^31 voxels
    const int b = (fz * d.ny + fy) * d.nx + fx;
    const int sy = d.nx, sz = d.nx * d.ny;
    c[0] = __ldg(a + b);
    c[1] = __ldg(a + b + 1);
    c[2] = __ldg(a + b + sy + 1);
    c[3] = __ldg(a + b + sy);
    c[4] = __ldg(a + b + sy + sz);
    c[5] = __ldg(a + b + sy + sz + 1);
    c[6] = __ldg(a + b + sz + 1);
    c[7] = __ldg(a + b + sz);
  } else {
    const bool fxi = fx >= 0 && fx < d.nx, fyi = fy >= 0 && fy < d.ny, fzi = fz >= 0 && fz < d.nz;
    const bool cxi = cx >= 0 && cx < d.nx, cyi = cy >= 0 && cy < d.ny, czi = cz >= 0 && cz < d.nz;
    c[0] = (fxi && fyi && fzi) ? __ldg(a + d.idx(fx, fy, fz)) : bg;
    c[1] = (cxi && fyi && fzi) ? __ldg(a + d.idx(cx, fy, fz)) : bg;
    c[2] = (cxi && cyi && fzi) ? __ldg(a + d.idx(cx, cy, fz)) : bg;
    c[3] = (fxi && cyi && fzi) ? __ldg(a + d.idx(fx, cy, fz)) : bg;
    c[4] = (fxi && cyi && czi) ? __ldg(a + d.idx(fx, cy, cz)) : bg;
    c[5] = (cxi && cyi && czi) ? __ldg(a + d.idx(cx, cy, cz)) : bg;
    c[6] = (cxi && fyi && czi) ? __ldg(a + d.idx(cx, fy, cz)) : bg;
    c[7] = (fxi && fyi && czi) ? __ldg(a + d.idx(fx, fy, cz)) : bg;
  }
  if (FAST) return lerp_tree_f(c, (float)t, (float)u, (float)v);
  return __double2float_rn(lerp_tree(c, t, u, v, omt, omu, omv));
}

AW_D int safe_mod(int r, int m) {
  r %= m;
  return r < 0 ? r + m : r;
}

// Vector trilinear sample with the reference's background strategies
// (HField3DUtils::trilerp, HField3DUtils.txx:1972-2300). Position in float,
// fractional part formed in float, weights and sums in double. `scale`
// multiplies each fetched corner value in float first (it reproduces
// interpolating a field that the reference scaled in place beforehand);
// pass 1.0f for none. FAST: the float tree (lerp_tree_f).
template <bool FAST = false>
AW_D void trilerp_vector(const float *__restrict__ hx, const float *__restrict__ hy,
                         const float *__restrict__ hz, const Dims d, float x, float y, float z,
                         int bgs, float scale, float &ox, float &oy, float &oz) {
  int fx = ref_floor_f(x), fy = ref_floor_f(y), fz = ref_floor_f(z);
  int cx = fx + 1, cy = fy + 1, cz = fz + 1;
  const float tf = fsub(x, __int2float_rn(fx));
  const float uf = fsub(y, __int2float_rn(fy));
  const float vf = fsub(z, __int2float_rn(fz));
  const double t = (double)tf, u = (double)uf, v = (double)vf;
  const double omt = FAST ? 0.0 : dsub(1.0, t), omu = FAST ? 0.0 : dsub(1.0, u),
               omv = FAST ? 0.0 : dsub(1.0, v);
  bool inside = true;
  if (bgs == BG_WRAP) {
    fx = safe_mod(fx, d.nx); fy = safe_mod(fy, d.ny); fz = safe_mod(fz, d.nz);
    cx = safe_mod(cx, d.nx); cy = safe_mod(cy, d.ny); cz = safe_mod(cz, d.nz);
  } else if (bgs == BG_CLAMP) {
    if (fx < 0) { fx = 0; if (cx < 0) cx = 0; }
    if (cx >= d.nx) { cx = d.nx - 1; if (fx >= d.nx) fx = d.nx - 1; }
    if (fy < 0) { fy = 0; if (cy < 0) cy = 0; }
    if (cy >= d.ny) { cy = d.ny - 1; if (fy >= d.ny) fy = d.ny - 1; }
    if (fz < 0) { fz = 0; if (cz < 0) cz = 0; }
    if (cz >= d.nz) { cz = d.nz - 1; if (fz >= d.nz) fz = d.nz - 1; }
  } else {
    inside = fx >= 0 && cx < d.nx && fy >= 0 && cy < d.ny && fz >= 0 && cz < d.nz;
  }
  const int X[8] = {fx, cx, cx, fx, fx, cx, cx, fx};
  const int Y[8] = {fy, fy, cy, cy, cy, cy, fy, fy};
  const int Z[8] = {fz, fz, fz, fz, cz, cz, cz, cz};
  float cxv[8], cyv[8], czv[8];
  if (inside) {
    // corner offsets from one 32-bit base (grids have < 2^31 voxels); CLAMP
    // and WRAP corners are not a unit cube, so they index each corner
    const int sy = d.nx, sz = d.nx * d.ny;
    int off[8];
    if (bgs == BG_WRAP || bgs == BG_CLAMP) {
#pragma unroll
      for (int c = 0; c < 8; ++c) off[c] = (Z[c] * d.ny + Y[c]) * d.nx + X[c];
    } else {
      const int b = (fz * d.ny + fy) * d.nx + fx;
      off[0] = b;
      off[1] = b + 1;
      off[2] = b + sy + 1;
      off[3] = b + sy;
      off[4] = b + sy + sz;
      off[5] = b + sy + sz + 1;
      off[6] = b + sz + 1;
      off[7] = b + sz;
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      cxv[c] = __ldg(hx + off[c]);
      cyv[c] = __ldg(hy + off[c]);
      czv[c] = __ldg(hz + off[c]);
    }
    if (scale != 1.0f) {
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        cxv[c] = fmul(cxv[c], scale);
        cyv[c] = fmul(cyv[c], scale);
        czv[c] = fmul(czv[c], scale);
      }
    }
  } else if (bgs == BG_ID) {
    ox = x; oy = y; oz = z;
    return;
  } else if (bgs == BG_ZERO) {
    ox = 0.f; oy = 0.f; oz = 0.f;
    return;
  } else {
    const bool pid = (bgs == BG_PARTIAL_ID);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const bool in = X[c] >= 0 && X[c] < d.nx && Y[c] >= 0 && Y[c] < d.ny && Z[c] >= 0 && Z[c] < d.nz;
      if (in) {
        const long i = d.idx(X[c], Y[c], Z[c]);
        cxv[c] = fmul(__ldg(hx + i), scale);
        cyv[c] = fmul(__ldg(hy + i), scale);
        czv[c] = fmul(__ldg(hz + i), scale);
      } else if (pid) {
        cxv[c] = __int2float_rn(X[c]);
        cyv[c] = __int2float_rn(Y[c]);
        czv[c] = __int2float_rn(Z[c]);
      } else {
        cxv[c] = 0.f; cyv[c] = 0.f; czv[c] = 0.f;
      }
    }
  }
  if (FAST) {
    ox = lerp_tree_f(cxv, tf, uf, vf);
    oy = lerp_tree_f(cyv, tf, uf, vf);
    oz = lerp_tree_f(czv, tf, uf, vf);
    return;
  }
  ox = __double2float_rn(lerp_tree(cxv, t, u, v, omt, omu, omv));
  oy = __double2float_rn(lerp_tree(cyv, t, u, v, omt, omu, omv));
  oz = __double2float_rn(lerp_tree(czv, t, u, v, omt, omu, omv));
}

// ---- warp reductions --------------------------------------------------------
AW_D double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
AW_D float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

}  // namespace aw
