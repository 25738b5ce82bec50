/*
 * aw_oracle.c — CPU restatement of the AtlasWerks greedy-fluid / LDMM inner
 * loop, used as the parity checker for the CUDA path.
 *
 * TEST INFRASTRUCTURE. Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg may load this library. The product (atlaswerks_b200/)
 * never links or calls it.
 *
 * Every routine follows a reference CPU routine statement by statement and
 * reproduces its floating-point types: float data, double interpolation
 * weights, float position arithmetic. Build with -ffp-contract=off so that no
 * fused multiply-add changes a rounding. The fluid operator is evaluated in
 * FP64 end to end (the "FP64 oracle"): the reference applies it in FP32 with
 * FFTW, which is not available here.
 *
 * Vector fields are planar (three float planes x|y|z, each nx*ny*nz, x
 * fastest) — the same values the reference holds as Array3D<Vector3D<float>>.
 */
#include "aw_oracle.h"

#include <math.h>
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#include <stdlib.h>
#include <string.h>

#include "fft64.h"

#define IDX(x, y, z) (((long)(z) * ny + (y)) * nx + (x))

/* ------------------------------------------------------------------------
 * Scalar trilinear interpolation, background value per corner.
 * Follows Array3DUtils::trilerp<T, BACKGROUND_STRATEGY_VAL>
 * (UtilitiesDataTypes/Array3DUtils.txx:59-232): positions and weights in
 * double, result rounded to float.
 * ---------------------------------------------------------------------- */
static float trilerp_val(const float *a, int nx, int ny, int nz, double x, double y, double z,
                         float bg) {
  int fx = (int)x, fy = (int)y, fz = (int)z;
  if (x < 0 && x != (int)x) --fx;
  if (y < 0 && y != (int)y) --fy;
  if (z < 0 && z != (int)z) --fz;
  const int cx = fx + 1, cy = fy + 1, cz = fz + 1;
  const double t = x - fx, u = y - fy, v = z - fz;
  const double omt = 1.0 - t, omu = 1.0 - u, omv = 1.0 - v;
  float v0, v1, v2, v3, v4, v5, v6, v7;
  const int inside = fx >= 0 && cx < nx && fy >= 0 && cy < ny && fz >= 0 && cz < nz;
  if (inside) {
    v0 = a[IDX(fx, fy, fz)];
    v1 = a[IDX(cx, fy, fz)];
    v2 = a[IDX(cx, cy, fz)];
    v3 = a[IDX(fx, cy, fz)];
    v4 = a[IDX(fx, cy, cz)];
    v5 = a[IDX(cx, cy, cz)];
    v6 = a[IDX(cx, fy, cz)];
    v7 = a[IDX(fx, fy, cz)];
  } else {
    const int fxi = fx >= 0 && fx < nx, fyi = fy >= 0 && fy < ny, fzi = fz >= 0 && fz < nz;
    const int cxi = cx >= 0 && cx < nx, cyi = cy >= 0 && cy < ny, czi = cz >= 0 && cz < nz;
    v0 = (fxi && fyi && fzi) ? a[IDX(fx, fy, fz)] : bg;
    v1 = (cxi && fyi && fzi) ? a[IDX(cx, fy, fz)] : bg;
    v2 = (cxi && cyi && fzi) ? a[IDX(cx, cy, fz)] : bg;
    v3 = (fxi && cyi && fzi) ? a[IDX(fx, cy, fz)] : bg;
    v4 = (fxi && cyi && czi) ? a[IDX(fx, cy, cz)] : bg;
    v5 = (cxi && cyi && czi) ? a[IDX(cx, cy, cz)] : bg;
    v6 = (cxi && fyi && czi) ? a[IDX(cx, fy, cz)] : bg;
    v7 = (fxi && fyi && czi) ? a[IDX(fx, fy, cz)] : bg;
  }
  return (float)(omt * (omu * (v0 * omv + v7 * v) + u * (v3 * omv + v4 * v)) +
                 t * (omu * (v1 * omv + v6 * v) + u * (v2 * omv + v5 * v)));
}

/* ------------------------------------------------------------------------
 * Vector trilinear interpolation with the reference's background strategies.
 * Follows HField3DUtils::trilerp (UtilitiesDataTypes/HField3DUtils.txx:
 * 1972-2300). The position is float; the fractional part is formed in float
 * (float - int), widened to double, and the corner sums run in double.
 * ---------------------------------------------------------------------- */
static int safe_mod(int r, int m) {
  r %= m;
  if (r < 0) r += m;
  return r;
}

static void trilerp_vec(const float *hxp, const float *hyp, const float *hzp, int nx, int ny,
                        int nz, float x, float y, float z, float *ox, float *oy, float *oz,
                        int bgs) {
  int fx = (int)x, fy = (int)y, fz = (int)z;
  if (x < 0 && x != (float)(int)x) --fx;
  if (y < 0 && y != (float)(int)y) --fy;
  if (z < 0 && z != (float)(int)z) --fz;
  int cx = fx + 1, cy = fy + 1, cz = fz + 1;
  const double t = (double)(x - (float)fx), u = (double)(y - (float)fy),
               v = (double)(z - (float)fz);
  const double omt = 1.0 - t, omu = 1.0 - u, omv = 1.0 - v;
  float vX[8] = {0}, vY[8] = {0}, vZ[8] = {0};
  int inside = 1;
  if (bgs == AW_BG_WRAP) {
    fx = safe_mod(fx, nx); fy = safe_mod(fy, ny); fz = safe_mod(fz, nz);
    cx = safe_mod(cx, nx); cy = safe_mod(cy, ny); cz = safe_mod(cz, nz);
  } else if (bgs == AW_BG_CLAMP) {
    if (fx < 0) { fx = 0; if (cx < 0) cx = 0; }
    if (cx >= nx) { cx = nx - 1; if (fx >= nx) fx = nx - 1; }
    if (fy < 0) { fy = 0; if (cy < 0) cy = 0; }
    if (cy >= ny) { cy = ny - 1; if (fy >= ny) fy = ny - 1; }
    if (fz < 0) { fz = 0; if (cz < 0) cz = 0; }
    if (cz >= nz) { cz = nz - 1; if (fz >= nz) fz = nz - 1; }
  } else {
    inside = fx >= 0 && cx < nx && fy >= 0 && cy < ny && fz >= 0 && cz < nz;
  }
  /* corner order v0..v7 as in the reference */
  const int X[8] = {fx, cx, cx, fx, fx, cx, cx, fx};
  const int Y[8] = {fy, fy, cy, cy, cy, cy, fy, fy};
  const int Z[8] = {fz, fz, fz, fz, cz, cz, cz, cz};
  if (inside) {
    for (int c = 0; c < 8; ++c) {
      const long i = IDX(X[c], Y[c], Z[c]);
      vX[c] = hxp[i]; vY[c] = hyp[i]; vZ[c] = hzp[i];
    }
  } else if (bgs == AW_BG_ID) {
    *ox = x; *oy = y; *oz = z;
    return;
  } else if (bgs == AW_BG_ZERO) {
    *ox = 0; *oy = 0; *oz = 0;
    return;
  } else { /* PARTIAL_ID / PARTIAL_ZERO */
    for (int c = 0; c < 8; ++c) {
      if (bgs == AW_BG_PARTIAL_ID) {
        vX[c] = (float)X[c]; vY[c] = (float)Y[c]; vZ[c] = (float)Z[c];
      }
      const int in = X[c] >= 0 && X[c] < nx && Y[c] >= 0 && Y[c] < ny && Z[c] >= 0 && Z[c] < nz;
      if (in) {
        const long i = IDX(X[c], Y[c], Z[c]);
        vX[c] = hxp[i]; vY[c] = hyp[i]; vZ[c] = hzp[i];
      }
    }
  }
  /* v0..v7 = index 0..7 */
  *ox = (float)(omt * (omu * (vX[0] * omv + vX[7] * v) + u * (vX[3] * omv + vX[4] * v)) +
                t * (omu * (vX[1] * omv + vX[6] * v) + u * (vX[2] * omv + vX[5] * v)));
  *oy = (float)(omt * (omu * (vY[0] * omv + vY[7] * v) + u * (vY[3] * omv + vY[4] * v)) +
                t * (omu * (vY[1] * omv + vY[6] * v) + u * (vY[2] * omv + vY[5] * v)));
  *oz = (float)(omt * (omu * (vZ[0] * omv + vZ[7] * v) + u * (vZ[3] * omv + vZ[4] * v)) +
                t * (omu * (vZ[1] * omv + vZ[6] * v) + u * (vZ[2] * omv + vZ[5] * v)));
}

/* I_def(x) = I(h(x)); HField3DUtils::apply (HField3DUtils.txx:734-752). */
void aw_oracle_apply(const float *img, const float *hx, const float *hy, const float *hz,
                     float *out, int nx, int ny, int nz, float bg) {
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const long i = IDX(x, y, z);
        out[i] = trilerp_val(img, nx, ny, nz, (double)hx[i], (double)hy[i], (double)hz[i], bg);
      }
}

/* I(x + v(x)/sp): HField3DUtils::applyU (HField3DUtils.txx, used by LDMM
 * IterateOrig at LDMM/LDMMIteratorCPU.cxx:426). Position in float. */
void aw_oracle_apply_u(const float *img, const float *vx, const float *vy, const float *vz,
                       float *out, int nx, int ny, int nz, double spx, double spy, double spz,
                       float bg) {
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const long i = IDX(x, y, z);
        const float px = (float)x + vx[i] / (float)spx;
        const float py = (float)y + vy[i] / (float)spy;
        const float pz = (float)z + vz[i] / (float)spz;
        out[i] = trilerp_val(img, nx, ny, nz, (double)px, (double)py, (double)pz, bg);
      }
}

/* Array3DUtils::computeGradient (Array3DUtils.txx:783-900). */
void aw_oracle_gradient(const float *a, float *gx, float *gy, float *gz, int nx, int ny, int nz,
                        double spx, double spy, double spz, int wrap) {
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 1; x < nx - 1; ++x)
        gx[IDX(x, y, z)] = (float)((double)(a[IDX(x + 1, y, z)] - a[IDX(x - 1, y, z)]) / (2.0 * spx));
  for (int z = 0; z < nz; ++z)
    for (int y = 1; y < ny - 1; ++y)
      for (int x = 0; x < nx; ++x)
        gy[IDX(x, y, z)] = (float)((double)(a[IDX(x, y + 1, z)] - a[IDX(x, y - 1, z)]) / (2.0 * spy));
  for (int z = 1; z < nz - 1; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x)
        gz[IDX(x, y, z)] = (float)((double)(a[IDX(x, y, z + 1)] - a[IDX(x, y, z - 1)]) / (2.0 * spz));
  if (wrap) {
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y) {
        gx[IDX(0, y, z)] = (float)((double)(a[IDX(1, y, z)] - a[IDX(nx - 1, y, z)]) / (2.0 * spx));
        gx[IDX(nx - 1, y, z)] = (float)((double)(a[IDX(0, y, z)] - a[IDX(nx - 2, y, z)]) / (2.0 * spx));
      }
    for (int z = 0; z < nz; ++z)
      for (int x = 0; x < nx; ++x) {
        gy[IDX(x, 0, z)] = (float)((double)(a[IDX(x, 1, z)] - a[IDX(x, ny - 1, z)]) / (2.0 * spy));
        gy[IDX(x, ny - 1, z)] = (float)((double)(a[IDX(x, 0, z)] - a[IDX(x, ny - 2, z)]) / (2.0 * spy));
      }
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        gz[IDX(x, y, 0)] = (float)((double)(a[IDX(x, y, 1)] - a[IDX(x, y, nz - 1)]) / (2.0 * spz));
        gz[IDX(x, y, nz - 1)] = (float)((double)(a[IDX(x, y, 0)] - a[IDX(x, y, nz - 2)]) / (2.0 * spz));
      }
  } else {
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y) {
        gx[IDX(0, y, z)] = (float)((double)(a[IDX(1, y, z)] - a[IDX(0, y, z)]) / spx);
        gx[IDX(nx - 1, y, z)] = (float)((double)(a[IDX(nx - 1, y, z)] - a[IDX(nx - 2, y, z)]) / spx);
      }
    for (int z = 0; z < nz; ++z)
      for (int x = 0; x < nx; ++x) {
        gy[IDX(x, 0, z)] = (float)((double)(a[IDX(x, 1, z)] - a[IDX(x, 0, z)]) / spy);
        gy[IDX(x, ny - 1, z)] = (float)((double)(a[IDX(x, ny - 1, z)] - a[IDX(x, ny - 2, z)]) / spy);
      }
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        gz[IDX(x, y, 0)] = (float)((double)(a[IDX(x, y, 1)] - a[IDX(x, y, 0)]) / spz);
        gz[IDX(x, y, nz - 1)] = (float)((double)(a[IDX(x, y, nz - 1)] - a[IDX(x, y, nz - 2)]) / spz);
      }
  }
}

/* h(x) = g(x + dir * v(x)/sp): composeHV (dir=+1, HField3DUtils.txx:436-455)
 * and composeHVInv (dir=-1, HField3DUtils.txx:461-480). */
void aw_oracle_compose_hv(const float *gx, const float *gy, const float *gz, const float *vx,
                          const float *vy, const float *vz, float *ox, float *oy, float *oz,
                          int nx, int ny, int nz, double spx, double spy, double spz, int dir,
                          int bgs) {
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const long i = IDX(x, y, z);
        float px, py, pz;
        if (dir > 0) {
          px = (float)x + vx[i] / (float)spx;
          py = (float)y + vy[i] / (float)spy;
          pz = (float)z + vz[i] / (float)spz;
        } else {
          px = (float)x - vx[i] / (float)spx;
          py = (float)y - vy[i] / (float)spy;
          pz = (float)z - vz[i] / (float)spz;
        }
        trilerp_vec(gx, gy, gz, nx, ny, nz, px, py, pz, &ox[i], &oy[i], &oz[i], bgs);
      }
}

/* h(x) = g(x) + dir * v(g(x))/sp: composeVH (dir=+1) and composeVHInv
 * (dir=-1, HField3DUtils.txx:405-430). The interpolated value is rounded to
 * float, divided by (dir*sp) in float, then g(x) is added in float. */
void aw_oracle_compose_vh(const float *vx, const float *vy, const float *vz, const float *gx,
                          const float *gy, const float *gz, float *ox, float *oy, float *oz,
                          int nx, int ny, int nz, double spx, double spy, double spz, int dir,
                          int bgs) {
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const long i = IDX(x, y, z);
        float hx, hy, hz;
        trilerp_vec(vx, vy, vz, nx, ny, nz, gx[i], gy[i], gz[i], &hx, &hy, &hz, bgs);
        if (dir > 0) {
          hx /= (float)spx; hy /= (float)spy; hz /= (float)spz;
        } else {
          hx /= -((float)spx); hy /= -((float)spy); hz /= -((float)spz);
        }
        ox[i] = hx + gx[i];
        oy[i] = hy + gy[i];
        oz[i] = hz + gz[i];
      }
}

/* Splat, the adjoint of interpolation: HField3DUtils::forwardApply with
 * hFieldStart = 0 and normalize = false (HField3DUtils.txx:1058-1279).
 * Contributions land in source (z,y,x) order, accumulated in float. */
void aw_oracle_splat(const float *img, const float *hx, const float *hy, const float *hz,
                     float *out, int nx, int ny, int nz, float bg) {
  const long n = (long)nx * ny * nz;
  for (long i = 0; i < n; ++i) out[i] = bg;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const long i = IDX(x, y, z);
        const float ix = img[i];
        const float px = hx[i], py = hy[i], pz = hz[i];
        int fx = (int)px, fy = (int)py, fz = (int)pz;
        if (px < 0 && px != (float)(int)px) --fx;
        if (py < 0 && py != (float)(int)py) --fy;
        if (pz < 0 && pz != (float)(int)pz) --fz;
        if (px > -1 && px < (float)nx && py > -1 && py < (float)ny && pz > -1 && pz < (float)nz) {
          const float rx = px - (float)fx, ry = py - (float)fy, rz = pz - (float)fz;
          const float w000 = (float)((1.0 - rx) * (1.0 - ry) * (1.0 - rz));
          const float w001 = (float)((1.0 - rx) * (1.0 - ry) * (rz));
          const float w010 = (float)((1.0 - rx) * (ry) * (1.0 - rz));
          const float w011 = (float)((1.0 - rx) * (ry) * (rz));
          const float w100 = (float)((rx) * (1.0 - ry) * (1.0 - rz));
          const float w101 = (float)((rx) * (1.0 - ry) * (rz));
          const float w110 = (float)((rx) * (ry) * (1.0 - rz));
          const float w111 = (float)((rx) * (ry) * (rz));
          const int fxi = fx >= 0, cxi = fx < nx - 1, fyi = fy >= 0, cyi = fy < ny - 1,
                    fzi = fz >= 0, czi = fz < nz - 1;
          if (fxi && fyi && fzi) out[IDX(fx, fy, fz)] += w000 * ix;
          if (fxi && fyi && czi) out[IDX(fx, fy, fz + 1)] += w001 * ix;
          if (fxi && cyi && fzi) out[IDX(fx, fy + 1, fz)] += w010 * ix;
          if (fxi && cyi && czi) out[IDX(fx, fy + 1, fz + 1)] += w011 * ix;
          if (cxi && fyi && fzi) out[IDX(fx + 1, fy, fz)] += w100 * ix;
          if (cxi && fyi && czi) out[IDX(fx + 1, fy, fz + 1)] += w101 * ix;
          if (cxi && cyi && fzi) out[IDX(fx + 1, fy + 1, fz)] += w110 * ix;
          if (cxi && cyi && czi) out[IDX(fx + 1, fy + 1, fz + 1)] += w111 * ix;
        }
      }
}

/* ------------------------------------------------------------------------
 * Fluid operator L = -alpha*Lap - beta*grad(div) + gamma and its inverse,
 * evaluated per wavenumber exactly as DiffOperT::ApplyInverseOperatorOnTheFly
 * / ApplyOperatorOnTheFly (Algorithms/Common/DiffOper.cxx:755-905) with the
 * LUT of DiffOper.cxx:590-639 and the Cholesky solve of DiffOper.cxx:
 * 1005-1083, all in double. The forward transform covers the full complex
 * spectrum of the real input; the result is its real part (equal to FFTW's
 * r2c -> solve -> c2r on the non-redundant half).
 * ---------------------------------------------------------------------- */
static void lut_axis(int n, double sp, double *cw, double *sw) {
  const double s = 2.0 * M_PI / n;
  for (int k = 0; k < n; ++k) {
    cw[k] = (2.0 * cos(s * (double)k) - 2.0) / (sp * sp);
    sw[k] = sin(s * (double)k) / sp;
  }
}

void aw_oracle_fluid_apply_f64(double *vx, double *vy, double *vz, int nx, int ny, int nz,
                               double spx, double spy, double spz, double alpha, double beta,
                               double gamma, int inverse) {
  const long n = (long)nx * ny * nz;
  fft64_cplx *F[3];
  double *V[3] = {vx, vy, vz};
  for (int c = 0; c < 3; ++c) {
    F[c] = (fft64_cplx *)malloc(sizeof(fft64_cplx) * (size_t)n);
    for (long i = 0; i < n; ++i) {
      F[c][i].re = V[c][i] / (double)n;
      F[c][i].im = 0.0;
    }
    fft64_3d(F[c], nx, ny, nz, -1);
  }
  double *cwx = (double *)malloc(sizeof(double) * (size_t)(2 * (nx + ny + nz)));
  double *swx = cwx + nx, *cwy = swx + nx, *swy = cwy + ny, *cwz = swy + ny, *swz = cwz + nz;
  lut_axis(nx, spx, cwx, swx);
  lut_axis(ny, spy, cwy, swy);
  lut_axis(nz, spz, cwz, swz);
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const long i = IDX(x, y, z);
        const double lambda = -alpha * (cwx[x] + cwy[y] + cwz[z]) + gamma;
        const double L00 = lambda - beta * cwx[x];
        const double L11 = lambda - beta * cwy[y];
        const double L22 = lambda - beta * cwz[z];
        const double L10 = beta * swx[x] * swy[y];
        const double L20 = beta * swx[x] * swz[z];
        const double L21 = beta * swy[y] * swz[z];
        double b[2][3] = {{F[0][i].re, F[1][i].re, F[2][i].re},
                          {F[0][i].im, F[1][i].im, F[2][i].im}};
        double o[2][3];
        if (inverse) {
          const double G00 = sqrt(L00);
          const double G10 = L10 / G00;
          const double G20 = L20 / G00;
          double G11 = L11 - G10 * G10;
          double G21 = L21 - G20 * G10;
          G11 = sqrt(G11);
          G21 = G21 / G11;
          double G22 = L22 - (G20 * G20 + G21 * G21);
          G22 = sqrt(G22);
          for (int p = 0; p < 2; ++p) {
            const double y0 = b[p][0] / G00;
            const double y1 = (b[p][1] - G10 * y0) / G11;
            const double y2 = (b[p][2] - G20 * y0 - G21 * y1) / G22;
            o[p][2] = y2 / G22;
            o[p][1] = (y1 - G21 * o[p][2]) / G11;
            o[p][0] = (y0 - G10 * o[p][1] - G20 * o[p][2]) / G00;
          }
        } else {
          for (int p = 0; p < 2; ++p) {
            o[p][0] = L00 * b[p][0] + L10 * b[p][1] + L20 * b[p][2];
            o[p][1] = L10 * b[p][0] + L11 * b[p][1] + L21 * b[p][2];
            o[p][2] = L20 * b[p][0] + L21 * b[p][1] + L22 * b[p][2];
          }
        }
        for (int c = 0; c < 3; ++c) {
          F[c][i].re = o[0][c];
          F[c][i].im = o[1][c];
        }
      }
  for (int c = 0; c < 3; ++c) {
    fft64_3d(F[c], nx, ny, nz, +1);
    for (long i = 0; i < n; ++i) V[c][i] = F[c][i].re;
    free(F[c]);
  }
  free(cwx);
}

/* float in/out wrapper: widen, apply in FP64, round back */
void aw_oracle_fluid_apply(float *vx, float *vy, float *vz, int nx, int ny, int nz, double spx,
                           double spy, double spz, double alpha, double beta, double gamma,
                           int inverse) {
  const long n = (long)nx * ny * nz;
  double *d = (double *)malloc(sizeof(double) * (size_t)(3 * n));
  float *V[3] = {vx, vy, vz};
  for (int c = 0; c < 3; ++c)
    for (long i = 0; i < n; ++i) d[c * n + i] = V[c][i];
  aw_oracle_fluid_apply_f64(d, d + n, d + 2 * n, nx, ny, nz, spx, spy, spz, alpha, beta, gamma,
                            inverse);
  for (int c = 0; c < 3; ++c)
    for (long i = 0; i < n; ++i) V[c][i] = (float)d[c * n + i];
  free(d);
}

/* max_x |v(x)|, the float norm of Vector3D::normL2 (DataTypes/Vector3D.txx:
 * 100-103) as used by GreedyIteratorCPU::calcMaxDisplacement
 * (Greedy/GreedyIteratorCPU.cxx:65-79). */
float aw_oracle_max_norm(const float *vx, const float *vy, const float *vz, long n) {
  float m = 0.0f;
  for (long i = 0; i < n; ++i) {
    const float l = sqrtf(vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]);
    if (l > m) m = l;
  }
  return m;
}

/* ------------------------------------------------------------------------
 * One greedy-fluid iteration, GreedyIteratorCPU::Iterate
 * (Algorithms/Greedy/GreedyIteratorCPU.cxx:99-138) with updateDeformation
 * (:83-95). h (and hinv when non-NULL) are updated in place. *step is read,
 * and replaced by maxPert / max|v| when update_step is set. Returns the
 * energy spacing^3 * sum (I1 - I0(h))^2 of the incoming h, accumulated in
 * double (the reference accumulates in float).
 * ---------------------------------------------------------------------- */
/* The iteration after I0(h): GreedyIteratorCPU::Iterate from the gradient
 * on (Greedy/GreedyIteratorCPU.cxx:105-137). idef = I0(h). */
static double greedy_iterate_idef(const float *idef, const float *I1, float *hx, float *hy,
                                  float *hz, float *hix, float *hiy, float *hiz, int nx, int ny,
                                  int nz, double spx, double spy, double spz, double alpha,
                                  double beta, double gamma, float max_pert, int update_step,
                                  float *step) {
  const long n = (long)nx * ny * nz;
  float *f = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *o = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *fx = f, *fy = f + n, *fz = f + 2 * n;
  aw_oracle_gradient(idef, fx, fy, fz, nx, ny, nz, spx, spy, spz, 0);
  double e = 0.0;
  for (long i = 0; i < n; ++i) {
    float r = idef[i] - I1[i];
    r = r * -1.0f;
    fx[i] *= r;
    fy[i] *= r;
    fz[i] *= r;
    e += (double)r * (double)r;
  }
  e *= spx * spy * spz;
  aw_oracle_fluid_apply(fx, fy, fz, nx, ny, nz, spx, spy, spz, alpha, beta, gamma, 1);
  if (update_step) {
    const float m = aw_oracle_max_norm(fx, fy, fz, n);
    *step = max_pert / m;
  }
  const float s = *step;
  for (long i = 0; i < 3 * n; ++i) f[i] *= s;
  aw_oracle_compose_hv(hx, hy, hz, fx, fy, fz, o, o + n, o + 2 * n, nx, ny, nz, spx, spy, spz, 1,
                       AW_BG_PARTIAL_ID);
  memcpy(hx, o, sizeof(float) * (size_t)n);
  memcpy(hy, o + n, sizeof(float) * (size_t)n);
  memcpy(hz, o + 2 * n, sizeof(float) * (size_t)n);
  if (hix) {
    aw_oracle_compose_vh(fx, fy, fz, hix, hiy, hiz, o, o + n, o + 2 * n, nx, ny, nz, spx, spy,
                         spz, -1, AW_BG_PARTIAL_ZERO);
    memcpy(hix, o, sizeof(float) * (size_t)n);
    memcpy(hiy, o + n, sizeof(float) * (size_t)n);
    memcpy(hiz, o + 2 * n, sizeof(float) * (size_t)n);
  }
  free(f);
  free(o);
  return e;
}

double aw_oracle_greedy_iterate(const float *I0, const float *I1, float *hx, float *hy, float *hz,
                                float *hix, float *hiy, float *hiz, int nx, int ny, int nz,
                                double spx, double spy, double spz, double alpha, double beta,
                                double gamma, float max_pert, int update_step, float *step) {
  const long n = (long)nx * ny * nz;
  float *idef = (float *)malloc(sizeof(float) * (size_t)n);
  aw_oracle_apply(I0, hx, hy, hz, idef, nx, ny, nz, 0.0f);
  const double e = greedy_iterate_idef(idef, I1, hx, hy, hz, hix, hiy, hiz, nx, ny, nz, spx, spy,
                                       spz, alpha, beta, gamma, max_pert, update_step, step);
  free(idef);
  return e;
}

/* I(h) for an atlas subject on its own grid (mx, my, mz) with h on the
 * template grid (nx, ny, nz): the sample point is (h + 0.5) * (m / n) - 0.5
 * per axis in double; with equal grids it is h itself
 * (HField3DUtils::apply, UtilitiesDataTypes/HField3DUtils.txx:734-752). */
void aw_oracle_apply_atlas(const float *img, int mx, int my, int mz, const float *hx,
                           const float *hy, const float *hz, float *out, int nx, int ny, int nz) {
  const int same = mx == nx && my == ny && mz == nz;
  const double rx = (double)mx / (double)nx, ry = (double)my / (double)ny,
               rz = (double)mz / (double)nz;
  const long n = (long)nx * ny * nz;
  for (long i = 0; i < n; ++i) {
    double px = (double)hx[i], py = (double)hy[i], pz = (double)hz[i];
    if (!same) {
      px = (px + 0.5) * rx - 0.5;
      py = (py + 0.5) * ry - 0.5;
      pz = (pz + 0.5) * rz - 0.5;
    }
    out[i] = trilerp_val(img, mx, my, mz, px, py, pz, 0.0f);
  }
}

/* One greedy iteration of atlas subject (I0 on its own grid) toward the
 * mean I1 (template grid): the iteration of AtlasThread::AtlasThreadMain
 * (Common/AtlasThread.txx:137-152) for one image. */
double aw_oracle_atlas_iterate(const float *I0, int mx, int my, int mz, const float *I1, float *hx,
                               float *hy, float *hz, int nx, int ny, int nz, double spx,
                               double spy, double spz, double alpha, double beta, double gamma,
                               float max_pert, int update_step, float *step) {
  const long n = (long)nx * ny * nz;
  float *idef = (float *)malloc(sizeof(float) * (size_t)n);
  aw_oracle_apply_atlas(I0, mx, my, mz, hx, hy, hz, idef, nx, ny, nz);
  const double e = greedy_iterate_idef(idef, I1, hx, hy, hz, NULL, NULL, NULL, nx, ny, nz, spx,
                                       spy, spz, alpha, beta, gamma, max_pert, update_step, step);
  free(idef);
  return e;
}

/* The thread mean of GreedyAtlasThreadCPU::ComputeThreadMean
 * (Greedy/GreedyAtlasThreadCPU.cxx): mean = 0, then for each subject in
 * order mean[j] += I_i(h_i)[j] * w_i in float. dims holds (mx, my, mz) per
 * subject, h holds 3 pointers per subject. */
void aw_oracle_atlas_mean(const float *const *imgs, const int *dims, const float *const *h,
                          const float *w, int ns, float *mean, int nx, int ny, int nz) {
  const long n = (long)nx * ny * nz;
  float *d = (float *)malloc(sizeof(float) * (size_t)n);
  for (long j = 0; j < n; ++j) mean[j] = 0.0f;
  for (int k = 0; k < ns; ++k) {
    aw_oracle_apply_atlas(imgs[k], dims[3 * k], dims[3 * k + 1], dims[3 * k + 2], h[3 * k],
                          h[3 * k + 1], h[3 * k + 2], d, nx, ny, nz);
    for (long j = 0; j < n; ++j) mean[j] += d[j] * w[k];
  }
  free(d);
}

void aw_oracle_identity(float *hx, float *hy, float *hz, int nx, int ny, int nz) {
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const long i = IDX(x, y, z);
        hx[i] = (float)x;
        hy[i] = (float)y;
        hz[i] = (float)z;
      }
}

/* ------------------------------------------------------------------------
 * LDMM relaxation, LDMMIteratorCPU::IterateNew (LDMM/LDMMIteratorCPU.cxx:
 * 529-631): forward integration by composeHVInv + apply, the residual
 * J0_{T-1} - I1, then for t = T-1..0: composeVHInv (PARTIAL_ZERO), splat of
 * the residual (forwardApply), body force grad(J0_{t-1}) * splat, K, and
 * v_t <- (1 - 2 eps) v_t + (2 eps / sigma^2) K f (updateVelocity, :177-190).
 * With update_step set, v is left unchanged and *step becomes
 * max_pert / max_t max_x |2 v_t - (2/sigma^2) K f_t| (calcMaxDisplacement,
 * :192-212). v is [T][3][N]. Returns the image energy sp^3 * sum diff^2
 * (accumulated in double).
 * ---------------------------------------------------------------------- */
/* <L v, v> sp^3 of LDMMIteratorCPU's debug mode (HField3DUtils::l2DotProd of
 * L v and v, LDMMIteratorCPU.cxx:493-505, 601-610): L applied by the FP32
 * operator, the float products summed in double */
static double vec_step_energy(const float *vt, long n, int nx, int ny, int nz, double spx,
                              double spy, double spz, double alpha, double beta, double gamma) {
  float *lv = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  memcpy(lv, vt, sizeof(float) * (size_t)(3 * n));
  aw_oracle_fluid_apply(lv, lv + n, lv + 2 * n, nx, ny, nz, spx, spy, spz, alpha, beta, gamma, 0);
  double e = 0.0;
  for (long k = 0; k < 3 * n; ++k) e += (double)(lv[k] * vt[k]);
  free(lv);
  return e * spx * spy * spz;
}

double aw_oracle_ldmm_iterate(const float *I0, const float *I1, float *v, int T, int nx, int ny,
                              int nz, double spx, double spy, double spz, double alpha,
                              double beta, double gamma, float sigma, float *step,
                              int update_step, float max_pert, double *vec_energy) {
  const long n = (long)nx * ny * nz;
  float *h = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *o = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *J0 = (float *)malloc(sizeof(float) * (size_t)(T * n));
  float *diff = (float *)malloc(sizeof(float) * (size_t)n);
  float *S = (float *)malloc(sizeof(float) * (size_t)n);
  float *f = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  aw_oracle_identity(h, h + n, h + 2 * n, nx, ny, nz);
  for (int i = 0; i < T; ++i) {
    float *vi = v + (long)i * 3 * n;
    aw_oracle_compose_hv(h, h + n, h + 2 * n, vi, vi + n, vi + 2 * n, o, o + n, o + 2 * n, nx, ny,
                         nz, spx, spy, spz, -1, AW_BG_PARTIAL_ID);
    memcpy(h, o, sizeof(float) * (size_t)(3 * n));
    aw_oracle_apply(I0, h, h + n, h + 2 * n, J0 + (long)i * n, nx, ny, nz, 0.0f);
  }
  double e = 0.0;
  for (long k = 0; k < n; ++k) {
    diff[k] = J0[(long)(T - 1) * n + k] - I1[k];
    e += (double)diff[k] * (double)diff[k];
  }
  e *= spx * spy * spz;
  const float vfac = 1.f - 2 * *step;
  const float ufac = 2 * *step / (sigma * sigma);
  float total_max = 0.f;
  double vsum = 0.0;
  aw_oracle_identity(h, h + n, h + 2 * n, nx, ny, nz);
  for (int t = T - 1; t >= 0; --t) {
    float *vt = v + (long)t * 3 * n;
    aw_oracle_compose_vh(vt, vt + n, vt + 2 * n, h, h + n, h + 2 * n, o, o + n, o + 2 * n, nx, ny,
                         nz, spx, spy, spz, -1, AW_BG_PARTIAL_ZERO);
    memcpy(h, o, sizeof(float) * (size_t)(3 * n));
    aw_oracle_splat(diff, h, h + n, h + 2 * n, S, nx, ny, nz, 0.0f);
    const float *G = (t > 0) ? J0 + (long)(t - 1) * n : I0;
    aw_oracle_gradient(G, f, f + n, f + 2 * n, nx, ny, nz, spx, spy, spz, 0);
    for (long k = 0; k < n; ++k) {
      f[k] *= S[k];
      f[n + k] *= S[k];
      f[2 * n + k] *= S[k];
    }
    aw_oracle_fluid_apply(f, f + n, f + 2 * n, nx, ny, nz, spx, spy, spz, alpha, beta, gamma, 1);
    if (update_step) {
      const float a = 2.0f, b = -2.0f / (sigma * sigma);
      for (long k = 0; k < n; ++k) {
        const float x = a * vt[k] + b * f[k];
        const float y = a * vt[n + k] + b * f[n + k];
        const float zz = a * vt[2 * n + k] + b * f[2 * n + k];
        const float len = (float)sqrt((double)(x * x + y * y + zz * zz));
        if (len > total_max) total_max = len;
      }
    } else {
      for (long k = 0; k < 3 * n; ++k) vt[k] = vfac * vt[k] + ufac * f[k];
      if (vec_energy)
        vsum += vec_step_energy(vt, n, nx, ny, nz, spx, spy, spz, alpha, beta, gamma);
    }
  }
  if (update_step) *step = max_pert / total_max;
  if (vec_energy) *vec_energy = vsum;
  free(h);
  free(o);
  free(J0);
  free(diff);
  free(S);
  free(f);
  return e;
}

/* LDMMIteratorCPU::IterateNew with computeAlphasOnly (LDMM/LDMMIteratorCPU.cxx:
 * 543-586): the forward deformed images, the residual J0_{T-1} - I1, then per
 * t from T-1 down: h = composeVHInv(v_t, h) [PARTIAL_ZERO], the residual
 * splatted by h (forwardApply, normalize off) and scaled by
 * (float)(1.0 / (sigma*sigma)) into alphas[t]. Returns the image energy. */
double aw_oracle_ldmm_alphas(const float *I0, const float *I1, const float *v, int T, int nx,
                             int ny, int nz, double spx, double spy, double spz, float sigma,
                             float *alphas) {
  const long n = (long)nx * ny * nz;
  float *h = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *o = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *J = (float *)malloc(sizeof(float) * (size_t)n);
  float *diff = (float *)malloc(sizeof(float) * (size_t)n);
  aw_oracle_identity(h, h + n, h + 2 * n, nx, ny, nz);
  for (int i = 0; i < T; ++i) {
    const float *vi = v + (long)i * 3 * n;
    aw_oracle_compose_hv(h, h + n, h + 2 * n, vi, vi + n, vi + 2 * n, o, o + n, o + 2 * n, nx, ny,
                         nz, spx, spy, spz, -1, AW_BG_PARTIAL_ID);
    memcpy(h, o, sizeof(float) * (size_t)(3 * n));
  }
  aw_oracle_apply(I0, h, h + n, h + 2 * n, J, nx, ny, nz, 0.0f);
  double e = 0.0;
  for (long k = 0; k < n; ++k) {
    diff[k] = J[k] - I1[k];
    e += (double)diff[k] * (double)diff[k];
  }
  e *= spx * spy * spz;
  const float f = (float)(1.0 / (sigma * sigma));
  aw_oracle_identity(h, h + n, h + 2 * n, nx, ny, nz);
  for (int t = T - 1; t >= 0; --t) {
    const float *vt = v + (long)t * 3 * n;
    aw_oracle_compose_vh(vt, vt + n, vt + 2 * n, h, h + n, h + 2 * n, o, o + n, o + 2 * n, nx, ny,
                         nz, spx, spy, spz, -1, AW_BG_PARTIAL_ZERO);
    memcpy(h, o, sizeof(float) * (size_t)(3 * n));
    float *a = alphas + (long)t * n;
    aw_oracle_splat(diff, h, h + n, h + 2 * n, a, nx, ny, nz, 0.0f);
    for (long k = 0; k < n; ++k) a[k] = a[k] * f;
  }
  free(h);
  free(o);
  free(J);
  free(diff);
  return e;
}

/* |D(x*sp + v)|: HField3DUtils::jacobian (UtilitiesDataTypes/HField3DUtils.txx:
 * 2374-2420) of the world-coordinate map that LDMMIteratorCPU::IterateOrig
 * forms (LDMM/LDMMIteratorCPU.cxx:409-417: identity scaled by the float
 * spacing, plus v): float components, gradients by computeGradient
 * (wrap = false), the determinant expanded along its first row in float. */
void aw_oracle_jacobian(const float *vx, const float *vy, const float *vz, float *jac, int nx,
                        int ny, int nz, double spx, double spy, double spz) {
  const long n = (long)nx * ny * nz;
  float *w = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *g = (float *)malloc(sizeof(float) * (size_t)(9 * n));
  const float sx = (float)spx, sy = (float)spy, sz = (float)spz;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const long i = IDX(x, y, z);
        w[i] = (float)x * sx + vx[i];
        w[n + i] = (float)y * sy + vy[i];
        w[2 * n + i] = (float)z * sz + vz[i];
      }
  for (int c = 0; c < 3; ++c)
    aw_oracle_gradient(w + c * n, g + 3 * c * n, g + (3 * c + 1) * n, g + (3 * c + 2) * n, nx, ny,
                       nz, spx, spy, spz, 0);
  for (long i = 0; i < n; ++i) {
    const float ax = g[i], ay = g[n + i], az = g[2 * n + i];           /* grad h1 */
    const float bx = g[3 * n + i], by = g[4 * n + i], bz = g[5 * n + i]; /* grad h2 */
    const float cx = g[6 * n + i], cy = g[7 * n + i], cz = g[8 * n + i]; /* grad h3 */
    const float t1 = ax * (by * cz - bz * cy);
    const float t2 = ay * (bx * cz - bz * cx);
    const float t3 = az * (bx * cy - by * cx);
    jac[i] = t1 - t2 + t3;
  }
  free(w);
  free(g);
}

/* ------------------------------------------------------------------------
 * LDMM relaxation, LDMMIteratorCPU::IterateOrig (LDMM/LDMMIteratorCPU.cxx:
 * 377-527): a backward sweep t = T-1..0 composing h <- h(x + v_t/sp)
 * [PARTIAL_ID], JT_t = I1(h) and the Jacobian transport
 * JacDet_t = JacDet_{t+1}(x + v_t/sp) * |D(x + v_t)| (applyU); then a
 * forward sweep t = 0..T-1 with S = I0 (t = 0) or I0(h), the body force
 * grad(S) * ((S - JT_t) * JacDet_t), K, the velocity update (or, with
 * update_step, the max of |(-2/sigma^2) K f + 2 v_t|), and
 * h <- h(x - v_t/sp) [PARTIAL_ID] with the updated v_t. Returns the image
 * energy sp^3 * sum (I0(h) - I1)^2 after the sweep (0 with update_step).
 * ---------------------------------------------------------------------- */
double aw_oracle_ldmm_iterate_orig(const float *I0, const float *I1, float *v, int T, int nx,
                                   int ny, int nz, double spx, double spy, double spz,
                                   double alpha, double beta, double gamma, float sigma,
                                   float *step, int update_step, float max_pert,
                                   double *vec_energy) {
  const long n = (long)nx * ny * nz;
  float *h = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *o = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *JT = (float *)malloc(sizeof(float) * (size_t)(T * n));
  float *JD = (float *)malloc(sizeof(float) * (size_t)(T * n));
  float *S = (float *)malloc(sizeof(float) * (size_t)n);
  float *jac = (float *)malloc(sizeof(float) * (size_t)n);
  float *f = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  aw_oracle_identity(h, h + n, h + 2 * n, nx, ny, nz);
  for (int t = T - 1; t >= 0; --t) {
    float *vt = v + (long)t * 3 * n;
    aw_oracle_compose_hv(h, h + n, h + 2 * n, vt, vt + n, vt + 2 * n, o, o + n, o + 2 * n, nx, ny,
                         nz, spx, spy, spz, 1, AW_BG_PARTIAL_ID);
    memcpy(h, o, sizeof(float) * (size_t)(3 * n));
    aw_oracle_apply(I1, h, h + n, h + 2 * n, JT + (long)t * n, nx, ny, nz, 0.0f);
    aw_oracle_jacobian(vt, vt + n, vt + 2 * n, jac, nx, ny, nz, spx, spy, spz);
    float *jd = JD + (long)t * n;
    if (t == T - 1) {
      memcpy(jd, jac, sizeof(float) * (size_t)n);
    } else {
      aw_oracle_apply_u(JD + (long)(t + 1) * n, vt, vt + n, vt + 2 * n, jd, nx, ny, nz, spx, spy,
                        spz, 0.0f);
      for (long k = 0; k < n; ++k) jd[k] *= jac[k];
    }
  }
  const float vfac = 1.f - 2 * *step;
  const float ufac = 2 * *step / (sigma * sigma);
  float total_max = 0.f;
  double vsum = 0.0;
  aw_oracle_identity(h, h + n, h + 2 * n, nx, ny, nz);
  for (int t = 0; t < T; ++t) {
    float *vt = v + (long)t * 3 * n;
    if (t == 0)
      memcpy(S, I0, sizeof(float) * (size_t)n);
    else
      aw_oracle_apply(I0, h, h + n, h + 2 * n, S, nx, ny, nz, 0.0f);
    aw_oracle_gradient(S, f, f + n, f + 2 * n, nx, ny, nz, spx, spy, spz, 0);
    const float *jt = JT + (long)t * n, *jd = JD + (long)t * n;
    for (long k = 0; k < n; ++k) {
      float m = S[k] - jt[k];
      m = m * jd[k];
      f[k] *= m;
      f[n + k] *= m;
      f[2 * n + k] *= m;
    }
    aw_oracle_fluid_apply(f, f + n, f + 2 * n, nx, ny, nz, spx, spy, spz, alpha, beta, gamma, 1);
    if (update_step) {
      const float b = -2.0f / (sigma * sigma);
      for (long k = 0; k < n; ++k) {
        const float x = b * f[k] + 2.0f * vt[k];
        const float y = b * f[n + k] + 2.0f * vt[n + k];
        const float zz = b * f[2 * n + k] + 2.0f * vt[2 * n + k];
        const float len = (float)sqrt((double)(x * x + y * y + zz * zz));
        if (len > total_max) total_max = len;
      }
    } else {
      for (long k = 0; k < 3 * n; ++k) vt[k] = vfac * vt[k] + ufac * f[k];
      if (vec_energy)
        vsum += vec_step_energy(vt, n, nx, ny, nz, spx, spy, spz, alpha, beta, gamma);
    }
    aw_oracle_compose_hv(h, h + n, h + 2 * n, vt, vt + n, vt + 2 * n, o, o + n, o + 2 * n, nx, ny,
                         nz, spx, spy, spz, -1, AW_BG_PARTIAL_ID);
    memcpy(h, o, sizeof(float) * (size_t)(3 * n));
  }
  if (vec_energy) *vec_energy = vsum;
  double e = 0.0;
  if (update_step) {
    *step = max_pert / total_max;
  } else {
    aw_oracle_apply(I0, h, h + n, h + 2 * n, S, nx, ny, nz, 0.0f);
    for (long k = 0; k < n; ++k) {
      const float r = S[k] - I1[k];
      e += (double)r * (double)r;
    }
    e *= spx * spy * spz;
  }
  free(h);
  free(o);
  free(JT);
  free(JD);
  free(S);
  free(jac);
  free(f);
  return e;
}

/* ------------------------------------------------------------------------
 * LDMM atlas pieces. GetI1At0: I1 pulled back to time 0 through
 * h_{0->1} = (((id)(x + v_{T-1}/sp)) ... )(x + v_0/sp), composeHV with
 * PARTIAL_ID from t = T-1 down to 0, then apply with background 0
 * (LDMMDeformationData::GetDefTTo1 / GetI1AtT, LDMM/LDMMDeformationData.cxx:
 * 255-265, 325-336). ComputeJacDet: JacDet = |D(x*sp + v_0)| *
 * (|D(x*sp + v_1)| * (...)(x + v_1/sp))(x + v_0/sp), the transport of
 * LDMMIteratorCPU::ComputeJacDet (LDMM/LDMMIteratorCPU.cxx:309-340).
 * jd may be NULL.
 * ---------------------------------------------------------------------- */
void aw_oracle_ldmm_i1_at_0(const float *I1, const float *v, int T, int nx, int ny, int nz,
                            double spx, double spy, double spz, float *img, float *jd) {
  const long n = (long)nx * ny * nz;
  float *h = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *o = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *jac = (float *)malloc(sizeof(float) * (size_t)n);
  float *tmp = (float *)malloc(sizeof(float) * (size_t)n);
  aw_oracle_identity(h, h + n, h + 2 * n, nx, ny, nz);
  for (int t = T - 1; t >= 0; --t) {
    const float *vt = v + (long)t * 3 * n;
    aw_oracle_compose_hv(h, h + n, h + 2 * n, vt, vt + n, vt + 2 * n, o, o + n, o + 2 * n, nx, ny,
                         nz, spx, spy, spz, 1, AW_BG_PARTIAL_ID);
    memcpy(h, o, sizeof(float) * (size_t)(3 * n));
    if (jd) {
      aw_oracle_jacobian(vt, vt + n, vt + 2 * n, jac, nx, ny, nz, spx, spy, spz);
      if (t == T - 1) {
        memcpy(jd, jac, sizeof(float) * (size_t)n);
      } else {
        aw_oracle_apply_u(jd, vt, vt + n, vt + 2 * n, tmp, nx, ny, nz, spx, spy, spz, 0.0f);
        for (long k = 0; k < n; ++k) jd[k] = tmp[k] * jac[k];
      }
    }
  }
  aw_oracle_apply(I1, h, h + n, h + 2 * n, img, nx, ny, nz, 0.0f);
  free(h);
  free(o);
  free(jac);
  free(tmp);
}

/* ------------------------------------------------------------------------
 * LDMM geodesic shooting from the initial momentum alpha0,
 * LDMMShootingIteratorCPU::Iterate (LDMM/LDMMShootingIteratorCPU.cxx:
 * 199-304): phi0T = phiT0 = id, alphaT = alpha0, v = K(grad(I0) alphaT);
 * for t = 1..T-1: phi0T = composeVH(v, phi0T) [PARTIAL_ZERO],
 * alphaT = forwardApply(alpha0, phi0T), phiT0 = composeHVInv(phiT0, v)
 * [PARTIAL_ID], I = I0(phiT0), v = K(grad(I) alphaT); then both maps take
 * the last v, diff = I0(phiT0) - I1, alphaT = forwardApply(diff, phiT0) and
 * alpha0 <- (1 - step) alpha0 + (step / sigma^2) alphaT. Returns the image
 * energy sp^3 sum diff^2 (the velocity terms of LDMMEnergy are not formed).
 * ---------------------------------------------------------------------- */
/* <L v, v> sp^3 as HField3DUtils::l2DotProd forms it (HField3DUtils.txx:
 * 190-200): float products, a float sum per component, the three sums
 * added in float, times the spacing product, kept as a float (Real) */
static double l_energy(const float *v, float *scratch, int nx, int ny, int nz, double spx,
                       double spy, double spz, double alpha, double beta, double gamma) {
  const long n = (long)nx * ny * nz;
  memcpy(scratch, v, sizeof(float) * (size_t)(3 * n));
  aw_oracle_fluid_apply(scratch, scratch + n, scratch + 2 * n, nx, ny, nz, spx, spy, spz, alpha,
                        beta, gamma, 0);
  float sx = 0.0f, sy = 0.0f, sz = 0.0f;
  for (long k = 0; k < n; ++k) {
    sx += scratch[k] * v[k];
    sy += scratch[n + k] * v[n + k];
    sz += scratch[2 * n + k] * v[2 * n + k];
  }
  return (double)(float)(spx * spy * spz * (double)(sx + sy + sz));
}

double aw_oracle_ldmm_shoot_iterate(const float *I0, const float *I1, float *alpha0, float *phi0T,
                                    float *phiT0, int T, int nx, int ny, int nz, double spx,
                                    double spy, double spz, double alpha, double beta,
                                    double gamma, float sigma, float step, double *vec_energy) {
  const long n = (long)nx * ny * nz;
  float *v = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *o = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *aT = (float *)malloc(sizeof(float) * (size_t)n);
  float *I = (float *)malloc(sizeof(float) * (size_t)n);
  float *p0 = phi0T, *p1 = phiT0;
  aw_oracle_identity(p0, p0 + n, p0 + 2 * n, nx, ny, nz);
  aw_oracle_identity(p1, p1 + n, p1 + 2 * n, nx, ny, nz);
  memcpy(aT, alpha0, sizeof(float) * (size_t)n);
  /* v = K(grad(G) * alphaT) */
#define AW_SHOOT_VELOCITY(G)                                                                  \
  do {                                                                                        \
    aw_oracle_gradient((G), v, v + n, v + 2 * n, nx, ny, nz, spx, spy, spz, 0);               \
    for (long k = 0; k < n; ++k) {                                                            \
      v[k] *= aT[k];                                                                          \
      v[n + k] *= aT[k];                                                                      \
      v[2 * n + k] *= aT[k];                                                                  \
    }                                                                                         \
    aw_oracle_fluid_apply(v, v + n, v + 2 * n, nx, ny, nz, spx, spy, spz, alpha, beta, gamma, \
                          1);                                                                 \
  } while (0)
  AW_SHOOT_VELOCITY(I0);
  /* sum over t of the step energies <L v_t, v_t> (.cxx:216-221, 257-262) */
  double ev = 0.0;
  for (int t = 1; t < T; ++t) {
    if (vec_energy) ev += l_energy(v, o, nx, ny, nz, spx, spy, spz, alpha, beta, gamma);
    aw_oracle_compose_vh(v, v + n, v + 2 * n, p0, p0 + n, p0 + 2 * n, o, o + n, o + 2 * n, nx, ny,
                         nz, spx, spy, spz, 1, AW_BG_PARTIAL_ZERO);
    memcpy(p0, o, sizeof(float) * (size_t)(3 * n));
    aw_oracle_splat(alpha0, p0, p0 + n, p0 + 2 * n, aT, nx, ny, nz, 0.0f);
    aw_oracle_compose_hv(p1, p1 + n, p1 + 2 * n, v, v + n, v + 2 * n, o, o + n, o + 2 * n, nx, ny,
                         nz, spx, spy, spz, -1, AW_BG_PARTIAL_ID);
    memcpy(p1, o, sizeof(float) * (size_t)(3 * n));
    aw_oracle_apply(I0, p1, p1 + n, p1 + 2 * n, I, nx, ny, nz, 0.0f);
    AW_SHOOT_VELOCITY(I);
  }
#undef AW_SHOOT_VELOCITY
  if (vec_energy) *vec_energy = ev + l_energy(v, o, nx, ny, nz, spx, spy, spz, alpha, beta, gamma);
  aw_oracle_compose_hv(p1, p1 + n, p1 + 2 * n, v, v + n, v + 2 * n, o, o + n, o + 2 * n, nx, ny,
                       nz, spx, spy, spz, -1, AW_BG_PARTIAL_ID);
  memcpy(p1, o, sizeof(float) * (size_t)(3 * n));
  aw_oracle_compose_vh(v, v + n, v + 2 * n, p0, p0 + n, p0 + 2 * n, o, o + n, o + 2 * n, nx, ny,
                       nz, spx, spy, spz, 1, AW_BG_PARTIAL_ZERO);
  memcpy(p0, o, sizeof(float) * (size_t)(3 * n));
  aw_oracle_apply(I0, p1, p1 + n, p1 + 2 * n, I, nx, ny, nz, 0.0f);
  double e = 0.0;
  for (long k = 0; k < n; ++k) {
    I[k] = I[k] - I1[k];
    e += (double)I[k] * (double)I[k];
  }
  e *= spx * spy * spz;
  aw_oracle_splat(I, p1, p1 + n, p1 + 2 * n, aT, nx, ny, nz, 0.0f);
  const float vfac = (float)(1.0 - (double)step);
  const float ufac = step / (sigma * sigma);
  for (long k = 0; k < n; ++k) alpha0[k] = vfac * alpha0[k] + ufac * aT[k];
  free(v);
  free(o);
  free(aT);
  free(I);
  return e;
}

/* LDMMGeodesicShootingCPU::ShootImage(I0, alpha0, T) (Algorithms/LDMM/
 * LDMMGeodesicShootingCPU.cxx:37-157): v = K(grad(I0) alpha0); for t = 1..T-1
 * phi0T = composeVH(v, phi0T) [PARTIAL_ZERO], alphaT = forwardApply(alpha0,
 * phi0T), phiT0 = composeHVInv(phiT0, v) [PARTIAL_ID], I = apply(I0, phiT0),
 * v = K(grad(I) alphaT); then the last step of phiT0 and phi0T and the final
 * image I0(phiT0). */
void aw_oracle_geodesic_shoot(const float *I0, const float *alpha0, int T, int nx, int ny, int nz,
                              double spx, double spy, double spz, double alpha, double beta,
                              double gamma, float *phi0T, float *phiT0, float *img) {
  const long n = (long)nx * ny * nz;
  float *v = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *o = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *aT = (float *)malloc(sizeof(float) * (size_t)n);
  float *p0 = phi0T, *p1 = phiT0;
  aw_oracle_identity(p0, p0 + n, p0 + 2 * n, nx, ny, nz);
  aw_oracle_identity(p1, p1 + n, p1 + 2 * n, nx, ny, nz);
  memcpy(aT, alpha0, sizeof(float) * (size_t)n);
  memcpy(img, I0, sizeof(float) * (size_t)n);
  for (int t = 0; t < T; ++t) {
    /* v = K(grad(I) alphaT) with I = I0 at t = 0 */
    aw_oracle_gradient(img, v, v + n, v + 2 * n, nx, ny, nz, spx, spy, spz, 0);
    for (long k = 0; k < n; ++k) {
      v[k] *= aT[k];
      v[n + k] *= aT[k];
      v[2 * n + k] *= aT[k];
    }
    aw_oracle_fluid_apply(v, v + n, v + 2 * n, nx, ny, nz, spx, spy, spz, alpha, beta, gamma, 1);
    if (t + 1 < T) {
      aw_oracle_compose_vh(v, v + n, v + 2 * n, p0, p0 + n, p0 + 2 * n, o, o + n, o + 2 * n, nx,
                           ny, nz, spx, spy, spz, 1, AW_BG_PARTIAL_ZERO);
      memcpy(p0, o, sizeof(float) * (size_t)(3 * n));
      aw_oracle_splat(alpha0, p0, p0 + n, p0 + 2 * n, aT, nx, ny, nz, 0.0f);
      aw_oracle_compose_hv(p1, p1 + n, p1 + 2 * n, v, v + n, v + 2 * n, o, o + n, o + 2 * n, nx,
                           ny, nz, spx, spy, spz, -1, AW_BG_PARTIAL_ID);
      memcpy(p1, o, sizeof(float) * (size_t)(3 * n));
      aw_oracle_apply(I0, p1, p1 + n, p1 + 2 * n, img, nx, ny, nz, 0.0f);
    }
  }
  aw_oracle_compose_hv(p1, p1 + n, p1 + 2 * n, v, v + n, v + 2 * n, o, o + n, o + 2 * n, nx, ny,
                       nz, spx, spy, spz, -1, AW_BG_PARTIAL_ID);
  memcpy(p1, o, sizeof(float) * (size_t)(3 * n));
  aw_oracle_compose_vh(v, v + n, v + 2 * n, p0, p0 + n, p0 + 2 * n, o, o + n, o + 2 * n, nx, ny,
                       nz, spx, spy, spz, 1, AW_BG_PARTIAL_ZERO);
  memcpy(p0, o, sizeof(float) * (size_t)(3 * n));
  aw_oracle_apply(I0, p1, p1 + n, p1 + 2 * n, img, nx, ny, nz, 0.0f);
  free(v);
  free(o);
  free(aT);
}

/* LDMMVelShootingIteratorCPU::Iterate (Algorithms/LDMM/
 * LDMMVelShootingIteratorCPU.cxx:186-344): the geodesic in velocity form
 * from v0, v_t = K(|D phiT0| (D phiT0)^T (L v0)(phiT0)), D phiT0 accumulated
 * as identity plus the gradients of the velocity components pulled back by
 * phiT0, both maps advanced by composeHVInv [PARTIAL_ID] / composeVH
 * [PARTIAL_ZERO]; then the residual I0(phiT0) - I1 splatted by phiT0,
 * K(grad(I0) * splat) and the velocity update v0 = (1 - 2 step) v0 +
 * (2 step / sigma^2) K(...) (or, with update_step, step = max_pert / max
 * |2 v0 - (2/sigma^2) K(...)|). v0, phi0T, phiT0 are [3][N]. Returns the
 * image energy sp^3 sum diff^2; *vec_energy = sum_t <L v_t, v_t>. */
double aw_oracle_ldmm_velshoot_iterate(const float *I0, const float *I1, float *v0, float *phi0T,
                                       float *phiT0, int T, int nx, int ny, int nz, double spx,
                                       double spy, double spz, double alpha, double beta,
                                       double gamma, float sigma, float *step, int update_step,
                                       float max_pert, double *vec_energy) {
  const long n = (long)nx * ny * nz;
  float *vt = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *lv0 = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *dp = (float *)malloc(sizeof(float) * (size_t)(9 * n)); /* rows x | y | z, each [3][N] */
  float *o = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *g = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  float *si = (float *)malloc(sizeof(float) * (size_t)n);
  float *p0 = phi0T, *p1 = phiT0;
  aw_oracle_identity(p0, p0 + n, p0 + 2 * n, nx, ny, nz);
  aw_oracle_identity(p1, p1 + n, p1 + 2 * n, nx, ny, nz);
  memcpy(vt, v0, sizeof(float) * (size_t)(3 * n));
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      for (long k = 0; k < n; ++k) dp[(long)(3 * r + c) * n + k] = r == c ? 1.0f : 0.0f;
  memcpy(lv0, v0, sizeof(float) * (size_t)(3 * n));
  aw_oracle_fluid_apply(lv0, lv0 + n, lv0 + 2 * n, nx, ny, nz, spx, spy, spz, alpha, beta, gamma,
                        0);
  double ev = 0.0;
  for (int t = 0; t < T; ++t) {
    ev += l_energy(vt, o, nx, ny, nz, spx, spy, spz, alpha, beta, gamma);
    aw_oracle_compose_hv(p1, p1 + n, p1 + 2 * n, vt, vt + n, vt + 2 * n, o, o + n, o + 2 * n, nx,
                         ny, nz, spx, spy, spz, -1, AW_BG_PARTIAL_ID);
    memcpy(p1, o, sizeof(float) * (size_t)(3 * n));
    aw_oracle_compose_vh(vt, vt + n, vt + 2 * n, p0, p0 + n, p0 + 2 * n, o, o + n, o + 2 * n, nx,
                         ny, nz, spx, spy, spz, 1, AW_BG_PARTIAL_ZERO);
    memcpy(p0, o, sizeof(float) * (size_t)(3 * n));
    if (t == T - 1) break;
    for (int r = 0; r < 3; ++r) {
      aw_oracle_apply(vt + (long)r * n, p1, p1 + n, p1 + 2 * n, si, nx, ny, nz, 0.0f);
      aw_oracle_gradient(si, g, g + n, g + 2 * n, nx, ny, nz, spx, spy, spz, 0);
      float *row = dp + (long)3 * r * n;
      for (long k = 0; k < 3 * n; ++k) row[k] += g[k];
    }
    /* (L v0)(phiT0) with PARTIAL_ZERO, then (D phiT0)^T times it and |D phiT0| */
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
          const long i = IDX(x, y, z);
          float lx, ly, lz;
          trilerp_vec(lv0, lv0 + n, lv0 + 2 * n, nx, ny, nz, p1[i], p1[n + i], p1[2 * n + i], &lx,
                      &ly, &lz, AW_BG_PARTIAL_ZERO);
          const float xx = dp[i], xy = dp[n + i], xz = dp[2 * n + i];
          const float yx = dp[3 * n + i], yy = dp[4 * n + i], yz = dp[5 * n + i];
          const float zx = dp[6 * n + i], zy = dp[7 * n + i], zz = dp[8 * n + i];
          const float fx = xx * lx + yx * ly + zx * lz;
          const float fy = xy * lx + yy * ly + zy * lz;
          const float fz = xz * lx + yz * ly + zz * lz;
          const float t1 = xx * (yy * zz - yz * zy);
          const float t2 = xy * (yx * zz - yz * zx);
          const float t3 = xz * (yx * zy - yy * zx);
          const float det = t1 - t2 + t3;
          o[i] = fx * det;
          o[n + i] = fy * det;
          o[2 * n + i] = fz * det;
        }
    aw_oracle_fluid_apply(o, o + n, o + 2 * n, nx, ny, nz, spx, spy, spz, alpha, beta, gamma, 1);
    memcpy(vt, o, sizeof(float) * (size_t)(3 * n));
  }
  if (vec_energy) *vec_energy = ev;
  /* residual, its energy, its splat by phiT0 and K(grad(I0) * splat) */
  aw_oracle_apply(I0, p1, p1 + n, p1 + 2 * n, si, nx, ny, nz, 0.0f);
  double e = 0.0;
  for (long k = 0; k < n; ++k) {
    si[k] = si[k] - I1[k];
    e += (double)si[k] * (double)si[k];
  }
  e *= spx * spy * spz;
  float *sp_img = (float *)malloc(sizeof(float) * (size_t)n);
  aw_oracle_splat(si, p1, p1 + n, p1 + 2 * n, sp_img, nx, ny, nz, 0.0f);
  aw_oracle_gradient(I0, g, g + n, g + 2 * n, nx, ny, nz, spx, spy, spz, 0);
  for (long k = 0; k < n; ++k) {
    g[k] *= sp_img[k];
    g[n + k] *= sp_img[k];
    g[2 * n + k] *= sp_img[k];
  }
  aw_oracle_fluid_apply(g, g + n, g + 2 * n, nx, ny, nz, spx, spy, spz, alpha, beta, gamma, 1);
  if (update_step) {
    const float a = 2.0f, b = -2.0f / (sigma * sigma);
    float mx = 0.f;
    for (long k = 0; k < n; ++k) {
      const float x = a * v0[k] + b * g[k];
      const float y = a * v0[n + k] + b * g[n + k];
      const float zz = a * v0[2 * n + k] + b * g[2 * n + k];
      const float len = (float)sqrt((double)(x * x + y * y + zz * zz));
      if (len > mx) mx = len;
    }
    *step = max_pert / mx;
  } else {
    const float vfac = (float)(1.0 - 2.0 * (double)*step);
    const float ufac = (2 * *step) / (sigma * sigma);
    for (long k = 0; k < 3 * n; ++k) v0[k] = vfac * v0[k] + ufac * g[k];
  }
  free(vt); free(lv0); free(dp); free(o); free(g); free(si); free(sp_img);
  return e;
}

/* ------------------------------------------------------------------------
 * Adjoint geodesic shooting: LDMMAdShootingIteratorCPU::Iterate
 * (Algorithms/LDMM/LDMMAdShootingIteratorCPU.cxx:237-323) and
 * backwardAdIntegration (:325-431).
 * ---------------------------------------------------------------------- */

/* HField3DUtils::divergence with wrap = false (UtilitiesDataTypes/
 * HField3DUtils.txx:2306-2349): d wx/dx + d wy/dy + d wz/dz, each partial
 * from computeGradient of one component, summed in float */
static void divergence(const float *w, float *out, float *g, int nx, int ny, int nz, double spx,
                       double spy, double spz) {
  const long n = (long)nx * ny * nz;
  float *t1 = g, *t2 = g + n, *t3 = g + 2 * n;
  float *scratch = (float *)malloc(sizeof(float) * (size_t)(2 * n));
  /* only the diagonal partials are used: the others land in scratch */
  aw_oracle_gradient(w, t1, scratch, scratch + n, nx, ny, nz, spx, spy, spz, 0);
  aw_oracle_gradient(w + n, scratch, t2, scratch + n, nx, ny, nz, spx, spy, spz, 0);
  aw_oracle_gradient(w + 2 * n, scratch, scratch + n, t3, nx, ny, nz, spx, spy, spz, 0);
  for (long k = 0; k < n; ++k) out[k] = t1[k] + t2[k] + t3[k];
  free(scratch);
}

/* Vector3D::dot in float, x first (HField3DUtils::pointwiseL2DotProd,
 * HField3DUtils.txx:204-221) */
static void dot3(const float *a, const float *b, float *out, long n) {
  for (long k = 0; k < n; ++k) out[k] = a[k] * b[k] + a[n + k] * b[n + k] + a[2 * n + k] * b[2 * n + k];
}

/* w (3 planes) *= s, component-wise (Array3D<Vector3D>::pointwiseMultiplyBy) */
static void scale3(float *w, const float *s, long n) {
  for (long k = 0; k < n; ++k) {
    w[k] *= s[k];
    w[n + k] *= s[k];
    w[2 * n + k] *= s[k];
  }
}

double aw_oracle_ldmm_adshoot_iterate(const float *I0, const float *I1, float *alpha0,
                                      float *phi0T, float *phiT0, float *V, int T, int nx, int ny,
                                      int nz, double spx, double spy, double spz, double alpha,
                                      double beta, double gamma, float sigma, float step,
                                      double *vec_energy) {
  const long n = (long)nx * ny * nz;
  const size_t f1 = sizeof(float) * (size_t)n, f3 = 3 * f1;
  float *o = (float *)malloc(f3), *w = (float *)malloc(f3), *w2 = (float *)malloc(f3);
  float *aT = (float *)malloc(f1), *I = (float *)malloc(f1), *IHat = (float *)malloc(f1);
  float *aHat = (float *)malloc(f1), *IT = (float *)malloc(f1), *aTil = (float *)malloc(f1);
  float *ITil = (float *)malloc(f1), *s1 = (float *)malloc(f1), *s2 = (float *)malloc(f1);
  float *p0 = phi0T, *p1 = phiT0;
#define AD_V(t) (V + (long)(t) * 3 * n)
  /* phi0T = composeVH(v, phi0T) [PARTIAL_ZERO]; phiT0 = composeHVInv(phiT0, v) [PARTIAL_ID] */
#define AD_ADVANCE_P0(v)                                                                       \
  do {                                                                                         \
    aw_oracle_compose_vh((v), (v) + n, (v) + 2 * n, p0, p0 + n, p0 + 2 * n, o, o + n, o + 2 * n, \
                         nx, ny, nz, spx, spy, spz, 1, AW_BG_PARTIAL_ZERO);                    \
    memcpy(p0, o, f3);                                                                         \
  } while (0)
#define AD_ADVANCE_P1(v)                                                                       \
  do {                                                                                         \
    aw_oracle_compose_hv(p1, p1 + n, p1 + 2 * n, (v), (v) + n, (v) + 2 * n, o, o + n, o + 2 * n, \
                         nx, ny, nz, spx, spy, spz, -1, AW_BG_PARTIAL_ID);                     \
    memcpy(p1, o, f3);                                                                         \
  } while (0)
  /* v_t = -K(grad(G) * alpha_t) */
#define AD_VELOCITY(G, t)                                                                      \
  do {                                                                                         \
    float *vt = AD_V(t);                                                                       \
    aw_oracle_gradient((G), vt, vt + n, vt + 2 * n, nx, ny, nz, spx, spy, spz, 0);             \
    scale3(vt, aT, n);                                                                         \
    aw_oracle_fluid_apply(vt, vt + n, vt + 2 * n, nx, ny, nz, spx, spy, spz, alpha, beta,      \
                          gamma, 1);                                                           \
    for (long k = 0; k < 3 * n; ++k) vt[k] = vt[k] * -1.0f;                                    \
  } while (0)

  /* part 1: shooting, every v_t kept (Iterate, .cxx:245-322) */
  aw_oracle_identity(p0, p0 + n, p0 + 2 * n, nx, ny, nz);
  aw_oracle_identity(p1, p1 + n, p1 + 2 * n, nx, ny, nz);
  memcpy(aT, alpha0, f1);
  AD_VELOCITY(I0, 0);
  for (int t = 1; t < T; ++t) {
    AD_ADVANCE_P0(AD_V(t - 1));
    aw_oracle_splat(alpha0, p0, p0 + n, p0 + 2 * n, aT, nx, ny, nz, 0.0f);
    AD_ADVANCE_P1(AD_V(t - 1));
    aw_oracle_apply(I0, p1, p1 + n, p1 + 2 * n, I, nx, ny, nz, 0.0f);
    AD_VELOCITY(I, t);
  }
  AD_ADVANCE_P1(AD_V(T - 1));
  AD_ADVANCE_P0(AD_V(T - 1));
  /* <L v0, v0> (.cxx:305-311) */
  if (vec_energy) *vec_energy = l_energy(AD_V(0), w, nx, ny, nz, spx, spy, spz, alpha, beta, gamma);
  aw_oracle_apply(I0, p1, p1 + n, p1 + 2 * n, I, nx, ny, nz, 0.0f);
  double e = 0.0;
  for (long k = 0; k < n; ++k) {
    const float r = I[k] - I1[k];
    e += (double)r * (double)r;
  }
  e *= spx * spy * spz;

  /* part 2: backward integration of the adjoint equations
   * (backwardAdIntegration, .cxx:325-431) */
  memset(aTil, 0, f1);
  {
    const float inv = 1.0f / (sigma * sigma);
    for (long k = 0; k < n; ++k) IHat[k] = (I1[k] - I[k]) * inv;
  }
  aw_oracle_splat(IHat, p1, p1 + n, p1 + 2 * n, ITil, nx, ny, nz, 0.0f);
  for (int i = T - 1; i >= 0; --i) {
    if (i != T - 1) {
      aw_oracle_identity(p0, p0 + n, p0 + 2 * n, nx, ny, nz);
      aw_oracle_identity(p1, p1 + n, p1 + 2 * n, nx, ny, nz);
      for (int j = 1; j <= i + 1; ++j) {
        AD_ADVANCE_P0(AD_V(j - 1));
        AD_ADVANCE_P1(AD_V(j - 1));
      }
    }
    aw_oracle_apply(I0, p1, p1 + n, p1 + 2 * n, IT, nx, ny, nz, 0.0f);
    aw_oracle_splat(alpha0, p0, p0 + n, p0 + 2 * n, aT, nx, ny, nz, 0.0f);
    aw_oracle_apply(aTil, p1, p1 + n, p1 + 2 * n, aHat, nx, ny, nz, 0.0f);
    aw_oracle_splat(ITil, p0, p0 + n, p0 + 2 * n, IHat, nx, ny, nz, 0.0f);
    /* vhat = K(grad(aHat) * aT - grad(IT) * IHat) */
    aw_oracle_gradient(aHat, w, w + n, w + 2 * n, nx, ny, nz, spx, spy, spz, 0);
    aw_oracle_gradient(IT, w2, w2 + n, w2 + 2 * n, nx, ny, nz, spx, spy, spz, 0);
    scale3(w, aT, n);
    scale3(w2, IHat, n);
    for (long k = 0; k < 3 * n; ++k) w[k] = w[k] - w2[k];
    aw_oracle_fluid_apply(w, w + n, w + 2 * n, nx, ny, nz, spx, spy, spz, alpha, beta, gamma, 1);
    /* aTilde -= (grad(IT) . vhat)(phi0T) */
    aw_oracle_gradient(IT, w2, w2 + n, w2 + 2 * n, nx, ny, nz, spx, spy, spz, 0);
    dot3(w2, w, s1, n);
    aw_oracle_apply(s1, p0, p0 + n, p0 + 2 * n, s2, nx, ny, nz, 0.0f);
    for (long k = 0; k < n; ++k) aTil[k] = aTil[k] - s2[k];
    /* ITilde += splat(div(aT vhat), phiT0) */
    scale3(w, aT, n);
    divergence(w, s1, w2, nx, ny, nz, spx, spy, spz);
    aw_oracle_splat(s1, p1, p1 + n, p1 + 2 * n, s2, nx, ny, nz, 0.0f);
    for (long k = 0; k < n; ++k) ITil[k] = ITil[k] + s2[k];
  }
  /* alpha0 -= step * (-(grad(I0) . v0) - aTilde) */
  aw_oracle_gradient(I0, w, w + n, w + 2 * n, nx, ny, nz, spx, spy, spz, 0);
  dot3(w, AD_V(0), s1, n);
  for (long k = 0; k < n; ++k) {
    float g = s1[k] * -1.0f;
    g = g - aTil[k];
    g = g * step;
    alpha0[k] = alpha0[k] - g;
  }
#undef AD_V
#undef AD_ADVANCE_P0
#undef AD_ADVANCE_P1
#undef AD_VELOCITY
  free(o);
  free(w);
  free(w2);
  free(aT);
  free(I);
  free(IHat);
  free(aHat);
  free(IT);
  free(aTil);
  free(ITil);
  free(s1);
  free(s2);
  return e;
}

/* ImageUtils::resampleNew (UtilitiesDataTypes/ImageUtils.txx:306-349) with
 * the default BACKGROUND_STRATEGY_CLAMP / linear interpolation
 * (Array3DUtils::trilerp, Array3DUtils.txx:63-210), origin 0: destination
 * voxel x samples the source at ((x*dsp + (dsp - ssp)/2) / ssp). The
 * reference keeps a floor equal to the size (a position at or beyond the
 * last cell plus one); such a corner is clamped here as well — the
 * multiscale upsampling never reaches it. */
static float trilerp_clamp(const float *a, int nx, int ny, int nz, double x, double y, double z) {
  int fx = (int)x, fy = (int)y, fz = (int)z;
  if (x < 0 && x != (int)x) --fx;
  if (y < 0 && y != (int)y) --fy;
  if (z < 0 && z != (int)z) --fz;
  int cx = fx + 1, cy = fy + 1, cz = fz + 1;
  const double t = x - fx, u = y - fy, v = z - fz;
  const double omt = 1.0 - t, omu = 1.0 - u, omv = 1.0 - v;
#define AD_CLAMP(f, c, s)           \
  do {                              \
    if (f < 0) {                    \
      f = 0;                        \
      if (c < 0) c = 0;             \
    }                               \
    if (c >= s) {                   \
      c = s - 1;                    \
      if (f > s - 1) f = s - 1;     \
    }                               \
  } while (0)
  AD_CLAMP(fx, cx, nx);
  AD_CLAMP(fy, cy, ny);
  AD_CLAMP(fz, cz, nz);
#undef AD_CLAMP
  const float v0 = a[IDX(fx, fy, fz)], v1 = a[IDX(cx, fy, fz)], v2 = a[IDX(cx, cy, fz)],
              v3 = a[IDX(fx, cy, fz)], v4 = a[IDX(fx, cy, cz)], v5 = a[IDX(cx, cy, cz)],
              v6 = a[IDX(cx, fy, cz)], v7 = a[IDX(fx, fy, cz)];
  return (float)(omt * (omu * (v0 * omv + v7 * v) + u * (v3 * omv + v4 * v)) +
                 t * (omu * (v1 * omv + v6 * v) + u * (v2 * omv + v5 * v)));
}

void aw_oracle_resample_image(const float *in, int nx, int ny, int nz, double ssx, double ssy,
                              double ssz, float *out, int mx, int my, int mz, double dsx,
                              double dsy, double dsz) {
  const double ox = (dsx - ssx) / 2.0, oy = (dsy - ssy) / 2.0, oz = (dsz - ssz) / 2.0;
  for (int z = 0; z < mz; ++z)
    for (int y = 0; y < my; ++y)
      for (int x = 0; x < mx; ++x) {
        const double wx = dsx * x + 0.0 + ox, wy = dsy * y + 0.0 + oy, wz = dsz * z + 0.0 + oz;
        out[((long)z * my + y) * mx + x] =
            trilerp_clamp(in, nx, ny, nz, (wx - 0.0) / ssx, (wy - 0.0) / ssy, (wz - 0.0) / ssz);
      }
}

/* ------------------------------------------------------------------------
 * Multiscale (Algorithms/Common/MultiscaleManager.cxx:301-366).
 * ---------------------------------------------------------------------- */

/* GaussianFilter3D::filter_generate_gauss_full
 * (Utilities/DownsampleFilter/GaussianFilter3D.cxx): row 0 is the
 * normalised half filter, row j the filter renormalised for an element j
 * voxels from the border. float arithmetic as written there. */
static void gauss_filter_rows(float sigma, int size, float *rows /* (size+1)^2 */) {
  float *f0 = rows;
  const float exp_scale = (float)(1.0 / (2.0 * sigma * sigma));
  float scale = f0[0] = 1.0f;
  for (int i = 1; i <= size; ++i) {
    f0[i] = expf(-(float)(i * i) * exp_scale);
    scale = (float)(scale + 2.0 * f0[i]);
  }
  scale = (float)(1.0 / scale);
  for (int i = 0; i <= size; ++i) f0[i] *= scale;
  scale = 0.0f;
  for (int j = 1; j <= size; ++j) {
    scale += f0[size + 1 - j];
    for (int i = 0; i <= size; ++i) rows[j * (size + 1) + i] = (float)(f0[i] / (1. - scale));
  }
}

/* one axis of GaussianFilter3D::filter_symmetric_full: n samples spaced
 * `stride` apart, K the half kernel size */
static void gauss_line(const float *in, float *out, int n, long stride, int K, const float *rows) {
  const float *f = rows;
  for (int x = K; x < n - K; ++x) {
    float o = in[x * stride] * f[0];
    for (int i = 1; i <= K; ++i) o += (in[(x - i) * stride] + in[(x + i) * stride]) * f[i];
    out[x * stride] = o;
  }
  for (int x = K - 1; x >= 0; --x) {
    f = rows + (K - x) * (K + 1);
    float o = in[x * stride] * f[0];
    for (int i = 1; i <= x; ++i) o += (in[(x - i) * stride] + in[(x + i) * stride]) * f[i];
    for (int i = x + 1; i <= K; ++i) o += in[(x + i) * stride] * f[i];
    out[x * stride] = o;
    const int r = n - 1 - x;
    o = in[r * stride] * f[0];
    for (int i = 1; i <= x; ++i) o += (in[(r + i) * stride] + in[(r - i) * stride]) * f[i];
    for (int i = x + 1; i <= K; ++i) o += in[(r - i) * stride] * f[i];
    out[r * stride] = o;
  }
}

/* Separable Gaussian blur, x then y then z; kernel half sizes clamped to
 * n/2 - 1 as filter_symmetric_full does. */
void aw_oracle_gauss_blur(const float *in, float *out, int nx, int ny, int nz, float sx, float sy,
                          float sz, int kx, int ky, int kz) {
  const long n = (long)nx * ny * nz;
  int K[3] = {kx, ky, kz};
  const int N[3] = {nx, ny, nz};
  for (int a = 0; a < 3; ++a)
    if (K[a] > N[a] / 2 - 1) K[a] = N[a] / 2 - 1;
  float *b1 = (float *)calloc((size_t)n, sizeof(float));
  float *b2 = (float *)calloc((size_t)n, sizeof(float));
  float *rows;
  rows = (float *)malloc(sizeof(float) * (size_t)((K[0] + 1) * (K[0] + 1)));
  gauss_filter_rows(sx, K[0], rows);
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y) gauss_line(in + IDX(0, y, z), b1 + IDX(0, y, z), nx, 1, K[0], rows);
  free(rows);
  rows = (float *)malloc(sizeof(float) * (size_t)((K[1] + 1) * (K[1] + 1)));
  gauss_filter_rows(sy, K[1], rows);
  for (int z = 0; z < nz; ++z)
    for (int x = 0; x < nx; ++x) gauss_line(b1 + IDX(x, 0, z), b2 + IDX(x, 0, z), ny, nx, K[1], rows);
  free(rows);
  rows = (float *)malloc(sizeof(float) * (size_t)((K[2] + 1) * (K[2] + 1)));
  gauss_filter_rows(sz, K[2], rows);
  for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x)
      gauss_line(b2 + IDX(x, y, 0), out + IDX(x, y, 0), nz, (long)nx * ny, K[2], rows);
  free(rows);
  free(b1);
  free(b2);
}

/* ImageUtils::gaussianDownsample + resampleNew (UtilitiesDataTypes/
 * ImageUtils.txx:259-349): sigma = sqrt(factor/2), half kernel 2*ceil(sigma),
 * then a trilinear sample of the blurred image at the centres of the
 * coarse voxels, background 0. Spacing of the input is (spx, spy, spz). */
void aw_oracle_downsample(const float *in, int nx, int ny, int nz, double spx, double spy,
                          double spz, float *out, int mx, int my, int mz) {
  const double fx = (double)nx / mx, fy = (double)ny / my, fz = (double)nz / mz;
  const double sgx = sqrt(fx / 2.0), sgy = sqrt(fy / 2.0), sgz = sqrt(fz / 2.0);
  const int kx = 2 * (int)ceil(sgx), ky = 2 * (int)ceil(sgy), kz = 2 * (int)ceil(sgz);
  const long n = (long)nx * ny * nz;
  float *blur = (float *)malloc(sizeof(float) * (size_t)n);
  aw_oracle_gauss_blur(in, blur, nx, ny, nz, (float)sgx, (float)sgy, (float)sgz, kx, ky, kz);
  const double dsx = spx * fx, dsy = spy * fy, dsz = spz * fz;
  const double ox = (dsx - spx) / 2.0, oy = (dsy - spy) / 2.0, oz = (dsz - spz) / 2.0;
  for (int z = 0; z < mz; ++z)
    for (int y = 0; y < my; ++y)
      for (int x = 0; x < mx; ++x) {
        const double wx = dsx * x + 0.0 + ox, wy = dsy * y + 0.0 + oy, wz = dsz * z + 0.0 + oz;
        const double vx = (wx - 0.0) / spx, vy = (wy - 0.0) / spy, vz = (wz - 0.0) / spz;
        out[((long)z * my + y) * mx + x] = trilerp_val(blur, nx, ny, nz, vx, vy, vz, 0.0f);
      }
  free(blur);
}

/* Upsampling a deformation to the next scale level, as
 * GreedyDeformationData::SetScaleLevel does it (Greedy/GreedyDeformationData.cxx:
 * 211-221): hToVelocity, HField3DUtils::resampleNew with CLAMP and the
 * vectors rescaled by out/in size (HField3DUtils.txx:1816-1881), velocityToH. */
void aw_oracle_upsample_hfield(const float *h, int nx, int ny, int nz, float *out, int mx, int my,
                               int mz, int rescale) {
  const long n = (long)nx * ny * nz, m = (long)mx * my * mz;
  float *v = (float *)malloc(sizeof(float) * (size_t)(3 * n));
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const long i = IDX(x, y, z);
        v[i] = (float)((double)(h[i] - (float)x) * 1.0);
        v[n + i] = (float)((double)(h[n + i] - (float)y) * 1.0);
        v[2 * n + i] = (float)((double)(h[2 * n + i] - (float)z) * 1.0);
      }
  const double rX = (double)nx / mx, rY = (double)ny / my, rZ = (double)nz / mz;
  const double oX = (rX - 1.0) / 2.0, oY = (rY - 1.0) / 2.0, oZ = (rZ - 1.0) / 2.0;
  const float s[3] = {(float)(1.0 / rX), (float)(1.0 / rY), (float)(1.0 / rZ)};
  for (int z = 0; z < mz; ++z) {
    const double iz = oZ + z * rZ;
    for (int y = 0; y < my; ++y) {
      const double iy = oY + y * rY;
      for (int x = 0; x < mx; ++x) {
        const double ix = oX + x * rX;
        const long o = ((long)z * my + y) * mx + x;
        float a, b, c;
        trilerp_vec(v, v + n, v + 2 * n, nx, ny, nz, (float)ix, (float)iy, (float)iz, &a, &b, &c,
                    AW_BG_CLAMP);
        if (rescale) {
          a *= s[0];
          b *= s[1];
          c *= s[2];
        }
        out[o] = (float)(x + a / 1.0);
        out[m + o] = (float)(y + b / 1.0);
        out[2 * m + o] = (float)(z + c / 1.0);
      }
    }
  }
  free(v);
}

/* MedianCalculator::Select(std::vector<RealImage*>, k, rtn)
 * (Algorithms/Common/MedianCalculator.cxx:264-389) with MinMax (:170-199) and
 * GetIndex (:201-258), one process: all voxels advance round by round, as in
 * the reference. */
int aw_oracle_voxel_median(const float *imgs, int n, long nvox, int k, float *out) {
  if (n <= 0 || nvox <= 0 || k < 0 || k >= n) return 2;
  float *gmin = malloc(sizeof(float) * nvox), *gmax = malloc(sizeof(float) * nvox);
  float *cmin = malloc(sizeof(float) * nvox), *cmax = malloc(sizeof(float) * nvox);
  float *p = malloc(sizeof(float) * nvox), *vp = malloc(sizeof(float) * nvox);
  float *vn = malloc(sizeof(float) * nvox);
  unsigned *idx = malloc(sizeof(unsigned) * nvox);
  char *fin = calloc((size_t)nvox, 1);
  int rc = 0;
  /* MinMax: per-voxel min / max starting from image 0 */
  for (long i = 0; i < nvox; ++i) gmin[i] = gmax[i] = imgs[i];
  for (int m = 1; m < n; ++m)
    for (long i = 0; i < nvox; ++i) {
      const float v = imgs[(long)m * nvox + i];
      gmin[i] = v < gmin[i] ? v : gmin[i];
      gmax[i] = v > gmax[i] ? v : gmax[i];
    }
  /* Array3DUtils::getMinMax of gmin (its min) and of gmax (its max) */
  float tmin = gmin[0], tmax = gmax[0];
  for (long i = 1; i < nvox; ++i) {
    if (gmin[i] < tmin) tmin = gmin[i];
    if (gmax[i] > tmax) tmax = gmax[i];
  }
  const float eps = (tmax - tmin) / 10000.f;
  for (long i = 0; i < nvox; ++i) {
    cmin[i] = gmin[i];
    cmax[i] = gmax[i];
  }
  long finished = 0;
  const unsigned uk = (unsigned)k;
  for (unsigned iter = 0;; ++iter) {
    for (long i = 0; i < nvox; ++i) {
      if (fin[i]) continue;
      if (eps > fabsf(cmax[i] - cmin[i])) {
        out[i] = cmin[i];
        fin[i] = 1;
        ++finished;
        continue;
      }
      p[i] = (float)((double)(cmin[i] + cmax[i]) / 2.0);
    }
    /* GetIndex: count below p, largest below (from gmin), smallest at or above (from gmax) */
    for (long i = 0; i < nvox; ++i) {
      vp[i] = gmin[i];
      vn[i] = gmax[i];
      idx[i] = 0;
    }
    for (int m = 0; m < n; ++m)
      for (long i = 0; i < nvox; ++i) {
        const float v = imgs[(long)m * nvox + i];
        if (v < p[i]) {
          idx[i]++;
          if (v > vp[i]) vp[i] = v;
        } else if (v < vn[i]) {
          vn[i] = v;
        }
      }
    for (long i = 0; i < nvox; ++i) {
      if (fin[i]) continue;
      if (idx[i] == uk) {
        out[i] = vn[i];
        fin[i] = 1;
        ++finished;
      } else if (idx[i] - 1u == uk) {
        out[i] = vp[i];
        fin[i] = 1;
        ++finished;
      } else if (idx[i] > uk) {
        cmax[i] = vp[i];
      } else if (idx[i] < uk) {
        cmin[i] = vn[i];
      }
    }
    if (iter > (unsigned)n && finished < nvox) {
      rc = 1;
      for (long i = 0; i < nvox; ++i)
        if (!fin[i]) out[i] = cmin[i];
      break;
    }
    if (finished == nvox) break;
  }
  free(gmin); free(gmax); free(cmin); free(cmax); free(p); free(vp); free(vn); free(idx); free(fin);
  return rc;
}
