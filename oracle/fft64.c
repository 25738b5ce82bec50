/*
 * fft64.c — recursive mixed-radix decimation-in-time DFT in double precision.
 *
 * TEST INFRASTRUCTURE ONLY (see fft64.h). Any length n >= 1 is supported:
 * n is split by its smallest prime factor p; prime lengths fall through to
 * an O(p^2) direct DFT. Twiddles come from one table of exact cos/sin of
 * 2*pi*j/N in double. The FFTW float plans used by the reference
 * (Common/DiffOper.cxx:30-77) are replaced by this FP64 transform, rounded
 * to float at the shim boundary.
 */
#include "fft64.h"

#include <math.h>
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#include <stdlib.h>
#include <string.h>

static int smallest_factor(int n) {
  if (n % 4 == 0 && n > 4) return 4;
  for (int p = 2; (long)p * p <= n; ++p)
    if (n % p == 0) return p;
  return n;
}

/* out[k] = sum_j in[j*istride] * W_n^(j*k), W_n = tw[(N/n) * 1]. */
static void dft_rec(const fft64_cplx *in, long istride, fft64_cplx *out, int n,
                    const fft64_cplx *tw, long twscale, fft64_cplx *scratch) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  const int p = smallest_factor(n);
  const int m = n / p;
  if (m == 1) {
    for (int k = 0; k < n; ++k) {
      double sr = 0.0, si = 0.0;
      for (int j = 0; j < n; ++j) {
        const fft64_cplx w = tw[(((long)j * k) % n) * twscale];
        const fft64_cplx v = in[j * istride];
        sr += v.re * w.re - v.im * w.im;
        si += v.re * w.im + v.im * w.re;
      }
      out[k].re = sr;
      out[k].im = si;
    }
    return;
  }
  for (int q = 0; q < p; ++q)
    dft_rec(in + q * istride, istride * p, out + q * m, m, tw, twscale * p, scratch + n);
  fft64_cplx *t = scratch;
  for (int k = 0; k < m; ++k) {
    for (int q = 0; q < p; ++q) {
      const fft64_cplx y = out[q * m + k];
      const fft64_cplx w = tw[(((long)q * k) % n) * twscale];
      t[q].re = y.re * w.re - y.im * w.im;
      t[q].im = y.re * w.im + y.im * w.re;
    }
    for (int u = 0; u < p; ++u) {
      double sr = 0.0, si = 0.0;
      for (int q = 0; q < p; ++q) {
        const fft64_cplx w = tw[((((long)q * u) % p) * m) * twscale];
        sr += t[q].re * w.re - t[q].im * w.im;
        si += t[q].re * w.im + t[q].im * w.re;
      }
      t[p + u].re = sr;
      t[p + u].im = si;
    }
    for (int u = 0; u < p; ++u) out[k + u * m] = t[p + u];
  }
}

typedef struct {
  int n, sign;
  fft64_cplx *tw, *in, *out, *scratch;
} line_plan;

static void plan_init(line_plan *pl, int n, int sign) {
  pl->n = n;
  pl->sign = sign;
  pl->tw = (fft64_cplx *)malloc(sizeof(fft64_cplx) * (size_t)n);
  pl->in = (fft64_cplx *)malloc(sizeof(fft64_cplx) * (size_t)n);
  pl->out = (fft64_cplx *)malloc(sizeof(fft64_cplx) * (size_t)n);
  pl->scratch = (fft64_cplx *)malloc(sizeof(fft64_cplx) * (size_t)(6 * n + 8));
  for (int j = 0; j < n; ++j) {
    const double a = sign * 2.0 * M_PI * (double)j / (double)n;
    pl->tw[j].re = cos(a);
    pl->tw[j].im = sin(a);
  }
}

static void plan_free(line_plan *pl) {
  free(pl->tw);
  free(pl->in);
  free(pl->out);
  free(pl->scratch);
}

static void plan_exec(line_plan *pl, fft64_cplx *data, long stride) {
  const int n = pl->n;
  for (int i = 0; i < n; ++i) pl->in[i] = data[i * stride];
  dft_rec(pl->in, 1, pl->out, n, pl->tw, 1, pl->scratch);
  for (int i = 0; i < n; ++i) data[i * stride] = pl->out[i];
}

void fft64_1d(fft64_cplx *data, int n, long stride, int sign) {
  if (n <= 1) return;
  line_plan pl;
  plan_init(&pl, n, sign);
  plan_exec(&pl, data, stride);
  plan_free(&pl);
}

void fft64_3d(fft64_cplx *data, int nx, int ny, int nz, int sign) {
  const long sxy = (long)nx * ny;
  line_plan pl;
  if (nx > 1) {
    plan_init(&pl, nx, sign);
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y) plan_exec(&pl, data + z * sxy + (long)y * nx, 1);
    plan_free(&pl);
  }
  if (ny > 1) {
    plan_init(&pl, ny, sign);
    for (int z = 0; z < nz; ++z)
      for (int x = 0; x < nx; ++x) plan_exec(&pl, data + z * sxy + x, nx);
    plan_free(&pl);
  }
  if (nz > 1) {
    plan_init(&pl, nz, sign);
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) plan_exec(&pl, data + (long)y * nx + x, nz == 1 ? 1 : sxy);
    plan_free(&pl);
  }
}
