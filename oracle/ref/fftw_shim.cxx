/*
 * fftw_shim.cxx — the subset of the FFTW3 API that the reference CPU path
 * calls, implemented on the project's FP64 FFT (oracle/fft64.c).
 *
 * TEST INFRASTRUCTURE: linked only into oracle/_ref/libawref.so, the
 * reference's own CPU code built from its sources so that the oracle can be
 * checked against it. FFTW is not installed in this image.
 *
 * Supported exactly as DiffOperFFTWWrapper uses it
 * (Algorithms/Common/DiffOper.cxx:30-77): rank-3 r2c/c2r, NULL embeds
 * (in-place => real rows padded to 2*(nx/2+1), per the FFTW manual),
 * arbitrary howmany/stride/dist. The transform runs in double and is
 * rounded to the plan's precision when written back, so this shim is more
 * accurate than FFTW's single-precision plans. Every other entry point
 * aborts: they are not on the greedy/LDMM path.
 */
#include <fftw3.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../fft64.h"

namespace {

struct ShimPlan {
  bool r2c;
  bool dbl;
  int n[3];  // z, y, x as passed
  int howmany;
  void *in;
  void *out;
  int istride, idist, ostride, odist;
  bool inplace;
};

template <class T>
void exec(const ShimPlan &p) {
  const int nz = p.n[0], ny = p.n[1], nx = p.n[2];
  const int nxh = nx / 2 + 1;
  const long ntot = (long)nx * ny * nz;
  // row length of the real array in T units: padded when in-place
  const int rx = p.inplace ? 2 * nxh : nx;
  // In-place interleaved transforms overlap across the howmany
  // components, so every component is read before any is written.
  std::vector<std::vector<fft64_cplx> > bufs(p.howmany, std::vector<fft64_cplx>(ntot));
  const T *in = (const T *)p.in;
  for (int h = 0; h < p.howmany; ++h) {
    std::vector<fft64_cplx> &buf = bufs[h];
    if (p.r2c) {
      for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
          for (int x = 0; x < nx; ++x) {
            long ri = ((long)(z * ny + y) * rx + x) * p.istride + (long)h * p.idist;
            fft64_cplx &c = buf[((long)z * ny + y) * nx + x];
            c.re = (double)in[ri];
            c.im = 0.0;
          }
    } else {
      for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
          for (int kx = 0; kx < nxh; ++kx) {
            long ci = (((long)(z * ny + y) * nxh + kx) * p.istride + (long)h * p.idist) * 2;
            fft64_cplx &c = buf[((long)z * ny + y) * nx + kx];
            c.re = (double)in[ci];
            c.im = (double)in[ci + 1];
          }
    }
  }
  for (int h = 0; h < p.howmany; ++h) {
    std::vector<fft64_cplx> &buf = bufs[h];
    T *out = (T *)p.out;
    if (p.r2c) {
      fft64_3d(buf.data(), nx, ny, nz, -1);
      for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
          for (int kx = 0; kx < nxh; ++kx) {
            long ci = (((long)(z * ny + y) * nxh + kx) * p.ostride + (long)h * p.odist) * 2;
            const fft64_cplx &c = buf[((long)z * ny + y) * nx + kx];
            out[ci] = (T)c.re;
            out[ci + 1] = (T)c.im;
          }
    } else {
      // Hermitian completion of the non-redundant half
      for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
          for (int kx = nxh; kx < nx; ++kx) {
            const int mz = (nz - z) % nz, my = (ny - y) % ny, mx = nx - kx;
            const fft64_cplx &s = buf[((long)mz * ny + my) * nx + mx];
            fft64_cplx &c = buf[((long)z * ny + y) * nx + kx];
            c.re = s.re;
            c.im = -s.im;
          }
      fft64_3d(buf.data(), nx, ny, nz, +1);
      for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
          for (int x = 0; x < nx; ++x) {
            long ri = ((long)(z * ny + y) * rx + x) * p.ostride + (long)h * p.odist;
            out[ri] = (T)buf[((long)z * ny + y) * nx + x].re;
          }
    }
  }
}

ShimPlan *make(bool r2c, bool dbl, int rank, const int *n, int howmany, void *in,
               const int *inembed, int istride, int idist, void *out, const int *onembed,
               int ostride, int odist) {
  if (rank != 3 || inembed || onembed) {
    std::fprintf(stderr, "fftw shim: only rank-3 transforms with NULL embeds are supported\n");
    std::abort();
  }
  ShimPlan *p = new ShimPlan;
  p->r2c = r2c;
  p->dbl = dbl;
  for (int i = 0; i < 3; ++i) p->n[i] = n[i];
  p->howmany = howmany;
  p->in = in;
  p->out = out;
  p->istride = istride;
  p->idist = idist;
  p->ostride = ostride;
  p->odist = odist;
  p->inplace = (in == out);
  return p;
}

[[noreturn]] void unsupported(const char *what) {
  std::fprintf(stderr, "fftw shim: %s is not on the registration path\n", what);
  std::abort();
}

}  // namespace

extern "C" {

fftwf_plan fftwf_plan_many_dft_r2c(int rank, const int *n, int howmany, float *in,
                                   const int *inembed, int istride, int idist, fftwf_complex *out,
                                   const int *onembed, int ostride, int odist, unsigned) {
  return (fftwf_plan)make(true, false, rank, n, howmany, in, inembed, istride, idist, out,
                          onembed, ostride, odist);
}
fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int *n, int howmany, fftwf_complex *in,
                                   const int *inembed, int istride, int idist, float *out,
                                   const int *onembed, int ostride, int odist, unsigned) {
  return (fftwf_plan)make(false, false, rank, n, howmany, in, inembed, istride, idist, out,
                          onembed, ostride, odist);
}
void fftwf_execute(const fftwf_plan p) {
  const ShimPlan *s = (const ShimPlan *)p;
  if (s->dbl) unsupported("mixed precision plan");
  exec<float>(*s);
}
void fftwf_destroy_plan(fftwf_plan p) { delete (ShimPlan *)p; }
void fftwf_plan_with_nthreads(int) {}
fftwf_plan fftwf_plan_many_dft(int, const int *, int, fftwf_complex *, const int *, int, int,
                               fftwf_complex *, const int *, int, int, int, unsigned) {
  unsupported("fftwf_plan_many_dft");
}
fftwf_plan fftwf_plan_dft(int, const int *, fftwf_complex *, fftwf_complex *, int, unsigned) {
  unsupported("fftwf_plan_dft");
}

fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany, double *in,
                                 const int *inembed, int istride, int idist, fftw_complex *out,
                                 const int *onembed, int ostride, int odist, unsigned) {
  return (fftw_plan)make(true, true, rank, n, howmany, in, inembed, istride, idist, out, onembed,
                         ostride, odist);
}
fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany, fftw_complex *in,
                                 const int *inembed, int istride, int idist, double *out,
                                 const int *onembed, int ostride, int odist, unsigned) {
  return (fftw_plan)make(false, true, rank, n, howmany, in, inembed, istride, idist, out, onembed,
                         ostride, odist);
}
void fftw_execute(const fftw_plan p) {
  const ShimPlan *s = (const ShimPlan *)p;
  if (!s->dbl) unsupported("mixed precision plan");
  exec<double>(*s);
}
void fftw_destroy_plan(fftw_plan p) { delete (ShimPlan *)p; }
void fftw_plan_with_nthreads(int) {}

}  // extern "C"
