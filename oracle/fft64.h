/*
 * fft64 — double-precision mixed-radix complex FFT used only by the test
 * oracle (oracle/aw_oracle.c) and by the FFTW-API shim that lets the
 * reference CPU path link without FFTW (oracle/ref/fftw_shim.cxx).
 *
 * TEST INFRASTRUCTURE: nothing in the product (atlaswerks_b200/) links this.
 *
 * Transform convention matches FFTW: forward sign = -1, backward sign = +1,
 * both unnormalised.
 */
#ifndef AW_ORACLE_FFT64_H
#define AW_ORACLE_FFT64_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double re, im; } fft64_cplx;

/* In-place 1D transform of n elements spaced `stride` apart. */
void fft64_1d(fft64_cplx *data, int n, long stride, int sign);

/* In-place 3D transform of a dense array laid out [nz][ny][nx] (x fastest). */
void fft64_3d(fft64_cplx *data, int nx, int ny, int nz, int sign);

#ifdef __cplusplus
}
#endif
#endif
