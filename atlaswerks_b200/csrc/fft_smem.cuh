// fft_smem.cuh — batched mixed-radix complex FFTs on lines held in shared
// memory, the building block of the fused fluid-operator kernels.
//
// Each stage is a self-sorting (Stockham) decimation-in-time pass that
// reads one shared-memory buffer and writes the other; radices 2, 4, 8 and 3
// have hand-written butterflies, any other prime factor goes through a
// direct DFT with table twiddles. Twiddles W_n^m = exp(-2*pi*i*m/n) are
// computed on the host in double and rounded to float once. Forward is
// sign -1, inverse +1; both unnormalised, as FFTW/cuFFT.
#pragma once

#include "aw_common.cuh"

namespace aw {

constexpr int kMaxStages = 12;

struct FFTAxis {
  int n;
  int nstages;
  int radix[kMaxStages];
  const float2 *tw;  // n entries, W_n^m (forward sign)
};

AW_D float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
AW_D float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
AW_D float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// multiply by sign*i
template <int SIGN>
AW_D float2 mul_si(float2 a) {
  return SIGN < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}

template <int SIGN>
AW_D float2 twiddle(const float2 *__restrict__ tw, int m) {
  const float2 w = __ldg(tw + m);
  return SIGN < 0 ? w : make_float2(w.x, -w.y);
}

template <int SIGN>
AW_D void bfly2(float2 *v) {
  const float2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <int SIGN>
AW_D void bfly4(float2 *v) {
  const float2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
  const float2 s13 = cadd(v[1], v[3]), d13 = mul_si<SIGN>(csub(v[1], v[3]));
  v[0] = cadd(s02, s13);
  v[2] = csub(s02, s13);
  v[1] = cadd(d02, d13);
  v[3] = csub(d02, d13);
}

template <int SIGN>
AW_D void bfly8(float2 *v) {
  float2 e[4] = {v[0], v[2], v[4], v[6]};
  float2 o[4] = {v[1], v[3], v[5], v[7]};
  bfly4<SIGN>(e);
  bfly4<SIGN>(o);
  const float r = 0.70710678118654752440f;
  // W8^u for u = 1, 2, 3 with the transform's sign
  const float2 w1 = make_float2(r, SIGN * r);
  const float2 w3 = make_float2(-r, SIGN * r);
  o[1] = cmul(o[1], w1);
  o[2] = mul_si<SIGN>(o[2]);
  o[3] = cmul(o[3], w3);
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    v[u] = cadd(e[u], o[u]);
    v[u + 4] = csub(e[u], o[u]);
  }
}

template <int SIGN>
AW_D void bfly3(float2 *v) {
  const float s = SIGN * 0.86602540378443864676f;  // sign * sin(2*pi/3)
  const float2 t1 = cadd(v[1], v[2]);
  const float2 t2 = csub(v[1], v[2]);
  const float2 m = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
  const float2 j = make_float2(-s * t2.y, s * t2.x);  // i*s*t2
  v[0] = cadd(v[0], t1);
  v[1] = cadd(m, j);
  v[2] = csub(m, j);
}

// One Stockham stage of radix R (compile-time) over `batch` lines.
template <int SIGN, int R>
AW_D void stage_fixed(const float2 *__restrict__ src, float2 *__restrict__ dst, int batch, int ld,
                      int n, int Ns, const float2 *__restrict__ tw) {
  const int nb = n / R;
  const int total = batch * nb;
  const int tws = n / (Ns * R);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int line = t / nb;
    const int j = t - line * nb;
    const int k = j % Ns;
    const float2 *sl = src + line * ld;
    float2 *dl = dst + line * ld;
    float2 v[R];
    v[0] = sl[j];
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = cmul(sl[j + r * nb], twiddle<SIGN>(tw, r * k * tws));
    if (R == 2) bfly2<SIGN>(v);
    if (R == 3) bfly3<SIGN>(v);
    if (R == 4) bfly4<SIGN>(v);
    if (R == 8) bfly8<SIGN>(v);
    const int base = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dl[base + r * Ns] = v[r];
  }
}

// Generic prime radix: direct DFT, twiddles from the length-n table.
template <int SIGN>
AW_D void stage_generic(const float2 *__restrict__ src, float2 *__restrict__ dst, int batch, int ld,
                        int n, int Ns, int R, const float2 *__restrict__ tw) {
  const int nb = n / R;
  const int total = batch * nb;
  const int tws = n / (Ns * R);
  const int step = n / R;  // W_R^1 = W_n^(n/R)
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int line = t / nb;
    const int j = t - line * nb;
    const int k = j % Ns;
    const float2 *sl = src + line * ld;
    float2 *dl = dst + line * ld;
    const int base = (j / Ns) * Ns * R + k;
    for (int u = 0; u < R; ++u) {
      float2 acc = sl[j];
      for (int q = 1; q < R; ++q) {
        const float2 a = cmul(sl[j + q * nb], twiddle<SIGN>(tw, q * k * tws));
        acc = cadd(acc, cmul(a, twiddle<SIGN>(tw, ((q * u) % R) * step)));
      }
      dl[base + u * Ns] = acc;
    }
  }
}

// Runs all stages over `batch` lines (line b at offset b*ld) starting in
// buffer a; returns the buffer that holds the result. Ends with a barrier.
template <int SIGN>
__device__ float2 *fft_lines(float2 *a, float2 *b, int batch, int ld, const FFTAxis &ax) {
  float2 *src = a, *dst = b;
  int Ns = 1;
  for (int s = 0; s < ax.nstages; ++s) {
    const int R = ax.radix[s];
    switch (R) {
      case 2: stage_fixed<SIGN, 2>(src, dst, batch, ld, ax.n, Ns, ax.tw); break;
      case 3: stage_fixed<SIGN, 3>(src, dst, batch, ld, ax.n, Ns, ax.tw); break;
      case 4: stage_fixed<SIGN, 4>(src, dst, batch, ld, ax.n, Ns, ax.tw); break;
      case 8: stage_fixed<SIGN, 8>(src, dst, batch, ld, ax.n, Ns, ax.tw); break;
      default: stage_generic<SIGN>(src, dst, batch, ld, ax.n, Ns, R, ax.tw); break;
    }
    __syncthreads();
    float2 *t = src;
    src = dst;
    dst = t;
    Ns *= R;
  }
  return src;
}

}  // namespace aw
