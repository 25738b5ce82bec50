// fft_reg.cuh — register-resident line FFTs for compile-time lengths.
//
// A line of N = T*E complex values is owned by T consecutive lanes of one
// warp (32/T lines per warp), each lane holding E values. The transform is
// the four-step split N = E x T:
//   1. every lane takes a length-E DFT of its strided values x[t + T*j],
//   2. multiplies by W_N^(t*k1),
//   3. the T lanes exchange through N shared-memory slots of the line
//      (XOR-swizzled so neither the writes nor the reads conflict),
//   4. every lane takes E/T length-T DFTs.
// Only __syncwarp separates the steps. On exit lane t holds
//   v[i*T + k2] = X[(t + T*i) + E*k2],  i < E/T, k2 < T.
// Twiddles come from the host-computed float table W_N^m (forward sign),
// read from global memory or from a copy in shared memory (SmemTw).
#pragma once

#include "fft_smem.cuh"

namespace aw {

// A twiddle table the calling CTA copied into shared memory (the line
// transforms read it instead of the global table: shorter latency, no L1
// traffic competing with the producers' loads)
struct SmemTw {
  const float2 *p;
};
template <int SIGN>
AW_D float2 twiddle(const SmemTw &tw, int m) {
  const float2 w = tw.p[m];
  return SIGN < 0 ? w : make_float2(w.x, -w.y);
}

template <int N>
struct LineCfg;
template <>
struct LineCfg<16> { static constexpr int T = 4, E = 4; };
template <>
struct LineCfg<32> { static constexpr int T = 4, E = 8; };
template <>
struct LineCfg<64> { static constexpr int T = 8, E = 8; };
template <>
struct LineCfg<128> { static constexpr int T = 8, E = 16; };
template <>
struct LineCfg<256> { static constexpr int T = 16, E = 16; };

template <int SIGN>
AW_D void dft4r(float2 &a0, float2 &a1, float2 &a2, float2 &a3) {
  const float2 s02 = cadd(a0, a2), d02 = csub(a0, a2);
  const float2 s13 = cadd(a1, a3), d13 = mul_si<SIGN>(csub(a1, a3));
  a0 = cadd(s02, s13);
  a2 = csub(s02, s13);
  a1 = cadd(d02, d13);
  a3 = csub(d02, d13);
}

template <int SIGN, int E>
struct DFT;

template <int SIGN>
struct DFT<SIGN, 4> {
  static AW_D void run(float2 *v) { dft4r<SIGN>(v[0], v[1], v[2], v[3]); }
};

template <int SIGN>
struct DFT<SIGN, 8> {
  static AW_D void run(float2 *v) { bfly8<SIGN>(v); }
};

// 16 = 4 x 4 with W16 twiddles; natural order in and out
template <int SIGN>
struct DFT<SIGN, 16> {
  static AW_D void run(float2 *v) {
    // columns s: elements v[s + 4m]
#pragma unroll
    for (int s = 0; s < 4; ++s) dft4r<SIGN>(v[s], v[s + 4], v[s + 8], v[s + 12]);
    // now v[s + 4*k1] = A[s][k1]; twiddle by W16^(s*k1)
    const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f;
    const float r2 = 0.70710678118654752440f;
    const float2 w1 = make_float2(c1, SIGN * s1), w2 = make_float2(r2, SIGN * r2),
                 w3 = make_float2(s1, SIGN * c1), w6 = make_float2(-r2, SIGN * r2),
                 w9 = make_float2(-c1, -SIGN * s1);
    v[1 + 4] = cmul(v[5], w1);
    v[1 + 8] = cmul(v[9], w2);
    v[1 + 12] = cmul(v[13], w3);
    v[2 + 4] = cmul(v[6], w2);
    v[2 + 8] = mul_si<SIGN>(v[10]);
    v[2 + 12] = cmul(v[14], w6);
    v[3 + 4] = cmul(v[7], w3);
    v[3 + 8] = cmul(v[11], w6);
    v[3 + 12] = cmul(v[15], w9);
    // rows k1: DFT over s of v[s + 4*k1] -> X[k1 + 4*k2]
    float2 o[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      float2 a0 = v[0 + 4 * k1], a1 = v[1 + 4 * k1], a2 = v[2 + 4 * k1], a3 = v[3 + 4 * k1];
      dft4r<SIGN>(a0, a1, a2, a3);
      o[k1 + 0] = a0;
      o[k1 + 4] = a1;
      o[k1 + 8] = a2;
      o[k1 + 12] = a3;
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = o[i];
  }
};

// Four-step line FFT; see the file comment for the register mapping.
// `slot(m)` returns the address of exchange slot m (0 <= m < N), storage
// that belongs to this line only: the line's own elements in a slab or tile
// when the transform runs in place. Slot (a, b) of the E x T exchange matrix
// is stored at m = a*T + (b ^ (a mod T)): the XOR keeps both the row-wise
// writes and the column-wise reads on distinct banks. `t` is the lane within
// the line. The lanes' inputs must already be in registers: the first write
// to a slot comes after a __syncwarp.
template <int N, int SIGN, class Slot, class Tw>
AW_D void line_fft(float2 *v, int t, const Slot &slot, const Tw &tw) {
  constexpr int T = LineCfg<N>::T, E = LineCfg<N>::E;
  static_assert(E % T == 0, "line split");
  DFT<SIGN, E>::run(v);
#pragma unroll
  for (int k1 = 1; k1 < E; ++k1) v[k1] = cmul(v[k1], twiddle<SIGN>(tw, t * k1));
  __syncwarp();
#pragma unroll
  for (int k1 = 0; k1 < E; ++k1) *slot(k1 * T + (t ^ (k1 & (T - 1)))) = v[k1];
  __syncwarp();
#pragma unroll
  for (int i = 0; i < E / T; ++i) {
    float2 w[T];
#pragma unroll
    for (int s = 0; s < T; ++s) w[s] = *slot((t + T * i) * T + (s ^ t));
    DFT<SIGN, T>::run(w);
#pragma unroll
    for (int k2 = 0; k2 < T; ++k2) v[i * T + k2] = w[k2];
  }
  __syncwarp();
}

// index of the output held in v[r] by lane t
template <int N>
AW_D int line_out_index(int t, int r) {
  constexpr int T = LineCfg<N>::T, E = LineCfg<N>::E;
  return (t + T * (r / T)) + E * (r % T);
}

}  // namespace aw
