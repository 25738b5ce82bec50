// multiscale.cu — scale-level changes on the device: Gaussian downsampling
// of images and trilinear upsampling of deformation fields, so a multiscale
// registration never leaves HBM (the reference round-trips through the
// host, Greedy/GreedyDeformationDataGPU.cxx:91-130).
//
// Arithmetic follows the reference CPU routines exactly:
//  * GaussianFilter3D::filter_symmetric_full (separable x, y, z passes with
//    border-renormalised filters, Utilities/DownsampleFilter/GaussianFilter3D.cxx)
//    and ImageUtils::gaussianDownsample + resampleNew
//    (UtilitiesDataTypes/ImageUtils.txx:259-349);
//  * hToVelocity, HField3DUtils::resampleNew with CLAMP and rescaled vectors,
//    velocityToH (UtilitiesDataTypes/HField3DUtils.txx:57-110, 1816-1881).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "multiscale.cuh"

namespace aw {

namespace {

// one axis of the separable blur; rows = (K+1) x (K+1) filter table. KT > 0
// fixes K at compile time, so the interior taps' loads are all issued before
// the first add (same arithmetic, same order); KT = 0 takes K at run time.
template <int KT>
__global__ void __launch_bounds__(kRowThreads)
    k_gauss_axis(const float *__restrict__ in, float *__restrict__ out, Dims d, int axis, int Kr,
                 const float *__restrict__ rows) {
  Voxel v;
  if (!voxel_of(d, v)) return;
  const int K = KT > 0 ? KT : Kr;
  const int pos = axis == 0 ? v.x : (axis == 1 ? v.y : v.z);
  const int n = axis == 0 ? d.nx : (axis == 1 ? d.ny : d.nz);
  const long st = axis == 0 ? 1 : (axis == 1 ? (long)d.nx : (long)d.nx * d.ny);
  const long i = v.i;
  float o;
  if (pos >= K && pos < n - K) {
    const float *f = rows;
    if (KT > 0) {
      float lo[KT > 0 ? KT : 1], hi[KT > 0 ? KT : 1], fk[KT > 0 ? KT : 1];
#pragma unroll
      for (int k = 1; k <= KT; ++k) {
        lo[k - 1] = __ldg(in + i - k * st);
        hi[k - 1] = __ldg(in + i + k * st);
        fk[k - 1] = __ldg(f + k);
      }
      o = fmul(__ldg(in + i), __ldg(f));
#pragma unroll
      for (int k = 1; k <= KT; ++k) o = fadd(o, fmul(fadd(lo[k - 1], hi[k - 1]), fk[k - 1]));
    } else {
      o = fmul(in[i], f[0]);
      for (int k = 1; k <= K; ++k) o = fadd(o, fmul(fadd(in[i - k * st], in[i + k * st]), f[k]));
    }
  } else if (pos < K) {
    const int x = pos;
    const float *f = rows + (K - x) * (K + 1);
    o = fmul(in[i], f[0]);
    for (int k = 1; k <= x; ++k) o = fadd(o, fmul(fadd(in[i - k * st], in[i + k * st]), f[k]));
    for (int k = x + 1; k <= K; ++k) o = fadd(o, fmul(in[i + k * st], f[k]));
  } else {
    const int x = n - 1 - pos;
    const float *f = rows + (K - x) * (K + 1);
    o = fmul(in[i], f[0]);
    for (int k = 1; k <= x; ++k) o = fadd(o, fmul(fadd(in[i + k * st], in[i - k * st]), f[k]));
    for (int k = x + 1; k <= K; ++k) o = fadd(o, fmul(in[i - k * st], f[k]));
  }
  out[i] = o;
}

// coarse voxel centres sampled from the blurred fine image
__global__ void __launch_bounds__(kRowThreads)
    k_resample_down(const float *__restrict__ blur, Dims din, float *__restrict__ out, Dims dout,
                    Spacing sin, Spacing sout) {
  Voxel v;
  if (!voxel_of(dout, v)) return;
  const double ox = (sout.x - sin.x) / 2.0, oy = (sout.y - sin.y) / 2.0,
               oz = (sout.z - sin.z) / 2.0;
  const double wx = dadd(dadd(dmul(sout.x, (double)v.x), 0.0), ox);
  const double wy = dadd(dadd(dmul(sout.y, (double)v.y), 0.0), oy);
  const double wz = dadd(dadd(dmul(sout.z, (double)v.z), 0.0), oz);
  const double px = __ddiv_rn(dsub(wx, 0.0), sin.x), py = __ddiv_rn(dsub(wy, 0.0), sin.y),
               pz = __ddiv_rn(dsub(wz, 0.0), sin.z);
  out[v.i] = trilerp_scalar(blur, din, px, py, pz, 0.0f);
}

// v = (h - x) * 1.0, the field hToVelocity hands to resampleNew
__global__ void __launch_bounds__(kRowThreads)
    k_h_to_v(const float *__restrict__ hx, const float *__restrict__ hy,
             const float *__restrict__ hz, float *__restrict__ v, Dims d) {
  Voxel p;
  if (!voxel_of(d, p)) return;
  const long n = d.n();
  v[p.i] = fsub(hx[p.i], __int2float_rn(p.x));
  v[n + p.i] = fsub(hy[p.i], __int2float_rn(p.y));
  v[2 * n + p.i] = fsub(hz[p.i], __int2float_rn(p.z));
}

__global__ void __launch_bounds__(kRowThreads)
    k_upsample_field(const float *__restrict__ v, Dims din, float *__restrict__ ox,
                     float *__restrict__ oy, float *__restrict__ oz, Dims dout, int rescale) {
  Voxel p;
  if (!voxel_of(dout, p)) return;
  const double rX = (double)din.nx / dout.nx, rY = (double)din.ny / dout.ny,
               rZ = (double)din.nz / dout.nz;
  const double oX = (rX - 1.0) / 2.0, oY = (rY - 1.0) / 2.0, oZ = (rZ - 1.0) / 2.0;
  const float ix = __double2float_rn(dadd(oX, dmul((double)p.x, rX)));
  const float iy = __double2float_rn(dadd(oY, dmul((double)p.y, rY)));
  const float iz = __double2float_rn(dadd(oZ, dmul((double)p.z, rZ)));
  const long n = din.n();
  float a, b, c;
  trilerp_vector(v, v + n, v + 2 * n, din, ix, iy, iz, BG_CLAMP, 1.0f, a, b, c);
  if (rescale) {
    a = fmul(a, __double2float_rn(1.0 / rX));
    b = fmul(b, __double2float_rn(1.0 / rY));
    c = fmul(c, __double2float_rn(1.0 / rZ));
  }
  ox[p.i] = fadd(__int2float_rn(p.x), a);
  oy[p.i] = fadd(__int2float_rn(p.y), b);
  oz[p.i] = fadd(__int2float_rn(p.z), c);
}

// ImageUtils::resampleNew with BACKGROUND_STRATEGY_CLAMP and linear
// interpolation (UtilitiesDataTypes/ImageUtils.txx:306-349,
// Array3DUtils::trilerp, Array3DUtils.txx:63-210), origin 0: destination
// voxel x samples the source at (x dsp + (dsp - ssp)/2) / ssp, the weights
// formed from the unclamped floor, the corners clamped into the grid.
__global__ void __launch_bounds__(kRowThreads)
    k_resample_image(const float *__restrict__ in, Dims din, double ssx, double ssy, double ssz,
                     float *__restrict__ out, Dims dout, double dsx, double dsy, double dsz) {
  Voxel p;
  if (!voxel_of(dout, p)) return;
  const double pos[3] = {
      __ddiv_rn(dadd(dmul(dsx, (double)p.x), __ddiv_rn(dsub(dsx, ssx), 2.0)), ssx),
      __ddiv_rn(dadd(dmul(dsy, (double)p.y), __ddiv_rn(dsub(dsy, ssy), 2.0)), ssy),
      __ddiv_rn(dadd(dmul(dsz, (double)p.z), __ddiv_rn(dsub(dsz, ssz), 2.0)), ssz)};
  const int size[3] = {din.nx, din.ny, din.nz};
  int f[3], c[3];
  double w[3], omw[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    f[a] = ref_floor_d(pos[a]);
    c[a] = f[a] + 1;
    w[a] = dsub(pos[a], (double)f[a]);
    omw[a] = dsub(1.0, w[a]);
    // the reference's clamp, then (for positions past the last cell plus
    // one, which the reference reads out of bounds) into the grid
    if (f[a] < 0) {
      f[a] = 0;
      if (c[a] < 0) c[a] = 0;
    }
    if (c[a] >= size[a]) {
      c[a] = size[a] - 1;
      if (f[a] > size[a] - 1) f[a] = size[a] - 1;
    }
  }
  float v[8];
  v[0] = __ldg(in + din.idx(f[0], f[1], f[2]));
  v[1] = __ldg(in + din.idx(c[0], f[1], f[2]));
  v[2] = __ldg(in + din.idx(c[0], c[1], f[2]));
  v[3] = __ldg(in + din.idx(f[0], c[1], f[2]));
  v[4] = __ldg(in + din.idx(f[0], c[1], c[2]));
  v[5] = __ldg(in + din.idx(c[0], c[1], c[2]));
  v[6] = __ldg(in + din.idx(c[0], f[1], c[2]));
  v[7] = __ldg(in + din.idx(f[0], f[1], c[2]));
  out[p.i] = __double2float_rn(lerp_tree(v, w[0], w[1], w[2], omw[0], omw[1], omw[2]));
}

// GaussianFilter3D::filter_generate_gauss_full, float arithmetic as there
void gauss_rows(float sigma, int size, std::vector<float> &rows) {
  rows.assign((size_t)(size + 1) * (size + 1), 0.0f);
  float *f0 = rows.data();
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
    for (int i = 0; i <= size; ++i) rows[(size_t)j * (size + 1) + i] = (float)(f0[i] / (1. - scale));
  }
}

}  // namespace

size_t downsample_scratch_bytes(const Dims &din) {
  // two blur buffers
  return sizeof(float) * 2 * (size_t)din.n();
}

namespace {

// The Gaussian tables live in device memory for the life of the process,
// one per (device, sigma, half-width), uploaded by the first call that
// needs them. A later call issues no host copy, so a stream capture of the
// downsampling (a CUDA graph) replays without host data. A table missing
// while the stream is being captured is an error: the first call must run
// outside the capture.
std::mutex g_gauss_mu;
std::map<std::tuple<int, uint32_t, int>, float *> g_gauss;

cudaError_t gauss_table(float sigma, int K, cudaStream_t s, const float **table) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  uint32_t bits;
  std::memcpy(&bits, &sigma, sizeof(bits));
  const auto key = std::make_tuple(dev, bits, K);
  std::lock_guard<std::mutex> lock(g_gauss_mu);
  auto it = g_gauss.find(key);
  if (it != g_gauss.end()) {
    *table = it->second;
    return cudaSuccess;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if ((e = cudaStreamIsCapturing(s, &cs)) != cudaSuccess) return e;
  if (cs != cudaStreamCaptureStatusNone) return cudaErrorStreamCaptureUnsupported;
  std::vector<float> rows;
  gauss_rows(sigma, K, rows);
  float *t = nullptr;
  if ((e = cudaMalloc(&t, rows.size() * sizeof(float))) != cudaSuccess) return e;
  e = cudaMemcpyAsync(t, rows.data(), rows.size() * sizeof(float), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // rows outlives the copy
  if (e != cudaSuccess) {
    cudaFree(t);
    return e;
  }
  g_gauss[key] = t;
  *table = t;
  return cudaSuccess;
}

}  // namespace

cudaError_t downsample(const float *in, Dims din, Spacing sin, float *out, Dims dout,
                       void *scratch, cudaStream_t s) {
  const double f[3] = {(double)din.nx / dout.nx, (double)din.ny / dout.ny,
                       (double)din.nz / dout.nz};
  const int n[3] = {din.nx, din.ny, din.nz};
  float *b1 = static_cast<float *>(scratch);
  float *b2 = b1 + din.n();
  const float *src = in;
  float *dst[3] = {b1, b2, b1};
  for (int a = 0; a < 3; ++a) {
    const double sg = std::sqrt(f[a] / 2.0);
    int K = 2 * (int)std::ceil(sg);
    if (K > n[a] / 2 - 1) K = n[a] / 2 - 1;
    if (K < 0) K = 0;
    const float *t = nullptr;
    cudaError_t e = gauss_table((float)sg, K, s, &t);
    if (e != cudaSuccess) return e;
    switch (K) {
      case 1: k_gauss_axis<1><<<row_grid(din), kRowThreads, 0, s>>>(src, dst[a], din, a, K, t); break;
      case 2: k_gauss_axis<2><<<row_grid(din), kRowThreads, 0, s>>>(src, dst[a], din, a, K, t); break;
      case 3: k_gauss_axis<3><<<row_grid(din), kRowThreads, 0, s>>>(src, dst[a], din, a, K, t); break;
      case 4: k_gauss_axis<4><<<row_grid(din), kRowThreads, 0, s>>>(src, dst[a], din, a, K, t); break;
      default: k_gauss_axis<0><<<row_grid(din), kRowThreads, 0, s>>>(src, dst[a], din, a, K, t);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    src = dst[a];
  }
  // the blur's output spacing is the input's; the coarse grid's is
  // sin * (nin / nout) (gaussianDownsample)
  const Spacing sout{sin.x * f[0], sin.y * f[1], sin.z * f[2]};
  k_resample_down<<<row_grid(dout), kRowThreads, 0, s>>>(src, din, out, dout, sin, sout);
  return cudaGetLastError();
}

cudaError_t resample_image(const float *in, Dims din, Spacing sin, float *out, Dims dout,
                           Spacing sout, cudaStream_t s) {
  k_resample_image<<<row_grid(dout), kRowThreads, 0, s>>>(in, din, sin.x, sin.y, sin.z, out, dout,
                                                         sout.x, sout.y, sout.z);
  return cudaGetLastError();
}

cudaError_t upsample_hfield(const float *const h[3], Dims din, float *const out[3], Dims dout,
                            int rescale, void *scratch, cudaStream_t s) {
  float *v = static_cast<float *>(scratch);
  k_h_to_v<<<row_grid(din), kRowThreads, 0, s>>>(h[0], h[1], h[2], v, din);
  k_upsample_field<<<row_grid(dout), kRowThreads, 0, s>>>(v, din, out[0], out[1], out[2], dout,
                                                          rescale);
  return cudaGetLastError();
}

}  // namespace aw
