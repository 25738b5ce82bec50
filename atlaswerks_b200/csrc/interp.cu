// interp.cu — trilinear apply / compose / gradient kernels and the greedy
// force-side and update-side kernels that use them.
//
// One thread per output voxel, consecutive threads on consecutive x, so the
// streamed planes (h, v, I1, outputs) are read and written fully coalesced;
// the gathers (I0 at h(x), h at x + v) hit L1/L2 because displacements are
// small. Arithmetic follows the reference CPU routines exactly (see
// aw_common.cuh), so with identical inputs the outputs are bit-identical.
#include "interp.cuh"

namespace aw {

namespace {

constexpr int kThreads = kRowThreads;

// HField3DUtils::apply (UtilitiesDataTypes/HField3DUtils.txx:734-752)
__global__ void __launch_bounds__(kThreads)
    k_apply(const float *__restrict__ img, const float *__restrict__ hx, const float *__restrict__ hy,
            const float *__restrict__ hz, float *__restrict__ out, Dims d, float bg) {
  Voxel vx;
  if (!voxel_of(d, vx)) return;
  const long i = vx.i;
  out[i] = trilerp_scalar(img, d, (double)hx[i], (double)hy[i], (double)hz[i], bg);
}

// Array3DUtils::computeGradient (Array3DUtils.txx:783-900)
__global__ void __launch_bounds__(kThreads)
    k_gradient(const float *__restrict__ a, float *__restrict__ gx, float *__restrict__ gy,
               float *__restrict__ gz, Dims d, Spacing sp, int wrap) {
  Voxel vx;
  if (!voxel_of(d, vx)) return;
  const long i = vx.i;
  const int pos[3] = {vx.x, vx.y, vx.z};
  const int n[3] = {d.nx, d.ny, d.nz};
  const long stride[3] = {1, d.nx, (long)d.nx * d.ny};
  const double s[3] = {sp.x, sp.y, sp.z};
  float *g[3] = {gx, gy, gz};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float r;
    if (pos[c] > 0 && pos[c] < n[c] - 1) {
      r = __double2float_rn((double)fsub(a[i + stride[c]], a[i - stride[c]]) / (2.0 * s[c]));
    } else if (wrap) {
      const long ip = pos[c] == n[c] - 1 ? i - (long)(n[c] - 1) * stride[c] : i + stride[c];
      const long im = pos[c] == 0 ? i + (long)(n[c] - 1) * stride[c] : i - stride[c];
      r = __double2float_rn((double)fsub(a[ip], a[im]) / (2.0 * s[c]));
    } else if (pos[c] == 0) {
      r = __double2float_rn((double)fsub(a[i + stride[c]], a[i]) / s[c]);
    } else {
      r = __double2float_rn((double)fsub(a[i], a[i - stride[c]]) / s[c]);
    }
    g[c][i] = r;
  }
}

// composeHV (dir=+1, HField3DUtils.txx:436-455) / composeHVInv (dir=-1,
// :461-480): h(x) = g(x +- (scale*v(x))/sp)
__global__ void __launch_bounds__(kThreads)
    k_compose_hv(const float *__restrict__ gx, const float *__restrict__ gy, const float *__restrict__ gz,
                 const float *__restrict__ vx, const float *__restrict__ vy, const float *__restrict__ vz,
                 float *__restrict__ ox, float *__restrict__ oy, float *__restrict__ oz, Dims d,
                 Spacing sp, int dir, int bgs, const float *__restrict__ scale_ptr, float scale_val) {
  Voxel vox;
  if (!voxel_of(d, vox)) return;
  const long i = vox.i;
  const int x = vox.x, y = vox.y, z = vox.z;
  const float scale = scale_ptr ? *scale_ptr : scale_val;
  const float dx = fdiv(fmul(vx[i], scale), (float)sp.x);
  const float dy = fdiv(fmul(vy[i], scale), (float)sp.y);
  const float dz = fdiv(fmul(vz[i], scale), (float)sp.z);
  float px, py, pz;
  if (dir > 0) {
    px = fadd(__int2float_rn(x), dx); py = fadd(__int2float_rn(y), dy); pz = fadd(__int2float_rn(z), dz);
  } else {
    px = fsub(__int2float_rn(x), dx); py = fsub(__int2float_rn(y), dy); pz = fsub(__int2float_rn(z), dz);
  }
  float rx, ry, rz;
  trilerp_vector(gx, gy, gz, d, px, py, pz, bgs, 1.0f, rx, ry, rz);
  ox[i] = rx;
  oy[i] = ry;
  oz[i] = rz;
}

// composeVH (dir=+1) / composeVHInv (dir=-1, HField3DUtils.txx:405-430):
// h(x) = g(x) +- (scale*v)(g(x))/sp
__global__ void __launch_bounds__(kThreads)
    k_compose_vh(const float *__restrict__ vx, const float *__restrict__ vy, const float *__restrict__ vz,
                 const float *__restrict__ gx, const float *__restrict__ gy, const float *__restrict__ gz,
                 float *__restrict__ ox, float *__restrict__ oy, float *__restrict__ oz, Dims d,
                 Spacing sp, int dir, int bgs, const float *__restrict__ scale_ptr, float scale_val) {
  Voxel vox;
  if (!voxel_of(d, vox)) return;
  const long i = vox.i;
  const float scale = scale_ptr ? *scale_ptr : scale_val;
  const float g0 = gx[i], g1 = gy[i], g2 = gz[i];
  float hx, hy, hz;
  trilerp_vector(vx, vy, vz, d, g0, g1, g2, bgs, scale, hx, hy, hz);
  const float sx = (float)sp.x, sy = (float)sp.y, sz = (float)sp.z;
  if (dir > 0) {
    hx = fdiv(hx, sx); hy = fdiv(hy, sy); hz = fdiv(hz, sz);
  } else {
    hx = fdiv(hx, -sx); hy = fdiv(hy, -sy); hz = fdiv(hz, -sz);
  }
  ox[i] = fadd(hx, g0);
  oy[i] = fadd(hy, g1);
  oz[i] = fadd(hz, g2);
}

}  // namespace

cudaError_t launch_apply(const float *img, const float *hx, const float *hy, const float *hz,
                         float *out, Dims d, float bg, cudaStream_t s) {
  k_apply<<<row_grid(d), kThreads, 0, s>>>(img, hx, hy, hz, out, d, bg);
  return cudaGetLastError();
}

cudaError_t launch_gradient(const float *a, float *gx, float *gy, float *gz, Dims d, Spacing sp,
                            int wrap, cudaStream_t s) {
  k_gradient<<<row_grid(d), kThreads, 0, s>>>(a, gx, gy, gz, d, sp, wrap);
  return cudaGetLastError();
}

cudaError_t launch_compose_hv(const float *const g[3], const float *const v[3], float *const o[3],
                              Dims d, Spacing sp, int dir, int bgs, const float *scale_ptr,
                              float scale_val, cudaStream_t s) {
  k_compose_hv<<<row_grid(d), kThreads, 0, s>>>(g[0], g[1], g[2], v[0], v[1], v[2], o[0], o[1],
                                                    o[2], d, sp, dir, bgs, scale_ptr, scale_val);
  return cudaGetLastError();
}

cudaError_t launch_compose_vh(const float *const v[3], const float *const g[3], float *const o[3],
                              Dims d, Spacing sp, int dir, int bgs, const float *scale_ptr,
                              float scale_val, cudaStream_t s) {
  k_compose_vh<<<row_grid(d), kThreads, 0, s>>>(v[0], v[1], v[2], g[0], g[1], g[2], o[0], o[1],
                                                    o[2], d, sp, dir, bgs, scale_ptr, scale_val);
  return cudaGetLastError();
}

}  // namespace aw
