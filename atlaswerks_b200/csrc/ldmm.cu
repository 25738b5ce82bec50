// ldmm.cu — one LDMM relaxation iteration on the device,
// LDMMIteratorCPU::IterateNew / LDMMIteratorGPU::IterateNew
// (LDMM/LDMMIteratorCPU.cxx:529-631, LDMM/LDMMIteratorGPU.cxx:159-293):
//
//   forward   for i = 0..T-1: h <- h(x - v_i(x)/sp)  [PARTIAL_ID],
//             J0_i = I0(h)                      (one fused kernel per step)
//   residual  diff = J0_{T-1} - I1, image energy
//   backward  for t = T-1..0:
//               h <- h - v_t(h)/sp               [PARTIAL_ZERO]
//               S = splat(diff, h)               (deterministic, splat.cu)
//               f = grad(J0_{t-1} or I0) * S     (fused into the xy FFT)
//               v_t <- (1 - 2 eps) v_t + (2 eps/sigma^2) K f
//                                                (fused into the inverse FFT)
//
// With a step-size update (UseAdaptiveStepSize at iteration 0) v is left
// unchanged and eps = MaxPert / max_t max_x |2 v_t - (2/sigma^2) K f_t| is
// formed on the device (LDMMIteratorCPU.cxx:192-212, 625-628).
#include <algorithm>
#include <cstring>

#include "interp.cuh"
#include "ldmm.cuh"

namespace aw {

namespace {

__global__ void __launch_bounds__(kRowThreads)
    k_identity(float *__restrict__ hx, float *__restrict__ hy, float *__restrict__ hz, Dims d) {
  Voxel v;
  if (!voxel_of(d, v)) return;
  hx[v.i] = __int2float_rn(v.x);
  hy[v.i] = __int2float_rn(v.y);
  hz[v.i] = __int2float_rn(v.z);
}

// h_out(x) = h_in(x - v(x)/sp) [PARTIAL_ID]; J(x) = I0(h_out(x))
// (composeHVInv + apply, LDMMIteratorCPU.cxx:549-554); with PLUS,
// h_in(x + v(x)/sp) (composeHV, IterateOrig's backward sweep :397-405)
template <bool PLUS>
__global__ void __launch_bounds__(kRowThreads)
    k_forward_step(const float *__restrict__ hx, const float *__restrict__ hy,
                   const float *__restrict__ hz, const float *__restrict__ vx,
                   const float *__restrict__ vy, const float *__restrict__ vz,
                   float *__restrict__ ox, float *__restrict__ oy, float *__restrict__ oz,
                   const float *__restrict__ I0, float *__restrict__ J, Dims d, Spacing sp) {
  Voxel vox;
  if (!voxel_of(d, vox)) return;
  const long i = vox.i;
  const float ux = fdiv(vx[i], (float)sp.x), uy = fdiv(vy[i], (float)sp.y),
              uz = fdiv(vz[i], (float)sp.z);
  const float px = PLUS ? fadd(__int2float_rn(vox.x), ux) : fsub(__int2float_rn(vox.x), ux);
  const float py = PLUS ? fadd(__int2float_rn(vox.y), uy) : fsub(__int2float_rn(vox.y), uy);
  const float pz = PLUS ? fadd(__int2float_rn(vox.z), uz) : fsub(__int2float_rn(vox.z), uz);
  float a, b, c;
  trilerp_vector(hx, hy, hz, d, px, py, pz, BG_PARTIAL_ID, 1.0f, a, b, c);
  ox[i] = a;
  oy[i] = b;
  oz[i] = c;
  if (J) J[i] = trilerp_scalar(I0, d, (double)a, (double)b, (double)c, 0.0f);
}

// float component c of IterateOrig's world-coordinate map x*sp + v
// (setToIdentity, scale by the float spacing, pointwiseAdd v:
// LDMMIteratorCPU.cxx:409-414)
AW_D float world(const float *__restrict__ vc, long i, int coord, float spc) {
  return fadd(fmul(__int2float_rn(coord), spc), __ldg(vc + i));
}

// d/d(axis) of component c of the world map at voxel (x,y,z): computeGradient
// with wrap = false (Array3DUtils.txx:783-900), as SrcForce forms it
AW_D float world_grad(const float *__restrict__ vc, int c, int axis, int x, int y, int z,
                      const Dims &d, float spc, const DivD &c2, const DivD &c1) {
  const int p[3] = {x, y, z};
  const int n = axis == 0 ? d.nx : (axis == 1 ? d.ny : d.nz);
  const long st = axis == 0 ? 1 : (axis == 1 ? (long)d.nx : (long)d.nx * d.ny);
  const long i = d.idx(x, y, z);
  const int pos = p[axis];
  const int cc = p[c];  // the coordinate that component c adds to v
  // the neighbours' own coordinate along c moves only when axis == c
  const int dlo = (axis == c) ? -1 : 0, dhi = (axis == c) ? 1 : 0;
  if (pos > 0 && pos < n - 1)
    return __double2float_rn(ddiv((double)fsub(world(vc, i + st, cc + dhi, spc),
                                                world(vc, i - st, cc + dlo, spc)), c2));
  if (pos == 0)
    return __double2float_rn(ddiv((double)fsub(world(vc, i + st, cc + dhi, spc),
                                                world(vc, i, cc, spc)), c1));
  return __double2float_rn(ddiv((double)fsub(world(vc, i, cc, spc),
                                              world(vc, i - st, cc + dlo, spc)), c1));
}

// JacDet_t = (t < T-1 ? JacDet_{t+1}(x + v_t/sp) : 1) * |D(x*sp + v_t)|
// (HField3DUtils::jacobian + applyU + pointwiseMultiplyBy,
// LDMMIteratorCPU.cxx:416-427; the determinant of HField3DUtils.txx:2408-2419)
__global__ void __launch_bounds__(kRowThreads)
    k_jacdet(const float *__restrict__ vx, const float *__restrict__ vy,
             const float *__restrict__ vz, const float *__restrict__ next,
             float *__restrict__ out, Dims d, Spacing sp, DivD a2, DivD b2, DivD e2, DivD a1,
             DivD b1, DivD e1) {
  Voxel vox;
  if (!voxel_of(d, vox)) return;
  const int x = vox.x, y = vox.y, z = vox.z;
  const float s[3] = {(float)sp.x, (float)sp.y, (float)sp.z};
  const DivD c2[3] = {a2, b2, e2}, c1[3] = {a1, b1, e1};
  const float *vc[3] = {vx, vy, vz};
  float g[3][3];  // g[c][axis]
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int a = 0; a < 3; ++a) g[c][a] = world_grad(vc[c], c, a, x, y, z, d, s[c], c2[a], c1[a]);
  const float t1 = fmul(g[0][0], fsub(fmul(g[1][1], g[2][2]), fmul(g[1][2], g[2][1])));
  const float t2 = fmul(g[0][1], fsub(fmul(g[1][0], g[2][2]), fmul(g[1][2], g[2][0])));
  const float t3 = fmul(g[0][2], fsub(fmul(g[1][0], g[2][1]), fmul(g[1][1], g[2][0])));
  const float jac = fadd(fsub(t1, t2), t3);
  const long i = vox.i;
  if (next) {
    // applyU: coord = v/sp + (x,y,z), default scalar background 0
    const float px = fadd(fdiv(vx[i], s[0]), __int2float_rn(x));
    const float py = fadd(fdiv(vy[i], s[1]), __int2float_rn(y));
    const float pz = fadd(fdiv(vz[i], s[2]), __int2float_rn(z));
    out[i] = fmul(trilerp_scalar(next, d, (double)px, (double)py, (double)pz, 0.0f), jac);
  } else {
    out[i] = jac;
  }
}

__global__ void __launch_bounds__(kRowThreads)
    k_residual(const float *__restrict__ J, const float *__restrict__ I1, float *__restrict__ diff,
               double *__restrict__ partials, Dims d) {
  Voxel v;
  double e = 0.0;
  if (voxel_of(d, v)) {
    const float r = fsub(J[v.i], I1[v.i]);
    diff[v.i] = r;
    e = (double)r * (double)r;
  }
  __shared__ double ws[kRowThreads / 32];
  e = warp_sum(e);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < kRowThreads / 32 ? ws[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0)
      partials[((long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = t;
  }
}

// energy[(count - back) % cap] = scale * sum(partials) (add: +=); advance:
// count += 1 (the image energy, recorded last in an iteration)
// one block of kRecThreads; four independent partial sums per thread keep
// four loads in flight (a fixed order: the same sum on every run)
constexpr int kRecThreads = 1024;
__global__ void __launch_bounds__(kRecThreads)
    k_record_energy(const double *__restrict__ partials, int nparts, double scale,
                    double *__restrict__ energy, int *__restrict__ count, int cap,
                    int advance = 1, int add = 0, int back = 0) {
  double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
  int i = threadIdx.x;
  for (; i + 3 * kRecThreads < nparts; i += 4 * kRecThreads) {
    t0 += __ldg(partials + i);
    t1 += __ldg(partials + i + kRecThreads);
    t2 += __ldg(partials + i + 2 * kRecThreads);
    t3 += __ldg(partials + i + 3 * kRecThreads);
  }
  for (; i < nparts; i += kRecThreads) t0 += __ldg(partials + i);
  double t = (t0 + t1) + (t2 + t3);
  __shared__ double ws[kRecThreads / 32];
  t = warp_sum(t);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kRecThreads / 32; ++w) s += ws[w];
    const int k = *count - back;
    energy[k % cap] = add ? energy[k % cap] + s * scale : s * scale;
    if (advance) *count = *count + 1;
  }
}

// max |2 v - (2/sigma^2) u| in the reference's float arithmetic
// (calcMaxDisplacement, LDMMIteratorCPU.cxx:192-212)
__global__ void __launch_bounds__(256)
    k_max_disp(const float *__restrict__ vx, const float *__restrict__ vy,
               const float *__restrict__ vz, const float *__restrict__ ux,
               const float *__restrict__ uy, const float *__restrict__ uz, long n, float sigma,
               unsigned *__restrict__ maxbits) {
  const float a = 2.0f, b = fdiv(-2.0f, fmul(sigma, sigma));
  float m = 0.0f;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float x = fadd(fmul(a, vx[i]), fmul(b, ux[i]));
    const float y = fadd(fmul(a, vy[i]), fmul(b, uy[i]));
    const float z = fadd(fmul(a, vz[i]), fmul(b, uz[i]));
    m = fmaxf(m, sqrtf(fadd(fadd(fmul(x, x), fmul(y, y)), fmul(z, z))));
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) atomicMax(maxbits, __float_as_uint(m));
}

__global__ void k_step_from_max(const unsigned *__restrict__ maxbits, float max_pert,
                                float *__restrict__ step) {
  *step = fdiv(max_pert, __uint_as_float(*maxbits));
}

// ---- adjoint shooting (LDMMAdShootingIteratorCPU.cxx:237-453) ----------

// central (2 sp) and one-sided (sp) divisors per axis of computeGradient
struct GradDiv {
  DivD c2[3], c1[3];
};

GradDiv grad_div(const Spacing &sp) {
  return GradDiv{{make_div(2.0 * sp.x), make_div(2.0 * sp.y), make_div(2.0 * sp.z)},
                 {make_div(sp.x), make_div(sp.y), make_div(sp.z)}};
}

// along axis c of voxel v: the offset to the two samples computeGradient
// (wrap = false, Array3DUtils.txx:783-900) differences, and whether the
// voxel is interior (central difference) or on a face (one-sided)
struct GradTaps {
  long lo, hi;
  bool in;
};
AW_D GradTaps grad_taps(int c, const Voxel &v, const Dims &d) {
  const int pos = c == 0 ? v.x : (c == 1 ? v.y : v.z);
  const int n = c == 0 ? d.nx : (c == 1 ? d.ny : d.nz);
  const long st = c == 0 ? 1 : (c == 1 ? (long)d.nx : (long)d.nx * d.ny);
  return GradTaps{pos > 0 ? -st : 0, pos < n - 1 ? st : 0, pos > 0 && pos < n - 1};
}
AW_D float grad_of(float diff, int c, const GradTaps &t, const GradDiv &g) {
  return __double2float_rn(ddiv((double)diff, t.in ? g.c2[c] : g.c1[c]));
}
// component c of computeGradient(a) at voxel v
AW_D float ref_grad(const float *__restrict__ a, int c, const Voxel &v, const Dims &d,
                    const GradDiv &g) {
  const GradTaps t = grad_taps(c, v, d);
  return grad_of(fsub(__ldg(a + v.i + t.hi), __ldg(a + v.i + t.lo)), c, t, g);
}

// f = grad(alphaHat) * alpha_t - grad(I_t) * IHat, component-wise in float
// (backwardAdIntegration, LDMMAdShootingIteratorCPU.cxx:384-392)
__global__ void __launch_bounds__(kRowThreads)
    k_ad_force(const float *__restrict__ aHat, const float *__restrict__ aT,
               const float *__restrict__ IT, const float *__restrict__ IHat, float *__restrict__ fx,
               float *__restrict__ fy, float *__restrict__ fz, Dims d, GradDiv g) {
  Voxel v;
  if (!voxel_of(d, v)) return;
  const float at = __ldg(aT + v.i), ih = __ldg(IHat + v.i);
  float *const f[3] = {fx, fy, fz};
#pragma unroll
  for (int c = 0; c < 3; ++c)
    f[c][v.i] = fsub(fmul(ref_grad(aHat, c, v, d, g), at), fmul(ref_grad(IT, c, v, d, g), ih));
}

// dot = grad(I_t) . vhat (Vector3D::dot in float, x first) and
// div = div(alpha_t * vhat) (HField3DUtils::divergence, wrap = false: the
// products formed in float at each tap, the partials summed in float)
// (LDMMAdShootingIteratorCPU.cxx:398-417)
__global__ void __launch_bounds__(kRowThreads)
    k_ad_dot_div(const float *__restrict__ IT, const float *__restrict__ vx,
                 const float *__restrict__ vy, const float *__restrict__ vz,
                 const float *__restrict__ aT, float *__restrict__ dot, float *__restrict__ div,
                 Dims d, GradDiv g) {
  Voxel v;
  if (!voxel_of(d, v)) return;
  const float *const vc[3] = {vx, vy, vz};
  float dp = 0.0f, dv = 0.0f;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float gi = ref_grad(IT, c, v, d, g);
    const float p = fmul(gi, __ldg(vc[c] + v.i));
    dp = c == 0 ? p : fadd(dp, p);
    const GradTaps t = grad_taps(c, v, d);
    const float hi = fmul(__ldg(vc[c] + v.i + t.hi), __ldg(aT + v.i + t.hi));
    const float lo = fmul(__ldg(vc[c] + v.i + t.lo), __ldg(aT + v.i + t.lo));
    const float part = grad_of(fsub(hi, lo), c, t, g);
    dv = c == 0 ? part : fadd(dv, part);
  }
  dot[v.i] = dp;
  div[v.i] = dv;
}

// out = src(h) with background 0 (HField3DUtils::apply); sub: out -= src(h)
template <bool SUB>
__global__ void __launch_bounds__(kRowThreads)
    k_ad_pull(const float *__restrict__ src, const float *__restrict__ hx,
              const float *__restrict__ hy, const float *__restrict__ hz, float *__restrict__ out,
              Dims d) {
  Voxel v;
  if (!voxel_of(d, v)) return;
  const float r = trilerp_scalar(src, d, (double)__ldg(hx + v.i), (double)__ldg(hy + v.i),
                                 (double)__ldg(hz + v.i), 0.0f);
  out[v.i] = SUB ? fsub(out[v.i], r) : r;
}

__global__ void __launch_bounds__(256) k_ad_add(float *__restrict__ a, const float *__restrict__ b,
                                                long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = fadd(a[i], b[i]);
}

// IHat = (I1 - I0(phiT0)) * (1 / sigma^2) and the image-energy partials of
// (I0(phiT0) - I1)^2 (LDMMAdShootingIteratorCPU.cxx:313-316, 338-342)
__global__ void __launch_bounds__(kRowThreads)
    k_ad_residual(const float *__restrict__ J, const float *__restrict__ I1, float inv,
                  float *__restrict__ ihat, double *__restrict__ partials, Dims d) {
  Voxel v;
  double e = 0.0;
  if (voxel_of(d, v)) {
    const float j = J[v.i], i1 = I1[v.i];
    ihat[v.i] = fmul(fsub(i1, j), inv);
    const float r = fsub(j, i1);
    e = (double)r * (double)r;
  }
  __shared__ double ws[kRowThreads / 32];
  e = warp_sum(e);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < kRowThreads / 32 ? ws[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0)
      partials[((long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = t;
  }
}

// partials of <L v, v> for v = sign * K f without applying L: L K f = f,
// so it is sum_c sum_x (sign f_c) v_c with the body force f = grad(G) A
// formed again on the fly as the forward transform formed it (SrcForce);
// float products summed in double, as HField3DUtils::l2DotProd sums
// (L v)_c v_c. Equal to the explicit L v route up to the transforms' float
// rounding.
__global__ void __launch_bounds__(kRowThreads)
    k_force_vdot(SrcForce f, const float *__restrict__ v, float sign,
                 double *__restrict__ partials, Dims d) {
  Voxel p;
  double e = 0.0;
  if (voxel_of(d, p)) {
    const long n = d.n();
#pragma unroll
    for (int c = 0; c < 3; ++c)
      e += (double)fmul(sign * f.value(c, p.x, p.y, p.z, d), v[c * n + p.i]);
  }
  __shared__ double ws[kRowThreads / 32];
  e = warp_sum(e);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < kRowThreads / 32 ? ws[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0)
      partials[((long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = t;
  }
}

// sum_c u_c v_c per block (float products summed in double), the step
// energy <L v, v> of HField3DUtils::l2DotProd with u = L v
__global__ void __launch_bounds__(kRowThreads)
    k_field_dot(const float *__restrict__ u, const float *__restrict__ v,
                double *__restrict__ partials, Dims d) {
  Voxel p;
  double e = 0.0;
  if (voxel_of(d, p)) {
    const long n = d.n();
#pragma unroll
    for (int c = 0; c < 3; ++c) e += (double)fmul(u[c * n + p.i], v[c * n + p.i]);
  }
  __shared__ double ws[kRowThreads / 32];
  e = warp_sum(e);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < kRowThreads / 32 ? ws[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0)
      partials[((long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = t;
  }
}

// alpha0 -= step * (-(grad(I0) . v0) - alphaTilde), float in the
// reference's order (LDMMAdShootingIteratorCPU.cxx:421-430)
__global__ void __launch_bounds__(kRowThreads)
    k_ad_alpha(const float *__restrict__ I0, const float *__restrict__ v0,
               const float *__restrict__ aTil, const float *__restrict__ step,
               float *__restrict__ alpha0, Dims d, GradDiv g) {
  Voxel v;
  if (!voxel_of(d, v)) return;
  const long n = d.n();
  float dp = 0.0f;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float p = fmul(ref_grad(I0, c, v, d, g), __ldg(v0 + c * n + v.i));
    dp = c == 0 ? p : fadd(dp, p);
  }
  const float gr = fmul(fsub(fmul(dp, -1.0f), aTil[v.i]), *step);
  alpha0[v.i] = fsub(alpha0[v.i], gr);
}

#define AW_TRY(x)                     \
  do {                                \
    cudaError_t _e = (x);             \
    if (_e != cudaSuccess) return _e; \
  } while (0)

}  // namespace

int ldmm_create(LdmmCtx *c, int nx, int ny, int nz, double spx, double spy, double spz,
                float alpha, float beta, float gamma, int T, float sigma, float max_pert) {
  std::memset(c, 0, sizeof(*c));
  const int rc = fluid_plan_create(&c->plan, nx, ny, nz, spx, spy, spz, alpha, beta, gamma);
  if (rc) return rc;
  c->d = c->plan.d;
  c->sp = c->plan.sp;
  c->T = T;
  c->sigma = sigma;
  c->max_pert = max_pert;
  c->cap = 4096;
  const long n = c->d.n();
  const dim3 gr = row_grid(c->d);
  c->nparts = (int)(gr.x * gr.y * gr.z);
  if (cudaMalloc(&c->J0, sizeof(float) * n * T) != cudaSuccess) return 3;
  if (cudaMalloc(&c->hbuf, sizeof(float) * 6 * n) != cudaSuccess) return 3;
  if (cudaMalloc(&c->diff, sizeof(float) * n) != cudaSuccess) return 3;
  if (cudaMalloc(&c->S, sizeof(float) * n) != cudaSuccess) return 3;
  if (cudaMalloc(&c->u, sizeof(float) * 3 * n) != cudaSuccess) return 3;
  if (cudaMalloc(&c->splat_scratch, splat_scratch_bytes(c->d)) != cudaSuccess) return 3;
  if (cudaMalloc(&c->partials, sizeof(double) * c->nparts) != cudaSuccess) return 3;
  if (cudaMalloc(&c->energy, sizeof(double) * c->cap) != cudaSuccess) return 3;
  if (cudaMalloc(&c->venergy, sizeof(double) * c->cap) != cudaSuccess) return 3;
  cudaMemset(c->venergy, 0, sizeof(double) * c->cap);
  if (cudaMalloc(&c->scalars, 64) != cudaSuccess) return 3;
  cudaMemset(c->scalars, 0, 64);
  c->step = reinterpret_cast<float *>(c->scalars);
  c->count = reinterpret_cast<int *>(c->scalars + 4);
  c->maxbits = reinterpret_cast<unsigned *>(c->scalars + 8);
  c->zero = reinterpret_cast<int *>(c->scalars + 12);
  if (cudaMalloc(&c->vstep, sizeof(double) * T) != cudaSuccess) return 3;
  cudaMemset(c->vstep, 0, sizeof(double) * T);
  splat_work_bind(&c->sw, c->d, c->splat_scratch);
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

void ldmm_destroy(LdmmCtx *c) {
  fluid_plan_destroy(&c->plan);
  void *ptrs[] = {c->J0,     c->hbuf,   c->diff, c->S,   c->u,   c->splat_scratch,
                  c->partials, c->energy, c->scalars, c->JT, c->JD, c->adV,
                  c->adP,    c->adA,    c->adI,  c->venergy, c->adSortMem, c->vstep,
                  c->vsBuf};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  std::memset(c, 0, sizeof(*c));
}

cudaError_t ldmm_iterate_orig(LdmmCtx *c, const float *I0, const float *I1, float *v,
                              int update_step, cudaStream_t s);

cudaError_t identity_field(float *hx, float *hy, float *hz, Dims d, cudaStream_t s) {
  k_identity<<<row_grid(d), kRowThreads, 0, s>>>(hx, hy, hz, d);
  return cudaGetLastError();
}

namespace {
// IterateNew's forward integration (J0_t = I0 at the composed map of every
// time point) and the residual J0_{T-1} - I1 with its energy partials; the
// energy is recorded unless the step is being recomputed
// (LDMMIteratorCPU.cxx:543-556, 616-627)
cudaError_t ldmm_forward(LdmmCtx *c, const float *I0, const float *I1, const float *v,
                         int update_step, cudaStream_t s) {
  const Dims d = c->d;
  const long n = d.n();
  const int T = c->T;
  float *H[2] = {c->hbuf, c->hbuf + 3 * n};
  auto comp = [&](float *base, int k) { return base + k * n; };
  auto vcomp = [&](const float *base, int k) { return base + k * n; };
  k_identity<<<row_grid(d), kRowThreads, 0, s>>>(comp(H[0], 0), comp(H[0], 1), comp(H[0], 2), d);
  AW_TRY(cudaGetLastError());
  int cur = 0;
  for (int i = 0; i < T; ++i) {
    const float *vi = v + (long)i * 3 * n;
    k_forward_step<false><<<row_grid(d), kRowThreads, 0, s>>>(
        comp(H[cur], 0), comp(H[cur], 1), comp(H[cur], 2), vcomp(vi, 0), vcomp(vi, 1),
        vcomp(vi, 2), comp(H[1 - cur], 0), comp(H[1 - cur], 1), comp(H[1 - cur], 2), I0,
        c->J0 + (long)i * n, d, c->sp);
    AW_TRY(cudaGetLastError());
    cur = 1 - cur;
  }
  k_residual<<<row_grid(d), kRowThreads, 0, s>>>(c->J0 + (long)(T - 1) * n, I1, c->diff,
                                                 c->partials, d);
  AW_TRY(cudaGetLastError());
  if (!update_step) {
    const double spprod = c->sp.x * c->sp.y * c->sp.z;
    k_record_energy<<<1, kRecThreads, 0, s>>>(c->partials, c->nparts, spprod, c->energy,
                                              c->count, c->cap);
    AW_TRY(cudaGetLastError());
  }
  return cudaSuccess;
}

// The vector energy of LDMMIteratorCPU's debug mode (LDMMIteratorCPU.cxx:
// 493-505 for IterateOrig, 601-610 for IterateNew): <L v_t, v_t> of the
// updated v_t, through one more forward transform, L and inverse; added up
// over the time steps of the iteration at energy index count - back.
static cudaError_t vec_step_energy(LdmmCtx *c, const float *vt, int t, int first, int back,
                                   cudaStream_t s) {
  const long n = c->d.n();
  float *u = c->u;
  AW_TRY(fluid_forward_field(c->plan, vt, vt + n, vt + 2 * n, s));
  AW_TRY(fluid_solve(c->plan, 0, s));
  AW_TRY(fluid_inverse_store(c->plan, u, u + n, u + 2 * n, s));
  k_field_dot<<<row_grid(c->d), kRowThreads, 0, s>>>(u, vt, c->partials, c->d);
  AW_TRY(cudaGetLastError());
  const double spprod = c->sp.x * c->sp.y * c->sp.z;
  k_record_energy<<<1, kRecThreads, 0, s>>>(c->partials, c->nparts, spprod, c->venergy, c->count,
                                            c->cap, 0, first ? 0 : 1, back);
  AW_TRY(cudaGetLastError());
  k_record_energy<<<1, kRecThreads, 0, s>>>(c->partials, c->nparts, spprod, c->vstep + t, c->zero,
                                            1, 0, 0, 0);
  return cudaGetLastError();
}

// alpha_t = splat / sigma^2 in float, the factor (float)(1.0 / (sigma*sigma))
// as Array3D::scale receives it (LDMMIteratorCPU.cxx:583-585)
__global__ void __launch_bounds__(256)
    k_scale_to(float *__restrict__ dst, const float *__restrict__ src, float f, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = fmul(src[i], f);
}
}  // namespace

// IterateNew with computeAlphasOnly (LDMMIteratorCPU.cxx:529-631): the
// forward integration, the residual and its energy, then the backward sweep
// of composeVHInv and splats, each splat scaled by 1/sigma^2 into
// alphas[t]; v is left as it is.
cudaError_t ldmm_alphas(LdmmCtx *c, const float *I0, const float *I1, const float *v,
                        float *alphas, cudaStream_t s) {
  const Dims d = c->d;
  const long n = d.n();
  const int T = c->T;
  AW_TRY(ldmm_forward(c, I0, I1, v, 0, s));
  float *H[2] = {c->hbuf, c->hbuf + 3 * n};
  auto comp = [&](float *base, int k) { return base + k * n; };
  k_identity<<<row_grid(d), kRowThreads, 0, s>>>(comp(H[0], 0), comp(H[0], 1), comp(H[0], 2), d);
  AW_TRY(cudaGetLastError());
  const float f = (float)(1.0 / (double)(c->sigma * c->sigma));
  int cur = 0;
  for (int t = T - 1; t >= 0; --t) {
    const float *vt = v + (long)t * 3 * n;
    const float *vv[3] = {vt, vt + n, vt + 2 * n};
    const float *hh[3] = {comp(H[cur], 0), comp(H[cur], 1), comp(H[cur], 2)};
    float *oo[3] = {comp(H[1 - cur], 0), comp(H[1 - cur], 1), comp(H[1 - cur], 2)};
    AW_TRY(launch_compose_vh(vv, hh, oo, d, c->sp, -1, BG_PARTIAL_ZERO, nullptr, 1.0f, s));
    cur = 1 - cur;
    AW_TRY(splat(c->sw, c->diff, comp(H[cur], 0), comp(H[cur], 1), comp(H[cur], 2), c->S, 0.0f, s));
    k_scale_to<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(alphas + (long)t * n, c->S, f, n);
    AW_TRY(cudaGetLastError());
  }
  return cudaSuccess;
}

cudaError_t ldmm_iterate(LdmmCtx *c, const float *I0, const float *I1, float *v, int update_step,
                         cudaStream_t s) {
  if (c->orig) return ldmm_iterate_orig(c, I0, I1, v, update_step, s);
  const Dims d = c->d;
  const long n = d.n();
  const int T = c->T;
  float *H[2] = {c->hbuf, c->hbuf + 3 * n};
  auto comp = [&](float *base, int k) { return base + k * n; };
  AW_TRY(ldmm_forward(c, I0, I1, v, update_step, s));
  if (update_step) AW_TRY(cudaMemsetAsync(c->maxbits, 0, sizeof(unsigned), s));
  int cur = 0;
  // backward sweep
  k_identity<<<row_grid(d), kRowThreads, 0, s>>>(comp(H[0], 0), comp(H[0], 1), comp(H[0], 2), d);
  AW_TRY(cudaGetLastError());
  cur = 0;
  for (int t = T - 1; t >= 0; --t) {
    float *vt = v + (long)t * 3 * n;
    const float *vv[3] = {comp(vt, 0), comp(vt, 1), comp(vt, 2)};
    const float *hh[3] = {comp(H[cur], 0), comp(H[cur], 1), comp(H[cur], 2)};
    float *oo[3] = {comp(H[1 - cur], 0), comp(H[1 - cur], 1), comp(H[1 - cur], 2)};
    AW_TRY(launch_compose_vh(vv, hh, oo, d, c->sp, -1, BG_PARTIAL_ZERO, nullptr, 1.0f, s));
    cur = 1 - cur;
    AW_TRY(splat(c->sw, c->diff, comp(H[cur], 0), comp(H[cur], 1), comp(H[cur], 2), c->S, 0.0f, s));
    const float *G = t > 0 ? c->J0 + (long)(t - 1) * n : I0;
    AW_TRY(fluid_forward_force(c->plan, G, c->S, 0, s));
    AW_TRY(fluid_solve(c->plan, 1, s));
    if (update_step) {
      AW_TRY(fluid_inverse_store(c->plan, comp(c->u, 0), comp(c->u, 1), comp(c->u, 2), s));
      int sms = 148;
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->plan.device);
      k_max_disp<<<sms * 4, 256, 0, s>>>(comp(vt, 0), comp(vt, 1), comp(vt, 2), comp(c->u, 0),
                                         comp(c->u, 1), comp(c->u, 2), n, c->sigma, c->maxbits);
      AW_TRY(cudaGetLastError());
    } else {
      AW_TRY(fluid_inverse_axpby(c->plan, comp(vt, 0), comp(vt, 1), comp(vt, 2), c->step,
                                 c->sigma, s));
      // the image energy was recorded (and the count advanced) up front
      if (c->vec_energy) AW_TRY(vec_step_energy(c, vt, t, t == T - 1, 1, s));
    }
  }
  if (update_step) {
    k_step_from_max<<<1, 1, 0, s>>>(c->maxbits, c->max_pert, c->step);
    AW_TRY(cudaGetLastError());
  }
  return cudaSuccess;
}

// LDMMDeformationData::GetI1At0 (LDMM/LDMMDeformationData.cxx:255-265,
// 325-336: h_{0->1} by composeHV [PARTIAL_ID] from t = T-1 down to 0, then
// apply with background 0) and LDMMIteratorCPU::ComputeJacDet
// (LDMMIteratorCPU.cxx:309-340), the same backward sweep as IterateOrig's.
// The Jacobian ping-pongs between jd and the context's splat buffer so that
// t = 0 lands in jd; jd may be null.
cudaError_t ldmm_i1_at_0(LdmmCtx *c, const float *I1, const float *v, float *img, float *jd,
                         cudaStream_t s) {
  const Dims d = c->d;
  const long n = d.n();
  const int T = c->T;
  float *H[2] = {c->hbuf, c->hbuf + 3 * n};
  auto comp = [&](float *base, int k) { return base + k * n; };
  auto vcomp = [&](const float *base, int k) { return base + k * n; };
  const DivD a2 = make_div(2.0 * c->sp.x), b2 = make_div(2.0 * c->sp.y), e2 = make_div(2.0 * c->sp.z);
  const DivD a1 = make_div(c->sp.x), b1 = make_div(c->sp.y), e1 = make_div(c->sp.z);
  auto jbuf = [&](int t) { return (t % 2 == 0) ? jd : c->S; };
  k_identity<<<row_grid(d), kRowThreads, 0, s>>>(comp(H[0], 0), comp(H[0], 1), comp(H[0], 2), d);
  AW_TRY(cudaGetLastError());
  int cur = 0;
  for (int t = T - 1; t >= 0; --t) {
    const float *vt = v + (long)t * 3 * n;
    k_forward_step<true><<<row_grid(d), kRowThreads, 0, s>>>(
        comp(H[cur], 0), comp(H[cur], 1), comp(H[cur], 2), vcomp(vt, 0), vcomp(vt, 1),
        vcomp(vt, 2), comp(H[1 - cur], 0), comp(H[1 - cur], 1), comp(H[1 - cur], 2), I1,
        t == 0 ? img : nullptr, d, c->sp);
    AW_TRY(cudaGetLastError());
    cur = 1 - cur;
    if (jd) {
      k_jacdet<<<row_grid(d), kRowThreads, 0, s>>>(vcomp(vt, 0), vcomp(vt, 1), vcomp(vt, 2),
                                                   t == T - 1 ? nullptr : jbuf(t + 1), jbuf(t),
                                                   d, c->sp, a2, b2, e2, a1, b1, e1);
      AW_TRY(cudaGetLastError());
    }
  }
  return cudaSuccess;
}

namespace {
// LDMMAtlasThreadCPU::ComputeThreadMean's sums (LDMM/LDMMAtlasThreadCPU.cxx:
// 243-252), float in the reference's order: acc += (img * jd) * w and
// jsum += jd * w with JacobianScale (jd given), else acc += img * w
__global__ void k_atlas_accumulate(float *__restrict__ acc, float *__restrict__ jsum,
                                   const float *__restrict__ img, const float *__restrict__ jd,
                                   float w, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (jd) {
    acc[i] = fadd(acc[i], fmul(fmul(img[i], jd[i]), w));
    jsum[i] = fadd(jsum[i], fmul(jd[i], w));
  } else {
    acc[i] = fadd(acc[i], fmul(img[i], w));
  }
}
// mean = acc / jsum (RealImage::pointwiseDivideBy, LDMMAtlasBuilder.txx:332-334)
__global__ void k_atlas_normalize(float *__restrict__ acc, const float *__restrict__ jsum, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) acc[i] = fdiv(acc[i], jsum[i]);
}
}  // namespace

cudaError_t ldmm_atlas_accumulate(float *acc, float *jsum, const float *img, const float *jd,
                                  float w, long n, cudaStream_t s) {
  k_atlas_accumulate<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(acc, jsum, img, jd, w, n);
  return cudaGetLastError();
}

cudaError_t ldmm_atlas_normalize(float *acc, const float *jsum, long n, cudaStream_t s) {
  k_atlas_normalize<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(acc, jsum, n);
  return cudaGetLastError();
}

// ---- the per-voxel median of the deformed subjects ------------------------
// MedianCalculator::Select(std::vector<RealImage*>, k, rtn) (Algorithms/
// Common/MedianCalculator.cxx:264-389), used as the atlas with
// UsePerVoxelMedian (LDMMAtlasBuilder.txx:218-233, 336-338): per voxel a
// bisection on the value between the voxel's min and max over the images;
// each round counts the values below the midpoint p and takes the largest
// value below it and the smallest at or above it; the voxel ends when the
// count is k (the latter) or k + 1 (the former), or when its interval is
// narrower than eps = (max over the volume - min over the volume) / 10000
// (its lower end). Voxels are independent, so each thread runs its own
// rounds; a voxel still open after round nImages + 1 is the reference's
// "not converging" error.
namespace {

__device__ __forceinline__ unsigned order_key(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_value(unsigned k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// min / max over the images at one voxel (MedianCalculator::MinMax)
__device__ __forceinline__ void voxel_min_max(const VoxelImages &in, int nimg, long i, float &mn,
                                              float &mx) {
  mn = mx = in.img[0][i];
  for (int m = 1; m < nimg; ++m) {
    const float v = in.img[m][i];
    mn = v < mn ? v : mn;
    mx = v > mx ? v : mx;
  }
}

// range[0] / range[1]: order keys of the volume's smallest min and largest max
__global__ void k_median_range(const __grid_constant__ VoxelImages in, int nimg, long n,
                               unsigned *range) {
  __shared__ unsigned lo_s[8], hi_s[8];
  unsigned lo = 0xffffffffu, hi = 0u;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    float mn, mx;
    voxel_min_max(in, nimg, i, mn, mx);
    lo = min(lo, order_key(mn));
    hi = max(hi, order_key(mx));
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    lo_s[w] = lo;
    hi_s[w] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
      lo = min(lo, lo_s[k]);
      hi = max(hi, hi_s[k]);
    }
    atomicMin(&range[0], lo);
    atomicMax(&range[1], hi);
  }
}

__global__ void k_median_select(const __grid_constant__ VoxelImages in, int nimg, unsigned k,
                                long n, const unsigned *range, float *out, int *open) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float eps = fdiv(fsub(key_value(range[1]), key_value(range[0])), 10000.f);
  float gmin, gmax;
  voxel_min_max(in, nimg, i, gmin, gmax);
  float cmin = gmin, cmax = gmax, r = gmin;
  bool done = false;
  for (int iter = 0; !done; ++iter) {
    if (eps > fabsf(fsub(cmax, cmin))) {
      r = cmin;
      break;
    }
    // (curMin + curMax) / 2.0 stored as float: the float sum halved exactly
    const float p = fmul(fadd(cmin, cmax), 0.5f);
    unsigned idx = 0;
    float vp = gmin, vn = gmax;
    for (int m = 0; m < nimg; ++m) {
      const float v = in.img[m][i];
      if (v < p) {
        ++idx;
        if (v > vp) vp = v;
      } else if (v < vn) {
        vn = v;
      }
    }
    if (idx == k) {
      r = vn;
      done = true;
    } else if (idx - 1u == k) {
      r = vp;
      done = true;
    } else if (idx > k) {
      cmax = vp;
    } else if (idx < k) {
      cmin = vn;
    }
    if (!done && iter > nimg) {
      atomicExch(open, 1);
      r = cmin;
      break;
    }
  }
  out[i] = r;
}

}  // namespace

cudaError_t ldmm_voxel_median(const VoxelImages &in, int nimg, int k, long n, float *out,
                              unsigned *range, int *open, cudaStream_t s) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(range, 0xff, sizeof(unsigned), s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(range + 1, 0, sizeof(unsigned), s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(open, 0, sizeof(int), s)) != cudaSuccess) return e;
  int sms = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long blocks = std::min<long>((n + 255) / 256, 4L * sms);
  k_median_range<<<(unsigned)blocks, 256, 0, s>>>(in, nimg, n, range);
  k_median_select<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(in, nimg, (unsigned)k, n, range,
                                                             out, open);
  return cudaGetLastError();
}

namespace {
// alpha0 <- (1 - eps) alpha0 + (eps / sigma^2) alphaT, float, with
// 1 - eps formed in double as the reference's `Real vFac = 1.0 - StepSize()`
// (LDMMShootingIteratorCPU.cxx:287-297)
__global__ void k_shoot_alpha(float *__restrict__ a0, const float *__restrict__ aT,
                              const float *__restrict__ step, float sigma, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float eps = *step;
  const float vfac = __double2float_rn(1.0 - (double)eps);
  const float ufac = fdiv(eps, fmul(sigma, sigma));
  a0[i] = fadd(fmul(vfac, a0[i]), fmul(ufac, aT[i]));
}
}  // namespace

// The geodesic from I0 and the momentum alpha0 (LDMMGeodesicShootingCPU::
// ShootImage(I0, alpha0, T), LDMM/LDMMGeodesicShootingCPU.cxx:44-157; the
// shooting half of LDMMShootingIteratorCPU::Iterate, LDMMShootingIteratorCPU.
// cxx:199-262): v_0 = K(grad(I0) alpha0); for t = 1..T-1: phi0T =
// composeVH(v, phi0T) [PARTIAL_ZERO], alpha_t = splat(alpha0, phi0T), phiT0 =
// composeHVInv(phiT0, v) [PARTIAL_ID], I_t = I0(phiT0), v_t = K(grad(I_t)
// alpha_t); then the last step of both maps and the final image. The maps end
// in A[ca] (phi0T or the context's buffer) and B[cb], the image in c->J0.
// With record, each step energy <L v, v> (as <f, v>, k_force_vdot: no second
// transform) is added to the iteration's vector energy.
static cudaError_t shoot_geodesic(LdmmCtx *c, const float *I0, const float *alpha0, float *phi0T,
                                  float *phiT0, bool record, float *A[2], float *B[2], int &ca,
                                  int &cb, cudaStream_t s) {
  const Dims d = c->d;
  const long n = d.n();
  const int T = c->T;
  A[0] = phi0T;
  A[1] = c->hbuf;
  B[0] = phiT0;
  B[1] = c->hbuf + 3 * n;
  ca = cb = 0;
  auto comp = [&](float *base, int k) { return base + k * n; };
  float *v = c->u, *aT = c->S, *I = c->J0;
  const double spprod = c->sp.x * c->sp.y * c->sp.z;
  int vt = 0;  // velocities formed so far
  auto velocity = [&](const float *G) -> cudaError_t {
    AW_TRY(fluid_forward_force(c->plan, G, aT, 0, s));
    AW_TRY(fluid_solve(c->plan, 1, s));
    AW_TRY(fluid_inverse_store(c->plan, comp(v, 0), comp(v, 1), comp(v, 2), s));
    if (!record) return cudaSuccess;
    k_force_vdot<<<row_grid(d), kRowThreads, 0, s>>>(make_force(G, aT, 0, c->sp), v, 1.0f,
                                                      c->partials, d);
    AW_TRY(cudaGetLastError());
    k_record_energy<<<1, kRecThreads, 0, s>>>(c->partials, c->nparts, spprod, c->venergy,
                                              c->count, c->cap, 0, vt++ > 0);
    return cudaGetLastError();
  };
  auto advance_phi0T = [&]() -> cudaError_t {  // phi0T = composeVH(v, phi0T)
    const float *vv[3] = {comp(v, 0), comp(v, 1), comp(v, 2)};
    const float *hh[3] = {comp(A[ca], 0), comp(A[ca], 1), comp(A[ca], 2)};
    float *oo[3] = {comp(A[1 - ca], 0), comp(A[1 - ca], 1), comp(A[1 - ca], 2)};
    AW_TRY(launch_compose_vh(vv, hh, oo, d, c->sp, 1, BG_PARTIAL_ZERO, nullptr, 1.0f, s));
    ca = 1 - ca;
    return cudaSuccess;
  };
  auto advance_phiT0 = [&]() -> cudaError_t {  // phiT0 = composeHVInv(phiT0, v), I = I0(phiT0)
    k_forward_step<false><<<row_grid(d), kRowThreads, 0, s>>>(
        comp(B[cb], 0), comp(B[cb], 1), comp(B[cb], 2), comp(v, 0), comp(v, 1), comp(v, 2),
        comp(B[1 - cb], 0), comp(B[1 - cb], 1), comp(B[1 - cb], 2), I0, I, d, c->sp);
    cb = 1 - cb;
    return cudaGetLastError();
  };
  k_identity<<<row_grid(d), kRowThreads, 0, s>>>(comp(phi0T, 0), comp(phi0T, 1), comp(phi0T, 2), d);
  AW_TRY(cudaGetLastError());
  k_identity<<<row_grid(d), kRowThreads, 0, s>>>(comp(phiT0, 0), comp(phiT0, 1), comp(phiT0, 2), d);
  AW_TRY(cudaGetLastError());
  AW_TRY(cudaMemcpyAsync(aT, alpha0, sizeof(float) * n, cudaMemcpyDeviceToDevice, s));
  AW_TRY(velocity(I0));
  for (int t = 1; t < T; ++t) {
    AW_TRY(advance_phi0T());
    AW_TRY(splat(c->sw, alpha0, comp(A[ca], 0), comp(A[ca], 1), comp(A[ca], 2), aT, 0.0f, s));
    AW_TRY(advance_phiT0());
    AW_TRY(velocity(I));
  }
  AW_TRY(advance_phiT0());
  return advance_phi0T();
}

// LDMMShootingIteratorCPU::Iterate (LDMM/LDMMShootingIteratorCPU.cxx:
// 199-304): the geodesic, then alpha0 <- (1 - step) alpha0 + (step/sigma^2)
// splat(I_T - I1 by phiT0), the image energy of I_T - I1 and the vector
// energy recorded.
cudaError_t ldmm_shoot_iterate(LdmmCtx *c, const float *I0, const float *I1, float *alpha0,
                               float *phi0T, float *phiT0, cudaStream_t s) {
  const Dims d = c->d;
  const long n = d.n();
  float *A[2], *B[2];
  int ca, cb;
  auto comp = [&](float *base, int k) { return base + k * n; };
  AW_TRY(shoot_geodesic(c, I0, alpha0, phi0T, phiT0, true, A, B, ca, cb, s));
  float *aT = c->S, *I = c->J0;
  const double spprod = c->sp.x * c->sp.y * c->sp.z;
  k_residual<<<row_grid(d), kRowThreads, 0, s>>>(I, I1, c->diff, c->partials, d);
  AW_TRY(cudaGetLastError());
  AW_TRY(splat(c->sw, c->diff, comp(B[cb], 0), comp(B[cb], 1), comp(B[cb], 2), aT, 0.0f, s));
  k_shoot_alpha<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(alpha0, aT, c->step, c->sigma, n);
  AW_TRY(cudaGetLastError());
  k_record_energy<<<1, kRecThreads, 0, s>>>(c->partials, c->nparts, spprod, c->energy,
                                            c->count, c->cap);
  AW_TRY(cudaGetLastError());
  // the maps end in the caller's buffers
  if (ca) AW_TRY(cudaMemcpyAsync(phi0T, A[1], sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, s));
  if (cb) AW_TRY(cudaMemcpyAsync(phiT0, B[1], sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, s));
  return cudaSuccess;
}

// LDMMGeodesicShootingGPU::ShootImage(I0, alpha0, T): the geodesic alone;
// the maps Phi0To1 / Phi1To0 in the caller's buffers, the final image
// (GetFinalImage) in img; no energy is recorded
cudaError_t ldmm_geodesic_shoot(LdmmCtx *c, const float *I0, const float *alpha0, float *phi0T,
                                float *phiT0, float *img, cudaStream_t s) {
  const long n = c->d.n();
  float *A[2], *B[2];
  int ca, cb;
  AW_TRY(shoot_geodesic(c, I0, alpha0, phi0T, phiT0, false, A, B, ca, cb, s));
  if (ca) AW_TRY(cudaMemcpyAsync(phi0T, A[1], sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, s));
  if (cb) AW_TRY(cudaMemcpyAsync(phiT0, B[1], sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, s));
  return cudaMemcpyAsync(img, c->J0, sizeof(float) * n, cudaMemcpyDeviceToDevice, s);
}

namespace {

// D phiT0 = identity: rows x | y | z, each a vector field [3][N]
__global__ void k_dphi_identity(float *__restrict__ dp, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) dp[(long)(3 * r + c) * n + i] = r == c ? 1.0f : 0.0f;
}

// row += g (Array3D<Vector3D<Real>>::pointwiseAdd), 3N floats
__global__ void k_add3(float *__restrict__ row, const float *__restrict__ g, long n3) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n3) row[i] = fadd(row[i], g[i]);
}

// f = |D phiT0| (D phiT0)^T (L v0)(phiT0): the compose of L v0 at phiT0
// (HField3DUtils::compose, PARTIAL_ZERO), the transposed product and the
// determinant in the reference's float order (LDMMVelShootingIteratorCPU.
// cxx:276-320)
__global__ void __launch_bounds__(kRowThreads)
    k_velshoot_force(const float *__restrict__ dp, const float *__restrict__ lv0,
                     const float *__restrict__ hx, const float *__restrict__ hy,
                     const float *__restrict__ hz, float *__restrict__ f, Dims d) {
  Voxel v;
  if (!voxel_of(d, v)) return;
  const long n = d.n(), i = v.i;
  float lx, ly, lz;
  trilerp_vector<false>(lv0, lv0 + n, lv0 + 2 * n, d, hx[i], hy[i], hz[i], BG_PARTIAL_ZERO, 1.0f,
                        lx, ly, lz);
  const float xx = dp[i], xy = dp[n + i], xz = dp[2 * n + i];
  const float yx = dp[3 * n + i], yy = dp[4 * n + i], yz = dp[5 * n + i];
  const float zx = dp[6 * n + i], zy = dp[7 * n + i], zz = dp[8 * n + i];
  const float fx = fadd(fadd(fmul(xx, lx), fmul(yx, ly)), fmul(zx, lz));
  const float fy = fadd(fadd(fmul(xy, lx), fmul(yy, ly)), fmul(zy, lz));
  const float fz = fadd(fadd(fmul(xz, lx), fmul(yz, ly)), fmul(zz, lz));
  const float t1 = fmul(xx, fsub(fmul(yy, zz), fmul(yz, zy)));
  const float t2 = fmul(xy, fsub(fmul(yx, zz), fmul(yz, zx)));
  const float t3 = fmul(xz, fsub(fmul(yx, zy), fmul(yy, zx)));
  const float det = fadd(fsub(t1, t2), t3);
  f[i] = fmul(fx, det);
  f[n + i] = fmul(fy, det);
  f[2 * n + i] = fmul(fz, det);
}

}  // namespace

int ldmm_velshoot_prepare(LdmmCtx *c) {
  if (c->vsBuf) return 0;
  if (cudaMalloc(&c->vsBuf, sizeof(float) * 15 * (size_t)c->d.n()) != cudaSuccess) {
    cudaGetLastError();
    c->vsBuf = nullptr;
    return 3;
  }
  return 0;
}

// LDMMVelShootingIteratorCPU::Iterate (LDMM/LDMMVelShootingIteratorCPU.cxx:
// 186-344): the geodesic in velocity form from v0 — for t = 0..T-1 the step
// energy <L v_t, v_t>, phiT0 = composeHVInv(phiT0, v_t) [PARTIAL_ID], phi0T =
// composeVH(v_t, phi0T) [PARTIAL_ZERO], and before the next step D phiT0 +=
// grad(v_t,c(phiT0)) per component c and v_{t+1} = K(|D phiT0| (D phiT0)^T
// (L v0)(phiT0)) — then the residual I0(phiT0) - I1, its energy (recorded in
// the step-size pass too, as the reference adds it), its splat by phiT0 and
// K(grad(I0) splat), and the update of v0 (or the step). The step energies
// after the first are formed as <f_{t-1}, v_t> with v_t = K f_{t-1}: no
// further transform.
cudaError_t ldmm_velshoot_iterate(LdmmCtx *c, const float *I0, const float *I1, float *v0,
                                  float *phi0T, float *phiT0, int update_step, cudaStream_t s) {
  const Dims d = c->d;
  const long n = d.n();
  const int T = c->T;
  auto comp = [&](float *base, int k) { return base + k * n; };
  float *A[2] = {phi0T, c->hbuf}, *B[2] = {phiT0, c->hbuf + 3 * n};
  int ca = 0, cb = 0;
  float *vt = c->u, *lv0 = c->vsBuf, *dp = lv0 + 3 * n, *f = dp + 9 * n;
  float *img = c->S, *g = f;  // g (a gradient) and f are never live together
  const double spprod = c->sp.x * c->sp.y * c->sp.z;
  const unsigned flat = (unsigned)((n + 255) / 256), flat3 = (unsigned)((3 * n + 255) / 256);
  auto record_vec = [&](const float *a, const float *b, int t) -> cudaError_t {
    k_field_dot<<<row_grid(d), kRowThreads, 0, s>>>(a, b, c->partials, d);
    AW_TRY(cudaGetLastError());
    k_record_energy<<<1, kRecThreads, 0, s>>>(c->partials, c->nparts, spprod, c->venergy,
                                              c->count, c->cap, 0, t > 0 ? 1 : 0, 0);
    AW_TRY(cudaGetLastError());
    k_record_energy<<<1, kRecThreads, 0, s>>>(c->partials, c->nparts, spprod, c->vstep + t,
                                              c->zero, 1, 0, 0, 0);
    return cudaGetLastError();
  };
  k_identity<<<row_grid(d), kRowThreads, 0, s>>>(comp(phi0T, 0), comp(phi0T, 1), comp(phi0T, 2), d);
  AW_TRY(cudaGetLastError());
  k_identity<<<row_grid(d), kRowThreads, 0, s>>>(comp(phiT0, 0), comp(phiT0, 1), comp(phiT0, 2), d);
  AW_TRY(cudaGetLastError());
  AW_TRY(cudaMemcpyAsync(vt, v0, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, s));
  k_dphi_identity<<<flat, 256, 0, s>>>(dp, n);
  AW_TRY(cudaGetLastError());
  AW_TRY(fluid_forward_field(c->plan, comp(v0, 0), comp(v0, 1), comp(v0, 2), s));
  AW_TRY(fluid_solve(c->plan, 0, s));
  AW_TRY(fluid_inverse_store(c->plan, comp(lv0, 0), comp(lv0, 1), comp(lv0, 2), s));
  for (int t = 0; t < T; ++t) {
    AW_TRY(t == 0 ? record_vec(lv0, vt, 0) : record_vec(f, vt, t));
    {
      const float *gg[3] = {comp(B[cb], 0), comp(B[cb], 1), comp(B[cb], 2)};
      const float *vv[3] = {comp(vt, 0), comp(vt, 1), comp(vt, 2)};
      float *oo[3] = {comp(B[1 - cb], 0), comp(B[1 - cb], 1), comp(B[1 - cb], 2)};
      AW_TRY(launch_compose_hv(gg, vv, oo, d, c->sp, -1, BG_PARTIAL_ID, nullptr, 1.0f, s));
      cb = 1 - cb;
    }
    {
      const float *vv[3] = {comp(vt, 0), comp(vt, 1), comp(vt, 2)};
      const float *hh[3] = {comp(A[ca], 0), comp(A[ca], 1), comp(A[ca], 2)};
      float *oo[3] = {comp(A[1 - ca], 0), comp(A[1 - ca], 1), comp(A[1 - ca], 2)};
      AW_TRY(launch_compose_vh(vv, hh, oo, d, c->sp, 1, BG_PARTIAL_ZERO, nullptr, 1.0f, s));
      ca = 1 - ca;
    }
    if (t == T - 1) break;
    for (int r = 0; r < 3; ++r) {
      AW_TRY(launch_apply(comp(vt, r), comp(B[cb], 0), comp(B[cb], 1), comp(B[cb], 2), img, d,
                          0.0f, s));
      AW_TRY(launch_gradient(img, comp(g, 0), comp(g, 1), comp(g, 2), d, c->sp, 0, s));
      k_add3<<<flat3, 256, 0, s>>>(dp + (long)3 * r * n, g, 3 * n);
      AW_TRY(cudaGetLastError());
    }
    k_velshoot_force<<<row_grid(d), kRowThreads, 0, s>>>(dp, lv0, comp(B[cb], 0), comp(B[cb], 1),
                                                         comp(B[cb], 2), f, d);
    AW_TRY(cudaGetLastError());
    AW_TRY(fluid_forward_field(c->plan, comp(f, 0), comp(f, 1), comp(f, 2), s));
    AW_TRY(fluid_solve(c->plan, 1, s));
    AW_TRY(fluid_inverse_store(c->plan, comp(vt, 0), comp(vt, 1), comp(vt, 2), s));
  }
  // residual, image energy, its splat, K(grad(I0) splat), the update
  AW_TRY(launch_apply(I0, comp(B[cb], 0), comp(B[cb], 1), comp(B[cb], 2), img, d, 0.0f, s));
  k_residual<<<row_grid(d), kRowThreads, 0, s>>>(img, I1, c->diff, c->partials, d);
  AW_TRY(cudaGetLastError());
  k_record_energy<<<1, kRecThreads, 0, s>>>(c->partials, c->nparts, spprod, c->energy, c->count,
                                            c->cap);
  AW_TRY(cudaGetLastError());
  AW_TRY(splat(c->sw, c->diff, comp(B[cb], 0), comp(B[cb], 1), comp(B[cb], 2), img, 0.0f, s));
  AW_TRY(fluid_forward_force(c->plan, I0, img, 0, s));
  AW_TRY(fluid_solve(c->plan, 1, s));
  if (update_step) {
    AW_TRY(cudaMemsetAsync(c->maxbits, 0, sizeof(unsigned), s));
    AW_TRY(fluid_inverse_store(c->plan, comp(f, 0), comp(f, 1), comp(f, 2), s));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->plan.device);
    k_max_disp<<<sms * 4, 256, 0, s>>>(comp(v0, 0), comp(v0, 1), comp(v0, 2), comp(f, 0),
                                       comp(f, 1), comp(f, 2), n, c->sigma, c->maxbits);
    AW_TRY(cudaGetLastError());
    k_step_from_max<<<1, 1, 0, s>>>(c->maxbits, c->max_pert, c->step);
    AW_TRY(cudaGetLastError());
  } else {
    AW_TRY(fluid_inverse_axpby(c->plan, comp(v0, 0), comp(v0, 1), comp(v0, 2), c->step, c->sigma,
                               s));
  }
  if (ca) AW_TRY(cudaMemcpyAsync(phi0T, A[1], sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, s));
  if (cb) AW_TRY(cudaMemcpyAsync(phiT0, B[1], sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, s));
  return cudaSuccess;
}

int ldmm_adshoot_prepare(LdmmCtx *c) {
  if (c->adV) return 0;
  const size_t n = (size_t)c->d.n(), T = (size_t)c->T;
  const size_t sort_bytes = (splat_scratch_bytes(c->d) + 255) & ~size_t(255);
  if (c->T + 1 > kMaxAdSorts) return 3;
  if (cudaMalloc(&c->adV, sizeof(float) * T * 3 * n) != cudaSuccess ||
      cudaMalloc(&c->adP, sizeof(float) * 2 * (T + 1) * 3 * n) != cudaSuccess ||
      cudaMalloc(&c->adA, sizeof(float) * T * n) != cudaSuccess ||
      cudaMalloc(&c->adI, sizeof(float) * 6 * n) != cudaSuccess ||
      cudaMalloc(&c->adSortMem, sort_bytes * (T + 1)) != cudaSuccess) {
    cudaGetLastError();
    void *ptrs[] = {c->adV, c->adP, c->adA, c->adI, c->adSortMem};
    for (void *p : ptrs)
      if (p) cudaFree(p);
    c->adV = c->adP = c->adA = c->adI = nullptr;
    c->adSortMem = nullptr;
    return 3;
  }
  for (size_t k = 0; k <= T; ++k)
    splat_work_bind(&c->adSort[k], c->d, static_cast<char *>(c->adSortMem) + k * sort_bytes);
  return 0;
}

// the momentum shooting needs no device memory beyond the handle's own
int ldmm_shoot_prepare(LdmmCtx *) { return 0; }

// LDMMAdShootingIteratorCPU::Iterate (LDMM/LDMMAdShootingIteratorCPU.cxx:
// 237-323) and backwardAdIntegration (:325-431).
//
//   shoot     v_0 = -K(grad(I0) alpha0); for t = 1..T-1:
//               phi0T_t = composeVH(v_{t-1}, phi0T_{t-1})   [PARTIAL_ZERO]
//               alpha_t = splat(alpha0, phi0T_t)
//               phiT0_t = composeHVInv(phiT0_{t-1}, v_{t-1}) [PARTIAL_ID],
//               I_t = I0(phiT0_t)                 (one fused kernel)
//               v_t = -K(grad(I_t) alpha_t)       (force fused into the FFT)
//             then the maps, I_T and alpha_T at t = T
//   energies  image sp^3 sum (I_T - I1)^2, vector <L v0, v0>
//   adjoint   IHat = (I1 - I_T)/sigma^2, ITilde = splat(IHat, phiT0_T),
//             alphaTilde = 0; for i = T-1..0 at t = i+1:
//               alphaHat = alphaTilde(phiT0_t), IHat = splat(ITilde, phi0T_t)
//               vhat = K(grad(alphaHat) alpha_t - grad(I_t) IHat)
//               alphaTilde -= (grad(I_t) . vhat)(phi0T_t)
//               ITilde += splat(div(alpha_t vhat), phiT0_t)
//   update    alpha0 -= step (-(grad(I0) . v_0) - alphaTilde)
//
// The reference recomposes phi0T_t / phiT0_t from the identity at every
// backward step (O(T^2) compositions) and recomputes I_t and alpha_t; the
// same operations in the same order produce the same values, so here the
// shooting keeps every map, I_t and alpha_t resident in HBM and the
// backward sweep reads them back. The bucket sort of each phi0T_t (and of
// phiT0_T) is kept too: the backward sweep splats by those maps again and
// needs only the ordered sums.
cudaError_t ldmm_adshoot_iterate(LdmmCtx *c, const float *I0, const float *I1, float *alpha0,
                                 float *phi0T, float *phiT0, cudaStream_t s) {
  if (!c->adV) return cudaErrorNotReady;
  const Dims d = c->d;
  const long n = d.n();
  const int T = c->T;
  const GradDiv g = grad_div(c->sp);
  const dim3 grid = row_grid(d);
  const unsigned flat = (unsigned)((n + 255) / 256);
  auto V = [&](int t) { return c->adV + (long)t * 3 * n; };
  auto P0 = [&](int t) { return c->adP + (long)t * 3 * n; };
  auto P1 = [&](int t) { return c->adP + (long)(T + 1 + t) * 3 * n; };
  auto A = [&](int t) { return c->adA + (long)(t - 1) * n; };  // alpha_t, t >= 1
  auto I = [&](int t) { return c->J0 + (long)(t - 1) * n; };   // I_t, t >= 1
  float *aHat = c->adI, *IHat = aHat + n, *aTil = IHat + n, *ITil = aTil + n, *s1 = ITil + n,
        *s2 = s1 + n;
  auto comp = [&](float *base, int k) { return base + k * n; };
  auto velocity = [&](const float *G, const float *At, int t) -> cudaError_t {
    AW_TRY(fluid_forward_force(c->plan, G, At, 0, s));
    AW_TRY(fluid_solve(c->plan, 1, s));
    return fluid_inverse_store_neg(c->plan, comp(V(t), 0), comp(V(t), 1), comp(V(t), 2), s);
  };
  auto advance = [&](int t) -> cudaError_t {  // maps, I_t and alpha_t at t from t-1
    const float *vv[3] = {comp(V(t - 1), 0), comp(V(t - 1), 1), comp(V(t - 1), 2)};
    const float *hh[3] = {comp(P0(t - 1), 0), comp(P0(t - 1), 1), comp(P0(t - 1), 2)};
    float *oo[3] = {comp(P0(t), 0), comp(P0(t), 1), comp(P0(t), 2)};
    AW_TRY(launch_compose_vh(vv, hh, oo, d, c->sp, 1, BG_PARTIAL_ZERO, nullptr, 1.0f, s));
    AW_TRY(splat_sort(c->adSort[t], oo[0], oo[1], oo[2], s));
    AW_TRY(splat_gather(c->adSort[t], alpha0, oo[0], oo[1], oo[2], A(t), 0.0f, s));
    k_forward_step<false><<<grid, kRowThreads, 0, s>>>(
        comp(P1(t - 1), 0), comp(P1(t - 1), 1), comp(P1(t - 1), 2), vv[0], vv[1], vv[2],
        comp(P1(t), 0), comp(P1(t), 1), comp(P1(t), 2), I0, I(t), d, c->sp);
    return cudaGetLastError();
  };

  // shooting
  k_identity<<<grid, kRowThreads, 0, s>>>(comp(P0(0), 0), comp(P0(0), 1), comp(P0(0), 2), d);
  AW_TRY(cudaGetLastError());
  k_identity<<<grid, kRowThreads, 0, s>>>(comp(P1(0), 0), comp(P1(0), 1), comp(P1(0), 2), d);
  AW_TRY(cudaGetLastError());
  AW_TRY(velocity(I0, alpha0, 0));
  for (int t = 1; t < T; ++t) {
    AW_TRY(advance(t));
    AW_TRY(velocity(I(t), A(t), t));
  }
  AW_TRY(advance(T));

  // energies: <L v0, v0> (recorded without advancing the count), then the
  // image term; v0 = -K f0 with f0 = grad(I0) alpha0, so L v0 = -f0 and the
  // product is formed from the force again (k_force_vdot), no second transform
  const double spprod = c->sp.x * c->sp.y * c->sp.z;
  k_force_vdot<<<grid, kRowThreads, 0, s>>>(make_force(I0, alpha0, 0, c->sp), V(0), -1.0f,
                                             c->partials, d);
  AW_TRY(cudaGetLastError());
  k_record_energy<<<1, kRecThreads, 0, s>>>(c->partials, c->nparts, spprod, c->venergy,
                                            c->count, c->cap, 0);
  AW_TRY(cudaGetLastError());
  const float inv = 1.0f / (c->sigma * c->sigma);
  k_ad_residual<<<grid, kRowThreads, 0, s>>>(I(T), I1, inv, IHat, c->partials, d);
  AW_TRY(cudaGetLastError());
  k_record_energy<<<1, kRecThreads, 0, s>>>(c->partials, c->nparts, spprod, c->energy,
                                            c->count, c->cap, 1);
  AW_TRY(cudaGetLastError());

  // backward integration of the adjoint equations
  AW_TRY(splat_sort(c->adSort[0], comp(P1(T), 0), comp(P1(T), 1), comp(P1(T), 2), s));
  AW_TRY(splat_gather(c->adSort[0], IHat, comp(P1(T), 0), comp(P1(T), 1), comp(P1(T), 2), ITil,
                      0.0f, s));
  AW_TRY(cudaMemsetAsync(aTil, 0, sizeof(float) * n, s));
  for (int i = T - 1; i >= 0; --i) {
    const int t = i + 1;
    float *p0[3] = {comp(P0(t), 0), comp(P0(t), 1), comp(P0(t), 2)};
    float *p1[3] = {comp(P1(t), 0), comp(P1(t), 1), comp(P1(t), 2)};
    k_ad_pull<false><<<grid, kRowThreads, 0, s>>>(aTil, p1[0], p1[1], p1[2], aHat, d);
    AW_TRY(cudaGetLastError());
    AW_TRY(splat_gather(c->adSort[t], ITil, p0[0], p0[1], p0[2], IHat, 0.0f, s));
    k_ad_force<<<grid, kRowThreads, 0, s>>>(aHat, A(t), I(t), IHat, comp(c->u, 0), comp(c->u, 1),
                                            comp(c->u, 2), d, g);
    AW_TRY(cudaGetLastError());
    AW_TRY(fluid_forward_field(c->plan, comp(c->u, 0), comp(c->u, 1), comp(c->u, 2), s));
    AW_TRY(fluid_solve(c->plan, 1, s));
    AW_TRY(fluid_inverse_store(c->plan, comp(c->u, 0), comp(c->u, 1), comp(c->u, 2), s));
    k_ad_dot_div<<<grid, kRowThreads, 0, s>>>(I(t), comp(c->u, 0), comp(c->u, 1), comp(c->u, 2),
                                              A(t), s1, s2, d, g);
    AW_TRY(cudaGetLastError());
    k_ad_pull<true><<<grid, kRowThreads, 0, s>>>(s1, p0[0], p0[1], p0[2], aTil, d);
    AW_TRY(cudaGetLastError());
    if (t == T)
      AW_TRY(splat_gather(c->adSort[0], s2, p1[0], p1[1], p1[2], s1, 0.0f, s));
    else
      AW_TRY(splat(c->sw, s2, p1[0], p1[1], p1[2], s1, 0.0f, s));
    k_ad_add<<<flat, 256, 0, s>>>(ITil, s1, n);
    AW_TRY(cudaGetLastError());
  }
  k_ad_alpha<<<grid, kRowThreads, 0, s>>>(I0, V(0), aTil, c->step, alpha0, d, g);
  AW_TRY(cudaGetLastError());
  // the data's maps end at t_1, where the reference's backward sweep leaves them
  AW_TRY(cudaMemcpyAsync(phi0T, P0(1), sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, s));
  return cudaMemcpyAsync(phiT0, P1(1), sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, s);
}

// finalUpdatePhi0T / finalUpdatePhiT0 (LDMMAdShootingIteratorCPU.cxx:433-453)
// compose the maps from the identity through the last Iterate's velocities:
// the maps at t = T that Iterate kept
cudaError_t ldmm_adshoot_final_maps(LdmmCtx *c, float *phi0T, float *phiT0, cudaStream_t s) {
  if (!c->adV) return cudaErrorNotReady;
  const long n = c->d.n();
  const int T = c->T;
  AW_TRY(cudaMemcpyAsync(phi0T, c->adP + (long)T * 3 * n, sizeof(float) * 3 * n,
                         cudaMemcpyDeviceToDevice, s));
  return cudaMemcpyAsync(phiT0, c->adP + (long)(2 * T + 1) * 3 * n, sizeof(float) * 3 * n,
                         cudaMemcpyDeviceToDevice, s);
}

int ldmm_set_orig(LdmmCtx *c, int on) {
  c->orig = on ? 1 : 0;
  if (c->orig && !c->JT) {
    const size_t bytes = sizeof(float) * (size_t)c->T * c->d.n();
    if (cudaMalloc(&c->JT, bytes) != cudaSuccess || cudaMalloc(&c->JD, bytes) != cudaSuccess)
      return 3;
  }
  return 0;
}

// LDMMIteratorCPU::IterateOrig (LDMM/LDMMIteratorCPU.cxx:377-527)
cudaError_t ldmm_iterate_orig(LdmmCtx *c, const float *I0, const float *I1, float *v,
                              int update_step, cudaStream_t s) {
  const Dims d = c->d;
  const long n = d.n();
  const int T = c->T;
  float *H[2] = {c->hbuf, c->hbuf + 3 * n};
  auto comp = [&](float *base, int k) { return base + k * n; };
  const DivD a2 = make_div(2.0 * c->sp.x), b2 = make_div(2.0 * c->sp.y), e2 = make_div(2.0 * c->sp.z);
  const DivD a1 = make_div(c->sp.x), b1 = make_div(c->sp.y), e1 = make_div(c->sp.z);
  // backward sweep: h <- h(x + v_t/sp), JT_t = I1(h), Jacobian transport
  k_identity<<<row_grid(d), kRowThreads, 0, s>>>(comp(H[0], 0), comp(H[0], 1), comp(H[0], 2), d);
  AW_TRY(cudaGetLastError());
  int cur = 0;
  for (int t = T - 1; t >= 0; --t) {
    float *vt = v + (long)t * 3 * n;
    k_forward_step<true><<<row_grid(d), kRowThreads, 0, s>>>(
        comp(H[cur], 0), comp(H[cur], 1), comp(H[cur], 2), comp(vt, 0), comp(vt, 1), comp(vt, 2),
        comp(H[1 - cur], 0), comp(H[1 - cur], 1), comp(H[1 - cur], 2), I1, c->JT + (long)t * n,
        d, c->sp);
    AW_TRY(cudaGetLastError());
    cur = 1 - cur;
    k_jacdet<<<row_grid(d), kRowThreads, 0, s>>>(comp(vt, 0), comp(vt, 1), comp(vt, 2),
                                                 t == T - 1 ? nullptr : c->JD + (long)(t + 1) * n,
                                                 c->JD + (long)t * n, d, c->sp, a2, b2, e2, a1, b1,
                                                 e1);
    AW_TRY(cudaGetLastError());
  }
  if (update_step) AW_TRY(cudaMemsetAsync(c->maxbits, 0, sizeof(unsigned), s));
  // forward sweep: S = I0(h), force grad(S) * (S - JT_t) * JacDet_t, K, update,
  // h <- h(x - v_t/sp) with the updated v_t, and S for the next t
  k_identity<<<row_grid(d), kRowThreads, 0, s>>>(comp(H[0], 0), comp(H[0], 1), comp(H[0], 2), d);
  AW_TRY(cudaGetLastError());
  cur = 0;
  float *Sb = c->S;
  for (int t = 0; t < T; ++t) {
    float *vt = v + (long)t * 3 * n;
    const float *Sg = t == 0 ? I0 : Sb;
    AW_TRY(fluid_forward_force_jac(c->plan, Sg, c->JT + (long)t * n, c->JD + (long)t * n, s));
    AW_TRY(fluid_solve(c->plan, 1, s));
    if (update_step) {
      AW_TRY(fluid_inverse_store(c->plan, comp(c->u, 0), comp(c->u, 1), comp(c->u, 2), s));
      int sms = 148;
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->plan.device);
      k_max_disp<<<sms * 4, 256, 0, s>>>(comp(vt, 0), comp(vt, 1), comp(vt, 2), comp(c->u, 0),
                                         comp(c->u, 1), comp(c->u, 2), n, c->sigma, c->maxbits);
      AW_TRY(cudaGetLastError());
    } else {
      AW_TRY(fluid_inverse_axpby(c->plan, comp(vt, 0), comp(vt, 1), comp(vt, 2), c->step,
                                 c->sigma, s));
    }
    k_forward_step<false><<<row_grid(d), kRowThreads, 0, s>>>(
        comp(H[cur], 0), comp(H[cur], 1), comp(H[cur], 2), comp(vt, 0), comp(vt, 1), comp(vt, 2),
        comp(H[1 - cur], 0), comp(H[1 - cur], 1), comp(H[1 - cur], 2), I0, Sb, d, c->sp);
    AW_TRY(cudaGetLastError());
    cur = 1 - cur;
    // the image energy is recorded (and the count advanced) after the sweep
    if (c->vec_energy && !update_step) AW_TRY(vec_step_energy(c, vt, t, t == 0, 0, s));
  }
  if (update_step) {
    k_step_from_max<<<1, 1, 0, s>>>(c->maxbits, c->max_pert, c->step);
    return cudaGetLastError();
  }
  // image energy of the updated path: sp^3 * sum (I0(h) - I1)^2
  k_residual<<<row_grid(d), kRowThreads, 0, s>>>(Sb, I1, c->diff, c->partials, d);
  AW_TRY(cudaGetLastError());
  const double spprod = c->sp.x * c->sp.y * c->sp.z;
  k_record_energy<<<1, kRecThreads, 0, s>>>(c->partials, c->nparts, spprod, c->energy,
                                            c->count, c->cap);
  return cudaGetLastError();
}

}  // namespace aw
