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
// (composeHVInv + apply, LDMMIteratorCPU.cxx:549-554)
__global__ void __launch_bounds__(kRowThreads)
    k_forward_step(const float *__restrict__ hx, const float *__restrict__ hy,
                   const float *__restrict__ hz, const float *__restrict__ vx,
                   const float *__restrict__ vy, const float *__restrict__ vz,
                   float *__restrict__ ox, float *__restrict__ oy, float *__restrict__ oz,
                   const float *__restrict__ I0, float *__restrict__ J, Dims d, Spacing sp) {
  Voxel vox;
  if (!voxel_of(d, vox)) return;
  const long i = vox.i;
  const float px = fsub(__int2float_rn(vox.x), fdiv(vx[i], (float)sp.x));
  const float py = fsub(__int2float_rn(vox.y), fdiv(vy[i], (float)sp.y));
  const float pz = fsub(__int2float_rn(vox.z), fdiv(vz[i], (float)sp.z));
  float a, b, c;
  trilerp_vector(hx, hy, hz, d, px, py, pz, BG_PARTIAL_ID, 1.0f, a, b, c);
  ox[i] = a;
  oy[i] = b;
  oz[i] = c;
  J[i] = trilerp_scalar(I0, d, (double)a, (double)b, (double)c, 0.0f);
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

__global__ void __launch_bounds__(256)
    k_record_energy(const double *__restrict__ partials, int nparts, double scale,
                    double *__restrict__ energy, int *__restrict__ count, int cap) {
  double t = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) t += partials[i];
  __shared__ double ws[8];
  t = warp_sum(t);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < 8; ++w) s += ws[w];
    const int k = *count;
    energy[k % cap] = s * scale;
    *count = k + 1;
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
  if (cudaMalloc(&c->scalars, 64) != cudaSuccess) return 3;
  cudaMemset(c->scalars, 0, 64);
  c->step = reinterpret_cast<float *>(c->scalars);
  c->count = reinterpret_cast<int *>(c->scalars + 4);
  c->maxbits = reinterpret_cast<unsigned *>(c->scalars + 8);
  splat_work_bind(&c->sw, c->d, c->splat_scratch);
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

void ldmm_destroy(LdmmCtx *c) {
  fluid_plan_destroy(&c->plan);
  void *ptrs[] = {c->J0, c->hbuf, c->diff, c->S, c->u, c->splat_scratch, c->partials, c->energy,
                  c->scalars};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  std::memset(c, 0, sizeof(*c));
}

cudaError_t ldmm_iterate(LdmmCtx *c, const float *I0, const float *I1, float *v, int update_step,
                         cudaStream_t s) {
  const Dims d = c->d;
  const long n = d.n();
  const int T = c->T;
  float *H[2] = {c->hbuf, c->hbuf + 3 * n};
  auto comp = [&](float *base, int k) { return base + k * n; };
  // forward integration
  k_identity<<<row_grid(d), kRowThreads, 0, s>>>(comp(H[0], 0), comp(H[0], 1), comp(H[0], 2), d);
  AW_TRY(cudaGetLastError());
  int cur = 0;
  for (int i = 0; i < T; ++i) {
    float *vi = v + (long)i * 3 * n;
    k_forward_step<<<row_grid(d), kRowThreads, 0, s>>>(
        comp(H[cur], 0), comp(H[cur], 1), comp(H[cur], 2), comp(vi, 0), comp(vi, 1), comp(vi, 2),
        comp(H[1 - cur], 0), comp(H[1 - cur], 1), comp(H[1 - cur], 2), I0, c->J0 + (long)i * n,
        d, c->sp);
    AW_TRY(cudaGetLastError());
    cur = 1 - cur;
  }
  k_residual<<<row_grid(d), kRowThreads, 0, s>>>(c->J0 + (long)(T - 1) * n, I1, c->diff,
                                                 c->partials, d);
  AW_TRY(cudaGetLastError());
  if (!update_step) {
    const double spprod = c->sp.x * c->sp.y * c->sp.z;
    k_record_energy<<<1, 256, 0, s>>>(c->partials, c->nparts, spprod, c->energy, c->count,
                                      c->cap);
    AW_TRY(cudaGetLastError());
  } else {
    AW_TRY(cudaMemsetAsync(c->maxbits, 0, sizeof(unsigned), s));
  }
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
    }
  }
  if (update_step) {
    k_step_from_max<<<1, 1, 0, s>>>(c->maxbits, c->max_pert, c->step);
    AW_TRY(cudaGetLastError());
  }
  return cudaSuccess;
}

}  // namespace aw
