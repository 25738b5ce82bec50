// ldmm.cuh — device state of the LDMM relaxation iterator (ldmm.cu).
#pragma once

#include "fluid.cuh"
#include "splat.cuh"

namespace aw {

// time steps whose splat sorts the adjoint shooting keeps (T + 1 sets)
constexpr int kMaxAdSorts = 65;

struct LdmmCtx {
  FluidPlan plan;
  Dims d;
  Spacing sp;
  int T;
  float sigma;
  float max_pert;
  float *J0;        // T x N: I0 deformed to each time point
  float *hbuf;      // 2 x 3N ping-pong deformation
  float *diff;      // N: J0_{T-1} - I1
  float *S;         // N: splatted residual
  float *u;         // 3N: K f when the step size is being computed
  void *splat_scratch;
  SplatWork sw;
  double *partials;
  int nparts;
  char *scalars;    // step | count | maxbits
  float *step;
  int *count;
  unsigned *maxbits;
  double *energy;   // image-energy history ring
  int cap;
  int orig;         // IterateOrig (Jacobian path) instead of IterateNew
  int vec_energy;   // IterateNew / IterateOrig also record sum_t <L v_t, v_t>
  double *vstep;    // T: <L v_t, v_t> sp^3 of each t, of the last such iteration
  float *vsBuf;     // velocity shooting (ldmm_velshoot_prepare): L v0 3N | D phiT0 9N | f 3N
  int *zero;        // a device int that stays 0 (index of one-slot records)
  float *JT;        // T x N: I1 pulled back to each time point (IterateOrig)
  float *JD;        // T x N: transported Jacobian determinants (IterateOrig)
  // adjoint shooting (allocated by ldmm_adshoot_prepare)
  float *adV;       // T x 3N: the shot velocities v_0 .. v_{T-1}
  float *adP;       // 2 x (T+1) x 3N: phi0T then phiT0 at t = 0 .. T
  float *adA;       // T x N: alpha_t = splat(alpha0, phi0T_t), t = 1 .. T
  float *adI;       // 6N: alphaHat, IHat, alphaTilde, ITilde and two scratch images
  double *venergy;  // vector-energy history ring, indexed like energy
  void *adSortMem;  // T + 1 splat scratch sets
  SplatWork adSort[kMaxAdSorts];  // the sorts by phi0T_t (t = 1..T) and by phiT0_T (slot 0)
};

int ldmm_create(LdmmCtx *c, int nx, int ny, int nz, double spx, double spy, double spz,
                float alpha, float beta, float gamma, int T, float sigma, float max_pert);
void ldmm_destroy(LdmmCtx *c);
// LDMMIteratorCPU's UseOrigGradientCalc: 1 selects IterateOrig (the
// reference's default), 0 IterateNew; allocates the IterateOrig buffers
int ldmm_set_orig(LdmmCtx *c, int on);
cudaError_t ldmm_i1_at_0(LdmmCtx *c, const float *I1, const float *v, float *img, float *jd,
                         cudaStream_t s);
cudaError_t ldmm_atlas_accumulate(float *acc, float *jsum, const float *img, const float *jd,
                                  float w, long n, cudaStream_t s);
cudaError_t ldmm_atlas_normalize(float *acc, const float *jsum, long n, cudaStream_t s);
// the per-voxel k-th smallest value over up to kVoxelMedianMaxImages images
// by the reference's bisection (MedianCalculator::Select); range: 2 unsigned
// and open: 1 int of device scratch; *open = 1 when a voxel did not converge
constexpr int kVoxelMedianMaxImages = 256;
struct VoxelImages {
  const float *img[kVoxelMedianMaxImages];
};
cudaError_t ldmm_voxel_median(const VoxelImages &in, int nimg, int k, long n, float *out,
                              unsigned *range, int *open, cudaStream_t s);
// the momentum shooting's scratch (returns 3 when the allocation fails)
int ldmm_shoot_prepare(LdmmCtx *c);
cudaError_t ldmm_shoot_iterate(LdmmCtx *c, const float *I0, const float *I1, float *alpha0,
                               float *phi0T, float *phiT0, cudaStream_t s);
// LDMMVelShootingIteratorCPU (LDMM/LDMMVelShootingIteratorCPU.cxx): the
// buffers (returns 3 when the allocation fails) and one Iterate; v0, phi0T,
// phiT0 are [3][N]; update_step: set the step from the update's size
// instead of moving v0
int ldmm_velshoot_prepare(LdmmCtx *c);
cudaError_t ldmm_velshoot_iterate(LdmmCtx *c, const float *I0, const float *I1, float *v0,
                                  float *phi0T, float *phiT0, int update_step, cudaStream_t s);
// LDMMGeodesicShootingGPU::ShootImage(I0, alpha0, T): the geodesic alone
cudaError_t ldmm_geodesic_shoot(LdmmCtx *c, const float *I0, const float *alpha0, float *phi0T,
                                float *phiT0, float *img, cudaStream_t s);
// LDMMAdShootingIteratorCPU (LDMM/LDMMAdShootingIteratorCPU.cxx): the
// buffers (returns 3 when an allocation fails), one Iterate, and the final
// maps of finalUpdatePhi0T / finalUpdatePhiT0 from the last Iterate
int ldmm_adshoot_prepare(LdmmCtx *c);
cudaError_t ldmm_adshoot_iterate(LdmmCtx *c, const float *I0, const float *I1, float *alpha0,
                                 float *phi0T, float *phiT0, cudaStream_t s);
cudaError_t ldmm_adshoot_final_maps(LdmmCtx *c, float *phi0T, float *phiT0, cudaStream_t s);
// One iteration (IterateNew or IterateOrig); v is [T][3][N]. update_step:
// compute the step from max |2v - (2/sigma^2) K f| and leave v unchanged.
// h(x) = x (HField3DUtils::setToIdentity), three planes of grid d
cudaError_t identity_field(float *hx, float *hy, float *hz, Dims d, cudaStream_t s);
// IterateNew's alphas only: alphas[t] = splat of the residual to t / sigma^2
cudaError_t ldmm_alphas(LdmmCtx *c, const float *I0, const float *I1, const float *v,
                        float *alphas, cudaStream_t s);
cudaError_t ldmm_iterate(LdmmCtx *c, const float *I0, const float *I1, float *v, int update_step,
                         cudaStream_t s);

}  // namespace aw
