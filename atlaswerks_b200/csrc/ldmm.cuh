// ldmm.cuh — device state of the LDMM relaxation iterator (ldmm.cu).
#pragma once

#include "fluid.cuh"
#include "splat.cuh"

namespace aw {

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
  float *JT;        // T x N: I1 pulled back to each time point (IterateOrig)
  float *JD;        // T x N: transported Jacobian determinants (IterateOrig)
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
cudaError_t ldmm_shoot_iterate(LdmmCtx *c, const float *I0, const float *I1, float *alpha0,
                               float *phi0T, float *phiT0, cudaStream_t s);
// One iteration (IterateNew or IterateOrig); v is [T][3][N]. update_step:
// compute the step from max |2v - (2/sigma^2) K f| and leave v unchanged.
cudaError_t ldmm_iterate(LdmmCtx *c, const float *I0, const float *I1, float *v, int update_step,
                         cudaStream_t s);

}  // namespace aw
