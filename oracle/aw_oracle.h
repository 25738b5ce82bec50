/*
 * aw_oracle.h — CPU restatement of the AtlasWerks registration inner loop.
 *
 * TEST INFRASTRUCTURE: the checker for the CUDA path. Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg use it.
 */
#ifndef AW_ORACLE_H
#define AW_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* HField3DUtils::VectorBackgroundStrategy order (UtilitiesDataTypes/HField3DUtils.h:44-49) */
enum {
  AW_BG_PARTIAL_ID = 0,
  AW_BG_ID = 1,
  AW_BG_PARTIAL_ZERO = 2,
  AW_BG_ZERO = 3,
  AW_BG_CLAMP = 4,
  AW_BG_WRAP = 5
};

void aw_oracle_identity(float *hx, float *hy, float *hz, int nx, int ny, int nz);
void aw_oracle_apply(const float *img, const float *hx, const float *hy, const float *hz,
                     float *out, int nx, int ny, int nz, float bg);
void aw_oracle_apply_u(const float *img, const float *vx, const float *vy, const float *vz,
                       float *out, int nx, int ny, int nz, double spx, double spy, double spz,
                       float bg);
void aw_oracle_gradient(const float *a, float *gx, float *gy, float *gz, int nx, int ny, int nz,
                        double spx, double spy, double spz, int wrap);
void aw_oracle_compose_hv(const float *gx, const float *gy, const float *gz, const float *vx,
                          const float *vy, const float *vz, float *ox, float *oy, float *oz,
                          int nx, int ny, int nz, double spx, double spy, double spz, int dir,
                          int bgs);
void aw_oracle_compose_vh(const float *vx, const float *vy, const float *vz, const float *gx,
                          const float *gy, const float *gz, float *ox, float *oy, float *oz,
                          int nx, int ny, int nz, double spx, double spy, double spz, int dir,
                          int bgs);
void aw_oracle_splat(const float *img, const float *hx, const float *hy, const float *hz,
                     float *out, int nx, int ny, int nz, float bg);
void aw_oracle_fluid_apply_f64(double *vx, double *vy, double *vz, int nx, int ny, int nz,
                               double spx, double spy, double spz, double alpha, double beta,
                               double gamma, int inverse);
void aw_oracle_fluid_apply(float *vx, float *vy, float *vz, int nx, int ny, int nz, double spx,
                           double spy, double spz, double alpha, double beta, double gamma,
                           int inverse);
float aw_oracle_max_norm(const float *vx, const float *vy, const float *vz, long n);
double aw_oracle_greedy_iterate(const float *I0, const float *I1, float *hx, float *hy, float *hz,
                                float *hix, float *hiy, float *hiz, int nx, int ny, int nz,
                                double spx, double spy, double spz, double alpha, double beta,
                                double gamma, float max_pert, int update_step, float *step);

void aw_oracle_apply_atlas(const float *img, int mx, int my, int mz, const float *hx,
                           const float *hy, const float *hz, float *out, int nx, int ny, int nz);
double aw_oracle_atlas_iterate(const float *I0, int mx, int my, int mz, const float *I1, float *hx,
                               float *hy, float *hz, int nx, int ny, int nz, double spx,
                               double spy, double spz, double alpha, double beta, double gamma,
                               float max_pert, int update_step, float *step);
void aw_oracle_atlas_mean(const float *const *imgs, const int *dims, const float *const *h,
                          const float *w, int ns, float *mean, int nx, int ny, int nz);

double aw_oracle_ldmm_alphas(const float *I0, const float *I1, const float *v, int T, int nx,
                             int ny, int nz, double spx, double spy, double spz, float sigma,
                             float *alphas);
double aw_oracle_ldmm_iterate(const float *I0, const float *I1, float *v, int T, int nx, int ny,
                              int nz, double spx, double spy, double spz, double alpha,
                              double beta, double gamma, float sigma, float *step,
                              int update_step, float max_pert, double *vec_energy);

void aw_oracle_jacobian(const float *vx, const float *vy, const float *vz, float *jac, int nx,
                        int ny, int nz, double spx, double spy, double spz);
double aw_oracle_ldmm_iterate_orig(const float *I0, const float *I1, float *v, int T, int nx,
                                   int ny, int nz, double spx, double spy, double spz,
                                   double alpha, double beta, double gamma, float sigma,
                                   float *step, int update_step, float max_pert,
                                   double *vec_energy);
/* GetI1At0 (I1 pulled back through the velocities) and ComputeJacDet */
void aw_oracle_ldmm_i1_at_0(const float *I1, const float *v, int T, int nx, int ny, int nz,
                            double spx, double spy, double spz, float *img, float *jd);
/* LDMMShootingIteratorCPU::Iterate: alpha0, phi0T, phiT0 updated in place;
 * returns the image energy; *vec_energy (if not null) = sum over t of the
 * step energies <L v_t, v_t> */
double aw_oracle_ldmm_shoot_iterate(const float *I0, const float *I1, float *alpha0, float *phi0T,
                                    float *phiT0, int T, int nx, int ny, int nz, double spx,
                                    double spy, double spz, double alpha, double beta,
                                    double gamma, float sigma, float step, double *vec_energy);

/* LDMMAdShootingIteratorCPU::Iterate + backwardAdIntegration: alpha0
 * updated in place; V (T x 3N) receives the shot velocities; phi0T / phiT0
 * are left at time t_1 as the reference leaves them. Returns the image
 * energy sp^3 sum (I0(phiT0) - I1)^2; *vec_energy = <L v0, v0>. */
double aw_oracle_ldmm_adshoot_iterate(const float *I0, const float *I1, float *alpha0,
                                      float *phi0T, float *phiT0, float *V, int T, int nx, int ny,
                                      int nz, double spx, double spy, double spz, double alpha,
                                      double beta, double gamma, float sigma, float step,
                                      double *vec_energy);
/* LDMMGeodesicShootingCPU::ShootImage(I0, alpha0, T): phi0T, phiT0 and the
 * final image I0(phiT0) */
void aw_oracle_geodesic_shoot(const float *I0, const float *alpha0, int T, int nx, int ny, int nz,
                              double spx, double spy, double spz, double alpha, double beta,
                              double gamma, float *phi0T, float *phiT0, float *img);
/* LDMMVelShootingIteratorCPU::Iterate: v0 updated in place (or *step set
 * with update_step), phi0T / phiT0 the geodesic's maps; returns the image
 * energy, *vec_energy the sum of the step energies */
double aw_oracle_ldmm_velshoot_iterate(const float *I0, const float *I1, float *v0, float *phi0T,
                                       float *phiT0, int T, int nx, int ny, int nz, double spx,
                                       double spy, double spz, double alpha, double beta,
                                       double gamma, float sigma, float *step, int update_step,
                                       float max_pert, double *vec_energy);
/* ImageUtils::resampleNew, clamp background, linear (origin 0) */
void aw_oracle_resample_image(const float *in, int nx, int ny, int nz, double ssx, double ssy,
                              double ssz, float *out, int mx, int my, int mz, double dsx,
                              double dsy, double dsz);

/* MedianCalculator::Select over images (Algorithms/Common/MedianCalculator
 * .cxx:264-389): out = the k-th smallest (0-based) value per voxel of the n
 * images stacked in imgs [n][nvox], by the reference's rounds of bisection.
 * Returns 0, 1 when a voxel is still open after round n + 1 (the
 * reference throws "Select() not converging"), or 2 for no images, no
 * voxels or k outside [0, n). */
int aw_oracle_voxel_median(const float *imgs, int n, long nvox, int k, float *out);

void aw_oracle_gauss_blur(const float *in, float *out, int nx, int ny, int nz, float sx, float sy,
                          float sz, int kx, int ky, int kz);
void aw_oracle_downsample(const float *in, int nx, int ny, int nz, double spx, double spy,
                          double spz, float *out, int mx, int my, int mz);
void aw_oracle_upsample_hfield(const float *h, int nx, int ny, int nz, float *out, int mx, int my,
                               int mz, int rescale);

#ifdef __cplusplus
}
#endif
#endif
