/*
 * aw_b200.h — C ABI of the B200-native greedy-fluid / LDMM registration path.
 *
 * Every entry point takes plain device pointers (planar float32 arrays,
 * x fastest, nx*ny*nz elements each; vector fields as three such planes, the
 * layout of the reference's cplVector3DArray), sizes, spacings and an
 * optional CUDA stream passed as void* (NULL = legacy default stream). All
 * work is stream-ordered; only the explicit *_get_* readbacks synchronise.
 *
 * Return value: 0 on success, non-zero on error; aw_last_error() gives the
 * message (thread-local). The reference raises AtlasWerksException for the
 * same conditions (Algorithms/Common/DiffOperGPU.cxx:127-182,
 * Base/CUDAUtilities.cxx:137-170).
 *
 * Grid limits: every axis in [2, 512] (the reference caps FFT axes at 512,
 * CUDACommon/src/cudaFFTSolver.cu:21). Slabs whose half spectrum,
 * ny*(nx/2+1)*8 bytes plus batch buffers, fits one CTA's shared memory
 * (227 KB, e.g. up to 224 x 224) are transformed in x and y by one kernel;
 * larger ones (256 x 256, 512 x 512, ...) by an x pass and a y pass through
 * the spectrum in device memory, with the same arithmetic.
 */
#ifndef AW_B200_H
#define AW_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* HField3DUtils::VectorBackgroundStrategy (UtilitiesDataTypes/HField3DUtils.h:44-49) */
enum aw_background {
  AW_BG_PARTIAL_ID = 0,
  AW_BG_ID = 1,
  AW_BG_PARTIAL_ZERO = 2,
  AW_BG_ZERO = 3,
  AW_BG_CLAMP = 4,
  AW_BG_WRAP = 5
};

/* Message of the last failed call on this thread. */
const char *aw_last_error(void);

/* Library build/version string. */
const char *aw_version(void);

/* ---------------------------------------------------------------------------
 * Device primitives. Replace CUDACommon's cudaHField3DUtils / cudaImage3D
 * free functions (CUDACommon/inc/cudaHField3DUtils.h:150-353,
 * CUDACommon/inc/cudaImage3D.h:95-110) and the CPU HField3DUtils templates
 * they mirror (UtilitiesDataTypes/HField3DUtils.txx).
 * ------------------------------------------------------------------------- */

/* out(x) = img(h(x)), trilinear, `background` outside (per corner).
 * Replaces cudaHField3DUtils::apply (CUDACommon/src/cudaHField3DUtils.cu:636-642)
 * and HField3DUtils::apply (UtilitiesDataTypes/HField3DUtils.txx:734-752). */
int aw_apply(const float *img, const float *hx, const float *hy, const float *hz, float *out,
             int nx, int ny, int nz, float background, void *stream);

/* Central-difference gradient / (2 sp), one-sided at the borders unless wrap.
 * Replaces cplComputeGradient (CUDACommon/inc/cudaImage3D.h:95-110) and
 * Array3DUtils::computeGradient (UtilitiesDataTypes/Array3DUtils.txx:783-900). */
int aw_gradient(const float *img, float *gx, float *gy, float *gz, int nx, int ny, int nz,
                double spx, double spy, double spz, int wrap, void *stream);

/* o(x) = g(x + direction * scale * v(x) / sp).
 * direction=+1: composeHV (UtilitiesDataTypes/HField3DUtils.txx:436-455,
 * CUDACommon/src/cudaHField3DUtilsSp.cu:453-511); direction=-1: composeHVInv
 * (HField3DUtils.txx:461-480). `scale` multiplies v first (1 for none). */
int aw_compose_hv(const float *gx, const float *gy, const float *gz, const float *vx,
                  const float *vy, const float *vz, float *ox, float *oy, float *oz, int nx,
                  int ny, int nz, double spx, double spy, double spz, float scale, int direction,
                  int background, void *stream);

/* o(x) = g(x) + direction * (scale * v)(g(x)) / sp.
 * direction=-1: composeVHInv (HField3DUtils.txx:405-430,
 * CUDACommon/src/cudaHField3DUtilsSp.cu:359-445); +1: composeVH. */
int aw_compose_vh(const float *vx, const float *vy, const float *vz, const float *gx,
                  const float *gy, const float *gz, float *ox, float *oy, float *oz, int nx,
                  int ny, int nz, double spx, double spy, double spz, float scale, int direction,
                  int background, void *stream);

/* Splat img by h (the adjoint of aw_apply): out(y) = bg + sum over sources
 * x of w(h(x) -> y) * img(x), in source order, no float atomics; bitwise
 * reproducible. Replaces cplSplat3DH (CUDACommon/inc/cudaSplat.h:119-131,
 * CUDACommon/src/cudaSplatAtomic.cu:569-599) and HField3DUtils::forwardApply
 * with normalize=false (UtilitiesDataTypes/HField3DUtils.txx:1058-1279).
 * Scratch (about 16 bytes per voxel) comes from the stream-ordered allocator. */
int aw_splat(const float *img, const float *hx, const float *hy, const float *hz, float *out,
             int nx, int ny, int nz, float background, void *stream);

/* h(x) = x on an nx x ny x nz grid, three planes
 * (HField3DUtils::setToIdentity, UtilitiesDataTypes/HField3DUtils.txx:26-45). */
int aw_identity(float *hx, float *hy, float *hz, int nx, int ny, int nz, void *stream);

/* Gaussian downsampling of an image to a coarser grid (out: mx*my*mz):
 * ImageUtils::gaussianDownsample (UtilitiesDataTypes/ImageUtils.txx:259-298),
 * sigma = sqrt(n/m / 2) per axis, as MultiscaleManager::DownsampleToLevel
 * uses it (Algorithms/Common/MultiscaleManager.cxx:344-366). (spx, spy, spz)
 * is the input spacing. Scratch from the stream-ordered allocator. */
int aw_downsample(const float *in, int nx, int ny, int nz, double spx, double spy, double spz,
                  float *out, int mx, int my, int mz, void *stream);

/* Deformation upsampling to a finer grid: hToVelocity, trilinear resampling
 * with CLAMP background and vectors rescaled by the size ratio when rescale
 * is set, velocityToH — GreedyDeformationData::SetScaleLevel
 * (Algorithms/Greedy/GreedyDeformationData.cxx:211-221) through
 * MultiscaleManager::UpsampleToLevel (MultiscaleManager.cxx:326-342). */
int aw_upsample_hfield(const float *hx, const float *hy, const float *hz, int nx, int ny, int nz,
                       float *ox, float *oy, float *oz, int mx, int my, int mz, int rescale,
                       void *stream);

/* Image resampling onto another grid: ImageUtils::resampleNew
 * (UtilitiesDataTypes/ImageUtils.txx:306-349) with clamped linear
 * interpolation, origin 0, (sx, sy, sz) the input spacing and (tx, ty, tz)
 * the output spacing — MultiscaleManager::UpsampleToLevel for images
 * (Algorithms/Common/MultiscaleManager.cxx:301-323), which
 * LDMMShootingDefData::SetScaleLevel applies to Alpha0
 * (Algorithms/LDMM/LDMMShootingDefData.cxx:166-168). */
int aw_resample_image(const float *in, int nx, int ny, int nz, double sx, double sy, double sz,
                      float *out, int mx, int my, int mz, double tx, double ty, double tz,
                      void *stream);

/* Scratch capacity of aw_splat_static, fixed when the library is built. */
#define AW_SPLAT_STATIC_MAX_BYTES (8u << 20)

/* aw_splat for callers that must not allocate device memory while they run
 * (no counterpart in the reference): a host that owns all device memory
 * through its own pool, or a latency-critical loop where an allocation may
 * block or fail. Same result as aw_splat, bit for bit. The scratch is one
 * fixed array of AW_SPLAT_STATIC_MAX_BYTES in the library's device memory
 * (held on every device that loads the library until the process exits);
 * grids whose scratch exceeds it are rejected with an error. The scratch of
 * an nx x ny x nz grid, with m = (nx+1)(ny+1)(nz+1) and each term rounded up
 * to a multiple of 256 bytes, is 4(m+1) + 4m + 4 nx ny nz + 4 ceil(m/1024)
 * bytes (about 12 bytes per voxel: 88^3 fits, 89^3 does not);
 * aw_splat_static_fits answers for a grid. The first call on each device
 * looks up the array's device address and keeps it, so make it before any
 * stream capture, and do not reset the device (cudaDeviceReset) while the
 * library is loaded. All calls share the one array: calls that overlap on
 * the GPU (other streams, other host threads) race and must be serialised
 * by the caller. */
int aw_splat_static(const float *img, const float *hx, const float *hy, const float *hz,
                    float *out, int nx, int ny, int nz, float background, void *stream);
/* 1 when aw_splat_static takes an nx x ny x nz grid, else 0. */
int aw_splat_static_fits(int nx, int ny, int nz);

/* ---------------------------------------------------------------------------
 * Fluid kernel. Replaces KernelInterfaceGPU / DiffOperGPU
 * (Algorithms/Common/KernelInterfaceGPU.h:20-43, Common/DiffOperGPU.cxx:32-205)
 * and FFTSolverPlan3D (CUDACommon/inc/cudaFFTSolver.h:99-176).
 * ------------------------------------------------------------------------- */
typedef struct aw_fluid_s *aw_fluid_t;

/* KernelInterfaceGPU::SetSize + DiffOperParam{Alpha, Beta, Gamma}. */
int aw_fluid_create(int nx, int ny, int nz, double spx, double spy, double spz, float alpha,
                    float beta, float gamma, aw_fluid_t *out);
/* In place: inverse=1 ApplyInverseOperator (v <- L^-1 v), inverse=0
 * ApplyOperator (v <- L v). */
int aw_fluid_apply(aw_fluid_t k, float *vx, float *vy, float *vz, int inverse, void *stream);
int aw_fluid_destroy(aw_fluid_t k);
/* Launch shapes of the shared-memory FFT path (grids with an axis that is
 * not a power of two in [16, 256]): x-line pairs per batch, y-columns per
 * batch, (ky,kx) columns per z-pass CTA. The plan autotunes them when it is
 * created (each candidate timed on the device; the choice is kept per grid
 * and device for the process); aw_fluid_autotune re-runs the tuning,
 * aw_fluid_set_shapes overrides it. Results do not depend on the shapes.
 * On the register-FFT path (every axis a power of two in [16, 256]) the
 * only shape is the z pass's tile width, 16 or 8 (ky,kx) columns, also
 * chosen by timing when a plan is created: aw_fluid_get_shapes writes
 * {0, 0, width} and aw_fluid_set_shapes(k, 0, 0, width) overrides it. */
int aw_fluid_get_shapes(aw_fluid_t k, int *shapes /* [3] */);
int aw_fluid_set_shapes(aw_fluid_t k, int pairs, int cols, int zcols);
int aw_fluid_autotune(aw_fluid_t k, void *stream);
/* Every wait of the transform kernels on a bulk or TMA copy is bounded: a
 * wait that runs out records a timeout in the handle's status word and the
 * kernel returns early, leaving its output incomplete, instead of spinning.
 * aw_fluid_status synchronises `stream`, sets *timed_out to 1 when that
 * happened since the last call (else 0) and clears the word. No counterpart
 * in the reference, whose transforms have no waits. */
int aw_fluid_status(aw_fluid_t k, int *timed_out, void *stream);
/* Runs the timeout path on purpose: one CTA waits, with the same bounded
 * wait the transforms use but limited to `polls` polls (1..4096), on a
 * barrier that nothing arrives on, and records the timeout in the handle's
 * status word; the context stays usable. A check of the status reporting
 * for tests and health probes; no counterpart in the reference. */
int aw_fluid_wait_selftest(aw_fluid_t k, int polls, void *stream);

/* ---------------------------------------------------------------------------
 * Greedy iterator. Replaces GreedyIteratorGPU / GreedyIteratorCPU
 * (Algorithms/Greedy/GreedyIteratorGPU.h:32-58, GreedyIteratorCPU.cxx:99-138).
 * The step size, energy history and iteration count live on the device.
 * ------------------------------------------------------------------------- */
typedef struct aw_greedy_s *aw_greedy_t;

/* ctor + SetScaleLevel: grid, spacing, DiffOper parameters, MaxPert. */
int aw_greedy_create(int nx, int ny, int nz, double spx, double spy, double spz, float alpha,
                     float beta, float gamma, float max_pert, aw_greedy_t *out);
int aw_greedy_destroy(aw_greedy_t g);

/* GreedyDeformationData::StepSize(s) / StepSize(); get synchronises. */
int aw_greedy_set_step(aw_greedy_t g, float step);
int aw_greedy_get_step(aw_greedy_t g, float *step);
/* aw_fluid_status for the iterator's transforms and staged update. */
int aw_greedy_status(aw_greedy_t g, int *timed_out, void *stream);
/* GreedyParam::AutoStepReduce (Greedy/GreedyParam.h:61-65); off by default. */
int aw_greedy_set_auto_step_reduce(aw_greedy_t g, int on);
/* on = 1 (default): the update stages h over each tile (plus a one-voxel
 * halo) in shared memory by TMA where the grid allows (nx % 4 == 0, nx >= 40,
 * ny >= 10, nz >= 6, no inverse field); 0: every gather from global memory.
 * Both give the same bits; the switch exists to compare them. */
int aw_greedy_set_staged_update(aw_greedy_t g, int on);
/* on = 1 (default): an iteration without a step-size update or an inverse
 * field, on a grid of power-of-two axes, runs the inverse transform and the
 * update h' = h(x + eps v/sp) as one kernel, so v = K f never goes to HBM
 * (the stages GreedyIteratorGPU::Iterate runs as cplFFT inverse and
 * composeHV, Greedy/GreedyIteratorGPU.cxx:120-134); 0: v is stored and the
 * update is a kernel of its own. Both give the same bits. */
int aw_greedy_set_fused_update(aw_greedy_t g, int on);
/* on = 1: I0(h) in the force preparation and h(x + eps v/sp) in the fused
 * update interpolate with float fused multiply-adds instead of the
 * reference's double weights and sums: a few float ulps from the
 * bit-exact results (I0(h) within 1e-6 of it for images in [0, 1]); 0
 * (default): bit-exact with the reference CPU's interpolation. */
int aw_greedy_set_fast_interpolation(aw_greedy_t g, int on);
/* Tile shape of the staged update (x 32 voxels; index 0: 8 x 4 in y x z,
 * 1: 4 x 8, 2: 8 x 8, 3: 16 x 2), chosen when the handle is created by
 * timing each on the device (kept per grid and device for the process).
 * set = 0 reads it into *tile, set = 1 overrides it with *tile. */
int aw_greedy_update_tile(aw_greedy_t g, int set, int *tile);

/* One Iterate(): reads h (and hinv when non-NULL), writes the updated fields
 * to h_out / hinv_out (distinct buffers). update_step=1 recomputes the step
 * as MaxPert / max|v| first (UpdateStepSizeNextIteration). Records the
 * energy sp^3 * sum (I1 - I0(h))^2 of the incoming h. */
int aw_greedy_iterate(aw_greedy_t g, const float *I0, const float *I1, const float *hx,
                      const float *hy, const float *hz, float *ox, float *oy, float *oz,
                      const float *hix, const float *hiy, const float *hiz, float *hiox,
                      float *hioy, float *hioz, int update_step, void *stream);

/* n_iters iterations, ping-ponging between h (holds the initial field and
 * receives the final one) and the scratch field s; hinv / sinv likewise when
 * non-NULL. The loop body is captured once as a CUDA graph and replayed.
 * update_first=1 recomputes the step at the first iteration. */
int aw_greedy_run(aw_greedy_t g, const float *I0, const float *I1, float *hx, float *hy,
                  float *hz, float *sx, float *sy, float *sz, float *hix, float *hiy, float *hiz,
                  float *six, float *siy, float *siz, int n_iters, int update_first,
                  void *stream);

/* Per-kernel device time of one iteration: each stage (0 force-prep,
 * 1 energy, 2 xy-forward FFT, 3 z-solve, 4 xy-inverse FFT, 5 max-norm,
 * 6 update, 7 xy-inverse FFT fused with the update) is launched `reps` times
 * back to back between CUDA events on `stream`; ms_out[8] receives the mean
 * milliseconds per launch. Leaves h_out holding one iteration's result;
 * records extra energies. Synchronises. */
int aw_greedy_profile(aw_greedy_t g, const float *I0, const float *I1, const float *hx,
                      const float *hy, const float *hz, float *ox, float *oy, float *oz,
                      const float *hix, const float *hiy, const float *hiz, float *hiox,
                      float *hioy, float *hioz, int reps, void *stream, float *ms_out);

/* Copies the energy history (oldest first) to host; synchronises. */
int aw_greedy_get_energies(aw_greedy_t g, double *out, int max_count, int *count);
/* The most recent energy only (GreedyDeformationData's LastEnergy, what
 * GreedyIteratorGPU::Iterate adds to the data object in debug mode); waits
 * for work queued on the legacy default stream. Error before any iteration. */
int aw_greedy_last_energy(aw_greedy_t g, double *energy);

/* ---------------------------------------------------------------------------
 * Greedy atlas building over the subjects resident on one GPU. Replaces the
 * per-GPU thread of GreedyAtlasBuilder (Algorithms/Greedy/GreedyAtlasBuilder.txx:
 * 150-301, Algorithms/Common/AtlasThread.txx:97-181,
 * Algorithms/Greedy/GreedyAtlasThreadGPU.cxx:161-194). Every subject's
 * deformation h_i (template grid, identity at create) is owned by the handle;
 * the mean template (template grid) is the I1 of every subject. A subject
 * image may sit on its own grid: it is sampled at (h + 0.5) * m/n - 0.5 per
 * axis (voxel centres of equal physical extent); with equal grids the
 * iteration is the reference's. Across GPUs, shard the subjects, call
 * aw_atlas_compute_mean on each, sum the mean buffers (one all-reduce) and
 * continue: the weights are the global ones.
 * ------------------------------------------------------------------------- */
typedef struct aw_atlas_s *aw_atlas_t;

/* template grid, spacing, DiffOper parameters, MaxPert, local subject count */
int aw_atlas_create(int nx, int ny, int nz, double spx, double spy, double spz, float alpha,
                    float beta, float gamma, float max_pert, int n_subjects, aw_atlas_t *out);
int aw_atlas_destroy(aw_atlas_t a);
/* GreedyAtlasDefDataGPU(I, mean, weight): subject i's image (device, the
 * caller keeps it alive, grid snx x sny x snz) and its mean weight */
int aw_atlas_set_subject(aw_atlas_t a, int i, const float *img, int snx, int sny, int snz,
                         float weight);
/* device pointers of subject i's deformation (template grid; read or write
 * between calls, e.g. to resume from a checkpoint) and of the mean buffer */
int aw_atlas_field(aw_atlas_t a, int i, float **hx, float **hy, float **hz);
int aw_atlas_mean_buffer(aw_atlas_t a, float **mean);
/* ComputeThreadMean: mean = sum_i w_i I_i(h_i), float, in subject order */
int aw_atlas_compute_mean(aw_atlas_t a, void *stream);
/* n_iters greedy iterations of every subject toward the current mean;
 * update_first=1 recomputes each subject's step at the first one
 * (BeginImageIteration at iteration 0). Graph-captured, no host sync. */
int aw_atlas_iterate(aw_atlas_t a, int n_iters, int update_first, void *stream);
/* subject i's step size and energy history (oldest first); synchronise */
int aw_atlas_get_step(aw_atlas_t a, int i, float *step);
int aw_atlas_get_energies(aw_atlas_t a, int i, double *out, int max_count, int *count);

/* ---------------------------------------------------------------------------
 * LDMM iterator (relaxation, splatting gradient). Replaces LDMMIteratorGPU /
 * LDMMIteratorCPU::IterateNew (Algorithms/LDMM/LDMMIteratorGPU.cxx:159-293,
 * LDMMIteratorCPU.cxx:529-631). Velocity fields are one device buffer
 * [T][3][nz][ny][nx].
 * ------------------------------------------------------------------------- */
typedef struct aw_ldmm_s *aw_ldmm_t;

/* ctor + SetScaleLevel: grid, spacing, DiffOper parameters, NTimeSteps,
 * Sigma and MaxPert (LDMM/LDMMIteratorParam.h:28-54). */
int aw_ldmm_create(int nx, int ny, int nz, double spx, double spy, double spz, float alpha,
                   float beta, float gamma, int n_time_steps, float sigma, float max_pert,
                   aw_ldmm_t *out);
int aw_ldmm_destroy(aw_ldmm_t l);
/* LDMMIteratorCPU's UseOrigGradientCalc (LDMM/LDMMIteratorCPU.cxx:33,
 * 369-527): 1 = IterateOrig, the Jacobian-transport gradient (the
 * reference's default), 0 = IterateNew, the splatting gradient (this
 * handle's default). Allocates 2 T N floats for IterateOrig. */
int aw_ldmm_use_orig_gradient_calc(aw_ldmm_t l, int on);
/* LDMMIteratorCPU's debug-mode vector energy (LDMM/LDMMIteratorCPU.cxx:
 * 493-505, 601-610): on = 1 makes every IterateNew / IterateOrig iteration
 * that updates v also apply L to each updated v_t (one more forward
 * transform, L and inverse per time step) and record sum_t <L v_t, v_t> sp^3
 * beside its image energy (aw_ldmm_get_vec_energies; LDMMEnergy::VecEnergy
 * is that sum / T). Off by default. Synchronises. */
int aw_ldmm_set_vector_energy(aw_ldmm_t l, int on);
/* The step energies <L v_t, v_t> sp^3 (t = 0 .. T-1) of the last iteration
 * that recorded vector energies (LDMMEnergy::VecStepEnergy); out holds T
 * values. Synchronises. */
int aw_ldmm_get_vec_step_energies(aw_ldmm_t l, double *out, int n_time_steps);
/* LDMMDeformationData::StepSize(s) / StepSize(); get synchronises. */
int aw_ldmm_set_step(aw_ldmm_t l, float step);
int aw_ldmm_get_step(aw_ldmm_t l, float *step);
/* aw_fluid_status for the iterator's transforms. */
int aw_ldmm_status(aw_ldmm_t l, int *timed_out, void *stream);
/* One Iterate(): updates v in place. update_step=1 instead computes the step
 * from max |2v - (2/sigma^2) K f| and leaves v unchanged
 * (UseAdaptiveStepSize, LDMM/LDMMWarp.txx:99-104). */
int aw_ldmm_iterate(aw_ldmm_t l, const float *I0, const float *I1, float *v, int update_step,
                    void *stream);
/* LDMMIteratorCPU/GPU::Iterate(data, computeAlphasOnly = true) then GetAlpha(t)
 * (LDMM/LDMMIteratorCPU.cxx:529-631, LDMMIteratorGPU.h:84-90): the forward
 * integration and residual of IterateNew (its image energy recorded), then
 * the backward sweep of composeVHInv and splats; alphas[t] (T x N floats) =
 * splat of the residual to time t, times (float)(1 / sigma^2). v is not
 * changed. IterateNew only (error with the Jacobian-transport gradient). */
int aw_ldmm_alphas(aw_ldmm_t l, const float *I0, const float *I1, const float *v, float *alphas,
                   void *stream);
/* n_iters iterations replayed from a captured CUDA graph; adaptive_first=1
 * runs the step-size pass before the first iteration. */
int aw_ldmm_run(aw_ldmm_t l, const float *I0, const float *I1, float *v, int n_iters,
                int adaptive_first, void *stream);
/* Image energies sp^3 * sum (I0(h_T) - I1)^2, oldest first; synchronises. */
int aw_ldmm_get_energies(aw_ldmm_t l, double *out, int max_count, int *count);

/* LDMM geodesic shooting (LDMMShootingIteratorCPU / GPU::Iterate,
 * Algorithms/LDMM/LDMMShootingIteratorCPU.cxx:199-304) on an LDMM handle (its
 * T, sigma, step size and kernel): shoots from the initial momentum alpha0
 * (a scalar image, updated in place to (1 - step) alpha0 + (step/sigma^2)
 * times the splatted residual) and leaves phi0T and phiT0 ([3][N] each, the
 * maps LDMMShootingDefData::Phi0T / PhiT0) in the caller's buffers; records
 * the image energy (aw_ldmm_get_energies) and the sum over t of the step
 * energies <L v_t, v_t> (aw_ldmm_get_vec_energies). */
int aw_ldmm_shoot_iterate(aw_ldmm_t l, const float *I0, const float *I1, float *alpha0,
                          float *phi0T, float *phiT0, void *stream);
/* LDMMVelShootingIteratorCPU::Iterate (Algorithms/LDMM/
 * LDMMVelShootingIteratorCPU.cxx:186-344) on an LDMM handle (its T, sigma,
 * MaxPert, step size and kernel): shoots the geodesic in velocity form from
 * v0 ([3][N], updated in place to (1 - 2 step) v0 + (2 step / sigma^2)
 * K(grad(I0) splat(I0(phiT0) - I1 by phiT0))), leaves the maps phi0T / phiT0
 * ([3][N] each) in the caller's buffers and records the image energy and
 * the step energies (aw_ldmm_get_energies, aw_ldmm_get_vec_energies,
 * aw_ldmm_get_vec_step_energies). update_step = 1: the step-size pass
 * (step = MaxPert / max |2 v0 - (2/sigma^2) K(...)|, v0 unchanged). Its
 * buffers (15 N floats) are allocated at the first call. */
int aw_ldmm_velshoot_iterate(aw_ldmm_t l, const float *I0, const float *I1, float *v0,
                             float *phi0T, float *phiT0, int update_step, void *stream);
/* LDMMGeodesicShootingGPU / CPU::ShootImage(I0, alpha0, nTimeSteps)
 * (Algorithms/LDMM/LDMMGeodesicShootingCPU.cxx:44-157): the geodesic from I0
 * along the momentum alpha0 over the handle's T time steps and kernel,
 * without an update; phi0T / phiT0 receive GetPhi0To1 / GetPhi1To0 and image
 * the final image GetFinalImage = I0(phiT0). */
int aw_ldmm_geodesic_shoot(aw_ldmm_t l, const float *I0, const float *alpha0, float *phi0T,
                           float *phiT0, float *image, void *stream);

/* LDMM adjoint geodesic shooting (LDMMAdShootingIteratorCPU::Iterate and
 * backwardAdIntegration, Algorithms/LDMM/LDMMAdShootingIteratorCPU.cxx:
 * 237-431; GPU twin LDMMAdShootingIteratorGPU) on an LDMM handle (its T,
 * sigma, step size and kernel): shoots the geodesic from alpha0 keeping
 * every velocity, map, deformed image and momentum image of the T time
 * points in device memory (allocated at the first call), integrates the
 * adjoint equations backward and takes the gradient step
 * alpha0 -= step * (-(grad I0 . v0) - alphaTilde). phi0T / phiT0 end at
 * time t_1, as the reference's iteration leaves LDMMShootingDefData's maps.
 * Records the image energy sp^3 sum (I0(phiT0) - I1)^2 (aw_ldmm_get_energies)
 * and <L v0, v0> (aw_ldmm_get_vec_energies). */
int aw_ldmm_adshoot_iterate(aw_ldmm_t l, const float *I0, const float *I1, float *alpha0,
                            float *phi0T, float *phiT0, void *stream);
/* LDMMWarpAd::FinishWarp's finalUpdatePhi0T / finalUpdatePhiT0
 * (LDMMAdShootingIteratorCPU.cxx:433-453, LDMMWarpAd.txx:37-42): the maps
 * from time 0 to 1 and back composed through the last iteration's velocities. */
int aw_ldmm_adshoot_final_maps(aw_ldmm_t l, float *phi0T, float *phiT0, void *stream);
/* Vector energies, oldest first, of the shooting iterations and (with
 * aw_ldmm_set_vector_energy) of IterateNew / IterateOrig: the sum over
 * the time steps of LDMMEnergy::VecStepEnergy(t), i.e. sum_t <L v_t, v_t> sp^3
 * for aw_ldmm_shoot_iterate and <L v0, v0> sp^3 for aw_ldmm_adshoot_iterate
 * (0 for the relaxation iterations); synchronises. */
int aw_ldmm_get_vec_energies(aw_ldmm_t l, double *out, int max_count, int *count);

/* LDMM relaxation atlas (LDMMAtlasBuilder / LDMMAtlasThreadCPU,
 * Algorithms/LDMM/LDMMAtlasThreadCPU.cxx:207-264, LDMMAtlasBuilder.txx:274-335).
 * Every subject is an aw_ldmm_t whose I0 is the shared mean and I1 its image;
 * after the subjects' iterations the caller forms
 *   mean = sum_i w_i I1_i(h_{0->1}) JacDet_i / sum_i w_i JacDet_i
 * (JacobianScale), or sum_i w_i I1_i(h_{0->1}), from these three calls
 * (across processes: sum acc and jacsum, e.g. one all-reduce each, before
 * normalising).
 *
 * aw_ldmm_i1_at_0: LDMMDeformationData::GetI1At0 (I1 pulled back to time 0
 * through v) into img and LDMMIteratorCPU::ComputeJacDet into jacdet (NULL:
 * skipped); v is [T][3][N] of the handle's grid. Uses the handle's scratch:
 * not concurrent with its iterations. */
int aw_ldmm_i1_at_0(aw_ldmm_t l, const float *I1, const float *v, float *img, float *jacdet,
                    void *stream);
/* acc += (img * jacdet) * weight and jacsum += jacdet * weight (float, in
 * that order), or acc += img * weight when jacdet is NULL; n voxels */
int aw_ldmm_atlas_accumulate(float *acc, float *jacsum, const float *img, const float *jacdet,
                             float weight, long n, void *stream);
/* acc /= jacsum (float division), n voxels */
int aw_ldmm_atlas_normalize(float *acc, const float *jacsum, long n, void *stream);
/* The atlas as the per-voxel median of the subjects' deformed images
 * (LDMMAtlasParam UsePerVoxelMedian; MedianCalculator::Select over the
 * deformed images, Algorithms/Common/MedianCalculator.cxx:264-389, called
 * by LDMMAtlasBuilder::ComputeMedian, LDMM/LDMMAtlasBuilder.txx:218-233):
 * out = the k-th smallest (0-based) of the n_images values at each voxel, by
 * the reference's bisection, including its early end on intervals narrower
 * than (volume max - volume min) / 10000. images: a HOST array of n_images
 * (1..256) device pointers to nx*ny*nz floats. The builder's median index is
 * n/2 - 1 for even n, n/2 for odd n. Synchronises; an error when a voxel
 * does not converge (the reference throws). */
int aw_ldmm_atlas_voxel_median(const float *const *images, int n_images, int k, int nx, int ny,
                               int nz, float *out, void *stream);

/* ---------------------------------------------------------------------------
 * Learned warm start: the kernels of a 3D convolutional encoder-decoder
 * (no counterpart in the reference; it predicts an initial deformation
 * that the greedy iteration then refines). Convolutions run as implicit
 * GEMMs on the tcgen05 tensor cores, BF16 operands, FP32 accumulation.
 * Activations: BF16 [B][D][H][W][C], channels last, C a multiple of 16.
 * Weights: BF16 [Cout][taps][Cin] (taps 27 = 3x3x3 zero-padded, or 1);
 * the data gradient takes the transposed copy [Cin][taps][Cout] that
 * aw_nn_weights_bf16 writes. Output channels: 16 32 48 64 96 128 192.
 * ------------------------------------------------------------------------- */
/* Grids too small to fill the GPU with 128-voxel row tiles split K over
 * CTAs; the FP32 partials go to `scratch` (at least
 * aw_nn_conv3d_scratch_floats floats; NULL or smaller = no split). */
size_t aw_nn_conv3d_scratch_floats(int B, int D, int H, int W, int cin, int cout, int ntaps);
/* Planes per tile of the direct (TMA halo tile + shifted-descriptor MMA)
 * kernel that aw_nn_conv3d_fwd uses for this shape: 3x3x3 taps, W % 8 == 0,
 * H % 16 == 0, (cin, cout) in {(16,16), (48,16), (16,32), (32,32)};
 * 0 = the implicit-GEMM kernel. Needs a current CUDA device. */
int aw_nn_conv3d_direct_planes(int B, int D, int H, int W, int cin, int cout, int ntaps);
/* on = 1: every forward convolution takes the implicit-GEMM kernel (the
 * direct kernel off, process-wide), to compare the two paths; 0 restores
 * the shape-based choice */
void aw_nn_set_gemm_only(int on);
/* out = act(conv(x, w) + bias): BF16 out_bf16, or FP32 out_f32 when given */
int aw_nn_conv3d_fwd(const void *x, int B, int D, int H, int W, int cin, const void *w,
                     const float *bias, int cout, int ntaps, int relu, void *out_bf16,
                     float *out_f32, float *scratch, size_t scratch_floats, void *stream);
/* dx = conv^T(dy, w) times (mask > 0) (the ReLU derivative of the layer's
 * input, which is a post-ReLU activation); mask NULL = no mask */
int aw_nn_conv3d_dgrad(const void *dy, int B, int D, int H, int W, int cout, const void *wt,
                       int cin, int ntaps, const void *mask, void *dx, float *scratch,
                       size_t scratch_floats, void *stream);
/* dw [Cout][taps][Cin] (FP32) = sum over voxels of dy x shifted x; the
 * voxel sum is split over `splits` CTA columns whose partials go to
 * scratch (aw_nn_wgrad_scratch_floats floats) and are summed in order */
size_t aw_nn_wgrad_scratch_floats(int cin, int cout, int ntaps, int splits);
int aw_nn_conv3d_wgrad(const void *x, const void *dy, int B, int D, int H, int W, int cin,
                       int cout, int ntaps, int splits, float *scratch, float *dw, void *stream);
/* db[c] = sum over the M voxels of dy[.][c], through block partials in
 * scratch (aw_nn_bias_scratch_floats floats) added in order */
size_t aw_nn_bias_scratch_floats(long M, int cout);
int aw_nn_bias_grad(const void *dy, long M, int cout, float *scratch, float *db, void *stream);
/* 2x2x2 average pooling of the (D,H,W) grid; backward (D,H,W = the fine
 * grid) spreads dy/8, adds `add` and keeps it where mask > 0 (the pooled
 * post-ReLU activation); add and mask may be NULL */
int aw_nn_pool(const void *in, int B, int D, int H, int W, int C, void *out, int backward,
               const void *add, const void *mask, void *stream);
/* nearest x2 upsampling of the coarse (D,H,W) grid into channels
 * [c0, c0+C) of a Ct-channel fine tensor; backward sums the 8 children */
int aw_nn_upsample(const void *in, int B, int D, int H, int W, int C, void *out, int Ct, int c0,
                   int backward, void *stream);
/* copy (or add) C channels between channel slices of two tensors */
int aw_nn_slice(const void *src, int Cs, int cs0, void *dst, int Cd, int cd0, int C, long voxels,
                int accumulate, void *stream);
/* (I0, I1) planar float -> channels 0, 1 of a 16-channel BF16 input */
int aw_nn_pack_pair(const float *I0, const float *I1, long voxels, void *x, void *stream);
/* loss = mean over voxels and 3 channels of (pred[.][c] - target[c][.])^2
 * (pred FP32 [V][16], target planar [3][V]); grad BF16 [V][16] */
size_t aw_nn_mse_scratch_doubles(long voxels);
int aw_nn_mse(const float *pred, const float *target, long voxels, void *grad, double *scratch,
              float *loss, void *stream);
/* Adam on FP32 masters (step counts from 1) */
int aw_nn_adam(float *w, const float *g, float *m1, float *m2, long n, float lr, float beta1,
               float beta2, float eps, int step, void *stream);
/* BF16 copies of FP32 weights: [Cout][taps][Cin] and (wt_bf16 non-NULL)
 * the transposed [Cin][taps][Cout] */
int aw_nn_weights_bf16(const float *w, int cout, int ntaps, int cin, void *w_bf16,
                       void *wt_bf16, void *stream);
/* h = identity + the predicted displacement (channels 0..2 of FP32 [V][16]) */
int aw_nn_displacement_to_h(const float *pred, int D, int H, int W, float *hx, float *hy,
                            float *hz, void *stream);
/* 1 in *timed_out when a GEMM gave up a bounded wait since the last call */
int aw_nn_status(int *timed_out);

/* ---------------------------------------------------------------------------
 * The warm start as one handle (no counterpart in the reference): the
 * trained encoder-decoder predicts a deformation for a pair, and the greedy
 * iteration refines it, with the plain greedy solve from the identity as the
 * fallback. The network runs on its own grid (axes multiples of 8, at most
 * the pair's): the pair is Gaussian-downsampled to it (aw_downsample's
 * filter) and the predicted deformation upsampled back with its vectors
 * rescaled (aw_upsample_hfield). Unit spacing; fluid parameters alpha =
 * beta = 0.01, gamma = 0.001.
 * Parameters: host FP32, per layer in network order (e0a e0b e1a e1b e2a e2b
 * e3a e3b d2a d2b d1a d1b d0a d0b head) the weights [Cout][taps][Cin] then
 * the Cout biases; aw_warmstart_param_floats() of them in all. */
size_t aw_warmstart_param_floats(void);
typedef struct aw_warmstart_s *aw_warmstart_t;
int aw_warmstart_create(int nx, int ny, int nz, int net_nx, int net_ny, int net_nz,
                        const float *params, size_t n_params, float max_pert,
                        aw_warmstart_t *out);
int aw_warmstart_destroy(aw_warmstart_t w);
/* h = the predicted deformation of the pair (device, pair grid). The
 * prediction (downsampling, the network's 25 launches, upsampling) runs as
 * one CUDA graph on the handle's stream, captured at the first call and
 * again whenever the five pointers change; ordered after `stream`'s work
 * and before its later work. */
int aw_warmstart_predict(aw_warmstart_t w, const float *I0, const float *I1, float *hx, float *hy,
                         float *hz, void *stream);
/* Registration with the warm start: predict, then greedy iterations from
 * the prediction (the step set at the first from its own velocity and
 * halved whenever the energy rises) in chunks of `chunk`, until an
 * iteration's energy sp^3 sum (I1 - I0(h))^2 is <= target_energy. A chunk
 * that does not lower the best energy so far, or max_refine_iters without
 * reaching the target, falls back to the plain solve from the identity for
 * plain_iters iterations. h receives the result; *iters_run the iterations
 * executed, *fell_back 1 when the fallback ran. Reads the energies back
 * after every chunk (synchronises). */
int aw_warmstart_register(aw_warmstart_t w, const float *I0, const float *I1,
                          double target_energy, int max_refine_iters, int chunk, int plain_iters,
                          float *hx, float *hy, float *hz, int *iters_run, int *fell_back,
                          void *stream);

#ifdef __cplusplus
}
#endif
#endif /* AW_B200_H */
