// capi.cu — the extern "C" boundary declared in include/aw_b200.h.
//
// Thin: argument checks, handle lifetime, error strings, and the CUDA-graph
// replay of the greedy loop. All arithmetic lives in the kernels.
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/aw_b200.h"
#include "atlas.cuh"
#include "greedy.cuh"
#include "interp.cuh"
#include "ldmm.cuh"
#include "multiscale.cuh"
#include "splat.cuh"

namespace {

thread_local std::string g_last_error;

int fail(const std::string &msg) {
  g_last_error = msg;
  return 1;
}

int cuda_fail(cudaError_t e, const char *what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return 2;
}

#define AW_CUDA(call, what)                        \
  do {                                             \
    cudaError_t _e = (call);                       \
    if (_e != cudaSuccess) return cuda_fail(_e, what); \
  } while (0)

bool dims_ok(int nx, int ny, int nz, std::string &why) {
  if (nx < 2 || ny < 2 || nz < 2) {
    why = "every grid axis must be >= 2";
    return false;
  }
  if (nx > 512 || ny > 512 || nz > 512) {
    why = "grid axes are limited to 512 (the reference's FFT LUT cap)";
    return false;
  }
  return true;
}

bool spacing_ok(double a, double b, double c) { return a > 0 && b > 0 && c > 0; }

const char *plan_error(int rc) {
  switch (rc) {
    case 1: return "unsupported grid size for the fluid FFT plan";
    case 2: return "z-slab spectrum does not fit in shared memory (nx*ny too large)";
    case 3: return "device allocation failed";
    default: return "kernel configuration failed";
  }
}

inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace

namespace aw {
void set_last_error(const std::string &msg) { g_last_error = msg; }
}  // namespace aw

struct aw_fluid_s {
  aw::FluidPlan plan;
};

struct GraphKey {
  const void *p[14];
  int n;
  bool operator<(const GraphKey &o) const {
    for (int i = 0; i < 14; ++i)
      if (p[i] != o.p[i]) return p[i] < o.p[i];
    return n < o.n;
  }
};

struct aw_ldmm_s {
  aw::LdmmCtx ctx;
  cudaStream_t gstream = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  std::map<std::pair<const void *, const void *>, std::pair<const void *, cudaGraphExec_t>> graphs;
};

struct aw_atlas_s {
  aw::AtlasCtx ctx;
};

struct aw_greedy_s {
  aw::GreedyCtx ctx;
  int auto_reduce = 0;
  cudaStream_t gstream = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  std::map<GraphKey, cudaGraphExec_t> graphs;
};

extern "C" {

const char *aw_last_error(void) { return g_last_error.c_str(); }

const char *aw_version(void) { return "atlaswerks_b200 0.1 (sm_100a)"; }

int aw_apply(const float *img, const float *hx, const float *hy, const float *hz, float *out,
             int nx, int ny, int nz, float background, void *stream) {
  std::string why;
  if (!img || !hx || !hy || !hz || !out) return fail("aw_apply: null pointer");
  if (nx < 1 || ny < 1 || nz < 1) return fail("aw_apply: empty grid");
  AW_CUDA(aw::launch_apply(img, hx, hy, hz, out, aw::Dims{nx, ny, nz}, background, S(stream)),
          "aw_apply");
  return 0;
}

int aw_gradient(const float *img, float *gx, float *gy, float *gz, int nx, int ny, int nz,
                double spx, double spy, double spz, int wrap, void *stream) {
  std::string why;
  if (!img || !gx || !gy || !gz) return fail("aw_gradient: null pointer");
  if (nx < 2 || ny < 2 || nz < 2) return fail("aw_gradient: every grid axis must be >= 2");
  if (!spacing_ok(spx, spy, spz)) return fail("aw_gradient: spacing must be positive");
  AW_CUDA(aw::launch_gradient(img, gx, gy, gz, aw::Dims{nx, ny, nz}, aw::Spacing{spx, spy, spz},
                              wrap, S(stream)),
          "aw_gradient");
  return 0;
}

int aw_compose_hv(const float *gx, const float *gy, const float *gz, const float *vx,
                  const float *vy, const float *vz, float *ox, float *oy, float *oz, int nx,
                  int ny, int nz, double spx, double spy, double spz, float scale, int direction,
                  int background, void *stream) {
  if (!gx || !gy || !gz || !vx || !vy || !vz || !ox || !oy || !oz)
    return fail("aw_compose_hv: null pointer");
  if (nx < 1 || ny < 1 || nz < 1) return fail("aw_compose_hv: empty grid");
  if (!spacing_ok(spx, spy, spz)) return fail("aw_compose_hv: spacing must be positive");
  if (background < 0 || background > 5) return fail("aw_compose_hv: unknown background strategy");
  const float *g[3] = {gx, gy, gz}, *v[3] = {vx, vy, vz};
  float *o[3] = {ox, oy, oz};
  AW_CUDA(aw::launch_compose_hv(g, v, o, aw::Dims{nx, ny, nz}, aw::Spacing{spx, spy, spz},
                                direction >= 0 ? 1 : -1, background, nullptr, scale, S(stream)),
          "aw_compose_hv");
  return 0;
}

int aw_compose_vh(const float *vx, const float *vy, const float *vz, const float *gx,
                  const float *gy, const float *gz, float *ox, float *oy, float *oz, int nx,
                  int ny, int nz, double spx, double spy, double spz, float scale, int direction,
                  int background, void *stream) {
  if (!gx || !gy || !gz || !vx || !vy || !vz || !ox || !oy || !oz)
    return fail("aw_compose_vh: null pointer");
  if (nx < 1 || ny < 1 || nz < 1) return fail("aw_compose_vh: empty grid");
  if (!spacing_ok(spx, spy, spz)) return fail("aw_compose_vh: spacing must be positive");
  if (background < 0 || background > 5) return fail("aw_compose_vh: unknown background strategy");
  const float *g[3] = {gx, gy, gz}, *v[3] = {vx, vy, vz};
  float *o[3] = {ox, oy, oz};
  AW_CUDA(aw::launch_compose_vh(v, g, o, aw::Dims{nx, ny, nz}, aw::Spacing{spx, spy, spz},
                                direction >= 0 ? 1 : -1, background, nullptr, scale, S(stream)),
          "aw_compose_vh");
  return 0;
}

int aw_splat(const float *img, const float *hx, const float *hy, const float *hz, float *out,
             int nx, int ny, int nz, float background, void *stream) {
  if (!img || !hx || !hy || !hz || !out) return fail("aw_splat: null pointer");
  if (nx < 1 || ny < 1 || nz < 1) return fail("aw_splat: empty grid");
  if ((long)(nx + 1) * (ny + 1) * (nz + 1) >= (1L << 31))
    return fail("aw_splat: grid too large for 32-bit bucket offsets");
  const aw::Dims d{nx, ny, nz};
  cudaStream_t s = S(stream);
  void *scratch = nullptr;
  AW_CUDA(cudaMallocAsync(&scratch, aw::splat_scratch_bytes(d), s), "aw_splat (scratch)");
  aw::SplatWork w;
  aw::splat_work_bind(&w, d, scratch);
  const cudaError_t e = aw::splat(w, img, hx, hy, hz, out, background, s);
  cudaFreeAsync(scratch, s);
  if (e != cudaSuccess) return cuda_fail(e, "aw_splat");
  return 0;
}

int aw_downsample(const float *in, int nx, int ny, int nz, double spx, double spy, double spz,
                  float *out, int mx, int my, int mz, void *stream) {
  if (!in || !out) return fail("aw_downsample: null pointer");
  if (nx < 2 || ny < 2 || nz < 2 || mx < 1 || my < 1 || mz < 1 || mx > nx || my > ny || mz > nz)
    return fail("aw_downsample: output grid must be non-empty and no larger than the input");
  if (!spacing_ok(spx, spy, spz)) return fail("aw_downsample: spacing must be positive");
  const aw::Dims din{nx, ny, nz}, dout{mx, my, mz};
  cudaStream_t s = S(stream);
  void *scratch = nullptr;
  AW_CUDA(cudaMallocAsync(&scratch, aw::downsample_scratch_bytes(din), s), "aw_downsample (scratch)");
  const cudaError_t e =
      aw::downsample(in, din, aw::Spacing{spx, spy, spz}, out, dout, scratch, s);
  cudaFreeAsync(scratch, s);
  if (e != cudaSuccess) return cuda_fail(e, "aw_downsample");
  return 0;
}

int aw_identity(float *hx, float *hy, float *hz, int nx, int ny, int nz, void *stream) {
  if (!hx || !hy || !hz) return fail("aw_identity: null pointer");
  if (nx < 1 || ny < 1 || nz < 1) return fail("aw_identity: empty grid");
  AW_CUDA(aw::identity_field(hx, hy, hz, aw::Dims{nx, ny, nz}, S(stream)), "aw_identity");
  return 0;
}

int aw_resample_image(const float *in, int nx, int ny, int nz, double sx, double sy, double sz,
                      float *out, int mx, int my, int mz, double tx, double ty, double tz,
                      void *stream) {
  if (!in || !out) return fail("aw_resample_image: null pointer");
  if (nx < 1 || ny < 1 || nz < 1 || mx < 1 || my < 1 || mz < 1)
    return fail("aw_resample_image: empty grid");
  if (!spacing_ok(sx, sy, sz) || !spacing_ok(tx, ty, tz))
    return fail("aw_resample_image: spacing must be positive");
  AW_CUDA(aw::resample_image(in, aw::Dims{nx, ny, nz}, aw::Spacing{sx, sy, sz}, out,
                             aw::Dims{mx, my, mz}, aw::Spacing{tx, ty, tz}, S(stream)),
          "aw_resample_image");
  return 0;
}

int aw_upsample_hfield(const float *hx, const float *hy, const float *hz, int nx, int ny, int nz,
                       float *ox, float *oy, float *oz, int mx, int my, int mz, int rescale,
                       void *stream) {
  if (!hx || !hy || !hz || !ox || !oy || !oz) return fail("aw_upsample_hfield: null pointer");
  if (nx < 1 || ny < 1 || nz < 1 || mx < 1 || my < 1 || mz < 1)
    return fail("aw_upsample_hfield: empty grid");
  const aw::Dims din{nx, ny, nz}, dout{mx, my, mz};
  cudaStream_t s = S(stream);
  void *scratch = nullptr;
  AW_CUDA(cudaMallocAsync(&scratch, sizeof(float) * 3 * din.n(), s), "aw_upsample_hfield (scratch)");
  const float *h[3] = {hx, hy, hz};
  float *o[3] = {ox, oy, oz};
  const cudaError_t e = aw::upsample_hfield(h, din, o, dout, rescale, scratch, s);
  cudaFreeAsync(scratch, s);
  if (e != cudaSuccess) return cuda_fail(e, "aw_upsample_hfield");
  return 0;
}

int aw_fluid_create(int nx, int ny, int nz, double spx, double spy, double spz, float alpha,
                    float beta, float gamma, aw_fluid_t *out) {
  std::string why;
  if (!out) return fail("aw_fluid_create: null handle pointer");
  *out = nullptr;
  if (!dims_ok(nx, ny, nz, why)) return fail("aw_fluid_create: " + why);
  if (!spacing_ok(spx, spy, spz)) return fail("aw_fluid_create: spacing must be positive");
  if (!(gamma > 0.0f) || alpha < 0.0f || beta < 0.0f)
    return fail("aw_fluid_create: need gamma > 0, alpha >= 0, beta >= 0 (L must be SPD)");
  aw_fluid_s *k = new (std::nothrow) aw_fluid_s;
  if (!k) return fail("aw_fluid_create: out of host memory");
  const int rc = aw::fluid_plan_create(&k->plan, nx, ny, nz, spx, spy, spz, alpha, beta, gamma);
  if (rc) {
    aw::fluid_plan_destroy(&k->plan);
    delete k;
    return fail(std::string("aw_fluid_create: ") + plan_error(rc));
  }
  *out = k;
  return 0;
}

int aw_fluid_apply(aw_fluid_t k, float *vx, float *vy, float *vz, int inverse, void *stream) {
  if (!k) return fail("aw_fluid_apply: null handle");
  if (!vx || !vy || !vz) return fail("aw_fluid_apply: null pointer");
  cudaStream_t s = S(stream);
  AW_CUDA(aw::fluid_forward_field(k->plan, vx, vy, vz, s), "aw_fluid_apply (xy forward)");
  AW_CUDA(aw::fluid_solve(k->plan, inverse ? 1 : 0, s), "aw_fluid_apply (z solve)");
  AW_CUDA(aw::fluid_inverse_store(k->plan, vx, vy, vz, s), "aw_fluid_apply (xy inverse)");
  return 0;
}

int aw_fluid_get_shapes(aw_fluid_t k, int *shapes) {
  if (!k || !shapes) return fail("aw_fluid_get_shapes: null pointer");
  // the register-FFT path reports {0, 0, z-pass tile width}
  aw::fluid_get_shapes(k->plan, shapes, shapes + 1, shapes + 2);
  return 0;
}

int aw_fluid_set_shapes(aw_fluid_t k, int pairs, int cols, int zcols) {
  if (!k) return fail("aw_fluid_set_shapes: null handle");
  AW_CUDA(cudaDeviceSynchronize(), "aw_fluid_set_shapes (pending work)");
  const cudaError_t e = aw::fluid_set_shapes(&k->plan, pairs, cols, zcols);
  if (e == cudaErrorInvalidValue)
    return fail(k->plan.fast ? "aw_fluid_set_shapes: power-of-two grids take (0, 0, 16 or 8)"
                             : "aw_fluid_set_shapes: shapes out of range or beyond shared memory");
  AW_CUDA(e, "aw_fluid_set_shapes");
  return 0;
}

int aw_fluid_autotune(aw_fluid_t k, void *stream) {
  if (!k) return fail("aw_fluid_autotune: null handle");
  AW_CUDA(aw::fluid_autotune(&k->plan, S(stream)), "aw_fluid_autotune");
  return 0;
}

int aw_fluid_status(aw_fluid_t k, int *timed_out, void *stream) {
  if (!k || !timed_out) return fail("aw_fluid_status: null pointer");
  AW_CUDA(aw::fluid_take_status(&k->plan, timed_out, S(stream)), "aw_fluid_status");
  return 0;
}

int aw_fluid_wait_selftest(aw_fluid_t k, int polls, void *stream) {
  if (!k) return fail("aw_fluid_wait_selftest: null handle");
  if (polls < 1 || polls > 4096) return fail("aw_fluid_wait_selftest: polls must be in [1, 4096]");
  AW_CUDA(aw::fluid_wait_selftest(k->plan, polls, S(stream)), "aw_fluid_wait_selftest");
  return 0;
}

int aw_fluid_destroy(aw_fluid_t k) {
  if (!k) return 0;
  aw::fluid_plan_destroy(&k->plan);
  delete k;
  return 0;
}

int aw_greedy_create(int nx, int ny, int nz, double spx, double spy, double spz, float alpha,
                     float beta, float gamma, float max_pert, aw_greedy_t *out) {
  std::string why;
  if (!out) return fail("aw_greedy_create: null handle pointer");
  *out = nullptr;
  if (!dims_ok(nx, ny, nz, why)) return fail("aw_greedy_create: " + why);
  if (!spacing_ok(spx, spy, spz)) return fail("aw_greedy_create: spacing must be positive");
  if (!(gamma > 0.0f) || alpha < 0.0f || beta < 0.0f)
    return fail("aw_greedy_create: need gamma > 0, alpha >= 0, beta >= 0 (L must be SPD)");
  if (!(max_pert > 0.0f)) return fail("aw_greedy_create: MaxPert must be positive");
  aw_greedy_s *g = new (std::nothrow) aw_greedy_s;
  if (!g) return fail("aw_greedy_create: out of host memory");
  const int rc =
      aw::greedy_create(&g->ctx, nx, ny, nz, spx, spy, spz, alpha, beta, gamma, max_pert, 4096);
  if (rc) {
    aw::greedy_destroy(&g->ctx);
    delete g;
    return fail(std::string("aw_greedy_create: ") + plan_error(rc));
  }
  if (cudaStreamCreateWithFlags(&g->gstream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&g->ev_in, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&g->ev_out, cudaEventDisableTiming) != cudaSuccess) {
    aw::greedy_destroy(&g->ctx);
    delete g;
    return fail("aw_greedy_create: stream/event creation failed");
  }
  *out = g;
  return 0;
}

int aw_greedy_destroy(aw_greedy_t g) {
  if (!g) return 0;
  cudaDeviceSynchronize();
  for (auto &kv : g->graphs) cudaGraphExecDestroy(kv.second);
  if (g->gstream) cudaStreamDestroy(g->gstream);
  if (g->ev_in) cudaEventDestroy(g->ev_in);
  if (g->ev_out) cudaEventDestroy(g->ev_out);
  aw::greedy_destroy(&g->ctx);
  delete g;
  return 0;
}

int aw_greedy_set_step(aw_greedy_t g, float step) {
  if (!g) return fail("aw_greedy_set_step: null handle");
  AW_CUDA(cudaMemcpy(g->ctx.st.step, &step, sizeof(float), cudaMemcpyHostToDevice),
          "aw_greedy_set_step");
  return 0;
}

int aw_greedy_status(aw_greedy_t g, int *timed_out, void *stream) {
  if (!g || !timed_out) return fail("aw_greedy_status: null pointer");
  AW_CUDA(aw::fluid_take_status(&g->ctx.plan, timed_out, S(stream)), "aw_greedy_status");
  return 0;
}

int aw_greedy_get_step(aw_greedy_t g, float *step) {
  if (!g || !step) return fail("aw_greedy_get_step: null pointer");
  AW_CUDA(cudaDeviceSynchronize(), "aw_greedy_get_step (pending work)");
  AW_CUDA(cudaMemcpy(step, g->ctx.st.step, sizeof(float), cudaMemcpyDeviceToHost),
          "aw_greedy_get_step");
  return 0;
}

int aw_greedy_set_auto_step_reduce(aw_greedy_t g, int on) {
  if (!g) return fail("aw_greedy_set_auto_step_reduce: null handle");
  g->auto_reduce = on ? 1 : 0;
  return 0;
}

int aw_greedy_set_staged_update(aw_greedy_t g, int on) {
  if (!g) return fail("aw_greedy_set_staged_update: null handle");
  AW_CUDA(cudaDeviceSynchronize(), "aw_greedy_set_staged_update (pending work)");
  g->ctx.no_staged_update = on ? 0 : 1;
  for (auto &kv : g->graphs) cudaGraphExecDestroy(kv.second);
  g->graphs.clear();  // captured iterations hold the other update kernel
  return 0;
}

int aw_greedy_set_fused_update(aw_greedy_t g, int on) {
  if (!g) return fail("aw_greedy_set_fused_update: null handle");
  AW_CUDA(cudaDeviceSynchronize(), "aw_greedy_set_fused_update (pending work)");
  g->ctx.no_fused_update = on ? 0 : 1;
  for (auto &kv : g->graphs) cudaGraphExecDestroy(kv.second);
  g->graphs.clear();  // captured iterations hold the other inverse/update kernels
  return 0;
}

int aw_greedy_set_fast_interpolation(aw_greedy_t g, int on) {
  if (!g) return fail("aw_greedy_set_fast_interpolation: null handle");
  AW_CUDA(cudaDeviceSynchronize(), "aw_greedy_set_fast_interpolation (pending work)");
  g->ctx.fast_interp = on ? 1 : 0;
  for (auto &kv : g->graphs) cudaGraphExecDestroy(kv.second);
  g->graphs.clear();  // captured iterations hold the other kernels
  return 0;
}

int aw_greedy_update_tile(aw_greedy_t g, int set, int *tile) {
  if (!g || !tile) return fail("aw_greedy_update_tile: null pointer");
  if (set) {
    if (*tile < 0 || *tile >= 4) return fail("aw_greedy_update_tile: tile index must be 0..3");
    AW_CUDA(cudaDeviceSynchronize(), "aw_greedy_update_tile (pending work)");
    g->ctx.utile = *tile;
    for (auto &kv : g->graphs) cudaGraphExecDestroy(kv.second);
    g->graphs.clear();  // captured iterations hold the other tile's kernel
  } else {
    *tile = g->ctx.utile;
  }
  return 0;
}

int aw_greedy_iterate(aw_greedy_t g, const float *I0, const float *I1, const float *hx,
                      const float *hy, const float *hz, float *ox, float *oy, float *oz,
                      const float *hix, const float *hiy, const float *hiz, float *hiox,
                      float *hioy, float *hioz, int update_step, void *stream) {
  if (!g) return fail("aw_greedy_iterate: null handle");
  if (!I0 || !I1 || !hx || !hy || !hz || !ox || !oy || !oz)
    return fail("aw_greedy_iterate: null pointer");
  if (ox == hx || oy == hy || oz == hz) return fail("aw_greedy_iterate: h_out must not alias h");
  const bool inv = hix != nullptr;
  if (inv && (!hiy || !hiz || !hiox || !hioy || !hioz))
    return fail("aw_greedy_iterate: incomplete inverse field pointers");
  if (inv && (hiox == hix || hioy == hiy || hioz == hiz))
    return fail("aw_greedy_iterate: hinv_out must not alias hinv");
  const float *h[3] = {hx, hy, hz}, *hi[3] = {hix, hiy, hiz};
  float *o[3] = {ox, oy, oz}, *hio[3] = {hiox, hioy, hioz};
  AW_CUDA(aw::greedy_iterate(&g->ctx, I0, I1, h, o, inv ? hi : nullptr, inv ? hio : nullptr,
                             update_step, g->auto_reduce, S(stream)),
          "aw_greedy_iterate");
  return 0;
}

int aw_greedy_run(aw_greedy_t g, const float *I0, const float *I1, float *hx, float *hy,
                  float *hz, float *sx, float *sy, float *sz, float *hix, float *hiy, float *hiz,
                  float *six, float *siy, float *siz, int n_iters, int update_first,
                  void *stream) {
  if (!g) return fail("aw_greedy_run: null handle");
  if (!I0 || !I1 || !hx || !hy || !hz || !sx || !sy || !sz)
    return fail("aw_greedy_run: null pointer");
  if (n_iters < 0) return fail("aw_greedy_run: negative iteration count");
  const bool inv = hix != nullptr;
  if (inv && (!hiy || !hiz || !six || !siy || !siz))
    return fail("aw_greedy_run: incomplete inverse field pointers");
  if (n_iters == 0) return 0;
  cudaStream_t user = S(stream);
  cudaStream_t s = g->gstream;
  AW_CUDA(cudaEventRecord(g->ev_in, user), "aw_greedy_run (event)");
  AW_CUDA(cudaStreamWaitEvent(s, g->ev_in, 0), "aw_greedy_run (wait)");
  float *A[3] = {hx, hy, hz}, *B[3] = {sx, sy, sz};
  float *AI[3] = {hix, hiy, hiz}, *BI[3] = {six, siy, siz};
  int done = 0;
  bool in_a = true;
  auto one = [&](int upd) -> cudaError_t {
    float **src = in_a ? A : B, **dst = in_a ? B : A;
    float **isrc = in_a ? AI : BI, **idst = in_a ? BI : AI;
    const float *cs[3] = {src[0], src[1], src[2]}, *ci[3] = {isrc[0], isrc[1], isrc[2]};
    cudaError_t e = aw::greedy_iterate(&g->ctx, I0, I1, cs, dst, inv ? ci : nullptr,
                                       inv ? idst : nullptr, upd, g->auto_reduce, s);
    in_a = !in_a;
    return e;
  };
  if (update_first) {
    AW_CUDA(one(1), "aw_greedy_run (first iteration)");
    ++done;
  }
  // replay a captured pair of iterations (src->dst->src) as often as possible
  const int pairs = (n_iters - done) / 2;
  if (pairs > 0) {
    GraphKey key;
    std::memset(&key, 0, sizeof(key));
    float **src = in_a ? A : B, **dst = in_a ? B : A;
    float **isrc = in_a ? AI : BI, **idst = in_a ? BI : AI;
    const void *ptrs[14] = {I0,      I1,      src[0],  src[1],  src[2],  dst[0],  dst[1],
                            dst[2],  isrc[0], isrc[1], isrc[2], idst[0], idst[1], idst[2]};
    for (int i = 0; i < 14; ++i) key.p[i] = ptrs[i];
    key.n = 2;
    auto it = g->graphs.find(key);
    cudaGraphExec_t exec = nullptr;
    if (it == g->graphs.end()) {
      cudaGraph_t graph;
      AW_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "aw_greedy_run (capture)");
      const bool start = in_a;
      cudaError_t e1 = one(0), e2 = one(0);
      cudaError_t ec = cudaStreamEndCapture(s, &graph);
      in_a = start;
      if (e1 != cudaSuccess) return cuda_fail(e1, "aw_greedy_run (captured iteration)");
      if (e2 != cudaSuccess) return cuda_fail(e2, "aw_greedy_run (captured iteration)");
      if (ec != cudaSuccess) return cuda_fail(ec, "aw_greedy_run (end capture)");
      AW_CUDA(cudaGraphInstantiate(&exec, graph, 0), "aw_greedy_run (instantiate)");
      cudaGraphDestroy(graph);
      g->graphs[key] = exec;
    } else {
      exec = it->second;
    }
    for (int p = 0; p < pairs; ++p) AW_CUDA(cudaGraphLaunch(exec, s), "aw_greedy_run (launch)");
    done += 2 * pairs;
  }
  if (done < n_iters) {
    AW_CUDA(one(0), "aw_greedy_run (last iteration)");
    ++done;
  }
  if (!in_a) {  // final field is in the scratch buffers: bring it home
    const size_t bytes = sizeof(float) * (size_t)g->ctx.d.n();
    for (int c = 0; c < 3; ++c) {
      AW_CUDA(cudaMemcpyAsync(A[c], B[c], bytes, cudaMemcpyDeviceToDevice, s), "aw_greedy_run (copy)");
      if (inv) AW_CUDA(cudaMemcpyAsync(AI[c], BI[c], bytes, cudaMemcpyDeviceToDevice, s), "aw_greedy_run (copy)");
    }
  }
  AW_CUDA(cudaEventRecord(g->ev_out, s), "aw_greedy_run (event)");
  AW_CUDA(cudaStreamWaitEvent(user, g->ev_out, 0), "aw_greedy_run (wait)");
  return 0;
}

int aw_greedy_profile(aw_greedy_t g, const float *I0, const float *I1, const float *hx,
                      const float *hy, const float *hz, float *ox, float *oy, float *oz,
                      const float *hix, const float *hiy, const float *hiz, float *hiox,
                      float *hioy, float *hioz, int reps, void *stream, float *ms_out) {
  if (!g || !ms_out) return fail("aw_greedy_profile: null pointer");
  if (!I0 || !I1 || !hx || !hy || !hz || !ox || !oy || !oz)
    return fail("aw_greedy_profile: null pointer");
  if (reps < 1) return fail("aw_greedy_profile: reps must be >= 1");
  const bool inv = hix != nullptr;
  const float *h[3] = {hx, hy, hz}, *hi[3] = {hix, hiy, hiz};
  float *o[3] = {ox, oy, oz}, *hio[3] = {hiox, hioy, hioz};
  cudaStream_t s = S(stream);
  cudaEvent_t e0, e1;
  AW_CUDA(cudaEventCreate(&e0), "aw_greedy_profile (event)");
  AW_CUDA(cudaEventCreate(&e1), "aw_greedy_profile (event)");
  int rc = 0;
  for (int stage = 0; stage < aw::kNumStages && rc == 0; ++stage) {
    cudaError_t e = cudaEventRecord(e0, s);
    for (int r = 0; r < reps && e == cudaSuccess; ++r)
      e = aw::greedy_stage(&g->ctx, stage, I0, I1, h, o, inv ? hi : nullptr, inv ? hio : nullptr,
                           0, (r & 1) ? 0 : 1, s);
    // an even number of solves leaves the spectrum at its original scale
    if (e == cudaSuccess && stage == aw::kStageZSolve && (reps & 1))
      e = aw::greedy_stage(&g->ctx, stage, I0, I1, h, o, nullptr, nullptr, 0, 0, s);
    if (e == cudaSuccess) e = cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e != cudaSuccess) rc = cuda_fail(e, "aw_greedy_profile");
    ms_out[stage] = ms / reps;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

static int copy_energies(const aw::GreedyDevState &st, double *out, int max_count, int *count,
                         const char *what) {
  AW_CUDA(cudaDeviceSynchronize(), what);
  int n = 0;
  AW_CUDA(cudaMemcpy(&n, st.count, sizeof(int), cudaMemcpyDeviceToHost), what);
  const int cap = st.cap;
  const int avail = n < cap ? n : cap;
  std::vector<double> ring(cap);
  AW_CUDA(cudaMemcpy(ring.data(), st.energy, sizeof(double) * cap, cudaMemcpyDeviceToHost), what);
  const int m = (out && max_count < avail) ? max_count : avail;
  for (int i = 0; i < m && out; ++i) out[i] = ring[(n - avail + i) % cap];
  *count = avail;
  return 0;
}

int aw_greedy_last_energy(aw_greedy_t g, double *energy) {
  if (!g || !energy) return fail("aw_greedy_last_energy: null pointer");
  const aw::GreedyDevState &st = g->ctx.st;
  int n = 0;
  // cudaMemcpy on the legacy stream waits for the iteration that records it
  AW_CUDA(cudaMemcpy(&n, st.count, sizeof(int), cudaMemcpyDeviceToHost), "aw_greedy_last_energy");
  if (n < 1) return fail("aw_greedy_last_energy: no energy recorded yet");
  AW_CUDA(cudaMemcpy(energy, st.energy + (n - 1) % st.cap, sizeof(double), cudaMemcpyDeviceToHost),
          "aw_greedy_last_energy");
  return 0;
}

int aw_greedy_get_energies(aw_greedy_t g, double *out, int max_count, int *count) {
  if (!g || !count) return fail("aw_greedy_get_energies: null pointer");
  return copy_energies(g->ctx.st, out, max_count, count, "aw_greedy_get_energies");
}

int aw_atlas_create(int nx, int ny, int nz, double spx, double spy, double spz, float alpha,
                    float beta, float gamma, float max_pert, int n_subjects, aw_atlas_t *out) {
  std::string why;
  if (!out) return fail("aw_atlas_create: null handle pointer");
  *out = nullptr;
  if (!dims_ok(nx, ny, nz, why)) return fail("aw_atlas_create: " + why);
  if (!spacing_ok(spx, spy, spz)) return fail("aw_atlas_create: spacing must be positive");
  if (!(gamma > 0.0f) || alpha < 0.0f || beta < 0.0f)
    return fail("aw_atlas_create: need gamma > 0, alpha >= 0, beta >= 0 (L must be SPD)");
  if (!(max_pert > 0.0f)) return fail("aw_atlas_create: MaxPert must be positive");
  if (n_subjects < 1) return fail("aw_atlas_create: need at least one subject");
  aw_atlas_s *a = new (std::nothrow) aw_atlas_s;
  if (!a) return fail("aw_atlas_create: out of host memory");
  const int rc = aw::atlas_create(&a->ctx, nx, ny, nz, spx, spy, spz, alpha, beta, gamma,
                                  max_pert, n_subjects);
  if (rc) {
    aw::atlas_destroy(&a->ctx);
    delete a;
    return fail(std::string("aw_atlas_create: ") +
                (rc == 5 ? "stream/event/copy setup failed" : plan_error(rc)));
  }
  *out = a;
  return 0;
}

int aw_atlas_destroy(aw_atlas_t a) {
  if (!a) return 0;
  aw::atlas_destroy(&a->ctx);
  delete a;
  return 0;
}

int aw_atlas_set_subject(aw_atlas_t a, int i, const float *img, int snx, int sny, int snz,
                         float weight) {
  if (!a || !img) return fail("aw_atlas_set_subject: null pointer");
  if (i < 0 || i >= a->ctx.ns) return fail("aw_atlas_set_subject: subject index out of range");
  if (snx < 2 || sny < 2 || snz < 2) return fail("aw_atlas_set_subject: every grid axis must be >= 2");
  AW_CUDA(aw::atlas_set_subject(&a->ctx, i, img, aw::Dims{snx, sny, snz}, weight),
          "aw_atlas_set_subject");
  return 0;
}

int aw_atlas_field(aw_atlas_t a, int i, float **hx, float **hy, float **hz) {
  if (!a || !hx || !hy || !hz) return fail("aw_atlas_field: null pointer");
  if (i < 0 || i >= a->ctx.ns) return fail("aw_atlas_field: subject index out of range");
  *hx = aw::atlas_field(&a->ctx, i, 0);
  *hy = aw::atlas_field(&a->ctx, i, 1);
  *hz = aw::atlas_field(&a->ctx, i, 2);
  return 0;
}

int aw_atlas_mean_buffer(aw_atlas_t a, float **mean) {
  if (!a || !mean) return fail("aw_atlas_mean_buffer: null pointer");
  *mean = a->ctx.mean;
  return 0;
}

static bool atlas_ready(aw_atlas_t a) {
  for (int r : a->ctx.ready)
    if (!r) return false;
  return true;
}

int aw_atlas_compute_mean(aw_atlas_t a, void *stream) {
  if (!a) return fail("aw_atlas_compute_mean: null handle");
  if (!atlas_ready(a)) return fail("aw_atlas_compute_mean: a subject image is not set");
  AW_CUDA(aw::atlas_mean(&a->ctx, S(stream)), "aw_atlas_compute_mean");
  return 0;
}

int aw_atlas_iterate(aw_atlas_t a, int n_iters, int update_first, void *stream) {
  if (!a) return fail("aw_atlas_iterate: null handle");
  if (n_iters < 0) return fail("aw_atlas_iterate: negative iteration count");
  if (!atlas_ready(a)) return fail("aw_atlas_iterate: a subject image is not set");
  AW_CUDA(aw::atlas_iterate(&a->ctx, n_iters, update_first, S(stream)), "aw_atlas_iterate");
  return 0;
}

int aw_atlas_get_step(aw_atlas_t a, int i, float *step) {
  if (!a || !step) return fail("aw_atlas_get_step: null pointer");
  if (i < 0 || i >= a->ctx.ns) return fail("aw_atlas_get_step: subject index out of range");
  AW_CUDA(cudaDeviceSynchronize(), "aw_atlas_get_step (pending work)");
  AW_CUDA(cudaMemcpy(step, a->ctx.subj[i].st.step, sizeof(float), cudaMemcpyDeviceToHost),
          "aw_atlas_get_step");
  return 0;
}

int aw_atlas_get_energies(aw_atlas_t a, int i, double *out, int max_count, int *count) {
  if (!a || !count) return fail("aw_atlas_get_energies: null pointer");
  if (i < 0 || i >= a->ctx.ns) return fail("aw_atlas_get_energies: subject index out of range");
  return copy_energies(a->ctx.subj[i].st, out, max_count, count, "aw_atlas_get_energies");
}

int aw_ldmm_create(int nx, int ny, int nz, double spx, double spy, double spz, float alpha,
                   float beta, float gamma, int n_time_steps, float sigma, float max_pert,
                   aw_ldmm_t *out) {
  std::string why;
  if (!out) return fail("aw_ldmm_create: null handle pointer");
  *out = nullptr;
  if (!dims_ok(nx, ny, nz, why)) return fail("aw_ldmm_create: " + why);
  if (!spacing_ok(spx, spy, spz)) return fail("aw_ldmm_create: spacing must be positive");
  if (!(gamma > 0.0f) || alpha < 0.0f || beta < 0.0f)
    return fail("aw_ldmm_create: need gamma > 0, alpha >= 0, beta >= 0 (L must be SPD)");
  if (n_time_steps < 1) return fail("aw_ldmm_create: NTimeSteps must be >= 1");
  if (!(sigma > 0.0f)) return fail("aw_ldmm_create: Sigma must be positive");
  aw_ldmm_s *l = new (std::nothrow) aw_ldmm_s;
  if (!l) return fail("aw_ldmm_create: out of host memory");
  const int rc = aw::ldmm_create(&l->ctx, nx, ny, nz, spx, spy, spz, alpha, beta, gamma,
                                 n_time_steps, sigma, max_pert);
  if (rc) {
    aw::ldmm_destroy(&l->ctx);
    delete l;
    return fail(std::string("aw_ldmm_create: ") + plan_error(rc));
  }
  if (cudaStreamCreateWithFlags(&l->gstream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&l->ev_in, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&l->ev_out, cudaEventDisableTiming) != cudaSuccess) {
    aw::ldmm_destroy(&l->ctx);
    delete l;
    return fail("aw_ldmm_create: stream/event creation failed");
  }
  *out = l;
  return 0;
}

int aw_ldmm_destroy(aw_ldmm_t l) {
  if (!l) return 0;
  cudaDeviceSynchronize();
  for (auto &kv : l->graphs) cudaGraphExecDestroy(kv.second.second);
  if (l->gstream) cudaStreamDestroy(l->gstream);
  if (l->ev_in) cudaEventDestroy(l->ev_in);
  if (l->ev_out) cudaEventDestroy(l->ev_out);
  aw::ldmm_destroy(&l->ctx);
  delete l;
  return 0;
}

int aw_ldmm_use_orig_gradient_calc(aw_ldmm_t l, int on) {
  if (!l) return fail("aw_ldmm_use_orig_gradient_calc: null handle");
  AW_CUDA(cudaDeviceSynchronize(), "aw_ldmm_use_orig_gradient_calc (pending work)");
  if (aw::ldmm_set_orig(&l->ctx, on)) return fail("aw_ldmm_use_orig_gradient_calc: device allocation failed");
  for (auto &kv : l->graphs) cudaGraphExecDestroy(kv.second.second);
  l->graphs.clear();  // captured iterations belong to the other variant
  return 0;
}

int aw_ldmm_set_vector_energy(aw_ldmm_t l, int on) {
  if (!l) return fail("aw_ldmm_set_vector_energy: null handle");
  AW_CUDA(cudaDeviceSynchronize(), "aw_ldmm_set_vector_energy (pending work)");
  l->ctx.vec_energy = on ? 1 : 0;
  for (auto &kv : l->graphs) cudaGraphExecDestroy(kv.second.second);
  l->graphs.clear();  // captured iterations belong to the other setting
  return 0;
}

int aw_ldmm_set_step(aw_ldmm_t l, float step) {
  if (!l) return fail("aw_ldmm_set_step: null handle");
  AW_CUDA(cudaMemcpy(l->ctx.step, &step, sizeof(float), cudaMemcpyHostToDevice),
          "aw_ldmm_set_step");
  return 0;
}

int aw_ldmm_status(aw_ldmm_t l, int *timed_out, void *stream) {
  if (!l || !timed_out) return fail("aw_ldmm_status: null pointer");
  AW_CUDA(aw::fluid_take_status(&l->ctx.plan, timed_out, S(stream)), "aw_ldmm_status");
  return 0;
}

int aw_ldmm_get_step(aw_ldmm_t l, float *step) {
  if (!l || !step) return fail("aw_ldmm_get_step: null pointer");
  AW_CUDA(cudaDeviceSynchronize(), "aw_ldmm_get_step (pending work)");
  AW_CUDA(cudaMemcpy(step, l->ctx.step, sizeof(float), cudaMemcpyDeviceToHost),
          "aw_ldmm_get_step");
  return 0;
}

int aw_ldmm_iterate(aw_ldmm_t l, const float *I0, const float *I1, float *v, int update_step,
                    void *stream) {
  if (!l) return fail("aw_ldmm_iterate: null handle");
  if (!I0 || !I1 || !v) return fail("aw_ldmm_iterate: null pointer");
  AW_CUDA(aw::ldmm_iterate(&l->ctx, I0, I1, v, update_step, S(stream)), "aw_ldmm_iterate");
  return 0;
}

int aw_ldmm_alphas(aw_ldmm_t l, const float *I0, const float *I1, const float *v, float *alphas,
                   void *stream) {
  if (!l) return fail("aw_ldmm_alphas: null handle");
  if (!I0 || !I1 || !v || !alphas) return fail("aw_ldmm_alphas: null pointer");
  if (l->ctx.orig)
    return fail("aw_ldmm_alphas: the alphas come from the splatting gradient (IterateNew); "
                "switch aw_ldmm_use_orig_gradient_calc off");
  AW_CUDA(aw::ldmm_alphas(&l->ctx, I0, I1, v, alphas, S(stream)), "aw_ldmm_alphas");
  return 0;
}

int aw_ldmm_run(aw_ldmm_t l, const float *I0, const float *I1, float *v, int n_iters,
                int adaptive_first, void *stream) {
  if (!l) return fail("aw_ldmm_run: null handle");
  if (!I0 || !I1 || !v) return fail("aw_ldmm_run: null pointer");
  if (n_iters < 0) return fail("aw_ldmm_run: negative iteration count");
  cudaStream_t user = S(stream), s = l->gstream;
  AW_CUDA(cudaEventRecord(l->ev_in, user), "aw_ldmm_run (event)");
  AW_CUDA(cudaStreamWaitEvent(s, l->ev_in, 0), "aw_ldmm_run (wait)");
  if (adaptive_first) AW_CUDA(aw::ldmm_iterate(&l->ctx, I0, I1, v, 1, s), "aw_ldmm_run (step)");
  if (n_iters > 0) {
    const auto key = std::make_pair((const void *)I0, (const void *)I1);
    auto it = l->graphs.find(key);
    cudaGraphExec_t exec = nullptr;
    if (it != l->graphs.end() && it->second.first == v) {
      exec = it->second.second;
    } else {
      if (it != l->graphs.end()) {
        cudaGraphExecDestroy(it->second.second);
        l->graphs.erase(it);
      }
      cudaGraph_t graph;
      AW_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "aw_ldmm_run (capture)");
      const cudaError_t e1 = aw::ldmm_iterate(&l->ctx, I0, I1, v, 0, s);
      const cudaError_t ec = cudaStreamEndCapture(s, &graph);
      if (e1 != cudaSuccess) return cuda_fail(e1, "aw_ldmm_run (captured iteration)");
      if (ec != cudaSuccess) return cuda_fail(ec, "aw_ldmm_run (end capture)");
      AW_CUDA(cudaGraphInstantiate(&exec, graph, 0), "aw_ldmm_run (instantiate)");
      cudaGraphDestroy(graph);
      l->graphs[key] = std::make_pair((const void *)v, exec);
    }
    for (int k = 0; k < n_iters; ++k) AW_CUDA(cudaGraphLaunch(exec, s), "aw_ldmm_run (launch)");
  }
  AW_CUDA(cudaEventRecord(l->ev_out, s), "aw_ldmm_run (event)");
  AW_CUDA(cudaStreamWaitEvent(user, l->ev_out, 0), "aw_ldmm_run (wait)");
  return 0;
}

int aw_ldmm_i1_at_0(aw_ldmm_t l, const float *I1, const float *v, float *img, float *jacdet,
                    void *stream) {
  if (!l || !I1 || !v || !img) return fail("aw_ldmm_i1_at_0: null pointer");
  AW_CUDA(aw::ldmm_i1_at_0(&l->ctx, I1, v, img, jacdet, S(stream)), "aw_ldmm_i1_at_0");
  return 0;
}

int aw_ldmm_atlas_accumulate(float *acc, float *jacsum, const float *img, const float *jacdet,
                             float weight, long n, void *stream) {
  if (!acc || !img || (jacdet && !jacsum)) return fail("aw_ldmm_atlas_accumulate: null pointer");
  if (n < 0) return fail("aw_ldmm_atlas_accumulate: negative size");
  if (n == 0) return 0;
  AW_CUDA(aw::ldmm_atlas_accumulate(acc, jacsum, img, jacdet, weight, n, S(stream)),
          "aw_ldmm_atlas_accumulate");
  return 0;
}

int aw_ldmm_atlas_normalize(float *acc, const float *jacsum, long n, void *stream) {
  if (!acc || !jacsum) return fail("aw_ldmm_atlas_normalize: null pointer");
  if (n < 0) return fail("aw_ldmm_atlas_normalize: negative size");
  if (n == 0) return 0;
  AW_CUDA(aw::ldmm_atlas_normalize(acc, jacsum, n, S(stream)), "aw_ldmm_atlas_normalize");
  return 0;
}

int aw_ldmm_atlas_voxel_median(const float *const *images, int n_images, int k, int nx, int ny,
                               int nz, float *out, void *stream) {
  std::string why;
  if (!images || !out) return fail("aw_ldmm_atlas_voxel_median: null pointer");
  if (n_images < 1 || n_images > aw::kVoxelMedianMaxImages)
    return fail("aw_ldmm_atlas_voxel_median: n_images must be in [1, " +
                std::to_string(aw::kVoxelMedianMaxImages) + "]");
  if (k < 0 || k >= n_images) return fail("aw_ldmm_atlas_voxel_median: k must be in [0, n_images)");
  if (nx < 1 || ny < 1 || nz < 1) return fail("aw_ldmm_atlas_voxel_median: empty grid");
  aw::VoxelImages in{};
  for (int m = 0; m < n_images; ++m) {
    if (!images[m]) return fail("aw_ldmm_atlas_voxel_median: null image pointer");
    in.img[m] = images[m];
  }
  cudaStream_t s = S(stream);
  void *scratch = nullptr;
  AW_CUDA(cudaMallocAsync(&scratch, 4 * sizeof(unsigned), s), "aw_ldmm_atlas_voxel_median (scratch)");
  unsigned *range = static_cast<unsigned *>(scratch);
  int *open = reinterpret_cast<int *>(range + 2);
  cudaError_t e = aw::ldmm_voxel_median(in, n_images, k, (long)nx * ny * nz, out, range, open, s);
  int h_open = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_open, open, sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(scratch, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  AW_CUDA(e, "aw_ldmm_atlas_voxel_median");
  if (h_open) return fail("aw_ldmm_atlas_voxel_median: the per-voxel selection did not converge");
  return 0;
}

int aw_ldmm_shoot_iterate(aw_ldmm_t l, const float *I0, const float *I1, float *alpha0,
                          float *phi0T, float *phiT0, void *stream) {
  if (!l || !I0 || !I1 || !alpha0 || !phi0T || !phiT0)
    return fail("aw_ldmm_shoot_iterate: null pointer");
  if (aw::ldmm_shoot_prepare(&l->ctx))
    return fail("aw_ldmm_shoot_iterate: device allocation failed");
  AW_CUDA(aw::ldmm_shoot_iterate(&l->ctx, I0, I1, alpha0, phi0T, phiT0, S(stream)),
          "aw_ldmm_shoot_iterate");
  return 0;
}

int aw_ldmm_velshoot_iterate(aw_ldmm_t l, const float *I0, const float *I1, float *v0,
                             float *phi0T, float *phiT0, int update_step, void *stream) {
  if (!l || !I0 || !I1 || !v0 || !phi0T || !phiT0)
    return fail("aw_ldmm_velshoot_iterate: null pointer");
  if (aw::ldmm_velshoot_prepare(&l->ctx))
    return fail("aw_ldmm_velshoot_iterate: device allocation failed");
  AW_CUDA(aw::ldmm_velshoot_iterate(&l->ctx, I0, I1, v0, phi0T, phiT0, update_step ? 1 : 0,
                                    S(stream)),
          "aw_ldmm_velshoot_iterate");
  return 0;
}

int aw_ldmm_geodesic_shoot(aw_ldmm_t l, const float *I0, const float *alpha0, float *phi0T,
                           float *phiT0, float *image, void *stream) {
  if (!l || !I0 || !alpha0 || !phi0T || !phiT0 || !image)
    return fail("aw_ldmm_geodesic_shoot: null pointer");
  AW_CUDA(aw::ldmm_geodesic_shoot(&l->ctx, I0, alpha0, phi0T, phiT0, image, S(stream)),
          "aw_ldmm_geodesic_shoot");
  return 0;
}

int aw_ldmm_adshoot_iterate(aw_ldmm_t l, const float *I0, const float *I1, float *alpha0,
                            float *phi0T, float *phiT0, void *stream) {
  if (!l || !I0 || !I1 || !alpha0 || !phi0T || !phiT0)
    return fail("aw_ldmm_adshoot_iterate: null pointer");
  if (l->ctx.T + 1 > aw::kMaxAdSorts)
    return fail("aw_ldmm_adshoot_iterate: at most " + std::to_string(aw::kMaxAdSorts - 1) +
                " time steps");
  if (aw::ldmm_adshoot_prepare(&l->ctx))
    return fail("aw_ldmm_adshoot_iterate: device allocation failed");
  AW_CUDA(aw::ldmm_adshoot_iterate(&l->ctx, I0, I1, alpha0, phi0T, phiT0, S(stream)),
          "aw_ldmm_adshoot_iterate");
  return 0;
}

int aw_ldmm_adshoot_final_maps(aw_ldmm_t l, float *phi0T, float *phiT0, void *stream) {
  if (!l || !phi0T || !phiT0) return fail("aw_ldmm_adshoot_final_maps: null pointer");
  if (!l->ctx.adV) return fail("aw_ldmm_adshoot_final_maps: no adjoint shooting iteration yet");
  AW_CUDA(aw::ldmm_adshoot_final_maps(&l->ctx, phi0T, phiT0, S(stream)),
          "aw_ldmm_adshoot_final_maps");
  return 0;
}

namespace {
// the last min(count, cap) entries of a device ring, oldest first
int read_ring(aw_ldmm_t l, const double *ring_dev, double *out, int max_count, int *count,
              const char *who) {
  AW_CUDA(cudaDeviceSynchronize(), who);
  int n = 0;
  AW_CUDA(cudaMemcpy(&n, l->ctx.count, sizeof(int), cudaMemcpyDeviceToHost), who);
  const int cap = l->ctx.cap;
  const int avail = n < cap ? n : cap;
  std::vector<double> ring(cap);
  AW_CUDA(cudaMemcpy(ring.data(), ring_dev, sizeof(double) * cap, cudaMemcpyDeviceToHost), who);
  const int m = (out && max_count < avail) ? max_count : avail;
  for (int i = 0; i < m && out; ++i) out[i] = ring[(n - avail + i) % cap];
  *count = avail;
  return 0;
}
}  // namespace

int aw_ldmm_get_vec_energies(aw_ldmm_t l, double *out, int max_count, int *count) {
  if (!l || !count) return fail("aw_ldmm_get_vec_energies: null pointer");
  return read_ring(l, l->ctx.venergy, out, max_count, count, "aw_ldmm_get_vec_energies");
}

int aw_ldmm_get_vec_step_energies(aw_ldmm_t l, double *out, int n_time_steps) {
  if (!l || !out) return fail("aw_ldmm_get_vec_step_energies: null pointer");
  if (n_time_steps != l->ctx.T)
    return fail("aw_ldmm_get_vec_step_energies: n_time_steps must be the handle's T");
  AW_CUDA(cudaMemcpy(out, l->ctx.vstep, sizeof(double) * l->ctx.T, cudaMemcpyDeviceToHost),
          "aw_ldmm_get_vec_step_energies");
  return 0;
}

int aw_ldmm_get_energies(aw_ldmm_t l, double *out, int max_count, int *count) {
  if (!l || !count) return fail("aw_ldmm_get_energies: null pointer");
  return read_ring(l, l->ctx.energy, out, max_count, count, "aw_ldmm_get_energies");
}

}  // extern "C"
