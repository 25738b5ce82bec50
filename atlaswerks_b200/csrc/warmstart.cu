// warmstart.cu — the learned warm start behind the C ABI (aw_warmstart_*):
// the encoder-decoder's forward pass on the tensor-core convolution kernels,
// captured once per handle as a CUDA graph, the pair's Gaussian downsampling
// to the network's grid and the upsampling of the predicted deformation,
// and the refinement loop with its fallback to the plain greedy solve.
// The network has no counterpart in the reference; the refinement is the
// reference's greedy iteration (GreedyIteratorGPU::Iterate) started from
// the prediction instead of the identity.
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/aw_b200.h"
#include "capi_error.h"
#include "multiscale.cuh"

namespace {

// (input channels, output channels, taps, level) of the 15 layers, in the
// order their parameters are packed: 3x3x3 convolutions with ReLU, two per
// level down (16, 32, 64, 128 channels), two per level up after the skip
// concatenation, and the 1x1x1 head (16 channels, 3 used, no ReLU)
struct Layer {
  int ci, co, taps, level;
};
constexpr int kLayers = 15;
constexpr Layer kNet[kLayers] = {
    {16, 16, 27, 0},  {16, 16, 27, 0},  {16, 32, 27, 1},   {32, 32, 27, 1},  {32, 64, 27, 2},
    {64, 64, 27, 2},  {64, 128, 27, 3}, {128, 128, 27, 3}, {192, 64, 27, 2}, {64, 64, 27, 2},
    {96, 32, 27, 1},  {32, 32, 27, 1},  {48, 16, 27, 0},   {16, 16, 27, 0},  {16, 16, 1, 0}};

size_t layer_params(const Layer &l) { return (size_t)l.co * l.taps * l.ci + l.co; }

int wfail(const std::string &m) {
  aw::set_last_error(m);
  return 1;
}

#define WS_TRY(call)                 \
  do {                               \
    if (int _rc = (call)) return _rc; \
  } while (0)

#define WS_CUDA(call, what)                                                  \
  do {                                                                       \
    cudaError_t _e = (call);                                                 \
    if (_e != cudaSuccess)                                                   \
      return wfail(std::string(what) + ": " + cudaGetErrorString(_e));      \
  } while (0)

}  // namespace

struct aw_warmstart_s {
  int nx, ny, nz;            // pair grid
  int D, H, W;               // network grid (z, y, x)
  bool coarse;               // network grid differs from the pair grid
  cudaStream_t s = nullptr;  // private stream the graph is captured on
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  // device memory: one block
  char *block = nullptr;
  void *wb[kLayers];         // BF16 weights [co][taps][ci]
  float *bias[kLayers];
  void *act[24];             // BF16 activations, channels last
  float *out = nullptr;      // FP32 head output [V][16]
  float *cscratch = nullptr;
  size_t cfloats = 0;
  float *I0c = nullptr, *I1c = nullptr;  // the pair on the network grid
  float *hc = nullptr;       // predicted h on the network grid, 3 planes
  void *dscratch = nullptr;  // downsampling scratch
  float *uscratch = nullptr; // upsampling scratch
  const float *in0 = nullptr, *in1 = nullptr;  // pointers the graph was captured with
  float *hout[3] = {nullptr, nullptr, nullptr};
  cudaGraphExec_t graph = nullptr;
  aw_greedy_t refine = nullptr;  // greedy handle on the pair grid (refinement, fallback)
  float *scratch_h = nullptr;    // 3N: the refinement's ping-pong field
  float max_pert = 0.f;
};

namespace {

long vox(const aw_warmstart_s *w, int level) {
  return (long)(w->D >> level) * (w->H >> level) * (w->W >> level);
}

// the forward pass of the network on the pair already on the network grid
// (I0c, I1c), then h = x + u on that grid
int forward(aw_warmstart_s *w) {
  cudaStream_t s = w->s;
  void *const *a = w->act;
  auto conv = [&](int l, const void *x, void *y, float *yf) -> int {
    const Layer &L = kNet[l];
    const int f = 1 << L.level;
    return aw_nn_conv3d_fwd(x, 1, w->D / f, w->H / f, w->W / f, L.ci, w->wb[l], w->bias[l], L.co,
                            L.taps, l == kLayers - 1 ? 0 : 1, y, yf, w->cscratch, w->cfloats, s);
  };
  auto pool = [&](const void *x, int level, int c, void *y) {
    const int f = 1 << level;
    return aw_nn_pool(x, 1, w->D / f, w->H / f, w->W / f, c, y, 0, nullptr, nullptr, s);
  };
  auto up = [&](const void *x, int level, int c, void *y, int ct) {
    const int f = 1 << level;
    return aw_nn_upsample(x, 1, w->D / f, w->H / f, w->W / f, c, y, ct, 0, 0, s);
  };
  // activation slots: 0 x, 1 e0a, 2 e0b, 3 p0, 4 e1a, 5 e1b, 6 p1, 7 e2a, 8 e2b, 9 p2,
  // 10 e3a, 11 e3b, 12 c2, 13 d2a, 14 d2b, 15 c1, 16 d1a, 17 d1b, 18 c0, 19 d0a, 20 d0b
  WS_TRY(aw_nn_pack_pair(w->I0c, w->I1c, vox(w, 0), a[0], s));
  WS_TRY(conv(0, a[0], a[1], nullptr));
  WS_TRY(conv(1, a[1], a[2], nullptr));
  WS_TRY(pool(a[2], 0, 16, a[3]));
  WS_TRY(conv(2, a[3], a[4], nullptr));
  WS_TRY(conv(3, a[4], a[5], nullptr));
  WS_TRY(pool(a[5], 1, 32, a[6]));
  WS_TRY(conv(4, a[6], a[7], nullptr));
  WS_TRY(conv(5, a[7], a[8], nullptr));
  WS_TRY(pool(a[8], 2, 64, a[9]));
  WS_TRY(conv(6, a[9], a[10], nullptr));
  WS_TRY(conv(7, a[10], a[11], nullptr));
  WS_TRY(up(a[11], 3, 128, a[12], 192));
  WS_TRY(aw_nn_slice(a[8], 64, 0, a[12], 192, 128, 64, vox(w, 2), 0, s));
  WS_TRY(conv(8, a[12], a[13], nullptr));
  WS_TRY(conv(9, a[13], a[14], nullptr));
  WS_TRY(up(a[14], 2, 64, a[15], 96));
  WS_TRY(aw_nn_slice(a[5], 32, 0, a[15], 96, 64, 32, vox(w, 1), 0, s));
  WS_TRY(conv(10, a[15], a[16], nullptr));
  WS_TRY(conv(11, a[16], a[17], nullptr));
  WS_TRY(up(a[17], 1, 32, a[18], 48));
  WS_TRY(aw_nn_slice(a[2], 16, 0, a[18], 48, 32, 16, vox(w, 0), 0, s));
  WS_TRY(conv(12, a[18], a[19], nullptr));
  WS_TRY(conv(13, a[19], a[20], nullptr));
  WS_TRY(conv(14, a[20], nullptr, w->out));
  const long n = vox(w, 0);
  return aw_nn_displacement_to_h(w->out, w->D, w->H, w->W, w->hc, w->hc + n, w->hc + 2 * n, s);
}

// the whole prediction: pair -> network grid, forward, h back to the pair grid
int predict_body(aw_warmstart_s *w, const float *I0, const float *I1, float *const hout[3]) {
  cudaStream_t s = w->s;
  const aw::Dims fine{w->nx, w->ny, w->nz}, net{w->W, w->H, w->D};
  const long nf = fine.n(), nc = net.n();
  if (w->coarse) {
    const aw::Spacing unit{1.0, 1.0, 1.0};
    WS_CUDA(aw::downsample(I0, fine, unit, w->I0c, net, w->dscratch, s), "aw_warmstart (downsample)");
    WS_CUDA(aw::downsample(I1, fine, unit, w->I1c, net, w->dscratch, s), "aw_warmstart (downsample)");
  } else {
    WS_CUDA(cudaMemcpyAsync(w->I0c, I0, sizeof(float) * nf, cudaMemcpyDeviceToDevice, s),
            "aw_warmstart (copy)");
    WS_CUDA(cudaMemcpyAsync(w->I1c, I1, sizeof(float) * nf, cudaMemcpyDeviceToDevice, s),
            "aw_warmstart (copy)");
  }
  WS_TRY(forward(w));
  const float *hc[3] = {w->hc, w->hc + nc, w->hc + 2 * nc};
  if (w->coarse) {
    WS_CUDA(aw::upsample_hfield(hc, net, hout, fine, 1, w->uscratch, s), "aw_warmstart (upsample)");
  } else {
    for (int c = 0; c < 3; ++c)
      WS_CUDA(cudaMemcpyAsync(hout[c], hc[c], sizeof(float) * nf, cudaMemcpyDeviceToDevice, s),
              "aw_warmstart (copy)");
  }
  return 0;
}

}  // namespace

extern "C" {

size_t aw_warmstart_param_floats(void) {
  size_t n = 0;
  for (const Layer &l : kNet) n += layer_params(l);
  return n;
}

int aw_warmstart_create(int nx, int ny, int nz, int net_nx, int net_ny, int net_nz,
                        const float *params, size_t n_params, float max_pert,
                        aw_warmstart_t *out) {
  if (!out || !params) return wfail("aw_warmstart_create: null pointer");
  *out = nullptr;
  if (n_params != aw_warmstart_param_floats())
    return wfail("aw_warmstart_create: expected " + std::to_string(aw_warmstart_param_floats()) +
                 " parameters (aw_warmstart_param_floats)");
  if (net_nx < 8 || net_ny < 8 || net_nz < 8 || net_nx % 8 || net_ny % 8 || net_nz % 8)
    return wfail("aw_warmstart_create: network grid axes must be multiples of 8");
  if (net_nx > nx || net_ny > ny || net_nz > nz)
    return wfail("aw_warmstart_create: the network grid may not exceed the pair grid");
  if (!(max_pert > 0.0f)) return wfail("aw_warmstart_create: MaxPert must be positive");
  aw_warmstart_s *w = new (std::nothrow) aw_warmstart_s;
  if (!w) return wfail("aw_warmstart_create: out of host memory");
  w->nx = nx; w->ny = ny; w->nz = nz;
  w->W = net_nx; w->H = net_ny; w->D = net_nz;
  w->coarse = net_nx != nx || net_ny != ny || net_nz != nz;
  w->max_pert = max_pert;
  auto bail = [&](int rc) {
    aw_warmstart_destroy(w);
    return rc;
  };
  // device block layout, 256-byte aligned pieces
  std::vector<size_t> sizes;
  auto add = [&](size_t bytes) {
    sizes.push_back((bytes + 255) & ~size_t(255));
    return sizes.size() - 1;
  };
  size_t iw[kLayers], ib[kLayers], ia[21];
  for (int l = 0; l < kLayers; ++l) {
    iw[l] = add(2 * (size_t)kNet[l].co * kNet[l].taps * kNet[l].ci);
    ib[l] = add(sizeof(float) * kNet[l].co);
  }
  const int slot_level[21] = {0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 3, 2, 2, 2, 1, 1, 1, 0, 0, 0};
  const int slot_ch[21] = {16, 16, 16, 16, 32, 32, 32, 64, 64, 64, 128, 128, 192, 64, 64, 96,
                           32, 32, 48, 16, 16};
  for (int k = 0; k < 21; ++k) ia[k] = add(2 * (size_t)vox(w, slot_level[k]) * slot_ch[k]);
  const size_t iout = add(sizeof(float) * 16 * vox(w, 0));
  size_t cf = 1;
  for (const Layer &l : kNet) {
    const int f = 1 << l.level;
    const size_t need =
        aw_nn_conv3d_scratch_floats(1, w->D / f, w->H / f, w->W / f, l.ci, l.co, l.taps);
    if (need > cf) cf = need;
  }
  const size_t ics = add(sizeof(float) * cf);
  const long nf = (long)nx * ny * nz, nc = vox(w, 0);
  const size_t ii0 = add(sizeof(float) * nc), ii1 = add(sizeof(float) * nc);
  const size_t ihc = add(sizeof(float) * 3 * nc);
  const aw::Dims fine{nx, ny, nz};
  const size_t ids = add(w->coarse ? aw::downsample_scratch_bytes(fine) : 16);
  const size_t ius = add(sizeof(float) * 3 * nc);
  const size_t ish = add(sizeof(float) * 3 * nf);
  size_t total = 0;
  std::vector<size_t> off(sizes.size());
  for (size_t k = 0; k < sizes.size(); ++k) {
    off[k] = total;
    total += sizes[k];
  }
  if (cudaMalloc((void **)&w->block, total) != cudaSuccess) {
    cudaGetLastError();
    return bail(wfail("aw_warmstart_create: device allocation of " + std::to_string(total) +
                      " bytes failed"));
  }
  auto at = [&](size_t k) { return (void *)(w->block + off[k]); };
  for (int l = 0; l < kLayers; ++l) {
    w->wb[l] = at(iw[l]);
    w->bias[l] = (float *)at(ib[l]);
  }
  for (int k = 0; k < 21; ++k) w->act[k] = at(ia[k]);
  w->out = (float *)at(iout);
  w->cscratch = (float *)at(ics);
  w->cfloats = cf;
  w->I0c = (float *)at(ii0);
  w->I1c = (float *)at(ii1);
  w->hc = (float *)at(ihc);
  w->dscratch = at(ids);
  w->uscratch = (float *)at(ius);
  w->scratch_h = (float *)at(ish);
  if (cudaStreamCreateWithFlags(&w->s, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&w->ev_in, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&w->ev_out, cudaEventDisableTiming) != cudaSuccess)
    return bail(wfail("aw_warmstart_create: stream/event creation failed"));
  // activations start at zero (the padded input channels stay zero)
  if (cudaMemsetAsync(w->block, 0, total, w->s) != cudaSuccess)
    return bail(wfail("aw_warmstart_create: clearing device memory failed"));
  // parameters: FP32 weights to BF16 on the device, biases as they are
  float *wtmp = nullptr;
  size_t maxw = 0;
  for (const Layer &l : kNet) maxw = std::max(maxw, (size_t)l.co * l.taps * l.ci);
  if (cudaMalloc((void **)&wtmp, sizeof(float) * maxw) != cudaSuccess) {
    cudaGetLastError();
    return bail(wfail("aw_warmstart_create: device allocation failed"));
  }
  const float *p = params;
  int rc = 0;
  for (int l = 0; l < kLayers && rc == 0; ++l) {
    const Layer &L = kNet[l];
    const size_t nw = (size_t)L.co * L.taps * L.ci;
    if (cudaMemcpyAsync(wtmp, p, sizeof(float) * nw, cudaMemcpyHostToDevice, w->s) != cudaSuccess ||
        cudaMemcpyAsync(w->bias[l], p + nw, sizeof(float) * L.co, cudaMemcpyHostToDevice, w->s) !=
            cudaSuccess) {
      rc = wfail("aw_warmstart_create: parameter upload failed");
      break;
    }
    rc = aw_nn_weights_bf16(wtmp, L.co, L.taps, L.ci, w->wb[l], nullptr, w->s);
    if (rc == 0 && cudaStreamSynchronize(w->s) != cudaSuccess)
      rc = wfail("aw_warmstart_create: parameter conversion failed");
    p += layer_params(L);
  }
  cudaFree(wtmp);
  if (rc) return bail(rc);
  if (int r = aw_greedy_create(nx, ny, nz, 1.0, 1.0, 1.0, 0.01f, 0.01f, 0.001f, max_pert,
                               &w->refine))
    return bail(r);
  *out = w;
  return 0;
}

int aw_warmstart_predict(aw_warmstart_t w, const float *I0, const float *I1, float *hx, float *hy,
                         float *hz, void *stream) {
  if (!w) return wfail("aw_warmstart_predict: null handle");
  if (!I0 || !I1 || !hx || !hy || !hz) return wfail("aw_warmstart_predict: null pointer");
  cudaStream_t user = reinterpret_cast<cudaStream_t>(stream);
  float *const h[3] = {hx, hy, hz};
  // a new set of pointers: (re)capture the prediction as one graph
  if (!w->graph || w->in0 != I0 || w->in1 != I1 || w->hout[0] != hx || w->hout[1] != hy ||
      w->hout[2] != hz) {
    if (w->graph) cudaGraphExecDestroy(w->graph);
    w->graph = nullptr;
    // one run outside the capture first: the downsampling caches its
    // Gaussian tables on the device, the kernels their attributes
    WS_CUDA(cudaEventRecord(w->ev_in, user), "aw_warmstart_predict (event)");
    WS_CUDA(cudaStreamWaitEvent(w->s, w->ev_in, 0), "aw_warmstart_predict (wait)");
    WS_TRY(predict_body(w, I0, I1, h));
    WS_CUDA(cudaStreamSynchronize(w->s), "aw_warmstart_predict (first run)");
    cudaGraph_t g;
    WS_CUDA(cudaStreamBeginCapture(w->s, cudaStreamCaptureModeThreadLocal),
            "aw_warmstart_predict (capture)");
    const int rc = predict_body(w, I0, I1, h);
    const cudaError_t ec = cudaStreamEndCapture(w->s, &g);
    if (rc) return rc;
    WS_CUDA(ec, "aw_warmstart_predict (end capture)");
    const cudaError_t ei = cudaGraphInstantiate(&w->graph, g, 0);
    cudaGraphDestroy(g);
    WS_CUDA(ei, "aw_warmstart_predict (instantiate)");
    w->in0 = I0;
    w->in1 = I1;
    for (int c = 0; c < 3; ++c) w->hout[c] = h[c];
  }
  WS_CUDA(cudaEventRecord(w->ev_in, user), "aw_warmstart_predict (event)");
  WS_CUDA(cudaStreamWaitEvent(w->s, w->ev_in, 0), "aw_warmstart_predict (wait)");
  WS_CUDA(cudaGraphLaunch(w->graph, w->s), "aw_warmstart_predict (launch)");
  WS_CUDA(cudaEventRecord(w->ev_out, w->s), "aw_warmstart_predict (event)");
  WS_CUDA(cudaStreamWaitEvent(user, w->ev_out, 0), "aw_warmstart_predict (wait)");
  return 0;
}

int aw_warmstart_register(aw_warmstart_t w, const float *I0, const float *I1,
                          double target_energy, int max_refine_iters, int chunk, int plain_iters,
                          float *hx, float *hy, float *hz, int *iters_run, int *fell_back,
                          void *stream) {
  if (!w) return wfail("aw_warmstart_register: null handle");
  if (!I0 || !I1 || !hx || !hy || !hz) return wfail("aw_warmstart_register: null pointer");
  if (chunk < 1 || max_refine_iters < 0 || plain_iters < 0)
    return wfail("aw_warmstart_register: chunk >= 1, iteration counts >= 0");
  const long n = (long)w->nx * w->ny * w->nz;
  float *s3 = w->scratch_h;
  WS_TRY(aw_warmstart_predict(w, I0, I1, hx, hy, hz, stream));
  // refinement: the step is set at its first iteration from the warm
  // start's own velocity, halved whenever the energy rises
  WS_TRY(aw_greedy_set_auto_step_reduce(w->refine, 1));
  int done = 0, run = 0;
  double best = 1e300;
  bool reached = false;
  std::vector<double> en;
  while (done < max_refine_iters) {
    const int k = std::min(chunk, max_refine_iters - done);
    WS_TRY(aw_greedy_run(w->refine, I0, I1, hx, hy, hz, s3, s3 + n, s3 + 2 * n, nullptr, nullptr,
                         nullptr, nullptr, nullptr, nullptr, k, done == 0 ? 1 : 0, stream));
    done += k;
    run += k;
    int count = 0;
    WS_TRY(aw_greedy_get_energies(w->refine, nullptr, 0, &count));
    en.assign(count > 0 ? count : 1, 0.0);
    WS_TRY(aw_greedy_get_energies(w->refine, en.data(), count, &count));
    double cmin = 1e300;
    for (int i = count - k; i < count; ++i) {
      if (i < 0) continue;
      if (en[i] <= target_energy) reached = true;
      cmin = std::min(cmin, en[i]);
    }
    if (reached) break;
    if (!(cmin < best)) break;  // the refinement stopped falling
    best = cmin;
  }
  WS_TRY(aw_greedy_set_auto_step_reduce(w->refine, 0));
  const bool fallback = !reached;
  if (fallback) {
    // the plain solve from the identity, unassisted
    WS_TRY(aw_identity(hx, hy, hz, w->nx, w->ny, w->nz, stream));
    WS_TRY(aw_greedy_run(w->refine, I0, I1, hx, hy, hz, s3, s3 + n, s3 + 2 * n, nullptr, nullptr,
                         nullptr, nullptr, nullptr, nullptr, plain_iters, 1, stream));
    run += plain_iters;
  }
  if (iters_run) *iters_run = run;
  if (fell_back) *fell_back = fallback ? 1 : 0;
  return 0;
}

int aw_warmstart_destroy(aw_warmstart_t w) {
  if (!w) return 0;
  if (w->graph) cudaGraphExecDestroy(w->graph);
  if (w->refine) aw_greedy_destroy(w->refine);
  if (w->s) cudaStreamSynchronize(w->s);
  if (w->block) cudaFree(w->block);
  if (w->s) cudaStreamDestroy(w->s);
  if (w->ev_in) cudaEventDestroy(w->ev_in);
  if (w->ev_out) cudaEventDestroy(w->ev_out);
  delete w;
  return 0;
}

}  // extern "C"
