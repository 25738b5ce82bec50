// nn_capi.cu — extern "C" entry points of the warm-start network kernels
// (nn.cu), declared in include/aw_b200.h. Argument checks and error strings
// only; the arithmetic is in nn.cu.
#include <mutex>
#include <string>

#include "../../include/aw_b200.h"
#include "capi_error.h"

namespace aw {
bool nn_channels_ok(int c);
size_t nn_splitk_floats(long M, int N, int K);
int nn_conv_direct_planes(int B, int D, int H, int W, int cin, int cout, int ntaps);
void nn_set_gemm_only(int on);
cudaError_t nn_conv_fwd(const void *x, int B, int D, int H, int W, int cin, const void *w,
                        const float *bias, int cout, int ntaps, int relu, void *out, float *outf,
                        float *scratch, size_t scratch_floats, int *status, cudaStream_t s);
cudaError_t nn_conv_dgrad(const void *dy, int B, int D, int H, int W, int cout, const void *wt,
                          int cin, int ntaps, const void *mask, void *dx, float *scratch,
                          size_t scratch_floats, int *status, cudaStream_t s);
size_t nn_wgrad_part_floats(int cin, int cout, int ntaps, int splits);
cudaError_t nn_conv_wgrad(const void *x, const void *dy, int B, int D, int H, int W, int cin,
                          int cout, int ntaps, int splits, float *part, float *dw, int *status,
                          cudaStream_t s);
size_t nn_bias_scratch_floats(long M, int N);
cudaError_t nn_bias_grad(const void *dy, long M, int N, float *scratch, float *db, cudaStream_t s);
cudaError_t nn_pool(const void *in, int B, int D, int H, int W, int C, void *out, int backward,
                    const void *add, const void *mask, cudaStream_t s);
cudaError_t nn_upsample(const void *in, int B, int D, int H, int W, int C, void *out, int Ct,
                        int c0, int backward, cudaStream_t s);
cudaError_t nn_slice(const void *src, int Cs, int cs0, void *dst, int Cd, int cd0, int C,
                     long voxels, int accumulate, cudaStream_t s);
cudaError_t nn_pack_pair(const float *a, const float *b, long voxels, void *x, cudaStream_t s);
size_t nn_mse_partials(long voxels);
cudaError_t nn_mse(const float *pred, const float *tgt, long voxels, void *grad, double *partials,
                   float *loss, cudaStream_t s);
cudaError_t nn_adam(float *w, const float *g, float *m1, float *m2, long n, float lr, float b1,
                    float b2, float eps, int t, cudaStream_t s);
cudaError_t nn_weights_bf16(const float *w, int cout, int ntaps, int cin, void *wb, void *wt,
                            cudaStream_t s);
cudaError_t nn_disp_to_h(const float *pred, int D, int H, int W, float *hx, float *hy, float *hz,
                         cudaStream_t s);
}  // namespace aw

namespace {

int nfail(const std::string &m) {
  aw::set_last_error(m);
  return 1;
}
int ncuda(cudaError_t e, const char *what) {
  aw::set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
  return 2;
}
#define NN_CUDA(call, what)                        \
  do {                                             \
    cudaError_t _e = (call);                       \
    if (_e != cudaSuccess) return ncuda(_e, what); \
  } while (0)

inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// per-device word where a GEMM records a bounded wait that gave up
constexpr int kMaxDev = 64;
std::mutex g_mu;
int *g_status[kMaxDev] = {nullptr};

int status_word(int **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return ncuda(e, "aw_nn (device)");
  if (dev < 0 || dev >= kMaxDev) return nfail("aw_nn: device index out of range");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_status[dev]) {
    e = cudaMalloc(&g_status[dev], sizeof(int));
    if (e != cudaSuccess) return ncuda(e, "aw_nn (status word)");
    e = cudaMemset(g_status[dev], 0, sizeof(int));
    if (e != cudaSuccess) return ncuda(e, "aw_nn (status word)");
  }
  *out = g_status[dev];
  return 0;
}

bool grid_ok(int B, int D, int H, int W) { return B >= 1 && D >= 1 && H >= 1 && W >= 1; }

}  // namespace

extern "C" {

size_t aw_nn_conv3d_scratch_floats(int B, int D, int H, int W, int cin, int cout, int ntaps) {
  // the larger of the forward (N = cout, K = taps cin) and dgrad (N = cin,
  // K = taps cout) split-K partials
  const long M = (long)B * D * H * W;
  const size_t a = aw::nn_splitk_floats(M, cout, ntaps * cin);
  const size_t b = aw::nn_splitk_floats(M, cin, ntaps * cout);
  return a > b ? a : b;
}

void aw_nn_set_gemm_only(int on) { aw::nn_set_gemm_only(on); }

int aw_nn_conv3d_direct_planes(int B, int D, int H, int W, int cin, int cout, int ntaps) {
  if (!grid_ok(B, D, H, W)) return 0;
  return aw::nn_conv_direct_planes(B, D, H, W, cin, cout, ntaps);
}

int aw_nn_conv3d_fwd(const void *x, int B, int D, int H, int W, int cin, const void *w,
                     const float *bias, int cout, int ntaps, int relu, void *out_bf16,
                     float *out_f32, float *scratch, size_t scratch_floats, void *stream) {
  if (!x || !w || (!out_bf16 && !out_f32)) return nfail("aw_nn_conv3d_fwd: null pointer");
  if (!grid_ok(B, D, H, W)) return nfail("aw_nn_conv3d_fwd: empty grid");
  if (cin % 16 || cin <= 0) return nfail("aw_nn_conv3d_fwd: input channels must be a multiple of 16");
  if (!aw::nn_channels_ok(cout))
    return nfail("aw_nn_conv3d_fwd: output channels must be one of 16 32 48 64 96 128 192");
  if (ntaps != 27 && ntaps != 1) return nfail("aw_nn_conv3d_fwd: taps must be 27 (3x3x3) or 1");
  int *st = nullptr;
  if (int rc = status_word(&st)) return rc;
  NN_CUDA(aw::nn_conv_fwd(x, B, D, H, W, cin, w, bias, cout, ntaps, relu, out_bf16, out_f32,
                          scratch, scratch_floats, st, S(stream)),
          "aw_nn_conv3d_fwd");
  return 0;
}

int aw_nn_conv3d_dgrad(const void *dy, int B, int D, int H, int W, int cout, const void *wt,
                       int cin, int ntaps, const void *mask, void *dx, float *scratch,
                       size_t scratch_floats, void *stream) {
  if (!dy || !wt || !dx) return nfail("aw_nn_conv3d_dgrad: null pointer");
  if (!grid_ok(B, D, H, W)) return nfail("aw_nn_conv3d_dgrad: empty grid");
  if (cout % 16 || cout <= 0) return nfail("aw_nn_conv3d_dgrad: output channels must be a multiple of 16");
  if (!aw::nn_channels_ok(cin))
    return nfail("aw_nn_conv3d_dgrad: input channels must be one of 16 32 48 64 96 128 192");
  if (ntaps != 27 && ntaps != 1) return nfail("aw_nn_conv3d_dgrad: taps must be 27 or 1");
  int *st = nullptr;
  if (int rc = status_word(&st)) return rc;
  NN_CUDA(aw::nn_conv_dgrad(dy, B, D, H, W, cout, wt, cin, ntaps, mask, dx, scratch,
                            scratch_floats, st, S(stream)),
          "aw_nn_conv3d_dgrad");
  return 0;
}

size_t aw_nn_wgrad_scratch_floats(int cin, int cout, int ntaps, int splits) {
  return aw::nn_wgrad_part_floats(cin, cout, ntaps, splits);
}

int aw_nn_conv3d_wgrad(const void *x, const void *dy, int B, int D, int H, int W, int cin,
                       int cout, int ntaps, int splits, float *scratch, float *dw, void *stream) {
  if (!x || !dy || !scratch || !dw) return nfail("aw_nn_conv3d_wgrad: null pointer");
  if (!grid_ok(B, D, H, W)) return nfail("aw_nn_conv3d_wgrad: empty grid");
  if (cin % 16 || cin <= 0) return nfail("aw_nn_conv3d_wgrad: input channels must be a multiple of 16");
  if (!aw::nn_channels_ok(cout))
    return nfail("aw_nn_conv3d_wgrad: output channels must be one of 16 32 48 64 96 128 192");
  if (ntaps != 27 && ntaps != 1) return nfail("aw_nn_conv3d_wgrad: taps must be 27 or 1");
  if (splits < 1) return nfail("aw_nn_conv3d_wgrad: splits must be >= 1");
  int *st = nullptr;
  if (int rc = status_word(&st)) return rc;
  NN_CUDA(aw::nn_conv_wgrad(x, dy, B, D, H, W, cin, cout, ntaps, splits, scratch, dw, st,
                            S(stream)),
          "aw_nn_conv3d_wgrad");
  return 0;
}

size_t aw_nn_bias_scratch_floats(long M, int cout) { return aw::nn_bias_scratch_floats(M, cout); }

int aw_nn_bias_grad(const void *dy, long M, int cout, float *scratch, float *db, void *stream) {
  if (!dy || !db || !scratch) return nfail("aw_nn_bias_grad: null pointer");
  if (cout < 1 || cout > 256) return nfail("aw_nn_bias_grad: 1..256 channels");
  NN_CUDA(aw::nn_bias_grad(dy, M, cout, scratch, db, S(stream)), "aw_nn_bias_grad");
  return 0;
}

int aw_nn_pool(const void *in, int B, int D, int H, int W, int C, void *out, int backward,
               const void *add, const void *mask, void *stream) {
  if (!in || !out) return nfail("aw_nn_pool: null pointer");
  if (D % 2 || H % 2 || W % 2) return nfail("aw_nn_pool: grid axes must be even");
  NN_CUDA(aw::nn_pool(in, B, D, H, W, C, out, backward, add, mask, S(stream)), "aw_nn_pool");
  return 0;
}

int aw_nn_upsample(const void *in, int B, int D, int H, int W, int C, void *out, int Ct, int c0,
                   int backward, void *stream) {
  if (!in || !out) return nfail("aw_nn_upsample: null pointer");
  if (c0 < 0 || c0 + C > Ct) return nfail("aw_nn_upsample: channel slice out of range");
  NN_CUDA(aw::nn_upsample(in, B, D, H, W, C, out, Ct, c0, backward, S(stream)), "aw_nn_upsample");
  return 0;
}

int aw_nn_slice(const void *src, int Cs, int cs0, void *dst, int Cd, int cd0, int C, long voxels,
                int accumulate, void *stream) {
  if (!src || !dst) return nfail("aw_nn_slice: null pointer");
  if (cs0 < 0 || cs0 + C > Cs || cd0 < 0 || cd0 + C > Cd)
    return nfail("aw_nn_slice: channel slice out of range");
  NN_CUDA(aw::nn_slice(src, Cs, cs0, dst, Cd, cd0, C, voxels, accumulate, S(stream)), "aw_nn_slice");
  return 0;
}

int aw_nn_pack_pair(const float *I0, const float *I1, long voxels, void *x, void *stream) {
  if (!I0 || !I1 || !x) return nfail("aw_nn_pack_pair: null pointer");
  NN_CUDA(aw::nn_pack_pair(I0, I1, voxels, x, S(stream)), "aw_nn_pack_pair");
  return 0;
}

size_t aw_nn_mse_scratch_doubles(long voxels) { return aw::nn_mse_partials(voxels); }

int aw_nn_mse(const float *pred, const float *target, long voxels, void *grad, double *scratch,
              float *loss, void *stream) {
  if (!pred || !target || !grad || !scratch || !loss) return nfail("aw_nn_mse: null pointer");
  NN_CUDA(aw::nn_mse(pred, target, voxels, grad, scratch, loss, S(stream)), "aw_nn_mse");
  return 0;
}

int aw_nn_adam(float *w, const float *g, float *m1, float *m2, long n, float lr, float beta1,
               float beta2, float eps, int step, void *stream) {
  if (!w || !g || !m1 || !m2) return nfail("aw_nn_adam: null pointer");
  if (step < 1) return nfail("aw_nn_adam: step counts from 1");
  NN_CUDA(aw::nn_adam(w, g, m1, m2, n, lr, beta1, beta2, eps, step, S(stream)), "aw_nn_adam");
  return 0;
}

int aw_nn_weights_bf16(const float *w, int cout, int ntaps, int cin, void *w_bf16,
                       void *wt_bf16, void *stream) {
  if (!w || !w_bf16) return nfail("aw_nn_weights_bf16: null pointer");
  NN_CUDA(aw::nn_weights_bf16(w, cout, ntaps, cin, w_bf16, wt_bf16, S(stream)),
          "aw_nn_weights_bf16");
  return 0;
}

int aw_nn_displacement_to_h(const float *pred, int D, int H, int W, float *hx, float *hy,
                            float *hz, void *stream) {
  if (!pred || !hx || !hy || !hz) return nfail("aw_nn_displacement_to_h: null pointer");
  NN_CUDA(aw::nn_disp_to_h(pred, D, H, W, hx, hy, hz, S(stream)), "aw_nn_displacement_to_h");
  return 0;
}

int aw_nn_status(int *timed_out) {
  if (!timed_out) return nfail("aw_nn_status: null pointer");
  int *st = nullptr;
  if (int rc = status_word(&st)) return rc;
  NN_CUDA(cudaDeviceSynchronize(), "aw_nn_status (pending work)");
  int v = 0;
  NN_CUDA(cudaMemcpy(&v, st, sizeof(int), cudaMemcpyDeviceToHost), "aw_nn_status");
  NN_CUDA(cudaMemset(st, 0, sizeof(int)), "aw_nn_status");
  *timed_out = v;
  return 0;
}

}  // extern "C"
