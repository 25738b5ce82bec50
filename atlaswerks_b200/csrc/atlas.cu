// atlas.cu — greedy atlas building over the subjects resident on one GPU.
//
// One iteration runs the six greedy stages of every subject (greedy.cu) with
// I1 = the mean template. Subjects are spread over `branches` stream chains
// forked from the caller's stream, so independent subjects overlap on the
// GPU; two iterations of all subjects are captured once as a CUDA graph and
// replayed. The mean of GreedyAtlasThreadCPU::ComputeThreadMean
// (Algorithms/Greedy/GreedyAtlasThreadCPU.cxx: averageData += I0(h) * w, in
// subject order, float) is one kernel over the template grid.
#include <cstring>

#include "atlas.cuh"

namespace aw {

namespace {

__global__ void __launch_bounds__(kRowThreads)
    k_atlas_mean(const AtlasSubjectDev *__restrict__ t, int ns, float *__restrict__ mean, Dims d) {
  Voxel v;
  if (!voxel_of(d, v)) return;
  float acc = 0.0f;
  for (int k = 0; k < ns; ++k) {
    const AtlasSubjectDev s = t[k];
    double px = (double)s.h[0][v.i], py = (double)s.h[1][v.i], pz = (double)s.h[2][v.i];
    if (s.am.on) atlas_point(s.am, px, py, pz);
    const float val = trilerp_scalar(s.img, s.am.on ? s.di : d, px, py, pz, 0.0f);
    acc = fadd(acc, fmul(val, s.w));
  }
  mean[v.i] = acc;
}

#define AW_TRY(x)                     \
  do {                                \
    cudaError_t _e = (x);             \
    if (_e != cudaSuccess) return _e; \
  } while (0)

// one iteration of every subject, chains forked from s and joined back;
// src_a selects h (true) or the scratch (false) as the input field
cudaError_t iterate_all(AtlasCtx *a, bool src_a, int update_step, cudaStream_t s) {
  const long n = a->d.n();
  AW_TRY(cudaEventRecord(a->ev_fork, s));
  for (int b = 0; b < a->branches; ++b) AW_TRY(cudaStreamWaitEvent(a->bstream[b], a->ev_fork, 0));
  for (int i = 0; i < a->ns; ++i) {
    cudaStream_t bs = a->bstream[i % a->branches];
    float *H = a->hbuf + (size_t)i * 6 * n;
    float *A[3] = {H, H + n, H + 2 * n}, *B[3] = {H + 3 * n, H + 4 * n, H + 5 * n};
    float **src = src_a ? A : B, **dst = src_a ? B : A;
    const float *cs[3] = {src[0], src[1], src[2]};
    AW_TRY(greedy_iterate(&a->subj[i], a->table[i].img, a->mean, cs, dst, nullptr, nullptr,
                          update_step, 0, bs));
  }
  for (int b = 0; b < a->branches; ++b) {
    AW_TRY(cudaEventRecord(a->ev_join[b], a->bstream[b]));
    AW_TRY(cudaStreamWaitEvent(s, a->ev_join[b], 0));
  }
  return cudaSuccess;
}

void set_identity_host(std::vector<float> &h, const Dims &d) {
  const long n = d.n();
  h.resize(3 * n);
  for (int z = 0; z < d.nz; ++z)
    for (int y = 0; y < d.ny; ++y)
      for (int x = 0; x < d.nx; ++x) {
        const long i = d.idx(x, y, z);
        h[i] = (float)x;
        h[n + i] = (float)y;
        h[2 * n + i] = (float)z;
      }
}

}  // namespace

int atlas_create(AtlasCtx *a, int nx, int ny, int nz, double spx, double spy, double spz,
                 float alpha, float beta, float gamma, float max_pert, int n_subjects) {
  a->d = Dims{nx, ny, nz};
  a->sp = Spacing{spx, spy, spz};
  a->ns = n_subjects;
  a->subj.resize(n_subjects);
  for (auto &g : a->subj) std::memset(&g, 0, sizeof(g));
  for (int i = 0; i < n_subjects; ++i) {
    const int rc = greedy_create(&a->subj[i], nx, ny, nz, spx, spy, spz, alpha, beta, gamma,
                                 max_pert, 0);
    if (rc) return rc;
  }
  const long n = a->d.n();
  if (cudaMalloc(&a->mean, sizeof(float) * n) != cudaSuccess) return 3;
  if (cudaMalloc(&a->hbuf, sizeof(float) * 6 * n * (size_t)n_subjects) != cudaSuccess) return 3;
  if (cudaMalloc(&a->dtable, sizeof(AtlasSubjectDev) * n_subjects) != cudaSuccess) return 3;
  cudaMemset(a->mean, 0, sizeof(float) * n);
  std::vector<float> id;
  set_identity_host(id, a->d);
  a->table.resize(n_subjects);
  a->ready.assign(n_subjects, 0);
  for (int i = 0; i < n_subjects; ++i) {
    float *H = a->hbuf + (size_t)i * 6 * n;
    if (cudaMemcpy(H, id.data(), sizeof(float) * 3 * n, cudaMemcpyHostToDevice) != cudaSuccess)
      return 5;
    AtlasSubjectDev &t = a->table[i];
    std::memset(&t, 0, sizeof(t));
    t.di = a->d;
    t.h[0] = H;
    t.h[1] = H + n;
    t.h[2] = H + 2 * n;
  }
  a->branches = n_subjects < 16 ? (n_subjects > 0 ? n_subjects : 1) : 16;
  if (cudaStreamCreateWithFlags(&a->gstream, cudaStreamNonBlocking) != cudaSuccess) return 5;
  a->bstream.assign(a->branches, nullptr);
  a->ev_join.assign(a->branches, nullptr);
  for (int b = 0; b < a->branches; ++b) {
    if (cudaStreamCreateWithFlags(&a->bstream[b], cudaStreamNonBlocking) != cudaSuccess) return 5;
    if (cudaEventCreateWithFlags(&a->ev_join[b], cudaEventDisableTiming) != cudaSuccess) return 5;
  }
  if (cudaEventCreateWithFlags(&a->ev_in, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&a->ev_out, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&a->ev_fork, cudaEventDisableTiming) != cudaSuccess)
    return 5;
  return cudaGetLastError() == cudaSuccess ? 0 : 5;
}

void atlas_destroy(AtlasCtx *a) {
  cudaDeviceSynchronize();
  if (a->pair) cudaGraphExecDestroy(a->pair);
  for (auto &g : a->subj) greedy_destroy(&g);
  if (a->mean) cudaFree(a->mean);
  if (a->hbuf) cudaFree(a->hbuf);
  if (a->dtable) cudaFree(a->dtable);
  for (auto s : a->bstream)
    if (s) cudaStreamDestroy(s);
  for (auto e : a->ev_join)
    if (e) cudaEventDestroy(e);
  if (a->gstream) cudaStreamDestroy(a->gstream);
  if (a->ev_in) cudaEventDestroy(a->ev_in);
  if (a->ev_out) cudaEventDestroy(a->ev_out);
  if (a->ev_fork) cudaEventDestroy(a->ev_fork);
  *a = AtlasCtx();
}

cudaError_t atlas_set_subject(AtlasCtx *a, int i, const float *img, Dims di, float weight) {
  AtlasSubjectDev &t = a->table[i];
  t.img = img;
  t.di = di;
  t.w = weight;
  t.am.on = !(di.nx == a->d.nx && di.ny == a->d.ny && di.nz == a->d.nz);
  t.am.r[0] = (double)di.nx / (double)a->d.nx;
  t.am.r[1] = (double)di.ny / (double)a->d.ny;
  t.am.r[2] = (double)di.nz / (double)a->d.nz;
  a->subj[i].di = di;
  a->subj[i].am = t.am;
  a->ready[i] = 1;
  if (a->pair) {  // the captured graph holds the old image pointer
    cudaGraphExecDestroy(a->pair);
    a->pair = nullptr;
  }
  return cudaMemcpy(a->dtable + i, &t, sizeof(t), cudaMemcpyHostToDevice);
}

float *atlas_field(AtlasCtx *a, int i, int comp) {
  return a->hbuf + (size_t)i * 6 * a->d.n() + (size_t)comp * a->d.n();
}

cudaError_t atlas_mean(AtlasCtx *a, cudaStream_t s) {
  k_atlas_mean<<<row_grid(a->d), kRowThreads, 0, s>>>(a->dtable, a->ns, a->mean, a->d);
  return cudaGetLastError();
}

cudaError_t atlas_iterate(AtlasCtx *a, int n_iters, int update_first, cudaStream_t user) {
  if (n_iters <= 0) return cudaSuccess;
  cudaStream_t s = a->gstream;
  AW_TRY(cudaEventRecord(a->ev_in, user));
  AW_TRY(cudaStreamWaitEvent(s, a->ev_in, 0));
  const long n = a->d.n();
  auto scratch_to_h = [&]() -> cudaError_t {
    for (int i = 0; i < a->ns; ++i) {
      float *H = a->hbuf + (size_t)i * 6 * n;
      AW_TRY(cudaMemcpyAsync(H, H + 3 * n, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, s));
    }
    return cudaSuccess;
  };
  int done = 0;
  if (update_first) {
    // the step-size iteration, plus one more so the field is back in h
    AW_TRY(iterate_all(a, true, 1, s));
    if (n_iters == 1) {
      AW_TRY(scratch_to_h());
      done = 1;
    } else {
      AW_TRY(iterate_all(a, false, 0, s));
      done = 2;
    }
  }
  const int pairs = (n_iters - done) / 2;
  if (pairs > 0) {
    if (!a->pair) {
      cudaGraph_t graph;
      AW_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      cudaError_t e1 = iterate_all(a, true, 0, s);
      cudaError_t e2 = e1 == cudaSuccess ? iterate_all(a, false, 0, s) : e1;
      cudaError_t ec = cudaStreamEndCapture(s, &graph);
      AW_TRY(e1);
      AW_TRY(e2);
      AW_TRY(ec);
      cudaError_t ei = cudaGraphInstantiate(&a->pair, graph, 0);
      cudaGraphDestroy(graph);
      AW_TRY(ei);
    }
    for (int p = 0; p < pairs; ++p) AW_TRY(cudaGraphLaunch(a->pair, s));
    done += 2 * pairs;
  }
  if (done < n_iters) {
    AW_TRY(iterate_all(a, true, 0, s));
    AW_TRY(scratch_to_h());
  }
  AW_TRY(cudaEventRecord(a->ev_out, s));
  return cudaStreamWaitEvent(user, a->ev_out, 0);
}

}  // namespace aw
