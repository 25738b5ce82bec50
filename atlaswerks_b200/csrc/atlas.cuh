// atlas.cuh — greedy atlas building on one GPU (atlas.cu): every local
// subject runs the greedy-fluid iteration toward the current mean template,
// and the mean is the weighted sum of the deformed subjects
// (AtlasThread::AtlasThreadMain, Algorithms/Common/AtlasThread.txx:97-181;
// GreedyAtlasThreadCPU/GPU::ComputeThreadMean).
//
// Deformations live on the template grid. A subject image may sit on a grid
// of its own; it is then sampled through the voxel-centre map of equal
// physical extent (AtlasMap, aw_common.cuh). Across GPUs the subjects are
// sharded and the host sums the per-GPU means (one all-reduce).
#pragma once

#include <vector>

#include "greedy.cuh"

namespace aw {

struct AtlasSubjectDev {
  const float *img;
  Dims di;
  AtlasMap am;
  const float *h[3];
  float w;
};

struct AtlasCtx {
  Dims d;
  Spacing sp;
  int ns = 0;
  std::vector<GreedyCtx> subj;
  std::vector<AtlasSubjectDev> table;  // host copy of dtable
  AtlasSubjectDev *dtable = nullptr;
  std::vector<int> ready;              // subject image set
  float *mean = nullptr;               // template-grid mean: I1 of every subject
  float *hbuf = nullptr;               // per subject: h (3N), then scratch (3N)
  int branches = 4;                    // concurrent subject chains in one iteration
  cudaStream_t gstream = nullptr;
  std::vector<cudaStream_t> bstream;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr, ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_join;
  cudaGraphExec_t pair = nullptr;      // two iterations of every subject, h -> scratch -> h
};

// returns 0, or the fluid-plan error code (1..4), or 5 for other failures
int atlas_create(AtlasCtx *a, int nx, int ny, int nz, double spx, double spy, double spz,
                 float alpha, float beta, float gamma, float max_pert, int n_subjects);
void atlas_destroy(AtlasCtx *a);
cudaError_t atlas_set_subject(AtlasCtx *a, int i, const float *img, Dims di, float weight);
float *atlas_field(AtlasCtx *a, int i, int comp);
// mean = sum over subjects in index order of w_i * I_i(h_i), float accumulation
cudaError_t atlas_mean(AtlasCtx *a, cudaStream_t s);
// n greedy iterations of every subject toward the current mean; the first
// one recomputes each subject's step (MaxPert / max|v|) when update_first
cudaError_t atlas_iterate(AtlasCtx *a, int n_iters, int update_first, cudaStream_t s);

}  // namespace aw
