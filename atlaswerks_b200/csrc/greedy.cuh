// greedy.cuh — device state of the greedy-fluid iterator (greedy.cu).
#pragma once

#include "fluid.cuh"

namespace aw {

// scalars the iteration keeps on the device (no host round trip per step)
struct GreedyDevState {
  float *step;     // current step size (GreedyDeformationData::StepSize)
  int *count;      // number of energies recorded
  double *energy;  // energy history ring, cap entries
  int cap;
};

struct GreedyCtx {
  FluidPlan plan;
  Dims d;
  Dims di;          // grid of I0 (= d, except for atlas subjects on their own grid)
  AtlasMap am;      // template voxel -> I0 voxel map when di != d (atlas_point)
  Spacing sp;
  float max_pert;
  float *idef;      // I0(h), N
  float *vbuf;      // v = K f, 3N
  double *partials; // per-block energy sums
  int nparts;
  int sms;
  cudaStream_t aux;  // side stream of the energy sum
  cudaEvent_t ev_fork, ev_join;
  char *scalars;    // step | count | maxbits
  unsigned *maxbits;
  GreedyDevState st;
  void *hmaps;      // host cache of the h planes' tensor maps (greedy.cu)
  int no_staged_update;  // 1: the update gathers h from global memory only
  int no_fused_update;   // 1: v goes to HBM and a separate kernel updates h
  int fast_interp;       // 1: float-tree interpolation in force-prep and the fused update
  int utile;             // tile shape of the staged update (greedy.cu)
};

// stages of one iteration, in launch order
enum GreedyStage {
  kStageForcePrep = 0,
  kStageEnergy = 1,
  kStageXYForward = 2,
  kStageZSolve = 3,
  kStageXYInverse = 4,
  kStageMaxNorm = 5,
  kStageUpdate = 6,
  kStageInvCompose = 7,  // xy-inverse and update in one kernel (v stays on chip)
  kNumStages = 8
};

int greedy_create(GreedyCtx *g, int nx, int ny, int nz, double spx, double spy, double spz,
                  float alpha, float beta, float gamma, float max_pert, int history_cap);
void greedy_destroy(GreedyCtx *g);
cudaError_t greedy_stage(GreedyCtx *g, int stage, const float *I0, const float *I1,
                         const float *const h[3], float *const h_out[3], const float *const hinv[3],
                         float *const hinv_out[3], int auto_reduce, int solve_inverse,
                         cudaStream_t s);
cudaError_t greedy_iterate(GreedyCtx *g, const float *I0, const float *I1, const float *const h[3],
                           float *const h_out[3], const float *const hinv[3],
                           float *const hinv_out[3], int update_step, int auto_reduce,
                           cudaStream_t s);

}  // namespace aw
