/*
 * aw_b200_greedy_iterator.hpp — the reference-side binding of the C ABI:
 * a greedy iterator with the interface that GreedyWarp<T> and the greedy
 * atlas thread expect of GreedyIteratorGPU
 * (Algorithms/Greedy/GreedyIteratorGPU.h:32-58, GreedyIteratorGPU.cxx:60-135),
 * so an AtlasWerks build switches with one template argument:
 *
 *     GreedyWarp<GreedyIteratorB200> warp(I0, I1, param);
 *
 * Header-only; it is compiled inside the AtlasWerks tree (it uses the
 * reference's GreedyDeformationDataGPU, GreedyIteratorParam, KernelParam,
 * MultiscaleManager, Energy and AtlasWerksException) and links
 * libaw_b200.so. All arithmetic runs in the library; this class forwards
 * the data object's device pointers and keeps the data object in step:
 * Def1To0 / Def0To1 updated in place, the step size, the energy record.
 * The library's calls take the default stream (NULL), the stream the
 * reference's GPU path uses.
 */
#ifndef AW_B200_GREEDY_ITERATOR_HPP
#define AW_B200_GREEDY_ITERATOR_HPP

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "aw_b200.h"

#include "AtlasWerksException.h"
#include "DeformationIteratorInterface.h"
#include "Energy.h"
#include "GreedyDeformationDataGPU.h"
#include "GreedyIteratorParam.h"
#include "MultiscaleManager.h"

class GreedyIteratorB200 : public DeformationIteratorInterface {
 public:
  typedef GreedyDeformationDataGPU DeformationDataType;
  typedef GreedyIteratorParam ParamType;

  /* scratch sized once for the finest grid and reused across scale levels,
   * as GreedyIteratorGPU does (GreedyIteratorGPU.cxx:36-43) */
  GreedyIteratorB200(const SizeType &size, const OriginType &origin, const SpacingType &spacing,
                     bool debug = true)
      : DeformationIteratorInterface(size, origin, spacing), mDebug(debug) {
    const size_t n = (size_t)size.x * size.y * size.z;
    if (cudaMalloc((void **)&mScratch, 6 * n * sizeof(float)) != cudaSuccess)
      throw AtlasWerksException(__FILE__, __LINE__, "GreedyIteratorB200: scratch allocation");
  }

  ~GreedyIteratorB200() {
    if (mHandle) aw_greedy_destroy(mHandle);
    if (mScratch) cudaFree(mScratch);
  }

  /* GreedyIteratorGPU::SetScaleLevel: a plan for the level's grid and the
   * DiffOper kernel (the only kernel DiffOperGPU-style plans support) */
  void SetScaleLevel(const MultiscaleManager &scaleManager, const GreedyIteratorParam &param) {
    ScaleLevelDataInfo::SetScaleLevel(scaleManager);
    const DiffOperParam *k = param.Kernel().AsDiffOperParam();
    if (!k)
      throw AtlasWerksException(__FILE__, __LINE__,
                                "GreedyIteratorB200: only the DiffOper kernel is supported");
    if (mHandle) aw_greedy_destroy(mHandle);
    mHandle = nullptr;
    check(aw_greedy_create(mCurSize.x, mCurSize.y, mCurSize.z, mCurSpacing.x, mCurSpacing.y,
                           mCurSpacing.z, k->Alpha(), k->Beta(), k->Gamma(), param.MaxPert(),
                           &mHandle),
          "SetScaleLevel");
    mStepKnown = false;  // a new handle starts from step 0
  }

  void UpdateStepSizeNextIteration() { mUpdateStep = true; }

  /* GreedyIteratorGPU::Iterate. Everything is queued on the default stream
   * without a host synchronisation, except where the data object needs a
   * host value: the step after a step-size update, and the energy when the
   * iterator was built with debug = true (as GreedyIteratorGPU computes the
   * energy only then). The step goes to the device only when the data
   * object's differs from the last one written or read. The library writes
   * h' to this iterator's scratch (the update reads h around every voxel, so
   * it cannot run in place) and an asynchronous device copy puts it back
   * into the data object's planes, which may lie apart.
   * Difference from the reference: GreedyDeformationData::AddEnergy halves
   * the step when AutoStepReduce is set and the energy rose; the reference
   * adds the energy before its update, this binding after it, so the halved
   * step takes effect one iteration later. */
  void Iterate(DeformationDataInterface &deformationData) {
    GreedyDeformationDataGPU &data = dynamic_cast<GreedyDeformationDataGPU &>(deformationData);
    const size_t n = (size_t)mCurSize.x * mCurSize.y * mCurSize.z;
    if (!mStepKnown || data.StepSize() != mStep) {
      check(aw_greedy_set_step(mHandle, data.StepSize()), "Iterate (step)");
      mStep = data.StepSize();
      mStepKnown = true;
    }
    cplVector3DArray &h = data.dDef1To0();
    float *s = mScratch, *si = mScratch + 3 * n;
    const bool inv = data.ComputeInverseHField();
    cplVector3DArray *hi = inv ? &data.dDef0To1() : nullptr;
    check(aw_greedy_iterate(mHandle, data.dI0(), data.dI1(), h.x, h.y, h.z, s, s + n, s + 2 * n,
                            inv ? hi->x : nullptr, inv ? hi->y : nullptr, inv ? hi->z : nullptr,
                            inv ? si : nullptr, inv ? si + n : nullptr, inv ? si + 2 * n : nullptr,
                            mUpdateStep ? 1 : 0, nullptr),
          "Iterate");
    copy3(s, n, h);
    if (inv) copy3(si, n, *hi);
    if (mUpdateStep) {
      float step = 0.f;
      check(aw_greedy_get_step(mHandle, &step), "Iterate (step)");
      data.StepSize(step);
      mStep = step;
    }
    mUpdateStep = false;
    if (mDebug) {
      double e = 0.0;
      check(aw_greedy_last_energy(mHandle, &e), "Iterate (energy)");
      Energy energy;
      energy.SetEnergy((Real)e);
      data.AddEnergy(energy);
    }
  }

 private:
  static void check(int rc, const char *what) {
    if (rc != 0)
      throw AtlasWerksException(__FILE__, __LINE__,
                                std::string("libaw_b200 ") + what + ": " + aw_last_error());
  }
  /* stream-ordered device copies on the default stream, no host wait */
  static void copy3(const float *src, size_t n, cplVector3DArray &dst) {
    float *d[3] = {dst.x, dst.y, dst.z};
    for (int c = 0; c < 3; ++c)
      if (cudaMemcpyAsync(d[c], src + c * n, n * sizeof(float), cudaMemcpyDeviceToDevice, 0) !=
          cudaSuccess)
        throw AtlasWerksException(__FILE__, __LINE__, "GreedyIteratorB200: field copy");
  }

  aw_greedy_t mHandle = nullptr;
  float *mScratch = nullptr;
  bool mUpdateStep = false;
  bool mStepKnown = false;  // mStep mirrors the device step
  float mStep = 0.f;
  bool mDebug;
};

#endif
