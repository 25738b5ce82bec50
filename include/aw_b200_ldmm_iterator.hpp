/*
 * aw_b200_ldmm_iterator.hpp — the reference-side binding of the LDMM
 * relaxation: an iterator with the interface LDMMWarp<T> and the LDMM atlas
 * thread expect of LDMMIteratorGPU (Algorithms/LDMM/LDMMIteratorGPU.h:27-106),
 * over libaw_b200.so's aw_ldmm_* entry points:
 *
 *     LDMMWarp<LDMMIteratorB200> warp(I0, I1, param);
 *
 * Header-only; compiled inside the AtlasWerks tree (LDMMDeformationDataGPU,
 * LDMMIteratorParam, LDMMEnergy, MultiscaleManager, cplVector3DArray,
 * AtlasWerksException) and linked against libaw_b200.so.
 *
 * The library keeps the T velocity fields as one [T][3][N] block; the data
 * object keeps T separate cplVector3DArray. Iterate gathers them into the
 * block, runs the iteration and scatters them back with stream-ordered
 * device copies (2 x 12 T N bytes, a few percent of an iteration's own
 * traffic); no host synchronisation except where the data object needs a
 * host value (the step after an adaptive-step pass, the image energy in
 * debug mode).
 *
 * In debug mode the energy added to the data object holds the image term
 * and the per-time-step vector energies <L v_t, v_t> (the library forms
 * them with one more transform per time step, aw_ldmm_set_vector_energy, as
 * the reference's debug mode does). What differs from LDMMIteratorGPU:
 * ReParameterize is not provided (it throws; LDMMWarp calls it only when
 * ReparameterizeEveryNIterations > 0, default 0).
 */
#ifndef AW_B200_LDMM_ITERATOR_HPP
#define AW_B200_LDMM_ITERATOR_HPP

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "aw_b200.h"

#include "AtlasWerksException.h"
#include "DeformationIteratorInterface.h"
#include "LDMMDeformationDataGPU.h"
#include "LDMMEnergy.h"
#include "LDMMParam.h"
#include "MultiscaleManager.h"

class LDMMIteratorB200 : public DeformationIteratorInterface {
 public:
  typedef LDMMDeformationDataGPU DeformationDataType;
  typedef LDMMIteratorParam ParamType;

  /* scratch sized once for the finest grid (LDMMIteratorGPU's constructor) */
  LDMMIteratorB200(SizeType &size, OriginType &origin, SpacingType &spacing,
                   unsigned int &nTimeSteps, bool debug = true)
      : DeformationIteratorInterface(size, origin, spacing), mNTimeSteps(nTimeSteps),
        mDebug(debug) {
    const size_t n = (size_t)size.x * size.y * size.z;
    // v block [T][3][N], alphas [T][N], two images for ComputeJacDet
    if (cudaMalloc((void **)&mV, (3 * mNTimeSteps + mNTimeSteps + 2) * n * sizeof(float)) !=
        cudaSuccess)
      throw AtlasWerksException(__FILE__, __LINE__, "LDMMIteratorB200: scratch allocation");
    mAlphas = mV + 3 * mNTimeSteps * n;
    mImg = mAlphas + mNTimeSteps * n;
  }

  ~LDMMIteratorB200() {
    if (mHandle) aw_ldmm_destroy(mHandle);
    if (mV) cudaFree(mV);
  }

  /* LDMMIteratorGPU::SetScaleLevel: the level's grid and spacing, the
   * DiffOper kernel, sigma and MaxPert; the step comes from the data object
   * (LDMMWarp sets it from the parameter after this call) */
  void SetScaleLevel(const MultiscaleManager &scaleManager, const LDMMIteratorParam &param) {
    ScaleLevelDataInfo::SetScaleLevel(scaleManager);
    const DiffOperParam *k = param.Kernel().AsDiffOperParam();
    if (!k)
      throw AtlasWerksException(__FILE__, __LINE__,
                                "LDMMIteratorB200: only the DiffOper kernel is supported");
    if (mHandle) aw_ldmm_destroy(mHandle);
    mHandle = nullptr;
    check(aw_ldmm_create(mCurSize.x, mCurSize.y, mCurSize.z, mCurSpacing.x, mCurSpacing.y,
                         mCurSpacing.z, k->Alpha(), k->Beta(), k->Gamma(), (int)mNTimeSteps,
                         param.Sigma(), param.MaxPert(), &mHandle),
          "SetScaleLevel");
    if (mDebug) check(aw_ldmm_set_vector_energy(mHandle, 1), "SetScaleLevel");
    mSigma = param.Sigma();
    mStepKnown = false;
    mAlphasValid = false;
  }

  void UpdateStepSizeNextIteration() { mUpdateStep = true; }

  void Iterate(DeformationDataInterface &defData) { Iterate(defData, false); }

  /* LDMMIteratorGPU::Iterate(defData, computeAlphasOnly): the splatting
   * gradient (IterateNew); with computeAlphasOnly the velocities stay and
   * GetAlpha(t) returns alpha_t until the next Iterate without it */
  void Iterate(DeformationDataInterface &defData, bool computeAlphasOnly) {
    LDMMDeformationDataGPU &data = dynamic_cast<LDMMDeformationDataGPU &>(defData);
    const size_t n = curVox();
    gather(data.dV(), n);
    if (computeAlphasOnly) {
      check(aw_ldmm_alphas(mHandle, data.dI0(), data.dI1(), mV, mAlphas, nullptr), "Iterate");
      mAlphasValid = true;
    } else {
      if (!mStepKnown || data.StepSize() != mStep) {
        check(aw_ldmm_set_step(mHandle, data.StepSize()), "Iterate (step)");
        mStep = data.StepSize();
        mStepKnown = true;
      }
      check(aw_ldmm_iterate(mHandle, data.dI0(), data.dI1(), mV, mUpdateStep ? 1 : 0, nullptr),
            "Iterate");
      scatter(data.dV(), n);
      mAlphasValid = false;
      if (mUpdateStep) {
        float step = 0.f;
        check(aw_ldmm_get_step(mHandle, &step), "Iterate (step)");
        data.StepSize(step);
        mStep = step;
        mUpdateStep = false;
        return;  // the adaptive-step pass records no energy
      }
    }
    if (mDebug) {
      int count = 0;
      check(aw_ldmm_get_energies(mHandle, nullptr, 0, &count), "Iterate (energy)");
      std::vector<double> all(count > 0 ? count : 1);
      int got = 0;
      check(aw_ldmm_get_energies(mHandle, all.data(), count, &got), "Iterate (energy)");
      LDMMEnergy energy(mNTimeSteps, mSigma);
      if (!computeAlphasOnly) {
        // set in the iteration's order, t = T-1 down to 0 (IterateNew)
        std::vector<double> steps(mNTimeSteps);
        check(aw_ldmm_get_vec_step_energies(mHandle, steps.data(), (int)mNTimeSteps),
              "Iterate (energy)");
        for (unsigned int t = mNTimeSteps; t-- > 0;) energy.SetVecStepEnergy((Real)steps[t]);
      }
      energy.SetImageEnergy(got > 0 ? (Real)all[got - 1] : (Real)0);
      data.AddEnergy(energy);
    }
  }

  float *GetAlpha(unsigned int t) {
    if (!mAlphasValid || t >= mNTimeSteps)
      throw AtlasWerksException(__FILE__, __LINE__,
                                "LDMMIteratorB200::GetAlpha: call Iterate(data, true) first");
    return mAlphas + (size_t)t * curVox();
  }

  /* LDMMIteratorGPU::ComputeJacDet: |D h_{0->1}| transported along the
   * velocities (LDMMIteratorCPU::ComputeJacDet, LDMMIteratorCPU.cxx:309-340) */
  void ComputeJacDet(std::vector<cplVector3DArray> &dV, float *dJacDet) {
    const size_t n = curVox();
    gather(dV, n);
    check(cudaMemsetAsync(mImg, 0, n * sizeof(float), 0) == cudaSuccess ? 0 : 1,
          "ComputeJacDet (scratch)");
    check(aw_ldmm_i1_at_0(mHandle, mImg, mV, mImg + n, dJacDet, nullptr), "ComputeJacDet");
  }

  void ReParameterize(LDMMDeformationDataGPU &) {
    throw AtlasWerksException(__FILE__, __LINE__,
                              "LDMMIteratorB200: ReParameterize is not provided");
  }

 private:
  size_t curVox() const { return (size_t)mCurSize.x * mCurSize.y * mCurSize.z; }
  void gather(std::vector<cplVector3DArray> &dV, size_t n) {
    for (unsigned t = 0; t < mNTimeSteps; ++t)
      for (int c = 0; c < 3; ++c)
        copy(mV + (3 * t + c) * n, dV[t].elementArray(c), n);
  }
  void scatter(std::vector<cplVector3DArray> &dV, size_t n) {
    for (unsigned t = 0; t < mNTimeSteps; ++t)
      for (int c = 0; c < 3; ++c)
        copy(dV[t].elementArray(c), mV + (3 * t + c) * n, n);
  }
  static void copy(float *dst, const float *src, size_t n) {
    if (cudaMemcpyAsync(dst, src, n * sizeof(float), cudaMemcpyDeviceToDevice, 0) != cudaSuccess)
      throw AtlasWerksException(__FILE__, __LINE__, "LDMMIteratorB200: field copy");
  }
  static void check(int rc, const char *what) {
    if (rc != 0)
      throw AtlasWerksException(__FILE__, __LINE__,
                                std::string("libaw_b200 LDMMIteratorB200::") + what + ": " +
                                    aw_last_error());
  }

  const unsigned int mNTimeSteps;
  aw_ldmm_t mHandle = nullptr;
  float *mV = nullptr, *mAlphas = nullptr, *mImg = nullptr;
  Real mSigma = 0;
  bool mUpdateStep = false;
  bool mStepKnown = false;
  float mStep = 0.f;
  bool mAlphasValid = false;
  bool mDebug;
};

#endif
