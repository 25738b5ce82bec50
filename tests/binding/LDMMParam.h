// stand-in: LDMMIteratorParam (Algorithms/LDMM/LDMMIteratorParam.h:57-62)
#pragma once
#include "KernelParam.h"
class LDMMIteratorParam {
 public:
  LDMMIteratorParam(const KernelParam &k, Real sigma, Real step, Real maxPert)
      : mK(k), mSigma(sigma), mStep(step), mMaxPert(maxPert) {}
  const KernelParam &Kernel() const { return mK; }
  Real Sigma() const { return mSigma; }
  Real StepSize() const { return mStep; }
  Real MaxPert() const { return mMaxPert; }
 private:
  KernelParam mK;
  Real mSigma, mStep, mMaxPert;
};
