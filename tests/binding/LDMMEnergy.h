// stand-in: LDMMEnergy (Algorithms/LDMM/LDMMEnergy.h, .cxx): the image term
// and the per-time-step vector energies, GetEnergy = ImageEnergy() + VecEnergy()
#pragma once
#include <vector>
#include "Energy.h"
class LDMMEnergy : public Energy {
 public:
  LDMMEnergy(int nTimeSteps, Real sigma) : mSigma(sigma), mVec(nTimeSteps, 0.f) {}
  void SetImageEnergy(Real e) { mImage = e; }
  void SetVecStepEnergy(Real e) { mVec[mCur++] = e; }
  Real ImageEnergy() const { return (1.0 / (mSigma * mSigma)) * mImage; }
  Real VecEnergy() const {
    Real val = 0.0f;
    for (Real e : mVec) val += e;
    return val / mVec.size();
  }
  Real GetEnergy() const override { return ImageEnergy() + VecEnergy(); }
 private:
  Real mSigma;
  Real mImage = 0;
  std::vector<Real> mVec;
  unsigned mCur = 0;
};
