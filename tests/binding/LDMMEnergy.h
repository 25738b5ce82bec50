// stand-in: LDMMEnergy (Algorithms/LDMM/LDMMEnergy.h): image term only
#pragma once
#include "Energy.h"
class LDMMEnergy : public Energy {
 public:
  LDMMEnergy(int nTimeSteps, Real sigma) : mSigma(sigma) { (void)nTimeSteps; }
  void SetImageEnergy(Real e) { mEnergy = e; }
 private:
  Real mSigma;
};
