// stand-in: DiffOperParam (Algorithms/Common/DiffOperParam.h:33-75)
#pragma once
#include "MultiscaleManager.h"
class DiffOperParam {
 public:
  DiffOperParam(Real a = 0.01f, Real b = 0.01f, Real g = 0.001f) : mA(a), mB(b), mG(g) {}
  Real Alpha() const { return mA; }
  Real Beta() const { return mB; }
  Real Gamma() const { return mG; }
  Real LPow() const { return mLPow; }
  bool UseEigenLUT() const { return false; }
  bool DivergenceFree() const { return false; }
  Real mLPow = 1.0f;
 private:
  Real mA, mB, mG;
};
