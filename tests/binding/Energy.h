// stand-in: Energy (Algorithms/Common/Energy.h)
#pragma once
#include "MultiscaleManager.h"
class Energy {
 public:
  virtual ~Energy() {}
  void SetEnergy(Real e) { mEnergy = e; }
  virtual Real GetEnergy() const { return mEnergy; }
 protected:
  Real mEnergy = 0;
};
