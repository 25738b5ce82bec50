// stand-in: GreedyIteratorParam (Algorithms/Greedy/GreedyIteratorParam.h:27-34)
#pragma once
#include "KernelParam.h"
class GreedyIteratorParam {
 public:
  GreedyIteratorParam(const KernelParam &k, Real maxPert) : mK(k), mMaxPert(maxPert) {}
  const KernelParam &Kernel() const { return mK; }
  Real MaxPert() const { return mMaxPert; }
 private:
  KernelParam mK;
  Real mMaxPert;
};
