// stand-in: KernelParam (Algorithms/Common/KernelParam.h) holding a DiffOper parameter
#pragma once
#include "DiffOperParam.h"
class KernelParam {
 public:
  explicit KernelParam(const DiffOperParam &p) : mDiffOper(p) {}
  bool IsDiffOperParam() const { return true; }
  const DiffOperParam *AsDiffOperParam() const { return &mDiffOper; }
 private:
  DiffOperParam mDiffOper;
};
