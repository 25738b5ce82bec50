// stand-in: KernelInterfaceGPU (Algorithms/Common/KernelInterfaceGPU.h:20-43)
#pragma once
#include "KernelParam.h"
#include "cudaVector3DArray.h"
class KernelInterfaceGPU {
 public:
  virtual ~KernelInterfaceGPU() {}
  virtual void SetSize(const SizeType &s, const SpacingType &sp, const KernelParam &p) = 0;
  virtual void ApplyOperator(cplVector3DArray &dV) = 0;
  virtual void ApplyInverseOperator(cplVector3DArray &dF) = 0;
};
