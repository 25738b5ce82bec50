// stand-in: LDMMDeformationDataGPU (Algorithms/LDMM/LDMMDeformationDataGPU.h:30-70):
// device images and the T velocity fields
#pragma once
#include <vector>
#include "DeformationIteratorInterface.h"
#include "cudaVector3DArray.h"
class LDMMDeformationDataGPU : public DeformationDataInterface {
 public:
  LDMMDeformationDataGPU(SizeType s, SpacingType sp, float *I0, float *I1,
                         const std::vector<cplVector3DArray> &v)
      : DeformationDataInterface(s, OriginType{0, 0, 0}, sp), mI0(I0), mI1(I1), mV(v) {}
  float *dI0() { return mI0; }
  float *dI1() { return mI1; }
  std::vector<cplVector3DArray> &dV() { return mV; }
 private:
  float *mI0, *mI1;
  std::vector<cplVector3DArray> mV;
};
