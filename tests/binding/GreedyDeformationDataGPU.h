// stand-in: GreedyDeformationDataGPU (Algorithms/Greedy/GreedyDeformationDataGPU.h:29-51):
// device images and the deformation planes of one registration
#pragma once
#include "DeformationIteratorInterface.h"
#include "cudaVector3DArray.h"
class GreedyDeformationDataGPU : public DeformationDataInterface {
 public:
  GreedyDeformationDataGPU(SizeType s, SpacingType sp, float *I0, float *I1, cplVector3DArray h,
                           cplVector3DArray hinv, bool inverse)
      : DeformationDataInterface(s, OriginType{0, 0, 0}, sp), mI0(I0), mI1(I1), mH(h),
        mHinv(hinv), mInverse(inverse) {}
  float *dI0() { return mI0; }
  float *dI1() { return mI1; }
  cplVector3DArray &dDef1To0() { return mH; }
  cplVector3DArray &dDef0To1() { return mHinv; }
  bool ComputeInverseHField() const { return mInverse; }
 private:
  float *mI0, *mI1;
  cplVector3DArray mH, mHinv;
  bool mInverse;
};
