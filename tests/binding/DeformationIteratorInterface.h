// stand-in: ScaleLevelDataInfo / DeformationDataInterface / DeformationIteratorInterface
// (Algorithms/Common/DeformationIteratorInterface.h) with the members the bindings use
#pragma once
#include <vector>
#include "Energy.h"
#include "MultiscaleManager.h"
class ScaleLevelDataInfo {
 public:
  ScaleLevelDataInfo(SizeType size, OriginType origin, SpacingType spacing)
      : mImSize(size), mImOrigin(origin), mImSpacing(spacing), mCurSize(size),
        mCurSpacing(spacing) {}
  virtual ~ScaleLevelDataInfo() {}
  virtual void SetScaleLevel(const MultiscaleManager &m) {
    mCurSize = m.CurScaleSize();
    mCurSpacing = m.CurScaleSpacing();
  }
 protected:
  SizeType mImSize;
  OriginType mImOrigin;
  SpacingType mImSpacing;
  SizeType mCurSize;
  SpacingType mCurSpacing;
};
class DeformationDataInterface : public ScaleLevelDataInfo {
 public:
  DeformationDataInterface(SizeType s, OriginType o, SpacingType sp) : ScaleLevelDataInfo(s, o, sp) {}
  virtual ~DeformationDataInterface() {}
  virtual void AddEnergy(const Energy &e) { mEnergies.push_back(e.GetEnergy()); }
  Real StepSize() { return mStepSize; }
  void StepSize(Real s) { mStepSize = s; }
  std::vector<Real> mEnergies;
 protected:
  Real mStepSize = 0;
};
class DeformationIteratorInterface : public ScaleLevelDataInfo {
 public:
  DeformationIteratorInterface(SizeType s, OriginType o, SpacingType sp) : ScaleLevelDataInfo(s, o, sp) {}
  virtual ~DeformationIteratorInterface() {}
  virtual void Iterate(DeformationDataInterface &d) = 0;
};
