// stand-in: MultiscaleManager (Algorithms/Common/MultiscaleManager.h): the current level's grid
#pragma once
typedef float Real;
struct Vec3i { unsigned x, y, z; };
struct Vec3d { double x, y, z; };
typedef Vec3i SizeType;
typedef Vec3d SpacingType;
typedef Vec3d OriginType;
class MultiscaleManager {
 public:
  MultiscaleManager(SizeType s, SpacingType sp) : mSize(s), mSpacing(sp) {}
  SizeType CurScaleSize() const { return mSize; }
  SpacingType CurScaleSpacing() const { return mSpacing; }
 private:
  SizeType mSize;
  SpacingType mSpacing;
};
