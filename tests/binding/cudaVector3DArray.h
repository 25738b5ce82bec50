// stand-in: cplVector3DArray (CUDACommon/inc/cudaVector3DArray.h), three device planes
#pragma once
struct cplVector3DArray {
  float *x = nullptr, *y = nullptr, *z = nullptr;
  float *elementArray(int i) { return i == 0 ? x : i == 1 ? y : i == 2 ? z : nullptr; }
  const float *elementArray(int i) const { return i == 0 ? x : i == 1 ? y : i == 2 ? z : nullptr; }
};
