/* Compile-only stand-in for the ITK transform reader: declares just enough
   for AffineTransform3D::readITKStyle to parse; it is never called. */
#ifndef STUB_ITK_TFR_H
#define STUB_ITK_TFR_H
#include <list>
#include <stdexcept>
namespace itk {
template <class P> struct StubPtr {
  P *p;
  StubPtr(P *q = 0) : p(q) {}
  P *operator->() const { return p; }
  P *GetPointer() const { return p; }
  bool operator!() const { return !p; }
};
struct TransformBase { virtual ~TransformBase() {} };
template <class T, unsigned R, unsigned C> struct Matrix {
  T a[R][C];
  T operator()(unsigned r, unsigned c) const { return a[r][c]; }
};
template <class T, unsigned N> struct FixedArray {
  T a[N];
  T operator[](unsigned i) const { return a[i]; }
};
template <class T, unsigned D> struct AffineTransform : TransformBase {
  typedef StubPtr<AffineTransform> Pointer;
  Matrix<T, D, D> GetMatrix() const { return Matrix<T, D, D>(); }
  FixedArray<T, D> GetOffset() const { return FixedArray<T, D>(); }
};
struct TransformFileReader {
  typedef StubPtr<TransformFileReader> Pointer;
  typedef std::list<StubPtr<TransformBase> > TransformListType;
  static Pointer New() { throw std::runtime_error("ITK is not available"); }
  void SetFileName(const char *) {}
  void Update() {}
  TransformListType *GetTransformList() { return 0; }
};
}
#endif
