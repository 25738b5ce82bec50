/*
 * lapack_stub.cxx — LAPACK symbols referenced by the reference's Matrix3D
 * (eigen-decomposition and inverse; DataTypes/Matrix3D.txx). They serve the
 * eigen-LUT operator variant, which the registration path does not use, so
 * each one aborts if it is ever reached. TEST INFRASTRUCTURE only.
 */
#include <cstdio>
#include <cstdlib>

extern "C" {
static void lapack_missing(const char *name) {
  std::fprintf(stderr, "lapack stub: %s is not on the registration path\n", name);
  std::abort();
}
void dgetrf_() { lapack_missing("dgetrf"); }
void dgetri_() { lapack_missing("dgetri"); }
void dsyev_() { lapack_missing("dsyev"); }
}
