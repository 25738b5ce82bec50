/*
 * aw_b200_diffoper.hpp — the reference-side binding of the fluid operator:
 * a KernelInterfaceGPU (Algorithms/Common/KernelInterfaceGPU.h:20-43) over
 * libaw_b200.so's aw_fluid_* entry points, the drop-in for DiffOperGPU
 * (Algorithms/Common/DiffOperGPU.cxx). KernelFactory::NewGPUKernel
 * (Algorithms/Common/KernelFactory.cxx:45-60) returns one for a DiffOper
 * parameter with
 *
 *     if (param.IsDiffOperParam()) kernel = new DiffOperB200();
 *
 * Header-only; compiled inside the AtlasWerks tree (KernelInterfaceGPU,
 * KernelParam, DiffOperParam, cplVector3DArray, AtlasWerksException) and
 * linked against libaw_b200.so. Applies L (ApplyOperator) or K = L^-1
 * (ApplyInverseOperator) in place on the three planes of a device field,
 * on the default stream, as DiffOperGPU does.
 */
#ifndef AW_B200_DIFFOPER_HPP
#define AW_B200_DIFFOPER_HPP

#include <string>

#include "aw_b200.h"

#include "AtlasWerksException.h"
#include "DiffOperParam.h"
#include "KernelInterfaceGPU.h"
#include "KernelParam.h"

class DiffOperB200 : public KernelInterfaceGPU {
 public:
  DiffOperB200() {}
  ~DiffOperB200() {
    if (mPlan) aw_fluid_destroy(mPlan);
  }

  /* DiffOperGPU::SetSize plus its parameter checks: the GPU operator has
   * no powers of L, no eigen LUT and no divergence-free projection
   * (DiffOperGPU.cxx:127-160), and neither has this one */
  void SetSize(const SizeType &logicalSize, const SpacingType &spacing,
               const KernelParam &params) {
    const DiffOperParam *k = params.AsDiffOperParam();
    if (!k)
      throw AtlasWerksException(__FILE__, __LINE__, "DiffOperB200: not a DiffOper parameter");
    if (k->LPow() != 1.0)
      throw AtlasWerksException(__FILE__, __LINE__, "Error, powers of L not supported on the GPU!");
    if (k->UseEigenLUT())
      throw AtlasWerksException(__FILE__, __LINE__, "Error, eigen LUT not supported on the GPU!");
    if (k->DivergenceFree())
      throw AtlasWerksException(__FILE__, __LINE__,
                                "Error, divergence free projection not implemented on the GPU!");
    if (mPlan) aw_fluid_destroy(mPlan);
    mPlan = nullptr;
    check(aw_fluid_create(logicalSize.x, logicalSize.y, logicalSize.z, spacing.x, spacing.y,
                          spacing.z, k->Alpha(), k->Beta(), k->Gamma(), &mPlan),
          "SetSize");
  }

  /* f = L v, overwriting v */
  void ApplyOperator(cplVector3DArray &dV) { apply(dV, 0, "ApplyOperator"); }

  /* v = K f, overwriting f */
  void ApplyInverseOperator(cplVector3DArray &dF) { apply(dF, 1, "ApplyInverseOperator"); }

 private:
  void apply(cplVector3DArray &a, int inverse, const char *what) {
    if (!mPlan)
      throw AtlasWerksException(__FILE__, __LINE__,
                                "Error, DiffOperB200 not initialized, please call SetSize first!");
    check(aw_fluid_apply(mPlan, a.x, a.y, a.z, inverse, nullptr), what);
  }
  static void check(int rc, const char *what) {
    if (rc != 0)
      throw AtlasWerksException(__FILE__, __LINE__,
                                std::string("libaw_b200 DiffOperB200::") + what + ": " +
                                    aw_last_error());
  }

  aw_fluid_t mPlan = nullptr;
};

#endif
