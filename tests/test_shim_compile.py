"""The reference-side bindings (include/aw_b200_greedy_iterator.hpp,
aw_b200_ldmm_iterator.hpp, aw_b200_diffoper.hpp) compile against the
reference's own headers: a syntax-only g++ run over a translation unit that
makes the calls GreedyWarp<T>::RunWarp makes of its iterator
(Algorithms/Greedy/GreedyWarp.txx:40-125), the calls LDMMWarp<T>::RunWarp
and the LDMM atlas make of theirs (Algorithms/LDMM/LDMMWarp.txx:71-130), and
the KernelFactory::NewGPUKernel choice of a DiffOper kernel
(Algorithms/Common/KernelFactory.cxx:45-60). Runs where the reference tree
is present (the bindings are meant to be built inside it);
tests/test_bindings_run.py links and runs them over stand-in headers."""
import os
import subprocess

import pytest

from oracle import reference_root

REF = reference_root()
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

TU = r"""
#include "aw_b200_greedy_iterator.hpp"
#include "GreedyParam.h"

// the iterator concept of GreedyWarp<GreedyIteratorT>
template <class GreedyIteratorT>
void run_like_greedy_warp(const RealImage *I0, const RealImage *I1, const GreedyParam &param) {
  typedef typename GreedyIteratorT::DeformationDataType DeformationDataType;
  typedef typename GreedyIteratorT::ParamType IteratorParamType;
  SizeType size = I0->getSize();
  OriginType origin = I0->getOrigin();
  SpacingType spacing = I0->getSpacing();
  DeformationDataType data(I0, I1, param);
  MultiscaleManager scaleManager(size, spacing, origin, param);
  GreedyIteratorT *it = new GreedyIteratorT(size, origin, spacing, true);
  data.InitializeWarp();
  for (unsigned int level = 0; level < param.GetNumberOfScaleLevels(); ++level) {
    scaleManager.SetScaleLevel(level);
    const IteratorParamType &p = param.GetScaleLevel(level).Iterator();
    it->SetScaleLevel(scaleManager, p);
    data.SetScaleLevel(scaleManager);
    for (unsigned int iter = 0; iter < param.GetScaleLevel(level).NIterations(); ++iter) {
      data.SetCurIter(iter);
      if (iter == 0) it->UpdateStepSizeNextIteration();
      it->Iterate(data);
    }
  }
  data.FinalizeWarp();
  delete it;
}

template void run_like_greedy_warp<GreedyIteratorB200>(const RealImage *, const RealImage *,
                                                       const GreedyParam &);

#include "aw_b200_diffoper.hpp"
#include "aw_b200_ldmm_iterator.hpp"

// the iterator concept of LDMMWarp<LDMMIteratorT> and the LDMM atlas thread
template <class LDMMIteratorT>
void run_like_ldmm_warp(const RealImage *I0, const RealImage *I1, const LDMMParam &param) {
  typedef typename LDMMIteratorT::DeformationDataType DeformationDataType;
  typedef typename LDMMIteratorT::ParamType IteratorParamType;
  SizeType size = I0->getSize();
  OriginType origin = I0->getOrigin();
  SpacingType spacing = I0->getSpacing();
  unsigned int nt = param.NTimeSteps();
  DeformationDataType data(I0, I1, param);
  MultiscaleManager scaleManager(size, spacing, origin, param);
  LDMMIteratorT *it = new LDMMIteratorT(size, origin, spacing, nt, true);
  data.InitializeWarp();
  for (unsigned int level = 0; level < param.GetNumberOfScaleLevels(); ++level) {
    scaleManager.SetScaleLevel(level);
    const IteratorParamType &p = param.GetScaleLevel(level).Iterator();
    it->SetScaleLevel(scaleManager, p);
    data.SetScaleLevel(scaleManager);
    data.StepSize(p.StepSize());
    for (unsigned int iter = 0; iter < param.GetScaleLevel(level).NIterations(); ++iter) {
      if (iter == 0 && p.UseAdaptiveStepSize()) {
        it->UpdateStepSizeNextIteration();
        it->Iterate(data);
      }
      data.SetCurIter(iter);
      it->Iterate(data);
    }
  }
  it->Iterate(data, true);
  float *alpha0 = it->GetAlpha(0);
  it->ComputeJacDet(data.dV(), alpha0);
  data.FinalizeWarp();
  delete it;
}

template void run_like_ldmm_warp<LDMMIteratorB200>(const RealImage *, const RealImage *,
                                                   const LDMMParam &);

// KernelFactory::NewGPUKernel with the B200 operator for DiffOper parameters
KernelInterfaceGPU *new_gpu_kernel(const KernelParam &param, const SizeType &size,
                                   const SpacingType &spacing, cplVector3DArray &field) {
  KernelInterfaceGPU *kernel = nullptr;
  if (param.IsDiffOperParam()) kernel = new DiffOperB200();
  kernel->SetSize(size, spacing, param);
  kernel->ApplyInverseOperator(field);
  kernel->ApplyOperator(field);
  return kernel;
}
"""


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference tree not present")
def test_bindings_compile_in_the_reference_tree(tmp_path):
    (tmp_path / "cutil.h").write_text("/* the 2011 CUDA SDK header the reference includes */\n")
    (tmp_path / "tu.cxx").write_text(TU)
    L = os.path.join(REF, "Code", "Libraries")
    U = os.path.join(REF, "Utilities")
    inc = [os.path.join(ROOT, "include"), "/usr/local/cuda/include",
           os.path.join(ROOT, "oracle", "ref", "stubs"), str(tmp_path)]
    inc += [os.path.join(L, d) for d in ("", "Base", "DataTypes", "UtilitiesDataTypes", "Numerics",
                                         "Algorithms/Common", "Algorithms/Greedy",
                                         "Algorithms/LDMM", "CUDACommon/inc")]
    inc += [os.path.join(U, d) for d in ("DownsampleFilter", "Matrix", "PowerCrust", "tinyxml")]
    cmd = ["/usr/bin/g++", "-std=c++14", "-DTIXML_USE_STL", "-fsyntax-only", "-w"]
    cmd += ["-I" + d for d in inc] + [str(tmp_path / "tu.cxx")]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
