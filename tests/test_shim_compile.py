"""The reference-side binding (include/aw_b200_greedy_iterator.hpp) compiles
against the reference's own headers as the template argument of its
greedy loop: a syntax-only g++ run over a translation unit that makes the
calls GreedyWarp<T>::RunWarp makes of its iterator
(Algorithms/Greedy/GreedyWarp.txx:40-125). Runs where the reference tree
is present (the binding is meant to be built inside it)."""
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
"""


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference tree not present")
def test_greedy_iterator_binding_compiles_in_the_reference_tree(tmp_path):
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
