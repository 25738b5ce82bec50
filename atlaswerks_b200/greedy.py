"""Host-side mirror of the reference's greedy-fluid interfaces.

Names, arguments and error behaviour follow the reference C++ classes so a
reference user finds the same concepts:

* ``DiffOperB200`` — KernelInterfaceGPU / DiffOperGPU
  (Algorithms/Common/KernelInterfaceGPU.h:20-43): ``SetSize``,
  ``ApplyOperator``, ``ApplyInverseOperator`` on a device vector field, in
  place.
* ``GreedyDeformationDataB200`` — GreedyDeformationData(GPU)
  (Algorithms/Greedy/GreedyDeformationData.h:31-130): images, the
  deformation ``Def1To0`` and its inverse ``Def0To1``, ``StepSize``, energy
  history.
* ``GreedyIteratorB200`` — GreedyIteratorGPU
  (Algorithms/Greedy/GreedyIteratorGPU.h:32-58): ``SetScaleLevel``,
  ``Iterate``, ``UpdateStepSizeNextIteration``.

Every computation runs in libaw_b200.so through the C ABI.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import check
from .device import _check_field, _check_image, _dims, _stream, identity


@dataclass
class DiffOperParam:
    """DiffOperParam (Algorithms/Common/DiffOperParam.h:33-71) defaults."""
    Alpha: float = 0.01
    Beta: float = 0.01
    Gamma: float = 0.001
    LPow: float = 1.0
    UseEigenLUT: bool = False
    DivergenceFree: bool = False


class DiffOperB200:
    """The fluid kernel K = L^-1 on the GPU (DiffOperGPU equivalent)."""

    def __init__(self):
        self._h = ctypes.c_void_p()
        self.size = None

    def SetSize(self, size: Sequence[int], spacing: Sequence[float], param: DiffOperParam):
        """size = (nx, ny, nz). Rejects what DiffOperGPU rejects
        (Common/DiffOperGPU.cxx:127-156): LPow != 1, UseEigenLUT, DivergenceFree."""
        if param.LPow != 1.0:
            raise ValueError("LPow != 1 is not supported on the GPU path (DiffOperGPU)")
        if param.UseEigenLUT:
            raise ValueError("UseEigenLUT is not supported on the GPU path (DiffOperGPU)")
        if param.DivergenceFree:
            raise ValueError("DivergenceFree is not supported on the GPU path (DiffOperGPU)")
        self._free()
        nx, ny, nz = size
        check(_lib.lib().aw_fluid_create(nx, ny, nz, *map(float, spacing), param.Alpha,
                                         param.Beta, param.Gamma, ctypes.byref(self._h)))
        self.size = (nx, ny, nz)

    def _apply(self, v: torch.Tensor, inverse: int):
        _check_field(v, "v")
        if self.size is None:
            raise RuntimeError("SetSize() must be called first")
        if tuple(v.shape[1:]) != (self.size[2], self.size[1], self.size[0]):
            raise ValueError("field size does not match SetSize()")
        check(_lib.lib().aw_fluid_apply(self._h, v[0].data_ptr(), v[1].data_ptr(),
                                        v[2].data_ptr(), inverse, _stream()))
        return v

    def ApplyOperator(self, v: torch.Tensor) -> torch.Tensor:
        return self._apply(v, 0)

    def ApplyInverseOperator(self, v: torch.Tensor) -> torch.Tensor:
        return self._apply(v, 1)

    def TimedOut(self) -> bool:
        """True when a transform's bounded wait ran out since the last call
        (its output is then incomplete); synchronises the current stream and
        clears the flag."""
        flag = ctypes.c_int()
        check(_lib.lib().aw_fluid_status(self._h, ctypes.byref(flag), _stream()))
        return bool(flag.value)

    def _free(self):
        if self._h:
            _lib.lib().aw_fluid_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self._free()
        except Exception:
            pass


@dataclass
class GreedyIteratorParam:
    """GreedyIteratorParam (Algorithms/Greedy/GreedyIteratorParam.h:27-34)."""
    Kernel: DiffOperParam = None
    MaxPert: float = 0.1

    def __post_init__(self):
        if self.Kernel is None:
            self.Kernel = DiffOperParam()


class GreedyDeformationDataB200:
    """Images, deformation fields and step size of one registration."""

    def __init__(self, I0: torch.Tensor, I1: torch.Tensor, spacing=(1.0, 1.0, 1.0),
                 compute_inverse: bool = False):
        _check_image(I0, "I0")
        _check_image(I1, "I1")
        if I0.shape != I1.shape:
            raise ValueError("I0 and I1 must have the same grid")
        self.I0, self.I1 = I0, I1
        self.spacing = tuple(float(s) for s in spacing)
        self._compute_inverse = compute_inverse
        self._h = [identity(I0.shape, I0.device), torch.empty((3,) + tuple(I0.shape),
                                                               device=I0.device)]
        self._hi = ([identity(I0.shape, I0.device), torch.empty((3,) + tuple(I0.shape),
                                                                 device=I0.device)]
                    if compute_inverse else None)
        self._cur = 0
        self._step = 0.0

    def ComputeInverseHField(self) -> bool:
        return self._compute_inverse

    def SetToIdentity(self):
        """Def1To0 (and Def0To1) back to the identity, on the device and the
        current stream, as GreedyDeformationData::SetScaleLevel does at the
        initial scale level without an initial affine
        (GreedyDeformationData.cxx:193-208): the library's identity kernel,
        no allocation, so a registration can start again on the same data."""
        self._cur = 0
        nx, ny, nz = _dims(self.I0)
        for h in [self._h[0]] + ([self._hi[0]] if self._hi else []):
            check(_lib.lib().aw_identity(h[0].data_ptr(), h[1].data_ptr(), h[2].data_ptr(),
                                         nx, ny, nz, _stream()))

    def Def1To0(self) -> torch.Tensor:
        return self._h[self._cur]

    def Def0To1(self) -> torch.Tensor:
        if not self._compute_inverse:
            raise RuntimeError("Error, inverse HField not computed")
        return self._hi[self._cur]

    def _next(self):
        return self._h[1 - self._cur], (self._hi[1 - self._cur] if self._hi else None)

    def _swap(self):
        self._cur = 1 - self._cur


class GreedyIteratorB200:
    """GreedyIteratorGPU equivalent; state (step, energies) lives on the device."""

    DeformationDataType = GreedyDeformationDataB200
    ParamType = GreedyIteratorParam

    def __init__(self, size: Sequence[int], origin=(0.0, 0.0, 0.0), spacing=(1.0, 1.0, 1.0),
                 debug: bool = True):
        self.size = tuple(size)
        self.spacing = tuple(float(s) for s in spacing)
        self.debug = debug
        self._h = ctypes.c_void_p()
        self._update_step = False

    def SetScaleLevel(self, size: Sequence[int], spacing: Sequence[float],
                      param: GreedyIteratorParam):
        k = param.Kernel
        if k.LPow != 1.0 or k.UseEigenLUT or k.DivergenceFree:
            raise ValueError("LPow != 1, UseEigenLUT and DivergenceFree are not supported on the "
                             "GPU path (DiffOperGPU)")
        self._free()
        nx, ny, nz = size
        check(_lib.lib().aw_greedy_create(nx, ny, nz, *map(float, spacing), k.Alpha, k.Beta,
                                          k.Gamma, param.MaxPert, ctypes.byref(self._h)))
        self.size = (nx, ny, nz)
        self.spacing = tuple(float(s) for s in spacing)

    def UpdateStepSizeNextIteration(self):
        self._update_step = True

    def SetFastInterpolation(self, on: bool):
        """Float fused-multiply-add interpolation in the force preparation
        and the fused update (a few float ulps from the bit-exact path)."""
        check(_lib.lib().aw_greedy_set_fast_interpolation(self._h, int(on)))

    def SetAutoStepReduce(self, on: bool):
        check(_lib.lib().aw_greedy_set_auto_step_reduce(self._h, int(on)))

    def SetStepSize(self, step: float):
        check(_lib.lib().aw_greedy_set_step(self._h, float(step)))

    def StepSize(self) -> float:
        s = ctypes.c_float()
        check(_lib.lib().aw_greedy_get_step(self._h, ctypes.byref(s)))
        return float(s.value)

    def Iterate(self, data: GreedyDeformationDataB200):
        h, hi = data.Def1To0(), (data.Def0To1() if data.ComputeInverseHField() else None)
        ho, hio = data._next()
        z = [None, None, None]
        hp = [t.data_ptr() for t in h]
        op = [t.data_ptr() for t in ho]
        hip = [t.data_ptr() for t in hi] if hi is not None else z
        iop = [t.data_ptr() for t in hio] if hio is not None else z
        check(_lib.lib().aw_greedy_iterate(self._h, data.I0.data_ptr(), data.I1.data_ptr(), *hp,
                                           *op, *hip, *iop, int(self._update_step), _stream()))
        self._update_step = False
        data._swap()

    def Run(self, data: GreedyDeformationDataB200, n_iters: int, update_first: bool = True):
        """n_iters iterations replayed from a captured CUDA graph."""
        h, s = data.Def1To0(), data._next()[0]
        z = [None, None, None]
        if data.ComputeInverseHField():
            hi, si = data.Def0To1(), data._next()[1]
            hip, sip = [t.data_ptr() for t in hi], [t.data_ptr() for t in si]
        else:
            hip, sip = z, z
        check(_lib.lib().aw_greedy_run(self._h, data.I0.data_ptr(), data.I1.data_ptr(),
                                       *[t.data_ptr() for t in h], *[t.data_ptr() for t in s],
                                       *hip, *sip, int(n_iters), int(update_first), _stream()))

    def Energies(self) -> np.ndarray:
        n = ctypes.c_int()
        check(_lib.lib().aw_greedy_get_energies(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1), np.float64)
        check(_lib.lib().aw_greedy_get_energies(self._h, out.ctypes.data, n.value,
                                                ctypes.byref(n)))
        return out[: n.value]

    def _free(self):
        if self._h:
            _lib.lib().aw_greedy_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self._free()
        except Exception:
            pass


def greedy_register(I0: torch.Tensor, I1: torch.Tensor, n_iters: int,
                    spacing=(1.0, 1.0, 1.0), alpha=0.01, beta=0.01, gamma=0.001,
                    max_pert=0.5, compute_inverse=False):
    """Single-scale greedy registration from the identity (GreedyWarp at one
    scale level). Returns (h, hinv or None, energies, step)."""
    nz, ny, nx = I0.shape
    it = GreedyIteratorB200((nx, ny, nz), spacing=spacing)
    it.SetScaleLevel((nx, ny, nz), spacing,
                     GreedyIteratorParam(DiffOperParam(alpha, beta, gamma), max_pert))
    data = GreedyDeformationDataB200(I0, I1, spacing, compute_inverse)
    it.Run(data, n_iters, update_first=True)
    hinv = data.Def0To1() if compute_inverse else None
    return data.Def1To0(), hinv, it.Energies(), it.StepSize()
