"""Host-side mirror of the reference's LDMM geodesic shooting interfaces.

* ``LDMMShootingDefDataB200`` — LDMMShootingDefData
  (Algorithms/LDMM/LDMMShootingDefData.h): I0, I1, the initial momentum
  ``Alpha0`` (a scalar image, zero at the start) and the two maps
  ``Phi0T`` / ``PhiT0`` the shooting leaves behind (``GetDef0To1`` /
  ``GetDef1To0``).
* ``LDMMShootingIteratorB200`` — LDMMShootingIteratorCPU / GPU
  (LDMM/LDMMShootingIteratorCPU.h): ``SetScaleLevel``, ``Iterate``: shoot the
  geodesic from alpha0 over T time steps, pull the residual back by
  splatting and update alpha0 (LDMMShootingIteratorCPU.cxx:199-304).

The iteration runs in libaw_b200.so (``aw_ldmm_shoot_iterate`` on an LDMM
handle, which holds T, sigma, the step size and the fluid kernel). The
energy history holds the image term sp^3 sum (I0(phiT0) - I1)^2; the
velocity terms LDMMEnergy adds are not formed.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np
import torch

from . import _lib
from ._lib import check
from .device import _check_image, _stream, apply, identity
from .ldmm import LDMMIteratorParam


class LDMMShootingDefDataB200:
    def __init__(self, I0: torch.Tensor, I1: torch.Tensor, spacing=(1.0, 1.0, 1.0)):
        _check_image(I0, "I0")
        _check_image(I1, "I1")
        if I0.shape != I1.shape:
            raise ValueError("I0 and I1 must have the same grid")
        self.I0, self.I1 = I0, I1
        self.spacing = tuple(float(s) for s in spacing)
        shape = tuple(I0.shape)
        self.Alpha0 = torch.zeros(shape, device=I0.device, dtype=torch.float32)
        self.Phi0T = identity(shape, I0.device)
        self.PhiT0 = identity(shape, I0.device)

    def GetDef0To1(self) -> torch.Tensor:
        return self.Phi0T

    def GetDef1To0(self) -> torch.Tensor:
        return self.PhiT0

    def GetI0At1(self) -> torch.Tensor:
        """I0 carried to time 1: I0(phiT0) (LDMMShootingDefData::GetI0At1)."""
        return apply(self.I0, self.PhiT0)

    def GetI1At0(self) -> torch.Tensor:
        """I1 carried to time 0: I1(phi0T) (LDMMShootingDefData::GetI1At0)."""
        return apply(self.I1, self.Phi0T)


class LDMMShootingIteratorB200:
    DeformationDataType = LDMMShootingDefDataB200
    ParamType = LDMMIteratorParam

    def __init__(self, size: Sequence[int], origin=(0.0, 0.0, 0.0), spacing=(1.0, 1.0, 1.0),
                 n_time_steps: int = 5, debug: bool = True):
        self.size = tuple(size)
        self.spacing = tuple(float(s) for s in spacing)
        self.T = int(n_time_steps)
        self._h = ctypes.c_void_p()

    def SetScaleLevel(self, size: Sequence[int], spacing: Sequence[float],
                      param: LDMMIteratorParam):
        k = param.Kernel
        if k.LPow != 1.0 or k.UseEigenLUT or k.DivergenceFree:
            raise ValueError("LPow != 1, UseEigenLUT and DivergenceFree are not supported on the "
                             "GPU path (DiffOperGPU)")
        self._free()
        nx, ny, nz = size
        check(_lib.lib().aw_ldmm_create(nx, ny, nz, *map(float, spacing), k.Alpha, k.Beta,
                                        k.Gamma, self.T, param.Sigma, param.MaxPert,
                                        ctypes.byref(self._h)))
        self.param = param
        check(_lib.lib().aw_ldmm_set_step(self._h, float(param.StepSize)))

    def Iterate(self, data: LDMMShootingDefDataB200):
        check(_lib.lib().aw_ldmm_shoot_iterate(self._h, data.I0.data_ptr(), data.I1.data_ptr(),
                                               data.Alpha0.data_ptr(), data.Phi0T.data_ptr(),
                                               data.PhiT0.data_ptr(), _stream()))

    def Energies(self) -> np.ndarray:
        n = ctypes.c_int()
        check(_lib.lib().aw_ldmm_get_energies(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1), np.float64)
        check(_lib.lib().aw_ldmm_get_energies(self._h, out.ctypes.data, n.value,
                                              ctypes.byref(n)))
        return out[: n.value]

    def _free(self):
        if self._h:
            _lib.lib().aw_ldmm_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self._free()
        except Exception:
            pass


def shoot_register(I0: torch.Tensor, I1: torch.Tensor, n_time_steps: int, n_iters: int,
                   spacing=(1.0, 1.0, 1.0), sigma=0.1, step=0.005, alpha=0.01, beta=0.01,
                   gamma=0.001):
    """Geodesic shooting registration at one scale from alpha0 = 0 (the loop
    LDMMWarp runs for the shooting iterator). Returns (data, energies)."""
    from .greedy import DiffOperParam
    it = LDMMShootingIteratorB200(I0.shape[::-1], spacing=spacing, n_time_steps=n_time_steps)
    it.SetScaleLevel(I0.shape[::-1], spacing,
                     LDMMIteratorParam(DiffOperParam(alpha, beta, gamma), sigma, step, False))
    data = LDMMShootingDefDataB200(I0, I1, spacing)
    for _ in range(n_iters):
        it.Iterate(data)
    return data, it.Energies()
