"""Host-side mirror of the reference's LDMM relaxation interfaces.

* ``LDMMIteratorB200`` — LDMMIteratorGPU / LDMMIteratorCPU
  (Algorithms/LDMM/LDMMIteratorCPU.h:30-70): ``SetScaleLevel``, ``Iterate``,
  ``UpdateStepSizeNextIteration``; the splatting gradient (IterateNew,
  LDMM/LDMMIteratorCPU.cxx:529-631).
* ``LDMMDeformationDataB200`` — LDMMDeformationData (LDMM/LDMMDeformationData.h):
  images, the T velocity fields ``v(t)`` and ``StepSize``.

Computation runs in libaw_b200.so through the C ABI.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np
import torch

from . import _lib
from ._lib import check
from .device import _check_image, _stream
from .greedy import DiffOperParam


@dataclass
class LDMMIteratorParam:
    """LDMMIteratorParam (Algorithms/LDMM/LDMMIteratorParam.h:28-54) defaults."""
    Kernel: DiffOperParam = field(default_factory=DiffOperParam)
    Sigma: float = 5.0
    StepSize: float = 0.005
    UseAdaptiveStepSize: bool = True
    MaxPert: float = 0.1


class LDMMDeformationDataB200:
    def __init__(self, I0: torch.Tensor, I1: torch.Tensor, n_time_steps: int,
                 spacing=(1.0, 1.0, 1.0)):
        _check_image(I0, "I0")
        _check_image(I1, "I1")
        if I0.shape != I1.shape:
            raise ValueError("I0 and I1 must have the same grid")
        self.I0, self.I1 = I0, I1
        self.T = int(n_time_steps)
        self.spacing = tuple(float(s) for s in spacing)
        self.V = torch.zeros((self.T, 3) + tuple(I0.shape), device=I0.device,
                             dtype=torch.float32)

    def v(self, t: int) -> torch.Tensor:
        return self.V[t]


def ldmm_total_energy(image_energy: float, step_energies: Sequence[float], sigma: float,
                      T: int) -> np.float32:
    """LDMMEnergy::GetEnergy from an image energy sp^3 sum (I0(h) - I1)^2
    and the step energies <L v_t, v_t> sp^3 in the order the iteration set
    them: (1.0 / (sigma*sigma)) times the image term (LDMMEnergy.h:42) plus
    the float sum of the step energies / T (LDMMEnergy.cxx:55-64)."""
    f32 = np.float32
    img = f32(float(1.0 / float(f32(sigma) * f32(sigma))) * float(f32(image_energy)))
    val = f32(0.0)
    for e in step_energies:
        val = f32(val + f32(e))
    return f32(img + f32(val / f32(T)))


class LDMMIteratorB200:
    DeformationDataType = LDMMDeformationDataB200
    ParamType = LDMMIteratorParam

    def __init__(self, size: Sequence[int], origin=(0.0, 0.0, 0.0), spacing=(1.0, 1.0, 1.0),
                 n_time_steps: int = 5, debug: bool = True):
        self.size = tuple(size)
        self.spacing = tuple(float(s) for s in spacing)
        self.T = int(n_time_steps)
        self._h = ctypes.c_void_p()
        self._update_step = False
        self._orig = False
        self._vec = False
        self._alphas = None
        self._alphas_valid = False

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
        self.SetStepSize(param.StepSize)
        if self._orig:
            check(_lib.lib().aw_ldmm_use_orig_gradient_calc(self._h, 1))
        if self._vec:
            check(_lib.lib().aw_ldmm_set_vector_energy(self._h, 1))

    def SetUseOrigGradientCalc(self, on: bool):
        """LDMMIteratorCPU's mUseOrigGradientCalc: IterateOrig (Jacobian
        transport) instead of IterateNew (splatting)."""
        self._orig = bool(on)
        if self._h:
            check(_lib.lib().aw_ldmm_use_orig_gradient_calc(self._h, int(self._orig)))

    def SetVectorEnergy(self, on: bool):
        """The debug mode's vector energy (LDMMIteratorCPU.cxx:493-505,
        601-610): every iteration that updates v also records
        sum_t <L v_t, v_t> sp^3 (VecEnergies), at the cost of one more
        transform and L per time step."""
        self._vec = bool(on)
        if self._h:
            check(_lib.lib().aw_ldmm_set_vector_energy(self._h, int(self._vec)))

    def UpdateStepSizeNextIteration(self):
        self._update_step = True

    def SetStepSize(self, step: float):
        check(_lib.lib().aw_ldmm_set_step(self._h, float(step)))

    def StepSize(self) -> float:
        s = ctypes.c_float()
        check(_lib.lib().aw_ldmm_get_step(self._h, ctypes.byref(s)))
        return float(s.value)

    def Iterate(self, data: LDMMDeformationDataB200, computeAlphasOnly: bool = False):
        """One iteration; with computeAlphasOnly the velocities stay as they
        are and GetAlpha(t) returns the splatted residual at t over sigma^2
        (LDMMIteratorGPU::Iterate(defData, computeAlphasOnly))."""
        if data.T != self.T:
            raise ValueError("data has a different number of time steps")
        if computeAlphasOnly:
            if self._alphas is None or self._alphas.shape[1:] != data.I0.shape:
                self._alphas = torch.empty((self.T,) + tuple(data.I0.shape),
                                           device=data.I0.device)
            check(_lib.lib().aw_ldmm_alphas(self._h, data.I0.data_ptr(), data.I1.data_ptr(),
                                            data.V.data_ptr(), self._alphas.data_ptr(),
                                            _stream()))
            self._alphas_valid = True
            return
        check(_lib.lib().aw_ldmm_iterate(self._h, data.I0.data_ptr(), data.I1.data_ptr(),
                                         data.V.data_ptr(), int(self._update_step), _stream()))
        self._update_step = False
        self._alphas_valid = False

    def GetAlpha(self, t: int) -> torch.Tensor:
        """alpha_t of the last Iterate(data, computeAlphasOnly=True); valid
        until the next Iterate without it."""
        if not self._alphas_valid:
            raise RuntimeError("call Iterate(data, computeAlphasOnly=True) first")
        return self._alphas[t]

    def Run(self, data: LDMMDeformationDataB200, n_iters: int, adaptive_first: bool = False):
        check(_lib.lib().aw_ldmm_run(self._h, data.I0.data_ptr(), data.I1.data_ptr(),
                                     data.V.data_ptr(), int(n_iters), int(adaptive_first),
                                     _stream()))

    def Energies(self) -> np.ndarray:
        n = ctypes.c_int()
        check(_lib.lib().aw_ldmm_get_energies(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1), np.float64)
        check(_lib.lib().aw_ldmm_get_energies(self._h, out.ctypes.data, n.value,
                                              ctypes.byref(n)))
        return out[: n.value]

    def VecEnergies(self) -> np.ndarray:
        """sum_t <L v_t, v_t> sp^3 per iteration, aligned with Energies()
        (zero for iterations run without SetVectorEnergy)."""
        n = ctypes.c_int()
        check(_lib.lib().aw_ldmm_get_vec_energies(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1), np.float64)
        check(_lib.lib().aw_ldmm_get_vec_energies(self._h, out.ctypes.data, n.value,
                                                  ctypes.byref(n)))
        return out[: n.value]

    def VecStepEnergies(self) -> np.ndarray:
        """<L v_t, v_t> sp^3 for t = 0 .. T-1 of the last iteration that
        recorded vector energies."""
        out = np.zeros(self.T, np.float64)
        check(_lib.lib().aw_ldmm_get_vec_step_energies(self._h, out.ctypes.data, self.T))
        return out

    def TotalEnergy(self) -> float:
        """LDMMEnergy::GetEnergy of the last iteration, ImageEnergy() +
        VecEnergy(), in the reference's float arithmetic and the order its
        iteration sets the step energies (t = T-1 .. 0 for IterateNew, 0 ..
        T-1 for IterateOrig); 0 before any iteration."""
        e = self.Energies()
        if e.size == 0:
            return 0.0
        steps = self.VecStepEnergies() if self._vec else np.zeros(self.T)
        order = steps if self._orig else steps[::-1]
        return float(ldmm_total_energy(e[-1], order, self.param.Sigma, self.T))

    def _free(self):
        if self._h:
            _lib.lib().aw_ldmm_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self._free()
        except Exception:
            pass


def ldmm_register(I0: torch.Tensor, I1: torch.Tensor, n_time_steps: int, n_iters: int,
                  spacing=(1.0, 1.0, 1.0), sigma=0.1, step=0.005, adaptive=False, max_pert=0.1,
                  alpha=0.01, beta=0.01, gamma=0.001, orig_gradient=False):
    """LDMMWarp at one scale level (LDMM/LDMMWarp.txx:71-130); orig_gradient
    selects IterateOrig (the reference's default) over IterateNew."""
    nz, ny, nx = I0.shape
    it = LDMMIteratorB200((nx, ny, nz), spacing=spacing, n_time_steps=n_time_steps)
    it.SetUseOrigGradientCalc(orig_gradient)
    p = LDMMIteratorParam(DiffOperParam(alpha, beta, gamma), sigma, step, adaptive, max_pert)
    it.SetScaleLevel((nx, ny, nz), spacing, p)
    data = LDMMDeformationDataB200(I0, I1, n_time_steps, spacing)
    it.Run(data, n_iters, adaptive_first=adaptive)
    return data.V, it.Energies(), it.StepSize()
