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

* ``LDMMVelShootingIteratorB200`` / ``LDMMVelShootingDefDataB200`` —
  LDMMVelShootingIteratorCPU and its data (LDMM/LDMMVelShootingIteratorCPU.cxx:
  186-344): the geodesic in velocity form from v0, the Jacobian of phiT0
  carried along, the update of v0.
* ``LDMMGeodesicShootingB200`` — LDMMGeodesicShootingCPU / GPU
  (LDMM/LDMMGeodesicShooting.h): ``ShootImage(I0, alpha0, T)``, the geodesic
  alone, with ``GetFinalImage``, ``GetPhi0To1`` and ``GetPhi1To0``.
* ``LDMMAdShootingIteratorB200`` — LDMMAdShootingIteratorCPU / GPU
  (LDMM/LDMMAdShootingIteratorCPU.cxx:237-453): shoots the geodesic keeping
  every time point, integrates the adjoint equations backward and takes the
  gradient step on alpha0; ``finalUpdatePhi0T`` / ``finalUpdatePhiT0``.
* ``LDMMAdShootingWarpB200`` — LDMMWarpAd<LDMMAdShootingIterator*>: the
  RunWarp scale loop (LDMM/LDMMWarp.txx:72-133) with LDMMShootingDefData's
  scale change (alpha0 resampled, images Gaussian-downsampled:
  LDMMShootingDefData.cxx:133-176) and FinishWarp's final maps
  (LDMMWarpAd.txx:37-42).

The iterations run in libaw_b200.so (``aw_ldmm_shoot_iterate`` /
``aw_ldmm_adshoot_iterate`` on an LDMM handle, which holds T, sigma, the
step size and the fluid kernel). The energy history holds the image term
sp^3 sum (I0(phiT0) - I1)^2 (``Energies``) and the vector term
(``VecEnergies``): sum_t <L v_t, v_t> for the momentum shooting, <L v0, v0>
for the adjoint shooting — the step energies LDMMEnergy holds.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import check
from . import device as D
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

    def VecEnergies(self) -> np.ndarray:
        """The vector term per iteration: the sum over t of LDMMEnergy's step
        energies <L v_t, v_t> (only v0's for the adjoint iterator)."""
        n = ctypes.c_int()
        check(_lib.lib().aw_ldmm_get_vec_energies(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1), np.float64)
        check(_lib.lib().aw_ldmm_get_vec_energies(self._h, out.ctypes.data, n.value,
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


class LDMMAdShootingIteratorB200(LDMMShootingIteratorB200):
    """LDMMAdShootingIteratorCPU / GPU (LDMM/LDMMAdShootingIteratorCPU.h):
    the same handle and scale-level set-up as the momentum-shooting
    iterator, the adjoint Iterate."""

    def Iterate(self, data: LDMMShootingDefDataB200):
        check(_lib.lib().aw_ldmm_adshoot_iterate(self._h, data.I0.data_ptr(), data.I1.data_ptr(),
                                                 data.Alpha0.data_ptr(), data.Phi0T.data_ptr(),
                                                 data.PhiT0.data_ptr(), _stream()))

    def _final(self, data: LDMMShootingDefDataB200, which: int):
        other = torch.empty_like(data.Phi0T)
        p0, p1 = (data.Phi0T, other) if which == 0 else (other, data.PhiT0)
        check(_lib.lib().aw_ldmm_adshoot_final_maps(self._h, p0.data_ptr(), p1.data_ptr(),
                                                    _stream()))

    def finalUpdatePhi0T(self, data: LDMMShootingDefDataB200):
        """Phi0T composed from the identity through the last iteration's v_t."""
        self._final(data, 0)

    def finalUpdatePhiT0(self, data: LDMMShootingDefDataB200):
        """PhiT0 composed from the identity through the last iteration's v_t."""
        self._final(data, 1)



class LDMMVelShootingDefDataB200:
    """LDMMVelShootingDefData (Algorithms/LDMM/LDMMVelShootingDefData.h): I0,
    I1, the initial velocity ``V0`` [3, nz, ny, nx] (zero at the start) and
    the maps ``Phi0T`` / ``PhiT0`` of the last shooting."""

    def __init__(self, I0: torch.Tensor, I1: torch.Tensor, spacing=(1.0, 1.0, 1.0)):
        _check_image(I0, "I0")
        _check_image(I1, "I1")
        if I0.shape != I1.shape:
            raise ValueError("I0 and I1 must have the same grid")
        self.I0, self.I1 = I0, I1
        self.spacing = tuple(float(s) for s in spacing)
        shape = tuple(I0.shape)
        self.V0 = torch.zeros((3,) + shape, device=I0.device, dtype=torch.float32)
        self.Phi0T = identity(shape, I0.device)
        self.PhiT0 = identity(shape, I0.device)

    def GetDef0To1(self) -> torch.Tensor:
        return self.Phi0T

    def GetDef1To0(self) -> torch.Tensor:
        return self.PhiT0

    def GetI0At1(self) -> torch.Tensor:
        return apply(self.I0, self.PhiT0)

    def GetI1At0(self) -> torch.Tensor:
        return apply(self.I1, self.Phi0T)


class LDMMVelShootingIteratorB200(LDMMShootingIteratorB200):
    """LDMMVelShootingIteratorCPU (LDMM/LDMMVelShootingIteratorCPU.cxx:
    186-344): the geodesic in velocity form from v0; Iterate updates V0 (or,
    after UpdateStepSizeNextIteration, sets the step from the update's
    size); StepSize()."""
    DeformationDataType = LDMMVelShootingDefDataB200

    def __init__(self, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self._update_step = False

    def UpdateStepSizeNextIteration(self):
        self._update_step = True

    def StepSize(self) -> float:
        st = ctypes.c_float()
        check(_lib.lib().aw_ldmm_get_step(self._h, ctypes.byref(st)))
        return float(st.value)

    def Iterate(self, data: LDMMVelShootingDefDataB200):
        check(_lib.lib().aw_ldmm_velshoot_iterate(self._h, data.I0.data_ptr(),
                                                  data.I1.data_ptr(), data.V0.data_ptr(),
                                                  data.Phi0T.data_ptr(), data.PhiT0.data_ptr(),
                                                  int(self._update_step), _stream()))
        self._update_step = False


class LDMMGeodesicShootingB200:
    """LDMMGeodesicShootingGPU / CPU (LDMM/LDMMGeodesicShooting.h,
    LDMMGeodesicShootingCPU.cxx:37-157): ShootImage(I0, alpha0, nTimeSteps)
    follows the geodesic from I0 along the momentum alpha0 and keeps the
    final image and both maps (GetFinalImage, GetPhi0To1, GetPhi1To0).
    ``size`` is (nx, ny, nz); ``kernel`` a DiffOperParam."""

    def __init__(self, size: Sequence[int], spacing: Sequence[float], kernel):
        if kernel.LPow != 1.0 or kernel.UseEigenLUT or kernel.DivergenceFree:
            raise ValueError("LPow != 1, UseEigenLUT and DivergenceFree are not supported on the "
                             "GPU path (DiffOperGPU)")
        self.size = tuple(int(x) for x in size)
        self.spacing = tuple(float(x) for x in spacing)
        self.kernel = kernel
        self._h = ctypes.c_void_p()
        self._T = 0
        nx, ny, nz = self.size
        self._img = torch.empty((nz, ny, nx), device="cuda")
        self._p0 = identity((nz, ny, nx), self._img.device)
        self._p1 = identity((nz, ny, nx), self._img.device)

    def ShootImage(self, I0: torch.Tensor, alpha0: torch.Tensor, nTimeSteps: int) -> None:
        _check_image(I0, "I0")
        _check_image(alpha0, "alpha0")
        if tuple(I0.shape) != tuple(self._img.shape) or alpha0.shape != I0.shape:
            raise ValueError("I0 and alpha0 must be on the shooter's grid")
        if nTimeSteps < 1:
            raise ValueError("nTimeSteps must be positive")
        L = _lib.lib()
        if self._T != int(nTimeSteps):
            self._free()
            nx, ny, nz = self.size
            k = self.kernel
            check(L.aw_ldmm_create(nx, ny, nz, *self.spacing, k.Alpha, k.Beta, k.Gamma,
                                   int(nTimeSteps), 1.0, 0.1, ctypes.byref(self._h)))
            self._T = int(nTimeSteps)
        check(L.aw_ldmm_geodesic_shoot(self._h, I0.data_ptr(), alpha0.data_ptr(),
                                       self._p0.data_ptr(), self._p1.data_ptr(),
                                       self._img.data_ptr(), _stream()))

    def GetFinalImage(self) -> torch.Tensor:
        return self._img

    def GetPhi0To1(self) -> torch.Tensor:
        return self._p0

    def GetPhi1To0(self) -> torch.Tensor:
        return self._p1

    def _free(self):
        if self._h:
            _lib.lib().aw_ldmm_destroy(self._h)
            self._h = ctypes.c_void_p()
            self._T = 0

    def __del__(self):
        try:
            self._free()
        except Exception:
            pass


@dataclass
class LDMMShootingScaleLevel:
    """One LDMMScaleLevel of an adjoint-shooting warp: downsample factor,
    iterations, fixed step size (UseAdaptiveStepSize is false for shooting)."""
    DownsampleFactor: int
    NIterations: int
    StepSize: float


class LDMMAdShootingWarpB200:
    """LDMMWarpAd<LDMMAdShootingIteratorB200>::RunWarp over the scale levels,
    coarsest first: at the first level alpha0 = 0; at each later one alpha0
    is resampled onto the finer grid (MultiscaleManager::UpsampleToLevel, the
    images' resampleNew) and the images are Gaussian-downsampled from the
    originals except at factor 1. FinishWarp leaves the final maps."""

    def __init__(self, I0: torch.Tensor, I1: torch.Tensor,
                 levels: Sequence[LDMMShootingScaleLevel], n_time_steps: int = 5,
                 spacing=(1.0, 1.0, 1.0), sigma: float = 1.0, kernel=None):
        from .greedy import DiffOperParam
        _check_image(I0, "I0")
        _check_image(I1, "I1")
        self.I0, self.I1 = I0, I1
        self.T = int(n_time_steps)
        self.spacing = tuple(float(s) for s in spacing)
        self.levels = sorted(levels, key=lambda l: -l.DownsampleFactor)
        if len({l.DownsampleFactor for l in self.levels}) != len(self.levels):
            raise ValueError("cannot add multiple scale levels with the same downsample factor")
        self.sigma = float(sigma)
        self.kernel = kernel or DiffOperParam()
        self.energies: List[np.ndarray] = []
        self.vec_energies: List[np.ndarray] = []
        self.data = None

    def RunWarp(self) -> LDMMShootingDefDataB200:
        from .multiscale import level_geometry
        shape = tuple(self.I0.shape)
        alpha0, prev_sp = None, None
        for li, lev in enumerate(self.levels):
            size, sp = level_geometry(shape, self.spacing, lev.DownsampleFactor)
            if size == shape:
                I0, I1 = self.I0, self.I1
            else:
                I0 = D.downsample(self.I0, size, self.spacing)
                I1 = D.downsample(self.I1, size, self.spacing)
            data = LDMMShootingDefDataB200(I0, I1, sp)
            if li > 0:
                data.Alpha0.copy_(D.resample_image(alpha0, size, prev_sp, sp))
            it = LDMMAdShootingIteratorB200((size[2], size[1], size[0]), spacing=sp,
                                            n_time_steps=self.T)
            it.SetScaleLevel((size[2], size[1], size[0]), sp,
                             LDMMIteratorParam(self.kernel, self.sigma, lev.StepSize, False))
            for _ in range(lev.NIterations):
                it.Iterate(data)
            self.energies.append(it.Energies())
            self.vec_energies.append(it.VecEnergies())
            alpha0, prev_sp = data.Alpha0, sp
        it.finalUpdatePhi0T(data)
        it.finalUpdatePhiT0(data)
        self.data = data
        return data

    def GetDefImage(self) -> torch.Tensor:
        """I0 carried to time 1 (LDMMWarp::GetDefImage -> GetI0At1)."""
        return self.data.GetI0At1()

    def GetInvDefImage(self) -> torch.Tensor:
        return self.data.GetI1At0()

    def GetAlpha0(self) -> torch.Tensor:
        return self.data.Alpha0
