"""Multiscale greedy registration: the host loop of GreedyWarp::RunWarp
(Algorithms/Greedy/GreedyWarp.txx:71-125) with MultiscaleManager's scale
levels (Algorithms/Common/MultiscaleManager.cxx:105-127) and
GreedyDeformationData::SetScaleLevel (Greedy/GreedyDeformationData.cxx:
188-247), every scale change done on the device.

Scale levels are given as (downsample factor, iterations, MaxPert); they run
coarsest first. Level size = original size // factor per axis, level
spacing = spacing * factor. At the first level h (and h^-1) start at the
identity; at each later level they are upsampled from the previous level;
images are Gaussian-downsampled from the originals except at factor 1.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np
import torch

from . import device as D
from .greedy import (DiffOperParam, GreedyDeformationDataB200, GreedyIteratorB200,
                     GreedyIteratorParam)


@dataclass
class ScaleLevel:
    DownsampleFactor: int
    NIterations: int
    MaxPert: float = 0.1


def level_geometry(shape, spacing, factor):
    nz, ny, nx = shape
    size = (nz // factor, ny // factor, nx // factor)
    sp = tuple(float(np.float32(s) * np.float32(factor)) for s in spacing)
    return size, sp


class GreedyWarpB200:
    """GreedyWarp<GreedyIteratorB200>: RunWarp over the scale levels."""

    def __init__(self, I0: torch.Tensor, I1: torch.Tensor, levels: Sequence[ScaleLevel],
                 spacing=(1.0, 1.0, 1.0), kernel: DiffOperParam = None,
                 compute_inverse: bool = False, fast_interpolation: bool = False):
        self.I0, self.I1 = I0, I1
        self.spacing = tuple(float(s) for s in spacing)
        self.levels = sorted(levels, key=lambda l: -l.DownsampleFactor)
        if len({l.DownsampleFactor for l in self.levels}) != len(self.levels):
            raise ValueError("cannot add multiple scale levels with the same downsample factor")
        self.kernel = kernel or DiffOperParam()
        self.compute_inverse = compute_inverse
        self.fast_interpolation = fast_interpolation
        self.energies: List[np.ndarray] = []
        self.steps: List[float] = []

    def prepare(self):
        """Builds every level's iterator (FFT plans, tuned launch shapes,
        device state) ahead of RunWarp, which reuses them; the reference
        builds its iterator once too (GreedyWarp.txx:40-69)."""
        if getattr(self, "_its", None) is None:
            shape = tuple(self.I0.shape)
            self._its = []
            for lev in self.levels:
                size, sp = level_geometry(shape, self.spacing, lev.DownsampleFactor)
                it = GreedyIteratorB200((size[2], size[1], size[0]), spacing=sp)
                it.SetScaleLevel((size[2], size[1], size[0]), sp,
                                 GreedyIteratorParam(self.kernel, lev.MaxPert))
                if self.fast_interpolation:
                    it.SetFastInterpolation(True)
                self._its.append(it)
        return self

    def RunWarp(self) -> Tuple[torch.Tensor, torch.Tensor]:
        shape = tuple(self.I0.shape)
        h = hinv = None
        self.prepare()
        self.energies, self.steps = [], []
        for li, lev in enumerate(self.levels):
            size, sp = level_geometry(shape, self.spacing, lev.DownsampleFactor)
            if size == shape:
                I0, I1 = self.I0, self.I1
            else:
                I0 = D.downsample(self.I0, size, self.spacing)
                I1 = D.downsample(self.I1, size, self.spacing)
            data = GreedyDeformationDataB200(I0, I1, sp, self.compute_inverse)
            if li > 0:
                data.Def1To0().copy_(D.upsample_hfield(h, size, True))
                if self.compute_inverse:
                    data.Def0To1().copy_(D.upsample_hfield(hinv, size, True))
            it = self._its[li]
            it.Run(data, lev.NIterations, update_first=True)
            h = data.Def1To0()
            hinv = data.Def0To1() if self.compute_inverse else None
            self.energies.append(it.Energies())
            self.steps.append(it.StepSize())
        return h, hinv

    def GenerateOutput(self, prefix: str, h: torch.Tensor, hinv: torch.Tensor = None,
                       suffix: str = "mha", origin=(0.0, 0.0, 0.0)):
        """The files GreedyWarp writes at the end of a run (GreedyWarp.txx:
        150-230): <prefix>DefImage (I0 deformed to I1's frame, I0(h)),
        <prefix>DefField1To0 (h) and, with the inverse, <prefix>InvDefImage
        (I1(h^-1)) and <prefix>DefField0To1 (h^-1), as MetaImage. h holds
        voxel coordinates, as the reference's deformation fields do."""
        from .metaimage import write_mha
        written = []

        def out(name, arr):
            path = f"{prefix}{name}.{suffix}"
            write_mha(path, arr.detach().cpu().numpy(), self.spacing, origin)
            written.append(path)

        out("DefImage", D.apply(self.I0, h))
        out("DefField1To0", h)
        if hinv is not None:
            out("InvDefImage", D.apply(self.I1, hinv))
            out("DefField0To1", hinv)
        return written

