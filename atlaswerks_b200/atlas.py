"""Host-side mirror of the reference's greedy atlas builder.

``GreedyAtlasBuilderB200`` follows GreedyAtlasBuilder
(Algorithms/Greedy/GreedyAtlasBuilder.h, .txx:20-301) and the per-GPU loop of
AtlasThread::AtlasThreadMain (Algorithms/Common/AtlasThread.txx:97-181):

* the mean template starts as the weighted sum of the subjects and is the
  I1 of every subject's greedy iteration;
* every iteration runs one greedy step of every subject
  (GreedyAtlasThreadGPU: one GreedyIteratorGPU, the step recomputed at
  iteration 0), then the mean is recomputed
  (GreedyAtlasThreadGPU::ComputeThreadMean) — after every iteration as in
  the reference, or after every ``MeanPeriod``-th one;
* with several processes (one per GPU), rank r owns subjects
  {i : i mod world == r}; each rank sums its subjects' weighted deformed
  images and one all-reduce (sum) over the process group forms the mean,
  the exchange of GreedyAtlasBuilder::SumAcrossNodes (.txx:181-203,
  MPI_Allreduce there).

Subjects may have grids of their own (the template grid is ``size``); their
images are sampled through the voxel-centre map of equal physical extent.
The per-rank work runs in libaw_b200.so (``aw_atlas_*``) through
``CudaAtlasEngine``; the builder only sequences it and the collective.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import check
from .device import _check_image, _stream
from .greedy import DiffOperParam


@dataclass
class GreedyAtlasParam:
    """GreedyAtlasParam (Algorithms/Greedy/GreedyAtlasParam.h) at one scale
    level: kernel, MaxPert, NIterations, plus the mean-update period."""
    Kernel: DiffOperParam = field(default_factory=DiffOperParam)
    MaxPert: float = 0.1
    NIterations: int = 50
    MeanPeriod: int = 1


class _DeviceBuffer:
    """A raw float32 device buffer viewed as a torch tensor (no copy)."""

    def __init__(self, ptr: int, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f4",
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None}


class CudaAtlasEngine:
    """The subjects of one rank on its GPU (``aw_atlas_*``)."""

    def __init__(self, size: Sequence[int], spacing: Sequence[float], param: GreedyAtlasParam,
                 images: Sequence[torch.Tensor], weights: Sequence[float]):
        k = param.Kernel
        if k.LPow != 1.0 or k.UseEigenLUT or k.DivergenceFree:
            raise ValueError("LPow != 1, UseEigenLUT and DivergenceFree are not supported on the "
                             "GPU path (DiffOperGPU)")
        nx, ny, nz = size
        self.shape = (nz, ny, nx)
        self._images = list(images)  # kept alive: the handle reads them every iteration
        self._h = ctypes.c_void_p()
        check(_lib.lib().aw_atlas_create(nx, ny, nz, *map(float, spacing), k.Alpha, k.Beta,
                                         k.Gamma, param.MaxPert, len(images),
                                         ctypes.byref(self._h)))
        for i, (img, w) in enumerate(zip(images, weights)):
            _check_image(img, f"image {i}")
            snz, sny, snx = img.shape
            check(_lib.lib().aw_atlas_set_subject(self._h, i, img.data_ptr(), snx, sny, snz,
                                                  float(w)))
        p = ctypes.c_void_p()
        check(_lib.lib().aw_atlas_mean_buffer(self._h, ctypes.byref(p)))
        self._mean = torch.as_tensor(_DeviceBuffer(p.value, self.shape), device="cuda")

    def compute_mean(self) -> torch.Tensor:
        """This rank's sum of w_i I_i(h_i), in the tensor the iterations read."""
        check(_lib.lib().aw_atlas_compute_mean(self._h, _stream()))
        return self._mean

    def iterate(self, n_iters: int, update_first: bool) -> None:
        check(_lib.lib().aw_atlas_iterate(self._h, int(n_iters), int(update_first), _stream()))

    def field(self, i: int) -> torch.Tensor:
        px, py, pz = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        check(_lib.lib().aw_atlas_field(self._h, i, ctypes.byref(px), ctypes.byref(py),
                                        ctypes.byref(pz)))
        # the three planes are contiguous in the handle: x | y | z
        return torch.as_tensor(_DeviceBuffer(px.value, (3,) + self.shape), device="cuda")

    def step(self, i: int) -> float:
        s = ctypes.c_float()
        check(_lib.lib().aw_atlas_get_step(self._h, i, ctypes.byref(s)))
        return float(s.value)

    def energies(self, i: int) -> np.ndarray:
        n = ctypes.c_int()
        check(_lib.lib().aw_atlas_get_energies(self._h, i, None, 0, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1), np.float64)
        check(_lib.lib().aw_atlas_get_energies(self._h, i, out.ctypes.data, n.value,
                                               ctypes.byref(n)))
        return out[: n.value]

    def close(self) -> None:
        if self._h:
            torch.cuda.synchronize()
            _lib.lib().aw_atlas_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def local_subjects(n_total: int, rank: int, world: int) -> List[int]:
    """Subjects owned by `rank`: i mod world == rank."""
    return [i for i in range(n_total) if i % world == rank]


class GreedyAtlasBuilderB200:
    """GreedyAtlasBuilder over the subjects of this rank.

    images / weights are the GLOBAL lists (every rank passes the same
    weights; only the local images need to be real tensors, the others may
    be None). weights default to 1/N. ``group`` is a torch.distributed
    process group (None: one process). ``engine_factory(size, spacing,
    param, images, weights)`` builds the per-rank engine (default
    CudaAtlasEngine).
    """

    def __init__(self, images: Sequence[Optional[torch.Tensor]], size: Sequence[int],
                 param: GreedyAtlasParam, spacing=(1.0, 1.0, 1.0),
                 weights: Optional[Sequence[float]] = None, group=None, engine_factory=None):
        self.n_total = len(images)
        if self.n_total < 1:
            raise ValueError("an atlas needs at least one image")
        if weights is None:
            weights = [1.0 / self.n_total] * self.n_total
        if len(weights) != self.n_total:
            raise ValueError("one weight per image")
        self.param = param
        self.group = group
        if group is not None:
            import torch.distributed as dist
            self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        else:
            self.rank, self.world = 0, 1
        self.local = local_subjects(self.n_total, self.rank, self.world)
        if not self.local:
            raise ValueError(f"rank {self.rank} owns no subject: use at most {self.n_total} ranks")
        factory = engine_factory or CudaAtlasEngine
        self.engine = factory(tuple(size), tuple(float(s) for s in spacing), param,
                              [images[i] for i in self.local], [weights[i] for i in self.local])
        self.mean = None

    def _update_mean(self):
        m = self.engine.compute_mean()
        if self.group is not None and self.world > 1:
            import torch.distributed as dist
            dist.all_reduce(m, op=dist.ReduceOp.SUM, group=self.group)
        self.mean = m

    def BuildAtlas(self):
        """The AtlasThreadMain loop at one scale level."""
        p = self.param
        self._update_mean()
        done = 0
        while done < p.NIterations:
            # iterations until the next mean update
            k = min(p.MeanPeriod - (done % p.MeanPeriod), p.NIterations - done)
            self.engine.iterate(k, update_first=(done == 0))
            done += k
            if done % p.MeanPeriod == 0:
                self._update_mean()
        return self.mean

    def GetMeanImage(self) -> torch.Tensor:
        return self.mean

    def GetDeformationField(self, i: int) -> torch.Tensor:
        """h of global subject i (it must be local to this rank)."""
        return self.engine.field(self.local.index(i))

    def GetStepSize(self, i: int) -> float:
        return self.engine.step(self.local.index(i))

    def GetEnergies(self, i: int) -> np.ndarray:
        return self.engine.energies(self.local.index(i))
