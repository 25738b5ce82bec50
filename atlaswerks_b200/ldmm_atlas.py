"""Host-side mirror of the reference's LDMM relaxation atlas builder.

``LDMMAtlasBuilderB200`` follows LDMMAtlasBuilder (Algorithms/LDMM/
LDMMAtlasBuilder.h, .txx:20-335) and the per-thread hooks of
LDMMAtlasThreadCPU / LDMMAtlasThreadGPU inside AtlasThread::AtlasThreadMain
(Algorithms/Common/AtlasThread.txx:97-181):

* every subject i is an LDMM registration whose I0 is the shared mean
  template (not rescaled: LDMMAtlasDefDataCPU, LDMMAtlasThreadCPU.cxx:41-53)
  and whose I1 is the subject's image, with T velocity fields of its own;
* the mean starts from v = 0 (the weighted mean of the subjects) and, after
  every iteration of all subjects (BeginImageIteration's step-size pass
  first at iteration 0 with UseAdaptiveStepSize), becomes
  sum_i w_i I1_i(h_i,0->1) |D h_i| / sum_i w_i |D h_i| (JacobianScale, the
  default) or sum_i w_i I1_i(h_i,0->1): GetI1At0 and ComputeJacDet per
  subject (LDMMAtlasThreadCPU::ComputeThreadMean, .cxx:207-264), the sums of
  all threads and nodes, then the division (LDMMAtlasBuilder::ComputeMean,
  .txx:274-335);
* with several processes (one per GPU), rank r owns subjects
  {i : i mod world == r}; each rank forms its two partial sums and two
  all-reduces (sum) over the process group complete them, the exchange of
  LDMMAtlasBuilder::SumAcrossNodes (.txx:236-269, MPI_Allreduce there).

With UsePerVoxelMedian the mean is instead the per-voxel median of the
subjects' deformed images I1_i(h_i,0->1) (MedianCalculator::Select,
LDMMAtlasBuilder::ComputeMedian, .txx:218-233, 336-338), by the reference's
bisection in libaw_b200.so (``aw_ldmm_atlas_voxel_median``); with several
ranks every deformed image is broadcast by its owner first, so each rank
selects over all of them (the selection does not depend on their order).

ComputeMedian (the geometric-median iteration: each subject's weight
divided by its distance) and TrimmedMeanSize k (only the k subjects
nearest the mean, weights renormalised) re-weight the subjects by their
distance sqrt(LDMMEnergy::GetEnergy()) of the last iteration, image plus
velocity terms (LDMMAtlasThreadCPU::FinishImageIteration / ComputeThreadMean,
.cxx:175-181, 225-237; LDMMAtlasBuilder::ComputeWeights, .txx:437-500);
the subjects' iterators then record the vector energies too
(aw_ldmm_set_vector_energy). With several ranks the distances are summed
into one vector of all subjects before the selection.

With Shooting the subjects run the momentum shooting iterator instead
(LDMMShootingAtlasThreadCPU, .cxx:40-226: I0 the mean, I1 the subject,
the state alpha0) and the mean's sums take I1(phi0T) with the Jacobian
splat(ones, phiT0); the sharding and exchange are the same.

Not built: the PCA step; multiscale (one scale level per BuildAtlas call).

The per-rank work runs in libaw_b200.so (``aw_ldmm_*``) through
``CudaLDMMAtlasEngine``; the builder only sequences it and the collectives.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import check
from .atlas import local_subjects
from .device import _check_image, _stream
from .ldmm import LDMMDeformationDataB200, LDMMIteratorB200, LDMMIteratorParam


@dataclass
class LDMMAtlasParam:
    """LDMMAtlasParam (Algorithms/LDMM/LDMMAtlasParam.h:26-147) at one scale
    level: the iterator, NTimeSteps, NIterations, JacobianScale, and the
    gradient variant (IterateOrig with UseOrigGradientCalc)."""
    Iterator: LDMMIteratorParam = field(default_factory=LDMMIteratorParam)
    NTimeSteps: int = 5
    NIterations: int = 50
    JacobianScale: bool = True
    UseOrigGradientCalc: bool = False
    UsePerVoxelMedian: bool = False
    ComputeMedian: bool = False
    TrimmedMeanSize: int = 0
    Shooting: bool = False  # the shooting atlas (LDMMShootingAtlasThreadCPU)


def atlas_weights(weights: Sequence[float], dists: Sequence[float], compute_median: bool,
                  trimmed: int) -> List[np.float32]:
    """The per-subject weights of the mean (float, as the reference holds
    them): ComputeMedian divides each weight by the subject's distance (1
    before any energy exists; LDMMAtlasThreadCPU.cxx:225-232); TrimmedMeanSize
    k > 0 replaces them by the weights of the subjects whose distance is at
    most the k-th smallest (0-based, MedianCalculator::Select), at most k of
    them in subject order and all of them before any energy exists,
    renormalised to sum 1 (LDMMAtlasBuilder::ComputeWeights, .txx:437-500)."""
    f32 = np.float32
    out = [f32(w) for w in weights]
    if compute_median:
        for i, d in enumerate(dists):
            d = f32(d)
            if d == 0:
                d = f32(1.0)
            out[i] = f32(out[i] * f32(1.0 / float(d)))
    if trimmed > 0:
        dd = [f32(d) for d in dists]
        kval = sorted(dd)[trimmed]
        tm, wsum, sel = [f32(0.0)] * len(dd), f32(0.0), 0
        for i, d in enumerate(dd):
            if d == 0 or (d <= kval and sel < trimmed):
                tm[i] = f32(weights[i])
                wsum = f32(wsum + tm[i])
                sel += 1
        out = [f32(w / wsum) for w in tm]
    return out


class CudaLDMMAtlasEngine:
    """The subjects of one rank on its GPU: one LDMM handle per subject (the
    reference runs one thread, hence one iterator, per image), the shared
    mean they read as I0, and the two sums of the mean."""

    def __init__(self, size: Sequence[int], spacing: Sequence[float], param: LDMMAtlasParam,
                 images: Sequence[torch.Tensor], weights: Sequence[float]):
        nx, ny, nz = size
        self.shape = (nz, ny, nx)
        self.param = param
        self.w = [float(x) for x in weights]
        self.n = nx * ny * nz
        self.mean = torch.zeros(self.shape, device="cuda")
        self.acc = torch.zeros(self.shape, device="cuda")
        self.jsum = torch.zeros(self.shape, device="cuda")
        self._img = torch.zeros(self.shape, device="cuda")
        self._jd = torch.zeros(self.shape, device="cuda")
        self.images = list(images)
        reweigh = param.ComputeMedian or param.TrimmedMeanSize > 0
        self.its: List[LDMMIteratorB200] = []
        self.data: List[LDMMDeformationDataB200] = []
        for i, img in enumerate(self.images):
            _check_image(img, f"image {i}")
            if tuple(img.shape) != self.shape:
                raise ValueError("LDMM atlas subjects must be on the template grid")
            it = LDMMIteratorB200(size, spacing=spacing, n_time_steps=param.NTimeSteps)
            it.SetUseOrigGradientCalc(param.UseOrigGradientCalc)
            it.SetVectorEnergy(reweigh)
            it.SetScaleLevel(size, spacing, param.Iterator)
            self.its.append(it)
            self.data.append(LDMMDeformationDataB200(self.mean, img, param.NTimeSteps, spacing))

    def mean_sums(self):
        """This rank's (sum w I1At0 JacDet, sum w JacDet), or (sum w I1At0,
        None) without JacobianScale, in subject order."""
        L, s = _lib.lib(), _stream()
        js = self.param.JacobianScale
        self.acc.zero_()
        self.jsum.zero_()
        for it, d, w in zip(self.its, self.data, self.w):
            check(L.aw_ldmm_i1_at_0(it._h, d.I1.data_ptr(), d.V.data_ptr(), self._img.data_ptr(),
                                    self._jd.data_ptr() if js else None, s))
            check(L.aw_ldmm_atlas_accumulate(self.acc.data_ptr(), self.jsum.data_ptr(),
                                             self._img.data_ptr(),
                                             self._jd.data_ptr() if js else None, w, self.n, s))
        return self.acc, (self.jsum if js else None)

    def deformed(self) -> List[torch.Tensor]:
        """This rank's deformed images I1_i(h_i,0->1), in subject order."""
        L, s = _lib.lib(), _stream()
        if not hasattr(self, "_defs"):
            self._defs = [torch.empty(self.shape, device="cuda") for _ in self.its]
        for it, d, out in zip(self.its, self.data, self._defs):
            check(L.aw_ldmm_i1_at_0(it._h, d.I1.data_ptr(), d.V.data_ptr(), out.data_ptr(), None,
                                    s))
        return self._defs

    def set_median(self, images: Sequence[torch.Tensor], k: int) -> torch.Tensor:
        """The mean as the per-voxel k-th smallest of the given deformed
        images (all subjects')."""
        nz, ny, nx = self.shape
        ptrs = (ctypes.c_void_p * len(images))(*[t.data_ptr() for t in images])
        check(_lib.lib().aw_ldmm_atlas_voxel_median(ptrs, len(images), int(k), nx, ny, nz,
                                                    self.mean.data_ptr(), _stream()))
        return self.mean

    def set_mean(self, acc: torch.Tensor, jsum: Optional[torch.Tensor]) -> torch.Tensor:
        """The new mean from the (all-reduced) sums, into the I0 every
        subject's iterations read."""
        if jsum is not None:
            check(_lib.lib().aw_ldmm_atlas_normalize(acc.data_ptr(), jsum.data_ptr(), self.n,
                                                     _stream()))
        self.mean.copy_(acc)
        return self.mean

    def iterate(self, first: bool) -> None:
        adaptive = first and self.param.Iterator.UseAdaptiveStepSize
        for it, d in zip(self.its, self.data):
            it.Run(d, 1, adaptive_first=adaptive)

    def velocities(self, i: int) -> torch.Tensor:
        return self.data[i].V

    def distances(self) -> List[float]:
        """sqrt of each local subject's last total energy (0 before any)."""
        return [float(np.sqrt(np.float32(it.TotalEnergy()))) for it in self.its]

    def set_weights(self, weights: Sequence[float]) -> None:
        self.w = [float(w) for w in weights]

    def device_of_sums(self):
        return self.acc.device

    def step(self, i: int) -> float:
        return self.its[i].StepSize()

    def energies(self, i: int) -> np.ndarray:
        return self.its[i].Energies()


class CudaLDMMShootingAtlasEngine:
    """The shooting atlas's subjects on this rank (LDMMShootingAtlasThreadCPU,
    Algorithms/LDMM/LDMMShootingAtlasThreadCPU.cxx:40-226): one momentum
    shooting iterator per subject whose I0 is the shared mean and I1 the
    subject's image (LDMMShootingAtlasDefDataCPU, .cxx:42-52); the mean's
    sums take each subject's image deformed to the mean, I1(phi0T)
    (LDMMShootingDefData::GetI1At0, LDMMShootingDefData.cxx:78-84), and the
    Jacobian of phi0T as the splat of ones by phiT0
    (LDMMShootingIteratorCPU::ComputeJacDet, LDMMShootingIteratorCPU.cxx:
    108-119)."""

    def __init__(self, size: Sequence[int], spacing: Sequence[float], param: LDMMAtlasParam,
                 images: Sequence[torch.Tensor], weights: Sequence[float]):
        from .device import apply, splat
        from .shooting import LDMMShootingDefDataB200, LDMMShootingIteratorB200
        self._apply, self._splat = apply, splat
        nx, ny, nz = size
        self.shape = (nz, ny, nx)
        self.param = param
        self.w = [float(x) for x in weights]
        self.n = nx * ny * nz
        self.mean = torch.zeros(self.shape, device="cuda")
        self.acc = torch.zeros(self.shape, device="cuda")
        self.jsum = torch.zeros(self.shape, device="cuda")
        self._ones = torch.ones(self.shape, device="cuda")
        self.images = list(images)
        self.its, self.data = [], []
        for i, img in enumerate(self.images):
            _check_image(img, f"image {i}")
            if tuple(img.shape) != self.shape:
                raise ValueError("LDMM atlas subjects must be on the template grid")
            it = LDMMShootingIteratorB200(size, spacing=spacing, n_time_steps=param.NTimeSteps)
            it.SetScaleLevel(size, spacing, param.Iterator)
            self.its.append(it)
            self.data.append(LDMMShootingDefDataB200(self.mean, img, spacing))

    def mean_sums(self):
        L, s = _lib.lib(), _stream()
        js = self.param.JacobianScale
        self.acc.zero_()
        self.jsum.zero_()
        for d, w in zip(self.data, self.w):
            img = self._apply(d.I1, d.Phi0T)
            jd = self._splat(self._ones, d.PhiT0) if js else None
            check(L.aw_ldmm_atlas_accumulate(self.acc.data_ptr(), self.jsum.data_ptr(),
                                             img.data_ptr(), jd.data_ptr() if js else None, w,
                                             self.n, s))
        return self.acc, (self.jsum if js else None)

    def deformed(self) -> List[torch.Tensor]:
        return [self._apply(d.I1, d.Phi0T) for d in self.data]

    set_median = CudaLDMMAtlasEngine.set_median
    set_mean = CudaLDMMAtlasEngine.set_mean
    device_of_sums = CudaLDMMAtlasEngine.device_of_sums

    def iterate(self, first: bool) -> None:
        for it, d in zip(self.its, self.data):
            it.Iterate(d)

    def velocities(self, i: int) -> torch.Tensor:
        """The shooting subject's state: its initial momentum alpha0."""
        return self.data[i].Alpha0

    def step(self, i: int) -> float:
        return float(self.param.Iterator.StepSize)

    def energies(self, i: int) -> np.ndarray:
        return self.its[i].Energies()


class LDMMAtlasBuilderB200:
    """LDMMAtlasBuilder over the subjects of this rank (one scale level).

    images / weights are the GLOBAL lists (only the local images need to be
    real tensors); weights default to 1/N. ``group`` is a torch.distributed
    process group (None: one process). ``engine_factory(size, spacing,
    param, images, weights)`` builds the per-rank engine (default
    CudaLDMMAtlasEngine).
    """

    def __init__(self, images: Sequence[Optional[torch.Tensor]], size: Sequence[int],
                 param: LDMMAtlasParam, spacing=(1.0, 1.0, 1.0),
                 weights: Optional[Sequence[float]] = None, group=None, engine_factory=None):
        self.n_total = len(images)
        if self.n_total < 1:
            raise ValueError("an atlas needs at least one image")
        if weights is None:
            weights = [1.0 / self.n_total] * self.n_total
        if len(weights) != self.n_total:
            raise ValueError("one weight per image")
        self.param = param
        self.weights = [float(w) for w in weights]
        if param.TrimmedMeanSize and not 0 < param.TrimmedMeanSize < self.n_total:
            raise ValueError("TrimmedMeanSize must be smaller than the number of images")
        self.group = group
        if group is not None:
            import torch.distributed as dist
            self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        else:
            self.rank, self.world = 0, 1
        self.local = local_subjects(self.n_total, self.rank, self.world)
        if not self.local:
            raise ValueError(f"rank {self.rank} owns no subject: use at most {self.n_total} ranks")
        if param.Shooting and (param.ComputeMedian or param.TrimmedMeanSize):
            raise ValueError("ComputeMedian / TrimmedMeanSize are not supported with Shooting")
        factory = engine_factory or (CudaLDMMShootingAtlasEngine if param.Shooting
                                     else CudaLDMMAtlasEngine)
        self.engine = factory(tuple(size), tuple(float(s) for s in spacing), param,
                              [images[i] for i in self.local], [weights[i] for i in self.local])
        self.mean = None

    @staticmethod
    def median_index(n: int) -> int:
        """LDMMAtlasBuilder::ComputeMedian's index (LDMMAtlasBuilder.txx:222)."""
        return n // 2 - 1 if n % 2 == 0 else n // 2

    def _update_median(self):
        mine = self.engine.deformed()
        if self.group is None or self.world == 1:
            allimgs = list(mine)
        else:
            import torch.distributed as dist
            allimgs = []
            for i in range(self.n_total):
                owner = i % self.world
                t = (mine[self.local.index(i)] if owner == self.rank
                     else torch.empty_like(mine[0]))
                dist.broadcast(t, src=owner, group=self.group)
                allimgs.append(t)
        self.mean = self.engine.set_median(allimgs, self.median_index(self.n_total))

    def _reweigh(self):
        p = self.param
        mine = self.engine.distances()
        dists = np.zeros(self.n_total, np.float32)
        for i, d in zip(self.local, mine):
            dists[i] = d
        if p.TrimmedMeanSize > 0 and self.group is not None and self.world > 1:
            import torch.distributed as dist
            t = torch.from_numpy(dists).to(self.engine.device_of_sums())
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
            dists = t.cpu().numpy()
        w = atlas_weights(self.weights, dists, p.ComputeMedian, p.TrimmedMeanSize)
        self.engine.set_weights([w[i] for i in self.local])

    def _update_mean(self):
        if self.param.UsePerVoxelMedian:
            return self._update_median()
        if self.param.ComputeMedian or self.param.TrimmedMeanSize > 0:
            self._reweigh()
        acc, jsum = self.engine.mean_sums()
        if self.group is not None and self.world > 1:
            import torch.distributed as dist
            dist.all_reduce(acc, op=dist.ReduceOp.SUM, group=self.group)
            if jsum is not None:
                dist.all_reduce(jsum, op=dist.ReduceOp.SUM, group=self.group)
        self.mean = self.engine.set_mean(acc, jsum)

    def BuildAtlas(self):
        """The AtlasThreadMain loop at one scale level: the mean, then per
        iteration every subject's LDMM iteration and the mean again."""
        self._update_mean()
        for k in range(self.param.NIterations):
            self.engine.iterate(first=(k == 0))
            self._update_mean()
        return self.mean

    def GetMeanImage(self) -> torch.Tensor:
        return self.mean

    def GetVelocities(self, i: int) -> torch.Tensor:
        """v [T, 3, nz, ny, nx] of global subject i (local to this rank); with
        Shooting, its initial momentum alpha0 [nz, ny, nx]."""
        return self.engine.velocities(self.local.index(i))

    def GetStepSize(self, i: int) -> float:
        return self.engine.step(self.local.index(i))

    def GetEnergies(self, i: int) -> np.ndarray:
        return self.engine.energies(self.local.index(i))
