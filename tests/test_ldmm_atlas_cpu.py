"""CPU tests of the LDMM atlas host path: LDMMAtlasBuilderB200's sharding of
subjects over world_size-2 gloo ranks and the two all-reduces of the mean's
sums, with an oracle-backed per-rank engine standing in for the GPU,
against the oracle's one-process atlas loop (itself pinned against the
reference in tests/test_oracle_pin.py)."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from atlaswerks_b200.greedy import DiffOperParam  # noqa: E402
from atlaswerks_b200.ldmm import LDMMIteratorParam  # noqa: E402
from atlaswerks_b200.ldmm_atlas import LDMMAtlasBuilderB200, LDMMAtlasParam  # noqa: E402
from atlaswerks_b200.synth import greedy_pair  # noqa: E402

SHAPE = (12, 12, 12)


class OracleLDMMAtlasEngine:
    """Per-rank engine over the oracle (CPU), same interface as CudaLDMMAtlasEngine."""

    def __init__(self, size, spacing, param, images, weights):
        from oracle import Oracle
        self.o = Oracle()
        nx, ny, nz = size
        self.shape = (nz, ny, nx)
        self.sp, self.param = spacing, param
        self.imgs = [np.ascontiguousarray(a.numpy()) for a in images]
        self.w = list(weights)
        T = param.NTimeSteps
        self.vs = [np.zeros((T, 3) + self.shape, np.float32) for _ in images]
        self.steps = [param.Iterator.StepSize] * len(images)
        self.mean = np.zeros(self.shape, np.float32)
        self.dists = [0.0] * len(images)
        self.reweigh = param.ComputeMedian or param.TrimmedMeanSize > 0

    def mean_sums(self):
        acc, jsum = self.o.ldmm_atlas_mean_sums(self.imgs, self.vs, self.w, self.sp,
                                                self.param.JacobianScale)
        return torch.from_numpy(acc), (torch.from_numpy(jsum) if jsum is not None else None)

    def deformed(self):
        return [torch.from_numpy(self.o.ldmm_i1_at_0(img, v, self.sp, jacdet=False)[0])
                for img, v in zip(self.imgs, self.vs)]

    def set_median(self, images, k):
        self.mean = self.o.voxel_median([t.numpy() for t in images], k)
        return torch.from_numpy(self.mean)

    def set_mean(self, acc, jsum):
        m = acc.numpy() / jsum.numpy() if jsum is not None else acc.numpy()
        self.mean = np.ascontiguousarray(m, np.float32)
        return torch.from_numpy(self.mean)

    def iterate(self, first):
        p, k = self.param.Iterator, self.param.Iterator.Kernel
        it = self.o.ldmm_iterate_orig if self.param.UseOrigGradientCalc else self.o.ldmm_iterate
        kw = dict(sp=self.sp, alpha=k.Alpha, beta=k.Beta, gamma=k.Gamma, sigma=p.Sigma)
        for i, img in enumerate(self.imgs):
            if first and p.UseAdaptiveStepSize:
                _, self.steps[i] = it(self.mean, img, self.vs[i], step=self.steps[i],
                                      update_step=True, max_pert=p.MaxPert, **kw)
            r = it(self.mean, img, self.vs[i], step=self.steps[i], vec=self.reweigh, **kw)
            if self.reweigh:
                self.dists[i] = float(self.o.ldmm_distance(r[0], r[2], p.Sigma,
                                                           self.param.NTimeSteps))

    def distances(self):
        return list(self.dists)

    def set_weights(self, weights):
        self.w = list(weights)

    def device_of_sums(self):
        return torch.device("cpu")

    def velocities(self, i):
        return torch.from_numpy(self.vs[i])


def _param(median=False, compute_median=False, trimmed=0, iters=2):
    return LDMMAtlasParam(LDMMIteratorParam(DiffOperParam(), 1.0, 0.01, True, 0.2), NTimeSteps=3,
                          NIterations=iters, JacobianScale=True, UsePerVoxelMedian=median,
                          ComputeMedian=compute_median, TrimmedMeanSize=trimmed)


def _subjects():
    return [greedy_pair(SHAPE, 60 + k, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0),
                        smooth_sigma=3.0)[1] for k in range(4)]


def test_one_process_builder_equals_oracle_loop(oracle):
    imgs = _subjects()
    b = LDMMAtlasBuilderB200([torch.from_numpy(a) for a in imgs], SHAPE, _param(),
                             engine_factory=OracleLDMMAtlasEngine)
    mean = b.BuildAtlas().numpy()
    m_o, v_o, _ = oracle.ldmm_atlas_run(imgs, [0.25] * 4, 3, 2, sigma=1.0, step=0.01,
                                        adaptive=True, max_pert=0.2)
    assert np.array_equal(mean, m_o)
    for i in range(4):
        assert np.array_equal(b.GetVelocities(i).numpy(), v_o[i])


def test_one_process_voxel_median_builder_equals_oracle_loop(oracle):
    """UsePerVoxelMedian: the builder's mean is the per-voxel median of the
    deformed subjects, as the oracle's loop forms it (five subjects: an odd
    count, median index 2)."""
    imgs = _subjects() + [greedy_pair(SHAPE, 70, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0),
                                      smooth_sigma=3.0)[1]]
    b = LDMMAtlasBuilderB200([torch.from_numpy(a) for a in imgs], SHAPE, _param(True),
                             engine_factory=OracleLDMMAtlasEngine)
    mean = b.BuildAtlas().numpy()
    m_o, v_o, _ = oracle.ldmm_atlas_run(imgs, [0.2] * 5, 3, 2, sigma=1.0, step=0.01,
                                        adaptive=True, max_pert=0.2, voxel_median=True)
    assert np.array_equal(mean, m_o)
    for i in range(5):
        assert np.array_equal(b.GetVelocities(i).numpy(), v_o[i])


@pytest.mark.parametrize("compute_median,trimmed", [(True, 0), (False, 2), (True, 3)])
def test_one_process_reweighted_builder_equals_oracle_loop(oracle, compute_median, trimmed):
    """ComputeMedian and TrimmedMeanSize: the builder's weights (from the
    subjects' image and vector energies) and mean equal the oracle loop's
    bit for bit, three iterations so the trimming drops a subject."""
    imgs = _subjects()
    b = LDMMAtlasBuilderB200([torch.from_numpy(a) for a in imgs], SHAPE,
                             _param(compute_median=compute_median, trimmed=trimmed, iters=3),
                             engine_factory=OracleLDMMAtlasEngine)
    mean = b.BuildAtlas().numpy()
    m_o, v_o, _ = oracle.ldmm_atlas_run(imgs, [0.25] * 4, 3, 3, sigma=1.0, step=0.01,
                                        adaptive=True, max_pert=0.2,
                                        compute_median=compute_median, trimmed=trimmed)
    assert np.array_equal(mean, m_o)
    for i in range(4):
        assert np.array_equal(b.GetVelocities(i).numpy(), v_o[i])


def test_reweighting_changes_the_mean(oracle):
    """The trimmed mean of 2 of 4 subjects is not the plain mean."""
    imgs = _subjects()
    m_p, _, _ = oracle.ldmm_atlas_run(imgs, [0.25] * 4, 3, 2, sigma=1.0, step=0.01,
                                      adaptive=True, max_pert=0.2)
    m_t, _, _ = oracle.ldmm_atlas_run(imgs, [0.25] * 4, 3, 2, sigma=1.0, step=0.01,
                                      adaptive=True, max_pert=0.2, trimmed=2)
    assert np.abs(m_p - m_t).max() > 1e-4


def _rank_main(rank, world, port, imgs, q, median=False, trimmed=0):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        b = LDMMAtlasBuilderB200([torch.from_numpy(a) for a in imgs], SHAPE,
                                 _param(median, trimmed=trimmed),
                                 group=dist.group.WORLD, engine_factory=OracleLDMMAtlasEngine)
        mean = b.BuildAtlas().numpy().copy()
        q.put((rank, mean, {i: b.GetVelocities(i).numpy().copy() for i in b.local}))
    finally:
        dist.destroy_process_group()


def test_two_rank_ldmm_atlas_equals_one_process(oracle):
    import multiprocessing as mp
    imgs = _subjects()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() + 371) % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, imgs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    m_o, v_o, _ = oracle.ldmm_atlas_run(imgs, [0.25] * 4, 3, 2, sigma=1.0, step=0.01,
                                        adaptive=True, max_pert=0.2)
    for rank, mean, vs in res:
        # the all-reduces add the two ranks' partial sums: another float
        # summation order than one process's subject-order sum
        assert np.abs(mean - m_o).max() <= 1e-5 * np.abs(m_o).max()
        for i, v in vs.items():
            assert i % 2 == rank
            assert np.abs(v - v_o[i]).max() <= 1e-3 * np.abs(v_o[i]).max()


def test_two_rank_voxel_median_equals_one_process(oracle):
    """UsePerVoxelMedian over two gloo ranks: each deformed subject is
    broadcast by its owner, every rank selects over all four, and the mean
    and velocities equal the one-process oracle loop bit for bit (the
    selection does not depend on the images' order)."""
    import multiprocessing as mp
    imgs = _subjects()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() + 613) % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, imgs, q, True)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    m_o, v_o, _ = oracle.ldmm_atlas_run(imgs, [0.25] * 4, 3, 2, sigma=1.0, step=0.01,
                                        adaptive=True, max_pert=0.2, voxel_median=True)
    for rank, mean, vs in res:
        assert np.array_equal(mean, m_o)
        for i, v in vs.items():
            assert np.array_equal(v, v_o[i])


def test_two_rank_trimmed_mean_equals_one_process(oracle):
    """TrimmedMeanSize 2 over two gloo ranks: the distances of all four
    subjects are summed into one vector before the selection, so both ranks
    weigh the same two subjects as the one-process loop."""
    import multiprocessing as mp
    imgs = _subjects()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() + 811) % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, imgs, q, False, 2))
             for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    m_o, v_o, _ = oracle.ldmm_atlas_run(imgs, [0.25] * 4, 3, 2, sigma=1.0, step=0.01,
                                        adaptive=True, max_pert=0.2, trimmed=2)
    for rank, mean, vs in res:
        assert np.abs(mean - m_o).max() <= 1e-5 * np.abs(m_o).max()
        for i, v in vs.items():
            assert np.abs(v - v_o[i]).max() <= 1e-3 * np.abs(v_o[i]).max()
