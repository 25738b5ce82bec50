"""CPU tests of the atlas path: the oracle's atlas loop pinned against the
reference's own GreedyDeformationData / GreedyIteratorCPU driven through
the AtlasThreadMain loop, and the multi-process path of
GreedyAtlasBuilderB200 (subject sharding + one all-reduce of the mean) on
world_size-2 gloo ranks, with an oracle-backed per-rank engine standing in
for the GPU."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from atlaswerks_b200.atlas import GreedyAtlasBuilderB200, GreedyAtlasParam, local_subjects  # noqa: E402
from atlaswerks_b200.greedy import DiffOperParam  # noqa: E402
from atlaswerks_b200.synth import atlas_subjects  # noqa: E402
from oracle import identity  # noqa: E402

TEMPLATE = (16, 16, 16)


def test_oracle_atlas_pinned_to_reference(oracle, reference):
    imgs = atlas_subjects(3, 9, sizes=(16,), n_blobs=6, umax=2.0)
    w = [0.3, 0.3, 0.4]
    for period in (1, 2):
        m_o, h_o, e_o, _ = oracle.atlas_run(imgs, w, (16, 16, 16), 5, period)
        m_r, h_r, e_r = reference.atlas_run(imgs, w, 5, period)
        # the oracle's FP64 fluid solve vs the reference's FP32 one
        assert np.abs(m_o - m_r).max() <= 1e-5
        assert max(np.abs(a - b).max() for a, b in zip(h_o, h_r)) <= 1e-4
        assert np.allclose(e_o, e_r, rtol=1e-5)


def test_local_subjects_partition():
    for n in (1, 5, 32):
        for world in (1, 2, 3, 8):
            if world > n:
                continue
            parts = [local_subjects(n, r, world) for r in range(world)]
            assert sorted(sum(parts, [])) == list(range(n))


class OracleAtlasEngine:
    """Per-rank engine over the oracle (CPU), same interface as CudaAtlasEngine."""

    def __init__(self, size, spacing, param, images, weights):
        from oracle import Oracle
        self.o = Oracle()
        nx, ny, nz = size
        self.shape = (nz, ny, nx)
        self.sp, self.param = spacing, param
        self.imgs = [np.ascontiguousarray(a.numpy()) for a in images]
        self.w = list(weights)
        self.hs = [identity(self.shape) for _ in images]
        self.steps = [0.0] * len(images)
        self.mean = torch.zeros(self.shape)

    def compute_mean(self):
        self.mean = torch.from_numpy(self.o.atlas_mean(self.imgs, self.hs, self.w))
        return self.mean

    def iterate(self, n, update_first):
        k = self.param.Kernel
        m = np.ascontiguousarray(self.mean.numpy())
        for it in range(n):
            for i, img in enumerate(self.imgs):
                _, self.steps[i] = self.o.atlas_iterate(
                    img, m, self.hs[i], self.sp, k.Alpha, k.Beta, k.Gamma, self.param.MaxPert,
                    update_first and it == 0, self.steps[i])

    def field(self, i):
        return torch.from_numpy(self.hs[i])


def _rank_main(rank, world, port, imgs, q):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        param = GreedyAtlasParam(DiffOperParam(), 0.5, 4, 2)
        b = GreedyAtlasBuilderB200([torch.from_numpy(a) for a in imgs], TEMPLATE, param,
                                   group=dist.group.WORLD, engine_factory=OracleAtlasEngine)
        mean = b.BuildAtlas().numpy().copy()
        q.put((rank, mean, {i: b.GetDeformationField(i).numpy().copy() for i in b.local}))
    finally:
        dist.destroy_process_group()


def test_two_rank_atlas_equals_one_process(oracle):
    import multiprocessing as mp
    imgs = atlas_subjects(4, 21, sizes=(12, 16, 20), n_blobs=6, umax=2.0)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, imgs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    m_o, h_o, _, _ = oracle.atlas_run(imgs, [0.25] * 4, TEMPLATE[::-1], 4, 2)
    for rank, mean, fields in res:
        # the all-reduce adds the two ranks' partial sums: a different float
        # summation order than one process's subject-order sum
        assert np.abs(mean - m_o).max() <= 1e-5
        for i, h in fields.items():
            assert i % 2 == rank
            assert np.abs(h - h_o[i]).max() <= 1e-3
