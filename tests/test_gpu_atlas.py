"""GPU parity of the batched greedy atlas (aw_atlas_*) against the oracle's
restatement of the AtlasThreadMain loop (oracle.Oracle.atlas_run), itself
pinned to the reference's own GreedyDeformationData / GreedyIteratorCPU
(tests/test_atlas_cpu.py).

Tolerances:
* the mean of given deformations (pure interpolation + float sum in
  subject order): bit-exact;
* after the iterations (FP32 FFT vs the oracle's FP64 solve): mean within
  1e-4 absolute, deformation RMS <= 1e-3 voxel, max <= 1e-2 voxel;
  per-subject steps within 1e-5 relative.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from atlaswerks_b200.atlas import CudaAtlasEngine, GreedyAtlasBuilderB200, GreedyAtlasParam  # noqa: E402
from atlaswerks_b200.greedy import DiffOperParam  # noqa: E402
from atlaswerks_b200.synth import atlas_subjects  # noqa: E402
from oracle import identity  # noqa: E402

pytestmark = pytest.mark.gpu

TEMPLATE = (32, 32, 32)  # (nx, ny, nz)


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def subjects(n, sizes, seed=5):
    return atlas_subjects(n, seed, sizes=sizes, n_blobs=10, umax=2.0)


def run_gpu(imgs, iters, period, max_pert=0.5):
    param = GreedyAtlasParam(DiffOperParam(), max_pert, iters, period)
    b = GreedyAtlasBuilderB200([cu(a) for a in imgs], TEMPLATE, param)
    mean = b.BuildAtlas()
    torch.cuda.synchronize()
    hs = [b.GetDeformationField(i).cpu().numpy() for i in range(len(imgs))]
    steps = [b.GetStepSize(i) for i in range(len(imgs))]
    en = np.stack([b.GetEnergies(i) for i in range(len(imgs))], 1)
    return mean.cpu().numpy(), hs, steps, en, b


@pytest.mark.parametrize("sizes", [(32,), (24, 28, 32, 36, 40)], ids=["equal", "uneven"])
def test_mean_of_given_fields_bit_exact(oracle, sizes):
    rng = np.random.default_rng(11)
    imgs = subjects(3, sizes)
    shape = TEMPLATE[::-1]
    hs = [identity(shape) + rng.normal(0, 1.5, (3,) + shape).astype(np.float32) for _ in imgs]
    w = [0.2, 0.5, 0.3]
    eng = CudaAtlasEngine(TEMPLATE, (1.0, 1.0, 1.0), GreedyAtlasParam(), [cu(a) for a in imgs], w)
    for i, h in enumerate(hs):
        eng.field(i).copy_(cu(h))
    got = eng.compute_mean().cpu().numpy()
    want = oracle.atlas_mean(imgs, hs, w)
    assert np.array_equal(got, want)
    eng.close()


@pytest.mark.parametrize("sizes", [(32,), (24, 28, 32, 36, 40)], ids=["equal", "uneven"])
@pytest.mark.parametrize("period", [1, 3])
def test_atlas_matches_oracle(oracle, sizes, period):
    imgs = subjects(4, sizes)
    iters = 6
    mean, hs, steps, en, _ = run_gpu(imgs, iters, period)
    w = [0.25] * 4
    m_o, h_o, e_o, s_o = oracle.atlas_run(imgs, w, TEMPLATE[::-1], iters, period)
    assert np.allclose(steps, s_o, rtol=1e-5, atol=0)
    assert np.abs(mean - m_o).max() <= 1e-4
    for a, b in zip(hs, h_o):
        d = a - b
        assert np.sqrt(np.mean(d * d)) <= 1e-3
        assert np.abs(d).max() <= 1e-2
    assert np.allclose(en, e_o, rtol=1e-4)


def test_graph_replay_equals_single_iterations():
    imgs = subjects(3, (24, 32, 40))
    param = GreedyAtlasParam(DiffOperParam(), 0.5, 7, 7)
    a = GreedyAtlasBuilderB200([cu(x) for x in imgs], TEMPLATE, param)
    a._update_mean()
    a.engine.iterate(7, True)
    b = GreedyAtlasBuilderB200([cu(x) for x in imgs], TEMPLATE, param)
    b._update_mean()
    for k in range(7):
        b.engine.iterate(1, k == 0)
    torch.cuda.synchronize()
    for i in range(3):
        assert torch.equal(a.GetDeformationField(i), b.GetDeformationField(i))


def test_atlas_energy_decreases():
    imgs = subjects(4, (32,))
    mean, hs, steps, en, _ = run_gpu(imgs, 20, 5)
    total = en.sum(1)
    assert total[-1] < 0.6 * total[0]


def test_set_subject_rejects_bad_index():
    from atlaswerks_b200 import _lib
    import ctypes
    h = ctypes.c_void_p()
    assert _lib.lib().aw_atlas_create(16, 16, 16, 1.0, 1.0, 1.0, 0.01, 0.01, 0.001, 0.5, 2,
                                      ctypes.byref(h)) == 0
    img = torch.zeros((16, 16, 16), device="cuda")
    assert _lib.lib().aw_atlas_set_subject(h, 2, img.data_ptr(), 16, 16, 16, 0.5) != 0
    assert b"out of range" in _lib.lib().aw_last_error()
    # iterating before every subject has an image is an error, not a fault
    assert _lib.lib().aw_atlas_iterate(h, 1, 1, None) != 0
    assert b"not set" in _lib.lib().aw_last_error()
    _lib.lib().aw_atlas_destroy(h)
