"""GPU parity of the LDMM relaxation atlas (LDMMAtlasBuilderB200 over
libaw_b200.so) against the oracle's atlas loop, itself pinned against the
reference's LDMMDeformationData / LDMMIteratorCPU (tests/test_oracle_pin.py).

Tolerances:
* GetI1At0 and ComputeJacDet for given velocities: bit-exact (the
  interpolation, composition and Jacobian arithmetic follow the reference
  operation by operation);
* the atlas loop: mean within 1e-4 of max |mean|, velocities within 1e-3 of
  max |v| after 3 iterations of 3 subjects (FP32 FFT rounding of the fluid
  solve compounds through the mean that every subject reads), energies
  1e-4 relative.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from atlaswerks_b200 import _lib  # noqa: E402
from atlaswerks_b200.greedy import DiffOperParam  # noqa: E402
from atlaswerks_b200.ldmm import LDMMIteratorB200, LDMMIteratorParam  # noqa: E402
from atlaswerks_b200.ldmm_atlas import LDMMAtlasBuilderB200, LDMMAtlasParam  # noqa: E402
from atlaswerks_b200.synth import greedy_pair  # noqa: E402

pytestmark = pytest.mark.gpu


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.mark.parametrize("shape,sp", [((16, 16, 16), (1.0, 1.0, 1.0)),
                                      ((12, 14, 16), (1.5, 0.75, 1.25))])
def test_i1_at_0_bit_exact(oracle, shape, sp):
    T = 4
    rng = np.random.default_rng(3)
    _, I1 = greedy_pair(shape, 8, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0), smooth_sigma=3.0)
    v = rng.normal(0, 0.6, (T, 3) + shape).astype(np.float32)
    want_img, want_jd = oracle.ldmm_i1_at_0(I1, v, sp)
    it = LDMMIteratorB200(shape[::-1], spacing=sp, n_time_steps=T)
    it.SetScaleLevel(shape[::-1], sp, LDMMIteratorParam())
    img = torch.zeros(shape, device="cuda")
    jd = torch.zeros(shape, device="cuda")
    I1d, vd = cu(I1), cu(v)
    _lib.check(_lib.lib().aw_ldmm_i1_at_0(it._h, I1d.data_ptr(), vd.data_ptr(), img.data_ptr(),
                                          jd.data_ptr(), None))
    assert np.array_equal(host(img), want_img)
    assert np.array_equal(host(jd), want_jd)


@pytest.mark.parametrize("use_new,jacobian_scale,adaptive", [(True, True, False),
                                                              (False, True, True),
                                                              (True, False, True)])
def test_ldmm_atlas_vs_oracle(oracle, use_new, jacobian_scale, adaptive):
    shape, T, iters = (16, 16, 16), 3, 3
    imgs = [greedy_pair(shape, 40 + k, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0),
                        smooth_sigma=3.0)[1] for k in range(3)]
    w = [0.5, 0.3, 0.2]
    kw = dict(sigma=1.0, step=0.01, adaptive=adaptive, max_pert=0.2, use_new=use_new,
              jacobian_scale=jacobian_scale)
    m_o, v_o, e_o = oracle.ldmm_atlas_run(imgs, w, T, iters, **kw)
    param = LDMMAtlasParam(LDMMIteratorParam(DiffOperParam(), 1.0, 0.01, adaptive, 0.2),
                           NTimeSteps=T, NIterations=iters, JacobianScale=jacobian_scale,
                           UseOrigGradientCalc=not use_new)
    b = LDMMAtlasBuilderB200([cu(a) for a in imgs], shape[::-1], param, weights=w)
    mean = host(b.BuildAtlas())
    assert np.abs(mean - m_o).max() <= 1e-4 * np.abs(m_o).max()
    for i in range(3):
        vg = host(b.GetVelocities(i))
        assert np.abs(vg - v_o[i]).max() <= 1e-3 * np.abs(v_o[i]).max()
        assert np.allclose(b.GetEnergies(i)[-iters:], e_o[:, i], rtol=1e-4)
    assert np.abs(v_o[0]).max() > 0


def _device_median(imgs, k):
    t = [cu(a) for a in imgs]
    nz, ny, nx = imgs[0].shape
    out = torch.full(imgs[0].shape, float("nan"), device="cuda")
    import ctypes
    ptrs = (ctypes.c_void_p * len(t))(*[x.data_ptr() for x in t])
    rc = _lib.lib().aw_ldmm_atlas_voxel_median(ptrs, len(t), k, nx, ny, nz, out.data_ptr(), None)
    return rc, host(out)


def test_voxel_median_bit_exact(oracle):
    """aw_ldmm_atlas_voxel_median against the oracle's restatement of
    MedianCalculator::Select (pinned to the reference): random values, ties,
    every k, the eps rule (a volume whose range makes eps = 1, so voxels
    with values within 1 end at the lower end), and a constant volume,
    where the reference throws for k > 0 and the device reports an error."""
    rng = np.random.default_rng(8)
    shape = (9, 10, 11)
    for n in (1, 2, 3, 5, 8, 33):
        imgs = [rng.normal(0, 1, shape).astype(np.float32) for _ in range(n)]
        if n > 2:
            imgs[1][0] = imgs[0][0]
        for k in sorted({0, n // 2 - 1 if n % 2 == 0 else n // 2, n - 1}):
            rc, got = _device_median(imgs, k)
            assert rc == 0
            assert np.array_equal(got, oracle.voxel_median(imgs, k))
    imgs = [np.full(shape, 0.1 * (m + 1), np.float32) for m in range(5)]
    imgs[0][0, 0, 0] = 1e4
    rc, got = _device_median(imgs, 2)
    assert rc == 0 and np.array_equal(got, oracle.voxel_median(imgs, 2))
    assert got[1, 1, 1] == np.float32(0.1)
    const = [np.full(shape, 2.0, np.float32) for _ in range(3)]
    rc, _ = _device_median(const, 1)
    assert rc != 0 and b"converge" in _lib.lib().aw_last_error()
    rc, got = _device_median(const, 0)
    assert rc == 0 and np.all(got == 2.0)


def test_ldmm_atlas_voxel_median_vs_oracle(oracle):
    """UsePerVoxelMedian: the atlas whose mean is the per-voxel median of the
    deformed subjects (five subjects, median index 2) against the oracle's
    loop; same tolerances as the mean atlas."""
    shape, T, iters = (16, 16, 16), 3, 2
    imgs = [greedy_pair(shape, 50 + k, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0),
                        smooth_sigma=3.0)[1] for k in range(5)]
    w = [0.2] * 5
    m_o, v_o, e_o = oracle.ldmm_atlas_run(imgs, w, T, iters, sigma=1.0, step=0.01,
                                          adaptive=True, max_pert=0.2, voxel_median=True)
    param = LDMMAtlasParam(LDMMIteratorParam(DiffOperParam(), 1.0, 0.01, True, 0.2),
                           NTimeSteps=T, NIterations=iters, UsePerVoxelMedian=True)
    b = LDMMAtlasBuilderB200([cu(a) for a in imgs], shape[::-1], param, weights=w)
    mean = host(b.BuildAtlas())
    assert np.abs(mean - m_o).max() <= 1e-4 * np.abs(m_o).max()
    for i in range(5):
        vg = host(b.GetVelocities(i))
        assert np.abs(vg - v_o[i]).max() <= 1e-3 * np.abs(v_o[i]).max()
        assert np.allclose(b.GetEnergies(i)[-iters:], e_o[:, i], rtol=1e-4)


@pytest.mark.parametrize("compute_median,trimmed", [(True, 0), (False, 2)])
def test_ldmm_atlas_reweighted_vs_oracle(oracle, compute_median, trimmed):
    """ComputeMedian (weights divided by each subject's distance) and
    TrimmedMeanSize 2 of 4 (the two nearest subjects), distances from the
    image and vector energies, against the oracle's loop; same tolerances as
    the mean atlas."""
    shape, T, iters = (16, 16, 16), 3, 3
    imgs = [greedy_pair(shape, 60 + k, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0),
                        smooth_sigma=3.0)[1] for k in range(4)]
    w = [0.25] * 4
    m_o, v_o, e_o = oracle.ldmm_atlas_run(imgs, w, T, iters, sigma=1.0, step=0.01,
                                          adaptive=True, max_pert=0.2,
                                          compute_median=compute_median, trimmed=trimmed)
    param = LDMMAtlasParam(LDMMIteratorParam(DiffOperParam(), 1.0, 0.01, True, 0.2),
                           NTimeSteps=T, NIterations=iters, ComputeMedian=compute_median,
                           TrimmedMeanSize=trimmed)
    b = LDMMAtlasBuilderB200([cu(a) for a in imgs], shape[::-1], param, weights=w)
    mean = host(b.BuildAtlas())
    assert np.abs(mean - m_o).max() <= 1e-4 * np.abs(m_o).max()
    for i in range(4):
        vg = host(b.GetVelocities(i))
        assert np.abs(vg - v_o[i]).max() <= 1e-3 * np.abs(v_o[i]).max()
        assert np.allclose(b.GetEnergies(i)[-iters:], e_o[:, i], rtol=1e-4)


@pytest.mark.parametrize("jacobian_scale", [True, False])
def test_ldmm_shooting_atlas_vs_oracle(oracle, jacobian_scale):
    """The shooting atlas (LDMMShootingAtlasThreadCPU): every subject's
    momentum shooting toward the mean and the mean of I1(phi0T) weighted by
    splat(ones, phiT0), against the oracle's loop over its pinned shooting
    iteration: mean 1e-4 of max, alpha0 1e-3 of max, energies 1e-4."""
    shape, T, iters = (16, 16, 16), 3, 3
    imgs = [greedy_pair(shape, 70 + k, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0),
                        smooth_sigma=3.0)[1] for k in range(3)]
    w = [0.5, 0.3, 0.2]
    m_o, a_o, e_o = oracle.ldmm_shoot_atlas_run(imgs, w, T, iters, sigma=1.0, step=0.1,
                                                jacobian_scale=jacobian_scale)
    param = LDMMAtlasParam(LDMMIteratorParam(DiffOperParam(), 1.0, 0.1, False, 0.2),
                           NTimeSteps=T, NIterations=iters, JacobianScale=jacobian_scale,
                           Shooting=True)
    b = LDMMAtlasBuilderB200([cu(a) for a in imgs], shape[::-1], param, weights=w)
    mean = host(b.BuildAtlas())
    assert np.abs(mean - m_o).max() <= 1e-4 * np.abs(m_o).max()
    for i in range(3):
        ag = host(b.GetVelocities(i))
        assert np.abs(ag - a_o[i]).max() <= 1e-3 * np.abs(a_o[i]).max()
        assert np.allclose(b.GetEnergies(i)[-iters:], e_o[:, i], rtol=1e-4)
    assert np.abs(a_o[0]).max() > 0
