"""GPU parity of splatting and the LDMM relaxation (IterateNew) against the
oracle, through the C ABI.

Tolerances:
* splat: bit-exact — sources are merged per destination in source order and
  summed in float as forwardApply does; run to run bitwise identical.
* adjoint identity <I1(h), I2> = <I1, splat(I2, h)> to 1e-6 relative
  (cudaHField3DUtilsRoutineTests.cxx:61-72 uses 0.1 absolute on 32^3).
* LDMM velocity fields: max |v_gpu - v_oracle| <= 1e-4 * max |v_oracle| per
  iteration (FP32 FFT rounding only; the rest is bit-exact), energies 1e-5.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from atlaswerks_b200 import device as D  # noqa: E402
from atlaswerks_b200.greedy import DiffOperParam  # noqa: E402
from atlaswerks_b200.ldmm import (LDMMDeformationDataB200, LDMMIteratorB200,  # noqa: E402
                                  LDMMIteratorParam, ldmm_register)
from atlaswerks_b200.synth import bullseye, greedy_pair  # noqa: E402
from oracle import identity  # noqa: E402

pytestmark = pytest.mark.gpu


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.mark.parametrize("shape", [(16, 16, 16), (12, 11, 10), (9, 17, 31), (1, 8, 8),
                                   (32, 31, 36)])
@pytest.mark.parametrize("scale", [0.5, 2.0, 6.0])
def test_splat_bit_exact(oracle, shape, scale):
    rng = np.random.default_rng(11)
    img = rng.normal(0, 1, shape).astype(np.float32)
    h = identity(shape) + rng.normal(0, scale, (3,) + shape).astype(np.float32)
    want = oracle.splat(img, h)
    got = host(D.splat(cu(img), cu(h)))
    assert np.array_equal(got, want), np.abs(got - want).max()


def test_splat_compressing_map(oracle):
    """Many sources onto few cells (a contracting h): long buckets."""
    shape = (16, 16, 16)
    rng = np.random.default_rng(12)
    img = rng.random(shape, dtype=np.float32)
    h = (identity(shape) * 0.25 + 5.3).astype(np.float32)
    want = oracle.splat(img, h)
    got = host(D.splat(cu(img), cu(h)))
    assert np.array_equal(got, want)


@pytest.mark.parametrize("shape,scale,shift", [
    ((32, 32, 32), 0.0, 5.3),     # collapsed: every source in one cell (32768 sources)
    ((32, 32, 32), 0.0, -0.5),    # collapsed onto the cell (-1, 0) of every axis
    ((16, 16, 16), 0.2, 5.3),     # about 125 sources a cell: the CTA-wide sort
    ((32, 32, 32), 0.1, 3.3),     # about 1000 sources a cell, many long buckets
    ((24, 20, 28), 0.05, 1.1)])   # ragged grid, a few thousand sources a cell
def test_splat_collapsing_maps(oracle, shape, scale, shift):
    """Long buckets: bit-exact against forwardApply's source-order sums."""
    rng = np.random.default_rng(15)
    img = rng.random(shape, dtype=np.float32)
    h = (identity(shape) * np.float32(scale) + np.float32(shift)).astype(np.float32)
    want = oracle.splat(img, h)
    got = host(D.splat(cu(img), cu(h)))
    assert np.array_equal(got, want)
    again = host(D.splat(cu(img), cu(h)))
    assert np.array_equal(got, again)


def test_splat_deterministic_and_adjoint():
    shape = (64, 64, 64)
    rng = np.random.default_rng(13)
    h = cu(identity(shape) + rng.normal(0, 1.5, (3,) + shape).astype(np.float32))
    I1 = cu(rng.random(shape, dtype=np.float32))
    I2 = cu(rng.random(shape, dtype=np.float32))
    s1 = D.splat(I2, h)
    s2 = D.splat(I2, h)
    assert torch.equal(s1, s2)
    lhs = float((D.apply(I1, h).double() * I2.double()).sum())
    rhs = float((I1.double() * s1.double()).sum())
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)


def test_splat_bullseye_vs_oracle(oracle):
    """GPU splat = CPU forwardApply on a bullseye (cudaHField3DUtilsRoutineTests.cxx:84-100)."""
    shape = (32, 32, 32)
    img = bullseye(shape, [12, 8, 4])
    rng = np.random.default_rng(14)
    h = identity(shape) + rng.normal(0, 1.0, (3,) + shape).astype(np.float32)
    assert np.array_equal(host(D.splat(cu(img), cu(h))), oracle.splat(img, h))


def _ldmm(shape, T, sigma, step):
    nz, ny, nx = shape
    it = LDMMIteratorB200((nx, ny, nz), n_time_steps=T)
    it.SetScaleLevel((nx, ny, nz), (1.0, 1.0, 1.0),
                     LDMMIteratorParam(DiffOperParam(), sigma, step, False, 0.1))
    return it


@pytest.mark.parametrize("shape,T", [((16, 16, 16), 4), ((20, 18, 16), 3), ((32, 32, 32), 5),
                                     ((16, 16, 256), 2)])
def test_ldmm_iterations_vs_oracle(oracle, shape, T):
    I0, I1 = greedy_pair(shape, seed=21, n_blobs=4, umax=2.0)
    sigma, step = 1.0, 0.01
    it = _ldmm(shape, T, sigma, step)
    data = LDMMDeformationDataB200(cu(I0), cu(I1), T)
    v = np.zeros((T, 3) + shape, np.float32)
    for k in range(3):
        e_o, _ = oracle.ldmm_iterate(I0, I1, v, sigma=sigma, step=step)
        it.Iterate(data)
        got = host(data.V)
        err = np.abs(got - v).max() / max(np.abs(v).max(), 1e-12)
        assert err <= 1e-4, (k, err)
        data.V.copy_(cu(v))  # re-sync to the oracle's state
        assert abs(it.Energies()[-1] - e_o) <= 1e-5 * e_o


def test_ldmm_iterations_anisotropic_spacing_vs_oracle(oracle):
    """IterateNew on a power-of-two grid (the register-FFT path) with
    spacings whose gradient divisors are not powers of two: the same bar
    as at unit spacing."""
    shape, T, sp = (16, 16, 32), 3, (1.5, 0.75, 1.25)
    I0, I1 = greedy_pair(shape, seed=23, n_blobs=4, umax=2.0)
    sigma, step = 1.0, 0.01
    nz, ny, nx = shape
    it = LDMMIteratorB200((nx, ny, nz), spacing=sp, n_time_steps=T)
    it.SetScaleLevel((nx, ny, nz), sp, LDMMIteratorParam(DiffOperParam(), sigma, step, False, 0.1))
    data = LDMMDeformationDataB200(cu(I0), cu(I1), T, sp)
    v = np.zeros((T, 3) + shape, np.float32)
    for k in range(3):
        e_o, _ = oracle.ldmm_iterate(I0, I1, v, sp, sigma=sigma, step=step)
        it.Iterate(data)
        got = host(data.V)
        err = np.abs(got - v).max() / max(np.abs(v).max(), 1e-12)
        assert err <= 1e-4, (k, err)
        data.V.copy_(cu(v))
        assert abs(it.Energies()[-1] - e_o) <= 1e-5 * e_o


@pytest.mark.parametrize("shape,T,sp", [((16, 16, 16), 4, (1.0, 1.0, 1.0)),
                                        ((20, 18, 16), 3, (1.5, 0.75, 1.25))])
def test_ldmm_alphas_vs_oracle(oracle, shape, T, sp):
    """Iterate(computeAlphasOnly) + GetAlpha: bit-exact against the oracle's
    restatement (compose, apply, splat and one float scale per voxel), v
    unchanged, the image energy recorded."""
    I0, I1 = greedy_pair(shape, seed=25, n_blobs=4, umax=2.0)
    rng = np.random.default_rng(26)
    v = rng.normal(0, 0.3, (T, 3) + shape).astype(np.float32)
    nz, ny, nx = shape
    it = LDMMIteratorB200((nx, ny, nz), spacing=sp, n_time_steps=T)
    it.SetScaleLevel((nx, ny, nz), sp, LDMMIteratorParam(DiffOperParam(), 0.1, 0.005, False, 0.1))
    data = LDMMDeformationDataB200(cu(I0), cu(I1), T)
    data.V.copy_(cu(v))
    it.Iterate(data, computeAlphasOnly=True)
    want, e = oracle.ldmm_alphas(I0, I1, v, sp, sigma=0.1)
    for t in range(T):
        assert np.array_equal(host(it.GetAlpha(t)), want[t]), t
    assert np.array_equal(host(data.V), v)
    assert abs(it.Energies()[-1] - e) <= 1e-12 * e
    it.Iterate(data)
    with pytest.raises(RuntimeError):
        it.GetAlpha(0)


def test_ldmm_adaptive_step_vs_oracle(oracle):
    shape, T = (16, 16, 16), 4
    I0, I1 = greedy_pair(shape, seed=22, n_blobs=4, umax=2.0)
    it = _ldmm(shape, T, 0.1, 0.005)
    data = LDMMDeformationDataB200(cu(I0), cu(I1), T)
    data.V.normal_(0, 0.1, generator=torch.Generator(device="cuda").manual_seed(3))
    v = host(data.V).copy()
    _, step_o = oracle.ldmm_iterate(I0, I1, v, sigma=0.1, step=0.005, update_step=True,
                                    max_pert=0.1)
    it.UpdateStepSizeNextIteration()
    it.Iterate(data)
    assert abs(it.StepSize() - step_o) <= 1e-4 * step_o
    assert np.array_equal(host(data.V), v)  # no velocity update in the step pass


def test_ldmm_run_equals_iterate():
    shape, T = (16, 16, 16), 3
    I0, I1 = greedy_pair(shape, seed=23, n_blobs=4, umax=2.0)
    a = _ldmm(shape, T, 1.0, 0.01)
    da = LDMMDeformationDataB200(cu(I0), cu(I1), T)
    a.Run(da, 5)
    b = _ldmm(shape, T, 1.0, 0.01)
    db = LDMMDeformationDataB200(cu(I0), cu(I1), T)
    for _ in range(5):
        b.Iterate(db)
    assert torch.equal(da.V, db.V)
    assert np.array_equal(a.Energies(), b.Energies())


def test_ldmm_register_decreases_energy():
    shape = (32, 32, 32)
    I0, I1 = greedy_pair(shape, seed=24, n_blobs=6, umax=2.0)
    V, e, _ = ldmm_register(cu(I0), cu(I1), 5, 20, sigma=1.0, step=0.01)
    assert len(e) == 20
    assert e[-1] < 0.7 * e[0]


@pytest.mark.parametrize("shape,T,sp", [((16, 16, 16), 4, (1.0, 1.0, 1.0)),
                                        ((12, 14, 16), 3, (1.5, 0.75, 1.25)),
                                        ((32, 32, 32), 5, (1.0, 1.0, 1.0)),
                                        ((16, 16, 256), 2, (1.0, 1.0, 1.0)),
                                        ((16, 16, 32), 2, (1.5, 0.75, 1.25))])
def test_ldmm_orig_iterations_vs_oracle(oracle, shape, T, sp):
    """IterateOrig (Jacobian transport): same bar as IterateNew."""
    I0, I1 = greedy_pair(shape, seed=31, n_blobs=5, umax=1.5, sigma_range=(1.5, 3.0),
                         smooth_sigma=3.0)
    sigma, step = 1.0, 0.01
    nz, ny, nx = shape
    it = LDMMIteratorB200((nx, ny, nz), spacing=sp, n_time_steps=T)
    it.SetUseOrigGradientCalc(True)
    it.SetScaleLevel((nx, ny, nz), sp, LDMMIteratorParam(DiffOperParam(), sigma, step, False, 0.1))
    data = LDMMDeformationDataB200(cu(I0), cu(I1), T, sp)
    v = np.zeros((T, 3) + shape, np.float32)
    for k in range(3):
        e_o, _ = oracle.ldmm_iterate_orig(I0, I1, v, sp, sigma=sigma, step=step)
        it.Iterate(data)
        got = host(data.V)
        err = np.abs(got - v).max() / max(np.abs(v).max(), 1e-12)
        assert err <= 1e-4, (k, err)
        data.V.copy_(cu(v))
        assert abs(it.Energies()[-1] - e_o) <= 1e-5 * e_o


def test_ldmm_orig_adaptive_step_vs_oracle(oracle):
    shape, T = (16, 16, 16), 3
    I0, I1 = greedy_pair(shape, seed=32, n_blobs=5, umax=1.5, sigma_range=(1.5, 3.0),
                         smooth_sigma=3.0)
    nz, ny, nx = shape
    it = LDMMIteratorB200((nx, ny, nz), n_time_steps=T)
    it.SetUseOrigGradientCalc(True)
    it.SetScaleLevel((nx, ny, nz), (1.0, 1.0, 1.0),
                     LDMMIteratorParam(DiffOperParam(), 1.0, 0.01, True, 0.2))
    data = LDMMDeformationDataB200(cu(I0), cu(I1), T)
    data.V.normal_(0, 0.05, generator=torch.Generator(device="cuda").manual_seed(4))
    v = host(data.V).copy()
    _, step_o = oracle.ldmm_iterate_orig(I0, I1, v, sigma=1.0, step=0.01, update_step=True,
                                         max_pert=0.2)
    it.UpdateStepSizeNextIteration()
    it.Iterate(data)
    assert abs(it.StepSize() - step_o) <= 1e-4 * step_o
    assert np.array_equal(host(data.V), v)


@pytest.mark.parametrize("orig", [False, True])
def test_ldmm_vector_energies_vs_oracle(oracle, orig):
    """SetVectorEnergy (the reference's debug-mode <L v_t, v_t>): each
    iteration's sum over t against the oracle's (pinned to the reference),
    1e-4 relative (FP32 transforms on both sides, summed in double); the
    velocities and image energies equal those of a run without it."""
    shape, T, sp = (20, 18, 16), 3, (1.5, 0.75, 1.25)
    I0, I1 = greedy_pair(shape, seed=31, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0),
                         smooth_sigma=3.0)
    nz, ny, nx = shape
    its, datas = [], []
    for vec in (True, False):
        it = LDMMIteratorB200((nx, ny, nz), spacing=sp, n_time_steps=T)
        it.SetUseOrigGradientCalc(orig)
        it.SetVectorEnergy(vec)
        it.SetScaleLevel((nx, ny, nz), sp, LDMMIteratorParam(DiffOperParam(), 1.0, 0.01, False))
        its.append(it)
        datas.append(LDMMDeformationDataB200(cu(I0), cu(I1), T, sp))
    v = np.zeros((T, 3) + shape, np.float32)
    step_fn = oracle.ldmm_iterate_orig if orig else oracle.ldmm_iterate
    for k in range(3):
        _, _, ve = step_fn(I0, I1, v, sp, sigma=1.0, step=0.01, vec=True)
        for it, d in zip(its, datas):
            it.Iterate(d)
        got = its[0].VecEnergies()[-1]
        assert ve > 0 and abs(got - ve) <= 1e-4 * ve, (k, got, ve)
        assert torch.equal(datas[0].V, datas[1].V)
        assert its[0].Energies()[-1] == its[1].Energies()[-1]
        for d in datas:
            d.V.copy_(cu(v))  # re-sync to the oracle's state
    assert its[0].TotalEnergy() > 0
