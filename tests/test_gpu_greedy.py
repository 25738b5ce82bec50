"""GPU parity of the greedy-fluid path against the oracle (C restatement of
the reference CPU routines), through the C ABI.

Tolerances:
* interpolation, gradient, compose (apply / composeHV / composeVHInv ...):
  bit-exact — same float/double operation sequence as the reference.
* fluid operator L^-1 and L: max |gpu - fp64| / max |fp64| <= 1e-5.
* greedy run (deformation fields): RMS of (h_gpu - h_oracle) <= 1e-3 voxel
  after the full iteration count; energies within 1e-4 relative.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from atlaswerks_b200 import device as D  # noqa: E402
from atlaswerks_b200.greedy import (DiffOperB200, DiffOperParam, GreedyDeformationDataB200,  # noqa: E402
                                    GreedyIteratorB200, GreedyIteratorParam, greedy_register)
from atlaswerks_b200.synth import greedy_pair  # noqa: E402
from oracle import identity  # noqa: E402

pytestmark = pytest.mark.gpu

SHAPES = [(16, 16, 16), (12, 11, 10), (9, 17, 31), (36, 31, 32)]
SPACINGS = [(1.0, 1.0, 1.0), (2.0, 2.06452, 1.77778)]


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.mark.parametrize("shape", SHAPES)
def test_apply_bit_exact(oracle, shape):
    rng = np.random.default_rng(1)
    img = rng.random(shape, dtype=np.float32)
    h = identity(shape) + rng.normal(0, 2.0, (3,) + shape).astype(np.float32)
    want = oracle.apply(img, h)
    got = host(D.apply(cu(img), cu(h)))
    assert np.array_equal(got, want)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("sp", SPACINGS)
@pytest.mark.parametrize("wrap", [False, True])
def test_gradient_bit_exact(oracle, shape, sp, wrap):
    rng = np.random.default_rng(2)
    img = rng.random(shape, dtype=np.float32)
    want = oracle.gradient(img, sp, wrap)
    got = host(D.gradient(cu(img), sp, wrap))
    assert np.array_equal(got, want)


@pytest.mark.parametrize("bg", range(6))
@pytest.mark.parametrize("direction", [1, -1])
def test_compose_bit_exact(oracle, bg, direction):
    shape, sp = (12, 11, 10), (1.0, 1.3, 0.8)
    rng = np.random.default_rng(3)
    g = identity(shape) + rng.normal(0, 1.5, (3,) + shape).astype(np.float32)
    v = rng.normal(0, 1.5, (3,) + shape).astype(np.float32)
    want = oracle.compose_hv(g, v, sp, direction, bg)
    got = host(D.compose_hv(cu(g), cu(v), sp, 1.0, direction, bg))
    assert np.array_equal(got, want)
    want = oracle.compose_vh(v, g, sp, direction, bg)
    got = host(D.compose_vh(cu(v), cu(g), sp, 1.0, direction, bg))
    assert np.array_equal(got, want)


# power-of-two grids take the register-FFT kernels, the others the generic
# shared-memory Stockham kernels
FLUID_SHAPES = SHAPES + [(64, 64, 64), (32, 48, 40), (128, 128, 128), (32, 64, 128),
                         (128, 16, 64), (16, 32, 16), (256, 32, 16)]
# slabs too large for one CTA's shared memory: the split x / y passes
SPLIT_SHAPES = [(8, 256, 256), (6, 288, 320), (3, 512, 512), (4, 250, 462)]


@pytest.mark.parametrize("shape", FLUID_SHAPES + SPLIT_SHAPES)
@pytest.mark.parametrize("inverse", [True, False])
def test_fluid_operator_vs_fp64(oracle, shape, inverse):
    rng = np.random.default_rng(4)
    sp = (1.0, 1.3, 0.8)
    f = rng.normal(0, 1, (3,) + shape).astype(np.float32)
    want = oracle.fluid_f64(f, sp, inverse=inverse)
    op = DiffOperB200()
    op.SetSize((shape[2], shape[1], shape[0]), sp, DiffOperParam())
    v = cu(f)
    (op.ApplyInverseOperator if inverse else op.ApplyOperator)(v)
    got = host(v).astype(np.float64)
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err <= 1e-5, err


def test_fluid_roundtrip_identity():
    """L^-1 L = I (DiffOperRoutineTests.cxx:120-203, sum of squared diff <= 0.1)."""
    rng = np.random.default_rng(5)
    shape = (32, 32, 32)
    f = rng.normal(0, 1, (3,) + shape).astype(np.float32)
    op = DiffOperB200()
    op.SetSize((32, 32, 32), (1.0, 1.25, 1.0), DiffOperParam())
    v = cu(f)
    op.ApplyOperator(v)
    op.ApplyInverseOperator(v)
    d = host(v) - f
    assert float((d.astype(np.float64) ** 2).sum()) <= 0.1


def test_bounded_wait_runs_out_and_is_reported():
    """The transforms' bounded wait, run out on purpose (one CTA waiting 64
    polls on a barrier that nothing arrives on): the handle's status word
    reports the timeout once and is cleared by the read, and the context
    stays usable — the next L^-1 L round trip is correct with a clean status."""
    import ctypes
    from atlaswerks_b200 import _lib
    op = DiffOperB200()
    op.SetSize((32, 32, 32), (1.0, 1.0, 1.0), DiffOperParam())
    assert not op.TimedOut()
    s = torch.cuda.current_stream().cuda_stream
    assert _lib.lib().aw_fluid_wait_selftest(op._h, 64, s) == 0
    assert op.TimedOut()
    assert not op.TimedOut()
    assert _lib.lib().aw_fluid_wait_selftest(op._h, 0, s) != 0  # polls out of range
    f = np.random.default_rng(6).normal(0, 1, (3, 32, 32, 32)).astype(np.float32)
    v = cu(f)
    op.ApplyOperator(v)
    op.ApplyInverseOperator(v)
    d = host(v) - f
    assert float((d.astype(np.float64) ** 2).sum()) <= 0.1
    assert not op.TimedOut()
    flag = ctypes.c_int(-1)
    it = GreedyIteratorB200((32, 32, 32))
    it.SetScaleLevel((32, 32, 32), (1.0, 1.0, 1.0), GreedyIteratorParam(DiffOperParam(), 0.5))
    assert _lib.lib().aw_greedy_status(it._h, ctypes.byref(flag), s) == 0
    assert flag.value == 0


def test_diffoper_rejects_unsupported():
    op = DiffOperB200()
    with pytest.raises(ValueError):
        op.SetSize((16, 16, 16), (1, 1, 1), DiffOperParam(LPow=2.0))
    with pytest.raises(ValueError):
        op.SetSize((16, 16, 16), (1, 1, 1), DiffOperParam(DivergenceFree=True))


# (16, 32, 256): 256-wide rows, whose body-force loads go in chunks of two;
# (16, 32, 64) with spacings whose gradient divisors are not powers of two
# (the register path's body force divides in double there)
@pytest.mark.parametrize("shape,sp", [((16, 16, 16), (1.0, 1.0, 1.0)),
                                      ((24, 20, 18), (1.0, 1.0, 1.0)),
                                      ((6, 256, 256), (1.0, 1.0, 1.0)),
                                      ((16, 32, 256), (1.0, 1.0, 1.0)),
                                      ((16, 32, 64), (1.5, 0.75, 1.25))])
@pytest.mark.parametrize("inverse", [False, True])
def test_greedy_single_iterations(oracle, shape, sp, inverse):
    """Each Iterate from the same state as the oracle's (fields re-synchronised
    every step, so only one step of FP32 FFT error separates them)."""
    I0, I1 = greedy_pair(shape, seed=7, n_blobs=4, umax=2.0)
    nz, ny, nx = shape
    it = GreedyIteratorB200((nx, ny, nz), spacing=sp)
    it.SetScaleLevel((nx, ny, nz), sp, GreedyIteratorParam(DiffOperParam(), 0.5))
    data = GreedyDeformationDataB200(cu(I0), cu(I1), sp, compute_inverse=inverse)
    h = identity(shape)
    hi = identity(shape) if inverse else None
    step = 0.0
    for k in range(4):
        if k == 0:
            it.UpdateStepSizeNextIteration()
        e_o, step = oracle.greedy_iterate(I0, I1, h, hi, sp, max_pert=0.5,
                                          update_step=(k == 0), step=step)
        it.Iterate(data)
        assert abs(it.StepSize() - step) <= 1e-5 * step
        got = host(data.Def1To0())
        assert np.abs(got - h).max() <= 1e-4
        data.Def1To0().copy_(cu(h))  # re-sync
        if inverse:
            goti = host(data.Def0To1())
            assert np.abs(goti - hi).max() <= 1e-4
            data.Def0To1().copy_(cu(hi))
        e_g = it.Energies()[-1]
        assert abs(e_g - e_o) <= 1e-6 * max(1.0, e_o)


def test_greedy_run_matches_oracle_64(oracle):
    """Config-1 shape: 64^3, 50 iterations, MaxPert 0.5; final field within
    1e-3 voxel RMS of the oracle."""
    shape = (64, 64, 64)
    I0, I1 = greedy_pair(shape, seed=11, n_blobs=8, umax=3.0)
    h_o, _, e_o, step_o = oracle.greedy_run(I0, I1, 50, max_pert=0.5)
    h_g, _, e_g, step_g = greedy_register(cu(I0), cu(I1), 50, max_pert=0.5)
    h_g = host(h_g)
    rms = float(np.sqrt(((h_g - h_o).astype(np.float64) ** 2).sum(0).mean()))
    assert rms <= 1e-3, rms
    assert len(e_g) == 50
    assert np.allclose(e_g, e_o, rtol=1e-4)
    assert abs(step_g - step_o) <= 1e-5 * step_o


def test_set_to_identity_restarts_a_registration():
    """SetToIdentity (the library's identity kernel on the current stream)
    restores Def1To0 and Def0To1 to the identity exactly, and a second run
    on the same data object gives the first run's fields bit for bit."""
    shape = (16, 24, 32)
    I0, I1 = greedy_pair(shape, seed=4, n_blobs=4, umax=2.0)
    nz, ny, nx = shape
    it = GreedyIteratorB200((nx, ny, nz))
    it.SetScaleLevel((nx, ny, nz), (1.0, 1.0, 1.0), GreedyIteratorParam(DiffOperParam(), 0.5))
    d = GreedyDeformationDataB200(cu(I0), cu(I1), compute_inverse=True)
    it.Run(d, 5, update_first=True)
    first = (host(d.Def1To0()).copy(), host(d.Def0To1()).copy())
    assert np.abs(first[0] - identity(shape)).max() > 0.01
    d.SetToIdentity()
    assert np.array_equal(host(d.Def1To0()), identity(shape))
    assert np.array_equal(host(d.Def0To1()), identity(shape))
    it.Run(d, 5, update_first=True)
    assert np.array_equal(host(d.Def1To0()), first[0])
    assert np.array_equal(host(d.Def0To1()), first[1])


def test_greedy_run_iterate_equivalence():
    """aw_greedy_run (graph replay) == repeated aw_greedy_iterate, bitwise."""
    shape = (20, 18, 16)
    I0, I1 = greedy_pair(shape, seed=3, n_blobs=4, umax=2.0)
    sp = (1.0, 1.0, 1.0)
    p = GreedyIteratorParam(DiffOperParam(), 0.5)
    a = GreedyIteratorB200((16, 18, 20))
    a.SetScaleLevel((16, 18, 20), sp, p)
    da = GreedyDeformationDataB200(cu(I0), cu(I1), sp, True)
    a.Run(da, 7, update_first=True)
    b = GreedyIteratorB200((16, 18, 20))
    b.SetScaleLevel((16, 18, 20), sp, p)
    db = GreedyDeformationDataB200(cu(I0), cu(I1), sp, True)
    for k in range(7):
        if k == 0:
            b.UpdateStepSizeNextIteration()
        b.Iterate(db)
    assert torch.equal(da.Def1To0(), db.Def1To0())
    assert torch.equal(da.Def0To1(), db.Def0To1())
    assert np.array_equal(a.Energies(), b.Energies())


@pytest.mark.parametrize("shape,n", [((64, 64, 64), 9), ((32, 64, 128), 4), ((16, 16, 32), 3)])
def test_fused_run_equals_iterations(shape, n):
    """aw_greedy_run on power-of-two grids (the fused inverse-and-update
    kernel inside captured graphs, two calls in a row) equals repeated
    aw_greedy_iterate bit for bit, fields and energies."""
    nz, ny, nx = shape
    I0, I1 = greedy_pair(shape, seed=4, n_blobs=6, umax=2.0)
    p = GreedyIteratorParam(DiffOperParam(), 0.5)
    out = []
    for run in (True, False):
        it = GreedyIteratorB200((nx, ny, nz))
        it.SetScaleLevel((nx, ny, nz), (1.0, 1.0, 1.0), p)
        d = GreedyDeformationDataB200(cu(I0), cu(I1))
        if run:
            it.Run(d, n, update_first=True)
            it.Run(d, n, update_first=False)
        else:
            for k in range(2 * n):
                if k == 0:
                    it.UpdateStepSizeNextIteration()
                it.Iterate(d)
        out.append((host(d.Def1To0()).copy(), it.Energies()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_greedy_deterministic():
    shape = (32, 32, 32)
    I0, I1 = greedy_pair(shape, seed=5)
    r1 = greedy_register(cu(I0), cu(I1), 10)
    r2 = greedy_register(cu(I0), cu(I1), 10)
    assert torch.equal(r1[0], r2[0])
    assert np.array_equal(r1[2], r2[2])


# NaN, infinite and huge positions (a diverged or untrained deformation):
# every kernel treats them as far outside the volume and reads nothing out
# of range. Voxels whose positions are finite keep their exact values.
_BAD = np.array([np.nan, np.inf, -np.inf, 1e30, -1e30, 3e9, -3e9, 2.2e9], np.float32)


def _plant(field, rng, count=64):
    """A copy of field with `count` entries of every component replaced by
    the values of _BAD; returns (copy, mask of the voxels touched)."""
    out = field.copy()
    n = field[0].size
    mask = np.zeros(n, bool)
    for c in range(3):
        idx = rng.choice(n, count, replace=False)
        out[c].reshape(-1)[idx] = _BAD[rng.integers(0, len(_BAD), count)]
        mask[idx] = True
    return out, mask.reshape(field.shape[1:])


def test_nonfinite_positions_apply_splat(oracle):
    shape = (12, 11, 10)
    rng = np.random.default_rng(11)
    img = rng.random(shape, dtype=np.float32)
    h = identity(shape) + rng.normal(0, 2.0, (3,) + shape).astype(np.float32)
    bad, mask = _plant(h, rng)
    got = host(D.apply(cu(img), cu(bad), 0.5))
    assert np.array_equal(got[~mask], oracle.apply(img, h, 0.5)[~mask])
    # the splat skips sources outside the grown volume: the same sum as with
    # those sources moved far outside
    far = h.copy()
    for c in range(3):
        far[c][mask] = -1.0e4
    assert np.array_equal(host(D.splat(cu(img), cu(bad))), oracle.splat(img, far))


@pytest.mark.parametrize("bg", range(6))
def test_nonfinite_velocity_compose(oracle, bg):
    shape, sp = (12, 11, 10), (1.0, 1.3, 0.8)
    rng = np.random.default_rng(12)
    g = identity(shape) + rng.normal(0, 1.5, (3,) + shape).astype(np.float32)
    v = rng.normal(0, 1.5, (3,) + shape).astype(np.float32)
    bad, mask = _plant(v, rng)
    got = host(D.compose_hv(cu(g), cu(bad), sp, 1.0, 1, bg))
    want = oracle.compose_hv(g, v, sp, 1, bg)
    assert np.array_equal(got[:, ~mask], want[:, ~mask])


def test_nonfinite_deformation_iterates_without_fault():
    """A greedy iteration from a deformation holding NaN / inf / huge
    entries completes; the energy it records is not finite."""
    shape = (32, 32, 32)
    I0, I1 = greedy_pair(shape, seed=6)
    rng = np.random.default_rng(13)
    bad, _ = _plant(identity(shape), rng)
    it = GreedyIteratorB200(shape)
    it.SetScaleLevel(shape, (1.0, 1.0, 1.0), GreedyIteratorParam(DiffOperParam(0.01, 0.01, 0.001),
                                                                  0.5))
    d = GreedyDeformationDataB200(cu(I0), cu(I1))
    d.Def1To0().copy_(cu(bad))
    it.Run(d, 3, update_first=True)
    torch.cuda.synchronize()
    assert not np.isfinite(it.Energies()[0])


@pytest.mark.parametrize("shape,sp,max_pert", [((44, 42, 48), (1.0, 1.0, 1.0), 0.5),
                                               ((40, 37, 52), (1.25, 0.8, 1.0), 3.0),
                                               ((64, 64, 64), (1.0, 1.0, 1.0), 0.5)])
def test_staged_update_equals_global_gathers(shape, sp, max_pert):
    """The update with h staged in shared memory by TMA, in each of its four
    tile shapes, against the one that gathers every corner from global
    memory: bit-identical fields and energies after several iterations, on
    grids with partial edge tiles and a step large enough (MaxPert 3) that
    many corners leave the staged box."""
    from atlaswerks_b200 import _lib
    I0, I1 = greedy_pair(shape, seed=12)
    import ctypes
    L = _lib.lib()
    out = []
    # the global-gather kernel, then every staged tile shape
    for staged, tile in [(0, 0), (1, 0), (1, 1), (1, 2), (1, 3)]:
        it = GreedyIteratorB200(shape[::-1], spacing=sp)
        it.SetScaleLevel(shape[::-1], sp, GreedyIteratorParam(DiffOperParam(0.01, 0.01, 0.001),
                                                               max_pert))
        _lib.check(L.aw_greedy_set_staged_update(it._h, staged))
        t = ctypes.c_int(tile)
        _lib.check(L.aw_greedy_update_tile(it._h, 1, ctypes.byref(t)))
        d = GreedyDeformationDataB200(cu(I0), cu(I1), spacing=sp)
        it.Run(d, 5, update_first=True)
        out.append((host(d.Def1To0()).copy(), it.Energies()))
    for h, e in out[1:]:
        assert np.array_equal(h, out[0][0])
        assert np.array_equal(e, out[0][1])
    assert np.abs(out[0][0] - identity(shape)).max() > 0.5


@pytest.mark.parametrize("shape,sp,max_pert", [((64, 64, 64), (1.0, 1.0, 1.0), 0.5),
                                               ((16, 32, 128), (2.0, 1.3, 0.8), 3.0),
                                               ((128, 128, 128), (1.0, 1.0, 1.0), 0.5),
                                               ((32, 16, 16), (1.0, 1.0, 1.0), 2.0)])
def test_fused_update_equals_separate_kernels(shape, sp, max_pert):
    """The inverse transform fused with the update (v kept in the shared
    memory of a three-CTA cluster) against v stored to HBM and the update
    as a kernel of its own: bit-identical fields and energies, with large
    steps that send corners outside the volume and with anisotropic spacing."""
    from atlaswerks_b200 import _lib
    I0, I1 = greedy_pair(shape, seed=13)
    L = _lib.lib()
    out = []
    for fused in (0, 1):
        it = GreedyIteratorB200(shape[::-1], spacing=sp)
        it.SetScaleLevel(shape[::-1], sp, GreedyIteratorParam(DiffOperParam(0.01, 0.01, 0.001),
                                                               max_pert))
        _lib.check(L.aw_greedy_set_fused_update(it._h, fused))
        d = GreedyDeformationDataB200(cu(I0), cu(I1), spacing=sp)
        it.Run(d, 6, update_first=True)
        d2 = GreedyDeformationDataB200(cu(I0), cu(I1), spacing=sp)
        it.UpdateStepSizeNextIteration()
        for _ in range(3):
            it.Iterate(d2)
        out.append((host(d.Def1To0()).copy(), it.Energies(), host(d2.Def1To0()).copy()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])
    assert np.abs(out[0][0] - identity(shape)).max() > 0.1


def test_fast_interpolation_within_tolerance(oracle):
    """The float fused-multiply-add interpolation mode: a 64^3 run of 30
    iterations within 1e-3 voxel RMS of the oracle, energies (sums of
    (I1 - I0(h))^2 over the interpolated I0(h)) to 1e-4."""
    shape = (64, 64, 64)
    I0, I1 = greedy_pair(shape, seed=14, n_blobs=8, umax=3.0)
    h_o, _, e_o, _ = oracle.greedy_run(I0, I1, 30, max_pert=0.5)
    it = GreedyIteratorB200((64, 64, 64))
    it.SetScaleLevel((64, 64, 64), (1.0, 1.0, 1.0), GreedyIteratorParam(DiffOperParam(), 0.5))
    it.SetFastInterpolation(True)
    d = GreedyDeformationDataB200(cu(I0), cu(I1))
    it.Run(d, 30, update_first=True)
    dh = (host(d.Def1To0()) - h_o).astype(np.float64)
    assert float(np.sqrt((dh ** 2).sum(0).mean())) <= 1e-3
    assert np.allclose(it.Energies(), e_o, rtol=1e-4)


@pytest.mark.parametrize("shape", [(128, 128, 128), (64, 32, 16), (16, 32, 256)])
def test_register_path_z_width_result_independent(shape):
    """The register-FFT path's z pass in 16- and 8-column tiles (the width
    is chosen by timing when a plan is created): bit-identical operators."""
    import ctypes
    from atlaswerks_b200 import _lib
    L = _lib.lib()
    rng = np.random.default_rng(22)
    f = rng.normal(0, 1, (3,) + shape).astype(np.float32)
    op = DiffOperB200()
    op.SetSize(shape[::-1], (1.0, 1.3, 0.8), DiffOperParam(0.01, 0.01, 0.001))
    sh = (ctypes.c_int * 3)()
    _lib.check(L.aw_fluid_get_shapes(op._h, sh))
    assert sh[0] == 0 and sh[1] == 0 and sh[2] in (8, 16)
    outs = []
    for width in (16, 8):
        _lib.check(L.aw_fluid_set_shapes(op._h, 0, 0, width))
        for inverse in (1, 0):
            v = cu(f)
            (op.ApplyInverseOperator if inverse else op.ApplyOperator)(v)
            outs.append(host(v).copy())
    assert np.array_equal(outs[0], outs[2]) and np.array_equal(outs[1], outs[3])
    assert L.aw_fluid_set_shapes(op._h, 0, 0, 12) != 0


@pytest.mark.parametrize("shape", [(36, 31, 32), (48, 40, 44), (96, 80, 72)])
def test_fluid_shapes_autotuned_and_result_independent(shape):
    """The shared-memory FFT path picks its launch shapes by timing at plan
    creation; every legal shape gives the same bits, the register path
    reports fixed shapes, and a rejected shape leaves the plan unchanged."""
    import ctypes
    from atlaswerks_b200 import _lib
    L = _lib.lib()
    rng = np.random.default_rng(21)
    v = rng.normal(0, 1, (3,) + shape).astype(np.float32)
    op = DiffOperB200()
    op.SetSize(shape[::-1], (1.0, 1.3, 0.8), DiffOperParam(0.01, 0.01, 0.001))
    sh = (ctypes.c_int * 3)()
    _lib.check(L.aw_fluid_get_shapes(op._h, sh))
    tuned = tuple(sh)
    assert all(x >= 1 for x in tuned)
    ref = host(op.ApplyInverseOperator(cu(v)))
    for P, Q, K in [(1, 1, 1), (2, 3, 4), (tuned[0], tuned[1], 16)]:
        _lib.check(L.aw_fluid_set_shapes(op._h, P, Q, K))
        assert np.array_equal(host(op.ApplyInverseOperator(cu(v))), ref), (P, Q, K)
    assert L.aw_fluid_set_shapes(op._h, 0, 1, 1) != 0
    _lib.check(L.aw_fluid_get_shapes(op._h, sh))
    assert tuple(sh) == (tuned[0], tuned[1], 16)
    # a second plan of the grid reuses the tuned shapes
    op2 = DiffOperB200()
    op2.SetSize(shape[::-1], (1.0, 1.3, 0.8), DiffOperParam(0.01, 0.01, 0.001))
    _lib.check(L.aw_fluid_get_shapes(op2._h, sh))
    assert tuple(sh) == tuned
    # power-of-two grids: the register-FFT path's only shape, the z width
    op3 = DiffOperB200()
    op3.SetSize((32, 32, 32), (1.0, 1.0, 1.0), DiffOperParam(0.01, 0.01, 0.001))
    _lib.check(L.aw_fluid_get_shapes(op3._h, sh))
    assert tuple(sh)[:2] == (0, 0) and sh[2] in (8, 16)
