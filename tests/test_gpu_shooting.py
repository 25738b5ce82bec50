"""GPU parity of LDMM geodesic shooting (LDMMShootingIteratorB200 over
aw_ldmm_shoot_iterate) against the oracle's restatement of
LDMMShootingIteratorCPU::Iterate (itself pinned against the reference in
tests/test_oracle_pin.py).

Tolerances (four iterations): alpha0 within 1e-4 of max |alpha0|, the
maps within 1e-3 voxel, image and vector energies 1e-4 relative — the fluid solve
is FP32 on the device and FP64 in the oracle; interpolation, composition
and splatting are bit-exact operations.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from atlaswerks_b200.shooting import shoot_register  # noqa: E402
from atlaswerks_b200.synth import greedy_pair  # noqa: E402

pytestmark = pytest.mark.gpu


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.mark.parametrize("shape,sp,T", [((16, 16, 16), (1.0, 1.0, 1.0), 4),
                                        ((12, 14, 16), (1.5, 0.75, 1.25), 3),
                                        ((32, 32, 32), (1.0, 1.0, 1.0), 5)])
def test_shooting_vs_oracle(oracle, shape, sp, T):
    iters = 4
    I0, I1 = greedy_pair(shape, 7, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0), smooth_sigma=3.0)
    a = np.zeros(shape, np.float32)
    e_o, ev_o = [], []
    for _ in range(iters):
        e, ev, p0, p1 = oracle.ldmm_shoot_iterate(I0, I1, a, T, sp, sigma=1.0, step=0.05,
                                                  vec=True)
        e_o.append(e)
        ev_o.append(ev)
    from atlaswerks_b200.shooting import LDMMShootingIteratorB200
    from atlaswerks_b200.ldmm import LDMMIteratorParam
    from atlaswerks_b200.greedy import DiffOperParam
    it = LDMMShootingIteratorB200(shape[::-1], spacing=sp, n_time_steps=T)
    it.SetScaleLevel(shape[::-1], sp, LDMMIteratorParam(DiffOperParam(), 1.0, 0.05, False))
    from atlaswerks_b200.shooting import LDMMShootingDefDataB200
    data = LDMMShootingDefDataB200(cu(I0), cu(I1), sp)
    for _ in range(iters):
        it.Iterate(data)
    ag = host(data.Alpha0)
    assert np.abs(ag - a).max() <= 1e-4 * np.abs(a).max()
    assert np.abs(host(data.Phi0T) - p0).max() <= 1e-3
    assert np.abs(host(data.PhiT0) - p1).max() <= 1e-3
    assert np.allclose(it.Energies(), e_o, rtol=1e-4)
    # sum over t of <L v_t, v_t>: double sums here, float sums in the oracle
    assert np.allclose(it.VecEnergies(), ev_o, rtol=1e-4)
    assert e_o[-1] < e_o[0]


def test_shooting_converges_like_the_oracle(oracle):
    """15 iterations at 32^3 with step 0.03 (the oracle's mismatch falls
    from ~770 to ~21): the device run follows it to the end."""
    shape = (32, 32, 32)
    I0, I1 = greedy_pair(shape, 9, n_blobs=8, umax=3.0)
    a = np.zeros(shape, np.float32)
    e_o = [oracle.ldmm_shoot_iterate(I0, I1, a, 5, sigma=1.0, step=0.03)[0] for _ in range(15)]
    data, e = shoot_register(cu(I0), cu(I1), 5, 15, sigma=1.0, step=0.03)
    assert e[-1] < 0.05 * e[0]
    assert np.allclose(e, e_o, rtol=1e-3)
    assert np.abs(host(data.Alpha0) - a).max() <= 1e-3 * np.abs(a).max()


# ---- adjoint shooting (LDMMAdShootingIteratorB200 over aw_ldmm_adshoot_iterate) ----

import os  # noqa: E402

from atlaswerks_b200 import device as D  # noqa: E402
from atlaswerks_b200.greedy import DiffOperParam  # noqa: E402
from atlaswerks_b200.ldmm import LDMMIteratorParam  # noqa: E402
from atlaswerks_b200.shooting import (LDMMAdShootingIteratorB200,  # noqa: E402
                                      LDMMAdShootingWarpB200, LDMMShootingDefDataB200,
                                      LDMMShootingScaleLevel)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def adshoot_device(I0, I1, T, iters, sp, step, sigma=1.0):
    shape = I0.shape
    it = LDMMAdShootingIteratorB200(shape[::-1], spacing=sp, n_time_steps=T)
    it.SetScaleLevel(shape[::-1], sp, LDMMIteratorParam(DiffOperParam(), sigma, step, False))
    data = LDMMShootingDefDataB200(cu(I0), cu(I1), sp)
    for _ in range(iters):
        it.Iterate(data)
    torch.cuda.synchronize()
    return it, data


@pytest.mark.parametrize("shape,sp,T", [((16, 16, 16), (1.0, 1.0, 1.0), 4),
                                        ((12, 14, 16), (1.5, 0.75, 1.25), 3),
                                        ((32, 32, 32), (1.0, 1.0, 1.0), 5)])
def test_adjoint_shooting_vs_oracle(oracle, shape, sp, T):
    """Four iterations: alpha0 within 1e-4 of max |alpha0|, the maps the
    iteration leaves (time t_1) and the final maps within 1e-3 voxel, image
    and vector energies 1e-4 relative (FP32 fluid solve on the device, FP64
    in the oracle; the vector energy summed in double against float)."""
    iters, step = 4, 0.0005
    I0, I1 = greedy_pair(shape, 7, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0), smooth_sigma=3.0)
    a = np.zeros(shape, np.float32)
    ei, ev = [], []
    for _ in range(iters):
        e, v, V, q0, q1 = oracle.ldmm_adshoot_iterate(I0, I1, a, T, sp, sigma=1.0, step=step)
        ei.append(e)
        ev.append(v)
    f0, f1 = oracle.adshoot_final_maps(V, sp)
    it, data = adshoot_device(I0, I1, T, iters, sp, step)
    ag = host(data.Alpha0)
    assert np.abs(ag - a).max() <= 1e-4 * np.abs(a).max()
    assert np.abs(host(data.Phi0T) - q0).max() <= 1e-3
    assert np.abs(host(data.PhiT0) - q1).max() <= 1e-3
    assert np.allclose(it.Energies(), ei, rtol=1e-4)
    assert np.allclose(it.VecEnergies(), ev, rtol=1e-4, atol=1e-9)
    it.finalUpdatePhi0T(data)
    it.finalUpdatePhiT0(data)
    assert np.abs(host(data.Phi0T) - f0).max() <= 1e-3
    assert np.abs(host(data.PhiT0) - f1).max() <= 1e-3
    assert ei[-1] < ei[0]


def test_adjoint_shooting_vs_golden():
    """The reference's own LDMMAdShootingIteratorCPU run (tests/golden/
    adshoot_16x14x12_T4.npz: 5 iterations, T = 4, anisotropic spacing)."""
    g = np.load(os.path.join(GOLDEN, "adshoot_16x14x12_T4.npz"))
    sp = tuple(float(s) for s in g["sp"])
    it, data = adshoot_device(g["I0"], g["I1"], 4, 5, sp, 0.0002)
    it.finalUpdatePhi0T(data)
    it.finalUpdatePhiT0(data)
    assert np.abs(host(data.Alpha0) - g["alpha0"]).max() <= 1e-4 * np.abs(g["alpha0"]).max()
    assert np.abs(host(data.Phi0T) - g["phi0T"]).max() <= 1e-3
    assert np.abs(host(data.PhiT0) - g["phiT0"]).max() <= 1e-3
    assert np.allclose(it.Energies(), g["img_energy"], rtol=1e-4)
    assert np.allclose(it.VecEnergies(), g["vec_energy"], rtol=1e-4, atol=1e-9)


def test_adjoint_shooting_bullseye_regression():
    """The reference's regression LDMMAdShootingWarp on its bullseye pair
    (32x31x36, spacing (2, 2.06, 1.78); factors 2 then 1, 100 iterations
    each) through LDMMAdShootingWarpB200: the deformed image against the
    reference's Baseline by the regression's criterion (L1 sum < 1.0), and
    alpha0 against the reference build's."""
    g = np.load(os.path.join(GOLDEN, "adshoot_bullseye.npz"))
    sp = tuple(float(s) for s in g["sp"])
    warp = LDMMAdShootingWarpB200(
        cu(g["I0"]), cu(g["I1"]),
        [LDMMShootingScaleLevel(1, 100, 0.0002), LDMMShootingScaleLevel(2, 100, 0.0005)],
        n_time_steps=5, spacing=sp, sigma=1.0)
    warp.RunWarp()
    err = float(np.abs(host(warp.GetDefImage()) - g["baseline_def_image"]).sum())
    assert err < 1.0, err
    a = host(warp.GetAlpha0())
    assert np.abs(a - g["alpha0"]).max() <= 1e-3 * np.abs(g["alpha0"]).max()
    ei = np.concatenate(warp.energies)
    assert np.allclose(ei, g["img_energy"], rtol=1e-3)


@pytest.mark.parametrize("src_shape,dst_shape,ssp,dsp", [
    ((5, 6, 7), (10, 12, 14), (2.0, 2.0, 2.0), (1.0, 1.0, 1.0)),
    ((18, 15, 16), (36, 31, 32), (3.55556, 4.12904, 4.0), (1.77778, 2.06452, 2.0))])
def test_resample_image_vs_oracle(oracle, src_shape, dst_shape, ssp, dsp):
    """MultiscaleManager's image upsampling (resampleNew, clamp): bit-exact."""
    rng = np.random.default_rng(3)
    src = rng.random(src_shape, dtype=np.float32)
    ssp = tuple(float(np.float32(s)) for s in ssp)
    dsp = tuple(float(np.float32(s)) for s in dsp)
    out = host(D.resample_image(cu(src), dst_shape, ssp, dsp))
    assert np.array_equal(out, oracle.resample_image(src, dst_shape, ssp, dsp))


def test_adjoint_final_maps_before_any_iteration_fails_loudly():
    """finalUpdatePhi0T has nothing to compose before the first Iterate: the
    C ABI returns an error (raised by the host mirror) instead of copying
    unset buffers."""
    shape = (16, 16, 16)
    I0, I1 = greedy_pair(shape, 7, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0), smooth_sigma=3.0)
    it = LDMMAdShootingIteratorB200(shape[::-1], n_time_steps=3)
    it.SetScaleLevel(shape[::-1], (1.0, 1.0, 1.0),
                     LDMMIteratorParam(DiffOperParam(), 1.0, 0.0005, False))
    data = LDMMShootingDefDataB200(cu(I0), cu(I1))
    with pytest.raises(Exception, match="no adjoint shooting iteration"):
        it.finalUpdatePhi0T(data)
    it.Iterate(data)
    it.finalUpdatePhi0T(data)
    torch.cuda.synchronize()
    assert len(it.Energies()) == 1 and len(it.VecEnergies()) == 1


@pytest.mark.parametrize("sp", [(1.0, 1.0, 1.0), (1.5, 0.75, 1.25)])
@pytest.mark.parametrize("T", [1, 4])
def test_geodesic_shoot_vs_oracle(oracle, sp, T):
    """LDMMGeodesicShootingB200.ShootImage against the oracle's restatement of
    LDMMGeodesicShootingCPU::ShootImage (pinned to the reference build):
    maps within 1e-3 voxel, the final image within 1e-4 (FP32 transforms on
    both sides); a second shot from the same handle gives the same result."""
    from atlaswerks_b200.greedy import DiffOperParam
    from atlaswerks_b200.shooting import LDMMGeodesicShootingB200
    shape = (12, 14, 16)
    I0, I1 = greedy_pair(shape, 5, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0), smooth_sigma=3.0)
    alpha0 = ((I1 - I0) * 0.5).astype(np.float32)
    p0o, p1o, io = oracle.geodesic_shoot(I0, alpha0, T, sp)
    sh = LDMMGeodesicShootingB200(shape[::-1], sp, DiffOperParam())
    for _ in range(2):
        sh.ShootImage(cu(I0), cu(alpha0), T)
        assert np.abs(host(sh.GetPhi0To1()) - p0o).max() <= 1e-3
        assert np.abs(host(sh.GetPhi1To0()) - p1o).max() <= 1e-3
        assert np.abs(host(sh.GetFinalImage()) - io).max() <= 1e-4


@pytest.mark.parametrize("sp,adaptive", [((1.0, 1.0, 1.0), False), ((1.5, 0.75, 1.25), True)])
def test_velocity_shooting_vs_oracle(oracle, sp, adaptive):
    """LDMMVelShootingIteratorB200 against the oracle's restatement of
    LDMMVelShootingIteratorCPU (pinned to the reference build), three
    iterations, each from the oracle's v0: v0 within 1e-4 of max |v0|, maps
    1e-3 voxel, image energies 1e-5 and vector energies 1e-4 relative, the
    step of the step-size pass 1e-5."""
    from atlaswerks_b200.greedy import DiffOperParam
    from atlaswerks_b200.ldmm import LDMMIteratorParam
    from atlaswerks_b200.shooting import LDMMVelShootingDefDataB200, LDMMVelShootingIteratorB200
    shape, T = (12, 14, 16), 3
    I0, I1 = greedy_pair(shape, 9, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0), smooth_sigma=3.0)
    it = LDMMVelShootingIteratorB200(shape[::-1], spacing=sp, n_time_steps=T)
    it.SetScaleLevel(shape[::-1], sp, LDMMIteratorParam(DiffOperParam(), 1.0, 0.01, adaptive, 0.2))
    data = LDMMVelShootingDefDataB200(cu(I0), cu(I1), sp)
    v = np.zeros((3,) + shape, np.float32)
    step = 0.01
    if adaptive:
        _, _, step, _, _ = oracle.ldmm_velshoot_iterate(I0, I1, v, T, sp, sigma=1.0, step=step,
                                                        update_step=True, max_pert=0.2)
        it.UpdateStepSizeNextIteration()
        it.Iterate(data)
        assert abs(it.StepSize() - step) <= 1e-5 * step
        assert torch.count_nonzero(data.V0) == 0
    for k in range(3):
        e, ve, _, p0, p1 = oracle.ldmm_velshoot_iterate(I0, I1, v, T, sp, sigma=1.0, step=step)
        it.Iterate(data)
        got = host(data.V0)
        assert np.abs(got - v).max() <= 1e-4 * np.abs(v).max(), k
        assert np.abs(host(data.Phi0T) - p0).max() <= 1e-3
        assert np.abs(host(data.PhiT0) - p1).max() <= 1e-3
        assert abs(it.Energies()[-1] - e) <= 1e-5 * e
        assert abs(it.VecEnergies()[-1] - ve) <= 1e-4 * max(ve, 1e-12) or ve == 0
        data.V0.copy_(cu(v))  # re-sync to the oracle's state
