"""The oracle (C restatement, oracle/aw_oracle.c) against the reference's own
CPU code built from its sources (oracle/_ref): CPU only.

Interpolation, gradient, compose and splat must agree bit for bit; the fluid
operator to FP64 rounding of float-valued parameters; greedy and LDMM
iterations to the FP32 rounding of the reference's FFT.
"""
import numpy as np
import pytest

from atlaswerks_b200.synth import greedy_pair
from oracle import BG_PARTIAL_ID, identity

SHAPES = [(12, 11, 10), (8, 9, 17), (16, 16, 16)]
SP = (1.0, 1.3, 0.8)


@pytest.mark.parametrize("shape", SHAPES)
def test_interpolation_family_bit_exact(oracle, reference, shape):
    rng = np.random.default_rng(0)
    img = rng.random(shape, dtype=np.float32)
    h = identity(shape) + rng.normal(0, 1.5, (3,) + shape).astype(np.float32)
    v = rng.normal(0, 1.0, (3,) + shape).astype(np.float32)
    assert np.array_equal(oracle.apply(img, h), reference.apply(img, h))
    for wrap in (False, True):
        assert np.array_equal(oracle.gradient(img, SP, wrap), reference.gradient(img, SP, wrap))
    for bg in range(6):
        for d in (1, -1):
            assert np.array_equal(oracle.compose_hv(h, v, SP, d, bg),
                                  reference.compose_hv(h, v, SP, d, bg))
            assert np.array_equal(oracle.compose_vh(v, h, SP, d, bg),
                                  reference.compose_vh(v, h, SP, d, bg))
    assert np.array_equal(oracle.splat(img, h), reference.splat(img, h))


@pytest.mark.parametrize("inverse", [True, False])
def test_fluid_fp64_matches_reference_fp64(oracle, reference, inverse):
    rng = np.random.default_rng(1)
    f = rng.normal(0, 1, (3, 12, 11, 10)).astype(np.float32)
    # the reference holds alpha, beta, gamma as float (Real)
    a, b, g = (float(np.float32(x)) for x in (0.01, 0.01, 0.001))
    want = reference.fluid_f64(f, SP, a, b, g, inverse)
    got = oracle.fluid_f64(f, SP, a, b, g, inverse)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    # the reference's FP32 operator (FFT in FP64 through the shim, solve in FP32)
    w32 = reference.fluid(f, SP, a, b, g, inverse)
    assert np.abs(w32 - want).max() <= 1e-6 * np.abs(want).max()


def test_greedy_iterations_match_reference(oracle, reference):
    shape = (24, 20, 16)
    I0, I1 = greedy_pair(shape, 1, n_blobs=4, umax=2.0)
    hr, hir, er, sr = reference.greedy_run(I0, I1, [1], [10], [0.5], inverse=True)
    ho, hio, eo, so = oracle.greedy_run(I0, I1, 10, max_pert=0.5, inverse=True)
    assert np.abs(ho - hr).max() <= 1e-5
    assert abs(sr[-1] - so) <= 1e-6 * so
    assert np.allclose(eo, er, rtol=1e-5)
    # the inverse field agrees except where the reference interpolates v in
    # the padded FFTW array (x >= nx - 1; see the restatement's notes)
    m = hio[0] < shape[2] - 1.0
    assert np.abs(hio - hir)[:, m].max() <= 1e-5


def test_ldmm_iterations_match_reference(oracle, reference):
    shape, T = (16, 14, 12), 4
    I0, I1 = greedy_pair(shape, 3, n_blobs=4, umax=2.0)
    vr, er, _ = reference.ldmm_run(I0, I1, T, 3, sigma=1.0, step=0.01)
    v = np.zeros((T, 3) + shape, np.float32)
    eo = [oracle.ldmm_iterate(I0, I1, v, sigma=1.0, step=0.01)[0] for _ in range(3)]
    assert np.abs(v - vr).max() <= 1e-5 * np.abs(vr).max()
    assert np.allclose(eo, er, rtol=1e-5)


def test_ldmm_adaptive_step_matches_reference(oracle, reference):
    shape, T = (16, 14, 12), 4
    I0, I1 = greedy_pair(shape, 3, n_blobs=4, umax=2.0)
    _, _, sr = reference.ldmm_run(I0, I1, T, 1, sigma=0.1, step=0.005, adaptive=True,
                                  max_pert=0.1)
    v = np.zeros((T, 3) + shape, np.float32)
    _, so = oracle.ldmm_iterate(I0, I1, v, sigma=0.1, step=0.005, update_step=True, max_pert=0.1)
    assert abs(so - sr) <= 1e-5 * sr


def test_ldmm_orig_iterations_match_reference(oracle, reference):
    """IterateOrig (Jacobian transport), anisotropic spacing, against the
    reference's LDMMIteratorCPU with UseOrigGradientCalc."""
    shape, T = (12, 14, 16), 4
    I0, I1 = greedy_pair(shape, 3, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0), smooth_sigma=3.0)
    sp = (1.5, 0.75, 1.25)
    vr, er, _ = reference.ldmm_run(I0, I1, T, 3, sp=sp, sigma=1.0, step=0.01, use_new=False)
    v = np.zeros((T, 3) + shape, np.float32)
    eo = [oracle.ldmm_iterate_orig(I0, I1, v, sp, sigma=1.0, step=0.01)[0] for _ in range(3)]
    assert np.abs(v - vr).max() <= 1e-5 * np.abs(vr).max()
    assert np.allclose(eo, er, rtol=1e-5)


def test_jacobian_of_identity_map_is_spacing_volume(oracle):
    v = np.zeros((3, 6, 7, 8), np.float32)
    jac = oracle.jacobian(v, (1.5, 0.75, 1.25))
    assert np.allclose(jac, 1.0)  # d(x*sp)/dx / sp = 1 per axis


def test_ldmm_i1_at_0_matches_reference(oracle, reference):
    """GetI1At0 and ComputeJacDet for nonzero velocities (from three LDMM
    iterations), anisotropic spacing: the restatement against the
    reference's LDMMDeformationData / LDMMIteratorCPU."""
    shape, T = (12, 14, 16), 4
    sp = (1.5, 0.75, 1.25)
    I0, I1 = greedy_pair(shape, 5, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0), smooth_sigma=3.0)
    v, _, _ = reference.ldmm_run(I0, I1, T, 3, sp=sp, sigma=1.0, step=0.01)
    img_r, jd_r = reference.ldmm_i1_at_0(I1, v, sp)
    img_o, jd_o = oracle.ldmm_i1_at_0(I1, v, sp)
    assert np.array_equal(img_o, img_r)
    assert np.array_equal(jd_o, jd_r)
    assert np.abs(jd_o - 1.0).max() > 1e-3  # the velocities are not trivial


@pytest.mark.parametrize("use_new,jacobian_scale,adaptive", [(True, True, False),
                                                              (False, True, True),
                                                              (True, False, False)])
def test_ldmm_atlas_matches_reference(oracle, reference, use_new, jacobian_scale, adaptive):
    """Three subjects, three atlas iterations of LDMM relaxation (IterateNew
    or IterateOrig, with or without JacobianScale, fixed or adaptive step):
    the restated loop against the reference's classes driven through the
    AtlasThreadMain loop."""
    shape, T = (12, 12, 12), 3
    imgs = [greedy_pair(shape, 40 + k, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0),
                        smooth_sigma=3.0)[1] for k in range(3)]
    w = [0.5, 0.3, 0.2]
    kw = dict(sigma=1.0, step=0.01, adaptive=adaptive, max_pert=0.2, use_new=use_new,
              jacobian_scale=jacobian_scale)
    mr, vr, er = reference.ldmm_atlas_run(imgs, w, T, 3, **kw)
    mo, vo, eo = oracle.ldmm_atlas_run(imgs, w, T, 3, **kw)
    assert np.abs(mo - mr).max() <= 1e-5 * np.abs(mr).max()
    for a, b in zip(vo, vr):
        assert np.abs(a - b).max() <= 1e-4 * max(np.abs(b).max(), 1e-12)
    assert np.allclose(eo, er, rtol=1e-4)
    assert np.abs(vr[0]).max() > 0


@pytest.mark.parametrize("sp", [(1.0, 1.0, 1.0), (1.5, 0.75, 1.25)])
def test_ldmm_shooting_matches_reference(oracle, reference, sp):
    """Geodesic shooting from the initial momentum, four iterations from
    alpha0 = 0: the restatement against LDMMShootingIteratorCPU."""
    shape, T, iters = (12, 14, 16), 4, 4
    I0, I1 = greedy_pair(shape, 7, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0), smooth_sigma=3.0)
    a_r, p0_r, p1_r, e_r, ev_r = reference.shoot_run(I0, I1, T, iters, sp=sp, sigma=1.0,
                                                     step=0.05, vec=True)
    a = np.zeros(shape, np.float32)
    e_o, ev_o = [], []
    for _ in range(iters):
        e, ev, p0, p1 = oracle.ldmm_shoot_iterate(I0, I1, a, T, sp, sigma=1.0, step=0.05,
                                                  vec=True)
        e_o.append(e)
        ev_o.append(ev)
    # the vector energies: sum over t of <L v_t, v_t> (LDMMEnergy's step energies)
    assert np.allclose(ev_o, ev_r, rtol=1e-5, atol=1e-9)
    # the oracle's FP64 fluid solve vs the reference's FP32 one
    assert np.abs(a - a_r).max() <= 1e-5 * np.abs(a_r).max()
    assert np.abs(p0 - p0_r).max() <= 1e-4
    assert np.abs(p1 - p1_r).max() <= 1e-4
    assert np.allclose(e_o, e_r, rtol=1e-5)
    assert e_r[-1] < e_r[0]  # the shooting lowers the mismatch


@pytest.mark.parametrize("sp", [(1.0, 1.0, 1.0), (1.5, 0.75, 1.25)])
def test_ldmm_adjoint_shooting_matches_reference(oracle, reference, sp):
    """Adjoint geodesic shooting, four iterations from alpha0 = 0: the
    restatement of Iterate + backwardAdIntegration and of the final maps
    against LDMMAdShootingIteratorCPU."""
    shape, T, iters = (12, 14, 16), 4, 4
    I0, I1 = greedy_pair(shape, 7, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0), smooth_sigma=3.0)
    a_r, p0_r, p1_r, ei_r, ev_r = reference.adshoot_run(I0, I1, T, [(1, iters, 0.0005)], sp,
                                                        sigma=1.0)
    a = np.zeros(shape, np.float32)
    ei, ev = [], []
    for _ in range(iters):
        e, v, V, _, _ = oracle.ldmm_adshoot_iterate(I0, I1, a, T, sp, sigma=1.0, step=0.0005)
        ei.append(e)
        ev.append(v)
    p0, p1 = oracle.adshoot_final_maps(V, sp)
    # the oracle's FP64 fluid solve vs the reference's FP32 one
    assert np.abs(a - a_r).max() <= 1e-5 * np.abs(a_r).max()
    assert np.abs(p0 - p0_r).max() <= 1e-4
    assert np.abs(p1 - p1_r).max() <= 1e-4
    assert np.allclose(ei, ei_r, rtol=1e-5)
    assert np.allclose(ev, ev_r, rtol=1e-5, atol=1e-9)
    assert ei_r[-1] < ei_r[0]


def test_ldmm_adjoint_shooting_two_scales_matches_reference(oracle, reference):
    """The LDMMWarpAd scale loop at 20x18x24, factors 2 then 1: downsampled
    images, alpha0 resampled by resampleNew at the scale change."""
    shape = (24, 18, 20)
    sp = (1.0, 1.25, 0.8)
    I0, I1 = greedy_pair(shape, 12, n_blobs=6, umax=1.5, sigma_range=(2.0, 3.0), smooth_sigma=3.0)
    levels = [(1, 3, 0.0002), (2, 4, 0.0005)]
    a_r, p0_r, p1_r, ei_r, ev_r = reference.adshoot_run(I0, I1, 3, levels, sp, sigma=1.0)
    a, p0, p1, hist = oracle.adshoot_warp(I0, I1, 3, levels, sp, sigma=1.0)
    assert np.abs(a - a_r).max() <= 1e-5 * np.abs(a_r).max()
    assert np.abs(p0 - p0_r).max() <= 1e-4
    assert np.abs(p1 - p1_r).max() <= 1e-4
    ei = np.concatenate([h[0] for h in hist])
    assert np.allclose(ei, ei_r, rtol=1e-5)


def _median_cases():
    """Image stacks for MedianCalculator::Select: random values, exact ties,
    and a volume whose range (one voxel at 1e4) makes eps = 1, so voxels
    whose values lie within 1 end at their interval's lower end, not at the
    k-th value."""
    rng = np.random.default_rng(8)
    shape = (5, 6, 7)
    cases = []
    for n in (1, 2, 3, 4, 6, 9):
        imgs = [rng.normal(0, 1, shape).astype(np.float32) for _ in range(n)]
        if n > 2:
            imgs[1][0] = imgs[0][0]  # ties across images
        cases.append(imgs)
    imgs = [np.full(shape, 0.1 * (m + 1), np.float32) for m in range(5)]
    imgs[0][0, 0, 0] = 1e4
    cases.append(imgs)
    return cases


def test_voxel_median_matches_reference(oracle, reference):
    for imgs in _median_cases():
        k = oracle.median_index(len(imgs))
        got = oracle.voxel_median(imgs, k)
        assert np.array_equal(got, reference.voxel_median(imgs, k))
    # the eps rule: 0.1 .. 0.5 lie within eps = 1 of each other, so the
    # selection ends at the lower end 0.1 instead of the median 0.3
    assert got[1, 1, 1] == np.float32(0.1)


def test_voxel_median_not_converging_matches_reference(oracle, reference):
    # one constant volume: eps = 0 and no bisection separates the values,
    # so the reference throws for any k > 0, and the oracle reports it
    imgs = [np.full((3, 3, 3), 2.0, np.float32) for _ in range(3)]
    with pytest.raises(RuntimeError):
        reference.voxel_median(imgs, 1)
    with pytest.raises(RuntimeError):
        oracle.voxel_median(imgs, 1)
    assert np.array_equal(oracle.voxel_median(imgs, 0), reference.voxel_median(imgs, 0))


def test_voxel_median_rejects_empty_inputs_and_bad_index(oracle):
    """The restatement refuses no images, no voxels and k outside [0, n)
    before it reads anything."""
    imgs = [np.full((2, 2, 2), v, np.float32) for v in (0.1, 0.2, 0.3)]
    for k in (-1, 3):
        with pytest.raises(ValueError):
            oracle.voxel_median(imgs, k)
    with pytest.raises(ValueError):
        oracle.voxel_median([np.zeros((0, 2, 2), np.float32)] * 3, 1)


@pytest.mark.parametrize("use_new", [True, False])
def test_ldmm_vector_energies_match_reference(oracle, reference, use_new):
    """The debug-mode vector energy sum_t <L v_t, v_t> sp^3 of the updated
    velocities, IterateNew and IterateOrig, against the reference's
    LDMMEnergy::VecEnergy() * T (the reference sums each step's products in
    float, hence the tolerance)."""
    shape, T = (12, 14, 16), 4
    I0, I1 = greedy_pair(shape, 3, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0), smooth_sigma=3.0)
    sp = (1.5, 0.75, 1.25)
    ven = np.zeros(3)
    reference.ldmm_run(I0, I1, T, 3, sp=sp, sigma=1.0, step=0.01, use_new=use_new, vec_out=ven)
    v = np.zeros((T, 3) + shape, np.float32)
    it = oracle.ldmm_iterate if use_new else oracle.ldmm_iterate_orig
    vo = [it(I0, I1, v, sp, sigma=1.0, step=0.01, vec=True)[2] for _ in range(3)]
    assert np.all(ven > 0)
    assert np.allclose(vo, ven, rtol=1e-4)


@pytest.mark.parametrize("sp", [(1.0, 1.0, 1.0), (1.5, 0.75, 1.25)])
def test_geodesic_shoot_matches_reference(oracle, reference, sp):
    """LDMMGeodesicShootingCPU::ShootImage(I0, alpha0, T): the oracle's
    restatement against the reference build, maps to 1e-4 voxel and the
    final image to 1e-5 (the FFT shim's rounding through T transforms)."""
    shape, T = (12, 14, 16), 4
    I0, I1 = greedy_pair(shape, 5, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0), smooth_sigma=3.0)
    alpha0 = ((I1 - I0) * 0.5).astype(np.float32)
    p0o, p1o, io = oracle.geodesic_shoot(I0, alpha0, T, sp)
    p0r, p1r, ir = reference.geodesic_shoot(I0, alpha0, T, sp)
    assert np.abs(p0o - p0r).max() <= 1e-4
    assert np.abs(p1o - p1r).max() <= 1e-4
    assert np.abs(io - ir).max() <= 1e-5
    assert np.abs(p1r - identity(shape)).max() > 0.01  # the geodesic moved


@pytest.mark.parametrize("sp,adaptive", [((1.0, 1.0, 1.0), False), ((1.5, 0.75, 1.25), True)])
def test_velocity_shooting_matches_reference(oracle, reference, sp, adaptive):
    """LDMMVelShootingIteratorCPU: the oracle's restatement against the
    reference build over three iterations (the step-size pass first when
    adaptive): v0 1e-5 of max, maps 1e-4, image energies 1e-5, vector
    energies 1e-4 (the reference sums each step's products in float)."""
    shape, T = (12, 14, 16), 3
    I0, I1 = greedy_pair(shape, 9, n_blobs=4, umax=1.5, sigma_range=(1.5, 3.0), smooth_sigma=3.0)
    kw = dict(sigma=1.0, step=0.01, max_pert=0.2)
    vr, p0r, p1r, er, ver, sr = reference.velshoot_run(I0, I1, T, 3, sp, adaptive=adaptive, **kw)
    v = np.zeros((3,) + shape, np.float32)
    step = kw["step"]
    if adaptive:
        _, _, step, _, _ = oracle.ldmm_velshoot_iterate(I0, I1, v, T, sp, sigma=1.0, step=step,
                                                        update_step=True, max_pert=0.2)
        assert abs(step - sr) <= 1e-5 * sr
    eo, veo = [], []
    for _ in range(3):
        e, ve, _, p0, p1 = oracle.ldmm_velshoot_iterate(I0, I1, v, T, sp, sigma=1.0, step=step)
        eo.append(e)
        veo.append(ve)
    assert np.abs(v - vr).max() <= 1e-5 * np.abs(vr).max()
    assert np.abs(p0 - p0r).max() <= 1e-4 and np.abs(p1 - p1r).max() <= 1e-4
    assert np.allclose(eo, er, rtol=1e-5)
    assert np.allclose(veo, ver, rtol=1e-4)
    assert np.abs(vr).max() > 0 and eo[-1] < eo[0]
