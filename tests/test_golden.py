"""The oracle against the golden fixtures in tests/golden/ — outputs of the
reference's own CPU code (compiled from its sources; tests/golden/
make_golden.py made them). These run anywhere, without the reference tree.

Tolerances: interpolation family, gradient, splat, downsample, upsample:
bit-exact. Fluid operator: the oracle's FP64 solve vs the reference's FP32
one, 1e-5 of the field's maximum (the FP64 golden to 1e-12). Greedy, LDMM
and atlas runs: 1e-4 voxel (fields) and 1e-5 relative (energies), the FP32
rounding of the reference's transforms carried through the iterations.
"""
import os

import numpy as np
import pytest

from oracle import identity

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BG = ["partial_id", "id", "partial_zero", "zero", "clamp", "wrap"]


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def test_interpolation_family(oracle):
    z = load("interp_9x13x11")
    img, h, v, sp = z["img"], z["h"], z["v"], tuple(z["sp"])
    assert np.array_equal(oracle.apply(img, h), z["apply"])
    assert np.array_equal(oracle.gradient(img, sp, False), z["gradient"])
    assert np.array_equal(oracle.gradient(img, sp, True), z["gradient_wrap"])
    assert np.array_equal(oracle.splat(img, h), z["splat"])
    for b, name in enumerate(BG):
        assert np.array_equal(oracle.compose_hv(h, v, sp, 1, b), z["compose_hv_" + name]), name
        assert np.array_equal(oracle.compose_hv(h, v, sp, -1, b), z["compose_hvinv_" + name]), name
        assert np.array_equal(oracle.compose_vh(v, h, sp, -1, b), z["compose_vhinv_" + name]), name


def test_fluid_operator(oracle):
    z = load("fluid_16x12x20")
    f, sp = z["f"], tuple(z["sp"])
    # the reference holds alpha, beta, gamma as float (Real)
    a, b, g = (float(np.float32(z[k])) for k in ("alpha", "beta", "gamma"))
    inv = oracle.fluid(f, sp, a, b, g, True)
    assert np.abs(inv - z["inverse"]).max() <= 1e-5 * np.abs(z["inverse"]).max()
    fwd = oracle.fluid(f, sp, a, b, g, False)
    assert np.abs(fwd - z["forward"]).max() <= 1e-5 * np.abs(z["forward"]).max()
    inv64 = oracle.fluid_f64(f, sp, a, b, g, True)
    assert np.abs(inv64 - z["inverse_f64"]).max() <= 1e-12 * np.abs(z["inverse_f64"]).max()


def test_greedy_single_scale(oracle):
    z = load("greedy_16")
    h, hinv, en, step = oracle.greedy_run(z["I0"], z["I1"], len(z["energies"]), inverse=True)
    assert np.abs(h - z["h"]).max() <= 1e-4
    assert np.abs(hinv - z["hinv"]).max() <= 1e-4
    assert np.allclose(en, z["energies"], rtol=1e-5)
    assert abs(step - z["steps"][-1]) <= 1e-6 * z["steps"][-1]


def test_greedy_two_scales(oracle):
    z = load("greedy_24_two_scales")
    h, _, en = oracle.greedy_warp(z["I0"], z["I1"], [(2, 10, 0.5), (1, 6, 0.5)])
    assert np.abs(h - z["h"]).max() <= 1e-4
    assert np.allclose(np.concatenate(en), z["energies"], rtol=1e-5)


def test_multiscale_resampling(oracle):
    z = load("downsample_16x20x24")
    assert np.array_equal(oracle.downsample(z["img"], (12, 10, 8)), z["half"])
    z = load("upsample_12x10x8")
    assert np.array_equal(oracle.upsample_hfield(z["h"], (16, 20, 24), True), z["up"])
    assert np.array_equal(oracle.upsample_hfield(z["h"], (16, 20, 24), False), z["up_norescale"])


@pytest.mark.parametrize("adaptive", [False, True])
def test_ldmm_iterate_new(oracle, adaptive):
    z = load("ldmm_16_T4")
    sfx = "_adaptive" if adaptive else ""
    want_v, want_e = z["v" + sfx], z["energies" + sfx]
    v = np.zeros_like(want_v)
    step, en = 0.01, []
    if adaptive:
        # LDMMWarp: a step-size pass (v unchanged, no energy) before iteration 0
        _, step = oracle.ldmm_iterate(z["I0"], z["I1"], v, sigma=1.0, step=step,
                                      update_step=True, max_pert=0.2)
    for it in range(len(want_e)):
        e, step = oracle.ldmm_iterate(z["I0"], z["I1"], v, sigma=1.0, step=step)
        en.append(e)
    assert np.abs(v - want_v).max() <= 1e-4 * np.abs(want_v).max()
    assert np.allclose(en, want_e, rtol=1e-5)
    assert abs(step - float(z["step" + sfx])) <= 1e-6 * float(z["step" + sfx])


@pytest.mark.parametrize("adaptive", [False, True])
def test_ldmm_iterate_orig(oracle, adaptive):
    z = load("ldmm_orig_16x14x12_T4")
    sfx = "_adaptive" if adaptive else ""
    want_v, want_e, sp = z["v" + sfx], z["energies" + sfx], tuple(z["sp"])
    v = np.zeros_like(want_v)
    step, en = 0.01, []
    if adaptive:
        _, step = oracle.ldmm_iterate_orig(z["I0"], z["I1"], v, sp, sigma=1.0, step=step,
                                           update_step=True, max_pert=0.2)
    for it in range(len(want_e)):
        e, step = oracle.ldmm_iterate_orig(z["I0"], z["I1"], v, sp, sigma=1.0, step=step)
        en.append(e)
    assert np.abs(v - want_v).max() <= 1e-5 * np.abs(want_v).max()
    # the reference's energy: float sum of squares
    assert np.allclose(en, want_e, rtol=1e-5)
    assert abs(step - float(z["step" + sfx])) <= 1e-6 * float(z["step" + sfx])


@pytest.mark.parametrize("period", [1, 2])
def test_atlas(oracle, period):
    z = load("atlas_16x3")
    imgs = [a for a in z["imgs"]]
    mean, hs, en, _ = oracle.atlas_run(imgs, list(z["w"]), (16, 16, 16), 6, period)
    assert np.abs(mean - z[f"mean_p{period}"]).max() <= 1e-5
    assert np.abs(np.stack(hs) - z[f"h_p{period}"]).max() <= 1e-4
    assert np.allclose(en, z[f"energies_p{period}"], rtol=1e-5)


def test_identity_helper():
    h = identity((2, 3, 4))
    assert h.shape == (3, 2, 3, 4) and h[0, 1, 2, 3] == 3 and h[1, 1, 2, 3] == 2 and h[2, 1, 2, 3] == 1


def test_adshoot_single_scale(oracle):
    """LDMM adjoint shooting, 5 iterations at 12x14x16, T = 4, anisotropic
    spacing: the oracle's Iterate and final maps against the reference's
    LDMMAdShootingIteratorCPU through the LDMMWarpAd loop."""
    g = load("adshoot_16x14x12_T4")
    sp = tuple(g["sp"])
    a = np.zeros(g["I0"].shape, np.float32)
    ei, ev = [], []
    for _ in range(5):
        e, v, V, _, _ = oracle.ldmm_adshoot_iterate(g["I0"], g["I1"], a, 4, sp, sigma=1.0,
                                                    step=0.0002)
        ei.append(e)
        ev.append(v)
    p0, p1 = oracle.adshoot_final_maps(V, sp)
    assert np.abs(a - g["alpha0"]).max() <= 1e-5 * np.abs(g["alpha0"]).max()
    assert np.abs(p0 - g["phi0T"]).max() <= 1e-4
    assert np.abs(p1 - g["phiT0"]).max() <= 1e-4
    assert np.allclose(ei, g["img_energy"], rtol=1e-5)
    assert np.allclose(ev, g["vec_energy"], rtol=1e-5, atol=1e-9)
    assert ei[-1] < 0.5 * ei[0]


def test_adshoot_bullseye_fixture_is_the_reference_regression(oracle):
    """The fixture's reference-build result reproduces the reference's own
    regression baseline (LDMMAdShootingWarp Baseline DefImage) by the
    regression's criterion, L1 sum below 1.0 (AtlasWerksTestUtils.py:
    122-168)."""
    g = load("adshoot_bullseye")
    err = float(np.abs(oracle.apply(g["I0"], g["phiT0"]) - g["baseline_def_image"]).sum())
    assert err < 1.0, err
    assert err < 0.02, err  # measured 0.0040


def test_resample_image_is_clamped_trilinear(oracle):
    """resampleNew of a linear ramp onto a grid twice as fine reproduces the
    ramp inside and clamps to the edge values outside."""
    src = np.fromfunction(lambda z, y, x: x + 2 * y + 3 * z, (5, 6, 7), dtype=np.float32)
    out = oracle.resample_image(src, (10, 12, 14), (2.0, 2.0, 2.0), (1.0, 1.0, 1.0))
    z, y, x = np.meshgrid(*[np.clip(np.arange(n) / 2.0 - 0.25, 0, m - 1)
                            for n, m in ((10, 5), (12, 6), (14, 7))], indexing="ij")
    assert np.abs(out - (x + 2 * y + 3 * z)).max() < 1e-5


def test_adshoot_bullseye_regression(oracle):
    """The oracle's LDMMWarpAd loop on the reference's regression pair
    (factors 2 then 1, 100 iterations each, T = 5): the deformed image
    against the reference's Baseline by the regression's criterion, alpha0
    against the reference build's (about a minute on one core)."""
    g = load("adshoot_bullseye")
    sp = tuple(float(s) for s in g["sp"])
    a, _, p1, hist = oracle.adshoot_warp(g["I0"], g["I1"], 5, [(1, 100, 0.0002), (2, 100, 0.0005)],
                                         sp, sigma=1.0)
    err = float(np.abs(oracle.apply(g["I0"], p1) - g["baseline_def_image"]).sum())
    assert err < 1.0, err
    assert err < 0.02, err  # measured 0.0041
    assert np.abs(a - g["alpha0"]).max() <= 1e-5 * np.abs(g["alpha0"]).max()
    # the reference keeps the image energy as a float: 3e-5 relative
    assert np.allclose(np.concatenate([h[0] for h in hist]), g["img_energy"], rtol=3e-5)
