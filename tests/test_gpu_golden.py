"""The CUDA path against the golden fixtures in tests/golden/ — outputs of
the reference's own CPU code (tests/golden/make_golden.py). No oracle in the
loop: the C ABI's results against the reference's on the same inputs.

Tolerances: interpolation family, gradient, splat, downsample, upsample:
bit-exact. Fluid operator: max |gpu - ref| <= 1e-5 of max |ref| against the
reference's FP32 path and against its FP64 path. Registration runs (greedy,
LDMM, atlas): deformation fields within 1e-3 voxel max, energies within
1e-4 relative — FP32 transforms on both sides, rounded differently.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from atlaswerks_b200 import device as D  # noqa: E402
from atlaswerks_b200.atlas import GreedyAtlasBuilderB200, GreedyAtlasParam  # noqa: E402
from atlaswerks_b200.greedy import DiffOperB200, DiffOperParam, greedy_register  # noqa: E402
from atlaswerks_b200.ldmm import ldmm_register  # noqa: E402
from atlaswerks_b200.multiscale import GreedyWarpB200, ScaleLevel  # noqa: E402

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BG = ["partial_id", "id", "partial_zero", "zero", "clamp", "wrap"]


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def test_interpolation_family():
    z = load("interp_9x13x11")
    img, h, v, sp = cu(z["img"]), cu(z["h"]), cu(z["v"]), tuple(z["sp"])
    assert np.array_equal(host(D.apply(img, h)), z["apply"])
    assert np.array_equal(host(D.gradient(img, sp, False)), z["gradient"])
    assert np.array_equal(host(D.gradient(img, sp, True)), z["gradient_wrap"])
    assert np.array_equal(host(D.splat(img, h)), z["splat"])
    for b, name in enumerate(BG):
        assert np.array_equal(host(D.compose_hv(h, v, sp, 1.0, 1, b)), z["compose_hv_" + name])
        assert np.array_equal(host(D.compose_hv(h, v, sp, 1.0, -1, b)), z["compose_hvinv_" + name])
        assert np.array_equal(host(D.compose_vh(v, h, sp, 1.0, -1, b)), z["compose_vhinv_" + name])


def test_fluid_operator():
    z = load("fluid_16x12x20")
    sp = tuple(z["sp"])
    op = DiffOperB200()
    op.SetSize((16, 12, 20), sp, DiffOperParam(float(z["alpha"]), float(z["beta"]),
                                               float(z["gamma"])))
    got = host(op.ApplyInverseOperator(cu(z["f"])))
    for want in (z["inverse"], z["inverse_f64"]):
        assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()
    got = host(op.ApplyOperator(cu(z["f"])))
    assert np.abs(got - z["forward"]).max() <= 1e-5 * np.abs(z["forward"]).max()


def test_greedy_single_scale():
    z = load("greedy_16")
    h, hinv, en, step = greedy_register(cu(z["I0"]), cu(z["I1"]), len(z["energies"]),
                                        compute_inverse=True)
    assert np.abs(host(h) - z["h"]).max() <= 1e-3
    assert np.abs(host(hinv) - z["hinv"]).max() <= 1e-3
    assert np.allclose(en, z["energies"], rtol=1e-4)
    assert abs(step - z["steps"][-1]) <= 1e-5 * z["steps"][-1]


def test_greedy_two_scales():
    z = load("greedy_24_two_scales")
    w = GreedyWarpB200(cu(z["I0"]), cu(z["I1"]), [ScaleLevel(2, 10, 0.5), ScaleLevel(1, 6, 0.5)])
    h, _ = w.RunWarp()
    assert np.abs(host(h) - z["h"]).max() <= 1e-3
    assert np.allclose(np.concatenate(w.energies), z["energies"], rtol=1e-4)


def test_multiscale_resampling():
    z = load("downsample_16x20x24")
    assert np.array_equal(host(D.downsample(cu(z["img"]), (12, 10, 8))), z["half"])
    z = load("upsample_12x10x8")
    assert np.array_equal(host(D.upsample_hfield(cu(z["h"]), (16, 20, 24), True)), z["up"])
    assert np.array_equal(host(D.upsample_hfield(cu(z["h"]), (16, 20, 24), False)),
                          z["up_norescale"])


@pytest.mark.parametrize("adaptive", [False, True])
def test_ldmm_iterate_new(adaptive):
    z = load("ldmm_16_T4")
    sfx = "_adaptive" if adaptive else ""
    want_v, want_e = z["v" + sfx], z["energies" + sfx]
    v, en, step = ldmm_register(cu(z["I0"]), cu(z["I1"]), 4, len(want_e), sigma=1.0, step=0.01,
                                adaptive=adaptive, max_pert=0.2)
    assert np.abs(host(v) - want_v).max() <= 1e-3 * np.abs(want_v).max()
    assert np.allclose(en, want_e, rtol=1e-4)
    assert abs(step - float(z["step" + sfx])) <= 1e-5 * float(z["step" + sfx])


@pytest.mark.parametrize("adaptive", [False, True])
def test_ldmm_iterate_orig(adaptive):
    z = load("ldmm_orig_16x14x12_T4")
    sfx = "_adaptive" if adaptive else ""
    want_v, want_e = z["v" + sfx], z["energies" + sfx]
    v, en, step = ldmm_register(cu(z["I0"]), cu(z["I1"]), 4, len(want_e), tuple(z["sp"]),
                                sigma=1.0, step=0.01, adaptive=adaptive, max_pert=0.2,
                                orig_gradient=True)
    assert np.abs(host(v) - want_v).max() <= 1e-3 * np.abs(want_v).max()
    assert np.allclose(en, want_e, rtol=1e-4)
    assert abs(step - float(z["step" + sfx])) <= 1e-5 * float(z["step" + sfx])


@pytest.mark.parametrize("period", [1, 2])
def test_atlas(period):
    z = load("atlas_16x3")
    imgs = [cu(a) for a in z["imgs"]]
    b = GreedyAtlasBuilderB200(imgs, (16, 16, 16), GreedyAtlasParam(DiffOperParam(), 0.5, 6,
                                                                     period),
                               weights=list(z["w"]))
    mean = host(b.BuildAtlas())
    assert np.abs(mean - z[f"mean_p{period}"]).max() <= 1e-4
    for i in range(3):
        assert np.abs(host(b.GetDeformationField(i)) - z[f"h_p{period}"][i]).max() <= 1e-3
        assert np.allclose(b.GetEnergies(i), z[f"energies_p{period}"][:, i], rtol=1e-4)


@pytest.mark.parametrize("fast", [False, True], ids=["exact", "fast_interp"])
def test_greedy_bullseye_regression_on_device(tmp_path, fast):
    """The reference's own greedy regression (Testing/Applications/Greedy/
    GreedyWarp, GreedyWarpParams.xml) through GreedyWarpB200: the bullseye
    pair rescaled to [0, 1] at its anisotropic spacing, scale factors 2 and
    1 with 50 iterations each, MaxPert 0.3, the inverse field computed. The
    deformed image against the regression's Baseline by its criterion (L1
    sum < 1.0); the fields against the reference build's run on the same
    inputs (1e-3 voxel RMS); the DefImage written as MetaImage reads back."""
    from atlaswerks_b200.metaimage import read_mha
    z = load("greedy_bullseye")
    sp = tuple(float(s) for s in z["sp"])
    w = GreedyWarpB200(cu(z["I0"]), cu(z["I1"]), [ScaleLevel(2, 50, 0.3), ScaleLevel(1, 50, 0.3)],
                       sp, compute_inverse=True, fast_interpolation=fast)
    h, hinv = w.RunWarp()
    err = float(np.abs(host(D.apply(cu(z["I0"]), h)) - z["baseline_def_image"]).sum())
    assert err < 1.0, err
    for got, want in ((host(h), z["h"]), (host(hinv), z["hinv"])):
        d = (got - want).astype(np.float64)
        assert np.sqrt((d * d).sum(0).mean()) <= 1e-3
    files = w.GenerateOutput(str(tmp_path / "GreedyBullseye"), h, hinv)
    assert len(files) == 4
    img, rsp = read_mha(files[0])
    assert np.array_equal(img, host(D.apply(cu(z["I0"]), h)))
    assert np.allclose(rsp, sp)
    field, _ = read_mha(files[1])
    assert np.array_equal(field, host(h))
