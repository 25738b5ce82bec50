"""GPU parity of the multiscale scale-level changes and of multiscale greedy
registration (GreedyWarp::RunWarp over several levels) against the oracle.

Tolerances: Gaussian downsampling and deformation upsampling are bit-exact
(same float/double operation sequence as GaussianFilter3D,
ImageUtils::resampleNew and HField3DUtils::resampleNew); the multiscale
registration's final field is within 1e-3 voxel RMS of the oracle's.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from atlaswerks_b200 import device as D  # noqa: E402
from atlaswerks_b200.multiscale import GreedyWarpB200, ScaleLevel  # noqa: E402
from atlaswerks_b200.synth import bullseye, greedy_pair  # noqa: E402
from oracle import identity  # noqa: E402

pytestmark = pytest.mark.gpu


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.mark.parametrize("shape,new,sp", [((32, 31, 36), (16, 15, 18), (2.0, 2.06452, 1.77778)),
                                          ((64, 64, 64), (32, 32, 32), (1.0, 1.0, 1.0)),
                                          ((128, 128, 128), (32, 32, 32), (1.0, 1.0, 1.0)),
                                          ((20, 18, 16), (10, 9, 8), (1.0, 1.0, 1.0))])
def test_downsample_upsample_bit_exact(oracle, shape, new, sp):
    rng = np.random.default_rng(5)
    img = rng.random(shape, dtype=np.float32)
    assert np.array_equal(host(D.downsample(cu(img), new, sp)), oracle.downsample(img, new, sp))
    h = identity(new) + rng.normal(0, 1.0, (3,) + new).astype(np.float32)
    assert np.array_equal(host(D.upsample_hfield(cu(h), shape)), oracle.upsample_hfield(h, shape))


def test_multiscale_greedy_vs_oracle(oracle):
    """Three levels 4/2/1 on a 64^3 pair (the config-2 schedule shape)."""
    shape = (64, 64, 64)
    I0, I1 = greedy_pair(shape, seed=31, n_blobs=8, umax=4.0, noise_sd=0.02)
    levels = [(4, 20, 0.5), (2, 10, 0.5), (1, 5, 0.5)]
    h_o, _, e_o = oracle.greedy_warp(I0, I1, levels)
    w = GreedyWarpB200(cu(I0), cu(I1), [ScaleLevel(f, n, m) for f, n, m in levels])
    h_g, _ = w.RunWarp()
    rms = float(np.sqrt(((host(h_g) - h_o).astype(np.float64) ** 2).sum(0).mean()))
    assert rms <= 1e-3, rms
    for a, b in zip(w.energies, e_o):
        assert np.allclose(a, b, rtol=1e-4)


def test_multiscale_bullseye_anisotropic(oracle):
    """The reference regression's geometry (32 x 31 x 36, spacing 2 x 2.06 x 1.78,
    levels 2 and 1 x 50 iterations, MaxPert 0.3) on generated bullseyes."""
    shape, sp = (36, 31, 32), (2.0, 2.06452, 1.77778)
    I0 = bullseye(shape, [12, 8, 4])
    I1 = bullseye(shape, [13, 9, 5], center=(16.5, 15.0, 17.0))
    levels = [(2, 50, 0.3), (1, 50, 0.3)]
    h_o, hi_o, _ = oracle.greedy_warp(I0, I1, levels, sp, inverse=True)
    w = GreedyWarpB200(cu(I0), cu(I1), [ScaleLevel(f, n, m) for f, n, m in levels], sp,
                       compute_inverse=True)
    h_g, hi_g = w.RunWarp()
    rms = float(np.sqrt(((host(h_g) - h_o).astype(np.float64) ** 2).sum(0).mean()))
    assert rms <= 1e-3, rms
    # deformed images by the reference regression's criterion (L1 sum < 1.0)
    err = float(np.abs(oracle.apply(I0, host(h_g)) - oracle.apply(I0, h_o)).sum())
    assert err < 1.0, err
