"""GPU parity of LDMM geodesic shooting (LDMMShootingIteratorB200 over
aw_ldmm_shoot_iterate) against the oracle's restatement of
LDMMShootingIteratorCPU::Iterate (itself pinned against the reference in
tests/test_oracle_pin.py).

Tolerances (four iterations): alpha0 within 1e-4 of max |alpha0|, the
maps within 1e-3 voxel, image energies 1e-4 relative — the fluid solve
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
    e_o = []
    for _ in range(iters):
        e, p0, p1 = oracle.ldmm_shoot_iterate(I0, I1, a, T, sp, sigma=1.0, step=0.05)
        e_o.append(e)
    data, e_g = shoot_register(cu(I0), cu(I1), T, iters, sp, sigma=1.0, step=0.05)
    ag = host(data.Alpha0)
    assert np.abs(ag - a).max() <= 1e-4 * np.abs(a).max()
    assert np.abs(host(data.Phi0T) - p0).max() <= 1e-3
    assert np.abs(host(data.PhiT0) - p1).max() <= 1e-3
    assert np.allclose(e_g, e_o, rtol=1e-4)
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
