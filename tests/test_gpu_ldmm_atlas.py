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
