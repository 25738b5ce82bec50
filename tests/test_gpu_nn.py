"""GPU tests of the warm-start network kernels (tcgen05 implicit-GEMM
convolutions and the elementwise layers) against the numpy restatement in
oracle/nn_oracle.py, and the network's gradients against the same oracle.

Tolerances: the device multiplies BF16 operands exactly and accumulates in
FP32 in a different order than the float64 oracle, then rounds the stored
activations or gradients to BF16 (relative 2^-8):
* FP32 outputs (the head, the weight gradients): max |gpu - ref| <=
  1e-3 * max |ref|;
* BF16 outputs: max |gpu - ref| <= 1e-2 * max |ref|;
* the whole network's weight gradients, through 15 layers of BF16
  activations and gradients: ||gpu - ref|| <= 5e-2 ||ref|| per layer.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from atlaswerks_b200 import _lib  # noqa: E402
from atlaswerks_b200.warmstart import LAYERS, WarmStartNet, n_parameters  # noqa: E402
from oracle import nn_oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu

CONFIGS = [(16, 16, 27), (16, 32, 27), (48, 16, 27), (192, 64, 27), (16, 16, 1), (96, 32, 27),
           (32, 128, 27), (64, 64, 27)]


def bf(a):
    return torch.from_numpy(O.bf16(a)).to(torch.bfloat16).cuda()


def f32(t):
    torch.cuda.synchronize()
    return t.float().cpu().numpy()


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


def scratch_for(grid, cin, cout, taps, split):
    """Split-K scratch (None: the direct, unsplit GEMM)."""
    if not split:
        return None, 0
    n = int(_lib.lib().aw_nn_conv3d_scratch_floats(*grid, cin, cout, taps))
    return torch.zeros(max(n, 1), device="cuda"), n


@pytest.mark.parametrize("split", [False, True])
@pytest.mark.parametrize("grid", [(1, 8, 8, 8), (1, 4, 6, 10), (2, 4, 8, 8)])
@pytest.mark.parametrize("cin,cout,taps", CONFIGS)
def test_conv_forward(grid, cin, cout, taps, split):
    rng = np.random.default_rng(cin * 7 + cout + taps)
    B, D, H, W = grid
    x = O.bf16(rng.normal(0, 1, (B, D, H, W, cin)).astype(np.float32))
    w = O.bf16(rng.normal(0, 0.1, (cout, taps, cin)).astype(np.float32))
    b = rng.normal(0, 0.1, cout).astype(np.float32)
    want = O.conv_fwd(x, w, b, relu=False)
    # device copies held in names: a temporary's memory could be reused
    # by the next temporary before the kernel runs
    xd, wd, bd = bf(x), bf(w), torch.from_numpy(b).cuda()
    sc, nsc = scratch_for(grid, cin, cout, taps, split)
    scp = sc.data_ptr() if sc is not None else None
    outf = torch.zeros((B * D * H * W, cout), device="cuda")
    rc = _lib.lib().aw_nn_conv3d_fwd(xd.data_ptr(), B, D, H, W, cin, wd.data_ptr(), bd.data_ptr(),
                                     cout, taps, 0, None, outf.data_ptr(), scp, nsc, None)
    assert rc == 0, _lib.lib().aw_last_error()
    got = f32(outf).reshape(want.shape)
    assert rel(got, want) <= 1e-3
    # BF16 output with ReLU
    outb = torch.zeros((B * D * H * W, cout), dtype=torch.bfloat16, device="cuda")
    rc = _lib.lib().aw_nn_conv3d_fwd(xd.data_ptr(), B, D, H, W, cin, wd.data_ptr(), bd.data_ptr(),
                                     cout, taps, 1, outb.data_ptr(), None, scp, nsc, None)
    assert rc == 0
    assert rel(f32(outb).reshape(want.shape), np.maximum(want, 0)) <= 1e-2


# shapes that take the direct kernel (TMA halo tile + shifted-descriptor
# MMAs), with 1, 2 and 4 output planes per tile
DIRECT = [(16, 16), (48, 16), (16, 32), (32, 32)]
DIRECT_GRIDS = [(1, 8, 32, 16), (2, 6, 32, 24), (1, 32, 64, 64), (1, 64, 64, 64)]


@pytest.mark.parametrize("grid", DIRECT_GRIDS)
@pytest.mark.parametrize("cin,cout", DIRECT)
def test_conv_forward_direct(grid, cin, cout):
    L = _lib.lib()
    B, D, H, W = grid
    planes = L.aw_nn_conv3d_direct_planes(B, D, H, W, cin, cout, 27)
    assert planes in (1, 2, 4)
    rng = np.random.default_rng(cin * 3 + cout + D)
    x = O.bf16(rng.normal(0, 1, (B, D, H, W, cin)).astype(np.float32))
    w = O.bf16(rng.normal(0, 0.1, (cout, 27, cin)).astype(np.float32))
    b = rng.normal(0, 0.1, cout).astype(np.float32)
    want = O.conv_fwd(x, w, b, relu=False)
    xd, wd, bd = bf(x), bf(w), torch.from_numpy(b).cuda()
    outf = torch.zeros((B * D * H * W, cout), device="cuda")
    rc = L.aw_nn_conv3d_fwd(xd.data_ptr(), B, D, H, W, cin, wd.data_ptr(), bd.data_ptr(), cout, 27,
                            0, None, outf.data_ptr(), None, 0, None)
    assert rc == 0, L.aw_last_error()
    assert rel(f32(outf).reshape(want.shape), want) <= 1e-3
    outb = torch.zeros((B * D * H * W, cout), dtype=torch.bfloat16, device="cuda")
    rc = L.aw_nn_conv3d_fwd(xd.data_ptr(), B, D, H, W, cin, wd.data_ptr(), bd.data_ptr(), cout, 27,
                            1, outb.data_ptr(), None, None, 0, None)
    assert rc == 0
    assert rel(f32(outb).reshape(want.shape), np.maximum(want, 0)) <= 1e-2


def test_direct_plane_choice():
    """The dispatcher's tile depth: 4 planes for the 64^3 16-channel layers,
    2 for the 48-channel one (shared memory), 1 on small grids, and the
    GEMM path (0) where the box would not fit or the channels are other."""
    L = _lib.lib()
    assert L.aw_nn_conv3d_direct_planes(1, 64, 64, 64, 16, 16, 27) == 4
    assert L.aw_nn_conv3d_direct_planes(1, 64, 64, 64, 48, 16, 27) == 2
    assert L.aw_nn_conv3d_direct_planes(1, 32, 32, 32, 16, 32, 27) == 1
    assert L.aw_nn_conv3d_direct_planes(1, 16, 16, 16, 16, 16, 27) == 0
    assert L.aw_nn_conv3d_direct_planes(1, 64, 64, 64, 96, 32, 27) == 0
    assert L.aw_nn_conv3d_direct_planes(1, 64, 64, 64, 16, 16, 1) == 0


@pytest.mark.parametrize("split", [False, True])
@pytest.mark.parametrize("grid", [(1, 8, 8, 8), (1, 4, 6, 10)])
@pytest.mark.parametrize("cin,cout,taps", CONFIGS)
def test_conv_dgrad(grid, cin, cout, taps, split):
    rng = np.random.default_rng(cin + cout * 3 + taps)
    B, D, H, W = grid
    dy = O.bf16(rng.normal(0, 1, (B, D, H, W, cout)).astype(np.float32))
    w = O.bf16(rng.normal(0, 0.1, (cout, taps, cin)).astype(np.float32))
    mask = O.bf16(rng.normal(0, 1, (B, D, H, W, cin)).astype(np.float32))
    want = O.conv_dgrad(dy, w, mask)
    wt = np.ascontiguousarray(w.transpose(2, 1, 0))
    dyd, wtd, md = bf(dy), bf(wt), bf(mask)
    sc, nsc = scratch_for(grid, cin, cout, taps, split)
    dx = torch.zeros((B * D * H * W, cin), dtype=torch.bfloat16, device="cuda")
    rc = _lib.lib().aw_nn_conv3d_dgrad(dyd.data_ptr(), B, D, H, W, cout, wtd.data_ptr(), cin, taps,
                                       md.data_ptr(), dx.data_ptr(),
                                       sc.data_ptr() if sc is not None else None, nsc, None)
    assert rc == 0, _lib.lib().aw_last_error()
    assert rel(f32(dx).reshape(want.shape), want) <= 1e-2


@pytest.mark.parametrize("grid,splits", [((1, 8, 8, 8), 1), ((1, 8, 8, 8), 3), ((1, 4, 6, 10), 2),
                                         ((2, 8, 8, 16), 8)])
@pytest.mark.parametrize("cin,cout,taps", CONFIGS)
def test_conv_wgrad(grid, splits, cin, cout, taps):
    rng = np.random.default_rng(cin * 5 + cout + taps + splits)
    B, D, H, W = grid
    x = O.bf16(rng.normal(0, 1, (B, D, H, W, cin)).astype(np.float32))
    dy = O.bf16(rng.normal(0, 1, (B, D, H, W, cout)).astype(np.float32))
    want = O.conv_wgrad(x, dy, taps)
    L = _lib.lib()
    scratch = torch.zeros(int(L.aw_nn_wgrad_scratch_floats(cin, cout, taps, splits)), device="cuda")
    dw = torch.zeros((cout, taps, cin), device="cuda")
    xd, dyd = bf(x), bf(dy)
    rc = L.aw_nn_conv3d_wgrad(xd.data_ptr(), dyd.data_ptr(), B, D, H, W, cin, cout, taps, splits,
                              scratch.data_ptr(), dw.data_ptr(), None)
    assert rc == 0, L.aw_last_error()
    assert rel(f32(dw), want) <= 1e-3


def test_elementwise_layers():
    rng = np.random.default_rng(3)
    L = _lib.lib()
    x = O.bf16(rng.normal(0, 1, (1, 8, 6, 4, 32)).astype(np.float32))
    xd = bf(x)
    p = torch.zeros((4 * 3 * 2, 32), dtype=torch.bfloat16, device="cuda")
    assert L.aw_nn_pool(xd.data_ptr(), 1, 8, 6, 4, 32, p.data_ptr(), 0, None, None, None) == 0
    assert rel(f32(p).reshape(1, 4, 3, 2, 32), O.pool(x)) <= 1e-2
    dp = O.bf16(rng.normal(0, 1, (1, 4, 3, 2, 32)).astype(np.float32))
    add = O.bf16(rng.normal(0, 1, x.shape).astype(np.float32))
    dpd, addd = bf(dp), bf(add)
    dx = torch.zeros((8 * 6 * 4, 32), dtype=torch.bfloat16, device="cuda")
    assert L.aw_nn_pool(dpd.data_ptr(), 1, 8, 6, 4, 32, dx.data_ptr(), 1, addd.data_ptr(),
                        xd.data_ptr(), None) == 0
    want = (O.pool_bwd(dp) + add) * (x > 0)
    assert rel(f32(dx).reshape(x.shape), want) <= 1e-2
    c = O.bf16(rng.normal(0, 1, (1, 4, 3, 2, 32)).astype(np.float32))
    cd = bf(c)
    cat = torch.zeros((8 * 6 * 4, 48), dtype=torch.bfloat16, device="cuda")
    assert L.aw_nn_upsample(cd.data_ptr(), 1, 4, 3, 2, 32, cat.data_ptr(), 48, 0, 0, None) == 0
    assert np.array_equal(f32(cat).reshape(1, 8, 6, 4, 48)[..., :32], O.up(c))
    dc = torch.zeros((4 * 3 * 2, 32), dtype=torch.bfloat16, device="cuda")
    g = O.bf16(rng.normal(0, 1, (1, 8, 6, 4, 48)).astype(np.float32))
    gd = bf(g)
    assert L.aw_nn_upsample(gd.data_ptr(), 1, 4, 3, 2, 32, dc.data_ptr(), 48, 0, 1, None) == 0
    assert rel(f32(dc).reshape(1, 4, 3, 2, 32), O.up_bwd(g[..., :32])) <= 1e-2


def test_network_gradients_match_oracle():
    """Forward and backward of the whole encoder-decoder at 16^3."""
    n = 16
    shape = (n, n, n)
    net = WarmStartNet(shape, seed=5)
    # a head large enough that its gradient reaches every layer
    rng = np.random.default_rng(6)
    net.w["head"].copy_(torch.from_numpy(rng.normal(0, 0.2, (16, 1, 16)).astype(np.float32)))
    net.refresh_bf16()
    I0 = rng.random(shape, dtype=np.float32)
    I1 = rng.random(shape, dtype=np.float32)
    out = f32(net.forward(torch.from_numpy(I0).cuda(), torch.from_numpy(I1).cuda()))
    x = np.zeros((1,) + shape + (16,), np.float32)
    x[..., 0], x[..., 1] = O.bf16(I0), O.bf16(I1)
    layers = [(n, ci, co, t, n != "head") for n, ci, co, t in LAYERS]
    ref = O.UNetOracle(layers, {k: v.cpu().numpy() for k, v in net.w.items()},
                       {k: v.cpu().numpy() for k, v in net.b.items()})
    want = ref.forward(x).reshape(-1, 16)
    assert np.linalg.norm(out - want) <= 2e-2 * np.linalg.norm(want)
    dout = O.bf16(rng.normal(0, 1e-3, (n ** 3, 16)).astype(np.float32))
    doutd = bf(dout)
    net.backward(doutd)
    g = ref.backward(dout.reshape((1,) + shape + (16,)).astype(np.float64))
    torch.cuda.synchronize()
    for name, *_ in LAYERS:
        gw, gb = f32(net.gw[name]), f32(net.gb[name])
        rw, rb = g[name]
        assert np.linalg.norm(gw - rw) <= 5e-2 * np.linalg.norm(rw), name
        assert np.linalg.norm(gb - rb) <= 5e-2 * max(np.linalg.norm(rb), 1e-12), name
    assert not net.timed_out()


def test_network_direct_path_32():
    """At 32^3 the level-0 convolutions take the direct kernel. Its forward
    output agrees with the oracle and with the all-GEMM path; the weight
    gradients point the oracle's way (BF16 activations and gradients
    through 15 layers at 32^3 leave 4-16 % relative noise on either path,
    so the check is the cosine, >= 0.97 per layer)."""
    L = _lib.lib()
    shape = (32, 32, 32)
    assert L.aw_nn_conv3d_direct_planes(1, 32, 32, 32, 16, 16, 27) > 0
    rng = np.random.default_rng(7)
    I0 = rng.random(shape, dtype=np.float32)
    I1 = rng.random(shape, dtype=np.float32)
    dout = O.bf16(rng.normal(0, 1e-3, (32 ** 3, 16)).astype(np.float32))
    doutd = bf(dout)
    outs, grads = [], []
    try:
        for gemm_only in (0, 1):
            L.aw_nn_set_gemm_only(gemm_only)
            net = WarmStartNet(shape, seed=5)
            net.w["head"].copy_(torch.from_numpy(
                np.random.default_rng(6).normal(0, 0.2, (16, 1, 16)).astype(np.float32)))
            net.refresh_bf16()
            outs.append(f32(net.forward(torch.from_numpy(I0).cuda(), torch.from_numpy(I1).cuda())))
            net.backward(doutd)
            grads.append({k: f32(net.gw[k]) for k, *_ in LAYERS})
    finally:
        L.aw_nn_set_gemm_only(0)
    x = np.zeros((1,) + shape + (16,), np.float32)
    x[..., 0], x[..., 1] = O.bf16(I0), O.bf16(I1)
    layers = [(n, ci, co, t, n != "head") for n, ci, co, t in LAYERS]
    ref = O.UNetOracle(layers, {k: v.cpu().numpy() for k, v in net.w.items()},
                       {k: v.cpu().numpy() for k, v in net.b.items()})
    want = ref.forward(x).reshape(-1, 16)
    assert np.linalg.norm(outs[0] - want) <= 1e-2 * np.linalg.norm(want)
    assert np.linalg.norm(outs[0] - outs[1]) <= 1e-2 * np.linalg.norm(want)
    g = ref.backward(dout.reshape((1,) + shape + (16,)).astype(np.float64))
    for name, *_ in LAYERS:
        a, r = grads[0][name].ravel(), g[name][0].ravel()
        assert a @ r >= 0.97 * np.linalg.norm(a) * np.linalg.norm(r), name


def test_parameter_count():
    assert 1.4e6 <= n_parameters() <= 1.5e6
