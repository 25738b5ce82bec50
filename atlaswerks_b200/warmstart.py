"""Learned warm start for greedy-fluid registration.

A small 3D convolutional encoder-decoder (4 levels, 16/32/64/128 channels,
3x3x3 convolutions, skip connections, ~1.47 M parameters) maps an image pair
(I0, I1) to a displacement u; the greedy iteration then starts from
h = x + u instead of the identity and refines it, and falls back to the
plain solve from the identity when the warm start does not lower the
image mismatch. The network has no counterpart in the reference; it is
trained on pairs whose targets come from the GPU greedy solver itself.

Every layer runs in libaw_b200.so (``aw_nn_*``: tcgen05 implicit-GEMM
convolutions, BF16 activations, FP32 accumulation and master weights,
Adam); torch only holds the device buffers.
"""
from __future__ import annotations

import ctypes
import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import check
from .device import _stream

# (name, input channels, output channels, taps); every layer but the head
# is followed by a ReLU. The first layer's input has 2 real channels
# (I0, I1) padded to 16.
LAYERS: List[Tuple[str, int, int, int]] = [
    ("e0a", 16, 16, 27), ("e0b", 16, 16, 27),
    ("e1a", 16, 32, 27), ("e1b", 32, 32, 27),
    ("e2a", 32, 64, 27), ("e2b", 64, 64, 27),
    ("e3a", 64, 128, 27), ("e3b", 128, 128, 27),
    ("d2a", 192, 64, 27), ("d2b", 64, 64, 27),
    ("d1a", 96, 32, 27), ("d1b", 32, 32, 27),
    ("d0a", 48, 16, 27), ("d0b", 16, 16, 27),
    ("head", 16, 16, 1),
]


def n_parameters() -> int:
    return sum(co * t * ci + co for _, ci, co, t in LAYERS)


def _p(t: Optional[torch.Tensor]):
    return None if t is None else t.data_ptr()


class WarmStartNet:
    """The network on one grid (D, H, W divisible by 8), batch 1."""

    def __init__(self, shape: Sequence[int], seed: int = 0, device="cuda"):
        self.D, self.H, self.W = (int(s) for s in shape)
        if self.D % 8 or self.H % 8 or self.W % 8:
            raise ValueError("grid axes must be divisible by 8 (three 2x poolings)")
        self.dev = device
        rng = np.random.default_rng(seed)
        self.w: Dict[str, torch.Tensor] = {}
        self.b: Dict[str, torch.Tensor] = {}
        for name, ci, co, t in LAYERS:
            fan_in = t * (2 if name == "e0a" else ci)
            std = math.sqrt(2.0 / fan_in) if name != "head" else 1e-3
            w = rng.normal(0.0, std, (co, t, ci)).astype(np.float32)
            if name == "e0a":
                w[:, :, 2:] = 0.0  # padded input channels
            if name == "head":
                w[3:] = 0.0        # only 3 output channels are used
            self.w[name] = torch.from_numpy(w).to(device)
            self.b[name] = torch.zeros(co, device=device)
        self.m1 = {k: torch.zeros_like(v) for k, v in list(self.w.items())}
        self.m2 = {k: torch.zeros_like(v) for k, v in list(self.w.items())}
        self.bm1 = {k: torch.zeros_like(v) for k, v in self.b.items()}
        self.bm2 = {k: torch.zeros_like(v) for k, v in self.b.items()}
        self.gw = {k: torch.zeros_like(v) for k, v in self.w.items()}
        self.gb = {k: torch.zeros_like(v) for k, v in self.b.items()}
        self.wb = {k: torch.empty(v.shape, dtype=torch.bfloat16, device=device) for k, v in self.w.items()}
        self.wt = {k: torch.empty((v.shape[2], v.shape[1], v.shape[0]), dtype=torch.bfloat16,
                                  device=device) for k, v in self.w.items()}
        self.t = 0
        self._alloc()
        self.refresh_bf16()

    # ---- buffers ---------------------------------------------------------------
    def _grid(self, level):
        f = 2 ** level
        return (self.D // f, self.H // f, self.W // f)

    def _vox(self, level):
        d, h, w = self._grid(level)
        return d * h * w

    def _alloc(self):
        bf = lambda level, c: torch.zeros((self._vox(level), c), dtype=torch.bfloat16,
                                          device=self.dev)
        a = {}
        a["x"] = bf(0, 16)
        for n, lvl, c in [("e0a", 0, 16), ("e0b", 0, 16), ("p0", 1, 16), ("e1a", 1, 32),
                          ("e1b", 1, 32), ("p1", 2, 32), ("e2a", 2, 64), ("e2b", 2, 64),
                          ("p2", 3, 64), ("e3a", 3, 128), ("e3b", 3, 128), ("c2", 2, 192),
                          ("d2a", 2, 64), ("d2b", 2, 64), ("c1", 1, 96), ("d1a", 1, 32),
                          ("d1b", 1, 32), ("c0", 0, 48), ("d0a", 0, 16), ("d0b", 0, 16)]:
            a[n] = bf(lvl, c)
        self.a = a
        self.out = torch.zeros((self._vox(0), 16), device=self.dev)
        # gradients: one buffer per level and width, reused along the sweep
        self.g = {(lvl, c): bf(lvl, c) for lvl, c in [(0, 16), (0, 48), (1, 16), (1, 32),
                                                         (1, 96), (2, 32), (2, 64), (2, 192),
                                                         (3, 64), (3, 128)]}
        self.g2 = {(lvl, c): bf(lvl, c) for lvl, c in [(0, 16), (1, 32), (2, 64), (3, 128)]}
        self.skip = {0: bf(0, 16), 1: bf(1, 32), 2: bf(2, 64)}
        self.dout = bf(0, 16)
        L = _lib.lib()
        self.splits = {}
        need, cneed = 0, 0
        for name, ci, co, t in LAYERS:
            lvl = self._level_of(name)
            vox = self._vox(lvl)
            # weight gradient: K = voxels split so that ~8 CTAs per SM run
            mtiles = -(-t * ci // 128)
            s = max(1, min(vox // 512, -(-1184 // mtiles)))
            self.splits[name] = s
            need = max(need, L.aw_nn_wgrad_scratch_floats(ci, co, t, s))
            cneed = max(cneed, L.aw_nn_conv3d_scratch_floats(1, *self._grid(lvl), ci, co, t))
        self.wscratch = torch.zeros(int(need), device=self.dev)
        self.cscratch = torch.zeros(max(1, int(cneed)), device=self.dev)
        self.bscratch = torch.zeros(int(L.aw_nn_bias_scratch_floats(self._vox(0), 192)),
                                    device=self.dev)
        self.mse_scratch = torch.zeros(int(L.aw_nn_mse_scratch_doubles(self._vox(0))),
                                       dtype=torch.float64, device=self.dev)
        self.loss = torch.zeros(1, device=self.dev)

    @staticmethod
    def _level_of(name):
        return {"e0": 0, "e1": 1, "e2": 2, "e3": 3, "d2": 2, "d1": 1, "d0": 0, "he": 0}[name[:2]]

    def refresh_bf16(self):
        L, s = _lib.lib(), _stream()
        for name, ci, co, t in LAYERS:
            check(L.aw_nn_weights_bf16(_p(self.w[name]), co, t, ci, _p(self.wb[name]),
                                       _p(self.wt[name]), s))

    # ---- layers ----------------------------------------------------------------
    def _conv(self, name, x, lvl, out=None, outf=None, relu=True):
        _, ci, co, t = next(l for l in LAYERS if l[0] == name)
        d, h, w = self._grid(lvl)
        check(_lib.lib().aw_nn_conv3d_fwd(_p(x), 1, d, h, w, ci, _p(self.wb[name]),
                                          _p(self.b[name]), co, t, int(relu), _p(out), _p(outf),
                                          _p(self.cscratch), self.cscratch.numel(), _stream()))

    def _pool(self, src, lvl_fine, c, dst):
        d, h, w = self._grid(lvl_fine)
        check(_lib.lib().aw_nn_pool(_p(src), 1, d, h, w, c, _p(dst), 0, None, None, _stream()))

    def _up_into(self, src, lvl_coarse, c, dst, ct, c0):
        d, h, w = self._grid(lvl_coarse)
        check(_lib.lib().aw_nn_upsample(_p(src), 1, d, h, w, c, _p(dst), ct, c0, 0, _stream()))

    def _slice(self, src, cs, cs0, dst, cd, cd0, c, lvl, acc=0):
        check(_lib.lib().aw_nn_slice(_p(src), cs, cs0, _p(dst), cd, cd0, c, self._vox(lvl), acc,
                                     _stream()))

    def forward(self, I0: torch.Tensor, I1: torch.Tensor) -> torch.Tensor:
        """Predicted displacement as FP32 [V, 16] (channels 0..2 = x, y, z)."""
        a = self.a
        check(_lib.lib().aw_nn_pack_pair(_p(I0), _p(I1), self._vox(0), _p(a["x"]), _stream()))
        self._conv("e0a", a["x"], 0, a["e0a"])
        self._conv("e0b", a["e0a"], 0, a["e0b"])
        self._pool(a["e0b"], 0, 16, a["p0"])
        self._conv("e1a", a["p0"], 1, a["e1a"])
        self._conv("e1b", a["e1a"], 1, a["e1b"])
        self._pool(a["e1b"], 1, 32, a["p1"])
        self._conv("e2a", a["p1"], 2, a["e2a"])
        self._conv("e2b", a["e2a"], 2, a["e2b"])
        self._pool(a["e2b"], 2, 64, a["p2"])
        self._conv("e3a", a["p2"], 3, a["e3a"])
        self._conv("e3b", a["e3a"], 3, a["e3b"])
        self._up_into(a["e3b"], 3, 128, a["c2"], 192, 0)
        self._slice(a["e2b"], 64, 0, a["c2"], 192, 128, 64, 2)
        self._conv("d2a", a["c2"], 2, a["d2a"])
        self._conv("d2b", a["d2a"], 2, a["d2b"])
        self._up_into(a["d2b"], 2, 64, a["c1"], 96, 0)
        self._slice(a["e1b"], 32, 0, a["c1"], 96, 64, 32, 1)
        self._conv("d1a", a["c1"], 1, a["d1a"])
        self._conv("d1b", a["d1a"], 1, a["d1b"])
        self._up_into(a["d1b"], 1, 32, a["c0"], 48, 0)
        self._slice(a["e0b"], 16, 0, a["c0"], 48, 32, 16, 0)
        self._conv("d0a", a["c0"], 0, a["d0a"])
        self._conv("d0b", a["d0a"], 0, a["d0b"])
        self._conv("head", a["d0b"], 0, outf=self.out, relu=False)
        return self.out

    def _layer_bwd(self, name, inp, dy, lvl, dx=None, mask=None):
        """Weight and bias gradients of `name` from dy (the gradient of its
        pre-activation output); dx = the input gradient (x mask > 0)."""
        _, ci, co, t = next(l for l in LAYERS if l[0] == name)
        d, h, w = self._grid(lvl)
        L, s = _lib.lib(), _stream()
        check(L.aw_nn_conv3d_wgrad(_p(inp), _p(dy), 1, d, h, w, ci, co, t, self.splits[name],
                                   _p(self.wscratch), _p(self.gw[name]), s))
        check(L.aw_nn_bias_grad(_p(dy), self._vox(lvl), co, _p(self.bscratch), _p(self.gb[name]),
                                s))
        if dx is not None:
            check(L.aw_nn_conv3d_dgrad(_p(dy), 1, d, h, w, co, _p(self.wt[name]), ci, t, _p(mask),
                                       _p(dx), _p(self.cscratch), self.cscratch.numel(), s))

    def _pool_bwd(self, dp, lvl_fine, c, add, mask, dst):
        d, h, w = self._grid(lvl_fine)
        check(_lib.lib().aw_nn_pool(_p(dp), 1, d, h, w, c, _p(dst), 1, _p(add), _p(mask),
                                    _stream()))

    def _up_bwd(self, dcat, lvl_coarse, c, ct, dst):
        d, h, w = self._grid(lvl_coarse)
        check(_lib.lib().aw_nn_upsample(_p(dcat), 1, d, h, w, c, _p(dst), ct, 0, 1, _stream()))

    def backward(self, dout: torch.Tensor):
        """dout: BF16 [V, 16] gradient of the head output. Fills gw, gb."""
        a, g, g2, sk = self.a, self.g, self.g2, self.skip
        self._layer_bwd("head", a["d0b"], dout, 0, g[(0, 16)], a["d0b"])
        self._layer_bwd("d0b", a["d0a"], g[(0, 16)], 0, g2[(0, 16)], a["d0a"])
        self._layer_bwd("d0a", a["c0"], g2[(0, 16)], 0, g[(0, 48)], a["c0"])
        self._up_bwd(g[(0, 48)], 1, 32, 48, g[(1, 32)])
        self._slice(g[(0, 48)], 48, 32, sk[0], 16, 0, 16, 0)
        self._layer_bwd("d1b", a["d1a"], g[(1, 32)], 1, g2[(1, 32)], a["d1a"])
        self._layer_bwd("d1a", a["c1"], g2[(1, 32)], 1, g[(1, 96)], a["c1"])
        self._up_bwd(g[(1, 96)], 2, 64, 96, g[(2, 64)])
        self._slice(g[(1, 96)], 96, 64, sk[1], 32, 0, 32, 1)
        self._layer_bwd("d2b", a["d2a"], g[(2, 64)], 2, g2[(2, 64)], a["d2a"])
        self._layer_bwd("d2a", a["c2"], g2[(2, 64)], 2, g[(2, 192)], a["c2"])
        self._up_bwd(g[(2, 192)], 3, 128, 192, g[(3, 128)])
        self._slice(g[(2, 192)], 192, 128, sk[2], 64, 0, 64, 2)
        self._layer_bwd("e3b", a["e3a"], g[(3, 128)], 3, g2[(3, 128)], a["e3a"])
        self._layer_bwd("e3a", a["p2"], g2[(3, 128)], 3, g[(3, 64)], None)
        self._pool_bwd(g[(3, 64)], 2, 64, sk[2], a["e2b"], g[(2, 64)])
        self._layer_bwd("e2b", a["e2a"], g[(2, 64)], 2, g2[(2, 64)], a["e2a"])
        self._layer_bwd("e2a", a["p1"], g2[(2, 64)], 2, g[(2, 32)], None)
        self._pool_bwd(g[(2, 32)], 1, 32, sk[1], a["e1b"], g[(1, 32)])
        self._layer_bwd("e1b", a["e1a"], g[(1, 32)], 1, g2[(1, 32)], a["e1a"])
        self._layer_bwd("e1a", a["p0"], g2[(1, 32)], 1, g[(1, 16)], None)
        self._pool_bwd(g[(1, 16)], 0, 16, sk[0], a["e0b"], g[(0, 16)])
        self._layer_bwd("e0b", a["e0a"], g[(0, 16)], 0, g2[(0, 16)], a["e0a"])
        self._layer_bwd("e0a", a["x"], g2[(0, 16)], 0)

    def loss_and_grad(self, target: torch.Tensor) -> torch.Tensor:
        """MSE of the prediction against the planar [3, D, H, W] target; the
        gradient goes to self.dout. Returns the device loss scalar."""
        check(_lib.lib().aw_nn_mse(_p(self.out), _p(target), self._vox(0), _p(self.dout),
                                   _p(self.mse_scratch), _p(self.loss), _stream()))
        return self.loss

    def adam_step(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.t += 1
        L, s = _lib.lib(), _stream()
        for name, ci, co, t in LAYERS:
            check(L.aw_nn_adam(_p(self.w[name]), _p(self.gw[name]), _p(self.m1[name]),
                               _p(self.m2[name]), self.w[name].numel(), lr, beta1, beta2, eps,
                               self.t, s))
            check(L.aw_nn_adam(_p(self.b[name]), _p(self.gb[name]), _p(self.bm1[name]),
                               _p(self.bm2[name]), co, lr, beta1, beta2, eps, self.t, s))
        self.refresh_bf16()

    def train_step(self, I0, I1, target, lr=1e-3) -> torch.Tensor:
        self.forward(I0, I1)
        loss = self.loss_and_grad(target)
        self.backward(self.dout)
        self.adam_step(lr)
        return loss

    def predict_h(self, I0, I1) -> torch.Tensor:
        """The warm-start deformation h = x + u as [3, D, H, W]."""
        pred = self.forward(I0, I1)
        h = torch.empty((3, self.D, self.H, self.W), device=self.dev)
        check(_lib.lib().aw_nn_displacement_to_h(_p(pred), self.D, self.H, self.W, _p(h[0]),
                                                 _p(h[1]), _p(h[2]), _stream()))
        return h

    def timed_out(self) -> bool:
        v = ctypes.c_int()
        check(_lib.lib().aw_nn_status(ctypes.byref(v)))
        return bool(v.value)

    def state(self):
        return {"w": {k: v.cpu().numpy() for k, v in self.w.items()},
                "b": {k: v.cpu().numpy() for k, v in self.b.items()}}

    def load(self, st):
        for k in self.w:
            self.w[k].copy_(torch.from_numpy(st["w"][k]))
            self.b[k].copy_(torch.from_numpy(st["b"][k]))
        self.refresh_bf16()


# ---- data, training, refinement ---------------------------------------------
def _greedy(shape, max_pert=0.5, alpha=0.01, beta=0.01, gamma=0.001):
    from .greedy import DiffOperParam, GreedyIteratorB200, GreedyIteratorParam
    nz, ny, nx = shape
    it = GreedyIteratorB200((nx, ny, nz))
    it.SetScaleLevel((nx, ny, nz), (1.0, 1.0, 1.0),
                     GreedyIteratorParam(DiffOperParam(alpha, beta, gamma), max_pert))
    return it


def solver_target(I0: torch.Tensor, I1: torch.Tensor, iters: int = 50,
                  max_pert: float = 0.5) -> torch.Tensor:
    """The training target: the displacement h - x of the plain GPU greedy
    solve from the identity, planar [3, D, H, W]."""
    from .device import identity
    from .greedy import GreedyDeformationDataB200
    it = _greedy(tuple(I0.shape), max_pert)
    data = GreedyDeformationDataB200(I0, I1)
    it.Run(data, iters, update_first=True)
    return (data.Def1To0() - identity(tuple(I0.shape), I0.device)).contiguous()


def refine(I0: torch.Tensor, I1: torch.Tensor, h0: torch.Tensor, target: float,
           max_iters: int = 50, chunk: int = 5, max_pert: float = 0.5, it=None, data=None,
           step: Optional[float] = None, auto_reduce: bool = True):
    """Greedy refinement from h0 until the iteration energy (the mismatch
    sum (I1 - I0(h))^2 of the deformation entering an iteration, recorded
    on the device) is <= target, in chunks of `chunk` graph-replayed
    iterations. With `step` the iteration keeps that step size (the plain
    solve's, from the identity); without it the step is set at the first
    iteration from the warm start's own velocity. auto_reduce halves the
    step whenever the energy rises (GreedyParam::AutoStepReduce), which
    damps the oscillation of a step chosen from a small residual. Returns (h, iterations,
    energies, reached, fell): `fell` is False when a chunk did not improve
    on the best energy so far — the signal to fall back to the plain solve."""
    from .greedy import GreedyDeformationDataB200
    it = it or _greedy(tuple(I0.shape), max_pert)
    data = data or GreedyDeformationDataB200(I0, I1)
    data.Def1To0().copy_(h0)
    if step is not None:
        it.SetStepSize(step)
    it.SetAutoStepReduce(auto_reduce)
    done = 0
    en = np.zeros(0)
    best = np.inf
    while done < max_iters:
        k = min(chunk, max_iters - done)
        it.Run(data, k, update_first=(done == 0 and step is None))
        done += k
        en = it.Energies()[-done:]
        hit = np.nonzero(en <= target)[0]
        if hit.size:
            return data.Def1To0(), int(hit[0]) + 1, en, True, True
        cmin = float(en[-k:].min())
        if not cmin < best:
            return data.Def1To0(), done, en, False, False
        best = cmin
    return data.Def1To0(), done, en, False, True


def plain_step(I0: torch.Tensor, I1: torch.Tensor, it, data, max_pert: float = 0.5) -> float:
    """The plain solve's step size: MaxPert / max |v| of the first iteration
    from the identity (one iteration on scratch data)."""
    from .device import identity
    data.Def1To0().copy_(identity(tuple(I0.shape), I0.device))
    it.Run(data, 1, update_first=True)
    return it.StepSize()


def warm_h(net: "WarmStartNet", I0: torch.Tensor, I1: torch.Tensor) -> torch.Tensor:
    """The warm-start deformation on the pair's grid. When the network's
    grid is coarser, the pair is Gaussian-downsampled to it (the multiscale
    downsampling of the greedy path), the network predicts there, and the
    deformation is upsampled with its vectors rescaled — the network takes
    the place of the coarse levels of a multiscale solve."""
    from . import device as D
    fine = tuple(I0.shape)
    coarse = (net.D, net.H, net.W)
    if fine == coarse:
        return net.predict_h(I0, I1)
    hc = net.predict_h(D.downsample(I0, coarse), D.downsample(I1, coarse))
    return D.upsample_hfield(hc, fine, True)


class WarmStartPredictor:
    """warm_h for one pair grid as one CUDA graph replay: the pair is copied
    into static buffers, and the downsampling, the 25 launches of the
    network's forward pass, the displacement-to-h kernel and the
    upsampling replay from a graph captured once (no per-layer host work).
    The returned field is the predictor's own buffer, overwritten by the
    next call; the weights are read at replay, so a predictor follows
    later weight updates of its network."""

    def __init__(self, net: "WarmStartNet", shape: Sequence[int]):
        self.net = net
        self.shape = tuple(int(s) for s in shape)
        self.I0 = torch.zeros(self.shape, device=net.dev)
        self.I1 = torch.zeros(self.shape, device=net.dev)
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):  # first launches (module loads, attributes) outside capture
            warm_h(net, self.I0, self.I1)
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.h = warm_h(net, self.I0, self.I1)
        torch.cuda.synchronize()

    def __call__(self, I0: torch.Tensor, I1: torch.Tensor) -> torch.Tensor:
        if tuple(I0.shape) != self.shape or tuple(I1.shape) != self.shape:
            raise ValueError(f"pair grid {tuple(I0.shape)} != predictor grid {self.shape}")
        self.I0.copy_(I0)
        self.I1.copy_(I1)
        self.graph.replay()
        return self.h


def coarse_training_set(seeds: Sequence[int], n: int, coarse: int, workers: int = 0,
                        batch: int = 128, iters: int = 50):
    """Training pairs of the n^3 generator, downsampled on the device to the
    network's coarse^3 grid, with the plain solver's displacement there as
    the target; generated in batches so the host holds one batch at a time."""
    from . import device as D
    out_pairs, out_targets = [], []
    seeds = list(seeds)
    for i in range(0, len(seeds), batch):
        for a, b in make_pairs(seeds[i:i + batch], n, workers):
            ca = D.downsample(torch.from_numpy(a).cuda(), (coarse,) * 3)
            cb = D.downsample(torch.from_numpy(b).cuda(), (coarse,) * 3)
            out_pairs.append((ca, cb))
            out_targets.append(solver_target(ca, cb, iters))
    return out_pairs, out_targets


def make_pairs(seeds: Sequence[int], n: int, workers: int = 0):
    """(I0, I1) pairs of the pair-registration generator (8 blobs, smooth
    warp with max |u| = 3 voxels) on an n^3 grid, one per seed, generated in
    parallel worker processes (started with spawn, so they may be created
    after CUDA is initialised)."""
    import multiprocessing as mp
    from .synth import greedy_pair
    args = [((n, n, n), int(s), 8, 3.0) for s in seeds]
    if workers <= 1 or len(args) < 4:
        return [greedy_pair(*a) for a in args]
    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.starmap(greedy_pair, args, chunksize=max(1, len(args) // (4 * workers)))


# the multiscale schedule of the 3-level pair-registration config:
# (downsample factor, iterations, MaxPert), coarse to fine
MULTISCALE = [(4, 100, 0.5), (2, 50, 0.5), (1, 25, 0.5)]


def _multiscale(I0: torch.Tensor, I1: torch.Tensor):
    """The plain multiscale solve (GreedyWarp over MULTISCALE) with its
    iterators built (prepare), ready to run."""
    from .multiscale import GreedyWarpB200, ScaleLevel
    return GreedyWarpB200(I0, I1, [ScaleLevel(f, n, m) for f, n, m in MULTISCALE]).prepare()


def _plain_multiscale(w):
    """Runs a prepared multiscale solve from the identity; returns (h,
    energies of the finest level)."""
    h, _ = w.RunWarp()
    return h, np.asarray(w.energies[-1])


def evaluate(net: "WarmStartNet", pairs, plain_iters: int = 50, tol: float = 0.01,
             chunk: int = 3, max_pert: float = 0.5, policy: str = "own", plain: str = "single"):
    """Per pair: the plain solve from the identity for plain_iters
    iterations, then the warm start (network + refinement until the
    iteration energy is within (1 + tol) of the plain solve's last one,
    with the plain solve as fallback when a refinement chunk does not lower
    the energy). policy "own": the refinement sets its step from the warm
    start and halves it when the energy rises; "plain": it keeps the plain
    solve's step from the identity (one extra iteration to find it).
    The network runs as one graph replay (WarmStartPredictor, built once
    per grid before any clock starts). Device times from CUDA events;
    warm_iters counts the iterations needed, warm_iters_run the ones
    executed (whole chunks). plain "multiscale": the plain method is the
    3-level multiscale solve (MULTISCALE), its finest-level energy the
    target, and it is also the fallback. Returns a list of dicts."""
    from .greedy import GreedyDeformationDataB200
    out = []
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    predictors: Dict[tuple, WarmStartPredictor] = {}
    for I0n, I1n in pairs:
        if I0n.shape not in predictors:
            predictors[I0n.shape] = WarmStartPredictor(net, I0n.shape)
        I0 = torch.from_numpy(I0n).cuda()
        I1 = torch.from_numpy(I1n).cuda()
        shape = tuple(I0.shape)
        it = _greedy(shape, max_pert)
        data = GreedyDeformationDataB200(I0, I1)
        # the warm path's handles exist before its clock starts, as the plain one's do
        it_w, data_w = _greedy(shape, max_pert), GreedyDeformationDataB200(I0, I1)
        it2, d2 = _greedy(shape, max_pert), GreedyDeformationDataB200(I0, I1)
        if plain == "multiscale":
            ms, ms2 = _multiscale(I0, I1), _multiscale(I0, I1)
            _plain_multiscale(ms)  # downsampling tables and graphs, outside the clock
        torch.cuda.synchronize()
        ev[0].record()
        if plain == "multiscale":
            _, e_plain = _plain_multiscale(ms)
        else:
            it.Run(data, plain_iters, update_first=True)
        ev[1].record()
        torch.cuda.synchronize()
        if plain != "multiscale":
            e_plain = it.Energies()
        target = float(e_plain[-1]) * (1.0 + tol)
        ev[2].record()
        eps = plain_step(I0, I1, it_w, data_w, max_pert) if policy == "plain" else None
        h0 = predictors[I0n.shape](I0, I1)
        ev[4].record()
        # past half the plain iteration count the warm path cannot win: cap it there
        h, k, en, reached, fell = refine(I0, I1, h0, target, plain_iters // 2, chunk, max_pert,
                                         it_w, data_w, step=eps, auto_reduce=(policy == "own"))
        run = len(en)  # one recorded energy per executed iteration
        if policy == "plain":
            k += 1  # the step-size iteration
            run += 1
        fallback = not reached
        if fallback:  # the warm start did not get there: the plain solve, unassisted
            if plain == "multiscale":
                _plain_multiscale(ms2)
                k += sum(n for _, n, _ in MULTISCALE)
                run += sum(n for _, n, _ in MULTISCALE)
            else:
                it2.Run(d2, plain_iters, update_first=True)
                k += plain_iters
                run += plain_iters
        ev[3].record()
        torch.cuda.synchronize()
        out.append({"plain_ms": ev[0].elapsed_time(ev[1]), "warm_ms": ev[2].elapsed_time(ev[3]),
                    "predict_ms": ev[2].elapsed_time(ev[4]), "warm_iters_run": run,
                    "plain_iters": (sum(n for _, n, _ in MULTISCALE) if plain == "multiscale"
                                    else plain_iters),
                    "warm_iters": int(k), "reached": bool(reached),
                    "fallback": bool(fallback), "plain_energy": float(e_plain[-1]),
                    "warm_start_energy": float(en[0]) if len(en) else float("nan"),
                    "identity_energy": float(e_plain[0])})
    return out


def train(net: "WarmStartNet", pairs, targets, epochs: int = 1, lr: float = 1e-3,
          log_every: int = 0):
    """Adam on the MSE between the prediction and the solver's displacement,
    one pair per step, pairs visited in a fixed shuffled order per epoch.
    Returns the per-step losses."""
    rng = np.random.default_rng(1234)
    losses = []
    dev_pairs = [(a if torch.is_tensor(a) else torch.from_numpy(a).cuda(),
                  b if torch.is_tensor(b) else torch.from_numpy(b).cuda()) for a, b in pairs]
    for ep in range(epochs):
        order = rng.permutation(len(pairs))
        for j, i in enumerate(order):
            I0, I1 = dev_pairs[i]
            losses.append(net.train_step(I0, I1, targets[i], lr).clone())
            if log_every and (j + 1) % log_every == 0:
                print(f"epoch {ep} step {j + 1} loss {float(losses[-1]):.5f}", flush=True)
    torch.cuda.synchronize()
    return [float(l) for l in torch.cat(losses).cpu()]


def _bf16_bits(a: np.ndarray) -> np.ndarray:
    b = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    return (((b + 0x7FFF + ((b >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def save_weights(net: "WarmStartNet", path: str):
    """Weights as BF16 bit patterns (what the convolutions compute with),
    biases as float32."""
    st = net.state()
    np.savez_compressed(path, **{f"w_{k}": _bf16_bits(v) for k, v in st["w"].items()},
                        **{f"b_{k}": v for k, v in st["b"].items()})


# committed trained weights: pair grid -> (file in atlaswerks_b200/data, network grid).
# The network runs at half the pair's grid on the downsampled pair (warm_h),
# trained on 2000 pairs of the pair generator at the pair's grid with the
# solver's displacements at the network's grid as targets.
# (warmstart_64.npz: the network at 64^3 on 64^3 pairs, the native-grid variant.)
TRAINED = {64: ("warmstart_64_net32.npz", 32), 128: ("warmstart_128.npz", 64)}


def trained(grid: int) -> "WarmStartNet":
    """The committed network for n^3 pairs (n in TRAINED), weights loaded."""
    import os
    if grid not in TRAINED:
        raise ValueError(f"no trained weights for {grid}^3 pairs (have {sorted(TRAINED)})")
    name, net_grid = TRAINED[grid]
    net = WarmStartNet((net_grid,) * 3)
    load_weights(net, os.path.join(os.path.dirname(__file__), "data", name))
    return net


def param_blob(net: "WarmStartNet") -> np.ndarray:
    """The network's parameters as aw_warmstart_create takes them: per layer
    in LAYERS order the FP32 weights [Cout][taps][Cin], then the biases."""
    parts = []
    for name, _, _, _ in LAYERS:
        parts.append(net.w[name].detach().float().cpu().numpy().ravel())
        parts.append(net.b[name].detach().float().cpu().numpy().ravel())
    return np.ascontiguousarray(np.concatenate(parts), dtype=np.float32)


class WarmStartB200:
    """The warm start through the C ABI (aw_warmstart_*): prediction as one
    captured graph and the refinement/fallback loop in the library, the
    path a C or C++ host uses. ``shape`` is the pair grid (nz, ny, nx)."""

    def __init__(self, net: "WarmStartNet", shape: Sequence[int], max_pert: float = 0.5):
        nz, ny, nx = (int(s) for s in shape)
        self.shape = (nz, ny, nx)
        blob = param_blob(net)
        self._h = ctypes.c_void_p()
        check(_lib.lib().aw_warmstart_create(nx, ny, nz, net.W, net.H, net.D,
                                             blob.ctypes.data, blob.size, float(max_pert),
                                             ctypes.byref(self._h)))

    def predict(self, I0: torch.Tensor, I1: torch.Tensor, h: torch.Tensor) -> torch.Tensor:
        check(_lib.lib().aw_warmstart_predict(self._h, _p(I0), _p(I1), _p(h[0]), _p(h[1]),
                                              _p(h[2]), _stream()))
        return h

    def register(self, I0: torch.Tensor, I1: torch.Tensor, h: torch.Tensor,
                 target_energy: float, max_refine_iters: int = 25, chunk: int = 3,
                 plain_iters: int = 50):
        """Returns (iterations executed, fell back to the plain solve)."""
        run, fb = ctypes.c_int(), ctypes.c_int()
        check(_lib.lib().aw_warmstart_register(self._h, _p(I0), _p(I1), float(target_energy),
                                               int(max_refine_iters), int(chunk),
                                               int(plain_iters), _p(h[0]), _p(h[1]), _p(h[2]),
                                               ctypes.byref(run), ctypes.byref(fb), _stream()))
        return run.value, bool(fb.value)

    def close(self):
        if self._h:
            _lib.lib().aw_warmstart_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def load_weights(net: "WarmStartNet", path: str):
    z = np.load(path)
    w = {}
    for k in net.w:
        a = z[f"w_{k}"]
        w[k] = (a.astype(np.uint32) << 16).view(np.float32) if a.dtype == np.uint16 else a
    net.load({"w": w, "b": {k: z[f"b_{k}"] for k in net.b}})


def main(argv=None):
    """Train on solver-generated pairs and evaluate on held-out seeds:
    python -m atlaswerks_b200.warmstart --n 64 --train 2000 --eval 256"""
    import argparse
    import json
    import os
    import time
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--eval", type=int, default=256)
    ap.add_argument("--epochs", type=int, default=2)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--weights", default="", help="load instead of training")
    ap.add_argument("--save", default="", help="where to write the trained weights")
    ap.add_argument("--json", default="", help="where to write the evaluation summary")
    ap.add_argument("--workers", type=int, default=min(32, os.cpu_count() or 1))
    ap.add_argument("--policy", default="own", choices=["own", "plain"])
    ap.add_argument("--net", type=int, default=0,
                    help="the network's grid (default: --n); smaller = predict on the "
                         "downsampled pair and upsample the deformation")
    a = ap.parse_args(argv)
    t0 = time.time()
    nn_grid = a.net or a.n
    net = WarmStartNet((nn_grid,) * 3)
    summary = {"grid": a.n, "net_grid": nn_grid, "n_train": a.train, "n_eval": a.eval,
               "parameters": n_parameters()}
    if a.weights:
        load_weights(net, a.weights)
    else:
        if nn_grid == a.n:
            train_pairs = make_pairs(range(a.train), a.n, a.workers)
            t1 = time.time()
            targets = [solver_target(torch.from_numpy(p[0]).cuda(),
                                     torch.from_numpy(p[1]).cuda()) for p in train_pairs]
        else:
            t1 = time.time()
            train_pairs, targets = coarse_training_set(range(a.train), a.n, nn_grid, a.workers)
        torch.cuda.synchronize()
        t2 = time.time()
        losses = train(net, train_pairs, targets, a.epochs, a.lr, log_every=500)
        t3 = time.time()
        summary.update({"data_s": t1 - t0, "targets_s": t2 - t1, "train_s": t3 - t2,
                        "epochs": a.epochs, "steps": len(losses),
                        "loss_first": float(np.mean(losses[:50])),
                        "loss_last": float(np.mean(losses[-50:]))})
        if a.save:
            save_weights(net, a.save)
        del train_pairs, targets
    eval_pairs = make_pairs(range(10_000_000, 10_000_000 + a.eval), a.n, a.workers)
    evaluate(net, eval_pairs[:2], policy=a.policy)  # warm-up: module loads, pools, graphs
    res = evaluate(net, eval_pairs, policy=a.policy)
    summary["policy"] = a.policy
    pm = float(np.sum([r["plain_ms"] for r in res]))
    wm = float(np.sum([r["warm_ms"] for r in res]))
    summary.update({
        "plain_ms_total": pm, "warm_ms_total": wm, "wall_ratio": wm / pm,
        "plain_pairs_per_s": 1000.0 * len(res) / pm, "warm_pairs_per_s": 1000.0 * len(res) / wm,
        "iters_plain_mean": float(np.mean([r["plain_iters"] for r in res])),
        "iters_warm_mean": float(np.mean([r["warm_iters"] for r in res])),
        "iters_warm_run_mean": float(np.mean([r["warm_iters_run"] for r in res])),
        "predict_ms_median": float(np.median([r["predict_ms"] for r in res])),
        "warm_ms_median": float(np.median([r["warm_ms"] for r in res])),
        "plain_ms_median": float(np.median([r["plain_ms"] for r in res])),
        "reached_fraction": float(np.mean([r["reached"] for r in res])),
        "fallback_fraction": float(np.mean([r["fallback"] for r in res])),
        "warm_start_energy_over_identity": float(np.median(
            [r["warm_start_energy"] / r["identity_energy"] for r in res])),
    })
    print(json.dumps(summary))
    if a.json:
        with open(a.json, "w") as f:
            json.dump({"summary": summary, "pairs": res}, f)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
