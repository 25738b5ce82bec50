"""Device primitives over the C ABI, on torch CUDA tensors.

Torch supplies device memory and streams; every computation is a kernel of
libaw_b200.so. Images are float32 [nz, ny, nx] (x fastest); vector fields
float32 [3, nz, ny, nx] (planar x | y | z), the reference's cplVector3DArray
layout.
"""
from __future__ import annotations

from typing import Sequence, Tuple

import torch

from . import _lib
from ._lib import check

BG_PARTIAL_ID, BG_ID, BG_PARTIAL_ZERO, BG_ZERO, BG_CLAMP, BG_WRAP = range(6)


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _dims(t: torch.Tensor) -> Tuple[int, int, int]:
    nz, ny, nx = t.shape[-3:]
    return nx, ny, nz


def _check_image(t: torch.Tensor, name: str) -> None:
    if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous() and t.dim() == 3):
        raise ValueError(f"{name} must be a contiguous float32 CUDA tensor [nz, ny, nx]")


def _check_field(t: torch.Tensor, name: str) -> None:
    if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous() and t.dim() == 4
            and t.shape[0] == 3):
        raise ValueError(f"{name} must be a contiguous float32 CUDA tensor [3, nz, ny, nx]")


def _p(t: torch.Tensor) -> int:
    return t.data_ptr()


def identity(shape: Sequence[int], device="cuda") -> torch.Tensor:
    nz, ny, nx = shape
    z, y, x = torch.meshgrid(torch.arange(nz, device=device), torch.arange(ny, device=device),
                             torch.arange(nx, device=device), indexing="ij")
    return torch.stack([x, y, z]).float().contiguous()


def apply(img: torch.Tensor, h: torch.Tensor, background: float = 0.0) -> torch.Tensor:
    """img(h(x)) — HField3DUtils::apply / cudaHField3DUtils::apply."""
    _check_image(img, "img")
    _check_field(h, "h")
    out = torch.empty_like(img)
    check(_lib.lib().aw_apply(_p(img), _p(h[0]), _p(h[1]), _p(h[2]), _p(out), *_dims(img),
                              background, _stream()))
    return out


def gradient(img: torch.Tensor, spacing=(1.0, 1.0, 1.0), wrap: bool = False) -> torch.Tensor:
    """Array3DUtils::computeGradient / cplComputeGradient."""
    _check_image(img, "img")
    g = torch.empty((3,) + tuple(img.shape), device=img.device, dtype=torch.float32)
    check(_lib.lib().aw_gradient(_p(img), _p(g[0]), _p(g[1]), _p(g[2]), *_dims(img), *spacing,
                                 int(wrap), _stream()))
    return g


def compose_hv(g: torch.Tensor, v: torch.Tensor, spacing=(1.0, 1.0, 1.0), scale: float = 1.0,
               direction: int = 1, background: int = BG_PARTIAL_ID) -> torch.Tensor:
    """g(x + direction*scale*v(x)/sp) — composeHV (+1) / composeHVInv (-1)."""
    _check_field(g, "g")
    _check_field(v, "v")
    o = torch.empty_like(g)
    check(_lib.lib().aw_compose_hv(_p(g[0]), _p(g[1]), _p(g[2]), _p(v[0]), _p(v[1]), _p(v[2]),
                                   _p(o[0]), _p(o[1]), _p(o[2]), *_dims(g), *spacing, scale,
                                   direction, background, _stream()))
    return o


def compose_vh(v: torch.Tensor, g: torch.Tensor, spacing=(1.0, 1.0, 1.0), scale: float = 1.0,
               direction: int = -1, background: int = BG_PARTIAL_ZERO) -> torch.Tensor:
    """g(x) + direction*(scale*v)(g(x))/sp — composeVH (+1) / composeVHInv (-1)."""
    _check_field(g, "g")
    _check_field(v, "v")
    o = torch.empty_like(g)
    check(_lib.lib().aw_compose_vh(_p(v[0]), _p(v[1]), _p(v[2]), _p(g[0]), _p(g[1]), _p(g[2]),
                                   _p(o[0]), _p(o[1]), _p(o[2]), *_dims(g), *spacing, scale,
                                   direction, background, _stream()))
    return o


def splat(img: torch.Tensor, h: torch.Tensor, background: float = 0.0) -> torch.Tensor:
    """Adjoint of apply: HField3DUtils::forwardApply(normalize=false) /
    cplSplat3DH, deterministic (no float atomics)."""
    _check_image(img, "img")
    _check_field(h, "h")
    out = torch.empty_like(img)
    check(_lib.lib().aw_splat(_p(img), _p(h[0]), _p(h[1]), _p(h[2]), _p(out), *_dims(img),
                              background, _stream()))
    return out


def downsample(img: torch.Tensor, new_shape, spacing=(1.0, 1.0, 1.0)) -> torch.Tensor:
    """ImageUtils::gaussianDownsample to new_shape = (nz, ny, nx)."""
    _check_image(img, "img")
    out = torch.empty(tuple(new_shape), device=img.device, dtype=torch.float32)
    mz, my, mx = new_shape
    check(_lib.lib().aw_downsample(_p(img), *_dims(img), *map(float, spacing), _p(out), mx, my,
                                   mz, _stream()))
    return out


def resample_image(img: torch.Tensor, new_shape, spacing, new_spacing) -> torch.Tensor:
    """ImageUtils::resampleNew (clamped linear, origin 0) onto new_shape =
    (nz, ny, nx) with new_spacing: MultiscaleManager's image upsampling."""
    _check_image(img, "img")
    out = torch.empty(tuple(new_shape), device=img.device, dtype=torch.float32)
    mz, my, mx = new_shape
    check(_lib.lib().aw_resample_image(_p(img), *_dims(img), *map(float, spacing), _p(out), mx,
                                       my, mz, *map(float, new_spacing), _stream()))
    return out


def upsample_hfield(h: torch.Tensor, new_shape, rescale: bool = True) -> torch.Tensor:
    """hToVelocity + resampleNew(CLAMP) + velocityToH to new_shape."""
    _check_field(h, "h")
    out = torch.empty((3,) + tuple(new_shape), device=h.device, dtype=torch.float32)
    mz, my, mx = new_shape
    check(_lib.lib().aw_upsample_hfield(_p(h[0]), _p(h[1]), _p(h[2]), *_dims(h), _p(out[0]),
                                        _p(out[1]), _p(out[2]), mx, my, mz, int(rescale),
                                        _stream()))
    return out

