"""CPU-only checks: the oracle's FFT against numpy FP64, the C ABI library
loads and exports every entry point its header declares, and host-side
argument validation (no device calls)."""
import ctypes
import os

import numpy as np
import pytest

from atlaswerks_b200 import _lib


def test_fft64_vs_numpy(oracle):
    """The FP64 FFT under the oracle and the FFTW shim, via the fluid operator
    with alpha = beta = 0, gamma = 1: L = I, so L^-1 f must return f."""
    rng = np.random.default_rng(0)
    for shape in [(8, 9, 10), (17, 3, 31), (16, 16, 16)]:
        f = rng.normal(0, 1, (3,) + shape)
        out = oracle.fluid_f64(f, (1, 1, 1), 0.0, 0.0, 1.0, True)
        assert np.abs(out - f).max() <= 1e-12


def test_fluid_fp64_vs_numpy(oracle):
    rng = np.random.default_rng(1)
    shape, sp = (10, 12, 14), (1.0, 1.3, 0.8)
    f = rng.normal(0, 1, (3,) + shape)
    nz, ny, nx = shape
    F = [np.fft.fftn(f[c]) for c in range(3)]
    kz, ky, kx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    cw = [(2 * np.cos(2 * np.pi * k / n) - 2) / s ** 2 for k, n, s in ((kx, nx, sp[0]), (ky, ny, sp[1]), (kz, nz, sp[2]))]
    sw = [np.sin(2 * np.pi * k / n) / s for k, n, s in ((kx, nx, sp[0]), (ky, ny, sp[1]), (kz, nz, sp[2]))]
    a, b, g = 0.01, 0.01, 0.001
    lam = -a * (cw[0] + cw[1] + cw[2]) + g
    L = np.zeros(kx.shape + (3, 3))
    for i in range(3):
        L[..., i, i] = lam - b * cw[i]
        for j in range(3):
            if i != j:
                L[..., i, j] = b * sw[i] * sw[j]
    V = np.linalg.solve(L, np.stack(F, -1)[..., None])[..., 0]
    want = np.stack([np.fft.ifftn(V[..., c]).real for c in range(3)])
    got = oracle.fluid_f64(f, sp, a, b, g, True)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


def test_library_exports_every_header_symbol():
    path = _lib.build()
    lib = ctypes.CDLL(path)
    names = _lib.header_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # every declared entry point has a Python signature
    assert set(names) <= set(_lib.SIGNATURES)


def test_last_error_and_version_without_gpu():
    lib = _lib.lib()
    assert b"sm_100a" in lib.aw_version()
    # argument validation happens before any device call
    h = ctypes.c_void_p()
    assert lib.aw_fluid_create(1, 16, 16, 1.0, 1.0, 1.0, 0.01, 0.01, 0.001, ctypes.byref(h)) != 0
    assert b">= 2" in lib.aw_last_error()
    assert lib.aw_greedy_create(16, 16, 16, 1.0, 1.0, 1.0, 0.01, 0.01, 0.0, 0.5,
                                ctypes.byref(h)) != 0
    assert b"gamma" in lib.aw_last_error()
    assert lib.aw_apply(None, None, None, None, None, 4, 4, 4, 0.0, None) != 0
    assert b"null" in lib.aw_last_error()


def test_host_mirror_rejects_unsupported_kernel_params():
    from atlaswerks_b200.greedy import DiffOperB200, DiffOperParam
    op = DiffOperB200()
    with pytest.raises(ValueError):
        op.SetSize((16, 16, 16), (1, 1, 1), DiffOperParam(UseEigenLUT=True))


def test_static_splat_capacity_query():
    """aw_splat_static_fits answers from the scratch formula the header
    states, without a GPU: 88^3 fits the fixed array, 89^3 does not."""
    from atlaswerks_b200 import _lib
    L = _lib.lib()
    assert L.aw_splat_static_fits(88, 88, 88) == 1
    assert L.aw_splat_static_fits(89, 89, 89) == 0
    assert L.aw_splat_static_fits(0, 8, 8) == 0
    assert L.aw_splat_static_fits(400, 100, 1) == 1
