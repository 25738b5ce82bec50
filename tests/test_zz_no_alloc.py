"""aw_splat_static: the splat entry point for callers that may not allocate
device memory while they run (a host that owns all device memory through
its own pool, or a latency-critical loop where an allocation could block or
fail). Its scratch is a fixed array inside the library, so it must give the
same image as aw_splat, the entry point that takes scratch from the
stream-ordered allocator, on back-to-back calls that reuse that array.

Collected last on purpose (file name), so that a run stopping at the first
failure has already run every other test; it also passes alone.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from atlaswerks_b200 import _lib  # noqa: E402
from oracle import identity  # noqa: E402

pytestmark = pytest.mark.gpu


def _splat(fn, img, h, shape):
    nz, ny, nx = shape
    out = torch.full(shape, float("nan"), device="cuda")
    rc = getattr(_lib.lib(), fn)(img.data_ptr(), h[0].data_ptr(), h[1].data_ptr(),
                                 h[2].data_ptr(), out.data_ptr(), nx, ny, nz, 0.0,
                                 torch.cuda.current_stream().cuda_stream)
    assert rc == 0, _lib.lib().aw_last_error().decode()
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("shape", [(40, 36, 32), (17, 9, 31)])
def test_static_scratch_splat_matches_allocating_splat(shape):
    rng = np.random.default_rng(7)
    # two different inputs back to back: the second call must not see the
    # first call's bucket contents
    cases = []
    for k in range(2):
        img = torch.from_numpy(rng.normal(0, 1, shape).astype(np.float32)).cuda()
        h = torch.from_numpy(identity(shape) +
                             rng.normal(0, 1.0 + 2.0 * k, (3,) + shape).astype(np.float32)).cuda()
        cases.append((img, h))
    for img, h in cases:
        want = _splat("aw_splat", img, h, shape)
        got = _splat("aw_splat_static", img, h, shape)
        # the splat is deterministic and bit-exact, so equality is the tolerance
        assert torch.equal(got, want)


def test_static_scratch_rejects_grids_beyond_its_capacity():
    shape = (128, 128, 128)
    t = torch.zeros(shape, device="cuda")
    h = torch.zeros((3,) + shape, device="cuda")
    nz, ny, nx = shape
    rc = _lib.lib().aw_splat_static(t.data_ptr(), h[0].data_ptr(), h[1].data_ptr(),
                                    h[2].data_ptr(), t.data_ptr(), nx, ny, nz, 0.0, None)
    assert rc != 0
    assert b"more than the fixed" in _lib.lib().aw_last_error()
