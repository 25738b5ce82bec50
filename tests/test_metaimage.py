"""MetaImage writing and reading (atlaswerks_b200.metaimage): scalar volumes
and 3-component fields survive a round trip bit for bit, the header carries
spacing and origin, and the committed fixture from the reference's own
bullseye files reads back as stored."""
import os

import numpy as np
import pytest

from atlaswerks_b200.metaimage import read_mha, write_mha

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("shape", [(5, 7, 9), (3, 5, 7, 9)])
def test_round_trip(tmp_path, shape):
    rng = np.random.default_rng(0)
    a = rng.normal(0, 1, shape).astype(np.float32)
    p = str(tmp_path / "v.mha")
    write_mha(p, a, (2.0, 2.06452, 1.77778), (1.0, -2.0, 0.5))
    b, sp = read_mha(p)
    assert b.shape == a.shape and np.array_equal(a, b)
    assert sp == (2.0, 2.06452, 1.77778)
    hdr = open(p, "rb").read(600).decode("latin-1")
    assert "Offset = 1.0 -2.0 0.5" in hdr
    assert ("ElementNumberOfChannels = 3" in hdr) == (len(shape) == 4)


def test_fixture_images_write_and_read(tmp_path):
    z = np.load(os.path.join(HERE, "golden", "greedy_bullseye.npz"))
    p = str(tmp_path / "base.mha")
    write_mha(p, z["baseline_def_image"], tuple(z["sp"]))
    b, sp = read_mha(p)
    assert np.array_equal(b, z["baseline_def_image"])
    assert np.allclose(sp, z["sp"])


def test_rejects_what_it_cannot_read(tmp_path):
    p = tmp_path / "bad.mha"
    p.write_bytes(b"NDims = 3\nDimSize = 2 2 2\nElementType = MET_SHORT\nElementDataFile = LOCAL\n"
                  + bytes(16))
    with pytest.raises(ValueError):
        read_mha(str(p))
