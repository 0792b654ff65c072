"""The emulator's save format (JSON header + little-endian binary blob), on CPU."""
import json

import numpy as np
import pytest

from disort_b200 import surrogate


def test_blob_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    blocks = [("params", rng.standard_normal(1000).astype(np.float32)),
              ("fmean", rng.standard_normal(329)), ("mask", np.arange(12, dtype=np.int32).reshape(3, 4))]
    p = str(tmp_path / "w")
    surrogate.write_blob(p, dict(format="x", version=3, note="n"), blocks)
    h, b = surrogate.read_blob(p, "x", 3)
    assert h["note"] == "n" and h["blob_bytes"] == sum(a.nbytes for _, a in blocks)
    for name, a in blocks:
        assert b[name].dtype == a.dtype and b[name].shape == a.shape
        np.testing.assert_array_equal(b[name], a)


def test_blob_rejects_wrong_format_version_and_truncation(tmp_path):
    p = str(tmp_path / "w")
    surrogate.write_blob(p, dict(format="x", version=1), [("a", np.ones(8))])
    with pytest.raises(ValueError, match="format"):
        surrogate.read_blob(p, "y", 1)
    with pytest.raises(ValueError, match="version"):
        surrogate.read_blob(p, "x", 2)
    with open(p + ".bin", "r+b") as f:
        f.truncate(40)
    with pytest.raises(ValueError, match="40 bytes"):
        surrogate.read_blob(p, "x", 1)
    h = json.load(open(p + ".json"))
    assert h["blocks"][0]["dtype"] == "<f8"
