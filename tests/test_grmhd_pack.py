"""Reading simulation output in the reference's nubhlight_pack format
(include/bh_rt.h, bh_grmhd_packed_read) on the CPU: metadata, samples,
checksum and validation errors. The files are written by this test in the
schema of the reference's tools/nubhlight_pack.cpp."""
from __future__ import annotations

import json

import numpy as np
import pytest

from oracle import grmhd_oracle as G


def frame(seed=0, shape=(12, 8, 10)):
    rng = np.random.default_rng(seed)
    f = rng.uniform(0.1, 1.0, shape + (4,)).astype(np.float32)
    return f


def test_read_metadata_and_samples(lib, tmp_path):
    from blackhole_b200 import rt

    f = frame()
    path = G.write_pack(tmp_path, "a", f, r_range=(2.5, 30.0))
    info, got = rt.read_packed(path)
    assert (info.n_r, info.n_theta, info.n_phi) == f.shape[:3]
    assert info.r_min == pytest.approx(2.5) and info.r_max == pytest.approx(30.0)
    assert [info.channels[k].value for k in range(4)] == [b"rho", b"u", b"v1", b"v2"]
    np.testing.assert_allclose(list(info.min_value), f.reshape(-1, 4).min(0), rtol=1e-6)
    np.testing.assert_array_equal(got, f)


def test_legacy_binary_key_and_absent_checksum(lib, tmp_path):
    from blackhole_b200 import rt

    f = frame(1)
    path = G.write_pack(tmp_path, "b", f, checksum=False, bin_key="binary_file")
    info, got = rt.read_packed(path)
    np.testing.assert_array_equal(got, f)
    assert info.r_min == pytest.approx(2.0)


@pytest.mark.parametrize("what", ["checksum", "dims", "format", "missing_bin"])
def test_invalid_packs_are_rejected(lib, tmp_path, what):
    from blackhole_b200 import rt

    f = frame(2)
    path = G.write_pack(tmp_path, "c", f, fmt="RGBA16F" if what == "format" else "RGBA32F",
                        dims=(12, 8, 11) if what == "dims" else None)
    if what == "checksum":
        raw = bytearray(open(tmp_path / "c.bin", "rb").read())
        raw[100] ^= 1
        open(tmp_path / "c.bin", "wb").write(bytes(raw))
    if what == "missing_bin":
        meta = json.load(open(path))
        del meta["bin"]
        json.dump(meta, open(path, "w"))
    with pytest.raises(RuntimeError) as e:
        rt.read_packed(path)
    key = {"checksum": "checksum", "dims": "floats", "format": "RGBA32F", "missing_bin": "bin"}[what]
    assert key in str(e.value)


def test_fnv1a64_known_answer():
    # FNV-1a 64 of the empty input is its offset basis; of "a" a published value
    assert G.fnv1a64_hex(b"") == "cbf29ce484222325"
    assert G.fnv1a64_hex(b"a") == "af63dc4c8601ec8c"
