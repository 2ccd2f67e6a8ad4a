"""The oracle (CPU restatement of the reference decoder) against the
published per-frame MD5s of the reference's committed conformance vectors
(rivet-vp9 tests/committed_vectors.rs)."""
import hashlib
import os

import pytest

from conftest import expected_md5s, read_packets, vector_paths


def decode_md5s(oracle_mod, path, threads=1):
    dec = oracle_mod.OracleDecoder(threads=threads)
    out = []
    for p in read_packets(path):
        for f in dec.decode_all(p):
            out.append(hashlib.md5(f.packed()).hexdigest())
    return out


def test_fifteen_vectors_present():
    assert len(vector_paths()) == 15


@pytest.mark.parametrize("path", vector_paths(), ids=os.path.basename)
def test_oracle_matches_published_md5(oracle_lib, path):
    assert decode_md5s(oracle_lib, path) == expected_md5s(path)


@pytest.mark.parametrize("name", ["vp90-2-05-resize.ivf", "vp93-2-20-12bit-yuv422.webm"])
def test_tile_threads_do_not_change_output(oracle_lib, name):
    path = os.path.join(os.path.dirname(vector_paths()[0]), name)
    assert decode_md5s(oracle_lib, path, threads=4) == expected_md5s(path)


def test_legacy_profile1_444_is_detected(oracle_lib):
    # The pre-final profile 1 stream needs 4:2:0 chroma transform sizes; the
    # final-syntax 4:4:4 stream must not be taken for it.
    d = os.path.dirname(vector_paths()[0])
    for name in ("vp91-2-04-yv444.webm", "vp91-2-04-yuv444.webm"):
        p = os.path.join(d, name)
        assert decode_md5s(oracle_lib, p) == expected_md5s(p)


def test_bitstream_errors_are_values(oracle_lib):
    dec = oracle_lib.OracleDecoder()
    with pytest.raises(oracle_lib.OracleError) as e:
        dec.decode_all(b"\x00\x01\x02")
    assert e.value.status == 1
