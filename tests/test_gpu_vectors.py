"""GPU parity: the CUDA decoder (through its C ABI) against the published
per-frame MD5s of the 15 conformance vectors and, frame by frame, against the
oracle. Bit-exact."""
import hashlib
import os

import pytest

from conftest import expected_md5s, read_packets, vector_paths

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rv9mod():
    import rv9
    return rv9


@pytest.mark.parametrize("path", vector_paths(), ids=os.path.basename)
def test_gpu_matches_published_md5(rv9mod, path):
    dec = rv9mod.Decoder()
    got = []
    for p in read_packets(path):
        for f in dec.decode_all(p):
            got.append(hashlib.md5(f.packed()).hexdigest())
    assert got == expected_md5s(path)


@pytest.mark.parametrize("path", vector_paths(), ids=os.path.basename)
def test_gpu_equals_oracle_frame_by_frame(rv9mod, oracle_lib, path):
    dec = rv9mod.Decoder()
    ref = oracle_lib.OracleDecoder()
    for i, p in enumerate(read_packets(path)):
        a = dec.decode_all(p)
        b = ref.decode_all(p)
        assert len(a) == len(b)
        for fa, fb in zip(a, b):
            assert (fa.width, fa.height, fa.bit_depth) == (fb.width, fb.height, fb.bit_depth)
            assert fa.packed() == fb.packed(), f"packet {i}"
