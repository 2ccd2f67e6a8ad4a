"""Shared test setup: the `gpu` marker, paths, the conformance vectors."""
import glob
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "rivet-vp9_b200")
for p in (PKG, os.path.join(REPO, "oracle"), REPO):
    if p not in sys.path:
        sys.path.insert(0, p)

VECTORS_DIR = os.path.join(REPO, "tests", "golden", "vectors")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def vector_paths():
    return sorted(glob.glob(os.path.join(VECTORS_DIR, "*.webm")) + glob.glob(os.path.join(VECTORS_DIR, "*.ivf")))


def expected_md5s(path):
    with open(path + ".md5") as f:
        return [l.split()[0] for l in f if l.strip()]


def read_packets(path):
    from rv9.containers import packets
    with open(path, "rb") as f:
        return packets(f.read())


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle as oracle_mod
    oracle_mod.build()
    return oracle_mod


def oracle_frames(oracle_mod, packets, threads=4):
    """(md5, packed byte size) of every frame the oracle shows for `packets`,
    decoded in order from a fresh decoder."""
    import hashlib
    dec = oracle_mod.OracleDecoder(threads=threads)
    out = []
    for p in packets:
        for f in dec.decode_all(p):
            data = f.packed()
            out.append((hashlib.md5(data).hexdigest(), len(data)))
    return out


def split_md5s(buf, sizes):
    """MD5s of consecutive frames of the given sizes in `buf` (a frame
    sink's contents)."""
    import hashlib
    out, off = [], 0
    for n in sizes:
        out.append(hashlib.md5(buf[off:off + n]).hexdigest())
        off += n
    return out


class FrameSinks:
    """Pinned host frame sinks on decoders: every frame each decoder shows
    while they are attached is copied there (rv9_decoder_set_frame_sink)."""

    def __init__(self, decs, cap):
        import torch
        self.decs = list(decs)
        self.bufs = [torch.empty(cap, dtype=torch.uint8, pin_memory=True) for _ in self.decs]
        self.cap = cap
        self.reset()

    def reset(self):
        for d, b in zip(self.decs, self.bufs):
            d.set_frame_sink(b.data_ptr(), self.cap)

    def md5s(self, i, sizes):
        """Decoder i's sink split by `sizes`; asserts nothing was dropped and
        the sink holds exactly those frames."""
        frames, used, dropped = self.decs[i].frame_sink_state()
        assert dropped == 0, f"decoder {i}: {dropped} frames did not fit the sink"
        assert frames == len(sizes) and used == sum(sizes), (frames, len(sizes), used, sum(sizes))
        return split_md5s(bytes(self.bufs[i][:used].numpy()), sizes)

    def detach(self):
        for d in self.decs:
            d.set_frame_sink(0, 0)
