"""rv9_sequence_run_noalloc (the replay that allocates no device memory)
against rv9_sequence_run, both called through the C ABI.

The no-allocation entry point keeps the wavefront scratch in a fixed static
device array shared by every call on the device and takes its frames from the
decoder's pool. Each case runs the existing entry point twice, the new one
twice in a row, then the existing one again, and requires every reference
slot to come out byte-identical each time. This file sorts last so that it
also runs after every other GPU test in the same process."""
import ctypes
import os

import pytest

from conftest import VECTORS_DIR, read_packets

pytestmark = pytest.mark.gpu

RV9_OK = 0
RV9_INVALID_INPUT = 3
SLOT_CAP = 4 << 20

CASES = [
    "vp90-2-02-size-130x132.webm",
    "vp90-2-05-resize.ivf",                  # several frame sizes in the pool
    "vp90-2-10-show-existing-frame2.webm",
    "vp90-2-13-mv-with-scaling.ivf",         # scaled references
    "vp91-2-04-yuv444.webm",
    "vp92-2-20-10bit-yuv420.webm",           # 16-bit samples
    "vp93-2-20-12bit-yuv422.webm",
]


def _slots(lib, dec):
    """The packed planes of the eight reference slots (None when empty)."""
    out = []
    buf = ctypes.create_string_buffer(SLOT_CAP)
    n = ctypes.c_size_t()
    for s in range(8):
        st = lib.rv9_decoder_download_slot(dec._dec, s, buf, SLOT_CAP, ctypes.byref(n))
        out.append(buf.raw[:n.value] if st == RV9_OK else None)
    return out


def _run(lib, dec, seq):
    ms = ctypes.c_double()
    st = lib.rv9_sequence_run(dec._dec, seq._h, 0, ctypes.byref(ms))
    assert st == RV9_OK, lib.rv9_last_error(dec._dec)


def _run_noalloc(lib, dec, seq):
    ms = ctypes.c_double()
    st = lib.rv9_sequence_run_noalloc(dec._dec, seq._h, ctypes.byref(ms))
    assert st == RV9_OK, lib.rv9_last_error(dec._dec)
    assert ms.value > 0


@pytest.mark.parametrize("name", CASES)
def test_noalloc_matches_sequence_run(name):
    import torch

    import rv9
    lib = rv9.load_library()
    dec = rv9.Decoder(0)
    seq = dec.load_sequence(read_packets(os.path.join(VECTORS_DIR, name)))
    try:
        _run(lib, dec, seq)
        want = _slots(lib, dec)
        assert any(s is not None for s in want)
        _run(lib, dec, seq)
        assert _slots(lib, dec) == want
        free0 = torch.cuda.mem_get_info(0)[0]
        for call in range(2):
            _run_noalloc(lib, dec, seq)
            assert _slots(lib, dec) == want, f"no-alloc call {call + 1}"
        assert torch.cuda.mem_get_info(0)[0] == free0
        _run(lib, dec, seq)
        assert _slots(lib, dec) == want
    finally:
        seq.free()
        dec.close()


def test_noalloc_refuses_an_empty_pool():
    import rv9
    lib = rv9.load_library()
    dec = rv9.Decoder(0)
    seq = dec.load_sequence(read_packets(os.path.join(VECTORS_DIR, "vp90-2-02-size-130x132.webm")))
    try:
        ms = ctypes.c_double()
        st = lib.rv9_sequence_run_noalloc(dec._dec, seq._h, ctypes.byref(ms))
        assert st == RV9_INVALID_INPUT
        assert b"pool" in lib.rv9_last_error(dec._dec)
        # The decoder stays usable, and the pool then covers the sequence.
        _run(lib, dec, seq)
        want = _slots(lib, dec)
        _run_noalloc(lib, dec, seq)
        assert _slots(lib, dec) == want
    finally:
        seq.free()
        dec.close()


def test_noalloc_refuses_a_frame_beyond_the_scratch():
    # 8192x2048: 262144 8x8 blocks need 1 MiB of loop-filter records alone,
    # past the fixed 1 MiB array.
    import rv9
    from rv9 import streams
    pkts = streams.generate(streams.config(8192, 2048, 1, 120, tile_cols_log2=2))
    lib = rv9.load_library()
    dec = rv9.Decoder(0)
    seq = dec.load_sequence(pkts)
    try:
        _run(lib, dec, seq)
        ms = ctypes.c_double()
        st = lib.rv9_sequence_run_noalloc(dec._dec, seq._h, ctypes.byref(ms))
        assert st == RV9_INVALID_INPUT
        assert b"fixed scratch" in lib.rv9_last_error(dec._dec)
    finally:
        seq.free()
        dec.close()
