"""Error behaviour through the C ABI, against the oracle (both share the
reference's error model: Bitstream / Unsupported / InvalidInput, the decoder
state "as far as it got"). Corrupted, truncated and garbage packets, a stream
entered mid-way, and the pixel limit: after each error both decoders go on
with the same packets and must keep agreeing, frame for frame."""
import ctypes
import hashlib
import os

import numpy as np
import pytest

from conftest import VECTORS_DIR, read_packets

pytestmark = pytest.mark.gpu


def _status(fn, *a):
    """(status, [frame md5s]) of one decode_all call."""
    try:
        return 0, [hashlib.md5(f.packed()).hexdigest() for f in fn(*a)]
    except Exception as e:  # the binding's errors carry the status
        import rv9
        st = {rv9.BitstreamError: 1, rv9.UnsupportedError: 2, rv9.InvalidInputError: 3, rv9.DeviceError: 4}
        for cls, v in st.items():
            if isinstance(e, cls):
                return v, []
        if hasattr(e, "status"):
            return e.status, []
        raise


def _run_both(oracle_lib, packets, max_pixels=None):
    import rv9
    g = rv9.Decoder(0)
    o = oracle_lib.OracleDecoder()
    if max_pixels:
        g.set_max_pixels(max_pixels)
        o.set_max_pixels(max_pixels)
    got = []
    for i, p in enumerate(packets):
        a = _status(g.decode_all, p)
        b = _status(o.decode_all, p)
        assert a == b, f"packet {i}: gpu {a[0]}, oracle {b[0]}"
        got.append(a[0])
    g.close()
    return got


def test_corrupted_packets_match_the_oracle(oracle_lib):
    rng = np.random.default_rng(21)
    base = read_packets(os.path.join(VECTORS_DIR, "vp90-2-02-size-130x132.webm"))
    packets = list(base)
    # Truncations, header bit flips, garbage, an empty packet.
    packets[3] = packets[3][: len(packets[3]) // 2]
    b = bytearray(packets[5])
    b[1] ^= 0x40
    packets[5] = bytes(b)
    packets.insert(7, bytes(rng.integers(0, 256, 40, dtype=np.uint8)))
    packets.insert(8, b"")
    statuses = _run_both(oracle_lib, packets)
    assert any(s != 0 for s in statuses) and statuses[0] == 0


def test_stream_entered_midway_matches_the_oracle(oracle_lib):
    packets = read_packets(os.path.join(VECTORS_DIR, "vp90-2-05-resize.ivf"))
    statuses = _run_both(oracle_lib, packets[3:] + packets)
    assert statuses[0] == 1  # an inter frame with empty reference slots
    assert statuses[-1] == 0  # the full stream from its keyframe decodes


def test_pixel_limit_matches_the_oracle(oracle_lib):
    packets = read_packets(os.path.join(VECTORS_DIR, "vp90-2-02-size-130x132.webm"))
    statuses = _run_both(oracle_lib, packets[:3], max_pixels=100 * 100)
    assert statuses[0] == 2


def test_decode_returns_the_last_shown_frame():
    # rv9_decode (reference Decoder::decode): the last frame a packet shows.
    import rv9
    lib = rv9.load_library()
    packets = read_packets(os.path.join(VECTORS_DIR, "vp90-2-10-show-existing-frame2.webm"))
    a, b = rv9.Decoder(0), rv9.Decoder(0)
    try:
        for p in packets:
            frames = a.decode_all(p)
            out = rv9.CFrame()
            shown = ctypes.c_int()
            st = lib.rv9_decode(b._dec, p, len(p), ctypes.byref(out), ctypes.byref(shown))
            assert st == 0
            assert shown.value == (1 if frames else 0)
            if frames:
                assert ctypes.string_at(out.data, out.size) == frames[-1].packed()
                lib.rv9_frame_release(ctypes.byref(out))
    finally:
        a.close()
        b.close()
