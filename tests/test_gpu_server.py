"""The serving engine (include/rv9_server.h): each stream's frames are the
same in the mix as alone (the published MD5s), requests complete in order
per stream, admission waits for the HBM budget, and a bad packet fails only
its own request. Every test runs on the plain engine (each stream on its own
CUDA stream), on the plain engine with device parsing
(rv9_engine_set_device_parse: a stream's queued requests parsed on the GPU as
one batch) and on the batched one (rv9_engine_create_batched: the streams'
frames reconstructed together, one launch per stage per step). The
device-parse tests at the end decode generated streams whose frames the
device parser takes, mixed with frames it leaves to the host, against the
oracle."""
import hashlib
import os
import time

import pytest

from conftest import VECTORS_DIR, expected_md5s, read_packets

pytestmark = pytest.mark.gpu

MIX = [
    ("vp90-2-02-size-130x132.webm", 8),
    ("vp90-2-05-resize.ivf", 8),
    ("vp90-2-10-show-existing-frame2.webm", 8),
    ("vp90-2-13-mv-with-scaling.ivf", 8),
    ("vp91-2-04-yuv444.webm", 8),
    ("vp92-2-20-10bit-yuv420.webm", 10),
    ("vp93-2-20-12bit-yuv422.webm", 12),
    ("vp90-2-15-fuzz-flicker.webm", 8),
]


@pytest.fixture(params=[0, "dp", 1, 3], ids=["plain", "plain_device_parse", "batched_1group", "batched_3groups"])
def groups(request):
    return request.param


def _engine(groups, **kw):
    """An engine of the form `groups` names: 0 plain, "dp" plain with device
    parsing (batches of up to 4 requests), n > 0
    batched in n groups."""
    from rv9 import server
    if groups == "dp":
        return server.Engine(0, device_parse=True, window=4, **kw)
    return server.Engine(0, groups=groups, **kw)


def _drain(eng, expect, timeout_s=120):
    got = []
    t0 = time.time()
    while len(got) < expect and time.time() - t0 < timeout_s:
        got += eng.poll(timeout_ms=100)
    return got


def _md5s(done, sid):
    return [hashlib.md5(f.packed()).hexdigest() for c in done if c.stream == sid for f in c.frames]


def test_mix_equals_alone(groups):
    eng = _engine(groups, workers=8)
    try:
        sids, packets = {}, {}
        for name, bd in MIX:
            sids[name] = eng.open_stream(1920, 1080, bit_depth=bd, chroma=(0, 0))
            packets[name] = read_packets(os.path.join(VECTORS_DIR, name))
        # The streams' packets interleaved, as if they arrived together.
        total = 0
        for i in range(max(len(p) for p in packets.values())):
            for name, _ in MIX:
                if i < len(packets[name]):
                    eng.submit(sids[name], packets[name][i], tag=i)
                    total += 1
        for name, _ in MIX:
            eng.close_stream(sids[name])
        done = _drain(eng, total)
        assert len(done) == total
        for name, _ in MIX:
            cs = [c for c in done if c.stream == sids[name]]
            assert [c.tag for c in cs] == list(range(len(packets[name])))  # in order
            assert all(c.ok for c in cs), name
            assert all(c.latency_ms > 0 for c in cs)
            assert _md5s(done, sids[name]) == expected_md5s(os.path.join(VECTORS_DIR, name)), name
        st = eng.stats()
        assert st["streams_open"] == 0 and st["reserved_bytes"] == 0
        assert st["requests_completed"] == st["requests_submitted"] == total
        if groups == "dp":
            # The requests queued together went as batches (the vectors'
            # frames all adapt probabilities, so the host parsed them).
            assert st["device_parse_batches"] > 0
        elif groups:
            # Every reconstructed frame went through a step (steps of one
            # frame or more, as the frames arrived).
            assert 0 < st["batched_steps"] <= st["batched_frames"]
    finally:
        eng.close()


def test_admission_waits_for_the_budget(groups):
    from rv9 import server
    one = server.reservation(1920, 1080, 12, (0, 0))
    if groups == "dp":
        # The reservation with the device parser's buffers.
        probe = _engine(groups, workers=1)
        try:
            probe.open_stream(1920, 1080, bit_depth=12, chroma=(0, 0))
            one = probe.stats()["reserved_bytes"]
            assert one > server.reservation(1920, 1080, 12, (0, 0))
        finally:
            probe.close()
    eng = _engine(groups, hbm_budget=int(one * 1.5), workers=4)
    try:
        names = MIX[:3]
        sids = [eng.open_stream(1920, 1080, bit_depth=12, chroma=(0, 0)) for _ in names]
        st = eng.stats()
        assert st["streams_pending"] == 2 and st["reserved_bytes"] == one
        packets = [read_packets(os.path.join(VECTORS_DIR, n)) for n, _ in names]
        total = 0
        for sid, pk in zip(sids, packets):
            for i, p in enumerate(pk):
                eng.submit(sid, p, tag=i)
                total += 1
            eng.close_stream(sid)
        done = _drain(eng, total)
        assert len(done) == total and all(c.ok for c in done)
        for sid, (name, _) in zip(sids, names):
            assert _md5s(done, sid) == expected_md5s(os.path.join(VECTORS_DIR, name)), name
        assert eng.stats()["reserved_bytes"] == 0
    finally:
        eng.close()


def test_spec_over_budget_is_refused(groups):
    import rv9
    eng = _engine(groups, hbm_budget=1 << 20, workers=1)
    try:
        with pytest.raises(rv9.UnsupportedError):
            eng.open_stream(1920, 1080)
    finally:
        eng.close()


def test_a_bad_packet_fails_only_its_request(groups):
    name = "vp90-2-02-size-130x132.webm"
    eng = _engine(groups, workers=4)
    try:
        good = eng.open_stream(352, 288)
        bad = eng.open_stream(352, 288)
        pk = read_packets(os.path.join(VECTORS_DIR, name))
        eng.submit(bad, b"\x00\x01\x02garbage", tag=99)
        for i, p in enumerate(pk):
            eng.submit(good, p, tag=i)
        eng.close_stream(good)
        eng.close_stream(bad)
        done = _drain(eng, len(pk) + 1)
        assert len(done) == len(pk) + 1
        badc = [c for c in done if c.stream == bad]
        assert len(badc) == 1 and not badc[0].ok and badc[0].tag == 99
        assert _md5s(done, good) == expected_md5s(os.path.join(VECTORS_DIR, name))
    finally:
        eng.close()


def test_free_with_requests_in_flight(groups):
    # Freeing the engine drains every stream, with completions never polled.
    eng = _engine(groups, workers=2)
    sid = eng.open_stream(352, 288)
    for i, p in enumerate(read_packets(os.path.join(VECTORS_DIR, "vp90-2-02-size-130x132.webm"))):
        eng.submit(sid, p, tag=i)
    eng.close()


def _submit_all(eng, sid, packets, first_tag=0):
    for i, p in enumerate(packets):
        eng.submit(sid, p, tag=first_tag + i)


@pytest.mark.parametrize("window", [2, 8])
def test_device_parse_streams_match_the_oracle(window, oracle_lib):
    """Generated streams, their requests queued deep: error-resilient ones
    (every frame parsed on the device) and linked ones (frames that read the
    previous frame's motion vectors, every few a probability-adapting frame
    the host parses between device batches). Every request's frames against
    the oracle's, in order."""
    from rv9 import server
    from conftest import oracle_frames
    from streams_cases import CASES, LINKED, generate, generate_linked
    cases = [("cif_8bit_q60", generate("cif_8bit_q60")[0], CASES["cif_8bit_q60"]),
             ("720p_10bit_422_q50", generate("720p_10bit_422_q50")[0], CASES["720p_10bit_422_q50"]),
             ("cif_8bit_linked", generate_linked("cif_8bit_linked"), LINKED["cif_8bit_linked"]),
             ("720p_8bit_linked", generate_linked("720p_8bit_linked"), LINKED["720p_8bit_linked"])]
    eng = server.Engine(0, workers=4, device_parse=True, window=window)
    try:
        sids = {}
        for name, packets, shape in cases:
            sids[name] = eng.open_stream(shape[0], shape[1], bit_depth=shape[2], chroma=shape[3])
        total = 0
        for name, packets, _ in cases:
            _submit_all(eng, sids[name], packets)
            total += len(packets)
            eng.close_stream(sids[name])
        done = _drain(eng, total)
        assert len(done) == total
        for name, packets, _ in cases:
            cs = [c for c in done if c.stream == sids[name]]
            assert [c.tag for c in cs] == list(range(len(packets))), name
            assert all(c.ok for c in cs), name
            want = [m for m, _ in oracle_frames(oracle_lib, packets)]
            assert _md5s(done, sids[name]) == want, name
        st = eng.stats()
        assert st["device_parse_batches"] > 0
        assert 0 < st["device_parsed_frames"] <= total
    finally:
        eng.close()


def test_device_parse_corrupted_request(oracle_lib):
    """A request whose tile data is corrupted fails as it does with host
    parsing, the requests before it decode exactly, and the stream decodes
    exactly again from its next key frame."""
    from rv9 import server
    from conftest import oracle_frames
    from streams_cases import generate
    packets, _ = generate("cif_8bit_q60")
    bad = list(packets)
    flipped = bytearray(bad[3])
    for i in range(len(flipped) // 2, len(flipped)):
        flipped[i] ^= 0xA5
    bad[3] = bytes(flipped)
    want = [m for m, _ in oracle_frames(oracle_lib, packets)]
    status = {}
    for form in ("host", "device"):
        eng = server.Engine(0, workers=2, window=8, device_parse=form == "device")
        try:
            sid = eng.open_stream(352, 288)
            _submit_all(eng, sid, bad)
            done = _drain(eng, len(bad))
            assert [c.tag for c in done] == list(range(len(bad))), form
            assert all(c.ok for c in done[:3]), form
            assert _md5s(done[:3], sid) == want[:3], form
            status[form] = done[3].status
            # Then the stream from its key frame again.
            _submit_all(eng, sid, packets[:3], first_tag=100)
            again = _drain(eng, 3)
            assert all(c.ok for c in again) and _md5s(again, sid) == want[:3], form
            eng.close_stream(sid)
        finally:
            eng.close()
    assert status["host"] == status["device"]



def _superframe(frames):
    """The frames as one VP9 superframe (the index of Annex B: a marker byte,
    4-byte little-endian sizes, the marker again)."""
    marker = 0xC0 | (3 << 3) | (len(frames) - 1)
    index = bytes([marker]) + b"".join(len(f).to_bytes(4, "little") for f in frames) + bytes([marker])
    return b"".join(frames) + index


def test_a_request_showing_two_frames(groups, oracle_lib):
    """A request whose packet shows two frames (two shown frames joined in a
    superframe): the first goes to the request's output buffer, the second
    to its own heap buffer; both exact, in order."""
    from conftest import oracle_frames
    from streams_cases import generate
    packets, _ = generate("cif_8bit_q60")
    want = [m for m, _ in oracle_frames(oracle_lib, packets)]
    joined = [packets[0], _superframe([packets[1], packets[2]])] + packets[3:]
    eng = _engine(groups, workers=2)
    try:
        sid = eng.open_stream(352, 288)
        _submit_all(eng, sid, joined)
        done = _drain(eng, len(joined))
        assert [c.tag for c in done] == list(range(len(joined)))
        assert all(c.ok for c in done)
        assert [c.n_frames for c in done][:3] == [1, 2, 1]
        assert _md5s(done, sid) == want
        eng.close_stream(sid)
    finally:
        eng.close()
