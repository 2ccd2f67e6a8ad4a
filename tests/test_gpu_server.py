"""The serving engine (include/rv9_server.h): each stream's frames are the
same in the mix as alone (the published MD5s), requests complete in order
per stream, admission waits for the HBM budget, and a bad packet fails only
its own request. Every test runs on the plain engine (each stream on its own
CUDA stream) and on the batched one (rv9_engine_create_batched: the streams'
frames reconstructed together, one launch per stage per step)."""
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


@pytest.fixture(params=[0, 1, 3], ids=["plain", "batched_1group", "batched_3groups"])
def groups(request):
    return request.param


def _drain(eng, expect, timeout_s=120):
    got = []
    t0 = time.time()
    while len(got) < expect and time.time() - t0 < timeout_s:
        got += eng.poll(timeout_ms=100)
    return got


def _md5s(done, sid):
    return [hashlib.md5(f.packed()).hexdigest() for c in done if c.stream == sid for f in c.frames]


def test_mix_equals_alone(groups):
    from rv9 import server
    eng = server.Engine(0, workers=8, groups=groups)
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
        if groups:
            # Every reconstructed frame went through a step (steps of one
            # frame or more, as the frames arrived).
            assert 0 < st["batched_steps"] <= st["batched_frames"]
    finally:
        eng.close()


def test_admission_waits_for_the_budget(groups):
    from rv9 import server
    one = server.reservation(1920, 1080, 12, (0, 0))
    eng = server.Engine(0, hbm_budget=int(one * 1.5), workers=4, groups=groups)
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
    from rv9 import server
    eng = server.Engine(0, hbm_budget=1 << 20, workers=1, groups=groups)
    try:
        with pytest.raises(rv9.UnsupportedError):
            eng.open_stream(1920, 1080)
    finally:
        eng.close()


def test_a_bad_packet_fails_only_its_request(groups):
    from rv9 import server
    name = "vp90-2-02-size-130x132.webm"
    eng = server.Engine(0, workers=4, groups=groups)
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
    from rv9 import server
    eng = server.Engine(0, workers=2, groups=groups)
    sid = eng.open_stream(352, 288)
    for i, p in enumerate(read_packets(os.path.join(VECTORS_DIR, "vp90-2-02-size-130x132.webm"))):
        eng.submit(sid, p, tag=i)
    eng.close()
