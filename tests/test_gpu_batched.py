"""One launch per stage across streams (rv9_sequences_run_batched): the next
frames of many sequences of different sizes, bit depths and chroma formats go
through shared launches, and every decoder ends with the same reference slots
as when its sequence runs alone."""
import os

import pytest

from conftest import VECTORS_DIR, read_packets
from streams_cases import generate

pytestmark = pytest.mark.gpu

NAMES = [
    "vp90-2-02-size-130x132.webm",
    "vp90-2-05-resize.ivf",
    "vp90-2-13-mv-with-scaling.ivf",
    "vp91-2-04-yuv444.webm",
    "vp92-2-20-10bit-yuv420.webm",
    "vp93-2-20-12bit-yuv422.webm",
    "vp90-2-15-fuzz-flicker.webm",
    "vp90-2-10-show-existing-frame2.webm",
]
CAP = 32 << 20


def _slots(dec):
    import rv9
    out = []
    for s in range(8):
        try:
            out.append(dec.download_slot(s, CAP))
        except rv9.Rv9Error:
            out.append(None)
    return out


def _load(names):
    import rv9
    decs = [rv9.Decoder(0) for _ in names]
    seqs = [d.load_sequence(read_packets(os.path.join(VECTORS_DIR, n))) for d, n in zip(decs, names)]
    return decs, seqs


def _close(decs, seqs):
    for d, s in zip(decs, seqs):
        s.free()
        d.close()


def test_batched_equals_alone(oracle_lib):
    # Every shown frame of every batched run (through the frame sinks) is the
    # oracle's, and the reference slots end as after the sequence alone.
    import rv9
    from conftest import FrameSinks, oracle_frames
    decs, seqs = _load(NAMES)
    want = [oracle_frames(oracle_lib, read_packets(os.path.join(VECTORS_DIR, n))) for n in NAMES]
    sinks = FrameSinks(decs, 64 << 20)
    try:
        alone = []
        for i, (d, s) in enumerate(zip(decs, seqs)):
            s.run()
            alone.append(_slots(d))
            assert sinks.md5s(i, [sz for _, sz in want[i]]) == [m for m, _ in want[i]], NAMES[i]
        for groups in (1, 2, 3, len(NAMES)):
            sinks.reset()
            ms = rv9.run_batched(list(zip(decs, seqs)), groups=groups)
            assert ms > 0
            for i, (d, slots) in enumerate(zip(decs, alone)):
                assert sinks.md5s(i, [sz for _, sz in want[i]]) == [m for m, _ in want[i]], (groups, NAMES[i])
                assert _slots(d) == slots, groups
        # An ordinary run after batched ones still matches.
        seqs[1].run()
        assert _slots(decs[1]) == alone[1]
    finally:
        sinks.detach()
        _close(decs, seqs)


def test_batched_large_frames_equal_alone(oracle_lib):
    # Generated streams at the benchmark shapes (1080p 8-bit with 4 tile
    # columns, 2160p 10-bit, 720p 12-bit 4:4:4, 720p 10-bit 4:2:2), several
    # decoders per content, so that the wavefront stages share each launch
    # among many large frames. Every shown frame is the oracle's.
    import rv9
    from conftest import FrameSinks, oracle_frames
    contents = [generate(name)[0] for name in ("1080p_8bit_q40", "2160p_10bit_q30", "720p_12bit_444_q30",
                                               "720p_10bit_422_q50", "cif_8bit_q60")]
    want = [oracle_frames(oracle_lib, pk) for pk in contents]
    decs, seqs, which = [], [], []
    try:
        for rep in range(3):
            for k, pk in enumerate(contents):
                d = rv9.Decoder(0)
                decs.append(d)
                seqs.append(d.load_sequence(pk))
                which.append(k)
        alone = []
        for d, s in zip(decs, seqs):
            s.run()
            alone.append(_slots(d))
        sinks = FrameSinks(decs, 96 << 20)
        try:
            for groups in (1, 4):
                sinks.reset()
                rv9.run_batched(list(zip(decs, seqs)), groups=groups)
                for i, (d, slots) in enumerate(zip(decs, alone)):
                    w = want[which[i]]
                    assert sinks.md5s(i, [sz for _, sz in w]) == [m for m, _ in w], (groups, i)
                    assert _slots(d) == slots, (groups, i)
        finally:
            sinks.detach()
    finally:
        _close(decs, seqs)


def test_batched_rejects_bad_calls():
    import rv9
    d = rv9.Decoder(0)
    s1 = d.load_sequence(read_packets(os.path.join(VECTORS_DIR, NAMES[0])))
    s2 = d.load_sequence(read_packets(os.path.join(VECTORS_DIR, NAMES[0])))
    try:
        with pytest.raises(rv9.InvalidInputError):
            rv9.run_batched([(d, s1), (d, s2)])
        with pytest.raises(rv9.InvalidInputError):
            rv9.run_batched([(d, s1)], groups=0)
        assert rv9.run_batched([(d, s1)]) > 0
    finally:
        s1.free()
        s2.free()
        d.close()


def test_batched_autotune_keeps_results_exact():
    import rv9
    decs, seqs = _load(NAMES[:5])
    try:
        alone = []
        for d, s in zip(decs, seqs):
            s.run()
            alone.append(_slots(d))
        pairs = list(zip(decs, seqs))
        tuned = rv9.autotune_batched(pairs)
        assert 1 <= tuned["groups"] <= len(pairs)
        assert tuned["intra_ctas_per_sm_x4"] in (2, 4, 8)
        assert 0 < tuned["best_ms"] <= tuned["default_ms"]
        rv9.run_batched(pairs, groups=tuned["groups"])
        for d, want in zip(decs, alone):
            assert _slots(d) == want
    finally:
        _close(decs, seqs)


def test_batched_on_fresh_decoders(oracle_lib):
    # Decoders that have never run: their frames are allocated (and zeroed)
    # by the batched run itself, on the group streams that first use them,
    # with fewer groups than decoders so that most decoders' launches go on
    # another decoder's stream. Every shown frame is checked, through the
    # frame sink, against the oracle and the published MD5s.
    import rv9
    from conftest import FrameSinks, expected_md5s, oracle_frames
    names = NAMES[:6]
    decs, seqs = _load(names)
    sinks = FrameSinks(decs, 64 << 20)
    try:
        rv9.run_batched(list(zip(decs, seqs)), groups=2)
        for i, n in enumerate(names):
            path = os.path.join(VECTORS_DIR, n)
            want = oracle_frames(oracle_lib, read_packets(path))
            got = sinks.md5s(i, [sz for _, sz in want])
            assert got == [m for m, _ in want] == expected_md5s(path), n
    finally:
        sinks.detach()
        _close(decs, seqs)
