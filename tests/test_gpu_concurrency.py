"""Several decoders reconstructing at once on their own CUDA streams
(rv9_sequences_run) give each stream the same reference slots as running it
alone, and the shown frames match the published MD5s."""
import hashlib
import os

import pytest

from conftest import VECTORS_DIR, expected_md5s, read_packets

pytestmark = pytest.mark.gpu

NAMES = [
    "vp90-2-02-size-130x132.webm",
    "vp90-2-05-resize.ivf",
    "vp90-2-13-mv-with-scaling.ivf",
    "vp91-2-04-yuv444.webm",
    "vp92-2-20-10bit-yuv420.webm",
    "vp93-2-20-12bit-yuv422.webm",
    "vp90-2-15-fuzz-flicker.webm",
]
CAP = 4 << 20


def _slots(dec):
    import rv9
    out = []
    for s in range(8):
        try:
            out.append(dec.download_slot(s, CAP))
        except rv9.Rv9Error:
            out.append(None)
    return out


def test_concurrent_equals_alone(oracle_lib):
    # Every shown frame of each concurrent run (through the frame sinks) is
    # the oracle's, and the reference slots end as after the sequence alone.
    import rv9
    from conftest import FrameSinks, oracle_frames
    decs = [rv9.Decoder(0) for _ in NAMES]
    seqs = [d.load_sequence(read_packets(os.path.join(VECTORS_DIR, n))) for d, n in zip(decs, NAMES)]
    want = [oracle_frames(oracle_lib, read_packets(os.path.join(VECTORS_DIR, n))) for n in NAMES]
    sinks = FrameSinks(decs, 64 << 20)
    try:
        alone = []
        for d, s in zip(decs, seqs):
            s.run()
            alone.append(_slots(d))
        for rep in range(3):
            sinks.reset()
            ms = rv9.run_concurrent(list(zip(decs, seqs)), per_kernel=(rep == 1))
            assert ms > 0
            for i, (d, slots) in enumerate(zip(decs, alone)):
                assert sinks.md5s(i, [sz for _, sz in want[i]]) == [m for m, _ in want[i]], (rep, NAMES[i])
                assert _slots(d) == slots
    finally:
        sinks.detach()
        for d, s in zip(decs, seqs):
            s.free()
            d.close()


def test_concurrent_public_decodes_match_md5():
    # Public-API decoding on host threads at once, one decoder each.
    import threading

    import rv9
    results = {}

    def run(name):
        dec = rv9.Decoder(0)
        got = []
        for pkt in read_packets(os.path.join(VECTORS_DIR, name)):
            for f in dec.decode_all(pkt):
                got.append(hashlib.md5(f.packed()).hexdigest())
        dec.close()
        results[name] = got

    threads = [threading.Thread(target=run, args=(n,)) for n in NAMES]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for n in NAMES:
        assert results.get(n) == expected_md5s(os.path.join(VECTORS_DIR, n)), n


def test_rejects_a_decoder_twice():
    import rv9
    d = rv9.Decoder(0)
    s1 = d.load_sequence(read_packets(os.path.join(VECTORS_DIR, NAMES[0])))
    s2 = d.load_sequence(read_packets(os.path.join(VECTORS_DIR, NAMES[0])))
    try:
        with pytest.raises(rv9.InvalidInputError):
            rv9.run_concurrent([(d, s1), (d, s2)])
    finally:
        s1.free()
        s2.free()
        d.close()


def test_clone_replays_the_same():
    import rv9
    a, b = rv9.Decoder(0), rv9.Decoder(0)
    seq = a.load_sequence(read_packets(os.path.join(VECTORS_DIR, NAMES[1])))
    try:
        seq.run()
        want = _slots(a)
        copy = b.clone_sequence(seq)
        assert copy.frames == seq.frames and copy.luma_samples == seq.luma_samples
        seq.free()  # the copy owns its records
        copy.run()
        assert _slots(b) == want
        copy.free()
    finally:
        a.close()
        b.close()


def test_graph_replay_equals_run():
    # RV9_RUN_GRAPH: the run captured as a CUDA graph and replayed gives the
    # same reference slots, replay after replay, alone and concurrently.
    import rv9
    decs = [rv9.Decoder(0) for _ in NAMES[:4]]
    seqs = [d.load_sequence(read_packets(os.path.join(VECTORS_DIR, n))) for d, n in zip(decs, NAMES[:4])]
    try:
        want = []
        for d, s in zip(decs, seqs):
            s.run()
            want.append(_slots(d))
        for rep in range(2):
            for d, s, w in zip(decs, seqs, want):
                assert s.run(graph=True) > 0
                assert _slots(d) == w
        for rep in range(2):
            rv9.run_concurrent(list(zip(decs, seqs)), graph=True)
            for d, w in zip(decs, want):
                assert _slots(d) == w
        # An ordinary run after replays still matches.
        seqs[0].run()
        assert _slots(decs[0]) == want[0]
    finally:
        for d, s in zip(decs, seqs):
            s.free()
            d.close()


def test_autotune_keeps_results_exact():
    # The autotuner's launch shapes change no sample: every vector's slots
    # are the same after tuning as before.
    import rv9
    for name in NAMES[:3] + NAMES[4:6]:
        d = rv9.Decoder(0)
        s = d.load_sequence(read_packets(os.path.join(VECTORS_DIR, name)))
        try:
            s.run()
            want = _slots(d)
            r = d.autotune(s)
            assert r["intra_ctas_per_sm_x4"] in (1, 2, 4, 8, 16) and r["inter_threads"] in (64, 128, 256)
            assert 0 < r["best_ms"] <= r["default_ms"]
            s.run()
            assert _slots(d) == want, name
        finally:
            s.free()
            d.close()


def test_concurrent_autotune_keeps_results_exact():
    # One shape for decoders reconstructed together: every decoder's slots
    # after tuning are the same as after a plain run of its sequence alone.
    import rv9
    names = NAMES[:3] + NAMES[4:6]
    decs = [rv9.Decoder(0) for _ in names]
    seqs = [d.load_sequence(read_packets(os.path.join(VECTORS_DIR, n))) for d, n in zip(decs, names)]
    try:
        want = []
        for d, s in zip(decs, seqs):
            s.run()
            want.append(_slots(d))
        pairs = list(zip(decs, seqs))
        r = rv9.autotune_concurrent(pairs)
        assert r["intra_ctas_per_sm_x4"] in (1, 2, 4, 8, 16) and r["inter_threads"] in (64, 128, 256)
        assert 0 < r["best_ms"] <= r["default_ms"]
        rv9.run_concurrent(pairs)
        for d, w, n in zip(decs, want, names):
            assert _slots(d) == w, n
    finally:
        for d, s in zip(decs, seqs):
            s.free()
            d.close()


def test_event_mask_brackets_only_the_chosen_kernels():
    # rv9_decoder_set_event_mask: a per-kernel run with only the loop filter
    # bracketed times only it, and the frames are the same either way.
    import rv9
    name = NAMES[0]
    d = rv9.Decoder(0)
    s = d.load_sequence(read_packets(os.path.join(VECTORS_DIR, name)))
    try:
        s.run(per_kernel=True)
        want = _slots(d)
        full = d.kernel_stats(reset=True)
        assert all(v["launches"] > 0 for k, v in full.items() if k in ("k_lf", "k_prep"))
        d.set_event_mask(["k_lf"])
        s.run(per_kernel=True)
        only = d.kernel_stats(reset=True)
        assert only["k_lf"]["launches"] == full["k_lf"]["launches"] and only["k_lf"]["ms"] > 0
        assert all(v["launches"] == 0 for k, v in only.items() if k != "k_lf")
        assert _slots(d) == want
        d.set_event_mask(None)
        s.run(per_kernel=True)
        assert d.kernel_stats(reset=True)["k_prep"]["launches"] == full["k_prep"]["launches"]
    finally:
        s.free()
        d.close()
