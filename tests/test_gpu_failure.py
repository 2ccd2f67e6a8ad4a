"""Device-side failure detection through the C ABI.

Every wait of the intra and loop-filter wavefronts is bounded. Here a wait is
made to run out without faulting anything: rv9_decoder_set_test_fault leaves
a frame's first intra job (bit 0) or first loop-filter row (bit 1) untaken,
so the jobs that depend on it poll until rv9_decoder_set_wait_limit's short
limit runs out. The kernel then records the error, the frame's other jobs
give up, and the call returns RV9_DEVICE (rv9.DeviceError). The decoder must
then decode cleanly again, bit-exact against the oracle.

Each entry point that launches the wavefronts is covered: rv9_decode_all,
rv9_sequence_run, rv9_sequence_run_noalloc and rv9_sequences_run_batched
(the reference's abort model: src/decoder/loopfilter.rs:300-338)."""
import hashlib

import pytest

from streams_cases import generate

pytestmark = pytest.mark.gpu

SHORT_LIMIT = 4096  # polls: about a millisecond
CAP = 8 << 20


@pytest.fixture(scope="module")
def stream(oracle_lib):
    packets, _ = generate("cif_8bit_q60")
    o = oracle_lib.OracleDecoder()
    md5s = [hashlib.md5(f.packed()).hexdigest() for p in packets for f in o.decode_all(p)]
    return packets, md5s


def _slots(dec):
    import rv9
    out = []
    for s in range(8):
        try:
            out.append(dec.download_slot(s, CAP))
        except rv9.Rv9Error:
            out.append(None)
    return out


def _decode(dec, packets):
    return [hashlib.md5(f.packed()).hexdigest() for p in packets for f in dec.decode_all(p)]


@pytest.mark.parametrize("mask", [1, 2], ids=["intra", "loop_filter"])
def test_decode_all_reports_a_wait_that_ran_out(stream, mask):
    import rv9
    packets, md5s = stream
    dec = rv9.Decoder(0)
    try:
        dec.set_wait_limit(SHORT_LIMIT)
        dec.set_test_fault(mask)
        with pytest.raises(rv9.DeviceError, match="timed out"):
            dec.decode_all(packets[0])
        dec.set_test_fault(0)
        dec.set_wait_limit(0)
        # From the key frame again: bit-exact.
        assert _decode(dec, packets) == md5s
    finally:
        dec.close()


@pytest.mark.parametrize("mask", [1, 2], ids=["intra", "loop_filter"])
def test_sequence_runs_report_a_wait_that_ran_out(stream, mask):
    import rv9
    packets, _ = stream
    dec = rv9.Decoder(0)
    seq = dec.load_sequence(packets)
    try:
        seq.run()  # also fills the pool for the no-allocation run
        want = _slots(dec)
        dec.set_wait_limit(SHORT_LIMIT)
        dec.set_test_fault(mask)
        with pytest.raises(rv9.DeviceError):
            seq.run()
        with pytest.raises(rv9.DeviceError):
            seq.run_noalloc()
        dec.set_test_fault(0)
        dec.set_wait_limit(0)
        seq.run()
        assert _slots(dec) == want
        for _ in range(2):
            seq.run_noalloc()
            assert _slots(dec) == want
    finally:
        seq.free()
        dec.close()


@pytest.mark.parametrize("mask", [1, 2], ids=["intra", "loop_filter"])
def test_batched_run_reports_a_wait_that_ran_out(stream, mask):
    # One faulted decoder among healthy ones: the batch reports the error,
    # and the healthy decoders' results are unaffected.
    import rv9
    packets, _ = stream
    decs = [rv9.Decoder(0) for _ in range(3)]
    seqs = [d.load_sequence(packets) for d in decs]
    try:
        for s in seqs:
            s.run()
        want = _slots(decs[0])
        pairs = list(zip(decs, seqs))
        decs[1].set_wait_limit(SHORT_LIMIT)
        decs[1].set_test_fault(mask)
        with pytest.raises(rv9.DeviceError):
            rv9.run_batched(pairs, groups=2)
        assert _slots(decs[0]) == want and _slots(decs[2]) == want
        decs[1].set_test_fault(0)
        decs[1].set_wait_limit(0)
        rv9.run_batched(pairs, groups=2)
        for d in decs:
            assert _slots(d) == want
    finally:
        for d, s in zip(decs, seqs):
            s.free()
            d.close()
