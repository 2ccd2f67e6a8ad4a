"""The benchmark configurations' streams at full length, on the GPU, frame by
frame against the oracle.

Configuration 1 (30 frames 352x288), configuration 2 (the two 60-frame 1080p
streams at q40 and q80 that bench.py times) and configuration 3 (60 frames
3840x2160 10-bit, 30 frames 1280x720 12-bit 4:4:4; LAST and GOLDEN
references, golden every 8 frames) are decoded through the C ABI two ways:
rv9_decode_packets from host packets into pinned host memory (the end-to-end
path), and the device-resident replay (rv9_sequence_load + rv9_sequence_run
with a frame sink), and for the frames that fit the fixed scratch array the
no-allocation replay too. Every shown frame's MD5 must equal the oracle's.

Streams come from the workload cache (rv9.workloads): generated once, then
read as IVF files. The reference-run recipe is tests/common/mod.rs:123-182
(per-frame MD5 of every shown frame)."""
import os

import pytest

from conftest import FrameSinks, oracle_frames, split_md5s

pytestmark = pytest.mark.gpu


def _cases():
    from rv9 import workloads
    return workloads.CONFIG1 + workloads.CONFIG2 + workloads.CONFIG3


def _ids():
    return [s["name"] for s in _cases()]


@pytest.mark.parametrize("spec", _cases(), ids=_ids())
def test_config_stream_matches_oracle(spec, oracle_lib):
    import torch

    import rv9
    from rv9 import workloads
    packets = workloads.packets(spec)
    want = oracle_frames(oracle_lib, packets, threads=os.cpu_count() or 4)
    assert len(want) == spec["frames"]
    sizes = [sz for _, sz in want]
    md5s = [m for m, _ in want]
    total = sum(sizes)
    dec = rv9.Decoder(0)
    try:
        # End to end: host packets in, packed frames out to pinned memory.
        out = torch.empty(total + (1 << 20), dtype=torch.uint8, pin_memory=True)
        nf, nb = dec.decode_packets_to(packets, out.data_ptr(), out.numel())
        assert (nf, nb) == (len(sizes), total)
        assert split_md5s(bytes(out[:nb].numpy()), sizes) == md5s
        del out
        # Device-resident replay, every shown frame through the sink.
        seq = dec.load_sequence(packets)
        sinks = FrameSinks([dec], total)
        try:
            seq.run()
            assert sinks.md5s(0, sizes) == md5s
            sinks.reset()
            seq.run_noalloc()  # the pool is filled by the run above
            assert sinks.md5s(0, sizes) == md5s
        finally:
            sinks.detach()
            seq.free()
    finally:
        dec.close()
