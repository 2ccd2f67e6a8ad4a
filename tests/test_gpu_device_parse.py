"""Device parsing on the GPU: the tile syntax and the work lists built on the
device (rv9_decoder_set_device_parse), frame by frame against the oracle.

tests/test_device_parse_cpu.py holds the same parser code, compiled for the
CPU, to the host parser's records byte for byte; here the device build runs
inside the decoder. Through the C ABI, every shown frame's MD5 must equal the
oracle's:
  * rv9_decode_packets (host packets in, packed frames out) on the generated
    streams of every configuration shape, in small and large batch windows;
  * the benchmark's full-length streams (configurations 1-3);
  * rv9_sequence_load + rv9_sequence_run (the device-built records resident);
  * streams whose frames read the previous frame's motion vectors, with
    probability-adapting frames (parsed on the host) among them, so that the
    vectors pass between the device parser's batches and to and from the host
    parser;
  * the conformance vectors (whose frames all adapt probabilities, so they
    stay with the host parser: the device-parse mode must leave them exact);
  * a stream with a corrupted frame: the same error as host parsing, and the
    frames before it decoded.
"""
import os

import pytest

from conftest import FrameSinks, expected_md5s, oracle_frames, read_packets, split_md5s, vector_paths
from streams_cases import CASES, LINKED, generate, generate_linked

pytestmark = pytest.mark.gpu


def _decode(dec, packets, total):
    import torch
    out = torch.empty(total + (1 << 20), dtype=torch.uint8, pin_memory=True)
    nf, nb = dec.decode_packets_to(packets, out.data_ptr(), out.numel())
    return nf, nb, bytes(out[:nb].numpy())


@pytest.mark.parametrize("window", [1, 3, 64])
@pytest.mark.parametrize("name", sorted(CASES))
def test_generated_streams(name, window, oracle_lib):
    import rv9
    packets, _ = generate(name)
    want = oracle_frames(oracle_lib, packets)
    sizes = [s for _, s in want]
    dec = rv9.Decoder(0)
    try:
        dec.set_device_parse(True, window)
        nf, nb, buf = _decode(dec, packets, sum(sizes))
        assert (nf, nb) == (len(sizes), sum(sizes))
        assert split_md5s(buf, sizes) == [m for m, _ in want]
        frames, bools, ms = dec.device_parse_stats()
        assert frames == len(packets) - (CASES[name][3] != (1, 1)) and bools > 0 and ms > 0
    finally:
        dec.close()


@pytest.mark.parametrize("window", [1, 3, 8])
@pytest.mark.parametrize("name", sorted(LINKED))
def test_linked_streams(name, window, oracle_lib):
    # Frames that read the previous frame's motion vectors, some of them
    # adapting probabilities (those parse on the host): the vectors pass
    # between the batch's frames, from the host parser to the device and
    # back, and between batches.
    import rv9
    packets = generate_linked(name)
    want = oracle_frames(oracle_lib, packets)
    sizes = [s for _, s in want]
    dec = rv9.Decoder(0)
    try:
        dec.set_device_parse(True, window)
        nf, nb, buf = _decode(dec, packets, sum(sizes))
        assert (nf, nb) == (len(sizes), sum(sizes))
        assert split_md5s(buf, sizes) == [m for m, _ in want]
        assert dec.device_parse_stats()[0] > 0
    finally:
        dec.close()


def _config_cases():
    from rv9 import workloads
    return workloads.CONFIG1 + workloads.CONFIG2 + workloads.CONFIG3


@pytest.mark.parametrize("spec", _config_cases(), ids=[s["name"] for s in _config_cases()])
def test_config_streams(spec, oracle_lib):
    import rv9
    from rv9 import workloads
    packets = workloads.packets(spec)
    want = oracle_frames(oracle_lib, packets, threads=os.cpu_count() or 4)
    sizes = [s for _, s in want]
    md5s = [m for m, _ in want]
    dec = rv9.Decoder(0)
    try:
        dec.set_device_parse(True)
        nf, nb, buf = _decode(dec, packets, sum(sizes))
        assert (nf, nb) == (len(sizes), sum(sizes))
        assert split_md5s(buf, sizes) == md5s
        # The device-built records, resident: a replay through the sink.
        seq = dec.load_sequence(packets)
        sinks = FrameSinks([dec], sum(sizes))
        try:
            seq.run()
            assert sinks.md5s(0, sizes) == md5s
        finally:
            sinks.detach()
            seq.free()
    finally:
        dec.close()


@pytest.mark.parametrize("path", vector_paths(), ids=os.path.basename)
def test_vectors(path):
    import hashlib

    import rv9
    packets = read_packets(path)
    want = expected_md5s(path)
    dec = rv9.Decoder(0)
    try:
        dec.set_device_parse(True, 4)
        # Frame sizes: each frame through decode_all of a host-parsing decoder.
        ref = rv9.Decoder(0)
        try:
            sizes = [len(f.packed()) for p in packets for f in ref.decode_all(p)]
        finally:
            ref.close()
        nf, nb, buf = _decode(dec, packets, sum(sizes))
        assert nf == len(want)
        got = split_md5s(buf, sizes)
        assert got == want
    finally:
        dec.close()


def test_corrupted_frame_reports_like_host_parsing(oracle_lib):
    import rv9
    packets, _ = generate("cif_8bit_q60")
    bad = list(packets)
    flipped = bytearray(bad[3])
    for i in range(len(flipped) // 2, len(flipped)):
        flipped[i] ^= 0xA5
    bad[3] = bytes(flipped)
    results = []
    for device_parse in (False, True):
        dec = rv9.Decoder(0)
        try:
            dec.set_device_parse(device_parse, 8)
            try:
                _decode(dec, bad, 8 << 20)
                results.append(("ok", None))
            except rv9.Rv9Error as e:
                results.append((type(e).__name__, str(e)))
            # The decoder goes on from the next key frame.
            want = oracle_frames(oracle_lib, packets[:2])
            sizes = [s for _, s in want]
            nf, nb, buf = _decode(dec, packets[:2], sum(sizes))
            assert split_md5s(buf, sizes) == [m for m, _ in want]
        finally:
            dec.close()
    assert results[0] == results[1]


@pytest.mark.parametrize("window", [4, 64])
@pytest.mark.parametrize("name", ["cif_8bit_q60", "1080p_8bit_q40", "720p_10bit_422_q50", "cif_8bit_linked",
                                  "720p_8bit_linked"])
def test_shared_batches(name, window, oracle_lib):
    """RV9_DEVICE_PARSE_SHARED: a batch of independent frames split between
    the host's threads and the device (the split moving between calls), the
    linked streams' batches left whole on the device; every frame exact."""
    import rv9
    packets = generate(name)[0] if name in CASES else generate_linked(name)
    want = oracle_frames(oracle_lib, packets)
    sizes = [s for _, s in want]
    dec = rv9.Decoder(0)
    try:
        dec.set_device_parse(rv9.DEVICE_PARSE_SHARED, window)
        for _ in range(3):
            nf, nb, buf = _decode(dec, packets, sum(sizes))
            assert (nf, nb) == (len(sizes), sum(sizes))
            assert split_md5s(buf, sizes) == [m for m, _ in want]
        frames, bools, ms = dec.device_parse_stats()
        assert 0 < frames <= 3 * len(packets)
        if name in CASES:
            assert frames < 3 * len(packets)  # the host took its part
    finally:
        dec.close()
