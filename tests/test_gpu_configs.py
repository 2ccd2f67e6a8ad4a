"""GPU parity on streams in the benchmark configurations' formats (8-bit
4:2:0 CIF and 1080p, 10-bit 2160p, 12-bit 4:4:4 and 10-bit 4:2:2 720p, with
4 tile columns and LAST + GOLDEN references): frame by frame against the
oracle, and the last frame against the generator's own reconstruction."""
import hashlib

import pytest

from streams_cases import CASES, generate

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_equals_oracle_and_generator(oracle_lib, name):
    import rv9
    packets, last_md5 = generate(name)
    dec = rv9.Decoder(0)
    ref = oracle_lib.OracleDecoder(threads=4)
    last = None
    for i, p in enumerate(packets):
        a = dec.decode_all(p)
        b = ref.decode_all(p)
        assert len(a) == len(b) == 1
        assert a[0].packed() == b[0].packed(), f"{name}: frame {i}"
        last = a[0].packed()
    assert hashlib.md5(last).hexdigest() == last_md5
    dec.close()


@pytest.mark.parametrize("name", ["cif_8bit_q60", "720p_12bit_444_q30", "720p_10bit_422_q50"])
def test_decode_packets_frame_parallel_parse(name):
    # rv9_decode_packets parses several frames at once on these
    # error-resilient streams: the output is the frame-by-frame one.
    import torch

    import rv9
    packets, last_md5 = generate(name)
    ref = rv9.Decoder(0)
    want = b"".join(f.packed() for p in packets for f in ref.decode_all(p))
    ref.close()
    for depth in (1, 3, 8):
        dec = rv9.Decoder(0)
        dec.set_parse_depth(depth)
        buf = torch.empty(len(want), dtype=torch.uint8, pin_memory=True)
        nf, nb = dec.decode_packets_to(packets, buf.data_ptr(), len(want))
        assert (nf, nb) == (len(packets), len(want))
        assert bytes(buf.numpy()) == want, f"depth {depth}"
        dec.close()


def test_decode_packets_on_vectors():
    # Conformance vectors through the multi-packet call (the pipeline settles
    # their dependent frames in turn): the published MD5s.
    import torch

    import rv9
    from conftest import expected_md5s, read_packets, vector_paths
    for path in vector_paths():
        packets = read_packets(path)
        dec = rv9.Decoder(0)
        dec.set_parse_depth(4)
        cap = 64 << 20
        buf = torch.empty(cap, dtype=torch.uint8, pin_memory=True)
        ref = rv9.Decoder(0)
        sizes = [len(f.packed()) for p in packets for f in ref.decode_all(p)]
        ref.close()
        nf, nb = dec.decode_packets_to(packets, buf.data_ptr(), cap)
        assert nf == len(sizes) and nb == sum(sizes), path
        data = bytes(buf[:nb].numpy())
        got, off = [], 0
        for s in sizes:
            got.append(hashlib.md5(data[off:off + s]).hexdigest())
            off += s
        assert got == expected_md5s(path), path
        dec.close()
