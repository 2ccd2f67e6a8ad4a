"""On-device frame digests (rv9_decoder_set_frame_digests): the MD5 of every
shown frame computed on the GPU from its device planes must be the published
per-frame MD5 of the reference's Frame::packed() — through the drop-in
decode calls, the device-resident replay and the batched runs — with no
frame read back."""
import os

import pytest

from conftest import VECTORS_DIR, expected_md5s, read_packets

pytestmark = pytest.mark.gpu

NAMES = [
    "vp90-2-02-size-130x132.webm",           # odd sizes
    "vp90-2-05-resize.ivf",                  # frame size changes
    "vp90-2-10-show-existing-frame2.webm",   # frames shown again
    "vp91-2-04-yuv444.webm",
    "vp92-2-20-10bit-yuv420.webm",           # 16-bit samples
    "vp93-2-20-12bit-yuv422.webm",
]


@pytest.mark.parametrize("name", NAMES)
def test_decode_digests_equal_published_md5s(name):
    import rv9
    path = os.path.join(VECTORS_DIR, name)
    dec = rv9.Decoder(0)
    try:
        dec.set_frame_digests(1024)
        for p in read_packets(path):
            dec.decode_all(p)
        assert dec.frame_digests() == expected_md5s(path)
    finally:
        dec.close()


def test_replay_and_batched_digests():
    import rv9
    decs = [rv9.Decoder(0) for _ in NAMES]
    seqs = [d.load_sequence(read_packets(os.path.join(VECTORS_DIR, n))) for d, n in zip(decs, NAMES)]
    want = [expected_md5s(os.path.join(VECTORS_DIR, n)) for n in NAMES]
    try:
        for d, s, w in zip(decs, seqs, want):
            d.set_frame_digests(1024)
            s.run()
            assert d.frame_digests() == w
        for d in decs:
            d.set_frame_digests(1024)
        rv9.run_batched(list(zip(decs, seqs)), groups=2)
        for d, w, n in zip(decs, want, NAMES):
            assert d.frame_digests() == w, n
    finally:
        for d, s in zip(decs, seqs):
            d.set_frame_digests(0)
            s.free()
            d.close()
