"""The synthetic streams decoded by an independent VP9 decoder.

The oracle links the product's host parser, so on the repository's synthetic
streams it checks reconstruction, not parsing; only the 15 conformance
vectors' published MD5s pin the parser. This test pins both on synthetic
content against a decoder that shares no code with this repository: FFmpeg's
native VP9 decoder, reached through OpenCV's video reader (cv2 is built with
FFmpeg in this image). With colour conversion off, OpenCV hands out the
decoded luma plane's bytes unconverted for BT.601 streams (for other colour
spaces it converts, which would not be a decoder comparison), so the streams
here are the benchmark shapes coded as BT.601: the colour-space field is the
only header difference and changes no sample. At 8 bits the whole luma plane
is compared; at 10 bits OpenCV returns the first `width` bytes of each luma
row (the left half of the row's little-endian u16 samples), which are
compared.

Runs on the CPU (no GPU): the oracle is the decoder under comparison here,
and the GPU path is held to the oracle frame by frame by the GPU tests."""
import numpy as np
import pytest

CASES = {
    # name: (width, height, bit_depth, frames, q, tile_cols_log2, noise)
    "cif_8bit_q60_30f": (352, 288, 8, 30, 60, 0, 8),       # the small CPU configuration, full length
    "1080p_8bit_q40_6f": (1920, 1080, 8, 6, 40, 2, 6),     # the GPU configuration's two quantisers
    "1080p_8bit_q80_6f": (1920, 1080, 8, 6, 80, 2, 6),
    "720p_8bit_q60_10f": (1280, 720, 8, 10, 60, 2, 6),
    "360p_10bit_q45_10f": (640, 360, 10, 10, 45, 0, 24),
}


def _ffmpeg_planes(path):
    cv2 = pytest.importorskip("cv2")
    if not hasattr(cv2, "CAP_FFMPEG"):
        pytest.skip("cv2 without its FFmpeg backend")
    cap = cv2.VideoCapture(path, cv2.CAP_FFMPEG)
    if not cap.isOpened():
        pytest.skip("cv2's FFmpeg backend cannot open IVF/VP9 here")
    cap.set(cv2.CAP_PROP_CONVERT_RGB, 0)
    out = []
    while True:
        ok, f = cap.read()
        if not ok:
            break
        out.append(np.ascontiguousarray(f).view(np.uint8).reshape(-1))
    cap.release()
    return out


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_equals_ffmpeg_on_synthetic_streams(name, oracle_lib, tmp_path):
    from rv9 import containers, streams
    w, h, bd, frames, q, tcl, noise = CASES[name]
    cfg = streams.config(w, h, frames, q, bit_depth=bd, tile_cols_log2=tcl, golden_interval=4, seed=7, pan=(3, 2),
                         rectangles=12, noise=noise, color_space=1)
    packets = streams.generate(cfg)
    path = str(tmp_path / f"{name}.ivf")
    with open(path, "wb") as f:
        f.write(containers.ivf_write(packets, w, h))
    theirs = _ffmpeg_planes(path)
    dec = oracle_lib.OracleDecoder(threads=4)
    ours = [fr for p in packets for fr in dec.decode_all(p)]
    assert len(ours) == frames and len(theirs) == frames
    n = w * h
    bps = 2 if bd > 8 else 1
    for i, (a, b) in enumerate(zip(ours, theirs)):
        assert b.size == n, f"frame {i}: OpenCV returned {b.size} bytes"
        mine = np.frombuffer(a.packed()[:n * bps], np.uint8).reshape(h, w * bps)[:, :w].reshape(-1)
        if not np.array_equal(mine, b):
            bad = int(np.count_nonzero(mine != b))
            pytest.fail(f"frame {i}: {bad} of {n} luma bytes differ from FFmpeg's decode")
