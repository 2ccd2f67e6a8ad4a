"""The device tile parser, compiled for the CPU, against the host parser.

rivet-vp9_b200/csrc/gpu/tile_parse.cuh is plain C++ with __host__ __device__
qualifiers; tests/cpp/device_parse_shim.cpp builds it with g++ and splits each
stream's frames the way the decoder's device-parse mode does (frames that
Parser::external_tiles admits go to the device parser, the others to the host
parser, which is handed the device-held motion vectors when it reads them).
Every frame's status, message and records must equal frame-by-frame host
parsing byte for byte: on the conformance vectors (mostly host-parsed, since
their frames adapt probabilities, with the key frames and the non-adapting
frames on the device parser), on the generated error-resilient streams of
every configuration shape (all device-parsed), on the benchmark streams'
first frames, and across corrupted packets. The GPU tests run the same code
on the device (tests/test_gpu_device_parse.py)."""
import ctypes
import os
import subprocess

import pytest

from conftest import REPO, read_packets, vector_paths
from streams_cases import CASES, LINKED, generate, generate_linked

SRC = os.path.join(REPO, "tests", "cpp", "device_parse_shim.cpp")
LIB = os.path.join(REPO, "tests", "cpp", "_build", "libdevice_parse_shim.so")
CSRC = os.path.join(REPO, "rivet-vp9_b200", "csrc")


@pytest.fixture(scope="module")
def shim():
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    deps = [SRC] + [os.path.join(CSRC, "host", f) for f in os.listdir(os.path.join(CSRC, "host"))]
    deps += [os.path.join(CSRC, "gpu", f) for f in ("tile_parse.cuh", "parse_plan.h")]
    if not os.path.exists(LIB) or max(os.path.getmtime(d) for d in deps) > os.path.getmtime(LIB):
        subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-pthread", SRC,
                        os.path.join(CSRC, "host", "parser.cpp"), os.path.join(CSRC, "host", "probs.cpp"), "-o",
                        LIB], check=True)
    lib = ctypes.CDLL(LIB)
    lib.device_parse_check.restype = ctypes.c_int
    lib.device_parse_check.argtypes = [ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_size_t),
                                       ctypes.c_size_t, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t,
                                       ctypes.POINTER(ctypes.c_uint64)]
    return lib


def check(lib, packets, window=4):
    n = len(packets)
    arr = (ctypes.c_char_p * n)(*packets)
    lens = (ctypes.c_size_t * n)(*[len(p) for p in packets])
    msg = ctypes.create_string_buffer(512)
    bools = ctypes.c_uint64(0)
    r = lib.device_parse_check(arr, lens, n, window, msg, 512, ctypes.byref(bools))
    assert r >= 0, msg.value.decode()
    return r, bools.value


@pytest.mark.parametrize("window", [1, 4])
@pytest.mark.parametrize("path", vector_paths(), ids=os.path.basename)
def test_vectors(shim, path, window):
    check(shim, read_packets(path), window)


@pytest.mark.parametrize("name", sorted(CASES))
def test_generated_streams(shim, name):
    packets, _ = generate(name)
    taken, bools = check(shim, packets)
    # All frames but a 4:2:2 / 4:4:4 key frame (which may need the legacy
    # layout probe, a host-parser matter).
    chroma = CASES[name][3]
    assert taken == len(packets) - (chroma != (1, 1)) and bools > 0


def test_benchmark_stream_frames(shim):
    # The first frames of the timed 1080p q40 stream and of one 10-bit
    # stream of the 64-stream batch (from the stream cache when present).
    from rv9 import workloads as W
    for spec in (W.CONFIG2[0], W.CONFIG4[20]):
        if not W.cached(spec):
            pytest.skip("benchmark streams not generated here")
        pk = W.packets(spec, generate=False)[:6]
        taken, _ = check(shim, pk, window=3)
        assert taken == len(pk)


@pytest.mark.parametrize("window", [1, 3, 8])
@pytest.mark.parametrize("name", sorted(LINKED))
def test_linked_streams(shim, name, window):
    # Frames that read the previous frame's motion vectors, with frames that
    # adapt probabilities (host-parsed) among them: every source of previous
    # vectors the batched flow has is taken, and each frame's records equal
    # host parsing.
    before = (ctypes.c_uint64 * 4)()
    shim.device_parse_prev_counts(before)
    packets = generate_linked(name)
    taken, _ = check(shim, packets, window)
    after = (ctypes.c_uint64 * 4)()
    shim.device_parse_prev_counts(after)
    used = [after[k] - before[k] for k in range(4)]
    adapt = LINKED[name][7]
    chroma = LINKED[name][3]
    host_frames = (len(packets) - 1) // adapt if adapt else 0
    host_frames = min(host_frames, 3) + (chroma != (1, 1))
    assert taken == len(packets) - host_frames, (taken, used)
    if window > 1:
        assert used[0] > 0, used            # from the batch's previous frame
    if window == 1 or adapt:
        assert used[1] + used[2] > 0, used  # from the state: host- or device-held
    if adapt:
        assert used[3] > 0, used            # device-held vectors given to the host parser


def test_corrupted_packets(shim):
    packets, _ = generate("cif_8bit_q60")
    bad = list(packets)
    bad[2] = bad[2][: len(bad[2]) // 3]             # a truncated inter frame
    bad.insert(4, b"\x82\x49\x83\x42\x00garbage")   # a garbage packet
    flipped = bytearray(bad[6])
    for i in range(len(flipped) // 2, len(flipped)):
        flipped[i] ^= 0xA5                           # corrupted tile data
    bad[6] = bytes(flipped)
    for window in (1, 3, 8):
        check(shim, bad, window)
    vec = read_packets(os.path.join(REPO, "tests", "golden", "vectors", "vp90-2-05-resize.ivf"))
    vec[5] = bytes(b ^ 0x5A for b in vec[5])
    for window in (1, 4):
        check(shim, vec, window)
