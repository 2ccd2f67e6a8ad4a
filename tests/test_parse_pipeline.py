"""Frame-parallel parsing (FramePipeline) gives exactly the records, statuses
and decoder state of frame-by-frame parsing: on every conformance vector
(whose frames mostly depend on each other, so the pipeline settles them in
turn), on generated error-resilient streams (which parse several frames at
once), and across corrupted packets. So does the host side of a shared
device-parse batch (RV9_DEVICE_PARSE_SHARED): frames begun in batches before
any finishes, an all-independent batch run on threads (Parser::run_async)
and finished in order."""
import ctypes
import os
import subprocess

import pytest

from conftest import REPO, read_packets, vector_paths
from streams_cases import LINKED, generate, generate_linked

SRC = os.path.join(REPO, "tests", "cpp", "parse_pipeline_shim.cpp")
LIB = os.path.join(REPO, "tests", "cpp", "_build", "libparse_pipeline_shim.so")
HOST = os.path.join(REPO, "rivet-vp9_b200", "csrc", "host")


@pytest.fixture(scope="module")
def shim():
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    deps = [SRC] + [os.path.join(HOST, f) for f in os.listdir(HOST)]
    if not os.path.exists(LIB) or max(os.path.getmtime(d) for d in deps) > os.path.getmtime(LIB):
        subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-pthread", SRC,
                        os.path.join(HOST, "parser.cpp"), os.path.join(HOST, "probs.cpp"), "-o", LIB], check=True)
    lib = ctypes.CDLL(LIB)
    lib.pipeline_check.restype = ctypes.c_int
    lib.pipeline_check.argtypes = [ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_size_t), ctypes.c_size_t,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]
    lib.shared_batch_check.restype = ctypes.c_int
    lib.shared_batch_check.argtypes = [ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_size_t),
                                       ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]
    return lib


def check(lib, packets, depth, tile_threads=2):
    n = len(packets)
    arr = (ctypes.c_char_p * n)(*packets)
    lens = (ctypes.c_size_t * n)(*[len(p) for p in packets])
    msg = ctypes.create_string_buffer(256)
    r = lib.pipeline_check(arr, lens, n, depth, tile_threads, msg, 256)
    assert r >= 0, msg.value.decode()
    return r


@pytest.mark.parametrize("path", vector_paths(), ids=os.path.basename)
def test_vectors(shim, path):
    assert check(shim, read_packets(path), depth=4) > 0


@pytest.mark.parametrize("name", ["cif_8bit_q60", "720p_12bit_444_q30"])
def test_error_resilient_streams(shim, name):
    packets, _ = generate(name)
    for depth in (1, 3, 8):
        assert check(shim, packets, depth=depth) == len(packets)


@pytest.mark.parametrize("name", sorted(LINKED))
def test_linked_streams(shim, name):
    # Frames that read the previous frame's motion vectors wait for it.
    packets = generate_linked(name)
    for depth in (1, 4):
        assert check(shim, packets, depth=depth) == len(packets)


def test_corrupted_packets(shim):
    packets, _ = generate("cif_8bit_q60")
    bad = list(packets)
    # A truncated inter frame and a garbage packet in the middle.
    bad[2] = bad[2][: len(bad[2]) // 3]
    bad.insert(4, b"\x82\x49\x83\x42\x00garbage")
    assert check(shim, bad, depth=4) == len(bad)
    vec = read_packets(os.path.join(REPO, "tests", "golden", "vectors", "vp90-2-05-resize.ivf"))
    vec[5] = bytes(b ^ 0x5A for b in vec[5])
    assert check(shim, vec, depth=3) == len(vec)


def shared_check(lib, packets, window, depth):
    n = len(packets)
    arr = (ctypes.c_char_p * n)(*packets)
    lens = (ctypes.c_size_t * n)(*[len(p) for p in packets])
    msg = ctypes.create_string_buffer(256)
    r = lib.shared_batch_check(arr, lens, n, window, depth, msg, 256)
    assert r >= 0, msg.value.decode()
    return r


@pytest.mark.parametrize("name", ["cif_8bit_q60", "720p_10bit_422_q50"])
def test_shared_batches_error_resilient(shim, name):
    # Every inter frame is independent: batches of two or more run on threads.
    packets, _ = generate(name)
    for window, depth in ((2, 1), (3, 2), (64, 8)):
        assert shared_check(shim, packets, window, depth) > 0


@pytest.mark.parametrize("name", sorted(LINKED))
def test_shared_batches_linked(shim, name):
    # Frames that read the previous frame's motion vectors are not independent:
    # their batches finish one by one.
    packets = generate_linked(name)
    for window in (2, 8):
        shared_check(shim, packets, window, 4)


def test_shared_batches_vectors_and_corruption(shim):
    for path in vector_paths()[:6]:
        shared_check(shim, read_packets(path), 8, 4)
    packets, _ = generate("cif_8bit_q60")
    bad = list(packets)
    bad[2] = bad[2][: len(bad[2]) // 3]
    bad.insert(4, b"\x82\x49\x83\x42\x00garbage")
    shared_check(shim, bad, 8, 4)
