"""The C ABI library loads and exports every symbol include/rv9.h declares;
without a GPU the decoder refuses to start (no CPU reconstruction path)."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import REPO


HEADERS = ("rv9.h", "rv9_server.h")


def declared_symbols():
    names = set()
    for h in HEADERS:
        text = open(os.path.join(REPO, "include", h)).read()
        names |= set(re.findall(r"\b(rv9_[a-z_]+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def built():
    import rv9
    subprocess.run(["python", os.path.join(REPO, "rivet-vp9_b200", "build.py")], check=True)
    return rv9


def test_exports_every_declared_symbol(built):
    lib = ctypes.CDLL(built.LIB_PATH)
    names = declared_symbols()
    from rv9 import server
    assert set(names) == set(built.EXPORTS) | set(server.EXPORTS)
    for n in names:
        assert hasattr(lib, n), n


def test_no_cpu_fallback_without_a_device(built):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(built.DeviceError):
        built.Decoder()


def test_stream_reservation_needs_no_device(built):
    from rv9 import server
    r720 = server.reservation(1280, 720)
    r1080 = server.reservation(1920, 1080)
    r2160 = server.reservation(3840, 2160, bit_depth=10)
    assert 0 < r720 < r1080 < r2160
    # Ten pooled 1080p frames (SB-aligned 1920x1088, 4:2:0, 1 byte per sample)
    # are the bulk of a 1080p reservation.
    frames = 10 * (1920 * 1088 * 3 // 2)
    assert frames < r1080 < 2 * frames
    # Ten 2160p 10-bit frames at 2 bytes per sample.
    assert r2160 > 10 * 3840 * 2176 * 3
    # 32 streams of the served mix fit a 120 GB budget many times over.
    assert 13 * r720 + 13 * r1080 + 6 * r2160 < 120 << 30


def test_engine_refuses_without_a_device(built):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from rv9 import server
    with pytest.raises(built.DeviceError):
        server.Engine()
