"""The CUDA kernels' per-sample arithmetic (csrc/gpu/dsp_math.cuh, compiled
for the host) against the oracle, on the reference's test recipes
(rivet-vp9 src/dsp/itx.rs:1252-1450, intra.rs:178-210, lf.rs:565-667):
every transform size and type at 8/10/12 bits including lossless and DC-only,
extreme coefficient magnitudes, every intra mode and edge availability, and
random loop-filter lines of every filter size. Bit-exact."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO

SHIM_SRC = os.path.join(REPO, "tests", "cpp", "gpu_math_shim.cpp")
SHIM = os.path.join(REPO, "tests", "cpp", "_build", "libgpumath_shim.so")


@pytest.fixture(scope="module")
def libs(oracle_lib):
    os.makedirs(os.path.dirname(SHIM), exist_ok=True)
    hdr = os.path.join(REPO, "rivet-vp9_b200", "csrc", "gpu", "dsp_math.cuh")
    if not os.path.exists(SHIM) or max(os.path.getmtime(SHIM_SRC), os.path.getmtime(hdr)) > os.path.getmtime(SHIM):
        subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", SHIM_SRC, "-o", SHIM], check=True)
    return oracle_lib.lib(), ctypes.CDLL(SHIM)


def P(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def test_inverse_transforms(libs):
    o, s = libs
    rng = np.random.default_rng(7)
    for trial in range(6000):
        n = int(rng.integers(2, 6))
        n0 = 1 << n
        bd = int(rng.choice([8, 10, 12]))
        lossless = int(n == 2 and rng.random() < 0.2)
        tx_type = 0 if (n == 5 or lossless) else int(rng.integers(0, 4))
        coefs = np.zeros(n0 * n0, np.int32)
        if rng.random() < 0.3:
            eob = 1
            coefs[0] = rng.integers(-40000, 40000)
        else:
            k = int(rng.integers(1, min(n0 * n0, 40)))
            idx = rng.integers(0, n0 * n0, k)
            mag = int(rng.choice([100, 2000, 1 << 15, 1 << 20, 1 << 30]))
            coefs[idx] = rng.integers(-mag, mag, k)
            eob = max(int(idx.max()) + 1, 2)
        pred = rng.integers(0, 1 << bd, (n0, n0)).astype(np.uint16)
        a, b = pred.copy(), pred.copy()
        o.rv9o_test_itx(P(coefs), n, tx_type, lossless, eob, bd, P(a), n0)
        s.shim_itx(P(coefs), n, tx_type, lossless, eob, bd, P(b), n0)
        assert np.array_equal(a, b), (n, tx_type, lossless, eob, bd)


def test_dc_only_matches_full_transform(libs):
    # The reference checks its DC shortcut over -40000..40000 (itx.rs:1433-1450).
    o, s = libs
    for bd in (8, 10):
        for n in (2, 3, 4, 5):
            n0 = 1 << n
            for dc in range(-40000, 40001, 997):
                c = np.zeros(n0 * n0, np.int32)
                c[0] = dc
                base = np.full((n0, n0), 1 << (bd - 1), np.uint16)
                a, b = base.copy(), base.copy()
                o.rv9o_test_itx(P(c), n, 0, 0, 2, bd, P(a), n0)  # eob 2: the full transform
                s.shim_itx(P(c), n, 0, 0, 1, bd, P(b), n0)       # eob 1: the shortcut
                assert np.array_equal(a, b), (bd, n, dc)


def test_intra_closed_forms(libs):
    o, s = libs
    rng = np.random.default_rng(11)
    for trial in range(6000):
        log2 = int(rng.integers(2, 6))
        size = 1 << log2
        bd = int(rng.choice([8, 10, 12]))
        mode = trial % 10
        above = rng.integers(0, 1 << bd, 65).astype(np.int32)
        left = rng.integers(0, 1 << bd, 32).astype(np.int32)
        hl, ha = int(rng.integers(0, 2)), int(rng.integers(0, 2))
        a = np.zeros((size, size), np.uint16)
        b = a.copy()
        o.rv9o_test_intra(mode, log2, P(above), P(left), hl, ha, bd, P(a), size)
        s.shim_intra(mode, log2, P(above), P(left), hl, ha, bd, P(b), size)
        assert np.array_equal(a, b), (mode, size, bd)


def test_loop_filter_lines(libs):
    o, s = libs
    rng = np.random.default_rng(13)
    for trial in range(60000):
        bd = int(rng.choice([8, 10, 12]))
        base = int(rng.integers(0, 1 << bd))
        spread = int(rng.choice([1, 2, 4, 16, 64])) << (bd - 8)
        line = np.clip(base + rng.integers(-spread, spread + 1, 16), 0, (1 << bd) - 1).astype(np.uint16)
        fs = int(rng.integers(0, 3))
        lvl = int(rng.integers(1, 64))
        sharp = int(rng.integers(0, 8))
        limit = max(lvl >> (2 if sharp > 4 else (1 if sharp else 0)), 1)
        if sharp:
            limit = min(limit, 9 - sharp)
        blimit, thresh = 2 * (lvl + 2) + limit, lvl >> 4
        a, b = line.copy(), line.copy()
        o.rv9o_test_lf(P(a), fs, limit, blimit, thresh, bd)
        s.shim_lf(P(b), fs, limit, blimit, thresh, bd)
        assert np.array_equal(a, b), (fs, bd)
