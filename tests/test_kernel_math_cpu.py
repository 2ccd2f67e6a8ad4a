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
    hdrs = [os.path.join(REPO, "rivet-vp9_b200", "csrc", "gpu", h) for h in ("dsp_math.cuh", "md5.cuh")]
    if not os.path.exists(SHIM) or max([os.path.getmtime(SHIM_SRC)] + [os.path.getmtime(h) for h in hdrs]) > \
            os.path.getmtime(SHIM):
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


def _lf_case(libs, rng, w, h, ss_x, ss_y, bd):
    from records_ctypes import FrameDesc, Block, random_blocks
    o, s = libs
    d = FrameDesc()
    d.width, d.height = w, h
    d.mi_cols, d.mi_rows = (w + 7) >> 3, (h + 7) >> 3
    d.sb64_cols, d.sb64_rows = (d.mi_cols + 7) >> 3, (d.mi_rows + 7) >> 3
    d.ss_x, d.ss_y, d.bit_depth = ss_x, ss_y, bd
    d.lf_level = int(rng.integers(1, 64))
    d.lf_sharpness = int(rng.integers(0, 8))
    d.lf_delta_enabled = int(rng.integers(0, 2))
    for i, v in enumerate(rng.integers(-15, 16, 4)):
        d.lf_ref_deltas[i] = int(v)
    for i, v in enumerate(rng.integers(-15, 16, 2)):
        d.lf_mode_deltas[i] = int(v)
    d.seg.enabled = int(rng.integers(0, 2))
    for sgi in range(8):
        d.seg.feature_enabled[sgi][1] = int(rng.integers(0, 2))
        d.seg.feature_data[sgi][1] = int(rng.integers(-63, 64))
    d.seg.abs_or_delta_update = int(rng.integers(0, 2))
    blocks = random_blocks(rng, d.mi_rows, d.mi_cols, ss_x, ss_y)
    arr = (Block * len(blocks))(*blocks)
    aw, ah = d.sb64_cols * 64, d.sb64_rows * 64
    planes = []
    for p in range(3):
        pw, ph = (aw >> ss_x, ah >> ss_y) if p else (aw, ah)
        yy, xx = np.mgrid[0:ph, 0:pw]
        base = (xx * 3 + yy * 2 + rng.integers(0, 64)) % (1 << bd)
        noise = rng.integers(-3, 4, (ph, pw)) << (bd - 8)
        blocky = ((xx // 8 + yy // 8) % 2) * int(rng.integers(0, 24)) << (bd - 8)
        planes.append(np.clip(base // 4 + noise + blocky, 0, (1 << bd) - 1).astype(np.uint16))
    a = [pl.copy() for pl in planes]
    b = [pl.copy() for pl in planes]
    o.rv9o_test_lf_frame(ctypes.byref(d), arr, len(blocks), P(a[0]), P(a[1]), P(a[2]))
    s.shim_lf_frame(ctypes.byref(d), arr, len(blocks), P(b[0]), P(b[1]), P(b[2]))
    changed = sum(int((a[p] != planes[p]).sum()) for p in range(3))
    for p in range(3):
        assert np.array_equal(a[p], b[p]), (w, h, ss_x, ss_y, bd, p, np.argwhere(a[p] != b[p])[:4].tolist())
    return changed


def test_loop_filter_frames(libs):
    """The loop-filter kernel's superblock procedure (edge decisions, row and
    column passes, tile copy) against the oracle's filter_frame, on random
    block layouts and levels, every chroma format, odd sizes."""
    rng = np.random.default_rng(17)
    changed = 0
    sizes = [(66, 66), (130, 132), (226, 226), (8, 8), (200, 120), (352, 288), (72, 40)]
    for i in range(40):
        w, h = sizes[i % len(sizes)]
        ss = [(1, 1), (1, 0), (0, 1), (0, 0)][i % 4]
        bd = [8, 10, 12][i % 3]
        changed += _lf_case(libs, rng, w, h, ss[0], ss[1], bd)
    assert changed > 0


def test_frame_digest_md5_matches_hashlib(libs):
    # The on-device frame digest's MD5 steps (csrc/gpu/md5.cuh, RFC 1321)
    # against Python's hashlib, at every padding boundary and on random data.
    import hashlib
    _, s = libs
    rng = np.random.default_rng(5)
    lengths = [0, 1, 3, 55, 56, 57, 63, 64, 65, 119, 120, 127, 128, 129, 1000, 4095, 4096, 4097, 100003]
    for n in lengths:
        data = rng.integers(0, 256, n, dtype=np.uint8)
        out = np.zeros(16, np.uint8)
        s.shim_md5(P(data), ctypes.c_uint64(n), P(out))
        assert bytes(out).hex() == hashlib.md5(data.tobytes()).hexdigest(), n
