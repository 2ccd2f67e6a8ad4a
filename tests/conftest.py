"""Shared test setup: the `gpu` marker, paths, the conformance vectors."""
import glob
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "rivet-vp9_b200")
for p in (PKG, os.path.join(REPO, "oracle"), REPO):
    if p not in sys.path:
        sys.path.insert(0, p)

VECTORS_DIR = os.path.join(REPO, "tests", "golden", "vectors")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def vector_paths():
    return sorted(glob.glob(os.path.join(VECTORS_DIR, "*.webm")) + glob.glob(os.path.join(VECTORS_DIR, "*.ivf")))


def expected_md5s(path):
    with open(path + ".md5") as f:
        return [l.split()[0] for l in f if l.strip()]


def read_packets(path):
    from rv9.containers import packets
    with open(path, "rb") as f:
        return packets(f.read())


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle as oracle_mod
    oracle_mod.build()
    return oracle_mod
