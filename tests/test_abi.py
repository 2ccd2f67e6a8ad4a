"""The C ABI library loads and exports every symbol include/rv9.h declares;
without a GPU the decoder refuses to start (no CPU reconstruction path)."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import REPO


def declared_symbols():
    text = open(os.path.join(REPO, "include", "rv9.h")).read()
    return sorted(set(re.findall(r"\b(rv9_[a-z_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def built():
    import rv9
    subprocess.run(["python", os.path.join(REPO, "rivet-vp9_b200", "build.py")], check=True)
    return rv9


def test_exports_every_declared_symbol(built):
    lib = ctypes.CDLL(built.LIB_PATH)
    names = declared_symbols()
    assert set(names) == set(built.EXPORTS)
    for n in names:
        assert hasattr(lib, n), n


def test_no_cpu_fallback_without_a_device(built):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(built.DeviceError):
        built.Decoder()
