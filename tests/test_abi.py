"""The C-ABI library builds for sm_100a, loads, and exports every symbol include/*.h declares.

No compute calls here (this runs without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

from cism_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(cismgpu_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    path = build.build()
    return ctypes.CDLL(path)


def test_header_declares_the_four_solvers():
    names = declared_symbols()
    for f in ("cismgpu_pcg_standard_3d", "cismgpu_pcg_chrongear_3d", "cismgpu_pcg_standard_2d",
              "cismgpu_pcg_chrongear_2d"):
        assert f in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_version_string(lib):
    lib.cismgpu_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.cismgpu_version()


def test_built_for_sm100a_only():
    flags = build.flags()
    assert "arch=compute_100a,code=sm_100a" in flags
    assert "--fmad=false" in flags
