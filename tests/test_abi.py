"""The C-ABI library loads and exports every entry point the headers declare."""
import ctypes as ct
import glob
import os
import re

import pytest

from parallelspectralfluids3d_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"^\s*(?:int|const char\s*\*)\s+(psf_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


def test_headers_declare_entry_points():
    names = declared_symbols()
    assert "psf_create" in names and "psf_step" in names


@pytest.mark.parametrize("name", declared_symbols())
def test_library_exports_symbol(name):
    lib = _lib.load()
    assert hasattr(lib, name), f"{name} declared in include/ but not exported"


def test_abi_version():
    assert _lib.load().psf_abi_version() == 1


def test_null_arguments_are_rejected_without_touching_a_device():
    lib = _lib.load()
    out = ct.c_void_p()
    rc = lib.psf_create(None, None, 0, ct.byref(out))
    assert rc == -1 and b"null" in lib.psf_last_error()
    assert lib.psf_step(None, 1) == -1
    assert lib.psf_device_count(None) == -1
