"""The C ABI without a GPU: the library and the drop-in libraries load, export every
entry point declared in include/hydro_b200.h (and `launcher`), and calls that touch no
device behave (version string, error latch)."""
from __future__ import annotations

import ctypes
import re

import pytest

from conftest import ROOT, load_pkg

hb = load_pkg()
HEADER = ROOT / "include" / "hydro_b200.h"


def declared_functions():
    txt = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?(?:double|float|int|void|char)\s*\*?\s*(hydro\w+)\s*\(", txt, flags=re.M)
    assert len(names) >= 18
    return sorted(set(names))


@pytest.fixture(scope="module")
def built():
    hb.build()
    return hb.lib()


def test_exports_every_declared_symbol(built):
    for name in declared_functions():
        assert hasattr(built, name), name


def test_dropin_libraries_export_launcher(built):
    for so in ("libhydro2d.so", "libhydro2d_float.so", "libhydro3d.so", "libhydro3d_float.so"):
        L = ctypes.CDLL(str(hb.LIB_DIR / so))
        assert hasattr(L, "launcher"), so


def test_version_and_error_latch(built):
    assert b"sm_100a" in built.hydro_version()
    built.hydro_clear_error()
    assert built.hydro_last_error() == 0
    assert built.hydro_last_error_string() == b""


def test_queue_struct_layout():
    """hydro_queue_t is {void*, int, int}: 16 bytes, passed like the C++ sycl::queue of
    include/compat/sycl/sycl.hpp (checked there by static_assert)."""
    assert ctypes.sizeof(hb.Queue) == 16
    assert ctypes.sizeof(hb.StepInfo) == 24
