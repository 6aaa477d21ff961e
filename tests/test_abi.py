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
    names = re.findall(r"^\s*(?:const\s+)?(?:double|float|int|void|char|unsigned|long long)\s*\*?\s*(hydro\w+)\s*\(",
                       txt, flags=re.M)
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


def test_noalloc_launch_shape_fits_the_fixed_scratch(built):
    """The allocation-free step's launch shape (host only): at most 65536 blocks, every
    row covered, and the chunk grown where the default shape would exceed the cap."""
    fn = built.hydro2d_noalloc_launch_shape
    fn.argtypes = [ctypes.c_size_t, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                   ctypes.POINTER(ctypes.c_uint), ctypes.POINTER(ctypes.c_uint)]
    fn.restype = ctypes.c_uint
    c, gx, gy = ctypes.c_int(), ctypes.c_uint(), ctypes.c_uint()
    for nb_x, nb_y, strip in ((60, 60, 1), (100000, 126 * 4096, 1), (40000, 20000, 1), (1 << 20, 126 * 65536, 1),
                              (3000, 8257536, 1), (100000, 126 * 4096, 0), (70000, 128 * 300, 0), (5, 7, 0)):
        n = fn(nb_x, nb_y, strip, 148, ctypes.byref(c), ctypes.byref(gx), ctypes.byref(gy))
        assert 0 < n <= 65536 and n == gx.value * gy.value
        assert gy.value <= 65535
        if strip:
            assert gx.value == -(-nb_y // 126)
            assert c.value * gy.value >= nb_x > c.value * (gy.value - 1)
        else:
            assert gx.value == -(-nb_y // 128) and c.value == 0
    # the default shape of 100000 x 516096 would need 391 chunks of 256 rows per strip:
    # 4096 strips leave room for 16, so the chunk grows to 6250 rows
    fn(100000, 126 * 4096, 1, 148, ctypes.byref(c), ctypes.byref(gx), ctypes.byref(gy))
    assert (c.value, gy.value) == (6250, 16)
    assert fn(10, 126 * 65536 + 1, 1, 148, ctypes.byref(c), ctypes.byref(gx), ctypes.byref(gy)) == 0


def test_launch_shape_settings(built):
    """hydro_set_launch_shape (host only): the tile heights the 3D kernels are built for (in
    rows with the halo: 8, 16, and in FP64 also 9 and 12) and the 2D register budgets are
    accepted, anything else rejected with HYDRO_ERR_ARG; 0 restores the built-in shape."""
    fn = built.hydro_set_launch_shape
    fn.argtypes = [ctypes.c_int] * 5
    fn.restype = ctypes.c_int
    for args in ((3, 8, 8, 0, 0), (3, 8, 9, 0, 0), (3, 8, 9, 128, 0), (3, 8, 12, 64, 0), (3, 8, 16, 32, 0),
                 (3, 4, 8, 0, 0), (3, 4, 16, 128, 0),
                 (2, 8, 0, 64, 0), (2, 4, 0, 0, 0), (2, 8, 0, 0, 5), (2, 4, 0, 32, 8), (2, 8, 0, 0, 4)):
        assert fn(*args) == 0, args
    for args in ((3, 4, 12, 0, 0), (3, 4, 9, 0, 0), (3, 8, 10, 0, 0), (3, 8, 7, 0, 0), (2, 8, 9, 0, 0),
                 (2, 8, 8, 0, 0), (4, 8, 0, 0, 0), (3, 2, 8, 0, 0),
                 (3, 8, 8, -1, 0), (2, 8, 0, 0, 8), (2, 4, 0, 0, 5), (3, 8, 8, 0, 4)):
        assert fn(*args) == hb.HYDRO_ERR_ARG, args
    for dim in (2, 3):
        for pb in (4, 8):
            assert fn(dim, pb, 0, 0, 0) == 0
    built.hydro_clear_error()


def test_step_arguments_rejected_before_any_device_call(built):
    """The step entry points reject null pointers and grids past their limits (NB > 2^30 per
    axis, more than 2^40 cells in 2D / 1e12 in 3D) with HYDRO_ERR_ARG and a message, before
    any CUDA call: the pointers below are never dereferenced."""
    fake = ctypes.c_void_p(256)
    d, f, sz = ctypes.c_double, ctypes.c_float, ctypes.c_size_t
    for suf, T in (("f64", d), ("f32", f)):
        fn2 = getattr(built, f"hydro2d_step_{suf}")
        fn2.argtypes = [ctypes.c_void_p] * 5 + [T] * 5 + [sz] * 2 + [T] * 2 + [ctypes.c_void_p, ctypes.c_int,
                                                                             ctypes.c_int, ctypes.c_void_p]
        fn2.restype = ctypes.c_int
        fn3 = getattr(built, f"hydro3d_step_{suf}")
        fn3.argtypes = [ctypes.c_void_p] * 5 + [T] * 5 + [sz] * 3 + [T] * 3 + [ctypes.c_void_p, ctypes.c_int,
                                                                              ctypes.c_int, ctypes.c_void_p]
        fn3.restype = ctypes.c_int
        phys = (0.1, 1.4, 0.4, 1 / 0.4, 1.1)
        cases2 = [((None, fake, fake, fake, fake), (16, 16), "null pointer"),
                  ((fake,) * 5, ((1 << 30) + 1, 4), "too large"),
                  ((fake,) * 5, (4, (1 << 30) + 1), "too large"),
                  ((fake,) * 5, ((1 << 21), (1 << 20)), "too large")]
        for ptrs, nb, msg in cases2:
            built.hydro_clear_error()
            assert fn2(*ptrs, *phys, *nb, 1e-3, 1e-3, None, 0, 1, None) == hb.HYDRO_ERR_ARG, (suf, nb)
            code, text = hb.last_error()
            assert code == hb.HYDRO_ERR_ARG and msg in text, text
        cases3 = [((fake, fake, None, fake, fake), (8, 8, 8), "null pointer"),
                  ((fake,) * 5, ((1 << 30) + 1, 2, 2), "too large"),
                  ((fake,) * 5, (2, 2, (1 << 30) + 1), "too large"),
                  ((fake,) * 5, (10000, 10000, 10001), "too large")]
        for ptrs, nb, msg in cases3:
            built.hydro_clear_error()
            assert fn3(*ptrs, *phys, *nb, 1e-3, 1e-3, 1e-3, None, 0, 1, None) == hb.HYDRO_ERR_ARG, (suf, nb)
            code, text = hb.last_error()
            assert code == hb.HYDRO_ERR_ARG and msg in text, text
    built.hydro_clear_error()
