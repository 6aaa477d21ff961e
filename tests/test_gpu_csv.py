"""CSV output formatted on the GPU (scope row f1): every value as std::ostream / printf
"%g" writes it (checked against the C library's snprintf on adversarial doubles), and
whole files byte-identical to the reference program's own CSV output."""
from __future__ import annotations

import ctypes
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_pkg

hb = load_pkg()
pytestmark = pytest.mark.gpu
REFDIR = ROOT / "oracle" / "_ref"
_libc = ctypes.CDLL(None)


def printf_g(v: float) -> str:
    buf = ctypes.create_string_buffer(64)
    _libc.snprintf(buf, 64, b"%g", ctypes.c_double(v))
    return buf.value.decode()


def adversarial_values(n_random=200000, seed=5):
    rng = np.random.default_rng(seed)
    bits = rng.integers(0, 2 ** 64, n_random, dtype=np.uint64)
    vals = list(bits.view(np.float64))
    # subnormals, extremes, zeros and non-finite values
    vals += [5e-324, -5e-324, 2.2250738585072014e-308, 2.225073858507201e-308, 1.7976931348623157e308,
             0.0, -0.0, float("inf"), -float("inf"), float("nan"), -float("nan")]
    vals += list(rng.integers(1, 2 ** 52, 2000).astype(np.float64) * 5e-324)
    # decade boundaries and values that round across them
    for e in range(-310, 309):
        for m in (1.0, 9.999995, 9.9999949999, 9.99999500001, 1.000005, 0.99999949999):
            try:
                vals.append(float(f"{m}e{e}"))
            except OverflowError:
                pass
    # exact ties at the 6th significant digit (half-even) and near-ties
    vals += [123456.5, 123457.5, 999999.5, 1000000.5, 0.5, 2.5, 1.5, 12345650.0, 12345750.0, 1.0000005,
             100000.0, 99999.95, 0.0001, 0.00001, 9.9999995e-5, 1e-4, 1e-5, 1e6, 999999.0, 1e5]
    vals += list(np.nextafter(np.array(vals[-20:]), np.inf)) + list(np.nextafter(np.array(vals[-20:]), -np.inf))
    # the ranges the solver prints (densities, energies, momenta down to subnormal tails)
    vals += list(rng.uniform(-30, 30, 20000)) + list(rng.uniform(0.1, 30, 20000).astype(np.float32).astype(np.float64))
    vals += list(10.0 ** rng.uniform(-330, 308, 20000))
    return np.array(vals, dtype=np.float64)


def test_format_g_matches_printf(cuda):
    v = adversarial_values()
    got = hb.format_g(v)
    bad = [(x, g, printf_g(float(x))) for x, g in zip(v, got) if g != printf_g(float(x))]
    assert not bad, bad[:10]


def _reference_csv(prog, args, tmp_path):
    exe = REFDIR / f"{prog}.cpu"
    if not exe.exists():
        pytest.skip("oracle/_ref reference programs not built")
    d = tmp_path / "ref"
    d.mkdir()
    p = subprocess.run([str(exe)] + args, cwd=d, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    return d


@pytest.mark.parametrize("prog,nb,T,steps", [("hydro", (60, 60), np.float64, 100), ("hydro", (200, 150), np.float64, 300),
                                             ("hydro_float", (60, 60), np.float32, 100),
                                             ("hydro3d", (20, 16, 12), np.float64, 40),
                                             ("hydro3d_float", (20, 16, 12), np.float32, 40)])
def test_write_csv_matches_reference_program(cuda, prog, nb, T, steps, tmp_path):
    """The state after `steps` steps written on the GPU equals, byte for byte, the file the
    reference program writes at that iteration (hydro2d/main.cxx:166-235)."""
    dims = ["-x", str(nb[0]), "-y", str(nb[1])] + (["-z", str(nb[2])] if len(nb) == 3 else [])
    ref = _reference_csv(prog, dims + ["-t", "100", "-i", str(steps), "-w", str(steps)], tmp_path)
    files = sorted(ref.glob(f"output_{steps}_*.csv"))
    assert len(files) == 1, list(ref.iterdir())
    run = hb.BlastRun(nb, T, arith="strict").run(1e9, steps)
    out = tmp_path / "gpu.csv"
    n = hb.write_csv(run.cur, nb, out)
    data = out.read_bytes()
    assert n == len(data)
    assert data == files[0].read_bytes()


@pytest.mark.parametrize("chunk_cells", [7000, 150, 1])
def test_write_csv_many_chunks(cuda, chunk_cells, tmp_path, monkeypatch):
    """The chunked pipeline (format, scan, compact, double-buffered copy and write) gives
    the same file whatever the chunk size: many chunks, one row per chunk, and chunks
    smaller than a row (one row each)."""
    nb, steps = (200, 150), 300
    ref = _reference_csv("hydro", ["-x", "200", "-y", "150", "-t", "100", "-i", str(steps), "-w", str(steps)],
                         tmp_path)
    files = sorted(ref.glob(f"output_{steps}_*.csv"))
    run = hb.BlastRun(nb, np.float64, arith="strict").run(1e9, steps)
    monkeypatch.setenv("HYDRO_B200_CSV_CHUNK_CELLS", str(chunk_cells))
    out = tmp_path / "gpu.csv"
    hb.write_csv(run.cur, nb, out)
    assert out.read_bytes() == files[0].read_bytes()
