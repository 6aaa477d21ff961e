"""Python host side of the B200 finite-volume library.

A thin ctypes layer over the C ABI of ``include/hydro_b200.h`` (``lib/libhydro_b200.so``)
plus ``BlastRun``, a restatement of the reference's host time loop for one rank and one
subdomain (hydro2d/main.cxx:595-836, hydro3d/main.cxx:642-900): blast initial condition,
first Dt, per-step DtDx = Dt/DX in the state's precision, launcher call, swap, Dt MIN,
``t += Dt`` with the newly reduced Dt (the reference's order), mass check.

PyTorch provides device memory and streams only; every kernel is this project's CUDA.
There is no CPU fallback: without the built library or a GPU the calls raise.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_DIR = PKG_DIR / "lib"
LIB_PATH = LIB_DIR / "libhydro_b200.so"

KERNEL_AUTO, KERNEL_STRIP, KERNEL_DIRECT = 0, 1, 2
# X neighbours of the first and last interior rows (planes) from the input's ghost rows
# instead of the in-kernel periodic wrap (include/hydro_b200.h)
X_GHOSTS_FROM_MEMORY = 0x100
# arithmetic of a step (include/hydro_b200.h): strict (the reference's order, bit-identical)
# or fused (fma contraction, refined hardware reciprocal / square root)
ARITH_FUSED, ARITH_STRICT = 0x200, 0x400
_ARITH_BITS = {None: 0, "strict": ARITH_STRICT, "fused": ARITH_FUSED}
HYDRO_OK, HYDRO_ERR_ARG, HYDRO_ERR_CUDA, HYDRO_ERR_NONPHYSICAL, HYDRO_ERR_TIMEOUT = 0, -1, -2, -3, -4

_c_size = ctypes.c_size_t
_vp = ctypes.c_void_p


class HydroError(RuntimeError):
    """A library entry point returned an error code."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"hydro_b200 error {code}: {msg}")
        self.code = code


class Queue(ctypes.Structure):
    """hydro_queue_t: the by-value queue argument of the drop-in launchers."""

    _fields_ = [("stream", _vp), ("device", ctypes.c_int), ("flags", ctypes.c_int)]


class StepInfo(ctypes.Structure):
    """hydro_step_info_t"""

    _fields_ = [("mass", ctypes.c_double), ("max_speed", ctypes.c_double), ("err", ctypes.c_uint),
                ("kernel", ctypes.c_int)]


def build(force: bool = False) -> None:
    """Compile the CUDA library in-tree (sm_100a) with the package Makefile. The make is
    incremental: it rebuilds whatever is older than its sources and headers, so a kernel
    edited since the last build is never run from a stale binary. Where no CUDA compiler
    is installed (a machine that only runs a prebuilt tree) an existing library is used."""
    nvcc = Path(os.environ.get("CUDA", "/usr/local/cuda")) / "bin" / "nvcc"
    if not nvcc.exists() and LIB_PATH.exists() and not force:
        return
    # one make at a time (ranks of one job build the same tree); make's report goes to
    # stderr: stdout belongs to the caller (bench.py prints one JSON line)
    import fcntl

    LIB_DIR.mkdir(exist_ok=True)
    with open(LIB_DIR / ".build.lock", "w") as lock:
        fcntl.flock(lock, fcntl.LOCK_EX)
        p = subprocess.run(["make", "-C", str(PKG_DIR), "-j8", "--no-print-directory"] + (["-B"] if force else []),
                           stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if p.stdout and "Nothing to be done" not in p.stdout:
        sys.stderr.write(p.stdout)
    if p.returncode != 0:
        raise HydroError(-1, f"building the CUDA library failed (make exit {p.returncode})")


_lib = None


def _declare(lib):
    d, f = ctypes.c_double, ctypes.c_float
    pd, pf = ctypes.POINTER(d), ctypes.POINTER(f)
    for T, P, suf in ((d, pd, "f64"), (f, pf, "f32")):
        fn = getattr(lib, f"hydro2d_launcher_{suf}")
        fn.argtypes = [_vp] * 5 + [T] * 5 + [_c_size] * 2 + [P, P, Queue]
        fn.restype = d
        fn = getattr(lib, f"hydro3d_launcher_{suf}")
        fn.argtypes = [_vp] * 5 + [T] * 5 + [_c_size] * 3 + [P, P, P, Queue]
        fn.restype = d
        fn = getattr(lib, f"hydro2d_step_{suf}")
        fn.argtypes = [_vp] * 5 + [T] * 5 + [_c_size] * 2 + [T] * 2 + [_vp, ctypes.c_int, ctypes.c_int,
                                                                      ctypes.POINTER(StepInfo)]
        fn.restype = ctypes.c_int
        fn = getattr(lib, f"hydro3d_step_{suf}")
        fn.argtypes = [_vp] * 5 + [T] * 5 + [_c_size] * 3 + [T] * 3 + [_vp, ctypes.c_int, ctypes.c_int,
                                                                      ctypes.POINTER(StepInfo)]
        fn.restype = ctypes.c_int
        fn = getattr(lib, f"hydro2d_init_blast_{suf}")
        fn.argtypes = [_vp, _vp, _c_size, _c_size] + [T] * 6 + [P, _vp]
        fn.restype = ctypes.c_int
        fn = getattr(lib, f"hydro3d_init_blast_{suf}")
        fn.argtypes = [_vp, _vp, _c_size, _c_size, _c_size] + [T] * 6 + [P, _vp]
        fn.restype = ctypes.c_int
        fn = getattr(lib, f"hydro_mass_{suf}")
        fn.argtypes = [_vp, _c_size, _c_size, _c_size, pd, _vp]
        fn.restype = ctypes.c_int
    lib.hydro_set_launch_shape.argtypes = [ctypes.c_int] * 5
    lib.hydro_set_launch_shape.restype = ctypes.c_int
    lib.hydro_last_launch_shape.argtypes = [ctypes.POINTER(ctypes.c_int)] * 4
    lib.hydro_last_launch_shape.restype = ctypes.c_int
    lib.hydro_last_step_info.argtypes = [ctypes.POINTER(StepInfo)]
    lib.hydro_last_step_info.restype = ctypes.c_int
    lib.hydro_last_error.restype = ctypes.c_int
    lib.hydro_last_error_string.restype = ctypes.c_char_p
    lib.hydro_clear_error.restype = None
    lib.hydro_version.restype = ctypes.c_char_p
    return lib


def lib():
    """The loaded C library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}`")
        _lib = _declare(ctypes.CDLL(str(LIB_PATH)))
    return _lib


def set_launch_shape(dim: int, dtype, warps: int = 0, chunk: int = 0, blocks: int = 0):
    """Launch shape of the plain strip kernels for (dim, precision): 3D warps per block
    (tile rows with halo), rows / planes per block, 2D register budget in blocks per SM
    (0 = built-in for each). Results do not depend on it."""
    _check(lib().hydro_set_launch_shape(int(dim), np.dtype(dtype).itemsize, int(warps), int(chunk), int(blocks)))


def last_launch_shape() -> dict:
    """The shape the last strip-kernel step on the current device used."""
    w, c, b, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _check(lib().hydro_last_launch_shape(ctypes.byref(w), ctypes.byref(c), ctypes.byref(b), ctypes.byref(t)))
    return dict(warps=w.value, chunk=c.value, blocks=b.value, tma=bool(t.value))


def last_error() -> tuple[int, str]:
    L = lib()
    return L.hydro_last_error(), L.hydro_last_error_string().decode()


def _check(rc: int):
    if rc != HYDRO_OK:
        code, msg = last_error()
        raise HydroError(rc, msg)


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("hydro_b200 needs a CUDA device; there is no CPU fallback")
    return torch


def _stream_handle(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class _nullctx:
    def __enter__(self):
        return None

    def __exit__(self, *a):
        return False


# --------------------------------------------------------------------------- physics ---
@dataclass
class Physics:
    """The reference's constants in the state's precision (hydro2d/main.cxx:595-607,
    hydro3d/main.cxx:642-655): C = 0.5 (2D) / 0.4 (3D), gamma = 1.4, K = 1.1,
    DX = 1/(NB_X+1), C_min = C * min(DX, DY[, DZ])."""

    dtype: type
    nb: tuple
    C: float = None
    gamma: float = 1.4
    K: float = 1.1
    consts: dict = field(default_factory=dict)

    def __post_init__(self):
        T = self.dtype
        if self.C is None:
            self.C = 0.4 if len(self.nb) == 3 else 0.5
        one = T(1)
        self.D = [one / T(n + 1) for n in self.nb]
        ms = self.D[0]
        for d in self.D[1:]:
            ms = d if d < ms else ms  # std::min({..}) keeps the first smallest
        self.min_spacing = ms
        self.Cc = T(self.C)
        self.C_min = T(self.Cc * ms)
        self.g = T(self.gamma)
        self.k = T(self.K)
        self.gm1 = T(self.g - one)
        self.divgamma = T(one / self.gm1)

    def dtd(self, dt):
        """DtDx, DtDy[, DtDz] = Dt / DX ... in the state's precision (main.cxx:703-704)."""
        T = self.dtype
        return [T(T(dt) / d) for d in self.D]


# ----------------------------------------------------------------------- drop-in ABI ---
def launcher2d(rhoE, uv, rhoE_next, uv_next, dt_next, C_min, gamma, gm1, divgamma, K, nb_x, nb_y, DtDx, DtDy,
               stream=None, device=-1, arith=None):
    """The reference launcher signature (hydro2d/kernel.hpp:63-68) over torch tensors;
    returns the elapsed microseconds like the reference (negative on error)."""
    L = lib()
    f64 = rhoE.dtype.itemsize == 8
    T, fn = (ctypes.c_double, L.hydro2d_launcher_f64) if f64 else (ctypes.c_float, L.hydro2d_launcher_f32)
    dx, dy = T(DtDx), T(DtDy)
    q = Queue(_stream_handle(stream), device, _ARITH_BITS[arith])
    return fn(_ptr(rhoE), _ptr(uv), _ptr(rhoE_next), _ptr(uv_next), _ptr(dt_next), C_min, gamma, gm1, divgamma, K,
              nb_x, nb_y, ctypes.byref(dx), ctypes.byref(dy), q)


def launcher3d(rhoE, uvw, rhoE_next, uvw_next, dt_next, C_min, gamma, gm1, divgamma, K, nb_x, nb_y, nb_z, DtDx,
               DtDy, DtDz, stream=None, device=-1, arith=None):
    """The reference launcher signature (hydro3d/kernel.hpp:64-69) over torch tensors."""
    L = lib()
    f64 = rhoE.dtype.itemsize == 8
    T, fn = (ctypes.c_double, L.hydro3d_launcher_f64) if f64 else (ctypes.c_float, L.hydro3d_launcher_f32)
    dx, dy, dz = T(DtDx), T(DtDy), T(DtDz)
    q = Queue(_stream_handle(stream), device, _ARITH_BITS[arith])
    return fn(_ptr(rhoE), _ptr(uvw), _ptr(rhoE_next), _ptr(uvw_next), _ptr(dt_next), C_min, gamma, gm1, divgamma,
              K, nb_x, nb_y, nb_z, ctypes.byref(dx), ctypes.byref(dy), ctypes.byref(dz), q)


def step(state_in, state_out, dt_next, phys: Physics, dtd, kernel=KERNEL_AUTO, sync=True, stream=None,
         check=True, x_ghosts=False, arith=None):
    """One step through hydro{2d,3d}_step_{f64,f32}. state_* = (rhoE, uvx) tensors.
    x_ghosts: read the X ghost rows (planes) of state_in instead of wrapping periodically.
    arith: "strict", "fused" or None (the library default)."""
    L = lib()
    if x_ghosts:
        kernel |= X_GHOSTS_FROM_MEMORY
    kernel |= _ARITH_BITS[arith]
    f64 = phys.dtype is np.float64
    suf = "f64" if f64 else "f32"
    info = StepInfo()
    p = phys
    if len(p.nb) == 2:
        fn = getattr(L, f"hydro2d_step_{suf}")
        rc = fn(_ptr(state_in[0]), _ptr(state_in[1]), _ptr(state_out[0]), _ptr(state_out[1]), _ptr(dt_next),
                p.C_min, p.g, p.gm1, p.divgamma, p.k, p.nb[0], p.nb[1], dtd[0], dtd[1], _stream_handle(stream),
                kernel, 1 if sync else 0, ctypes.byref(info))
    else:
        fn = getattr(L, f"hydro3d_step_{suf}")
        rc = fn(_ptr(state_in[0]), _ptr(state_in[1]), _ptr(state_out[0]), _ptr(state_out[1]), _ptr(dt_next),
                p.C_min, p.g, p.gm1, p.divgamma, p.k, p.nb[0], p.nb[1], p.nb[2], dtd[0], dtd[1], dtd[2],
                _stream_handle(stream), kernel, 1 if sync else 0, ctypes.byref(info))
    if check:
        _check(rc)
    return rc, info


def init_blast(state, phys: Physics, rho_in=1.0, rho_out=1.2, p_in=10.0, p_out=0.1, stream=None):
    """Device blast initial condition; returns the first Dt (state's precision)."""
    L = lib()
    T = phys.dtype
    f64 = T is np.float64
    CT = ctypes.c_double if f64 else ctypes.c_float
    out = CT(0)
    suf = "f64" if f64 else "f32"
    args = [T(rho_in), T(rho_out), T(p_in), T(p_out), phys.C_min, phys.g]
    if len(phys.nb) == 2:
        rc = getattr(L, f"hydro2d_init_blast_{suf}")(_ptr(state[0]), _ptr(state[1]), *phys.nb, *args,
                                                    ctypes.byref(out), _stream_handle(stream))
    else:
        rc = getattr(L, f"hydro3d_init_blast_{suf}")(_ptr(state[0]), _ptr(state[1]), *phys.nb, *args,
                                                    ctypes.byref(out), _stream_handle(stream))
    _check(rc)
    return T(out.value)


def init_blast_at(state, phys: Physics, blast, stream=None):
    """Device blast IC with the explicit centre/radius/densities of a `Blast`; first Dt."""
    L = lib()
    T = phys.dtype
    f64 = T is np.float64
    CT = ctypes.c_double if f64 else ctypes.c_float
    suf = "f64" if f64 else "f32"
    fn = getattr(L, f"hydro{len(phys.nb)}d_init_blast_at_{suf}")
    d = ctypes.c_double
    nd = len(phys.nb)
    fn.argtypes = [_vp, _vp] + [_c_size] * nd + [d] * (nd + 1) + [CT] * 6 + [ctypes.POINTER(CT), _vp]
    fn.restype = ctypes.c_int
    out = CT(0)
    _check(fn(_ptr(state[0]), _ptr(state[1]), *phys.nb, *[float(c) for c in blast.centre[:nd]], float(blast.radius),
              T(blast.rho_in), T(blast.rho_out), T(blast.p_in), T(blast.p_out), phys.C_min, phys.g,
              ctypes.byref(out), _stream_handle(stream)))
    return T(out.value)


def mass(rhoE, nb, stream=None) -> float:
    """Compensated FP64 sum of the interior density (device)."""
    L = lib()
    f64 = rhoE.dtype.itemsize == 8
    out = ctypes.c_double(0)
    nbz = nb[2] if len(nb) == 3 else 0
    fn = L.hydro_mass_f64 if f64 else L.hydro_mass_f32
    _check(fn(_ptr(rhoE), nb[0], nb[1], nbz, ctypes.byref(out), _stream_handle(stream)))
    return out.value


def write_csv(state, nb, path, i_offset=0, stream=None) -> int:
    """The state (reference layout, device tensors) as the reference's CSV output file,
    formatted on the GPU (hydro{2d,3d}_write_csv_*); returns the bytes written."""
    L = lib()
    f64 = state[0].dtype.itemsize == 8
    suf = "f64" if f64 else "f32"
    fn = getattr(L, f"hydro{len(nb)}d_write_csv_{suf}")
    fn.argtypes = [_vp, _vp] + [_c_size] * (len(nb) + 1) + [ctypes.c_char_p, _vp]
    fn.restype = ctypes.c_longlong
    n = fn(_ptr(state[0]), _ptr(state[1]), *[int(x) for x in nb], int(i_offset), str(path).encode(),
           _stream_handle(stream))
    if n < 0:
        raise HydroError(int(n), last_error()[1])
    return int(n)


def format_g(values) -> list:
    """printf("%g") of each double, formatted on the GPU (hydro_format_g)."""
    torch = _torch()
    v = torch.as_tensor(np.ascontiguousarray(values, dtype=np.float64)).cuda()
    out = torch.zeros(max(1, v.numel()) * 16, dtype=torch.uint8, device="cuda")
    L = lib()
    L.hydro_format_g.argtypes = [_vp, _c_size, _vp, _vp]
    L.hydro_format_g.restype = ctypes.c_int
    _check(L.hydro_format_g(_ptr(v), v.numel(), _ptr(out), None))
    raw = out.cpu().numpy().reshape(-1, 16)[:v.numel()]
    return [bytes(r).split(b"\0", 1)[0].decode() for r in raw]


def alloc_state(nb, dtype, device="cuda"):
    """(rhoE, uv[w]) device arrays of the reference layout, zero-initialised."""
    torch = _torch()
    tdt = torch.float64 if dtype is np.float64 else torch.float32
    ncell = 1
    for n in nb:
        ncell *= n + 2
    nv = 3 if len(nb) == 3 else 2
    return (torch.zeros(2 * ncell, dtype=tdt, device=device), torch.zeros(nv * ncell, dtype=tdt, device=device))


class BlastRun:
    """The reference's host loop for one rank and one subdomain covering the domain
    (hydro2d/main.cxx:686-815): state stays on the device; each step reads the new Dt
    back (the only per-step device-to-host copy the loop needs)."""

    def __init__(self, nb, dtype=np.float64, kernel=KERNEL_AUTO, stream=None, blast=None, arith=None):
        """`blast` (a hydro_b200.batch.Blast) overrides the reference's initial condition
        and constants with an explicit centre, radius, densities, pressures, gamma, K, C.
        `arith`: "strict", "fused" or None (the library default)."""
        torch = _torch()
        self.nb = tuple(int(n) for n in nb)
        self.T = dtype
        self.arith = arith
        if blast is None:
            self.phys = Physics(dtype, self.nb)
        else:
            self.phys = Physics(dtype, self.nb, C=blast.C, gamma=blast.gamma, K=blast.K)
        self.kernel = kernel
        self.stream = stream
        with torch.cuda.stream(stream) if stream is not None else _nullctx():
            self.cur = alloc_state(self.nb, dtype)
            self.nxt = alloc_state(self.nb, dtype)
        tdt = torch.float64 if dtype is np.float64 else torch.float32
        self.dt_dev = torch.zeros(1, dtype=tdt, device="cuda")
        if blast is None:
            self.first_dt = init_blast(self.cur, self.phys, stream=stream)
        else:
            self.first_dt = init_blast_at(self.cur, self.phys, blast, stream=stream)
        big = dtype(1e20)
        self.dt = self.first_dt if not (big < self.first_dt) else big
        self.t = 0.0
        self.it = 0
        self.t_log: list[float] = []
        self.dt_log: list = []
        self.mass0 = mass(self.cur[0], self.nb, stream)
        self.last_info = None

    def step_kernel_only(self):
        """Enqueue this step's kernel on the stream without waiting."""
        dtd = self.phys.dtd(self.dt)
        step(self.cur, self.nxt, self.dt_dev, self.phys, dtd, kernel=self.kernel, sync=False, stream=self.stream,
             arith=self.arith)

    def step_finish(self):
        """Wait for the step, check its status, swap buffers and read the new Dt back."""
        torch = _torch()
        (self.stream or torch.cuda.current_stream()).synchronize()
        info = StepInfo()
        _check(lib().hydro_last_step_info(ctypes.byref(info)))
        self.last_info = info
        self.cur, self.nxt = self.nxt, self.cur
        dtn = self.T(self.dt_dev.item())
        big = self.T(1e20)
        self.dt = dtn if dtn < big else big
        self.t_log.append(self.t)
        self.dt_log.append(self.dt)
        self.it += 1
        self.t += float(self.dt)

    def step(self):
        self.step_kernel_only()
        self.step_finish()

    def run(self, max_t: float, max_it: int):
        while self.t < max_t and self.it < max_it:
            self.step()
        return self

    def mass(self):
        return mass(self.cur[0], self.nb, self.stream)

    def host_state(self):
        """(rhoE, uvx) as numpy arrays of the reference layout."""
        return self.cur[0].cpu().numpy(), self.cur[1].cpu().numpy()
