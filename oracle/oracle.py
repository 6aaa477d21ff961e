"""Oracle bindings (test infrastructure only).

Loads
  * oracle/liboracle.so       the C restatement of the reference path (hydro_oracle.c)
  * oracle/_ref/libref*.so    the reference's own kernel.cxx compiled unchanged (when
                              the reference sources were present at build time)
and exposes them over numpy arrays. Only tests, the smoke check and the CPU-baseline
leg of the benchmark import this module; the product never does.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"

_c_size = ctypes.c_size_t
_vp = ctypes.c_void_p


def build():
    subprocess.run(["make", "-C", str(HERE), "oracle"], check=True, stdout=subprocess.DEVNULL)


def _np_ptr(a):
    return a.ctypes.data_as(_vp)


class Oracle:
    """ctypes view of liboracle.so."""

    def __init__(self):
        if not ORACLE_SO.exists():
            build()
        L = ctypes.CDLL(str(ORACLE_SO))
        d, f = ctypes.c_double, ctypes.c_float
        for T, suf in ((d, "f64"), (f, "f32")):
            fn = getattr(L, f"oracle2d_step_{suf}")
            fn.argtypes = [_vp] * 5 + [T] * 5 + [_c_size] * 2 + [T] * 2
            fn.restype = None
            fn = getattr(L, f"oracle3d_step_{suf}")
            fn.argtypes = [_vp] * 5 + [T] * 5 + [_c_size] * 3 + [T] * 3
            fn.restype = None
            fn = getattr(L, f"oracle2d_init_{suf}")
            fn.argtypes = [_vp, _vp, _c_size, _c_size] + [T] * 6
            fn.restype = T
            fn = getattr(L, f"oracle3d_init_{suf}")
            fn.argtypes = [_vp, _vp, _c_size, _c_size, _c_size] + [T] * 6
            fn.restype = T
            fn = getattr(L, f"oracle2d_ghost_x_{suf}")
            fn.argtypes = [_vp, _vp, _c_size, _c_size]
            fn.restype = None
            fn = getattr(L, f"oracle3d_ghost_x_{suf}")
            fn.argtypes = [_vp, _vp, _c_size, _c_size, _c_size]
            fn.restype = None
            fn = getattr(L, f"oracle_mass_{suf}")
            fn.argtypes = [_vp, _c_size, _c_size, _c_size]
            fn.restype = d
            fn = getattr(L, f"oracle_blast_stats_{suf}")
            fn.argtypes = [_c_size, _c_size, _c_size] + [T] * 6 + [ctypes.POINTER(T)]
            fn.restype = d
            fn = getattr(L, f"oracle_run_{suf}")
            fn.argtypes = [_c_size, _c_size, _c_size, d, _c_size, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(d),
                           ctypes.POINTER(d)]
            fn.restype = _c_size
        self.L = L

    @staticmethod
    def _suf(dtype):
        return "f64" if np.dtype(dtype) == np.float64 else "f32"

    def step(self, cur, nxt, phys, dtd):
        """One reference step on numpy state tuples (rhoE, uvx); returns Dt_next."""
        T = np.dtype(cur[0].dtype).type
        dt = np.zeros(1, dtype=T)
        nb = phys.nb
        if len(nb) == 2:
            getattr(self.L, f"oracle2d_step_{self._suf(T)}")(
                _np_ptr(cur[0]), _np_ptr(cur[1]), _np_ptr(nxt[0]), _np_ptr(nxt[1]), _np_ptr(dt), phys.C_min,
                phys.g, phys.gm1, phys.divgamma, phys.k, nb[0], nb[1], dtd[0], dtd[1])
        else:
            getattr(self.L, f"oracle3d_step_{self._suf(T)}")(
                _np_ptr(cur[0]), _np_ptr(cur[1]), _np_ptr(nxt[0]), _np_ptr(nxt[1]), _np_ptr(dt), phys.C_min,
                phys.g, phys.gm1, phys.divgamma, phys.k, nb[0], nb[1], nb[2], dtd[0], dtd[1], dtd[2])
        return T(dt[0])

    def ghost_x(self, st, nb):
        T = np.dtype(st[0].dtype).type
        if len(nb) == 2:
            getattr(self.L, f"oracle2d_ghost_x_{self._suf(T)}")(_np_ptr(st[0]), _np_ptr(st[1]), nb[0], nb[1])
        else:
            getattr(self.L, f"oracle3d_ghost_x_{self._suf(T)}")(_np_ptr(st[0]), _np_ptr(st[1]), *nb)

    def init(self, st, phys, rho_in=1.0, rho_out=1.2, p_in=10.0, p_out=0.1):
        T = np.dtype(st[0].dtype).type
        args = [T(rho_in), T(rho_out), T(p_in), T(p_out), phys.C_min, phys.g]
        if len(phys.nb) == 2:
            return T(getattr(self.L, f"oracle2d_init_{self._suf(T)}")(_np_ptr(st[0]), _np_ptr(st[1]), *phys.nb,
                                                                       *args))
        return T(getattr(self.L, f"oracle3d_init_{self._suf(T)}")(_np_ptr(st[0]), _np_ptr(st[1]), *phys.nb, *args))

    def blast_stats(self, nb, phys, rho_in=1.0, rho_out=1.2, p_in=10.0, p_out=0.1):
        """(initial mass, first Dt) of the blast IC without storing the grid."""
        T = phys.dtype
        CT = ctypes.c_double if T is np.float64 else ctypes.c_float
        out = CT(0)
        nbz = nb[2] if len(nb) == 3 else 0
        m = getattr(self.L, f"oracle_blast_stats_{self._suf(T)}")(nb[0], nb[1], nbz, T(rho_in), T(rho_out), T(p_in),
                                                                   T(p_out), phys.C_min, phys.g, ctypes.byref(out))
        return m, T(out.value)

    def mass(self, rhoE, nb):
        T = np.dtype(rhoE.dtype).type
        nbz = nb[2] if len(nb) == 3 else 0
        return getattr(self.L, f"oracle_mass_{self._suf(T)}")(_np_ptr(rhoE), nb[0], nb[1], nbz)

    def run(self, nb, dtype, max_t, max_it):
        """The reference host loop from the blast IC (one rank, one subdomain).
        Returns dict(state=(rhoE, uvx), t=[...], dt=[...], first_dt, mass0, mass1, it)."""
        T = np.dtype(dtype).type
        nb = tuple(int(n) for n in nb)
        ncell = int(np.prod([n + 2 for n in nb]))
        nv = 3 if len(nb) == 3 else 2
        rhoE = np.zeros(2 * ncell, dtype=T)
        uvx = np.zeros(nv * ncell, dtype=T)
        t_log = np.zeros(max(1, max_it), dtype=np.float64)
        dt_log = np.zeros(max(1, max_it), dtype=T)
        first = np.zeros(1, dtype=T)
        m0, m1 = ctypes.c_double(0), ctypes.c_double(0)
        nbz = nb[2] if len(nb) == 3 else 0
        it = getattr(self.L, f"oracle_run_{self._suf(T)}")(nb[0], nb[1], nbz, float(max_t), int(max_it),
                                                            _np_ptr(rhoE), _np_ptr(uvx), _np_ptr(t_log),
                                                            _np_ptr(dt_log), _np_ptr(first), ctypes.byref(m0),
                                                            ctypes.byref(m1))
        return dict(state=(rhoE, uvx), t=t_log[:it], dt=dt_log[:it], first_dt=T(first[0]), mass0=m0.value,
                    mass1=m1.value, it=int(it))


class RefKernel:
    """The reference's own kernel.cxx (unchanged, strict IEEE order) as a shared
    object exporting `launcher`; the SYCL stand-in runs its single_task inline."""

    def __init__(self, dim: int, dtype, fast: bool = False, level: str = ""):
        """fast: the reference Makefile's -O2 with FMA contraction (x86-64-v3, or the
        instruction-set level `level`, e.g. "v4"); else strict IEEE order."""
        T = np.dtype(dtype).type
        suf = ("f64" if T is np.float64 else "f32") + ("_fast" if fast else "") + (f"_{level}" if level else "")
        path = REF_DIR / f"libref{dim}d_{suf}.so"
        if not path.exists():
            raise FileNotFoundError(path)
        L = ctypes.CDLL(str(path))
        CT = ctypes.c_double if T is np.float64 else ctypes.c_float
        P = ctypes.POINTER(CT)
        # the empty sycl::queue argument of the stand-in occupies no register or stack
        # slot, so it is omitted from the foreign signature
        if dim == 2:
            L.launcher.argtypes = [_vp] * 5 + [CT] * 5 + [_c_size] * 2 + [P, P]
        else:
            L.launcher.argtypes = [_vp] * 5 + [CT] * 5 + [_c_size] * 3 + [P, P, P]
        L.launcher.restype = ctypes.c_double
        self.L, self.T, self.CT, self.dim = L, T, CT, dim

    def step(self, cur, nxt, phys, dtd):
        dt = np.zeros(1, dtype=self.T)
        refs = [self.CT(x) for x in dtd]
        nb = phys.nb
        self.L.launcher(_np_ptr(cur[0]), _np_ptr(cur[1]), _np_ptr(nxt[0]), _np_ptr(nxt[1]), _np_ptr(dt),
                        phys.C_min, phys.g, phys.gm1, phys.divgamma, phys.k, *nb, *[ctypes.byref(r) for r in refs])
        return self.T(dt[0])


def available_ref(dim: int, dtype, fast: bool = False, level: str = "") -> bool:
    suf = ("f64" if np.dtype(dtype) == np.float64 else "f32") + ("_fast" if fast else "") + (f"_{level}" if level else "")
    return (REF_DIR / f"libref{dim}d_{suf}.so").exists()


def host_loop(stepper, init_state, phys, first_dt, max_t, max_it):
    """The reference's host loop (hydro2d/main.cxx:686-815) around any step function
    stepper(cur, nxt, phys, dtd) -> Dt_next operating on numpy state tuples: periodic X
    ghost copy (main.cxx:349-378), DtDx = Dt/DX in T, swap, Dt = min(1e20, Dt_next),
    t += Dt. Returns (final state, t list, dt list)."""
    T = phys.dtype
    nb = phys.nb
    cur = tuple(a.copy() for a in init_state)
    nxt = tuple(np.zeros_like(a) for a in init_state)
    big = T(1e20)
    dt = first_dt if first_dt < big else big
    t, it = 0.0, 0
    t_log, dt_log = [], []
    while t < max_t and it < max_it:
        ghost_x_numpy(cur, nb)
        dtn = stepper(cur, nxt, phys, phys.dtd(dt))
        cur, nxt = nxt, cur
        dt = dtn if dtn < big else big
        t_log.append(t)
        dt_log.append(dt)
        it += 1
        t += float(dt)
    return cur, t_log, dt_log


def interior(st, nb):
    """The interior cells of a state tuple as (rhoE, uvx) arrays of shape nb + (nv,).
    Ghost cells are excluded: the reference host writes the X ghosts of its copy, the
    device kernels never read or write them."""
    nv = 3 if len(nb) == 3 else 2
    shape = tuple(n + 2 for n in nb)
    inner = tuple(slice(1, n + 1) for n in nb)
    return (st[0].reshape(shape + (2,))[inner], st[1].reshape(shape + (nv,))[inner])


def interior_digest(st, nb):
    """SHA-256 of the interior cells' bytes (rhoE then uvx, row-major)."""
    import hashlib

    h = hashlib.sha256()
    for a in interior(st, nb):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def ghost_x_numpy(st, nb):
    """Periodic X ghost rows/planes by copy (hydro2d/main.cxx:349-378)."""
    plane = int(np.prod([n + 2 for n in nb[1:]]))
    nv = 3 if len(nb) == 3 else 2
    for a, w in ((st[0], 2), (st[1], nv)):
        v = a.reshape(nb[0] + 2, plane * w)
        v[0] = v[nb[0]]
        v[nb[0] + 1] = v[1]
