"""ctypes wrapper of the oracle (oracle/tild_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / reference legs, as the checker the CUDA library is compared against.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        vp, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
        fp, dp, ip = C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_int32)
        sig = {
            "orc_create": ([vp, C.POINTER(vp)], i32), "orc_destroy": ([vp], None),
            "orc_set_topology": ([vp, ip, fp, ip, ip, ip], i32),
            "orc_forces": ([vp, fp, i64, dp, dp], i32), "orc_step": ([vp, fp, fp, fp, i64, i32, dp], i32),
            "orc_observables": ([vp, fp, vp], i32), "orc_sk": ([vp, i32, dp], i32),
            "orc_stencil": ([vp, fp, ip, dp], i32), "orc_grid_field": ([vp, dp], i32),
            "orc_nlist": ([vp, fp, C.c_float, i32, ip, ip, ip, ip], i32),
            "orc_fft": ([i32, ip, dp, i32], i32), "orc_noise3": ([C.c_uint64, C.c_uint32, i64, C.c_uint32, dp], i32),
            "orc_set_threads": ([i32], None), "orc_max_threads": ([], i32),
        }
        for n, (a, r) in sig.items():
            f = getattr(L, n)
            f.argtypes = a
            f.restype = r
        _lib = L
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def fft(data: np.ndarray, sign: int) -> np.ndarray:
    """Unnormalised FFT over all axes of `data` (axis order z, y, x with x fastest)."""
    a = np.ascontiguousarray(data, dtype=np.complex128).copy()
    nx = np.array(a.shape[::-1], dtype=np.int32)
    lib().orc_fft(len(nx), _p(nx, C.c_int32), a.ctypes.data_as(C.POINTER(C.c_double)), sign)
    return a


def noise3(seed: int, bead: int, step: int, integ: int) -> np.ndarray:
    out = np.zeros(3)
    lib().orc_noise3(seed, bead, step, integ, _p(out, C.c_double))
    return out


def set_threads(n: int):
    lib().orc_set_threads(n)


def max_threads() -> int:
    return lib().orc_max_threads()


class Oracle:
    """FP64 restatement of one system (same System description as the CUDA context)."""

    def __init__(self, system):
        import tild  # the shared System / Config description
        self.sys = system
        self._cfg = system.config()
        h = C.c_void_p()
        st = lib().orc_create(C.byref(self._cfg), C.byref(h))
        if st:
            raise RuntimeError(f"orc_create failed: {st}")
        self._h = h
        self.ns, self.dim = system.ns, system.dim
        self.M = int(np.prod([system.nx[d] for d in range(system.dim)]))
        self.S = (system.pmeorder + 1) ** system.dim
        s = system
        self._types = np.ascontiguousarray(s.types, np.int32)
        self._q = None if s.charges is None else np.ascontiguousarray(s.charges, np.float32)
        self._nb = np.ascontiguousarray(s.n_bonds, np.int32)
        self._bt = np.ascontiguousarray(s.bonded_to, np.int32).reshape(-1)
        self._by = np.ascontiguousarray(s.bond_type, np.int32).reshape(-1)
        st = lib().orc_set_topology(self._h, _p(self._types, C.c_int32), _p(self._q, C.c_float),
                                    _p(self._nb, C.c_int32), _p(self._bt, C.c_int32), _p(self._by, C.c_int32))
        if st:
            raise RuntimeError(f"orc_set_topology failed: {st}")
        self._tild = tild

    def close(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forces(self, x, step: int = 0, want_rho: bool = False):
        x = np.ascontiguousarray(x, np.float32)
        f = np.zeros((self.ns, self.dim), np.float64)
        nch = self.sys.ntypes + (1 if self.sys.charges is not None else 0)
        rho = np.zeros((nch, self.M)) if want_rho else None
        st = lib().orc_forces(self._h, _p(x, C.c_float), step, _p(f, C.c_double), _p(rho, C.c_double))
        if st:
            raise RuntimeError(f"orc_forces failed: {st}")
        return (f, rho) if want_rho else f

    def step(self, x, xo, noise, step: int, noise_on: bool = True):
        """One step in place on float32 arrays x, xo, noise [ns, dim]; returns the forces used."""
        f = np.zeros((self.ns, self.dim), np.float64)
        st = lib().orc_step(self._h, _p(x, C.c_float), _p(xo, C.c_float), _p(noise, C.c_float), step,
                            1 if noise_on else 0, _p(f, C.c_double))
        if st:
            raise RuntimeError(f"orc_step failed: {st}")
        return f

    def observables(self, x) -> dict:
        x = np.ascontiguousarray(x, np.float32)
        o = self._tild.Obs()
        st = lib().orc_observables(self._h, _p(x, C.c_float), C.byref(o))
        if st:
            raise RuntimeError(f"orc_observables failed: {st}")
        return o.as_dict()

    def sk(self, type_: int) -> np.ndarray:
        out = np.zeros((self.M, 2))
        st = lib().orc_sk(self._h, type_, _p(out, C.c_double))
        if st:
            raise RuntimeError(f"orc_sk failed: {st}")
        return out[:, 0] + 1j * out[:, 1]

    def stencil(self, x):
        x = np.ascontiguousarray(x, np.float32)
        inds = np.zeros((self.ns, self.S), np.int32)
        w = np.zeros((self.ns, self.S))
        st = lib().orc_stencil(self._h, _p(x, C.c_float), _p(inds, C.c_int32), _p(w, C.c_double))
        if st:
            raise RuntimeError(f"orc_stencil failed: {st}")
        return inds, w

    def grid_field(self) -> np.ndarray:
        out = np.zeros((self.sys.ntypes, self.dim, self.M))
        lib().orc_grid_field(self._h, _p(out, C.c_double))
        return out

    def nlist(self, x, rc: float, group_type: int = -1):
        x = np.ascontiguousarray(x, np.float32)
        cm = C.c_int32()
        lib().orc_nlist(self._h, _p(x, C.c_float), rc, group_type, None, None, None, C.byref(cm))
        cmax = cm.value
        cell = np.zeros(self.ns, np.int32)
        cnt = np.zeros(self.ns, np.int32)
        nb = np.zeros((self.ns, max(cmax, 1)), np.int32)
        st = lib().orc_nlist(self._h, _p(x, C.c_float), rc, group_type, _p(cell, C.c_int32), _p(cnt, C.c_int32),
                             _p(nb, C.c_int32), C.byref(cm))
        return st, cell, cnt, nb, cmax
