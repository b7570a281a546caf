"""ctypes binding of libtild (include/tild.h) — the Python face of the B200 TILD hot path.

The reference program exposes its per-step path only as argument-less functions over globals
(forces.cu:42, integrator.cu:24, calc_properties.cu:20).  This module mirrors those calls as
methods of :class:`Context` over the C ABI, so tests and benchmarks drive exactly the entry
points a C/C++ caller would bind.  There is no fallback: if ``lib/libtild.so`` is missing or
fails to load, importing the library raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libtild.so")

MAX_TYPES = 16
MAX_STYLES = 32
MAX_BOND_TYPES = 32
MAX_INTEGRATORS = 8
MAX_BONDS = 3
MAX_COMPUTES = 8

OK, ERR_CUDA, ERR_NAN, ERR_OOM, ERR_TIMEOUT, ERR_BAD_INPUT, ERR_UNSUPPORTED, ERR_STATE = range(8)

STYLE_GAUSSIAN, STYLE_ERF, STYLE_GAUSSIAN_ERF, STYLE_FIELDPHASE = range(4)
INTEGRATOR_EM, INTEGRATOR_GJF = 0, 1
RNG_PHILOX, RNG_XORWOW = 0, 1
TABLES_FP64, TABLES_REF_FP32 = 0, 1


class PairStyle(C.Structure):
    _fields_ = [("style", C.c_int32), ("type1", C.c_int32), ("type2", C.c_int32), ("ramp", C.c_int32),
                ("prefactor", C.c_float), ("final_prefactor", C.c_float), ("sigma", C.c_float), ("rp", C.c_float),
                ("phase", C.c_int32), ("dir", C.c_int32), ("n_periods", C.c_int32), ("reserved", C.c_int32)]


class Integrator(C.Structure):
    _fields_ = [("kind", C.c_int32), ("group_type", C.c_int32)]


class Config(C.Structure):
    _fields_ = [("dim", C.c_int32), ("nx", C.c_int32 * 3), ("box", C.c_float * 3), ("ns", C.c_int32),
                ("ntypes", C.c_int32), ("pmeorder", C.c_int32), ("delt", C.c_float), ("noise_mag", C.c_float),
                ("seed", C.c_uint64), ("rng", C.c_int32), ("max_steps", C.c_int32), ("n_styles", C.c_int32),
                ("styles", PairStyle * MAX_STYLES), ("do_charges", C.c_int32), ("bjerrum", C.c_float),
                ("smearing", C.c_float), ("n_bond_types", C.c_int32), ("bond_k", C.c_float * MAX_BOND_TYPES),
                ("bond_req", C.c_float * MAX_BOND_TYPES), ("mass", C.c_float * MAX_TYPES),
                ("diff", C.c_float * MAX_TYPES), ("n_integrators", C.c_int32),
                ("integrators", Integrator * MAX_INTEGRATORS), ("table_mode", C.c_int32),
                ("sort_interval", C.c_int32), ("flags", C.c_int32), ("reserved", C.c_int32 * 7)]


SPREAD_TILED, SPREAD_DIRECT = 0, 1
GATHER_DIRECT, GATHER_BOX = 0, 1
FIELD_LINEAR, FIELD_BRICK = 0, 1


class Tune(C.Structure):
    _fields_ = [("spread_mode", C.c_int32), ("spread_cap", C.c_int32), ("sort_interval", C.c_int32),
                ("fft_streams", C.c_int32), ("gather_mode", C.c_int32), ("gather_cap", C.c_int32),
                ("sort_brick", C.c_int32), ("field_layout", C.c_int32), ("fft_pipeline", C.c_int32),
                ("spread_ahead", C.c_int32), ("ms_per_step", C.c_double)]

    def as_dict(self) -> dict:
        return {"spread_mode": "tiled" if self.spread_mode == SPREAD_TILED else "direct",
                "spread_cap_words": self.spread_cap, "sort_interval": self.sort_interval,
                "fft_streams": self.fft_streams, "gather_mode": ("direct", "box")[self.gather_mode],
                "gather_cap_nodes": self.gather_cap, "sort_brick": hex(self.sort_brick),
                "field_layout": ("linear", "brick")[self.field_layout], "fft_pipeline": int(self.fft_pipeline),
                "spread_ahead": int(self.spread_ahead),
                "ms_per_step": self.ms_per_step}


class Obs(C.Structure):
    _fields_ = [("upe", C.c_double), ("ubond", C.c_double), ("uelec", C.c_double), ("ptens", C.c_double * 6),
                ("bond_vir", C.c_double * 6), ("style_energy", C.c_double * MAX_STYLES),
                ("style_virial", (C.c_double * 6) * MAX_STYLES), ("step", C.c_int64), ("n_styles", C.c_int32),
                ("n_p_comps", C.c_int32)]

    def as_dict(self) -> dict:
        n, npc = self.n_styles, self.n_p_comps
        return {"upe": self.upe, "ubond": self.ubond, "uelec": self.uelec,
                "ptens": np.array(self.ptens[:npc]), "bond_vir": np.array(self.bond_vir[:npc]),
                "style_energy": np.array(self.style_energy[:n]),
                "style_virial": np.array([list(self.style_virial[i])[:npc] for i in range(n)]).reshape(n, npc),
                "step": self.step}


_lib = None


def lib() -> C.CDLL:
    """Load libtild.so once; raises if the CUDA library is absent (no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libtild.so not built: {LIB_PATH} missing (run __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64p = C.c_void_p, C.c_int32, C.POINTER(C.c_int64)
    fp = C.POINTER(C.c_float)
    ip = C.POINTER(C.c_int32)
    dp = C.POINTER(C.c_double)
    sig = {
        "tild_abi_version": ([], i32), "tild_status_string": ([i32], C.c_char_p),
        "tild_last_error": ([vp], C.c_char_p),
        "tild_create": ([C.POINTER(Config), i32, C.POINTER(vp)], i32), "tild_destroy": ([vp], i32),
        "tild_set_topology": ([vp, ip, fp, ip, ip, ip], i32), "tild_set_state": ([vp, fp, fp, fp], i32),
        "tild_get_state": ([vp, fp, fp, fp], i32), "tild_forces": ([vp, fp], i32), "tild_step": ([vp, i32], i32),
        "tild_get_step": ([vp, i64p], i32), "tild_set_step": ([vp, C.c_int64], i32),
        "tild_observables": ([vp, C.POINTER(Obs)], i32), "tild_get_density": ([vp, fp], i32),
        "tild_get_stencil": ([vp, ip, fp], i32), "tild_sk_accumulate": ([vp, i32, i32], i32),
        "tild_sk_get": ([vp, i32, dp, ip], i32),
        "tild_nlist_build": ([vp, C.c_float, i32, ip, ip, ip, ip], i32),
        "tild_profile_steps": ([vp, i32, dp, i32, ip, C.c_char_p, i32], i32),
        "tild_time_steps": ([vp, i32, dp], i32), "tild_kernel_launches": ([vp, i64p], i32),
        "tild_sync": ([vp], i32),
        "tild_batch_create": ([C.POINTER(Config), i32, i32, C.POINTER(vp)], i32), "tild_batch_destroy": ([vp], i32),
        "tild_batch_last_error": ([vp], C.c_char_p),
        "tild_batch_set_topology": ([vp, i32, ip, fp, ip, ip, ip], i32),
        "tild_batch_set_state": ([vp, i32, fp, fp, fp], i32), "tild_batch_get_state": ([vp, i32, fp, fp, fp], i32),
        "tild_batch_set_active": ([vp, i32, i32], i32), "tild_batch_set_step": ([vp, i32, C.c_int64], i32),
        "tild_batch_get_step": ([vp, i32, i64p], i32), "tild_batch_step": ([vp, i32], i32),
        "tild_batch_forces": ([vp, i32, fp], i32), "tild_batch_observables": ([vp, i32, C.POINTER(Obs)], i32),
        "tild_batch_get_density": ([vp, i32, fp], i32), "tild_batch_time_steps": ([vp, i32, dp], i32),
        "tild_batch_sync": ([vp], i32),
        "tild_batch_sk_accumulate": ([vp, i32, i32, i32], i32), "tild_batch_sk_get": ([vp, i32, i32, dp, ip], i32),
        "tild_batch_create_slots": ([C.POINTER(Config), ip, i32, i32, C.POINTER(vp)], i32),
        "tild_batch_capacity": ([vp, i32, ip], i32), "tild_batch_load": ([vp, i32, C.POINTER(Config)], i32),
        "tild_batch_set_stop": ([vp, i32, C.c_int64], i32), "tild_batch_get_active": ([vp, i32, ip], i32),
        "tild_snapshot_async": ([vp, fp, fp, i64p], i32), "tild_snapshot_wait": ([vp, C.c_int64], i32),
        "tild_batch_snapshot_async": ([vp, i32, fp, fp, i64p], i32), "tild_batch_snapshot_wait": ([vp, C.c_int64], i32),
        "tild_host_alloc": ([C.c_size_t], vp), "tild_host_free": ([vp], None),
        "tild_autotune": ([vp, i32, C.POINTER(Tune)], i32), "tild_get_tune": ([vp, C.POINTER(Tune)], i32),
        "tild_set_tune": ([vp, C.POINTER(Tune)], i32), "tild_batch_autotune": ([vp, i32, C.POINTER(Tune)], i32),
        "tild_batch_get_tune": ([vp, C.POINTER(Tune)], i32), "tild_batch_set_tune": ([vp, C.POINTER(Tune)], i32),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


class HostArray:
    """A page-locked float32 host array (tild_host_alloc), freed with the object."""

    def __init__(self, shape):
        n = int(np.prod(shape))
        self._p = lib().tild_host_alloc(max(n, 1) * 4)
        if not self._p:
            raise MemoryError("page-locked host memory unavailable")
        self.array = np.ctypeslib.as_array(C.cast(self._p, C.POINTER(C.c_float)), shape=(n,)).reshape(shape)

    def __del__(self):
        if getattr(self, "_p", None):
            lib().tild_host_free(self._p)
            self._p = None


class TildError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{msg} [status {status}]")
        self.status = status


# ------------------------------------------------------------------------------------------
# System description shared by the CUDA library, the oracle and the file writers
# ------------------------------------------------------------------------------------------
@dataclass
class Style:
    kind: int
    type1: int
    type2: int
    prefactor: float
    sigma: float = 1.0
    rp: float = 0.0
    ramp: bool = False
    final_prefactor: Optional[float] = None
    phase: int = 0
    dir: int = 0
    n_periods: int = 1


@dataclass
class System:
    """One TILD system: the quantities read_input.cu + read_config() would produce."""
    dim: int
    nx: Sequence[int]
    box: Sequence[float]
    types: np.ndarray                      # int32 [ns], 0-based
    x: np.ndarray                          # float32 [ns, dim]
    n_bonds: np.ndarray                    # int32 [ns]
    bonded_to: np.ndarray                  # int32 [ns, 3]
    bond_type: np.ndarray                  # int32 [ns, 3]
    ntypes: int
    styles: List[Style] = field(default_factory=list)
    bond_k: Sequence[float] = (1.5,)
    bond_req: Sequence[float] = (0.0,)
    mass: Optional[Sequence[float]] = None
    diff: Optional[Sequence[float]] = None
    integrators: List[tuple] = field(default_factory=lambda: [(INTEGRATOR_GJF, -1)])
    pmeorder: int = 1
    delt: float = 0.005
    noise_mag: Optional[float] = None
    seed: int = 12345
    charges: Optional[np.ndarray] = None   # float32 [ns]
    bjerrum: float = 1.0
    smearing: float = 1.0
    max_steps: int = 100000
    molecule: Optional[np.ndarray] = None  # int32 [ns], 0-based molecule ids
    rng: int = RNG_PHILOX
    table_mode: int = TABLES_FP64

    @property
    def ns(self) -> int:
        return int(self.types.shape[0])

    def config(self) -> Config:
        c = Config()
        c.dim = self.dim
        for d in range(3):
            c.nx[d] = int(self.nx[d]) if d < self.dim else 1
            c.box[d] = float(self.box[d]) if d < self.dim else 1.0
        c.ns = self.ns
        c.ntypes = self.ntypes
        c.pmeorder = self.pmeorder
        c.delt = self.delt
        nm = self.noise_mag
        c.noise_mag = float(np.sqrt(np.float32(2.0) * np.float32(self.delt), dtype=np.float32)) if nm is None else nm
        c.seed = self.seed
        c.rng = self.rng
        c.max_steps = self.max_steps
        c.n_styles = len(self.styles)
        for i, s in enumerate(self.styles):
            p = c.styles[i]
            p.style, p.type1, p.type2 = s.kind, s.type1, s.type2
            p.ramp = 1 if s.ramp else 0
            p.prefactor = s.prefactor
            p.final_prefactor = s.prefactor if s.final_prefactor is None else s.final_prefactor
            p.sigma, p.rp = s.sigma, s.rp
            p.phase, p.dir, p.n_periods = s.phase, s.dir, s.n_periods
        c.do_charges = 1 if self.charges is not None else 0
        c.bjerrum, c.smearing = self.bjerrum, self.smearing
        c.n_bond_types = len(self.bond_k)
        for b, (k, r) in enumerate(zip(self.bond_k, self.bond_req)):
            c.bond_k[b], c.bond_req[b] = k, r
        mass = self.mass if self.mass is not None else [1.0] * self.ntypes
        diff = self.diff if self.diff is not None else [1.0] * self.ntypes
        for t in range(self.ntypes):
            c.mass[t], c.diff[t] = mass[t], diff[t]
        c.n_integrators = len(self.integrators)
        for k, (kind, grp) in enumerate(self.integrators):
            c.integrators[k].kind, c.integrators[k].group_type = kind, grp
        c.table_mode = self.table_mode
        return c


def _ptr(a: Optional[np.ndarray], ctype):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


class Context:
    """One device-resident TILD system (a tild_ctx)."""

    def __init__(self, system: System, device: int = 0):
        L = lib()
        self.sys = system
        self._cfg = system.config()
        h = C.c_void_p()
        st = L.tild_create(C.byref(self._cfg), device, C.byref(h))
        if st != OK:
            raise TildError(st, f"tild_create failed: {L.tild_status_string(st).decode()}")
        self._h = h
        self.ns, self.dim = system.ns, system.dim
        self.M = int(np.prod([system.nx[d] for d in range(system.dim)]))
        s = system
        self._types = np.ascontiguousarray(s.types, dtype=np.int32)
        self._q = None if s.charges is None else np.ascontiguousarray(s.charges, dtype=np.float32)
        self._nb = np.ascontiguousarray(s.n_bonds, dtype=np.int32)
        self._bt = np.ascontiguousarray(s.bonded_to, dtype=np.int32).reshape(-1)
        self._by = np.ascontiguousarray(s.bond_type, dtype=np.int32).reshape(-1)
        self._check(L.tild_set_topology(self._h, _ptr(self._types, C.c_int32), _ptr(self._q, C.c_float),
                                        _ptr(self._nb, C.c_int32), _ptr(self._bt, C.c_int32),
                                        _ptr(self._by, C.c_int32)), "tild_set_topology")
        self.set_state(s.x)

    def _check(self, st: int, what: str):
        if st != OK:
            L = lib()
            raise TildError(st, f"{what}: {L.tild_status_string(st).decode()}: {L.tild_last_error(self._h).decode()}")

    def close(self):
        if getattr(self, "_h", None):
            lib().tild_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- state ----------------------------------------------------------------------------
    def set_state(self, x, xo=None, noise=None):
        x = np.ascontiguousarray(x, dtype=np.float32)
        xo = None if xo is None else np.ascontiguousarray(xo, dtype=np.float32)
        noise = None if noise is None else np.ascontiguousarray(noise, dtype=np.float32)
        self._check(lib().tild_set_state(self._h, _ptr(x, C.c_float), _ptr(xo, C.c_float), _ptr(noise, C.c_float)),
                    "tild_set_state")

    def get_state(self):
        x = np.empty((self.ns, self.dim), np.float32)
        xo = np.empty_like(x)
        nz = np.empty_like(x)
        self._check(lib().tild_get_state(self._h, _ptr(x, C.c_float), _ptr(xo, C.c_float), _ptr(nz, C.c_float)),
                    "tild_get_state")
        return x, xo, nz

    # -- per step ------------------------------------------------------------------------
    def forces(self) -> np.ndarray:
        f = np.empty((self.ns, self.dim), np.float32)
        self._check(lib().tild_forces(self._h, _ptr(f, C.c_float)), "tild_forces")
        return f

    def step(self, n: int = 1):
        self._check(lib().tild_step(self._h, int(n)), "tild_step")

    @property
    def step_count(self) -> int:
        v = C.c_int64()
        self._check(lib().tild_get_step(self._h, C.byref(v)), "tild_get_step")
        return v.value

    def set_step(self, s: int):
        self._check(lib().tild_set_step(self._h, int(s)), "tild_set_step")

    def observables(self) -> dict:
        o = Obs()
        self._check(lib().tild_observables(self._h, C.byref(o)), "tild_observables")
        return o.as_dict()

    def density(self) -> np.ndarray:
        nch = self.sys.ntypes + (1 if self.sys.charges is not None else 0)
        r = np.empty((nch, self.M), np.float32)
        self._check(lib().tild_get_density(self._h, _ptr(r, C.c_float)), "tild_get_density")
        return r

    def stencil(self):
        S = (self.sys.pmeorder + 1) ** self.dim
        inds = np.empty((self.ns, S), np.int32)
        w = np.empty((self.ns, S), np.float32)
        self._check(lib().tild_get_stencil(self._h, _ptr(inds, C.c_int32), _ptr(w, C.c_float)), "tild_get_stencil")
        return inds, w

    def sk_accumulate(self, slot: int, type_: int):
        self._check(lib().tild_sk_accumulate(self._h, slot, type_), "tild_sk_accumulate")

    def sk_get(self, slot: int):
        out = np.empty((self.M, 2), np.float64)
        n = C.c_int32()
        self._check(lib().tild_sk_get(self._h, slot, _ptr(out, C.c_double), C.byref(n)), "tild_sk_get")
        return out[:, 0] + 1j * out[:, 1], n.value

    def nlist(self, rc: float, group_type: int = -1):
        cm = C.c_int32()
        self._check(lib().tild_nlist_build(self._h, rc, group_type, None, None, None, C.byref(cm)), "nlist geometry")
        cmax = cm.value
        cell = np.empty(self.ns, np.int32)
        cnt = np.empty(self.ns, np.int32)
        nb = np.empty((self.ns, max(cmax, 1)), np.int32)
        self._check(lib().tild_nlist_build(self._h, rc, group_type, _ptr(cell, C.c_int32), _ptr(cnt, C.c_int32),
                                           _ptr(nb, C.c_int32), C.byref(cm)), "tild_nlist_build")
        return cell, cnt, nb, cmax

    # -- measurement ---------------------------------------------------------------------
    def autotune(self, trial_steps: int = 64) -> dict:
        """Times schedule candidates (tild_autotune) and keeps the fastest; the state is restored."""
        t = Tune()
        self._check(lib().tild_autotune(self._h, int(trial_steps), C.byref(t)), "tild_autotune")
        return t.as_dict()

    def get_tune(self) -> Tune:
        t = Tune()
        self._check(lib().tild_get_tune(self._h, C.byref(t)), "tild_get_tune")
        return t

    def snapshot_async(self, x: Optional[np.ndarray], rho: Optional[np.ndarray]) -> int:
        """Starts copying the current positions [ns][dim] and/or densities [(T+C)][M] into the given
        float32 arrays (page-locked ones from host_array overlap with stepping); returns a ticket.
        The arrays must stay alive and untouched until snapshot_wait(ticket) returns."""
        for a in (x, rho):
            if a is not None and (a.dtype != np.float32 or not a.flags["C_CONTIGUOUS"]):
                raise ValueError("snapshot arrays must be C-contiguous float32")
        t = C.c_int64()
        self._check(lib().tild_snapshot_async(self._h, _ptr(x, C.c_float), _ptr(rho, C.c_float), C.byref(t)),
                    "tild_snapshot_async")
        return t.value

    def snapshot_wait(self, ticket: int):
        self._check(lib().tild_snapshot_wait(self._h, int(ticket)), "tild_snapshot_wait")

    def set_tune(self, t: Tune):
        self._check(lib().tild_set_tune(self._h, C.byref(t)), "tild_set_tune")

    def time_steps(self, n: int) -> float:
        ms = C.c_double()
        self._check(lib().tild_time_steps(self._h, int(n), C.byref(ms)), "tild_time_steps")
        return ms.value

    def profile_steps(self, n: int) -> dict:
        out = (C.c_double * 16)()
        ns = C.c_int32()
        names = C.create_string_buffer(512)
        self._check(lib().tild_profile_steps(self._h, int(n), out, 16, C.byref(ns), names, 512), "tild_profile_steps")
        keys = names.value.decode().split(",")
        return {k: out[i] for i, k in enumerate(keys)}

    def kernel_launches(self) -> int:
        v = C.c_int64()
        self._check(lib().tild_kernel_launches(self._h, C.byref(v)), "tild_kernel_launches")
        return v.value

    def sync(self):
        self._check(lib().tild_sync(self._h), "tild_sync")


class Batch:
    """Many independent systems advanced together (a tild_batch): one launch per stage for all
    systems, one batched cuFFT plan per grid shape.  Systems share dim, pmeorder and rng."""

    def __init__(self, systems: Sequence[System], device: int = 0, capacity: Optional[Sequence[int]] = None):
        """capacity: beads reserved per system (a slot batch, tild_batch_create_slots), so that
        load() can later put another system of the same grid shape into that slot."""
        L = lib()
        self.systems = list(systems)
        n = len(self.systems)
        self._cfgs = (Config * n)(*[s.config() for s in self.systems])
        h = C.c_void_p()
        if capacity is None:
            st = L.tild_batch_create(self._cfgs, n, device, C.byref(h))
        else:
            cap = np.ascontiguousarray(capacity, dtype=np.int32)
            if cap.shape != (n,):
                raise ValueError("one capacity per system")
            st = L.tild_batch_create_slots(self._cfgs, _ptr(cap, C.c_int32), n, device, C.byref(h))
        if st != OK:
            raise TildError(st, f"tild_batch_create failed: {L.tild_status_string(st).decode()}")
        self._h = h
        self._keep = []
        for i, s in enumerate(self.systems):
            self.set_topology(i, s)
            self.set_state(i, s.x)

    def _check(self, st: int, what: str):
        if st != OK:
            L = lib()
            raise TildError(st, f"{what}: {L.tild_status_string(st).decode()}: {L.tild_batch_last_error(self._h).decode()}")

    def close(self):
        if getattr(self, "_h", None):
            lib().tild_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_topology(self, i: int, s: System):
        types = np.ascontiguousarray(s.types, dtype=np.int32)
        q = None if s.charges is None else np.ascontiguousarray(s.charges, dtype=np.float32)
        nb = np.ascontiguousarray(s.n_bonds, dtype=np.int32)
        bt = np.ascontiguousarray(s.bonded_to, dtype=np.int32).reshape(-1)
        by = np.ascontiguousarray(s.bond_type, dtype=np.int32).reshape(-1)
        self._check(lib().tild_batch_set_topology(self._h, i, _ptr(types, C.c_int32), _ptr(q, C.c_float),
                                                  _ptr(nb, C.c_int32), _ptr(bt, C.c_int32), _ptr(by, C.c_int32)),
                    "tild_batch_set_topology")

    def set_state(self, i: int, x, xo=None, noise=None):
        x = np.ascontiguousarray(x, dtype=np.float32)
        xo = None if xo is None else np.ascontiguousarray(xo, dtype=np.float32)
        noise = None if noise is None else np.ascontiguousarray(noise, dtype=np.float32)
        self._check(lib().tild_batch_set_state(self._h, i, _ptr(x, C.c_float), _ptr(xo, C.c_float),
                                               _ptr(noise, C.c_float)), "tild_batch_set_state")

    def get_state(self, i: int):
        s = self.systems[i]
        x = np.empty((s.ns, s.dim), np.float32)
        xo = np.empty_like(x)
        nz = np.empty_like(x)
        self._check(lib().tild_batch_get_state(self._h, i, _ptr(x, C.c_float), _ptr(xo, C.c_float),
                                               _ptr(nz, C.c_float)), "tild_batch_get_state")
        return x, xo, nz

    def set_active(self, i: int, active: bool):
        self._check(lib().tild_batch_set_active(self._h, i, 1 if active else 0), "tild_batch_set_active")

    def set_step(self, i: int, step: int):
        self._check(lib().tild_batch_set_step(self._h, i, int(step)), "tild_batch_set_step")

    def step_count(self, i: int) -> int:
        v = C.c_int64()
        self._check(lib().tild_batch_get_step(self._h, i, C.byref(v)), "tild_batch_get_step")
        return v.value

    def step(self, n: int = 1):
        self._check(lib().tild_batch_step(self._h, int(n)), "tild_batch_step")

    def forces(self, i: int) -> np.ndarray:
        s = self.systems[i]
        f = np.empty((s.ns, s.dim), np.float32)
        self._check(lib().tild_batch_forces(self._h, i, _ptr(f, C.c_float)), "tild_batch_forces")
        return f

    def evaluate(self):
        """One force evaluation of every system at its current positions, without a step: the
        densities, spectra and observables afterwards describe the current state (systems that
        stopped or were set inactive included, their positions being held)."""
        self._check(lib().tild_batch_forces(self._h, 0, None), "tild_batch_forces")

    def observables(self, i: int) -> dict:
        o = Obs()
        self._check(lib().tild_batch_observables(self._h, i, C.byref(o)), "tild_batch_observables")
        return o.as_dict()

    def density(self, i: int) -> np.ndarray:
        s = self.systems[i]
        nch = s.ntypes + (1 if s.charges is not None else 0)
        r = np.empty((nch, int(np.prod(s.nx[:s.dim]))), np.float32)
        self._check(lib().tild_batch_get_density(self._h, i, _ptr(r, C.c_float)), "tild_batch_get_density")
        return r

    def autotune(self, trial_steps: int = 64) -> dict:
        """Times schedule candidates (tild_batch_autotune) and keeps the fastest; states are restored."""
        t = Tune()
        self._check(lib().tild_batch_autotune(self._h, int(trial_steps), C.byref(t)), "tild_batch_autotune")
        return t.as_dict()

    def get_tune(self) -> Tune:
        t = Tune()
        self._check(lib().tild_batch_get_tune(self._h, C.byref(t)), "tild_batch_get_tune")
        return t

    def set_tune(self, t: Tune):
        self._check(lib().tild_batch_set_tune(self._h, C.byref(t)), "tild_batch_set_tune")

    def time_steps(self, n: int) -> float:
        ms = C.c_double()
        self._check(lib().tild_batch_time_steps(self._h, int(n), C.byref(ms)), "tild_batch_time_steps")
        return ms.value

    def profile_steps(self, n: int) -> dict:
        """Per-stage CUDA-event times over n steps (a batch is a context of several systems)."""
        out = (C.c_double * 16)()
        cnt = C.c_int32()
        names = C.create_string_buffer(512)
        self._check(lib().tild_profile_steps(self._h, int(n), out, 16, C.byref(cnt), names, 512), "tild_profile_steps")
        return {k: out[i] for i, k in enumerate(names.value.decode().split(","))}

    def sync(self):
        self._check(lib().tild_batch_sync(self._h), "tild_batch_sync")

    # ---- avg_sk per system ----
    def sk_accumulate(self, i: int, slot: int, type_: int):
        self._check(lib().tild_batch_sk_accumulate(self._h, i, slot, type_), "tild_batch_sk_accumulate")

    def sk_get(self, i: int, slot: int):
        s = self.systems[i]
        out = np.empty(2 * int(np.prod(s.nx[:s.dim])), np.float64)
        n = C.c_int32()
        self._check(lib().tild_batch_sk_get(self._h, i, slot, _ptr(out, C.c_double), C.byref(n)), "tild_batch_sk_get")
        return out.view(np.complex128), n.value

    # ---- slots (continuous batching) ----
    def capacity(self, i: int) -> int:
        v = C.c_int32()
        self._check(lib().tild_batch_capacity(self._h, i, C.byref(v)), "tild_batch_capacity")
        return v.value

    def load(self, i: int, s: System, activate: bool = True):
        """Put system s into slot i (same grid shape and channel layout, s.ns <= capacity):
        tables rebuilt, topology and state uploaded, step counter 0."""
        cfg = s.config()
        self._check(lib().tild_batch_load(self._h, i, C.byref(cfg)), "tild_batch_load")
        self._cfgs[i] = cfg
        self.systems[i] = s
        self.set_topology(i, s)
        self.set_state(i, s.x)
        if activate:
            self.set_active(i, True)

    def set_stop(self, i: int, stop_at: int):
        self._check(lib().tild_batch_set_stop(self._h, i, int(stop_at)), "tild_batch_set_stop")

    def active(self, i: int) -> bool:
        v = C.c_int32()
        self._check(lib().tild_batch_get_active(self._h, i, C.byref(v)), "tild_batch_get_active")
        return bool(v.value)
