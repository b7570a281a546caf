"""Seeded synthetic TILD systems and the reference file formats.

The reference ships no configuration generator (its docs point to external utilities), so
systems here are built from a seeded random walk: bead 0 of a chain uniform in the box, each
next bead displaced by N(0, b^2/dim) per component, positions wrapped into [0, L).  Types are
assigned by block (diblocks) or by chain (blends).  Bonds are linear, type 0.

Writers produce the fixed-layout "LAMMPS-like" data file that read_config / read_charge_config
parse (config_utils.cu:5-364) and an input script in read_input's keyword grammar
(read_input.cu:23-523), so the reference build and this one read identical bytes.
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence

import numpy as np

from tild import (INTEGRATOR_EM, INTEGRATOR_GJF, STYLE_ERF, STYLE_FIELDPHASE, STYLE_GAUSSIAN,
                  STYLE_GAUSSIAN_ERF, Style, System)

SEED_BASE = 20261203


def topology_from_bonds(ns: int, bonds: np.ndarray):
    """n_bonds / bonded_to / bond_type exactly as read_config builds them (config_utils.cu:96-125):
    each bond line (type, i1, i2) is stored from both ends in file order, i1 < i2 after a swap."""
    n_bonds = np.zeros(ns, np.int32)
    bonded_to = np.zeros((ns, 3), np.int32)
    bond_type = np.zeros((ns, 3), np.int32)
    if len(bonds) == 0:
        return n_bonds, bonded_to, bond_type
    b = np.asarray(bonds, dtype=np.int64)
    bt, i1, i2 = b[:, 0], np.minimum(b[:, 1], b[:, 2]), np.maximum(b[:, 1], b[:, 2])
    # vectorised version of the sequential fill for the common case where every bead appears
    # in at most 3 bonds; ordering follows the file order per bead
    ends = np.concatenate([np.stack([i1, i2, bt, np.arange(len(b)) * 2], 1),
                           np.stack([i2, i1, bt, np.arange(len(b)) * 2 + 1], 1)])
    ends = ends[np.lexsort((ends[:, 3], ends[:, 0]))]
    owner = ends[:, 0]
    first = np.searchsorted(owner, owner, side="left")
    slot = np.arange(len(owner)) - first
    if slot.max() >= 3:
        raise ValueError("more than MAX_BONDS (3) bonds on a bead")
    bonded_to[owner, slot] = ends[:, 1]
    bond_type[owner, slot] = ends[:, 2]
    np.add.at(n_bonds, owner, 1)
    return n_bonds, bonded_to, bond_type


def random_walk_chains(rng: np.random.Generator, n_chains: int, N: int, box: Sequence[float], dim: int,
                       b: float = 1.0) -> np.ndarray:
    L = np.asarray(box[:dim], dtype=np.float64)
    start = rng.random((n_chains, 1, dim)) * L
    steps = rng.normal(0.0, b / math.sqrt(dim), size=(n_chains, N - 1, dim))
    x = np.concatenate([start, start + np.cumsum(steps, axis=1)], axis=1).reshape(-1, dim)
    x = np.mod(x, L)
    x = x.astype(np.float32)
    # float rounding can land exactly on L; the reference keeps x in [0, L]
    Lf = L.astype(np.float32)
    x = np.where(x >= Lf, x - Lf, x).astype(np.float32)
    return x


def linear_bonds(n_chains: int, N: int, offset: int = 0) -> np.ndarray:
    base = (offset + np.arange(n_chains)[:, None] * N + np.arange(N - 1)[None, :]).reshape(-1)
    return np.stack([np.zeros_like(base), base, base + 1], 1)


def helfand(kappa: float, chi: float, rho0: float):
    """Gaussian prefactors from Helfand compressibility and Flory chi: A_II = kappa/(2 rho0),
    A_IJ = (kappa + chi)/rho0."""
    return kappa / (2.0 * rho0), (kappa + chi) / rho0


def diblock_melt(n_chains=2000, N=20, fA=0.5, box=(20.0, 20.0, 20.0), nx=(40, 40, 40), a=0.5, kappa=50.0,
                 chiN=20.0, pmeorder=1, seed=SEED_BASE + 0, dim=3, integrator=INTEGRATOR_GJF, delt=0.005,
                 max_steps=1000) -> System:
    """AB diblock melt (default: 40,000 beads in a 20^3 box on a 40^3 grid, CIC spreading)."""
    rng = np.random.default_rng(seed)
    x = random_walk_chains(rng, n_chains, N, box, dim)
    ns = n_chains * N
    nA = int(round(fA * N))
    types = np.tile(np.array([0] * nA + [1] * (N - nA), np.int32), n_chains)
    V = float(np.prod(box[:dim]))
    rho0 = ns / V
    Aii, Aij = helfand(kappa, chiN / N, rho0)
    sigma = math.sqrt(2.0) * a
    styles = [Style(STYLE_GAUSSIAN, 0, 0, Aii, sigma), Style(STYLE_GAUSSIAN, 1, 1, Aii, sigma),
              Style(STYLE_GAUSSIAN, 0, 1, Aij, sigma)]
    nb, bt, by = topology_from_bonds(ns, linear_bonds(n_chains, N))
    return System(dim=dim, nx=nx, box=box, types=types, x=x, n_bonds=nb, bonded_to=bt, bond_type=by, ntypes=2,
                  styles=styles, bond_k=(1.5,), bond_req=(0.0,), integrators=[(integrator, -1)], pmeorder=pmeorder,
                  delt=delt, seed=seed, max_steps=max_steps,
                  molecule=np.repeat(np.arange(n_chains, dtype=np.int32), N))


def homopolymer_blend(n_chains=130000, N=20, box=(64.0, 64.0, 64.0), nx=(128, 128, 128), rp=0.5, sigma=0.5,
                      kappa=50.0, chi=0.2, pmeorder=3, seed=SEED_BASE + 1, dim=3, delt=0.005,
                      max_steps=2000) -> System:
    """A/B homopolymer blend 50:50 with gaussian_erf styles (default: 2.6M beads, 64^3 box, 128^3
    grid, 64-point stencil).  A is kappa/(2 rho0), (kappa+chi)/rho0 as given to the script."""
    rng = np.random.default_rng(seed)
    x = random_walk_chains(rng, n_chains, N, box, dim)
    ns = n_chains * N
    types = np.repeat((np.arange(n_chains) % 2).astype(np.int32), N)
    rho0 = ns / float(np.prod(box[:dim]))
    Aii, Aij = helfand(kappa, chi, rho0)
    styles = [Style(STYLE_GAUSSIAN_ERF, 0, 0, Aii, sigma, rp), Style(STYLE_GAUSSIAN_ERF, 1, 1, Aii, sigma, rp),
              Style(STYLE_GAUSSIAN_ERF, 0, 1, Aij, sigma, rp)]
    nb, bt, by = topology_from_bonds(ns, linear_bonds(n_chains, N))
    return System(dim=dim, nx=nx, box=box, types=types, x=x, n_bonds=nb, bonded_to=bt, bond_type=by, ntypes=2,
                  styles=styles, bond_k=(1.5,), bond_req=(0.0,), integrators=[(INTEGRATOR_GJF, -1)],
                  pmeorder=pmeorder, delt=delt, seed=seed, max_steps=max_steps,
                  molecule=np.repeat(np.arange(n_chains, dtype=np.int32), N))


def coacervate(n_poly=4000, N=25, n_solvent=20000, box=(48.0, 48.0, 48.0), nx=(96, 96, 96), kappa=30.0, a=0.5,
               bjerrum=1.0, smearing=0.5, pmeorder=1, seed=SEED_BASE + 2, dim=3, delt=0.002,
               max_steps=2000) -> System:
    """Polycations + polyanions (charge +-1 per bead) + neutral solvent, smeared charges plus
    Gaussian excluded volume (default: 220,000 beads, 48^3 box, 96^3 grid, EM)."""
    rng = np.random.default_rng(seed)
    xc = random_walk_chains(rng, n_poly, N, box, dim)
    xa = random_walk_chains(rng, n_poly, N, box, dim)
    xs = (rng.random((n_solvent, dim)) * np.asarray(box[:dim])).astype(np.float32)
    x = np.concatenate([xc, xa, xs]).astype(np.float32)
    ns = x.shape[0]
    types = np.concatenate([np.zeros(n_poly * N, np.int32), np.ones(n_poly * N, np.int32),
                            np.full(n_solvent, 2, np.int32)])
    q = np.concatenate([np.ones(n_poly * N, np.float32), -np.ones(n_poly * N, np.float32),
                        np.zeros(n_solvent, np.float32)])
    rho0 = ns / float(np.prod(box[:dim]))
    Aii, Aij = helfand(kappa, 0.0, rho0)
    sigma = math.sqrt(2.0) * a
    styles = []
    for i in range(3):
        for j in range(i, 3):
            styles.append(Style(STYLE_GAUSSIAN, i, j, Aii if i == j else Aij, sigma))
    bonds = np.concatenate([linear_bonds(n_poly, N, 0), linear_bonds(n_poly, N, n_poly * N)])
    nb, bt, by = topology_from_bonds(ns, bonds)
    mol = np.concatenate([np.repeat(np.arange(2 * n_poly, dtype=np.int32), N),
                          2 * n_poly + np.arange(n_solvent, dtype=np.int32)])
    return System(dim=dim, nx=nx, box=box, types=types, x=x, n_bonds=nb, bonded_to=bt, bond_type=by, ntypes=3,
                  styles=styles, bond_k=(1.5,), bond_req=(0.0,), integrators=[(INTEGRATOR_EM, -1)],
                  pmeorder=pmeorder, delt=delt, seed=seed, charges=q, bjerrum=bjerrum, smearing=smearing,
                  max_steps=max_steps, molecule=mol)


def ensemble_member(index: int, base_seed: int = SEED_BASE + 3, dx: float = 0.5, rho0: float = 5.0,
                    kappa: float = 50.0) -> System:
    """One system of the batched diblock ensemble: L ~ U(12, 24) snapped to the grid (grid =
    round(L/dx), 24^3..48^3), N ~ U{10..40}, f_A ~ U(0.3, 0.7), chi N ~ U(10, 30), rho0 = 5."""
    rng = np.random.default_rng(base_seed + index)
    g = int(round(rng.uniform(12.0, 24.0) / dx))
    L = g * dx
    N = int(rng.integers(10, 41))
    fA = float(rng.uniform(0.3, 0.7))
    chiN = float(rng.uniform(10.0, 30.0))
    n_chains = max(1, int(round(rho0 * L ** 3 / N)))
    return diblock_melt(n_chains=n_chains, N=N, fA=fA, box=(L, L, L), nx=(g, g, g), kappa=kappa, chiN=chiN,
                        seed=base_seed + 100000 + index, max_steps=5000)


def ensemble_grid_edges(dx: float = 0.5):
    """Grid edges the batched-ensemble distribution can draw: round(U(12, 24) / dx)."""
    return list(range(int(round(12.0 / dx)), int(round(24.0 / dx)) + 1))


def ensemble_capacity(g: int, dx: float = 0.5, rho0: float = 5.0, n_max: int = 40) -> int:
    """Largest bead count an ensemble member on a g^3 grid can have: round(rho0 L^3 / N) * N
    <= rho0 L^3 + N / 2 for every chain length N <= n_max."""
    L = g * dx
    return int(math.floor(rho0 * L ** 3 + n_max / 2)) + 1


def ensemble_slot_template(g: int, dx: float = 0.5, rho0: float = 5.0, seed: int = SEED_BASE + 7) -> System:
    """A placeholder diblock system of grid g^3 (same channel layout as every ensemble member)
    that initialises one slot of a serving batch before its first job arrives."""
    L = g * dx
    N = 20
    return diblock_melt(n_chains=max(1, int(round(rho0 * L ** 3 / N))), N=N, fA=0.5, box=(L, L, L), nx=(g, g, g),
                        kappa=50.0, chiN=20.0, seed=seed + g, max_steps=5000)


# ------------------------------------------------------------------------------------------
# reference file formats
# ------------------------------------------------------------------------------------------
def write_data_file(path: str, s: System):
    """Data file in the layout read_config / read_charge_config parse (config_utils.cu:5-364)."""
    ns, dim = s.ns, s.dim
    mol = s.molecule if s.molecule is not None else np.zeros(ns, np.int32)
    # bonds: one line per stored pair (i < j), in bead order
    pairs = []
    for i in range(ns):
        for k in range(int(s.n_bonds[i])):
            j = int(s.bonded_to[i, k])
            if j > i:
                pairs.append((int(s.bond_type[i, k]), i, j))
    box = list(s.box) + [1.0] * (3 - len(s.box))
    with open(path, "w") as f:
        f.write("synthetic TILD configuration\n\n")
        f.write(f"{ns} atoms\n{len(pairs)} bonds\n0 angles\n\n")
        f.write(f"{s.ntypes} atom types\n{len(s.bond_k)} bond types\n0 angle types\n\n")
        for d, (lo, hi) in enumerate((("xlo", "xhi"), ("ylo", "yhi"), ("zlo", "zhi"))):
            f.write(f"0.000000 {box[d]:.6f} {lo} {hi}\n")
        f.write("\nMasses\n\n")
        mass = s.mass if s.mass is not None else [1.0] * s.ntypes
        for t in range(s.ntypes):
            f.write(f"{t + 1} {mass[t]:.6f}\n")
        f.write("\nAtoms\n\n")
        lines = []
        for i in range(ns):
            xs = " ".join(f"{v:.6f}" for v in s.x[i, :dim])
            if s.charges is not None:
                lines.append(f"{i + 1} {int(mol[i]) + 1} {int(s.types[i]) + 1}  {float(s.charges[i]):.3f}  {xs}\n")
            else:
                lines.append(f"{i + 1} {int(mol[i]) + 1} {int(s.types[i]) + 1}  {xs}\n")
        f.write("".join(lines))
        f.write("\nBonds\n\n")
        f.write("".join(f"{n + 1} {bt + 1} {i + 1} {j + 1}\n" for n, (bt, i, j) in enumerate(pairs)))
        f.write("\nAngles\n\n")


def write_input_script(path: str, s: System, data_name: str = "input.data", max_steps: int = 1000,
                       log_freq: int = 100, binary_freq: int = 0, grid_freq: int = 0, traj_freq: int = 0,
                       extra: Optional[List[str]] = None):
    """Input script in read_input's grammar (read_input.cu:23-523)."""
    names = {STYLE_GAUSSIAN: ("n_gaussians", "gaussian"), STYLE_ERF: ("n_erfs", "erf"),
             STYLE_GAUSSIAN_ERF: ("n_gaussian_erfs", "gaussian_erf"), STYLE_FIELDPHASE: ("n_fieldphases", "fieldphase")}
    L = [f"Dim {s.dim}", "", f"max_steps {max_steps}", f"log_freq {log_freq}", f"binary_freq {binary_freq}",
         f"grid_freq {grid_freq}", f"traj_freq {traj_freq}", f"pmeorder {s.pmeorder}", f"rand_seed {s.seed}", ""]
    if s.charges is not None:
        L.append(f"charges {s.bjerrum} {s.smearing}")
    L += [f"delt {s.delt}", f"read_data {data_name}"]
    gnames = {-1: "all"}
    for kind, grp in s.integrators:
        if grp >= 0 and grp not in gnames:
            gnames[grp] = f"type{grp + 1}"
            L.append(f"group {gnames[grp]} type {grp + 1}")
    for kind, grp in s.integrators:
        L.append(f"integrator {gnames[grp]} {'GJF' if kind == INTEGRATOR_GJF else 'EM'}")
    L.append("")
    for d, key in enumerate(("Nx", "Ny", "Nz")[:s.dim]):
        L.append(f"{key} {s.nx[d]}")
    L.append("")
    for b, (k, r) in enumerate(zip(s.bond_k, s.bond_req)):
        L.append(f"bond {b + 1} harmonic {k} {r}")
    if s.diff is not None:
        for t, dval in enumerate(s.diff):
            L.append(f"diffusivity {t + 1} {dval}")
    for kind in (STYLE_GAUSSIAN, STYLE_ERF, STYLE_GAUSSIAN_ERF, STYLE_FIELDPHASE):
        group = [st for st in s.styles if st.kind == kind]
        if not group:
            continue
        L.append(f"{names[kind][0]} {len(group)}")
        for st in group:
            ramp = f" ramp {st.final_prefactor}" if st.ramp else ""
            if kind == STYLE_GAUSSIAN:
                L.append(f"gaussian {st.type1 + 1} {st.type2 + 1} {st.prefactor!r} {st.sigma!r}{ramp}")
            elif kind in (STYLE_ERF, STYLE_GAUSSIAN_ERF):
                L.append(f"{names[kind][1]} {st.type1 + 1} {st.type2 + 1} {st.prefactor!r} {st.rp!r} {st.sigma!r}{ramp}")
            else:
                L.append(f"fieldphase {st.type1 + 1} {st.type2 + 1} {st.prefactor!r} {st.phase} {st.dir} {st.n_periods}{ramp}")
    if extra:
        L += extra
    with open(path, "w") as f:
        f.write("\n".join(L) + "\n")


def read_data_file(path: str, dim: int, with_charges: bool):
    """Reader of the fixed-layout data file, following read_config / read_charge_config
    (config_utils.cu:5-364): whitespace tokens in the same order, FP32 positions (the charge
    variant parses with %f, the plain one with %lf then casts), bonds stored from both ends."""
    with open(path) as f:
        lines = f.read().split("\n")
    it = iter(lines)
    next(it); next(it)
    ns = int(next(it).split()[0]); nbonds = int(next(it).split()[0]); nangles = int(next(it).split()[0])
    next(it)
    ntypes = int(next(it).split()[0]); nbt = int(next(it).split()[0]); next(it)
    next(it)
    box = []
    for d in range(3):
        lo, hi = next(it).split()[:2]
        if with_charges:
            box.append(float(np.float32(np.float32(hi) - np.float32(lo))))
        else:
            box.append(float(np.float32(float(hi) - float(lo))))
    next(it); next(it); next(it)
    mass = [1.0] * ntypes
    for _ in range(ntypes):
        t, m = next(it).split()[:2]
        mass[int(t) - 1] = float(np.float32(m))
    next(it); next(it); next(it)
    rest = "\n".join(it).split()
    ncol = 3 + (1 if with_charges else 0) + dim
    atoms = np.array(rest[:ns * ncol], dtype=object).reshape(ns, ncol)
    idx = atoms[:, 0].astype(np.int64) - 1
    types = np.zeros(ns, np.int32); mol = np.zeros(ns, np.int32)
    types[idx] = atoms[:, 2].astype(np.int32) - 1
    mol[idx] = atoms[:, 1].astype(np.int32) - 1
    q = None
    if with_charges:
        q = np.zeros(ns, np.float32); q[idx] = atoms[:, 3].astype(np.float32)
    x = np.zeros((ns, dim), np.float32)
    cols = atoms[:, ncol - dim:]
    if with_charges:
        x[idx] = cols.astype(np.float32)
    else:
        x[idx] = cols.astype(np.float64).astype(np.float32)
    pos = ns * ncol
    # skip "Bonds" header word
    while rest[pos] != "Bonds":
        pos += 1
    pos += 1
    b = np.array(rest[pos:pos + 4 * nbonds], dtype=np.int64).reshape(nbonds, 4)
    bonds = np.stack([b[:, 1] - 1, b[:, 2] - 1, b[:, 3] - 1], 1)
    nb, bt, by = topology_from_bonds(ns, bonds)
    return dict(ns=ns, ntypes=ntypes, nbond_types=nbt, box=box, mass=mass, types=types, mol=mol, charges=q, x=x,
                n_bonds=nb, bonded_to=bt, bond_type=by, bonds=bonds, nangles=nangles)
