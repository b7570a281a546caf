"""Shared builders and comparisons for the parity tests (oracle = FP64 CPU restatement)."""
import math

import numpy as np

import tild
import tild_systems as ts
from tild import Style

# Force tolerance: relative L2 error ||F_gpu - F_oracle|| / ||F_oracle|| of the FP32 CUDA path
# against the FP64 oracle on identical FP32 positions (the 1e-5 bound of the target).
FORCE_RTOL = 1e-5
# Energies / virials: FP64 reductions of FP32 spectra.
ENERGY_RTOL = 2e-5


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def small_diblock(dim=3, pmeorder=1, nx=None, box=None, n_chains=120, N=10, seed=7, **kw):
    box = box or ((8.0, 8.0, 8.0) if dim == 3 else (10.0, 12.0))
    nx = nx or ((16, 16, 16) if dim == 3 else (20, 24))
    box = tuple(box) + (1.0,) * (3 - len(box))
    return ts.diblock_melt(n_chains=n_chains, N=N, box=box, nx=tuple(nx) + (1,) * (3 - len(nx)), dim=dim,
                           pmeorder=pmeorder, seed=seed, **kw)


def with_styles(s, styles):
    s.styles = styles
    return s


def erf_system(kind, pmeorder=3, nx=(18, 20, 22), box=(9.0, 10.0, 11.0), seed=11):
    s = small_diblock(3, pmeorder, nx=nx, box=box, seed=seed)
    A = 2.0
    s.styles = [Style(kind, 0, 0, A, 0.5, 0.5), Style(kind, 1, 1, A, 0.5, 0.5), Style(kind, 0, 1, 1.3 * A, 0.5, 0.5)]
    return s


def charged_system(pmeorder=1, nx=(16, 18, 20), box=(8.0, 9.0, 10.0), seed=5, bjerrum=1.0, smearing=0.5):
    return ts.coacervate(n_poly=30, N=10, n_solvent=300, box=box, nx=nx, pmeorder=pmeorder, seed=seed,
                         bjerrum=bjerrum, smearing=smearing)


def coacervate_golden_system():
    import json
    import os
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    z = np.load(os.path.join(here, "coacervate_config.npz"))
    g = json.load(open(os.path.join(here, "coacervate_step0.json")))
    ns = z["x"].shape[0]
    nb, bt, by = ts.topology_from_bonds(ns, z["bonds"])
    sc = g["script"]
    s = tild.System(dim=3, nx=tuple(sc["Nx"]), box=tuple(float(v) for v in z["box"]), types=z["types"].astype(np.int32),
                    x=z["x"], n_bonds=nb, bonded_to=bt, bond_type=by, ntypes=1,
                    styles=[Style(tild.STYLE_GAUSSIAN, 0, 0, sc["gaussian"][0][2], sc["gaussian"][0][3])],
                    bond_k=(sc["bond"][0],), bond_req=(sc["bond"][1],), pmeorder=sc["pmeorder"],
                    charges=z["charges"].astype(np.float32), bjerrum=sc["charges"][0], smearing=sc["charges"][1],
                    mass=[float(v) for v in z["mass"]], delt=sc["delt"], molecule=z["mol"])
    return s, g
