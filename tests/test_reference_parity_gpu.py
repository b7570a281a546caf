"""Parity with the reference's own CUDA build at the target's bounds, on the benchmark
configurations at their real sizes.

The reference build here is oracle/_ref/ref_harness: the unmodified reference objects plus a
harness main that runs initialize(); forces() and dumps d_f, d_all_rho, d_grid_inds/W (and, on
request, a neighbour list and the positions after N steps).  libtild runs with
table_mode = TABLES_REF_FP32, which evaluates the k-space multipliers with the reference's FP32
expressions (pair_style_erf.cu:122-158, pair_style_gaussian_erf.cu:82-115,
pair_style_gaussian.cu:72-90), so the comparison isolates the per-step path.  The FP64-table
path is held to the same 1e-5 against the FP64 oracle beside it.

Bounds written here (the target's):
  forces     ||F - F_ref||_2 / ||F_ref||_2 <= 1e-5
  densities  relative L2 <= 1e-6
  stencils   grid indices bit-exact
  positions  after N steps with the same cuRAND XORWOW stream: max |dx| <= 1e-5 * L
  neighbours cell ids bit-exact, rows equal as sets
Each test prints the measured errors.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle
import tild
import tild_systems as ts
from helpers import FORCE_RTOL, erf_system, rel_l2, small_diblock

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
RHO_RTOL = 1e-6


def harness(tmp_path, s, steps=0, nonoise=True, ninds=None, nlist=None, timeout=900):
    """Runs the reference harness on s written in the reference's file formats; returns its dumps."""
    if not os.path.exists(HARNESS):
        pytest.skip("reference build not present (oracle/_ref)")
    ts.write_data_file(str(tmp_path / "input.data"), s)
    extra = None
    if nlist is not None and nlist[1] != "all":
        extra = [f"group {nlist[1]} type {int(nlist[1][4:])}"]
    ts.write_input_script(str(tmp_path / "input"), s, max_steps=max(steps, 1), log_freq=10 ** 8, binary_freq=0,
                          extra=extra)
    args = [HARNESS, "-in", "input", "-out", "ref", "-steps", str(steps)]
    if nonoise:
        args.append("-nonoise")
    if ninds is not None:
        args += ["-ninds", str(ninds)]
    if nlist is not None:
        args += ["-nlist", repr(float(nlist[0])), nlist[1]]
    r = subprocess.run(args, cwd=tmp_path, capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    D = s.dim
    S = (s.pmeorder + 1) ** D
    M = int(np.prod(s.nx[:D]))
    K = s.ns if ninds is None else min(ninds, s.ns)
    rd = lambda n, dt, shape: np.fromfile(str(tmp_path / f"ref_{n}.bin"), dtype=dt).reshape(shape)
    out = {"x0": rd("x0", np.float32, (s.ns, D)), "f0": rd("f0", np.float32, (s.ns, D)),
           "rho0": rd("rho0", np.float32, (s.ntypes, M)), "inds": rd("inds", np.int32, (K, S)),
           "obs0": np.loadtxt(str(tmp_path / "ref_obs0.txt"))}
    if steps:
        out["xN"] = rd(f"x{steps}", np.float32, (s.ns, D))
    if nlist is not None:
        cmax, _ = (int(v) for v in open(tmp_path / "ref_nlist.txt").read().split())
        out["cell"] = rd("cell", np.int32, (s.ns,))
        out["ncount"] = rd("ncount", np.int32, (s.ns,))
        out["neigh"] = rd("neigh", np.int32, (s.ns, cmax))
        out["cmax"] = cmax
    for f in tmp_path.glob("ref_*.bin"):
        f.unlink()
    return out


def ref_fp32(s):
    s.table_mode = tild.TABLES_REF_FP32
    return s


# ---------------------------------------------------------------------------------------------
# erf-family styles with the reference's FP32 tables: 1e-5 against the reference build
# ---------------------------------------------------------------------------------------------
ERF_CASES = {
    "gaussian_erf_p3": lambda: erf_system(tild.STYLE_GAUSSIAN_ERF),
    "gaussian_erf_p1": lambda: erf_system(tild.STYLE_GAUSSIAN_ERF, pmeorder=1, nx=(20, 20, 24), box=(10.0, 10.0, 12.0)),
    "erf_p2": lambda: erf_system(tild.STYLE_ERF, pmeorder=2, nx=(16, 18, 20)),
    "erf_p3": lambda: erf_system(tild.STYLE_ERF, pmeorder=3, nx=(18, 20, 22)),
}


@pytest.mark.parametrize("name", sorted(ERF_CASES))
def test_erf_styles_with_reference_tables_match_reference_build(tmp_path, name):
    s = ref_fp32(ERF_CASES[name]())
    ref = harness(tmp_path, s)
    s.x = ref["x0"]
    with tild.Context(s) as c:
        f = c.forces()
        rho = c.density()
        ob = c.observables()
    ef, er = rel_l2(f, ref["f0"]), rel_l2(rho[:s.ntypes], ref["rho0"])
    print(f"{name}: force error {ef:.2e}, density error {er:.2e}")
    assert er < RHO_RTOL
    assert ef < FORCE_RTOL
    # the reference sums energies on the host in FP32; its own rounding sets this bound
    assert ob["upe"] == pytest.approx(ref["obs0"][0], rel=1e-4)


# ---------------------------------------------------------------------------------------------
# The benchmark configurations at their real sizes
# ---------------------------------------------------------------------------------------------
def check_full_size(tmp_path, s, name, ninds=20000):
    """One force evaluation of s: libtild (reference tables) against the reference build, and
    libtild (FP64 tables) against the FP64 oracle, both at 1e-5; stencil indices of the first
    `ninds` beads bit-exact; densities at 1e-6."""
    ref = harness(tmp_path, ref_fp32(s), ninds=ninds)
    s.x = ref["x0"]
    with tild.Context(s) as c:
        f_ref_tables = c.forces()
        rho = c.density()
        inds, _ = c.stencil()
    e_ref = rel_l2(f_ref_tables, ref["f0"])
    e_rho = rel_l2(rho[:s.ntypes], ref["rho0"])
    same_inds = np.array_equal(inds[:ninds], ref["inds"])
    s.table_mode = tild.TABLES_FP64
    o = oracle.Oracle(s)
    fo = o.forces(s.x, 0)
    o.close()
    with tild.Context(s) as c:
        f64 = c.forces()
    e_or = rel_l2(f64, fo)
    e_64_ref = rel_l2(f64, ref["f0"])
    print(f"{name}: ns={s.ns} grid={s.nx[:s.dim]} force error vs reference build {e_ref:.2e} (reference tables), "
          f"vs FP64 oracle {e_or:.2e} (FP64 tables); FP64 tables vs reference build {e_64_ref:.2e}; "
          f"density error {e_rho:.2e}; stencil indices of {ninds} beads bit-exact: {same_inds}")
    assert same_inds
    assert e_rho < RHO_RTOL
    assert e_ref < FORCE_RTOL
    assert e_or < FORCE_RTOL


def test_diblock_40k_full_size(tmp_path):
    """40,000-bead AB diblock melt, 40^3 grid, CIC, three gaussian styles."""
    check_full_size(tmp_path, ts.diblock_melt(), "diblock_40k")


def test_coacervate_220k_full_size(tmp_path):
    """220,000-bead charged coacervate, 96^3 grid, smeared charges + gaussian excluded volume."""
    check_full_size(tmp_path, ts.coacervate(), "coacervate_220k")


def test_blend_2_6M_full_size(tmp_path):
    """2.6M-bead A/B blend, 128^3 grid, 64-point stencil, three gaussian_erf styles: the
    configuration the throughput is quoted on."""
    check_full_size(tmp_path, ts.homopolymer_blend(), "blend_2.6M")


# ---------------------------------------------------------------------------------------------
# Noise on: the reference's cuRAND XORWOW stream (cuda_random_posits.cu:22-30,
# device_GJF_integrator.cu:36, device_EM_integrator.cu) reproduced with rng = RNG_XORWOW
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("integ", [tild.INTEGRATOR_GJF, tild.INTEGRATOR_EM])
def test_xorwow_noise_steps_match_reference_build(tmp_path, integ):
    s = small_diblock(3, 1)
    s.integrators = [(integ, -1)]
    s.rng = tild.RNG_XORWOW
    steps = 5
    ref = harness(tmp_path, s, steps=steps, nonoise=False)
    s.x = ref["x0"]
    with tild.Context(s) as c:
        c.step(steps)
        x, _, _ = c.get_state()
    L = np.array(s.box[:3], np.float32)
    d = x - ref["xN"]
    d -= L * np.round(d / L)
    moved = x - ref["x0"]
    moved -= L * np.round(moved / L)
    err = float(np.abs(d).max())
    print(f"XORWOW {'GJF' if integ == tild.INTEGRATOR_GJF else 'EM'}: {steps} steps, max |dx| {err:.2e}, "
          f"rms displacement {float(np.sqrt((moved ** 2).mean())):.3e}")
    assert err <= 1e-5 * float(L.max())


# ---------------------------------------------------------------------------------------------
# Neighbour list against the reference's NList kernels (nlist.cu:83-228)
# ---------------------------------------------------------------------------------------------
def nlist_fits(s, rc, group_type):
    """The reference kernels write without bounds checks: run them only when, in FP32 as they
    compute it, every cell id is in range and no cell or neighbour row exceeds CELL_MAX."""
    D = s.dim
    L = np.array(s.box[:D], np.float32)
    nc = np.array([int(np.float32(l) / np.float32(rc)) for l in L], np.int64)
    Lc = (L / nc.astype(np.float32)).astype(np.float32)
    sel = np.ones(s.ns, bool) if group_type < 0 else (s.types == group_type)
    cid = (s.x[sel, :D] / Lc).astype(np.int64)
    if (cid < 0).any() or (cid >= nc).any():
        return False
    st = oracle.Oracle(s).nlist(s.x, rc, group_type)[0]
    return st == 0


@pytest.mark.parametrize("rc,group", [(1.0, -1), (1.6, 1), (1.25, -1)])
def test_neighbour_list_matches_reference_build(tmp_path, rc, group):
    s = small_diblock(3, 1)
    # the harness reads the positions back from the data file: check the ones it will use
    ts.write_data_file(str(tmp_path / "probe.data"), s)
    s.x = ts.read_data_file(str(tmp_path / "probe.data"), 3, False)["x"]
    if not nlist_fits(s, rc, group):
        pytest.skip("this cut-off overflows the reference's fixed-size lists")
    gname = "all" if group < 0 else f"type{group + 1}"
    ref = harness(tmp_path, s, nlist=(rc, gname))
    assert np.array_equal(ref["x0"], s.x)
    with tild.Context(s) as c:
        gc, gn, gnb, gcm = c.nlist(rc, group)
    assert gcm == ref["cmax"]
    sel = np.ones(s.ns, bool) if group < 0 else (s.types == group)
    assert np.array_equal(gc[sel], ref["cell"][sel])
    assert np.array_equal(gn[sel], ref["ncount"][sel])
    for i in np.nonzero(sel)[0]:
        n = ref["ncount"][i]
        assert sorted(ref["neigh"][i, :n].tolist()) == gnb[i, :n].tolist()
    print(f"nlist rc={rc} group={gname}: {int(sel.sum())} beads, CELL_MAX {gcm}, "
          f"{int(gn[sel].sum())} neighbour entries equal as sets")


# ---------------------------------------------------------------------------------------------
# Beads on the faces of the box: x = 0 and x = L are both legal positions for the reference (its
# integrators wrap only x > L and x < 0, device_GJF_integrator.cu:52-55), and their stencils wrap
# across the periodic boundary (device_grid_utils.cu:305-325)
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("pmeorder", [1, 2, 3, 4])
def test_beads_on_the_box_faces(tmp_path, pmeorder):
    s = small_diblock(3, pmeorder)
    L = np.array(s.box[:3], np.float32)
    x = s.x.copy()
    x[0] = [0.0, 0.0, 0.0]
    x[1] = L
    x[2] = [L[0], 0.0, L[2] * 0.5]
    x[3] = [0.0, L[1], 0.0]
    x[4] = [L[0] * 0.25, L[1], 0.0]
    x[5] = (L - np.float32(1e-6)).astype(np.float32)     # just below the faces (6 decimals in the file)
    s.x = x.astype(np.float32)
    ref = harness(tmp_path, ref_fp32(s))
    assert np.array_equal(ref["x0"][:6], s.x[:6])      # the face beads reach the reference unrounded
    s.x = ref["x0"]                                     # the others as the data file rounded them
    with tild.Context(s) as c:
        f = c.forces()
        inds, _ = c.stencil()
        rho = c.density()
    assert np.array_equal(inds, ref["inds"])
    assert rel_l2(rho[:s.ntypes], ref["rho0"]) < RHO_RTOL
    e_ref = rel_l2(f, ref["f0"])
    s.table_mode = tild.TABLES_FP64
    fo = oracle.Oracle(s).forces(s.x, 0)
    with tild.Context(s) as c:
        e_or = rel_l2(c.forces(), fo)
    print(f"faces p{pmeorder}: force error vs reference build {e_ref:.2e}, vs oracle {e_or:.2e}")
    assert e_ref < FORCE_RTOL and e_or < FORCE_RTOL
