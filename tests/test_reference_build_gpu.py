"""Parity against the reference's own CUDA build (oracle/_ref/ref_harness: the unmodified
reference objects plus a harness main that dumps d_f, d_all_rho, d_grid_inds after forces()).

Runs only where that build exists (it is compiled from the reference sources by
oracle/ref.mk); skipped otherwise.  Inputs go through the reference's own readers: the system
is written as a data file + input script, and the positions the reference read back (x0) are
the ones fed to libtild.
"""
import os
import subprocess

import numpy as np
import pytest

import tild
import tild_systems as ts
from helpers import FORCE_RTOL, charged_system, erf_system, rel_l2, small_diblock

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")


def run_harness(tmp_path, s, steps=0, nonoise=True):
    if not os.path.exists(HARNESS):
        pytest.skip("reference build not present (oracle/_ref)")
    ts.write_data_file(str(tmp_path / "input.data"), s)
    ts.write_input_script(str(tmp_path / "input"), s, max_steps=max(steps, 1), log_freq=10 ** 6, binary_freq=0)
    args = [HARNESS, "-in", "input", "-out", "ref", "-steps", str(steps)] + (["-nonoise"] if nonoise else [])
    r = subprocess.run(args, cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    D = s.dim
    S = (s.pmeorder + 1) ** D
    M = int(np.prod(s.nx[:D]))
    rd = lambda n, dt, shape: np.fromfile(str(tmp_path / f"ref_{n}.bin"), dtype=dt).reshape(shape)
    out = {"x0": rd("x0", np.float32, (s.ns, D)), "f0": rd("f0", np.float32, (s.ns, D)),
           "rho0": rd("rho0", np.float32, (s.ntypes, M)), "inds": rd("inds", np.int32, (s.ns, S)),
           "w": rd("w", np.float32, (s.ns, S)),
           "obs0": np.loadtxt(str(tmp_path / "ref_obs0.txt"))}
    if steps:
        out["xN"] = rd(f"x{steps}", np.float32, (s.ns, D))
    return out


CASES = {
    "diblock3d_p1": lambda: small_diblock(3, 1),
    "diblock3d_p3_odd": lambda: small_diblock(3, 3, nx=(15, 17, 19), box=(7.5, 8.5, 9.5)),
    "diblock3d_p4": lambda: small_diblock(3, 4),
    "diblock2d_p2": lambda: small_diblock(2, 2),
    "gaussian_erf": lambda: erf_system(tild.STYLE_GAUSSIAN_ERF),
    "erf": lambda: erf_system(tild.STYLE_ERF, pmeorder=2, nx=(16, 18, 20)),
    "charges": lambda: charged_system(),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_forces_density_stencil_vs_reference_build(tmp_path, name):
    s = CASES[name]()
    ref = run_harness(tmp_path, s)
    s.x = ref["x0"]
    with tild.Context(s) as c:
        f = c.forces()
        rho = c.density()
        inds, w = c.stencil()
        ob = c.observables()
    assert np.array_equal(inds, ref["inds"]), "stencil indices must be bit-exact"
    np.testing.assert_allclose(w, ref["w"], rtol=2e-5, atol=1e-6 * np.abs(ref["w"]).max())
    assert rel_l2(rho[:s.ntypes], ref["rho0"]) < 1e-6
    # the reference's erf tables lose ~1e-4 to FP32 cancellation at small k
    tol = 2e-4 if name == "erf" or name == "gaussian_erf" else 2e-5
    assert rel_l2(f, ref["f0"]) < tol
    # observables: reference sums M floats on the host in FP32
    o = ref["obs0"]
    assert ob["ubond"] == pytest.approx(o[1], rel=1e-4)
    assert ob["upe"] == pytest.approx(o[0], rel=1e-4)


def test_one_step_noise_off_vs_reference_build(tmp_path):
    s = small_diblock(3, 1)
    ref = run_harness(tmp_path, s, steps=3, nonoise=True)
    s.x = ref["x0"]
    s.noise_mag = 0.0
    with tild.Context(s) as c:
        c.step(3)
        x, _, _ = c.get_state()
    L = np.array(s.box[:3], np.float32)
    d = x - ref["xN"]
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 1e-4
