"""CPU tests of the drop-in driver's script surface (gpu-tild -in <script> --dry-run): the
keyword grammar and ordering rules of read_input.cu, the data-file reader and the
NEED_A_NAME.input echo (read_input.cu:565-651), without a GPU."""
import json
import os
import subprocess

import numpy as np
import pytest

import tild_systems as ts
from helpers import coacervate_golden_system

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "gpu-tild_b200", "bin", "gpu-tild")
GOLD = json.load(open(os.path.join(ROOT, "tests", "golden", "coacervate_step0.json")))


def run(tmp_path, script_text, data_system=None, data_name="input.data"):
    if not os.path.exists(EXE):
        pytest.skip("driver not built")
    (tmp_path / "input").write_text(script_text)
    if data_system is not None:
        ts.write_data_file(str(tmp_path / data_name), data_system)
    return subprocess.run([EXE, "-in", "input", "--dry-run"], cwd=tmp_path, capture_output=True, text=True, timeout=120)


def test_echo_file_matches_reference_example(tmp_path):
    s, _ = coacervate_golden_system()
    r = run(tmp_path, GOLD["script_text"], s)
    assert r.returncode == 0, r.stdout + r.stderr
    mine = [l for l in (tmp_path / "NEED_A_NAME.input").read_text().splitlines() if not l.startswith("rand_seed")]
    ref = [l for l in GOLD["need_a_name_input"].splitlines() if not l.startswith("rand_seed")]
    assert mine == ref
    assert "Input file read!" in r.stdout


SMALL = """Dim 3
max_steps 10
log_freq 5
read_data input.data
integrator all GJF
Nx 8
Ny 8
Nz 8
bond 1 harmonic 1.5 0.0
n_gaussians 1
gaussian 1 1 1.0 1.0
"""


@pytest.mark.parametrize("script,message", [
    (SMALL.replace("read_data input.data", "read_data input.data\ncharges 1.0 0.5"),
     "charges keyword must come before read_data command!"),
    ("Dim 3\nbond 1 harmonic 1.5 0.0\nread_data input.data\n", "bond keyword before config read"),
    (SMALL + "integrator all VV\n", "VV is not a valid integrator!"),
    (SMALL + "integrator nogroup EM\n", "Group nogroup not found to integrate!"),
    (SMALL + "pmeorder 5\n", "PMEORDER greater than 4 not supported!"),
    (SMALL + "frobnicate 3\n", "Invalid keyword error"),
    (SMALL.replace("gaussian 1 1 1.0 1.0", "gaussian 1 3 1.0 1.0"), "Invalid particle type in Gaussian input!"),
    (SMALL + "group g1 molecule 1\n", "ERROR: Group type molecule not supported!"),
    (SMALL + "compute avg_sk 9\n", "Invalid type to calculate avg_sk"),
])
def test_script_errors_are_reported_like_the_reference(tmp_path, script, message):
    from helpers import small_diblock
    r = run(tmp_path, script, small_diblock(3, 1, n_chains=4, N=5))
    assert r.returncode == 1
    assert message in r.stdout


def test_groups_integrators_computes_and_ramps_parse(tmp_path):
    from helpers import small_diblock
    script = SMALL.replace("n_gaussians 1\ngaussian 1 1 1.0 1.0",
                           "n_gaussians 2\ngaussian 1 1 1.0 1.0\ngaussian 1 2 2.0 0.5 ramp 3.0") + \
        "group grpA type 1\nintegrator grpA EM\ncompute avg_sk 2 freq 5 wait 2\ndiffusivity 2 0.5\nrand_seed 77\n"
    r = run(tmp_path, script, small_diblock(3, 1, n_chains=4, N=5))
    assert r.returncode == 0, r.stdout
    echo = (tmp_path / "NEED_A_NAME.input").read_text().splitlines()
    assert "group grpA type 1" in echo
    assert "integrator all GJF" in echo and "integrator grpA EM" in echo
    assert "compute avg_sk 2 freq 5 wait 2" in echo
    assert "diffusivity 2 0.5" in echo and "rand_seed 77" in echo
    assert "gaussian1 2 2 0.25" in echo  # the reference's missing space and sigma^2
    assert "Calculating <S(k)> for component 2 every 5 steps after 2 steps have passed." in r.stdout


def test_data_reader_matches_python_reader(tmp_path):
    """The C++ reader and tild_systems.read_data_file agree (both follow config_utils.cu:5-183)."""
    from helpers import small_diblock
    s = small_diblock(3, 1, n_chains=6, N=7)
    ts.write_data_file(str(tmp_path / "input.data"), s)
    d = ts.read_data_file(str(tmp_path / "input.data"), 3, False)
    assert d["ns"] == s.ns and np.array_equal(d["types"], s.types)
    assert np.array_equal(d["n_bonds"], s.n_bonds) and np.array_equal(d["bonded_to"], s.bonded_to)
    np.testing.assert_allclose(d["x"], s.x, atol=1e-6)
    r = run(tmp_path, SMALL, None)
    assert r.returncode == 0 and f"ns {s.ns} M 512" in r.stdout
