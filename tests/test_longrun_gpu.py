"""Long-run statistics against the reference build.  The same diblock melt is run by the reference
program (its cuRAND XORWOW noise) and by the drop-in driver (Philox noise) for thousands of steps.
The noise streams are independent, so the trajectories differ, but the equilibrium averages must
agree: the mean potential and bond energies over the second half within statistical error (block
averages of the logged values), and the radially averaged avg_sk peak: its |S|-weighted centre
within 0.75 of a shell (shells of 0.2 in |k|) and its weight within 15 %."""
import os
import subprocess

import numpy as np
import pytest

import tild_systems as ts

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "gpu-tild_b200", "bin", "gpu-tild")
REF = os.path.join(ROOT, "oracle", "_ref", "gpu-tild")

STEPS, LOG, WAIT = 6000, 50, 3000
N_SIGMA = 4.0     # agreement bound on the difference of means, in combined standard errors


def run_program(exe, d):
    r = subprocess.run([exe, "-in", "input"], cwd=d, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]


def energies(path):
    rows = [np.array([float(v) for v in l.split()]) for l in open(path).read().strip().splitlines()[1:]]
    a = np.array(rows)
    return a[a[:, 0] > WAIT]


def mean_and_error(v, blocks=6):
    b = np.array([x.mean() for x in np.array_split(v, blocks)])
    return v.mean(), b.std(ddof=1) / np.sqrt(blocks)


def sk_profile(path, kmax=4.0, nbins=20):
    """Radial average of |S(k)| over shells of |k| (avg_sk_%d.dat columns: k, |S|, |k|, Re, Im)."""
    a = np.loadtxt(path)
    k, s = a[:, 4], a[:, 3]
    edges = np.linspace(0.0, kmax, nbins + 1)
    idx = np.digitize(k, edges)
    return np.array([s[idx == i].mean() if np.any(idx == i) else 0.0 for i in range(1, nbins + 1)])


def peak_centroid(prof, last=13):
    """|S(k)|-weighted mean shell index over the correlation-hole peak (shells below `last`):
    steadier than the arg-max of a broad, noisy peak."""
    i = np.arange(last)
    return float((i * prof[:last]).sum() / prof[:last].sum())


@pytest.mark.skipif(not os.path.exists(REF), reason="reference build not present")
def test_equilibrium_averages_match_reference_build(tmp_path):
    s = ts.diblock_melt(n_chains=480, N=20, fA=0.5, box=(12.0, 12.0, 12.0), nx=(24, 24, 24), chiN=8.0,
                        seed=ts.SEED_BASE + 41, max_steps=STEPS)
    dirs = {}
    for name, exe in (("ref", REF), ("ours", EXE)):
        d = tmp_path / name
        d.mkdir()
        ts.write_data_file(str(d / "input.data"), s)
        ts.write_input_script(str(d / "input"), s, max_steps=STEPS, log_freq=LOG, binary_freq=0,
                              extra=[f"compute avg_sk 1 freq {LOG} wait {WAIT}"])
        run_program(exe, d)
        dirs[name] = d
    er, eo = energies(dirs["ref"] / "data.dat"), energies(dirs["ours"] / "data.dat")
    for col, what in ((1, "Upe"), (2, "Ubond")):
        mr, sr = mean_and_error(er[:, col])
        mo, so = mean_and_error(eo[:, col])
        tol = N_SIGMA * np.hypot(sr, so) + 1e-6 * abs(mr)
        print(f"{what}: reference {mr:.6g} +- {sr:.2g}, ours {mo:.6g} +- {so:.2g}")
        assert abs(mr - mo) <= tol, what
    sr, so = sk_profile(dirs["ref"] / "avg_sk_0.dat"), sk_profile(dirs["ours"] / "avg_sk_0.dat")
    print("S(k) shells, reference:", np.array2string(sr, precision=1))
    print("S(k) shells, ours:     ", np.array2string(so, precision=1))
    pr, po = peak_centroid(sr), peak_centroid(so)
    print(f"S(k) peak centroid (shells of 0.2): reference {pr:.2f}, ours {po:.2f}")
    assert abs(pr - po) <= 0.75, (pr, po)
    assert abs(sr[:13].sum() - so[:13].sum()) <= 0.15 * sr[:13].sum()
