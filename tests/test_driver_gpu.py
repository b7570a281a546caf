"""The drop-in driver (gpu-tild -in <script>) on the GPU: every output file the reference
writes, in the reference's formats, with step-0 values checked against the oracle and — where
the reference's own build is present — against the reference program run on the same files."""
import os
import subprocess

import numpy as np
import pytest

import oracle
import tild_systems as ts
from helpers import charged_system, small_diblock

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "gpu-tild_b200", "bin", "gpu-tild")
REF = os.path.join(ROOT, "oracle", "_ref", "gpu-tild")


def setup_dir(d, s, steps=6, extra=None):
    ts.write_data_file(str(d / "input.data"), s)
    ts.write_input_script(str(d / "input"), s, max_steps=steps, log_freq=2, binary_freq=3, grid_freq=3, traj_freq=3,
                          extra=extra)


def run(exe, d):
    r = subprocess.run([exe, "-in", "input"], cwd=d, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return r.stdout


def read_data_dat(path):
    lines = open(path).read().strip().splitlines()
    return lines[0], [np.array([float(v) for v in l.split()]) for l in lines[1:]]


def traj_frames(path):
    text = open(path).read().split("ITEM: TIMESTEP\n")[1:]
    return [(int(f.split("\n")[0]), f) for f in text]


@pytest.mark.parametrize("kind", ["neutral", "charged"])
def test_driver_outputs_and_step0(tmp_path, kind):
    s = small_diblock(3, 1) if kind == "neutral" else charged_system()
    setup_dir(tmp_path, s, extra=["compute avg_sk 1 freq 2"])
    out = run(EXE, tmp_path)
    assert "Step 0 of 6" in out and "Step 6 of 6" in out
    header, rows = read_data_dat(tmp_path / "data.dat")
    assert header.startswith("# step Upe Ubond  Pxx Pyy Pzz Pxy Pxz Pyz Ugauss[0]")
    assert [int(r[0]) for r in rows] == [0, 2, 4, 6]
    # step-0 line against the oracle on the positions the driver read
    d = ts.read_data_file(str(tmp_path / "input.data"), 3, s.charges is not None)
    s.x = d["x"]
    o = oracle.Oracle(s)
    o.forces(s.x, 0)
    ob = o.observables(s.x)
    r0 = rows[0]
    assert r0[1] == pytest.approx(ob["upe"], rel=2e-5)
    assert r0[2] == pytest.approx(ob["ubond"], rel=2e-5)
    np.testing.assert_allclose(r0[3:9], ob["ptens"], rtol=2e-4, atol=1e-6 * np.abs(ob["ptens"]).max())
    np.testing.assert_allclose(r0[9:9 + len(s.styles)], ob["style_energy"], rtol=2e-5)
    # trajectory: frames 0, 3, 6 and the final frame stamped max_steps + 1
    frames = traj_frames(tmp_path / "traj.lammpstrj")
    assert [f[0] for f in frames] == [0, 3, 6, 7]
    # binary outputs: headers + two frames (steps 3, 6)
    M = int(np.prod(s.nx[:3]))
    g = np.fromfile(tmp_path / "grid_densities.bin", dtype=np.int32)
    assert g[0] == 3 and list(g[1:4]) == list(s.nx[:3]) and g[7] == s.ntypes
    assert (tmp_path / "grid_densities.bin").stat().st_size == 32 + 2 * 4 * M * s.ntypes
    hdr = 4 * (2 + 3 + 2 * s.ns + 1) + (4 * s.ns if s.charges is not None else 0)
    assert (tmp_path / "positions.bin").stat().st_size == hdr + 2 * 4 * 3 * s.ns
    for t in range(s.ntypes):
        assert len(open(tmp_path / f"rho{t}.dat").read().strip().splitlines()) == M
    sk = open(tmp_path / "avg_sk_0.dat").read().strip().splitlines()
    assert len(sk) == M - 1 and len(sk[0].split()) == 7


@pytest.mark.parametrize("kind", ["neutral", "charged"])
def test_read_resume_restarts_from_a_trajectory_frame(tmp_path, kind):
    """read_resume (config_utils.cu:405-454) takes positions from a trajectory frame: a run
    resumed from the step-3 frame of another run starts from those positions (its step-0 frame
    prints them again, its step-0 energies are the oracle's at them).  On the charged frame the
    reference program reads the same files to the same step-0 line; on a 3-D frame without
    charges its reader misparses (its "%f " format swallows the newline and the next line's first
    characters), so there only the oracle is compared."""
    s = small_diblock(3, 1) if kind == "neutral" else charged_system()
    a = tmp_path / "a"
    a.mkdir()
    setup_dir(a, s, steps=3)
    run(EXE, a)
    frame = [f for st, f in traj_frames(a / "traj.lammpstrj") if st == 3][0]
    text = "ITEM: TIMESTEP\n" + frame
    rows = [l.split() for l in frame.strip().split("\n")[8:]]
    x3 = np.array([[float(v) for v in r[3:6]] for r in rows], np.float32)
    assert x3.shape == (s.ns, 3)
    outs = {}
    for exe, sub in ((EXE, "b"), (REF, "c")):
        if not os.path.exists(exe) or (sub == "c" and kind == "neutral"):
            continue
        d = tmp_path / sub
        d.mkdir()
        (d / "resume.lammpstrj").write_text(text)
        setup_dir(d, s, steps=2, extra=["read_resume resume.lammpstrj"])
        run(exe, d)
        outs[sub] = d
    b = outs["b"]
    f0 = traj_frames(b / "traj.lammpstrj")[0]
    assert f0[0] == 0 and f0[1].split("\n")[8:] == frame.split("\n")[8:]
    assert "read_resume resume.lammpstrj" in open(b / "NEED_A_NAME.input").read()
    _, rb = read_data_dat(b / "data.dat")
    s.x = x3
    o = oracle.Oracle(s)
    o.forces(s.x, 0)
    ob = o.observables(s.x)
    assert rb[0][1] == pytest.approx(ob["upe"], rel=2e-5)
    assert rb[0][2] == pytest.approx(ob["ubond"], rel=2e-5)
    if "c" in outs:
        _, rc = read_data_dat(outs["c"] / "data.dat")
        # the reference sums in FP32 on the host: near-zero off-diagonal pressures carry its noise
        np.testing.assert_allclose(rb[0], rc[0], rtol=5e-5, atol=1e-5 * np.abs(rc[0][3:6]).max())
        assert open(b / "NEED_A_NAME.input").read() == open(outs["c"] / "NEED_A_NAME.input").read()


def test_driver_matches_reference_program(tmp_path):
    """Same files through both programs: identical step-0 trajectory text, step-0 data.dat line
    and rho files within FP32 print precision."""
    if not os.path.exists(REF):
        pytest.skip("reference build not present")
    s = small_diblock(3, 1)
    (tmp_path / "a").mkdir()
    (tmp_path / "b").mkdir()
    for sub in ("a", "b"):
        setup_dir(tmp_path / sub, s, steps=2)
    run(EXE, tmp_path / "a")
    run(REF, tmp_path / "b")
    fa, fb = traj_frames(tmp_path / "a" / "traj.lammpstrj"), traj_frames(tmp_path / "b" / "traj.lammpstrj")
    assert fa[0][1] == fb[0][1]
    assert [f[0] for f in fa] == [f[0] for f in fb]
    ha, ra = read_data_dat(tmp_path / "a" / "data.dat")
    hb, rb = read_data_dat(tmp_path / "b" / "data.dat")
    assert ha == hb
    np.testing.assert_allclose(ra[0], rb[0], rtol=5e-5, atol=1e-7)
    for t in range(s.ntypes):
        ga = np.loadtxt(tmp_path / "a" / f"rho{t}.dat")
        gb = np.loadtxt(tmp_path / "b" / f"rho{t}.dat")
        np.testing.assert_array_equal(ga[:, :3], gb[:, :3])
        np.testing.assert_allclose(ga[:, 3], gb[:, 3], rtol=1e-5, atol=1e-5)
    ea = open(tmp_path / "a" / "NEED_A_NAME.input").read()
    eb = open(tmp_path / "b" / "NEED_A_NAME.input").read()
    assert ea == eb
