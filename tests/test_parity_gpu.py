"""GPU parity: the CUDA path (libtild through the C ABI) against the FP64 oracle.

Tolerances (FP32 CUDA vs FP64 oracle on identical FP32 inputs):
  forces        relative L2 error <= 1e-5 (FORCE_RTOL)
  energies      relative error <= 2e-5 (ENERGY_RTOL), virials atol 1e-6 * scale
  stencils      grid indices bit-exact, weights rtol 1e-5
  cells/nlists  bit-exact as sets
"""
import numpy as np
import pytest

import oracle
import tild
from helpers import (ENERGY_RTOL, FORCE_RTOL, charged_system, coacervate_golden_system, erf_system, rel_l2,
                     small_diblock)
from tild import Style

pytestmark = pytest.mark.gpu


def _forces_pair(s, step=0):
    o = oracle.Oracle(s)
    fo = o.forces(s.x, step)
    with tild.Context(s) as c:
        if step:
            c.set_step(step)
        fg = c.forces()
    return fg, fo


CASES = {
    "diblock3d_p1": lambda: small_diblock(3, 1),
    "diblock3d_p0": lambda: small_diblock(3, 0),
    "diblock3d_p2_odd": lambda: small_diblock(3, 2, nx=(15, 17, 19), box=(7.5, 8.5, 9.5)),
    "diblock3d_p3": lambda: small_diblock(3, 3, nx=(18, 16, 20), box=(9.0, 8.0, 10.0)),
    "diblock3d_p4": lambda: small_diblock(3, 4, nx=(16, 16, 16)),
    "diblock2d_p1": lambda: small_diblock(2, 1),
    "diblock2d_p3": lambda: small_diblock(2, 3, nx=(21, 24)),
    "gaussian_erf_p3": lambda: erf_system(tild.STYLE_GAUSSIAN_ERF),
    "erf_p2": lambda: erf_system(tild.STYLE_ERF, pmeorder=2, nx=(17, 19, 21)),
    "charges_p1": lambda: charged_system(),
    "charges_p3": lambda: charged_system(pmeorder=3),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_forces_match_oracle(name):
    s = CASES[name]()
    fg, fo = _forces_pair(s)
    err = rel_l2(fg, fo)
    assert err < FORCE_RTOL, f"{name}: rel L2 force error {err:.3e}"


@pytest.mark.parametrize("phase,dir_", [(0, 0), (0, 2), (2, 1), (3, 0)])
def test_fieldphase_forces(phase, dir_):
    s = small_diblock(3, 1, nx=(16, 16, 16))
    s.styles = s.styles + [Style(tild.STYLE_FIELDPHASE, 0, 1, 0.7, phase=phase, dir=dir_, n_periods=2)]
    fg, fo = _forces_pair(s)
    assert rel_l2(fg, fo) < FORCE_RTOL


@pytest.mark.parametrize("name", ["diblock3d_p1", "diblock3d_p3", "diblock3d_p2_odd", "diblock2d_p3", "gaussian_erf_p3"])
def test_paired_inverse_matches_per_channel_inverse(name):
    """Two type channels take one complex transform each way (real part one channel's field,
    imaginary part the other's); a fieldphase style keeps a system on per-channel R2C and C2R.
    With the fieldphase at amplitude 0 the physics is the same, so both paths must agree to FP32
    rounding (odd grid edges and 2D included)."""
    s = CASES[name]()
    with tild.Context(s) as c:
        f_paired = c.forces()
        rho_paired = c.density()
        e_paired = c.observables()["upe"]
    s.styles = s.styles + [Style(tild.STYLE_FIELDPHASE, 0, 1, 0.0, phase=0, dir=0, n_periods=1)]
    with tild.Context(s) as c:
        f_c2r = c.forces()
        rho_c2r = c.density()
        e_c2r = c.observables()["upe"]
    err = rel_l2(f_paired, f_c2r)
    assert err < 1e-6, f"{name}: paired against per-channel inverse, rel L2 {err:.3e}"
    # the forward transforms are paired too: densities (read back de-interleaved) are the same
    # conversions bit for bit, and the energies read the unpacked spectra
    assert np.array_equal(rho_paired, rho_c2r), name
    assert e_paired == pytest.approx(e_c2r, rel=1e-6), name


def test_ramp_scales_forces_like_reference():
    s = small_diblock(3, 1)
    s.styles[2] = Style(tild.STYLE_GAUSSIAN, 0, 1, s.styles[2].prefactor, s.styles[2].sigma, ramp=True,
                        final_prefactor=2.0 * s.styles[2].prefactor)
    s.max_steps = 50
    for step in (0, 1, 2, 17):
        fg, fo = _forces_pair(s, step)
        assert rel_l2(fg, fo) < FORCE_RTOL, step


@pytest.mark.parametrize("name", ["diblock3d_p1", "diblock3d_p4", "diblock2d_p3", "diblock3d_p2_odd"])
def test_stencil_indices_bit_exact(name):
    s = CASES[name]()
    oi, ow = oracle.Oracle(s).stencil(s.x)
    with tild.Context(s) as c:
        gi, gw = c.stencil()
    assert np.array_equal(gi, oi)
    np.testing.assert_allclose(gw, ow, rtol=1e-5, atol=1e-6 * np.abs(ow).max())


@pytest.mark.parametrize("name", ["diblock3d_p1", "charges_p1", "diblock2d_p3"])
def test_density_matches_oracle(name):
    s = CASES[name]()
    o = oracle.Oracle(s)
    _, ro = o.forces(s.x, 0, want_rho=True)
    with tild.Context(s) as c:
        c.forces()
        rg = c.density()
    assert rel_l2(rg, ro) < 1e-6


@pytest.mark.parametrize("name", ["diblock3d_p1", "gaussian_erf_p3", "erf_p2", "charges_p1", "diblock2d_p1"])
def test_observables_match_oracle(name):
    s = CASES[name]()
    o = oracle.Oracle(s)
    o.forces(s.x, 0)
    oo = o.observables(s.x)
    with tild.Context(s) as c:
        og = c.observables()
    assert og["upe"] == pytest.approx(oo["upe"], rel=ENERGY_RTOL)
    assert og["ubond"] == pytest.approx(oo["ubond"], rel=1e-9)
    assert og["uelec"] == pytest.approx(oo["uelec"], rel=ENERGY_RTOL, abs=1e-9)
    np.testing.assert_allclose(og["style_energy"], oo["style_energy"], rtol=ENERGY_RTOL)
    scale = np.abs(oo["style_virial"]).max() + 1e-30
    np.testing.assert_allclose(og["style_virial"], oo["style_virial"], rtol=ENERGY_RTOL, atol=1e-5 * scale)
    np.testing.assert_allclose(og["ptens"], oo["ptens"], rtol=ENERGY_RTOL, atol=1e-5 * np.abs(oo["ptens"]).max())


def test_coacervate_golden_on_gpu():
    s, g = coacervate_golden_system()
    with tild.Context(s) as c:
        ob = c.observables()
    assert ob["upe"] == pytest.approx(g["Upe"], rel=2e-5)
    assert ob["ubond"] == pytest.approx(g["Ubond"], rel=2e-5)
    assert ob["style_energy"][0] == pytest.approx(g["Ugauss"][0], rel=2e-5)
    np.testing.assert_allclose(ob["ptens"], g["P"], rtol=2e-5, atol=1e-8)


@pytest.mark.parametrize("integ", [tild.INTEGRATOR_GJF, tild.INTEGRATOR_EM])
def test_one_step_with_matched_philox_noise(integ):
    s = small_diblock(3, 1)
    s.integrators = [(integ, -1)]
    x = s.x.copy()
    xo = x.copy()
    nz = np.zeros_like(x)
    o = oracle.Oracle(s)
    o.step(x, xo, nz, 1, True)
    with tild.Context(s) as c:
        c.step(1)
        gx, gxo, gnz = c.get_state()
    L = np.array(s.box[:3], np.float32)
    d = gx - x
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 2e-5
    if integ == tild.INTEGRATOR_GJF:
        np.testing.assert_allclose(gnz, nz, rtol=2e-5, atol=2e-6)
        np.testing.assert_array_equal(gxo, s.x)


def test_group_integrators_move_only_their_type():
    s = small_diblock(3, 1)
    s.integrators = [(tild.INTEGRATOR_EM, 1)]
    with tild.Context(s) as c:
        c.step(3)
        gx, _, _ = c.get_state()
    moved = np.any(gx != s.x, axis=1)
    assert not moved[s.types == 0].any() and moved[s.types == 1].all()


GROUP_LISTS = {
    # Integrate_2 runs every integrator of the input in order on its group (integrator.cu:24-39,
    # group.cu:44-60); a bead in two groups is moved twice with the step's forces
    "gjf_type1_em_type2": [(tild.INTEGRATOR_GJF, 0), (tild.INTEGRATOR_EM, 1)],
    "em_all_em_type2": [(tild.INTEGRATOR_EM, -1), (tild.INTEGRATOR_EM, 1)],
    "gjf_all_em_type1": [(tild.INTEGRATOR_GJF, -1), (tild.INTEGRATOR_EM, 0)],
}


@pytest.mark.parametrize("name", sorted(GROUP_LISTS))
def test_group_integrator_positions_match_oracle(name):
    """Positions of type-group and mixed integrator lists against the oracle: one step with
    matched Philox noise, then five noise-off steps."""
    s = small_diblock(3, 1)
    s.integrators = GROUP_LISTS[name]
    L = np.array(s.box[:3], np.float32)

    def dist(a, b):
        d = a - b
        d -= L * np.round(d / L)
        return float(np.abs(d).max())

    x, xo, nz = s.x.copy(), s.x.copy(), np.zeros_like(s.x)
    o = oracle.Oracle(s)
    o.step(x, xo, nz, 1, True)
    with tild.Context(s) as c:
        c.step(1)
        gx, gxo, gnz = c.get_state()
    assert dist(gx, x) < 2e-5
    np.testing.assert_allclose(gnz, nz, rtol=2e-5, atol=2e-6)
    s.noise_mag = 0.0
    x, xo, nz = s.x.copy(), s.x.copy(), np.zeros_like(s.x)
    o = oracle.Oracle(s)
    for k in range(1, 6):
        o.step(x, xo, nz, k, False)
    with tild.Context(s) as c:
        c.step(5)
        gx, _, _ = c.get_state()
    assert dist(gx, x) < 1e-4
    # beads outside every group stay where they were
    covered = np.zeros(s.ns, bool)
    for _, grp in s.integrators:
        covered |= (s.types == grp) if grp >= 0 else True
    assert np.array_equal(gx[~covered], s.x[~covered])


def test_ten_steps_track_oracle_without_noise():
    s = small_diblock(3, 1)
    s.noise_mag = 0.0
    x, xo, nz = s.x.copy(), s.x.copy(), np.zeros_like(s.x)
    o = oracle.Oracle(s)
    for k in range(1, 11):
        o.step(x, xo, nz, k, False)
    with tild.Context(s) as c:
        c.step(10)
        gx, _, _ = c.get_state()
    L = np.array(s.box[:3], np.float32)
    d = gx - x
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 1e-4


def test_sk_accumulator_matches_oracle():
    s = small_diblock(3, 1)
    o = oracle.Oracle(s)
    acc = 0
    with tild.Context(s) as c:
        x = s.x.copy()
        for k in range(3):
            c.forces()
            c.sk_accumulate(0, 1)
            o.forces(c.get_state()[0], 0)
            acc = acc + o.sk(1)
            c.step(1)
        sk, n = c.sk_get(0)
    assert n == 3
    ref = acc / 3
    assert np.abs(sk - ref).max() < 1e-5 * np.abs(ref).max()


@pytest.mark.parametrize("rc,group", [(1.0, -1), (1.6, 1), (1.0, 0), (1.3, -1)])
def test_neighbour_list_sets_match(rc, group):
    """Cells bit-exact, neighbour rows equal as sets.  When a row needs more than CELL_MAX
    entries (the reference's 7.5 x mean-occupancy heuristic, nlist.cu:100-102) the reference
    writes past its buffer; oracle and libtild both report it as an error instead."""
    s = small_diblock(3, 1)
    st, oc, on, onb, ocm = oracle.Oracle(s).nlist(s.x, rc, group)
    with tild.Context(s) as c:
        if st != 0:
            with pytest.raises(tild.TildError):
                c.nlist(rc, group)
            return
        gc, gn, gnb, gcm = c.nlist(rc, group)
    assert gcm == ocm
    assert np.array_equal(gc, oc)
    assert np.array_equal(gn, on)
    for i in range(s.ns):
        n = min(on[i], ocm)
        assert sorted(onb[i, :n].tolist()) == gnb[i, :n].tolist()
