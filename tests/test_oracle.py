"""CPU tests of the oracle: FFT, noise stream, and the pin against the reference's golden line."""
import math

import numpy as np
import pytest

import oracle
import tild
import tild_systems as ts
from helpers import coacervate_golden_system, small_diblock


@pytest.mark.parametrize("shape", [(7,), (12, 10), (6, 9, 10), (5, 7, 11), (4, 47), (29, 3, 8), (16, 16, 16)])
def test_fft_matches_numpy(shape):
    rng = np.random.default_rng(1)
    a = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    np.testing.assert_allclose(oracle.fft(a, -1), np.fft.fftn(a), rtol=0, atol=1e-12 * np.abs(a).sum())
    np.testing.assert_allclose(oracle.fft(a, +1), np.fft.ifftn(a) * a.size, rtol=0, atol=1e-12 * np.abs(a).sum())


def test_noise_is_standard_normal():
    z = np.array([oracle.noise3(99, b, s, 0) for b in range(400) for s in range(1, 6)]).reshape(-1)
    assert abs(z.mean()) < 0.06 and abs(z.std() - 1.0) < 0.05
    # counters are independent of each other
    assert not np.allclose(oracle.noise3(1, 0, 1, 0), oracle.noise3(1, 0, 2, 0))
    assert not np.allclose(oracle.noise3(1, 0, 1, 0), oracle.noise3(1, 1, 1, 0))
    assert not np.allclose(oracle.noise3(1, 0, 1, 0), oracle.noise3(1, 0, 1, 1))


def test_coacervate_step0_golden_line():
    """examples/Coacervate/data.dat step 0: spreading + charges + gaussian + bonds + virial.
    The reference sums on the host in FP32 (integ_utils.cu:3-13, bonds.cu:3-52,
    calc_properties.cu:113-115), so its printed values carry FP32 accumulation error; the FP64
    oracle must agree within 2e-5 relative."""
    s, g = coacervate_golden_system()
    o = oracle.Oracle(s)
    o.forces(s.x, 0)
    ob = o.observables(s.x)
    assert ob["upe"] == pytest.approx(g["Upe"], rel=2e-5)
    assert ob["ubond"] == pytest.approx(g["Ubond"], rel=2e-5)
    assert ob["style_energy"][0] == pytest.approx(g["Ugauss"][0], rel=2e-5)
    np.testing.assert_allclose(ob["ptens"], g["P"], rtol=2e-5, atol=1e-8)


def test_coacervate_bond_energy_fp32_order_reproduces_print():
    """Summing the bond energy in FP32 in host_bonds' loop order gives the printed 158706."""
    s, g = coacervate_golden_system()
    x = s.x
    L = np.array(s.box, np.float32)
    Lh = np.float32(0.5) * L
    i = np.repeat(np.arange(s.ns), 3).reshape(s.ns, 3)
    m = (np.arange(3)[None, :] < s.n_bonds[:, None]) & (s.bonded_to >= i)
    a, b = i[m], s.bonded_to[m]
    dr = (x[a] - x[b]).astype(np.float32)
    dr = np.where(dr > Lh, dr - L, np.where(dr < -Lh, dr + L, dr)).astype(np.float32)
    mdr2 = ((dr[:, 0] * dr[:, 0] + dr[:, 1] * dr[:, 1]).astype(np.float32) + dr[:, 2] * dr[:, 2]).astype(np.float32)
    e = (np.sqrt(mdr2).astype(np.float32) ** 2 * np.float32(1.5)).astype(np.float32)
    acc = np.float32(0)
    for v in e:  # sequential FP32 accumulation
        acc = np.float32(acc + v)
    assert "%g" % acc == "%g" % g["Ubond"]


@pytest.mark.parametrize("p", [0, 1, 2, 3])
def test_stencil_weights_partition_of_unity(p):
    s = small_diblock(3, p)
    o = oracle.Oracle(s)
    inds, w = o.stencil(s.x)
    gvol = np.prod([s.box[d] / s.nx[d] for d in range(3)])
    np.testing.assert_allclose(w.sum(1) * gvol, 1.0, rtol=1e-6)
    assert inds.min() >= 0 and inds.max() < np.prod(s.nx)


def test_density_integrates_to_bead_count():
    s = small_diblock(2, 2)
    o = oracle.Oracle(s)
    _, rho = o.forces(s.x, 0, want_rho=True)
    dV = np.prod([s.box[d] / s.nx[d] for d in range(2)])
    counts = np.bincount(s.types, minlength=s.ntypes)
    np.testing.assert_allclose(rho.sum(1) * dV, counts, rtol=1e-10)


def test_bond_topology_matches_reader_layout():
    """read_config stores each bond from both ends in file order (config_utils.cu:111-123)."""
    bonds = np.array([[0, 0, 1], [0, 2, 1], [1, 2, 3], [0, 5, 4]])
    nb, bt, by = ts.topology_from_bonds(6, bonds)
    assert nb.tolist() == [1, 2, 2, 1, 1, 1]
    assert bt[1, :2].tolist() == [0, 2] and bt[2, :2].tolist() == [1, 3]
    assert by[2, :2].tolist() == [0, 1] and bt[4, 0] == 5 and bt[5, 0] == 4


def test_forces_sum_to_zero_without_field():
    """Pair and bond forces are internal: total force ~ 0 (up to assignment error)."""
    s = small_diblock(3, 1)
    o = oracle.Oracle(s)
    f = o.forces(s.x, 0)
    assert np.abs(f.sum(0)).max() < 1e-6 * np.abs(f).sum()
