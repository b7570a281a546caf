"""Batched engine: several independent systems of different boxes, grids, types, styles and
integrators advanced together must give each system the results it gets alone (densities
bitwise, forces to FP32 noise, trajectories with matched noise counters)."""
import numpy as np
import pytest

import oracle
import tild
import tild_systems as ts
from helpers import FORCE_RTOL, charged_system, rel_l2, small_diblock

pytestmark = pytest.mark.gpu


def mixed_systems():
    a = small_diblock(3, 1, nx=(16, 16, 16), box=(8.0, 8.0, 8.0), seed=1)
    b = small_diblock(3, 1, nx=(12, 14, 16), box=(6.0, 7.0, 8.0), n_chains=70, seed=2)
    c = small_diblock(3, 1, nx=(16, 16, 16), box=(8.5, 8.5, 8.5), n_chains=90, N=7, seed=3)
    c.integrators = [(tild.INTEGRATOR_EM, -1)]
    d = charged_system()          # 3 types + charges, EM
    e = ts.ensemble_member(5)     # diblock ensemble member (random box/grid/N/chi)
    return [a, b, c, d, e]


def test_batch_forces_match_single_and_oracle():
    systems = mixed_systems()
    with tild.Batch(systems) as B:
        fb = [B.forces(i) for i in range(len(systems))]
        rb = [B.density(i) for i in range(len(systems))]
    for i, s in enumerate(systems):
        with tild.Context(s) as c:
            fs = c.forces()
            rs = c.density()
        assert np.array_equal(rb[i], rs), f"system {i}: densities differ"
        assert rel_l2(fb[i], fs) < 1e-6, i
        fo = oracle.Oracle(s).forces(s.x, 0)
        assert rel_l2(fb[i], fo) < FORCE_RTOL, i


def test_batch_mixes_paired_and_per_channel_inverses():
    """A grid shape whose systems all have an even channel count and no fieldphase takes the paired
    complex inverse; a fieldphase system turns its whole shape to per-channel C2R.  Here the 16^3
    shape holds a plain diblock (paired when alone) and a fieldphase system, the other shapes stay
    paired: every system must still match its single-system run and the oracle."""
    a = small_diblock(3, 1, nx=(16, 16, 16), box=(8.0, 8.0, 8.0), seed=1)
    f = small_diblock(3, 1, nx=(16, 16, 16), box=(8.5, 8.5, 8.5), n_chains=90, seed=4)
    f.styles = f.styles + [tild.Style(tild.STYLE_FIELDPHASE, 0, 1, 0.7, phase=0, dir=1, n_periods=2)]
    b = small_diblock(3, 1, nx=(12, 14, 16), box=(6.0, 7.0, 8.0), n_chains=70, seed=2)
    d = charged_system()
    systems = [a, f, b, d]
    with tild.Batch(systems) as B:
        fb = [B.forces(i) for i in range(len(systems))]
        rb = [B.density(i) for i in range(len(systems))]
    for i, s in enumerate(systems):
        with tild.Context(s) as c:
            fs = c.forces()
            rs = c.density()
        assert np.array_equal(rb[i], rs), f"system {i}: densities differ"
        assert rel_l2(fb[i], fs) < 1e-6, i
        assert rel_l2(fb[i], oracle.Oracle(s).forces(s.x, 0)) < FORCE_RTOL, i


def test_batch_steps_match_single_runs():
    systems = mixed_systems()
    with tild.Batch(systems) as B:
        B.step(7)
        xb = [B.get_state(i)[0] for i in range(len(systems))]
        ob = [B.observables(i) for i in range(len(systems))]
        steps = [B.step_count(i) for i in range(len(systems))]
    assert steps == [7] * len(systems)
    for i, s in enumerate(systems):
        with tild.Context(s) as c:
            c.step(7)
            xs = c.get_state()[0]
            os_ = c.observables()
        L = np.array(s.box[:3], np.float32)
        d = xb[i] - xs
        d -= L * np.round(d / L)
        assert np.abs(d).max() < 1e-4, i
        assert ob[i]["upe"] == pytest.approx(os_["upe"], rel=1e-5)


def test_inactive_system_keeps_its_state():
    systems = mixed_systems()[:3]
    with tild.Batch(systems) as B:
        B.set_active(1, False)
        B.step(3)
        x1 = B.get_state(1)[0]
        assert B.step_count(1) == 0 and B.step_count(0) == 3
        np.testing.assert_array_equal(x1, systems[1].x)
        B.set_active(1, True)
        B.step(2)
        assert B.step_count(1) == 2


def test_reloading_a_system_in_place():
    """Serving reuses a slot: new topology + state into system 0 of a running batch."""
    systems = mixed_systems()[:2]
    fresh = small_diblock(3, 1, nx=(16, 16, 16), box=(8.0, 8.0, 8.0), seed=99)
    with tild.Batch(systems) as B:
        B.step(20)  # sorts the slots
        B.set_topology(0, fresh)
        B.set_state(0, fresh.x)
        B.set_step(0, 0)
        f0 = B.forces(0)
    with tild.Context(fresh) as c:
        fs = c.forces()
    assert rel_l2(f0, fs) < 1e-6


def test_graph_replay_matches_direct_steps():
    """Whole step periods run as a captured CUDA graph: the trajectory must be bit-identical to
    stepping one call at a time (densities are deterministic, every kernel is the same)."""
    s = small_diblock(3, 1)
    with tild.Context(s) as c:
        c.step(70)                       # 2 graph periods of 32 (capture + replay) + 6 direct steps
        xg, xog, ng = c.get_state()
        assert c.step_count == 70
    with tild.Context(s) as c:
        for _ in range(70):
            c.step(1)
        xd, xod, nd = c.get_state()
    np.testing.assert_array_equal(xg, xd)
    np.testing.assert_array_equal(xog, xod)
    np.testing.assert_array_equal(ng, nd)


@pytest.mark.parametrize("pmeorder,chunks", [(1, [20] * 5), (1, [9, 45, 13, 8, 25]), (3, [20] * 5),
                                              (3, [31, 17, 10, 40])])
def test_graphs_of_any_length_match_direct_steps(pmeorder, chunks):
    """Runs shorter than a whole period, or starting between sorts, replay graphs of their own
    length (captured per starting configuration): bit-identical to one step per call, whatever
    the split, and the replays leave the host at the right buffers and sort phase."""
    s = small_diblock(3, pmeorder, nx=(16, 18, 20), box=(8.0, 9.0, 10.0))
    n = sum(chunks)
    with tild.Context(s) as c:
        for k in chunks:
            c.step(k)
        for k in chunks:                 # the same split again: every graph is replayed
            c.step(k)
        xg, xog, ng = c.get_state()
        assert c.step_count == 2 * n
    with tild.Context(s) as c:
        for _ in range(2 * n):
            c.step(1)
        xd, xod, nd = c.get_state()
    np.testing.assert_array_equal(xg, xd)
    np.testing.assert_array_equal(xog, xod)
    np.testing.assert_array_equal(ng, nd)


def test_batch_stops_inside_a_remainder_graph():
    systems = mixed_systems()[:3]
    with tild.Batch(systems) as B:
        B.set_stop(1, 13)
        B.step(20)                       # one graph of 20 steps; system 1 stops after its 13th
        assert [B.step_count(i) for i in range(3)] == [20, 13, 20] and not B.active(1)
        B.step(20)
        assert [B.step_count(i) for i in range(3)] == [40, 13, 40]


def test_batch_graph_with_inactive_system():
    systems = mixed_systems()[:3]
    with tild.Batch(systems) as B:
        B.step(64)
        B.set_active(2, False)
        x2 = B.get_state(2)[0]
        B.step(64)                       # replays the captured graph with one system inactive
        np.testing.assert_array_equal(B.get_state(2)[0], x2)
        assert [B.step_count(i) for i in range(3)] == [128, 128, 64]
