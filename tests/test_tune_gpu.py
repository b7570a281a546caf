"""Schedule tuning changes how, not what, a step computes: every setting gives bitwise the same
trajectory, and tild_autotune leaves the simulation state where it found it."""
import numpy as np
import pytest

import tild
from helpers import small_diblock

pytestmark = pytest.mark.gpu


def p3_system():
    return small_diblock(3, 3, nx=(20, 18, 16), box=(10.0, 9.0, 8.0), n_chains=150, N=10, seed=31)


def run(s, tune=None, steps=70):
    with tild.Context(s) as c:
        if tune is not None:
            t = c.get_tune()
            for k, v in tune.items():
                setattr(t, k, v)
            c.set_tune(t)
        c.step(steps)
        return c.get_state()


@pytest.mark.parametrize("tune", [
    {"spread_mode": tild.SPREAD_DIRECT},
    {"spread_cap": 1024},                 # most chunks overflow the box and fall back to global atomics
    {"sort_interval": 8},
    {"sort_interval": 32},
    {"sort_brick": 0x1222},
    {"sort_brick": 0x1113},
    {"sort_brick": 0x1123, "sort_interval": 8},
    {"gather_mode": tild.GATHER_BOX},
    {"gather_mode": tild.GATHER_BOX, "gather_cap": 1024},   # most chunks fall back to global reads
    {"field_layout": tild.FIELD_BRICK},
    {"field_layout": tild.FIELD_BRICK, "gather_mode": tild.GATHER_BOX},   # box needs linear: direct runs
    {"spread_ahead": 1},                  # the gather spreads for the next step (shared box)
    {"spread_ahead": 1, "spread_mode": tild.SPREAD_DIRECT},
    {"spread_ahead": 1, "spread_cap": 1024},
    {"spread_cap": 3072, "field_layout": tild.FIELD_BRICK},
])
def test_every_setting_gives_the_same_trajectory(tune):
    s = p3_system()
    ref = run(s)
    got = run(s, tune)
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)


def test_autotune_restores_state_and_keeps_results():
    s = p3_system()
    with tild.Context(s) as c:
        c.step(20)
        x0 = c.get_state()
        best = c.autotune(trial_steps=32)
        assert best["ms_per_step"] > 0
        assert c.step_count == 20
        for a, b in zip(x0, c.get_state()):
            assert np.array_equal(a, b)
        c.step(50)
        got = c.get_state()
    ref = run(s, steps=70)
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)


def test_batch_autotune_streams():
    systems = [small_diblock(3, 1, nx=(16, 16, 16), box=(8.0, 8.0, 8.0), seed=41),
               small_diblock(3, 1, nx=(12, 14, 16), box=(6.0, 7.0, 8.0), n_chains=70, seed=42),
               small_diblock(3, 1, nx=(20, 20, 20), box=(10.0, 10.0, 10.0), n_chains=200, seed=43)]
    with tild.Batch(systems) as B:
        before = [B.get_state(i) for i in range(3)]
        best = B.autotune(trial_steps=32)
        assert 0 <= best["fft_streams"] <= 8
        t = B.get_tune()
        t.fft_streams, t.fft_pipeline = 2, 2     # the per-shape pipeline must not change results
        B.set_tune(t)
        for i in range(3):
            assert B.step_count(i) == 0
            for a, b in zip(before[i], B.get_state(i)):
                assert np.array_equal(a, b)
        B.step(40)
        tuned = [B.get_state(i)[0] for i in range(3)]
    with tild.Batch(systems) as B:
        B.step(40)
        plain = [B.get_state(i)[0] for i in range(3)]
    for a, b in zip(tuned, plain):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("brick", [0x1033, 0x1014])
def test_2d_sort_bricks_give_the_same_trajectory(brick):
    s = small_diblock(2, 2, nx=(32, 28), box=(16.0, 14.0), n_chains=150, N=10, seed=61)
    ref = run(s)
    got = run(s, {"sort_brick": brick, "sort_interval": 8})
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("level", [1, 2])
def test_shape_pipeline_gives_the_same_trajectories(level):
    systems = [small_diblock(3, 1, nx=(16, 16, 16), box=(8.0, 8.0, 8.0), seed=71),
               small_diblock(3, 1, nx=(12, 14, 16), box=(6.0, 7.0, 8.0), n_chains=70, seed=72),
               small_diblock(3, 1, nx=(20, 20, 20), box=(10.0, 10.0, 10.0), n_chains=200, seed=73)]
    out = []
    for lv in (0, level):
        with tild.Batch(systems) as B:
            t = B.get_tune()
            t.fft_streams, t.fft_pipeline = 2, lv
            B.set_tune(t)
            B.step(70)
            out.append([B.get_state(i)[0] for i in range(3)])
    for a, b in zip(*out):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("pmeorder", [1, 3])
def test_spread_ahead_after_host_changes(pmeorder):
    """The gather spreads x_{n+1} for the next step; positions replaced on the host must discard
    those densities, and a force-only evaluation may use them."""
    s = small_diblock(3, pmeorder, nx=(20, 18, 16), box=(10.0, 9.0, 8.0), n_chains=150, N=10, seed=33)
    ref = run(s, {"spread_ahead": 0}, steps=40)
    with tild.Context(s) as c:
        t = c.get_tune()
        t.spread_ahead = 1
        c.set_tune(t)
        c.step(40)
        mid = c.get_state()
        f_mid = c.forces()                       # force-only evaluation on the spread-ahead densities
        c.step(5)
        c.set_state(s.x)                         # back to the start: the pending densities are stale
        c.set_step(0)
        c.step(40)
        again = c.get_state()
    with tild.Context(s) as c:
        c.set_state(mid[0], mid[1], mid[2])
        c.set_step(40)
        f_fresh = c.forces()
    assert np.array_equal(f_mid, f_fresh)
    for a, b, r in zip(mid, again, ref):
        assert np.array_equal(a, b)
        assert np.array_equal(a, r)
