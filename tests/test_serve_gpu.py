"""Continuous batching on the GPU: a slot reloaded with another system while its neighbours run
gives that system's own forces; a device-side stop ends a system after exactly its step count;
and every served job's energy trace and final positions are the same alone and in the mix."""
import numpy as np
import pytest

import tild
import tild_serve as sv
import tild_systems as ts
from helpers import rel_l2

pytestmark = pytest.mark.gpu

# Results of a job alone and in a mix may differ only through cuFFT rounding for a different
# number of batched transforms; these bounds are what the comparison allows.
ENERGY_RTOL = 1e-5
POS_ATOL = 1e-4


def job_system(g, seed, N=16, fA=0.4, chiN=15.0, n_chains=None):
    L = g * 0.5
    n_chains = n_chains or int(round(4.0 * L ** 3 / N))
    return ts.diblock_melt(n_chains=n_chains, N=N, fA=fA, box=(L, L, L), nx=(g, g, g), chiN=chiN, seed=seed,
                           max_steps=5000)


def min_image_maxdiff(a, b, box):
    d = np.abs(a - b)
    box = np.asarray(box[:a.shape[1]], np.float32)
    d = np.minimum(d, box - d)
    return float(d.max())


def test_slot_load_matches_fresh_context():
    g = 24
    tpl = ts.ensemble_slot_template(g)
    cap = ts.ensemble_capacity(g)
    job = job_system(g, 11)
    with tild.Batch([tpl, tpl], capacity=[cap, cap]) as B:
        B.step(40)
        B.load(1, job)
        B.step(0)
        f = B.forces(1)
        r = B.density(1)
        assert B.capacity(1) == cap and B.step_count(1) == 0
    with tild.Context(job) as c:
        fs = c.forces()
        rs = c.density()
    assert np.array_equal(r, rs)
    assert rel_l2(f, fs) < 1e-6


def test_device_stop_takes_exact_steps():
    g = 24
    tpl = ts.ensemble_slot_template(g)
    cap = ts.ensemble_capacity(g)
    job = job_system(g, 12)
    with tild.Batch([tpl, tpl], capacity=[cap, cap]) as B:
        B.load(1, job, activate=False)
        B.set_stop(1, 200)
        B.set_active(1, True)
        B.step(256)
        assert B.step_count(1) == 200 and not B.active(1)
        assert B.step_count(0) == 256 and B.active(0)
        x = B.get_state(1)[0]
        with pytest.raises(tild.TildError):
            B.set_active(1, True)          # at its stop step
    with tild.Context(job) as c:
        c.step(200)
        xs = c.get_state()[0]
    assert min_image_maxdiff(x, xs, job.box) < POS_ATOL


def test_served_results_same_alone_and_in_mix():
    systems = [job_system(24, 21), job_system(26, 22, N=20, fA=0.5, chiN=25.0), job_system(24, 23, N=10),
               job_system(26, 24, N=12, chiN=12.0), job_system(24, 25, fA=0.3)]
    steps = [300, 200, 150, 260, 128]
    arrivals = [0, 0, 1, 2, 2]
    jobs = [sv.Job(k, s, n, a) for k, (s, n, a) in enumerate(zip(systems, steps, arrivals))]
    with sv.Server({24: 2, 26: 2}, epoch=64, keep_positions=True, measure_memory=False) as srv:
        mixed = srv.run(jobs, clock="epochs")
    assert any(r.admitted > r.arrival for r in mixed)      # someone waited for a slot
    worst_e, worst_x = 0.0, 0.0
    for job, rm in zip(jobs, mixed):
        g = sv.grid_edge(job.system)
        with sv.Server({g: 1}, epoch=64, keep_positions=True, measure_memory=False) as alone_srv:
            ra = alone_srv.run([sv.Job(job.job_id, job.system, job.steps, 0)], clock="epochs")[0]
        assert [s for s, _ in rm.energy] == [s for s, _ in ra.energy]
        assert rm.energy[-1][0] == job.steps and rm.sk_calls == ra.sk_calls
        em = np.array([e for _, e in rm.energy])
        ea = np.array([e for _, e in ra.energy])
        worst_e = max(worst_e, float(np.max(np.abs(em - ea) / np.abs(ea))))
        worst_x = max(worst_x, min_image_maxdiff(rm.x, ra.x, job.system.box))
        assert np.allclose(rm.sk, ra.sk, rtol=1e-4, atol=1e-6 * np.abs(ra.sk).max())
    print(f"alone vs mix: max energy rel diff {worst_e:.3e}, max position diff {worst_x:.3e}")
    assert worst_e < ENERGY_RTOL and worst_x < POS_ATOL


def test_preempted_job_resumes_bitwise():
    """A job checkpointed off the GPU mid-run and resumed later in a slot that another job used in
    between gives the same energy trace and final positions as the same job run without a break."""
    a = sv.Job(0, job_system(24, 31), 320, 0)
    b = sv.Job(1, job_system(24, 32, N=10), 128, 0)
    with sv.Server({24: 1}, epoch=64, keep_positions=True, measure_memory=False) as srv:
        broken = srv.run([a, b], clock="epochs", preempt_at={0: 2})
    with sv.Server({24: 1}, epoch=64, keep_positions=True, measure_memory=False) as srv:
        whole = srv.run([sv.Job(0, a.system, a.steps, 0)], clock="epochs")[0]
    ra = broken[0]
    assert ra.admitted == 0 and ra.finished > whole.finished       # it waited while job 1 ran
    assert ra.energy == whole.energy
    assert np.array_equal(ra.x, whole.x)
    assert ra.sk_calls == whole.sk_calls
    assert np.allclose(ra.sk, whole.sk, rtol=1e-12, atol=1e-12 * np.abs(whole.sk).max())


def test_burst_of_one_shape_admitted_by_memory():
    """With pools grown inside the HBM budget, a burst of 14 jobs of one grid shape (2 initial
    slots) is admitted at once; each job's trace matches the same job served alone."""
    jobs = [sv.Job(k, job_system(24, 50 + k, N=10 + (k % 3) * 4), 128 + 64 * (k % 2), 0) for k in range(14)]
    with sv.Server({24: 2, 26: 1}, epoch=64, keep_positions=True, grow=True, group_slots=4) as srv:
        res = srv.run(jobs, clock="epochs")
        grown, peak = srv.pools_grown, srv.peak_bytes
    assert grown == 3 and peak <= 80e9
    assert all(r.admitted == 0 for r in res)
    for k in (0, 5, 13):
        with sv.Server({24: 1}, epoch=64, keep_positions=True, measure_memory=False) as alone_srv:
            ra = alone_srv.run([sv.Job(k, jobs[k].system, jobs[k].steps, 0)], clock="epochs")[0]
        em = np.array([e for _, e in res[k].energy])
        ea = np.array([e for _, e in ra.energy])
        assert [s for s, _ in res[k].energy] == [s for s, _ in ra.energy]
        assert np.max(np.abs(em - ea) / np.abs(ea)) < ENERGY_RTOL
        assert min_image_maxdiff(res[k].x, ra.x, jobs[k].system.box) < POS_ATOL
