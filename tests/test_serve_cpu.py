"""Request loop of the serving layer, on the host: admission by grid shape and free slots, first
come first served, device-side stops, retirement and the latency summary.  The slot batch is a
host stand-in with the same interface (no GPU): steps advance counters, a slot leaves the active
set when its counter reaches the stop step, exactly as k_advance_steps does."""
import numpy as np

import tild_serve as sv
import tild_systems as ts


class FakeBatch:
    def __init__(self, systems, caps):
        self.systems = list(systems)
        self.caps = list(caps)
        self.stepc = [0] * len(systems)
        self.act = [True] * len(systems)
        self.stop = [-1] * len(systems)
        self.loads = []
        self.sk = [0] * len(systems)

    def sync(self):
        pass

    def close(self):
        pass

    def set_active(self, i, a):
        assert not a or self.stop[i] < 0 or self.stepc[i] < self.stop[i]
        self.act[i] = bool(a)

    def load(self, i, s, activate=True):
        assert s.ns <= self.caps[i]
        assert tuple(s.nx) == tuple(self.systems[i].nx)
        self.systems[i] = s
        self.stepc[i] = 0
        self.stop[i] = -1
        self.sk[i] = 0
        self.act[i] = bool(activate)
        self.loads.append(i)

    def set_stop(self, i, n):
        self.stop[i] = n

    def step(self, n):
        for _ in range(n):
            for i in range(len(self.systems)):
                if self.act[i]:
                    self.stepc[i] += 1
                    if self.stop[i] >= 0 and self.stepc[i] >= self.stop[i]:
                        self.act[i] = False

    def evaluate(self):
        pass

    def observables(self, i):
        return {"upe": float(self.stepc[i]) + 0.5 * i}

    def step_count(self, i):
        return self.stepc[i]

    def sk_accumulate(self, i, slot, t):
        self.sk[i] += 1

    def active(self, i):
        return self.act[i]

    def sk_get(self, i, slot):
        return np.ones(4, np.complex128), self.sk[i]

    def get_state(self, i):
        x = np.full((self.systems[i].ns, 3), float(self.stepc[i]), np.float32)
        return x, x.copy(), x.copy()

    def set_state(self, i, x, xo=None, noise=None):
        pass

    def set_step(self, i, n):
        self.stepc[i] = n


class FakeServer(sv.Server):
    def _make_batch(self, systems, caps):
        return FakeBatch(systems, caps)


def tiny(g, seed):
    L = g * 0.5
    return ts.diblock_melt(n_chains=6, N=10, box=(L, L, L), nx=(g, g, g), seed=seed)


def test_fifo_admission_per_grid_shape_and_device_stops():
    srv = FakeServer({24: 1, 26: 2}, capacity_of=lambda g: 100, template_of=lambda g: tiny(g, 1), epoch=64,
                     measure_memory=False)
    jobs = [sv.Job(0, tiny(24, 2), 100, 0), sv.Job(1, tiny(24, 3), 64, 0), sv.Job(2, tiny(26, 4), 200, 1),
            sv.Job(3, tiny(26, 5), 10, 1), sv.Job(4, tiny(26, 6), 64, 5)]
    res = srv.run(jobs, clock="epochs")
    by = {r.job_id: r for r in res}
    # job 1 waits for job 0's slot (one edge-24 slot): 0 needs two epochs (100 steps, epoch 64)
    assert by[0].admitted == 0 and by[0].finished == 2
    assert by[1].admitted == 2 and by[1].finished == 3
    # both edge-26 jobs start at epoch 1; the 10-step job retires after one epoch
    assert by[2].admitted == 1 and by[3].admitted == 1 and by[3].finished == 2
    assert by[2].finished == 5
    # job 4 arrives at epoch 5 to a free slot
    assert by[4].admitted == 5 and by[4].finished == 6
    for r in res:
        steps = [s for s, _ in r.energy]
        assert steps[-1] == r.steps                                 # the last record is the stop step
        assert steps == sorted(steps) and len(steps) == -(-r.steps // 64)
        assert r.sk_calls == len(steps)
    summ = sv.latency_summary(res)
    assert summ["jobs"] == 5 and summ["p99_s"] >= summ["p50_s"] > 0


def test_job_without_slot_shape_is_rejected():
    srv = FakeServer({24: 1}, capacity_of=lambda g: 100, template_of=lambda g: tiny(g, 1), measure_memory=False)
    try:
        srv.run([sv.Job(0, tiny(30, 2), 10, 0)], clock="epochs")
    except ValueError as e:
        assert "grid edge 30" in str(e)
    else:
        raise AssertionError("a job without a slot of its grid shape must be rejected")


def test_poisson_stream_and_capacity():
    jobs = sv.poisson_jobs(8, rate=50.0, steps=5000, seed=3)
    t = np.array([j.arrival for j in jobs])
    assert t[0] == 0 and np.all(np.diff(t) > 0)
    for j in jobs:
        g = sv.grid_edge(j.system)
        assert g in ts.ensemble_grid_edges()
        assert j.system.ns <= ts.ensemble_capacity(g)


def test_time_slice_preempts_and_resumes_from_checkpoints():
    srv = FakeServer({24: 1}, capacity_of=lambda g: 100, template_of=lambda g: tiny(g, 1), epoch=64,
                     measure_memory=False)
    jobs = [sv.Job(0, tiny(24, 2), 256, 0), sv.Job(1, tiny(24, 3), 128, 0)]
    res = srv.run(jobs, clock="epochs", time_slice=1)
    by = {r.job_id: r for r in res}
    # one slot, slices of one epoch: the two jobs alternate until job 1 (2 epochs) is done
    assert [s for s, _ in by[0].energy] == [64, 128, 192, 256]
    assert [s for s, _ in by[1].energy] == [64, 128]
    assert by[1].finished == 4 and by[0].finished == 6
    assert by[0].sk_calls == 4 and by[1].sk_calls == 2


def test_growth_admits_a_burst_beyond_the_initial_slots():
    """Admission by memory: a burst of one grid shape larger than the initial slots of that shape
    is admitted at once into pools grown for it, while the budget allows."""
    srv = FakeServer({24: 1, 26: 1}, capacity_of=lambda g: 100, template_of=lambda g: tiny(g, 1), epoch=64,
                     measure_memory=False, grow=True, group_slots=2, hbm_budget=1e9)
    jobs = [sv.Job(k, tiny(24, 10 + k), 128, 0) for k in range(5)]
    res = srv.run(jobs, clock="epochs")
    assert all(r.admitted == 0 and r.finished == 2 for r in res)
    assert srv.pools_grown == 2 and len({r.slot for r in res}) == 5


def test_growth_stops_at_the_hbm_budget():
    one = sv.slot_bytes_estimate(24, 100)
    # the two-slot initial pool plus exactly one grown pool of two slots fit
    budget = 2 * one + 2 * one + one // 2
    srv = FakeServer({24: 1, 26: 1}, capacity_of=lambda g: 100, template_of=lambda g: tiny(g, 1), epoch=64,
                     measure_memory=False, grow=True, group_slots=2, hbm_budget=budget)
    jobs = [sv.Job(k, tiny(24, 20 + k), 64, 0) for k in range(5)]
    res = srv.run(jobs, clock="epochs")
    by = {r.job_id: r for r in res}
    assert srv.pools_grown == 1 and srv.peak_bytes <= budget
    assert [by[k].admitted for k in range(5)] == [0, 0, 0, 1, 1]      # two wait one epoch


def test_idle_grown_pools_release_their_memory():
    srv = FakeServer({24: 1}, capacity_of=lambda g: 100, template_of=lambda g: tiny(g, 1), epoch=64,
                     measure_memory=False, grow=True, group_slots=2, idle_epochs=2, hbm_budget=1e9)
    burst = [sv.Job(k, tiny(24, 30 + k), 64, 0) for k in range(3)]
    late = [sv.Job(3, tiny(24, 40), 64 * 6, 0)]            # keeps the loop running after the burst
    res = srv.run(burst + late, clock="epochs")
    assert srv.pools_grown == 2 and srv.pools_released >= 1
    assert all(r.finished == 1 for r in res[:3]) and res[3].finished == 6
    assert len(srv.pools) <= 2


def test_grow_policies_size_pools():
    """Pool sizes: one slot per queued job of the shape ("demand"), the whole group once the queue
    is long against the number of waiting shapes ("load"), twice the demand ("double")."""
    mk = lambda pol: FakeServer({24: 1}, capacity_of=lambda g: 100, template_of=lambda g: tiny(g, 1), epoch=64,
                                measure_memory=False, grow=True, group_slots=8, grow_policy=pol, hbm_budget=1e9)
    d, l, x = mk("demand"), mk("load"), mk("double")
    assert [d._pool_size(k, 40, 5) for k in (1, 3, 20)] == [1, 3, 8]
    assert [l._pool_size(k, 4, 3) for k in (1, 3)] == [1, 3] and l._pool_size(1, 40, 5) == 8
    assert [x._pool_size(k, 4, 3) for k in (1, 3, 6)] == [2, 6, 8]
    try:
        mk("sometimes")
    except ValueError:
        pass
    else:
        raise AssertionError("an unknown policy must be rejected")
