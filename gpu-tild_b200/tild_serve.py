"""Continuous batching of TILD simulation jobs on one GPU.

The reference runs one system per process (main.cu:47-290) and has no request loop; this module
is the serving form layered on the batched engine.  A pool of slots is created once: each slot
is a system of a slot batch (tild_batch_create_slots) with a fixed grid shape and a bead
capacity, so its state stays resident in HBM.  The loop

  1. admits arrived jobs, first come first served, into free slots of their grid shape while the
     pool's device footprint stays inside the HBM budget (tild_batch_load rebuilds the slot's
     k-space tables, then topology and state are uploaded and the slot is activated with a
     device-side stop at the job's step count);
  2. advances every active slot by one epoch of `epoch` steps in one stepping call (CUDA graphs,
     one launch per stage for all slots), so jobs admitted at different times overlap on the GPU;
  3. evaluates the densities of every slot at its current positions (one force evaluation without a
     step; stopped slots hold their last positions) and records each running job's energy (FP64
     observables) and accumulates its avg_sk, so every record describes the state at its step;
  4. retires the jobs whose slots left the active set on the device (their last step ran inside
     the epoch), returning the energy trace and S(k) and freeing the slot for the queue.

A job's result does not depend on what else runs: the spread is fixed point (order-independent),
the noise is keyed by (bead id, step, seed), and every other kernel is per bead or per grid
point of one system.  Only cuFFT's batched transforms could round differently with the batch
size; the serving test bounds that.
"""
from __future__ import annotations

import collections
import dataclasses
import math
import time
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

import tild
import tild_systems as ts


@dataclasses.dataclass
class Job:
    job_id: int
    system: tild.System
    steps: int
    arrival: float                 # seconds after the loop starts (epochs when clock="epochs")
    sk_type: int = 0               # bead type whose avg_sk is accumulated


@dataclasses.dataclass
class JobResult:
    job_id: int
    ns: int
    grid: int
    steps: int
    arrival: float
    admitted: float = math.nan
    finished: float = math.nan
    slot: int = -1
    energy: List[tuple] = dataclasses.field(default_factory=list)   # (step, upe) after each epoch
    sk: Optional[np.ndarray] = None                                  # avg_sk, full spectrum
    sk_calls: int = 0
    x: Optional[np.ndarray] = None                                   # final positions (keep_positions)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


@dataclasses.dataclass
class Checkpoint:
    """Full state of a preempted job: resuming it in any free slot of its grid shape continues
    the trajectory bitwise (positions, x_{n-1} and GJF noise restored, step counter restored, the
    noise being keyed by (bead id, step, seed)).  avg_sk is carried as the accumulated sum."""
    job: Job
    result: JobResult
    x: np.ndarray
    xo: np.ndarray
    noise: np.ndarray
    step: int
    sk_sum: Optional[np.ndarray]
    sk_calls: int
    epochs_run: int = 0


def grid_edge(s: tild.System) -> int:
    nx = tuple(int(v) for v in s.nx[:s.dim])
    if len(set(nx)) != 1:
        raise ValueError("serving slots are keyed by a cubic grid edge")
    return nx[0]


def device_free_bytes(device: int) -> int:
    import torch
    free, _ = torch.cuda.mem_get_info(device)
    return int(free)


class Server:
    """A slot pool plus the request loop.

    slots_per_edge: number of slots for each grid edge g (g^3 grids).
    capacity_of(g): bead capacity of a slot of edge g.
    template_of(g): a system of edge g that initialises the slot before its first job.
    hbm_budget: bytes the pool may occupy on the device; creation fails beyond it.
    epoch: steps per stepping call (a multiple of 32 keeps every call inside CUDA graphs).
    """

    def __init__(self, slots_per_edge: Dict[int, int], capacity_of: Callable[[int], int] = ts.ensemble_capacity,
                 template_of: Callable[[int], tild.System] = ts.ensemble_slot_template, device: int = 0,
                 hbm_budget: float = 80e9, epoch: int = 128, keep_positions: bool = False,
                 measure_memory: bool = True, tune: bool = False):
        self.device = device
        self.epoch = int(epoch)
        self.keep_positions = keep_positions
        self.hbm_budget = float(hbm_budget)
        systems, caps, self.edge_of_slot = [], [], []
        for g, n in sorted(slots_per_edge.items()):
            tpl = template_of(g)
            for _ in range(n):
                systems.append(tpl)
                caps.append(max(capacity_of(g), tpl.ns))
                self.edge_of_slot.append(g)
        free0 = device_free_bytes(device) if measure_memory else 0
        self.batch = self._make_batch(systems, caps)
        self.batch.sync()
        self.pool_bytes = (free0 - device_free_bytes(device)) if measure_memory else 0
        if self.pool_bytes > self.hbm_budget:
            self.batch.close()
            raise MemoryError(f"slot pool needs {self.pool_bytes / 1e9:.1f} GB, budget {self.hbm_budget / 1e9:.1f} GB")
        # schedule chosen on the full pool (every slot holding its template system)
        self.schedule = self.batch.autotune(trial_steps=64) if tune else None
        for i in range(len(systems)):
            self.batch.set_active(i, False)
        self.free: Dict[int, collections.deque] = collections.defaultdict(collections.deque)
        for i, g in enumerate(self.edge_of_slot):
            self.free[g].append(i)
        self.nslots = len(systems)
        self.epochs_run = 0
        self.stepping_s = 0.0     # wall time of the stepping calls and their force evaluation
        self.work_done = 0        # particle-steps the jobs advanced inside those calls

    def _make_batch(self, systems, caps):
        return tild.Batch(systems, device=self.device, capacity=caps)

    def close(self):
        self.batch.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---------------------------------------------------------------------------------------
    def checkpoint(self, slot: int, job: Job, r: JobResult, epochs_run: int = 0) -> Checkpoint:
        """Takes the full state of the job in `slot` off the GPU and frees the slot."""
        x, xo, nz = self.batch.get_state(slot)
        sk, n = self.batch.sk_get(slot, 0)
        ck = Checkpoint(job, r, x, xo, nz, self.batch.step_count(slot), sk * n if n else None, n, epochs_run)
        self.batch.set_active(slot, False)
        self.free[r.grid].append(slot)
        return ck

    def _start(self, slot: int, item, now: float):
        """Puts a new job or a checkpoint into `slot` and activates it."""
        if isinstance(item, Checkpoint):
            job, r = item.job, item.result
            self.batch.load(slot, job.system, activate=False)
            self.batch.set_state(slot, item.x, item.xo, item.noise)
            self.batch.set_step(slot, item.step)
            r.slot = slot
        else:
            job = item
            r = JobResult(job.job_id, job.system.ns, grid_edge(job.system), job.steps, job.arrival, admitted=now,
                          slot=slot)
            self.batch.load(slot, job.system, activate=False)
        self.batch.set_stop(slot, job.steps)
        self.batch.set_active(slot, True)
        return job, r

    def run(self, jobs: Sequence[Job], clock: str = "wall", time_slice: Optional[int] = None,
            preempt_at: Optional[Dict[int, int]] = None) -> List[JobResult]:
        """Serves `jobs` to completion.  clock="wall": arrivals in seconds of wall time since the
        call (a Poisson stream replayed in real time); clock="epochs": arrival k means the job
        arrives before epoch k (deterministic, for tests).  Times in the results use the same
        unit as the arrivals.

        time_slice: a job that has run this many epochs while another job of its grid shape
        waits is checkpointed and queued behind it (round-robin within a shape); None never
        preempts.  preempt_at: {job_id: epoch} checkpoints that job once, after that many of its
        epochs (tests)."""
        for j in jobs:
            if grid_edge(j.system) not in self.free:
                raise ValueError(f"job {j.job_id}: no slot has grid edge {grid_edge(j.system)}")
            if j.steps < 1:
                raise ValueError(f"job {j.job_id}: steps must be positive")
        pending = collections.deque(sorted(jobs, key=lambda j: j.arrival))
        queue: List = []                      # Jobs and Checkpoints, first come first served
        running: Dict[int, list] = {}         # slot -> [job, result, epochs run since (re)start]
        results: Dict[int, JobResult] = {}
        sk_parts: Dict[int, list] = collections.defaultdict(list)
        preempt_at = dict(preempt_at or {})
        t0 = time.perf_counter()
        epoch_no = 0

        def now() -> float:
            return (time.perf_counter() - t0) if clock == "wall" else float(epoch_no)

        def edge_of(item) -> int:
            return grid_edge((item.job if isinstance(item, Checkpoint) else item).system)

        while pending or queue or running:
            t = now()
            while pending and pending[0].arrival <= t:
                queue.append(pending.popleft())
            waiting = []
            for item in queue:
                g = edge_of(item)
                if self.free[g]:
                    slot = self.free[g].popleft()
                    job, r = self._start(slot, item, now())
                    running[slot] = [job, r, 0]
                    results[job.job_id] = r
                else:
                    waiting.append(item)
            queue = waiting
            if not running:
                if pending and clock == "wall":
                    time.sleep(max(0.0, pending[0].arrival - now()))
                elif pending:
                    epoch_no = max(epoch_no + 1, int(math.ceil(pending[0].arrival)))
                continue
            ts0 = time.perf_counter()
            before = {slot: self.batch.step_count(slot) for slot in running}
            self.batch.step(self.epoch)
            # records describe each job's state after the epoch (stopped jobs: their last step)
            self.batch.evaluate()
            self.stepping_s += time.perf_counter() - ts0
            self.epochs_run += 1
            epoch_no += 1
            waiting_edges = collections.Counter(edge_of(it) for it in queue)
            for slot in list(running):
                job, r, ran = running[slot]
                ran += 1
                running[slot][2] = ran
                o = self.batch.observables(slot)
                step_now = self.batch.step_count(slot)
                self.work_done += (step_now - before[slot]) * job.system.ns
                r.energy.append((step_now, o["upe"]))
                self.batch.sk_accumulate(slot, 0, job.sk_type)
                if not self.batch.active(slot):
                    sk, n = self.batch.sk_get(slot, 0)
                    parts = sk_parts.pop(job.job_id, []) + [(sk * n, n)]
                    r.sk_calls = sum(k for _, k in parts)
                    r.sk = sum(v for v, _ in parts) / r.sk_calls
                    if self.keep_positions:
                        r.x = self.batch.get_state(slot)[0]
                    r.finished = now()
                    del running[slot]
                    self.free[r.grid].append(slot)
                    continue
                forced = preempt_at.get(job.job_id) == ran
                if forced or (time_slice is not None and ran >= time_slice and waiting_edges[r.grid] > 0):
                    if forced:
                        del preempt_at[job.job_id]
                    ck = self.checkpoint(slot, job, r)
                    if ck.sk_sum is not None:
                        sk_parts[job.job_id].append((ck.sk_sum, ck.sk_calls))
                    ck.sk_sum, ck.sk_calls = None, 0
                    del running[slot]
                    queue.append(ck)
                    waiting_edges[r.grid] -= 1
        return [results[j.job_id] for j in jobs]


def poisson_jobs(n: int, rate: float, steps: int = 5000, seed: int = 20261208, first_index: int = 0) -> List[Job]:
    """n jobs drawn from the batched-ensemble distribution with Poisson arrivals of mean `rate`
    per second (seeded)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    t -= t[0]
    return [Job(k, ts.ensemble_member(first_index + k), steps, float(t[k])) for k in range(n)]


def latency_summary(results: Sequence[JobResult]) -> dict:
    lat = np.array([r.latency for r in results])
    wait = np.array([r.admitted - r.arrival for r in results])
    span = max(r.finished for r in results) - min(r.arrival for r in results)
    work = sum(r.ns * r.steps for r in results)
    return {"jobs": len(results), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max()), "queue_wait_p50_s": float(np.percentile(wait, 50)),
            "queue_wait_p99_s": float(np.percentile(wait, 99)), "span_s": float(span),
            "aggregate_particle_steps_per_s": work / span if span > 0 else math.nan}
