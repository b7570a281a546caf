"""Continuous batching of TILD simulation jobs on one GPU.

The reference runs one system per process (main.cu:47-290) and has no request loop; this module
is the serving form layered on the batched engine.  Slots live in pools: a pool is one slot batch
(tild_batch_create_slots), each slot a system with a fixed grid shape and a bead capacity, so its
state stays resident in HBM.  The server starts with one pool of a fixed number of slots per grid
edge; with grow=True, a job whose grid shape has no free slot gets a new pool of `group_slots`
slots of that shape whenever the device footprint of all pools stays inside the HBM budget, and
pools that have run no job for `idle_epochs` epochs are released.  Admission is therefore bounded
by memory, not by a fixed number of slots per shape.  The loop

  1. admits arrived jobs, first come first served, into free slots of their grid shape, growing
     a pool for the shape when none is free and the budget allows (tild_batch_load rebuilds the
     slot's k-space tables, then topology and state are uploaded and the slot is activated with a
     device-side stop at the job's step count);
  2. advances every pool with an active slot by one epoch of `epoch` steps (CUDA graphs, one
     launch per stage for all slots of a pool); pools step concurrently from worker threads, each
     on its own stream, so jobs admitted at different times overlap on the GPU;
  3. evaluates the densities of every slot at its current positions (one force evaluation without a
     step; stopped slots hold their last positions) and records each running job's energy (FP64
     observables) and accumulates its avg_sk, so every record describes the state at its step;
  4. retires the jobs whose slots left the active set on the device (their last step ran inside
     the epoch), returning the energy trace and S(k) and freeing the slot for the queue.

A job's result does not depend on what else runs or which pool holds it: the spread is fixed
point (order-independent), the noise is keyed by (bead id, step, seed), and every other kernel is
per bead or per grid point of one system.  Only cuFFT's batched transforms could round
differently with the batch size; the serving test bounds that.
"""
from __future__ import annotations

import collections
import concurrent.futures
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


def slot_bytes_estimate(g: int, capacity: int) -> int:
    """Device bytes of one slot of grid edge g (diblock: two density channels, three gaussian
    styles) from the engine's layout: per grid point and channel 8 (fixed-point) + 4 (density) +
    16 (float4 field) bytes and 16 bytes of half spectra (the two channels' inverse transforms run
    as one complex transform in the force spectra, so no planar fields), the multiplier and virial
    tables, and about 100 bytes per bead of capacity.  Used when the footprint is not measured on
    the device."""
    M = g ** 3
    return int(2 * 28 * M + 2 * 16 * M + 3 * 2 * M + 3 * 6 * 4 * M + 100 * capacity)


class _Pool:
    """One slot batch: its slots' grid edges, whether it was grown on demand, its device bytes."""

    def __init__(self, pid: int, batch, edges: List[int], grown: bool, nbytes: int):
        self.pid = pid
        self.batch = batch
        self.edges = list(edges)
        self.grown = grown
        self.nbytes = int(nbytes)
        self.idle = 0                      # consecutive epochs with no job in any slot


class Server:
    """Slot pools plus the request loop.

    slots_per_edge: slots of the initial pool for each grid edge g (g^3 grids).
    capacity_of(g): bead capacity of a slot of edge g.
    template_of(g): a system of edge g that initialises a slot before its first job.
    hbm_budget: bytes all pools may occupy on the device; the initial pool must fit, and pools
      are grown only while the total stays inside it.
    epoch: steps per stepping call (a multiple of 32 keeps every call inside CUDA graphs).
    grow: create a pool of `group_slots` slots for a grid shape whose slots are all busy while a
      job of that shape waits and the budget allows; release grown pools idle for `idle_epochs`.
      With grow, slots_per_edge may be empty: every slot is then grown on demand.
    workers: threads that step the pools of one epoch concurrently.
    grow_policy: how many slots a grown pool gets ("demand", "load", "double"; see _pool_size).
    Slots are named by integers that stay unique for the server's lifetime.
    """

    def __init__(self, slots_per_edge: Dict[int, int], capacity_of: Callable[[int], int] = ts.ensemble_capacity,
                 template_of: Callable[[int], tild.System] = ts.ensemble_slot_template, device: int = 0,
                 hbm_budget: float = 80e9, epoch: int = 128, keep_positions: bool = False,
                 measure_memory: bool = True, tune: bool = False, grow: bool = False, group_slots: int = 4,
                 idle_epochs: int = 2, workers: int = 16, grow_policy: str = "demand"):
        self.device = device
        self.epoch = int(epoch)
        self.keep_positions = keep_positions
        self.hbm_budget = float(hbm_budget)
        self.capacity_of = capacity_of
        self.template_of = template_of
        self.measure_memory = measure_memory
        self.grow = grow
        self.group_slots = int(group_slots)
        self.idle_epochs = int(idle_epochs)
        if grow_policy not in ("demand", "load", "double"):
            raise ValueError(f"unknown grow_policy {grow_policy}")
        self.grow_policy = grow_policy
        self.pools: Dict[int, _Pool] = {}
        self.slot_at: Dict[int, tuple] = {}          # slot -> (pool id, index in the pool)
        self.free: Dict[int, collections.deque] = collections.defaultdict(collections.deque)
        self.edges = set(slots_per_edge)
        self._next_pid = 0
        self._next_slot = 0
        self.pools_grown = 0
        self.pools_released = 0
        self.peak_bytes = 0
        edges = [g for g, n in sorted(slots_per_edge.items()) for _ in range(n)]
        if not edges and not grow:
            raise ValueError("no initial slots and no growth: nothing could run")
        self.schedule, self._tune = None, None
        if edges:
            pool = self._new_pool(edges, grown=False)
            if pool.nbytes > self.hbm_budget:
                pool.batch.close()
                raise MemoryError(f"slot pool needs {pool.nbytes / 1e9:.1f} GB, budget {self.hbm_budget / 1e9:.1f} GB")
            # schedule chosen on the initial pool (every slot holding its template system); grown
            # pools take it too, with their single grid shape's FFTs on the main stream
            if tune:
                self.schedule = pool.batch.autotune(trial_steps=64)
                self._tune = pool.batch.get_tune()
            self._register(pool)
        self.nslots = len(edges)
        self.epochs_run = 0
        self.stepping_s = 0.0     # wall time of the stepping calls and their force evaluation
        self.work_done = 0        # particle-steps the jobs advanced inside those calls
        self._exec = concurrent.futures.ThreadPoolExecutor(max_workers=workers)

    @property
    def pool_bytes(self) -> int:
        return sum(p.nbytes for p in self.pools.values())

    def _make_batch(self, systems, caps):
        return tild.Batch(systems, device=self.device, capacity=caps)

    def _new_pool(self, edges: List[int], grown: bool) -> _Pool:
        systems, caps = [], []
        for g in edges:
            tpl = self.template_of(g)
            systems.append(tpl)
            caps.append(max(self.capacity_of(g), tpl.ns))
        free0 = device_free_bytes(self.device) if self.measure_memory else 0
        batch = self._make_batch(systems, caps)
        batch.sync()
        if self.measure_memory:
            nbytes = free0 - device_free_bytes(self.device)
        else:
            nbytes = sum(slot_bytes_estimate(g, c) for g, c in zip(edges, caps))
        pool = _Pool(self._next_pid, batch, edges, grown, nbytes)
        self._next_pid += 1
        return pool

    def _register(self, pool: _Pool):
        for i in range(len(pool.edges)):
            pool.batch.set_active(i, False)
        self.pools[pool.pid] = pool
        for i, g in enumerate(pool.edges):
            sid = self._next_slot
            self._next_slot += 1
            self.slot_at[sid] = (pool.pid, i)
            self.free[g].append(sid)
        self.peak_bytes = max(self.peak_bytes, self.pool_bytes)

    def _release(self, pool: _Pool):
        mine = {sid for sid, (pid, _) in self.slot_at.items() if pid == pool.pid}
        for g in set(pool.edges):
            self.free[g] = collections.deque(sid for sid in self.free[g] if sid not in mine)
        for sid in mine:
            del self.slot_at[sid]
        del self.pools[pool.pid]
        pool.batch.close()
        self.pools_released += 1

    def _pool_size(self, demand: int, queued: int, shapes_waiting: int) -> int:
        """Slots of a pool grown for a shape with `demand` queued jobs, while `queued` jobs of
        `shapes_waiting` shapes wait in all.  "demand": one slot per queued job of the shape;
        "load": the same while the queue is short, group_slots once it is longer than two jobs
        per waiting shape (an overloaded stream keeps any slot busy); "double": twice the demand."""
        if self.grow_policy == "double":
            n = 2 * demand
        elif self.grow_policy == "load" and queued > 2 * max(1, shapes_waiting):
            n = self.group_slots
        else:
            n = demand
        return max(1, min(self.group_slots, n or self.group_slots))

    def _try_grow(self, g: int, running: dict, n: int) -> bool:
        """A pool of n slots of edge g, if the budget allows (idle grown pools of other shapes
        are released first when that makes room).  Returns whether slots were added."""
        caps = [max(self.capacity_of(g), self.template_of(g).ns)] * n
        need = sum(slot_bytes_estimate(g, c) for c in caps)
        known = [p for p in self.pools.values() if p.grown and p.edges[0] == g and len(p.edges) == n]
        if known:
            need = known[0].nbytes
        if self.pool_bytes + need > self.hbm_budget:
            busy = {self.slot_at[sid][0] for sid in running}
            for p in sorted(self.pools.values(), key=lambda p: -p.idle):
                if p.grown and p.pid not in busy and self.pool_bytes + need > self.hbm_budget:
                    self._release(p)
            if self.pool_bytes + need > self.hbm_budget:
                return False
        pool = self._new_pool([g] * n, grown=True)
        if self._tune is not None:
            t = pool.batch.get_tune()
            for f, _ in tild.Tune._fields_:
                if f not in ("fft_streams", "fft_pipeline", "ms_per_step"):
                    setattr(t, f, getattr(self._tune, f))
            pool.batch.set_tune(t)
        if self.pool_bytes + pool.nbytes > self.hbm_budget:
            pool.batch.close()
            return False
        self._register(pool)
        self.pools_grown += 1
        return True

    def close(self):
        self._exec.shutdown(wait=True)
        for p in list(self.pools.values()):
            p.batch.close()
        self.pools.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _b(self, slot: int):
        pid, i = self.slot_at[slot]
        return self.pools[pid].batch, i

    # ---------------------------------------------------------------------------------------
    def checkpoint(self, slot: int, job: Job, r: JobResult, epochs_run: int = 0) -> Checkpoint:
        """Takes the full state of the job in `slot` off the GPU and frees the slot."""
        b, i = self._b(slot)
        x, xo, nz = b.get_state(i)
        sk, n = b.sk_get(i, 0)
        ck = Checkpoint(job, r, x, xo, nz, b.step_count(i), sk * n if n else None, n, epochs_run)
        b.set_active(i, False)
        self.free[r.grid].append(slot)
        return ck

    def _start(self, slot: int, item, now: float):
        """Puts a new job or a checkpoint into `slot` and activates it."""
        b, i = self._b(slot)
        if isinstance(item, Checkpoint):
            job, r = item.job, item.result
            b.load(i, job.system, activate=False)
            b.set_state(i, item.x, item.xo, item.noise)
            b.set_step(i, item.step)
            r.slot = slot
        else:
            job = item
            r = JobResult(job.job_id, job.system.ns, grid_edge(job.system), job.steps, job.arrival, admitted=now,
                          slot=slot)
            b.load(i, job.system, activate=False)
        b.set_stop(i, job.steps)
        b.set_active(i, True)
        return job, r

    def _advance(self, running: dict):
        """One epoch on every pool with a running job (concurrently), then each pool's force
        evaluation at the new positions."""
        busy = sorted({self.slot_at[sid][0] for sid in running})

        def one(pid):
            b = self.pools[pid].batch
            b.step(self.epoch)
            b.evaluate()

        if len(busy) == 1:
            one(busy[0])
        else:
            for f in [self._exec.submit(one, pid) for pid in busy]:
                f.result()
        for pid, p in self.pools.items():
            p.idle = 0 if pid in busy else p.idle + 1

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
            if grid_edge(j.system) not in self.edges:
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
            blocked = set()                   # shapes the budget cannot grow this round
            demand = collections.Counter(edge_of(it) for it in queue)
            queued, shapes_waiting = len(queue), len(demand)
            for item in queue:
                g = edge_of(item)
                if not self.free[g] and self.grow and g not in blocked and \
                        not self._try_grow(g, running, self._pool_size(demand[g], queued, shapes_waiting)):
                    blocked.add(g)
                demand[g] -= 1
                queued -= 1
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
            before = {}
            for slot in running:
                b, i = self._b(slot)
                before[slot] = b.step_count(i)
            # records describe each job's state after the epoch (stopped jobs: their last step)
            self._advance(running)
            self.stepping_s += time.perf_counter() - ts0
            self.epochs_run += 1
            epoch_no += 1
            waiting_edges = collections.Counter(edge_of(it) for it in queue)
            for slot in list(running):
                job, r, ran = running[slot]
                b, i = self._b(slot)
                ran += 1
                running[slot][2] = ran
                o = b.observables(i)
                step_now = b.step_count(i)
                self.work_done += (step_now - before[slot]) * job.system.ns
                r.energy.append((step_now, o["upe"]))
                b.sk_accumulate(i, 0, job.sk_type)
                if not b.active(i):
                    sk, n = b.sk_get(i, 0)
                    parts = sk_parts.pop(job.job_id, []) + [(sk * n, n)]
                    r.sk_calls = sum(k for _, k in parts)
                    r.sk = sum(v for v, _ in parts) / r.sk_calls
                    if self.keep_positions:
                        r.x = b.get_state(i)[0]
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
            # grown pools with nothing to run for a while give their memory back
            if self.grow:
                busy = {self.slot_at[sid][0] for sid in running}
                for p in list(self.pools.values()):
                    if p.grown and p.pid not in busy and p.idle >= self.idle_epochs:
                        self._release(p)
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
