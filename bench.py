"""Benchmark of the B200 TILD hot path: particle-steps/s on one system per GPU.

Workload (default, --workload blend): A/B homopolymer blend, 130,000 chains x N=20 = 2.6M beads,
box 64^3, grid 128^3, three gaussian_erf pair styles (R_p = 0.5, smearing 0.5, kappa = 50,
chi = 0.2), 4th-order assignment (64-point stencil), GJF, dt = 0.005, seeded synthetic chains.
A "step" is one full TILD step: spread, R2C, k-space multiply, C2R, gather + bonds + GJF.
Other workloads: diblock (40k beads, 40^3), coacervate (220k, 96^3, charges, EM), ensemble
(256 systems batched), serving (Poisson job stream), blend_half (the blend at half the volume,
for multi-pass profiler captures).

Arms:
  --impl ours       (default) libtild through its C ABI.  value: device-timed (CUDA events on
                    the context stream) K steps with the state resident in HBM; e2e: the same K
                    steps through the public API from page-locked host buffers (initial state
                    uploaded, an observable record read back every 128 steps, final positions
                    read back).
  --impl reference  the reference algorithm on the host cores: the FP64 oracle port
                    (oracle/tild_oracle.c, OpenMP over all host threads) on a bounded sample of
                    the same workload.  When the reference's own CUDA build is present
                    (oracle/_ref/gpu-tild) its particle-steps/s on this GPU is added as
                    "reference_cuda".
The default line (workload blend) also carries, as extra keys on their own configurations:
  "ensemble": the 256-system batch (K steps, autotuned schedule) against the same systems run
              one at a time through libtild and through the reference build, with its roofline;
  "serving":  the Poisson stream of ensemble-distributed jobs at 50 jobs/s (overloaded: it offers
              more particle-steps than one B200 sustains) and at a rate below capacity, with p50/p99
              job latency, aggregate particle-steps/s and the ratio to the jobs run alone.
--no-extras leaves them out.  Exactly K = --steps steps are timed: whole CUDA-graph periods
plus direct launches for any remainder.
Multi-GPU (torchrun, N > 1): one independent replica per GPU (systems do not exchange
anything), timing = max over ranks, value = total particle-steps of all ranks / that time.
"""
from __future__ import annotations

import argparse
import collections
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "gpu-tild_b200")]

import numpy as np  # noqa: E402

import tild  # noqa: E402
import tild_dist  # noqa: E402
import tild_systems as ts  # noqa: E402

PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
C_SIZEOF_OBS = __import__("ctypes").sizeof(tild.Obs)


def graph_period(tune) -> int:
    """Steps per captured CUDA graph: two sort periods (32 when the sort is off)."""
    return 2 * tune.sort_interval if tune.sort_interval > 0 else 32


def warm_and_prime(obj, warmup: int, steps: int, period: int):
    """Warm-up in whole graph periods, then one untimed run of `steps` steps (its CUDA graphs are
    captured) and the steps to the next period boundary, so the timed run of `steps` steps starts
    from the same configuration and replays those graphs.  obj starts at a period boundary
    (fresh, or just tuned: the tuner restores the state)."""
    obj.step(period * max(1, -(-warmup // period)))
    obj.step(steps)
    pad = (period - steps % period) % period
    if pad:
        obj.step(pad)
    obj.sync()


def nvtx_range(name: str):
    """An NVTX range around a timed region, so a profiler can select exactly its launches."""
    try:
        import torch
        return torch.cuda.nvtx.range(name)
    except Exception:
        import contextlib
        return contextlib.nullcontext()


def ensemble(n: int = 256):
    return [ts.ensemble_member(i) for i in range(n)]


def apply_schedule(engine, spec: str) -> dict:
    """Sets the tild.Tune fields given as JSON on a context or batch (instead of the autotuner)."""
    t = engine.get_tune()
    for k, v in json.loads(spec).items():
        if k not in dict(tild.Tune._fields_):
            raise SystemExit(f"--schedule: unknown field {k}")
        setattr(t, k, v)
    engine.set_tune(t)
    return engine.get_tune().as_dict()


def ensemble_leg(grp, args) -> dict:
    """Batched ensemble: 256 independent diblock systems (box L ~ U(12, 24) snapped to dx = 0.5,
    grids 24^3..48^3, N ~ U{10..40}, f_A ~ U(0.3, 0.7), chi N ~ U(10, 30), rho0 = 5) advanced
    together for exactly args.steps steps, against the same systems run one at a time (a sample
    of them, scaled by bead counts), through libtild and through the reference build."""
    systems = ensemble(args.nsys)
    mine = tild_dist.shard([s.ns for s in systems], grp.rank, grp.world)
    local = [systems[i] for i in mine]
    B = tild.Batch(local, device=grp.local)
    schedule = apply_schedule(B, args.schedule) if args.schedule else (None if args.no_tune else B.autotune(trial_steps=64))
    steps = args.steps
    warm_and_prime(B, args.warmup, steps, graph_period(B.get_tune()))
    grp.barrier()
    with ClockSampler(grp.local) as clk, nvtx_range("timed_ensemble"):
        ms = B.time_steps(steps)
    ms = grp.max(ms)
    tot = grp.sum(sum(s.ns for s in local)) * steps
    value = tot / (ms / 1e3)
    prof = B.profile_steps(steps)
    B.close()
    Sall = ensemble_bytes(systems)
    dom = max(prof, key=lambda k: prof[k])
    peak, peak_kind = hbm_peak()
    out = {"value": value, "unit": "particle-steps/s", "steps": steps, "ms_per_step": ms / steps,
           "config": {"workload": f"ensemble_{args.nsys}_diblock_24^3-48^3_gaussian_p1_GJF",
                      "systems": args.nsys, "beads_total": sum(s.ns for s in systems),
                      "grid_points_total": int(sum(np.prod(s.nx) for s in systems)), "parallelism": f"shards{grp.world}",
                      "schedule": schedule},
           "clocks": clk.summary(), "stages_ms_per_step": {k: v / steps for k, v in prof.items()},
           "roofline": {"bound": "hbm", "kernel": dom, "achieved": Sall[dom] / (prof[dom] / steps / 1e3) / 1e9
                        if prof[dom] > 0 else 0.0, "peak": peak, "unit": "GB/s",
                        "frac": Sall[dom] / (prof[dom] / steps / 1e3) / 1e9 / peak if prof[dom] > 0 else 0.0,
                        "peak_source": peak_kind, "algorithmic_bytes_per_launch": Sall[dom]},
           "step_roofline": {"algorithmic_bytes_per_step": Sall["step"],
                             "frac": Sall["step"] / (ms / steps / 1e3) / 1e9 / peak}}
    if grp.rank == 0 and not args.no_serial:
        # one at a time: every 16th system alone, scaled to all systems by their bead counts
        sample = list(range(0, args.nsys, 16))
        t_serial, ns_sample = 0.0, 0
        for i in sample:
            s = systems[i]
            with tild.Context(s, device=grp.local) as c:
                warm_and_prime(c, args.warmup, steps, graph_period(c.get_tune()))
                t_serial += c.time_steps(steps) / 1e3
                ns_sample += s.ns
        serial_value = ns_sample * steps / t_serial
        out["serial"] = {"value": serial_value, "unit": "particle-steps/s",
                         "sample": f"{len(sample)} of {args.nsys} systems, each alone for {steps} steps"}
        out["batched_over_serial"] = value / serial_value
        if not args.no_reference_cuda:
            # the reference's own build, one system per process as it runs them
            ref_sample = sample[::4]
            t_ref, ns_ref = 0.0, 0
            for i in ref_sample:
                r = reference_cuda(systems[i], "ensemble_member", runs=1, target_s=0.5)
                if r is None or "unavailable" in r:
                    t_ref = None
                    break
                t_ref += r["ms_per_step"] / 1e3
                ns_ref += systems[i].ns
            if t_ref:
                ref_value = ns_ref / t_ref
                out["reference_cuda_serial"] = {
                    "value": ref_value, "unit": "particle-steps/s",
                    "sample": f"{len(ref_sample)} of {args.nsys} systems, each a separate run of the reference build "
                              "(its step loop timed inside the harness)"}
                out["batched_over_reference_serial"] = value / ref_value
    return out


def ensemble_bytes(systems) -> dict:
    """Algorithmic bytes of one launch of each stage over all systems, and of one whole step."""
    tot = collections.Counter()
    for s in systems:
        tot.update(stage_bytes(s))
        tot["step"] += step_bytes(s)
    return dict(tot)


def run_ensemble(args):
    grp = tild_dist.Group(backend="nccl")
    leg = ensemble_leg(grp, args)
    grp.close()
    if grp.rank == 0:
        out = {"metric": "particle-steps/s", "value": leg["value"], "unit": "particle-steps/s", "n_gpus": grp.world,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": leg["ms_per_step"], "higher_is_better": True,
               "scaling": "weak" if grp.world == 1 else "strong", "vs_baseline": None, "dtype": "f32",
               "data": "synthetic (seeded random-walk chains)"}
        out.update({k: v for k, v in leg.items() if k not in out})
        print(json.dumps(out))


def serving_leg(grp, args, rate: float, njobs: int, serial: bool = True, slots_per_edge: int = None) -> dict:
    """Serving: a seeded Poisson stream (mean `rate` jobs/s) of `njobs` jobs drawn from the
    batched-ensemble distribution, each --job-steps steps returning its energy trace and avg_sk,
    served by continuous batching over slot pools: --slots-per-edge initial slots for each grid
    edge 24..48 (12 for the 50 jobs/s stream, none for the stream below capacity) and pools grown
    on demand inside the HBM budget (one slot per queued job of a grid shape, up to
    --group-slots per pool).  value: aggregate particle-steps/s
    of all jobs over the span from the first arrival to the last completion; latency percentiles
    are arrival -> results on the host.  Against: the same jobs run one at a time alone (a sample
    of them, each for all its steps, set-up included)."""
    import tild_serve as sv
    jobs_all = sv.poisson_jobs(njobs, rate, steps=args.job_steps)
    mine = [j for k, j in enumerate(jobs_all) if k % grp.world == grp.rank]
    # each rank replays its share of the stream: arrivals keep their absolute times
    spe = args.slots_per_edge if slots_per_edge is None else slots_per_edge
    edges = {g: spe for g in ts.ensemble_grid_edges()}
    with sv.Server(edges, device=grp.local, hbm_budget=args.hbm_budget, epoch=args.epoch, tune=not args.no_tune,
                   grow=not args.no_grow, group_slots=args.group_slots,
                   grow_policy=getattr(args, "grow_policy", "demand")) as srv:
        pool0, nslots, schedule = srv.pool_bytes, srv.nslots, srv.schedule
        grp.barrier()
        res = srv.run(mine, clock="wall")
        stepping_s, work_stepping = srv.stepping_s, srv.work_done
        grown, peak_bytes = srv.pools_grown, srv.peak_bytes
    rows = grp.gather_lists([(r.job_id, r.ns, r.steps, r.arrival, r.admitted, r.finished) for r in res])
    rows.sort()
    results = [sv.JobResult(j, ns, 0, st, a, admitted=ad, finished=f) for j, ns, st, a, ad, f in rows]
    summ = sv.latency_summary(results)
    work = sum(r.ns * r.steps for r in results)
    offered = rate * work / len(results)
    out = {"metric": "particle-steps/s (aggregate, served jobs); p50/p99 job latency",
           "value": summ["aggregate_particle_steps_per_s"], "unit": "particle-steps/s",
           "config": {"workload": f"serving_poisson{rate:g}_{njobs}jobs_{args.job_steps}steps",
                      "initial_slots": nslots * grp.world, "slots_per_edge": spe,
                      "grown_pools_rank0": grown, "group_slots": args.group_slots, "epoch_steps": args.epoch,
                      "hbm_budget_gb": args.hbm_budget / 1e9, "initial_pool_gb_per_gpu": pool0 / 1e9,
                      "peak_pool_gb_rank0": peak_bytes / 1e9, "schedule": schedule,
                      "parallelism": f"replicas{grp.world}"},
           "latency": summ,
           "offered_particle_steps_per_s": offered,
           "stepping_fraction_rank0": stepping_s / summ["span_s"] if summ["span_s"] > 0 else None,
           "stepping_throughput_rank0": {
               "value": work_stepping / stepping_s if stepping_s > 0 else None, "unit": "particle-steps/s",
               "note": "particle-steps the jobs advanced / wall time of the stepping calls: the batched engine's rate "
                       "inside the request loop; the aggregate value also spans the stream's ramp-up and drain"}}
    if grp.rank == 0 and serial and not args.no_serial:
        sample = jobs_all[:: max(1, len(jobs_all) // args.serial_sample)][:args.serial_sample]
        t_serial, w_serial, lat = 0.0, 0, []
        for j in sample:
            t0 = time.perf_counter()
            with tild.Context(j.system, device=grp.local) as c:
                c.step(j.steps)
                c.observables()
                c.sync()
            dt = time.perf_counter() - t0
            t_serial += dt
            lat.append(dt)
            w_serial += j.system.ns * j.steps
        out["serial"] = {"value": w_serial / t_serial, "unit": "particle-steps/s",
                         "job_time_s_mean": float(np.mean(lat)),
                         "sample": f"{len(sample)} of {len(jobs_all)} jobs, each alone for all its steps "
                                   "(set-up included)"}
        out["served_over_serial"] = out["value"] / out["serial"]["value"]
    return out


def run_serving(args):
    grp = tild_dist.Group(backend="nccl")
    leg = serving_leg(grp, args, args.rate, args.jobs)
    grp.close()
    if grp.rank == 0:
        out = {"metric": leg["metric"], "value": leg["value"], "unit": "particle-steps/s", "n_gpus": grp.world,
               "steps": args.job_steps, "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "f32", "data": "synthetic (seeded random-walk chains, seeded Poisson arrivals)"}
        out.update({k: v for k, v in leg.items() if k not in out})
        print(json.dumps(out))


def make_system(workload: str):
    if workload == "blend":
        return ts.homopolymer_blend(), "blend_2.6M_128^3_gaussian_erf_p3_GJF"
    if workload == "blend_half":  # half the blend (same density and stencil) for multi-pass ncu captures
        return (ts.homopolymer_blend(n_chains=65000, box=(64.0, 64.0, 32.0), nx=(128, 128, 64)),
                "blend_1.3M_128x128x64_gaussian_erf_p3_GJF")
    if workload == "diblock":
        return ts.diblock_melt(), "diblock_40k_40^3_gaussian_p1_GJF"
    if workload == "coacervate":
        return ts.coacervate(), "coacervate_220k_96^3_charges_gaussian_p1_EM"
    raise SystemExit(f"unknown workload {workload}")


# ------------------------------------------------------------------------------------------
# algorithmic bytes per launch of each stage (the roofline numerators)
# ------------------------------------------------------------------------------------------
def stage_bytes(s) -> dict:
    """Compulsory HBM bytes of one launch of each stage's kernel, each array touched once."""
    ns, D, T = s.ns, s.dim, s.ntypes
    C = 1 if s.charges is not None else 0
    M = int(np.prod(s.nx[:D]))
    Mh = M // s.nx[0] * (s.nx[0] // 2 + 1)
    nfft = sum(1 for st in s.styles if st.kind != tild.STYLE_FIELDPHASE)
    gjf = any(k == tild.INTEGRATOR_GJF for k, _ in s.integrators)
    # x_n (16), bead id, bond info, partners (4 + 4 + 12), x_{n-1} read and x_{n+1} write (32),
    # GJF noise read and write (24), charge (4)
    per_bead_gather = 16 + 20 + 32 + (24 if gjf else 0) + 4 * C
    return {
        "sort": 0,
        "fix2float": (T + C) * M * (8 + 4 + 8),            # read u64, write f32, clear u64
        "spread": ns * (16 + 4 * C) + (T + C) * M * 16,     # positions; u64 accumulator RMW
        "r2c": (T + C) * (M * 4 + Mh * 8),
        "kmul": (T + C) * Mh * 8 + nfft * Mh * 4 + C * Mh * 4 + (T + C) * D * Mh * 8,
        "c2r": (T + C) * D * (Mh * 8 + M * 4),
        "fieldphase": 0,
        "interleave": (T + C) * M * (D * 4 + 16),
        "gather": ns * per_bead_gather + (T + C) * M * 16,  # every float4 field node read once
        "step_tail": 0,
    }


def step_bytes(s) -> int:
    """Compulsory bytes of one whole step of a fused design: ns * b_p + M * 48 * channels, with
    b_p = 104 B per bead for GJF (64 for EM, +4 with charges)."""
    D = s.dim
    M = int(np.prod(s.nx[:D]))
    C = 1 if s.charges is not None else 0
    gjf = any(k == tild.INTEGRATOR_GJF for k, _ in s.integrators)
    bp = (104 if gjf else 64) + 4 * C
    return s.ns * bp + M * 48 * (s.ntypes + C)


# dram__bytes_read.sum + dram__bytes_write.sum of one launch of the stage's kernel on this
# workload: one ncu capture of k_gather<3,3,GJF> and k_spread_tiled<3,3> on the half-size blend
# (--workload blend_half with the blend's tuned schedule given by --schedule, one launch each
# inside the timed region), doubled: the full blend has twice the beads and twice the grid
# points, and both kernels' traffic grows in proportion.
NCU_DRAM_BYTES_PER_LAUNCH = {
    "blend_2.6M_128^3_gaussian_erf_p3_GJF": {"gather": 2 * (119597824 + 15529216), "spread": 2 * (37655040 + 9216)},
}


def hbm_peak():
    try:
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.out = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        return self

    def __exit__(self, *a):
        if self.proc:
            # a timed region shorter than nvidia-smi's start-up has no sample yet: wait for the
            # first one (at most 2 s), taken just after the region with the GPU still at its clocks
            t0 = time.time()
            while time.time() - t0 < 2.0 and self.out.tell() == 0 and self.proc.poll() is None:
                time.sleep(0.02)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.out:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.out.seek(0)
        rows = [r.split(",") for r in self.out.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[0]))
                mx.append(float(r[1]))
                for k, v in zip(names, r[3:7]):
                    if v.strip() == "Active":
                        reasons.add(k)
            except (ValueError, IndexError):
                continue
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------------------------------
def run_ours(args):
    grp = tild_dist.Group(backend="nccl")
    rank, local, ws = grp.rank, grp.local, grp.world
    s, wname = make_system(args.workload)
    ctx = tild.Context(s, device=local)
    if args.schedule:  # a fixed schedule (profiling runs): no autotuner trials before the timed region
        schedule = apply_schedule(ctx, args.schedule)
    else:
        schedule = None if args.no_tune else ctx.autotune(trial_steps=64)
    period = graph_period(ctx.get_tune())
    warm_and_prime(ctx, args.warmup, args.steps, period)
    grp.barrier()
    with ClockSampler(local) as clk, nvtx_range("timed"):
        l0 = ctx.kernel_launches()
        ms = ctx.time_steps(args.steps)
        launches = ctx.kernel_launches() - l0
    ms = grp.max(ms)
    clocks = clk.summary()
    per_rank = s.ns * args.steps
    value = per_rank * ws / (ms / 1e3)

    # per-stage times over the same number of steps -> roofline of the dominant kernel
    prof = ctx.profile_steps(args.steps)
    sb = stage_bytes(s)
    dom = max(prof, key=lambda k: prof[k])
    dom_ms = prof[dom] / args.steps
    peak, peak_kind = hbm_peak()
    achieved = sb[dom] / (dom_ms / 1e3) / 1e9 if dom_ms > 0 else 0.0

    # end to end through the public API from host buffers
    e2e_steps = args.steps
    log_freq = 128                      # observables every 128 steps (a whole number of graph periods)
    x_in = tild.HostArray((s.ns, s.dim))   # page-locked host buffers, filled/allocated before timing
    x_in.array[:] = s.x
    x_out = tild.HostArray((s.ns, s.dim))
    def e2e_run():
        ctx.set_state(x_in.array)
        done, reads, ticket = 0, 0, None
        while done < e2e_steps:
            n = min(log_freq, e2e_steps - done)
            ctx.step(n)
            done += n
            if done == e2e_steps:   # final positions to the host, copied while the last record is computed
                ticket = ctx.snapshot_async(x_out.array, None)
            if done % log_freq == 0 or done == e2e_steps:   # a record every 128 steps and at the end
                ctx.observables()
                reads += 1
        ctx.snapshot_wait(ticket)
        return reads

    # one untimed rehearsal: the first observables call allocates the reduction scratch, the first
    # snapshot its device buffers and copy stream, and the run's CUDA graphs are captured
    e2e_run()
    ctx.sync()
    runs_s = []
    for _ in range(3):  # three whole runs (the host side of a short run varies by a few ms): the median
        grp.barrier()
        t0 = time.perf_counter()
        obs_reads = e2e_run()
        runs_s.append(grp.max(time.perf_counter() - t0))
    e2e_s = sorted(runs_s)[1]
    obs_bytes = C_SIZEOF_OBS
    h2d = s.ns * s.dim * 4
    d2h = s.ns * s.dim * 4 + obs_reads * obs_bytes
    e2e = {"value": per_rank * ws / e2e_s, "unit": "particle-steps/s",
           "h2d_bytes_per_step": h2d / e2e_steps, "d2h_bytes_per_step": d2h / e2e_steps,
           "runs_ms": [round(r * 1e3, 3) for r in runs_s],
           "note": "public C ABI from page-locked host arrays: upload positions, K steps, an FP64 observables "
                   "record every 128 steps and after the last step, download positions; median of 3 runs"}

    out = {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded random-walk chains)",
        "config": {"workload": wname, "ns_per_gpu": s.ns, "grid": list(s.nx[:s.dim]), "pmeorder": s.pmeorder,
                   "pair_styles": len(s.styles), "integrator": "GJF" if s.integrators[0][0] else "EM",
                   "parallelism": f"replicas{ws}", "schedule": schedule,
                   "l2": "per-step working set (positions, grids, spectra) exceeds the 126 MB L2"},
        "clocks": clocks,
        "e2e": e2e,
        "gpu_launches": int(launches),
        "stages_ms_per_step": {k: v / args.steps for k, v in prof.items()},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": f"{peak_kind} ({'MEASURED_PEAKS.json' if peak_kind == 'measured' else 'fallback'})",
                     "algorithmic_bytes_per_launch": sb[dom],
                     "traffic": NCU_DRAM_BYTES_PER_LAUNCH.get(wname, {}).get(dom)},
        "step_roofline": {"algorithmic_bytes_per_step": step_bytes(s),
                          "achieved": step_bytes(s) * args.steps / (ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                          "frac": step_bytes(s) * args.steps / (ms / 1e3) / 1e9 / peak},
    }
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(s, args)
    ctx.close()
    if args.workload == "blend" and not args.no_extras:
        out["ensemble"] = ensemble_leg(grp, args)
        # each stream with the pool policy that suits its load: an overloaded stream keeps one
        # large batched pool busy (plus growth), a stream below capacity is served fastest by
        # pools grown per queued job
        out["serving"] = [serving_leg(grp, args, 50.0, args.jobs),
                          serving_leg(grp, args, args.subsat_rate, args.subsat_jobs, serial=False,
                                      slots_per_edge=args.subsat_slots_per_edge)]
        if rank == 0 and "serial" in out["serving"][0]:
            out["serving"][1]["served_over_serial"] = out["serving"][1]["value"] / out["serving"][0]["serial"]["value"]
    grp.close()
    if rank == 0:
        print(json.dumps(out))


def cpu_baseline(s, args, target_s: float = 20.0):
    """FP64 oracle on the host cores: whole steps of the same system, as many as fit ~target_s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    o = oracle.Oracle(s)
    cores = oracle.max_threads()
    x, xo, nz = s.x.copy(), s.x.copy(), np.zeros_like(s.x)
    t0 = time.perf_counter()
    o.step(x, xo, nz, 1, True)
    t1 = time.perf_counter() - t0
    k = max(1, min(int(target_s / max(t1, 1e-3)), 50))
    t0 = time.perf_counter()
    for i in range(k):
        o.step(x, xo, nz, 2 + i, True)
    dt = time.perf_counter() - t0
    o.close()
    return {"value": s.ns * k / dt, "unit": "particle-steps/s", "cores": cores, "kind": "port",
            "sample": f"{k} full steps of the same {s.ns}-bead system after 1 untimed step "
                      f"(oracle/tild_oracle.c, FP64, OpenMP {cores} threads)"}


def reference_cuda(s, wname, runs: int = 3, target_s: float = 2.0):
    """The reference's own CUDA build on this GPU: oracle/_ref/ref_harness (the unmodified reference
    objects with a main that runs the reference's step loop, forces(); Integrate_2();
    update_pairstyles(), output off, main.cu:104-201) times N steps with the device synchronised
    on both sides after 10 untimed steps.  N is sized to about target_s seconds at a first
    estimate; `runs` runs of the program, median reported with every run's value."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(exe):
        return None
    per = []
    with tempfile.TemporaryDirectory() as td:
        ts.write_data_file(os.path.join(td, "input.data"), s)
        ts.write_input_script(os.path.join(td, "input"), s, max_steps=10 ** 6, log_freq=10 ** 8, binary_freq=0)
        n = 20
        for k in range(runs + 1):   # the first run sizes N
            r = subprocess.run([exe, "-in", "input", "-out", "t", "-steps", str(n), "-time", "10"], cwd=td,
                               stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, timeout=900)
            line = [l for l in r.stdout.splitlines() if l.startswith("harness timing:")]
            if r.returncode != 0 or not line:
                return {"unavailable": f"reference harness exited {r.returncode}"}
            ms = float(line[0].split()[4])
            if k == 0:
                n = int(min(20000, max(50, target_s * 1e3 / max(ms, 1e-3))))
            else:
                per.append(ms)
    per_step = float(np.median(per)) / 1e3
    return {"value": s.ns / per_step, "unit": "particle-steps/s", "ms_per_step": per_step * 1e3,
            "ms_per_step_runs": per, "steps_timed": n,
            "binary": "oracle/_ref/ref_harness (unmodified reference objects, nvcc -arch=sm_100a -O3, and a main "
                      "that times the reference's step loop)",
            "method": f"median over {runs} runs of {n} timed steps after 10 untimed ones, device synchronised on both "
                      "sides"}


def run_reference(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if ws > 1 and rank != 0:
        return
    s, wname = make_system(args.workload)
    cb = cpu_baseline(s, args, target_s=min(60.0, 4.0 * max(args.steps, 1)))
    out = {"impl": "reference", "metric": "particle-steps/s", "value": cb["value"], "unit": "particle-steps/s",
           "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded random-walk chains)",
           "config": {"workload": wname, "ns_per_gpu": s.ns, "grid": list(s.nx[:s.dim])},
           "cpu_baseline": cb,
           "e2e": {"value": cb["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    if not args.no_reference_cuda:
        rc = reference_cuda(s, wname)
        if rc is not None:
            out["reference_cuda"] = rc
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="blend", choices=["blend", "blend_half", "diblock", "coacervate", "ensemble", "serving"])
    ap.add_argument("--nsys", type=int, default=256)
    ap.add_argument("--jobs", type=int, default=300, help="serving: number of jobs in the stream")
    ap.add_argument("--rate", type=float, default=50.0, help="serving: mean arrivals per second")
    ap.add_argument("--job-steps", type=int, default=5000)
    ap.add_argument("--slots-per-edge", type=int, default=12,
                    help="serving: initial slots per grid edge (0: every slot grown on demand)")
    ap.add_argument("--subsat-slots-per-edge", type=int, default=0,
                    help="serving: initial slots per grid edge of the below-capacity stream")
    ap.add_argument("--group-slots", type=int, default=8,
                    help="serving: largest pool grown on demand (one slot per queued job of the shape)")
    ap.add_argument("--no-grow", action="store_true", help="serving: fixed slots only")
    ap.add_argument("--grow-policy", default="demand", choices=["demand", "load", "double"],
                    help="serving: slots of a grown pool (see tild_serve.Server)")
    ap.add_argument("--subsat-rate", type=float, default=4.0, help="serving: the below-capacity arrival rate")
    ap.add_argument("--subsat-jobs", type=int, default=40)
    ap.add_argument("--no-extras", action="store_true", help="blend line only (no ensemble and serving legs)")
    ap.add_argument("--epoch", type=int, default=128)
    ap.add_argument("--hbm-budget", type=float, default=80e9)
    ap.add_argument("--serial-sample", type=int, default=6)
    ap.add_argument("--no-tune", action="store_true", help="skip the schedule autotuner")
    ap.add_argument("--schedule", default="",
                    help='fixed schedule instead of the autotuner, as JSON of tild.Tune fields '
                         '(e.g. \'{"field_layout": 1, "spread_cap": 6144}\')')
    ap.add_argument("--no-serial", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-cuda", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "ensemble":
        run_ensemble(args)
    elif args.workload == "serving":
        run_serving(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
