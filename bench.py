"""Benchmark of the RealQM solver step on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload glycine128]
                    [--leg molecule_js_lobpcg|mol_fast_ch4|realqm_rb_h2]

Metric: grid-point updates per second (Gpt-updates/s): one update = one imaginary-time
update of psi at one interior voxel; one solver step updates (NN-1)^3 voxels.

A bench *step* is one schedule period of the solver.py flavour (100 solver steps: the
Poisson step every 2, normalisation every 20, labels every 100; cloud/solver.py:561-586)
on the glycine workload (10 atoms, 40 electrons, 128^3, h = 0.2 bohr, all-electron
reference idiom, seeded random rotation), run as one CUDA-graph replay -- the product path.
L2 is flushed (a 256 MB write, not timed) before every timed period.  The 129^3 fields
(~60 MB) fit in the 126 MB L2, so inside a period later steps find their inputs in L2, as
they do in a real run at this size; ``value_l2_flushed_every_solver_step`` repeats one
period with the flush before EVERY solver step (every kernel reads HBM cold).

``value``  device-resident throughput (state already in HBM);
``e2e``    the public API call a user makes per frame: upload the state (psi, labels, P)
           from pinned host memory, run one period (CUDA-graph replay), read the energies
           back -- copies inside the timed region;
``roofline`` the dominant kernel (k_step_sp: the ITP update and one Jacobi sweep in one pass,
           24 algorithmic B per interior point) against the measured HBM copy bandwidth;
``cpu_baseline`` the reference's own cloud/solver.py kernels compiled for the host
           (oracle/_ref, OpenMP over all host cores) on a bounded sample of the same workload.

``converge`` the second half of the metric, seconds to converge with the new flavour: glycine
           (40 electrons, 128^3) as one context in mixed precision and in FP64, and the 96 water
           clusters (1-12 waters, 64^3-128^3) as one mixed-precision batch against the plain FP64 path
           (one FP64 context per instance, one after another).  Converged: |dE| < 1e-9 Ha on 3
           consecutive checks 100 steps apart, which keeps every solve within 1e-6 Ha of its fixed
           point (the energy readout is P-stationary and, for fp32 fields, uses the FP64 nuclear
           potential, so the mixed path converges to the FP64 answer without an FP64 phase).
           ``max_abs_dE_Ha`` compares the mixed and FP64 answers; ``forces`` the mixed and FP64
           forces.  Times are CUDA events around initialise + solve on the solver stream.
``batch_step`` the C3 batch step alone (all 96 clusters active, mixed precision): Gpt/s, launches
           per step and the composite HBM roofline of its kernels, before and after the autotuner.
``geometry`` the C4 / C5 geometry workloads for a few geometry steps each (100 waters, 192^3, FIRE,
           200 iterations per step; 1000 waters, 320^3, velocity Verlet, 50 iterations per step;
           mixed precision, adjoint forces): wall time per geometry step and its parts.

``callers`` the other reference callers of the step through their drop-ins, each beside its CPU
           restatement: the recorded hairpin job (RealQMSolver), atom.js's He page, mol_fast.js's
           CH4 page, realqm_rb.js's H2 page and molecule.js's LOBPCG frames (water, 64^3).
           ``--leg NAME`` runs one of mol_fast_ch4, realqm_rb_h2 or molecule_js_lobpcg alone.

``--impl reference`` times that reference CPU implementation alone (the reference has no
GPU path that can run here: its kernels need CuPy, which is not installed).
Multi-GPU (torchrun): every rank runs an independent replica of the period (one grid does not
shard); value = all ranks' updates / max-over-ranks time; scaling "weak".  The cluster batch of
``converge`` is partitioned over the ranks by cost (realmolecule_b200.shard), max over ranks:
strong scaling of a fixed set of 96 solves.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gpt-updates/s"
PERIOD = 100


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="glycine128")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-converge", action="store_true")
    ap.add_argument("--leg", default=None, choices=["molecule_js_lobpcg", "mol_fast_ch4", "realqm_rb_h2"],
                    help="run only this caller leg on one GPU and print its JSON (for profiling)")
    return ap.parse_args()


def workload_config(name):
    from realmolecule_b200 import configs
    if name == "hairpin":
        with open(os.path.join(ROOT, "tests", "golden", "hairpin_config.json")) as f:
            cfg = json.load(f)
        return {"gridN": cfg["gridN"], "screen": cfg["screen"], "atoms": cfg["atoms"]}, "hairpin 267 atoms 300^3"
    g = configs.WORKLOADS[name]()
    return configs.reference_config(g), f"{name}: {len(g.elements)} atoms, {int(g.charges.sum())} electrons, " \
                                         f"{g.NN}^3 at h={g.h} bohr (solver.py schedule)"


def interior(NN):
    return (NN - 1) ** 3


def bench_config(desc, world):
    """The workload description both arms print (identical, so the two lines compare)."""
    return {"workload": desc,
            "step": f"one schedule period = {PERIOD} solver steps (GPU arm: one CUDA-graph replay)",
            "l2": "GPU arm: flushed (256 MB write) before every timed period; flush not timed",
            "parallelism": f"replicas x{world}"}


# ---------------------------------------------------------------------------------------
# reference CPU implementation (oracle/_ref: the reference's kernel text compiled for the host)
# ---------------------------------------------------------------------------------------
def cpu_reference_rate(cfg, steps, warmup):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    threads = len(os.sched_getaffinity(0))
    os.environ["OMP_NUM_THREADS"] = str(threads)
    d = orc.SolverPyDriver(cfg, kernels="reference")
    d.initialize(bootstrap=2)
    d.run(warmup)
    t0 = time.perf_counter()
    d.run(steps)
    dt = time.perf_counter() - t0
    return interior(cfg["gridN"]) * steps / dt / 1e9, threads, dt


def run_reference_arm(a):
    cfg, desc = workload_config(a.workload)
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # each bench step is one schedule period (100 solver steps) of the same workload
    per = PERIOD
    rate, threads, dt = cpu_reference_rate(cfg, per * a.steps, per * a.warmup)
    line = {"metric": METRIC, "value": rate, "unit": "Gpt/s", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": dt / a.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": bench_config(desc, a.gpus),
            "cpu_baseline": {"value": rate, "unit": "Gpt/s", "cores": threads, "kind": "reference",
                             "sample": f"{per * a.steps} solver steps after {per * a.warmup} warm-up"},
            "e2e": {"value": rate, "unit": "Gpt/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------------------
class Clocks:
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "20"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.5)  # nvidia-smi is sampling before the timed region starts
        except Exception:
            self.p = None
        return self

    def __exit__(self, *exc):
        self.rows = []
        if self.p is None:
            return
        time.sleep(0.15)
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except Exception:
            self.p.kill()
            out = ""
        for ln in out.strip().splitlines():
            f = [x.strip() for x in ln.split(",")]
            if len(f) >= 8:
                self.rows.append(f)

    def summary(self):
        if not getattr(self, "rows", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in self.rows for q in range(4) if r[4 + q].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(workload):
    """DRAM bytes per launch of the fused step kernel on this workload, from the committed ncu
    summary (line "traffic_bytes_per_launch <workload>: <bytes>"), or None."""
    p = os.path.join(ROOT, "profiles", "step_sp_glycine128.md")
    key = f"traffic_bytes_per_launch {workload}:"
    try:
        with open(p) as f:
            for ln in f:
                if ln.startswith(key):
                    return float(ln.split(":")[1])
    except Exception:
        pass
    return None


# ---------------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------------
def run_ours(a):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from realmolecule_b200 import Context, _lib as L

    cfg, desc = workload_config(a.workload)
    NN = cfg["gridN"]
    # one dedicated stream for the solver, the L2 flush and the timing events
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = Context(NN, cfg["screen"], cfg["atoms"], flavor="solver.py")
    ctx.set_stream(stream.cuda_stream)
    ctx.initialize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # warm-up: W periods (captures the CUDA graphs of the period for both buffer parities)
    for _ in range(max(a.warmup, 2)):
        ctx.step(PERIOD)
    torch.cuda.synchronize()

    # ---- device-resident timing: K periods, each one CUDA-graph replay of 100 solver steps,
    #      L2 flushed before every period (flush not timed), CUDA events on the solver stream
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    l0 = ctx.kernel_launches
    barrier()
    with Clocks(local) as clk:
        for s in range(a.steps):
            flush.fill_(float(s))
            ev[s][0].record(stream)
            ctx.step(PERIOD)
            ev[s][1].record(stream)
        torch.cuda.synchronize()
    barrier()
    launches = ctx.kernel_launches - l0
    ms = sum(e0.elapsed_time(e1) for e0, e1 in ev)
    if dist:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    pts = interior(NN) * PERIOD * a.steps * world
    value = pts / (ms * 1e-3) / 1e9

    # ---- per-kernel CUDA events over one more period run the same way (eager launches,
    #      each kernel bracketed on the solver stream) -> roofline of the dominant kernel
    flush.fill_(-1.0)
    ctx.profile_begin()
    ctx.step(PERIOD)
    prof = ctx.profile_end()
    # and the same period with L2 flushed before every solver step (every kernel cold)
    cold_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(PERIOD)]
    for s in range(PERIOD):
        flush.fill_(float(s))
        cold_ev[s][0].record(stream)
        ctx.step(1)
        cold_ev[s][1].record(stream)
    torch.cuda.synchronize()
    cold_ms = sum(e0.elapsed_time(e1) for e0, e1 in cold_ev)
    value_cold = interior(NN) * PERIOD / (cold_ms * 1e-3) / 1e9

    # ---- end to end through the public API with pinned host buffers
    st = ctx.download(psi=True, label=True, P=True)
    S3 = ctx.S3
    pin = {k: torch.empty(S3, dtype=torch.float32 if k != "label" else torch.int32).pin_memory() for k in st}
    for k in st:
        pin[k].numpy()[:] = st[k]
    e2e_steps = max(1, a.steps)
    barrier()
    t_e0, t_e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(1):  # untimed pass so the graph for this parity exists
        ctx.upload(psi=pin["psi"].numpy(), label=pin["label"].numpy(), P=pin["P"].numpy())
        ctx.step(PERIOD)
        ctx.energy(per_domain=True)
    barrier()
    t_e0.record(stream)
    for _ in range(e2e_steps):
        ctx.upload(psi=pin["psi"].numpy(), label=pin["label"].numpy(), P=pin["P"].numpy())
        ctx.step(PERIOD)
        ctx.energy(per_domain=True)
    t_e1.record(stream)
    barrier()
    e2e_ms = t_e0.elapsed_time(t_e1)
    if dist:
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e = interior(NN) * PERIOD * e2e_steps * world / (e2e_ms * 1e-3) / 1e9
    h2d = S3 * 12
    d2h = ctx.n_atoms * L.DOMAIN_LEN * 8

    ctx.close()
    conv = None if a.no_converge else converge_leg(stream, dist, rank, world)
    batch = None if a.no_converge or rank != 0 else batch_leg(stream, measured_peak()[0])
    callers = None if a.no_converge or rank != 0 else caller_legs(a)
    geometry = None if a.no_converge or rank != 0 else geometry_leg()

    if rank == 0:
        peak, peak_kind = measured_peak()
        up = prof.get("update", {"ms": 0, "bytes": 0, "launches": 1})
        upd_bytes = up["bytes"] / max(1, up["launches"])
        upd_ms = amortised_update_ms(prof, ms / a.steps)
        achieved = upd_bytes / (upd_ms * 1e-3) / 1e9 if upd_ms > 0 else None
        period_bytes = sum(v["bytes"] for v in prof.values())
        hbm = hbm_leg(stream, peak)
        cpu = None
        if world == 1 and not a.no_cpu_baseline:
            try:
                nsteps = 40 * PERIOD
                rate, threads, dt = cpu_reference_rate(cfg, nsteps, 2)
                cpu = {"value": rate, "unit": "Gpt/s", "cores": threads, "kind": "reference",
                       "sample": f"{nsteps} solver steps of {a.workload} after 2 warm-up ({dt:.1f} s)"}
            except Exception as e:  # the reference build is missing: say so
                cpu = {"value": None, "unit": "Gpt/s", "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}
        line = {
            "metric": METRIC, "value": value, "unit": "Gpt/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(desc, world),
            "value_l2_flushed_every_solver_step": value_cold,
            "e2e": {"value": e2e, "unit": "Gpt/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if achieved else None, "traffic": ncu_traffic(a.workload),
                         "kernel": "k_step_sp (ITP update fused with a Jacobi sweep)", "bytes_per_launch": upd_bytes,
                         "peak_kind": peak_kind,
                         "duration": "in-graph: (timed period - the eager event time of every other kernel class) "
                                     "/ update launches, so launches x duration <= ms_per_step",
                         "us_per_launch_in_graph": upd_ms * 1e3,
                         "us_per_launch_eager_events": up["ms"] / max(1, up["launches"]) * 1e3,
                         "hbm_bound_320": hbm,
                         # every kernel of the period: its algorithmic bytes over the timed period time
                         "composite": {"achieved": period_bytes / (ms / a.steps * 1e-3) / 1e9,
                                       "frac": period_bytes / (ms / a.steps * 1e-3) / 1e9 / peak,
                                       "bytes_per_period": period_bytes}},
            "kernels": {k: {"launches": v["launches"], "ms": round(v["ms"], 4), "GB/s": round(v["gbs"], 1)}
                        for k, v in prof.items()},
            "cpu_baseline": cpu,
            "converge": conv,
            "batch_step": batch,
            "callers": callers,
            "geometry": geometry,
            "clocks": clk.summary(),
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def amortised_update_ms(prof, period_ms):
    """Duration of one update launch inside the replayed period: the period's time less the eager
    CUDA-event time of every other kernel class, over the update launches of the period."""
    up = prof.get("update")
    if not up or not up["launches"]:
        return 0.0
    other = sum(v["ms"] for k, v in prof.items() if k != "update")
    return max(period_ms - other, 1e-6) / up["launches"]


def hbm_leg(stream, peak):
    """The same solver.py step on a 320^3 grid (the 1000-water geometry, 3000 atoms, all-electron
    idiom): 33 M points per field, every pass streams HBM (the 128^3 fields fit the 126 MB L2)."""
    import torch
    from realmolecule_b200 import Context, configs
    g = configs.water1000()
    cfg = configs.reference_config(g)
    ctx = Context(g.NN, cfg["screen"], cfg["atoms"], flavor="solver.py")
    ctx.set_stream(stream.cuda_stream)
    ctx.initialize()
    for _ in range(2):
        ctx.step(PERIOD)
    periods = 5
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    ctx.step(PERIOD * periods)
    e1.record(stream)
    torch.cuda.synchronize()
    period_ms = e0.elapsed_time(e1) / periods
    ctx.profile_begin()
    ctx.step(PERIOD)
    prof = ctx.profile_end()
    ctx.close()
    up = prof["update"]
    b = up["bytes"] / up["launches"]
    t = amortised_update_ms(prof, period_ms)
    return {"workload": f"water1000 geometry, {len(cfg['atoms'])} atoms, {g.NN}^3 at h={g.h} (solver.py schedule)",
            "value_gpts": interior(g.NN) * PERIOD / (period_ms * 1e-3) / 1e9, "ms_per_period": period_ms,
            "achieved": b / (t * 1e-3) / 1e9, "frac": b / (t * 1e-3) / 1e9 / peak, "us_per_launch_in_graph": t * 1e3,
            "bytes_per_launch": b}


def nm_step_bytes(NN, es=4, pi=4, pre=1, post=1):
    """Algorithmic bytes per new-flavour step on one grid (the byte counts of nm_flavor.cu's launches):
    the update every step (psi, K, P, label read; psi written); every pi steps the materialised
    normalisation (psi, label read; psi written) and one V(pre, post) cycle (each red-black colour
    2.5 field values per point, the fused residual + full weighting 2 fine + 2 coarse (the coarse
    right-hand side and the cleared correction), the prolongation 2 fine + 1 coarse, the coarsest
    level 2 values per point)."""
    levels, nn = [NN], NN
    while nn % 2 == 0 and nn // 2 >= 6:
        nn //= 2
        levels.append(nn)
    n_in = [(x - 1) ** 3 for x in levels]
    s3 = [(x + 1) ** 3 for x in levels]
    v = 0.0
    for l in range(len(levels) - 1):
        v += (pre + post) * 2 * 2.5 * es * n_in[l] + 2 * es * (n_in[l] + n_in[l + 1])
        v += es * (2 * n_in[l] + n_in[l + 1])
    v += 2 * es * s3[-1]
    return (4 * es + 4) * n_in[0] + ((2 * es + 4) * s3[0] + v) / pi


def batch_leg(stream, peak):
    """The C3 batch step on its own: all 96 clusters active in one mixed-precision batch (a period
    per CUDA-graph replay), timed with CUDA events over 200 steps with the default configuration,
    then autotuned (march tile x launch form, smoother sweeps) and timed over 400 steps; composite
    roofline = the algorithmic bytes of every kernel of the step (nm_step_bytes, at the tuned
    sweeps) over the step time."""
    import torch
    from realmolecule_b200 import configs
    from realmolecule_b200.batch import Batch
    geoms = configs.clusters96()
    inst = [{"NN": x.NN, "screen": x.screen, "atoms": configs.to_domain_atoms(x)} for x in geoms]
    b = Batch(inst, precision="mixed", label_until=LABEL_UNTIL)
    b.set_stream(stream.cuda_stream)
    b.initialize()
    b.step(LABEL_UNTIL + 200)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed_steps(n):
        torch.cuda.synchronize()
        e0.record(stream)
        b.step(n)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n
    ms_default = timed_steps(200)
    tune = b.autotune()  # march tile x launch form, then smoother sweeps (their steps are steps of the run)
    b.step(200)          # capture the tuned periods
    n = 400
    l0 = b.info()["kernel_launches"]
    ms = timed_steps(n)
    info = b.info()
    b.close()
    cfg = tune["config"]
    byts = sum(nm_step_bytes(x.NN, pre=cfg.get("mg_pre", 1), post=cfg.get("mg_post", 1)) for x in geoms)
    byts_default = sum(nm_step_bytes(x.NN) for x in geoms)
    return {"instances": len(geoms), "interior_points": info["interior_points"], "ms_per_step": ms,
            "ms_per_step_default_config": ms_default,
            "frac_default_config": byts_default / (ms_default * 1e-3) / 1e9 / peak, "autotune": tune,
            "value_gpts": info["interior_points"] / (ms * 1e-3) / 1e9,
            "launches_per_step": (info["kernel_launches"] - l0) / n,
            "roofline": {"bound": "hbm", "bytes_per_step": byts, "achieved": byts / (ms * 1e-3) / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": byts / (ms * 1e-3) / 1e9 / peak,
                         "kernels": "update + normalisation + V(1,1) multigrid, composite"}}


# ---------------------------------------------------------------------------------------
# seconds to converge: mixed / batched against plain FP64 (new flavour)
# ---------------------------------------------------------------------------------------
# Convergence: |dE| < TOL on CHECKS consecutive checks CHECK steps apart (molecule.js counts 3 frames
# within CONVERGENCE_THRESHOLD, :4645-4659).  On these workloads |dE| < 1e-6 between checks stops up to
# 3e-4 Ha short of the fixed point: the ITP energy has plateaus (an electron crossing its domain to a
# lower well) that a loose threshold takes for convergence; 1e-9 on 3 checks stays within 1e-6 Ha.
TOL, CHECK, CHECKS, MAX_STEPS = 1e-9, 100, 3, 60000
LABEL_UNTIL = 1    # the level set moves the labels for the first LABEL_UNTIL steps, then they are frozen
ADJ_STEPS = 48     # warm-started steps of the adjoint comparison


def _timed(stream, fn):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    out = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1) * 1e-3


def _max_over_ranks(dist, x):
    if not dist:
        return x
    import torch
    t = torch.tensor([x], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def geometry_leg():
    """C4 and C5 for a few geometry steps each, through dynamics.geometry_model (each evaluation:
    the warm-started iterations recorded for the adjoint, the energy, the adjoint forces and the
    nuclear terms).  Synchronised wall clock per geometry step; per-class CUDA-event kernel times of
    one evaluation's parts."""
    import time
    from realmolecule_b200 import configs, dynamics, _lib as L
    out = {}
    for name, g, iters, pre, n in (("water100_fire", configs.water100(), 200, 2000, 4),
                                    ("water1000_verlet", configs.water1000(), 50, 3000, 3)):
        model, Z, off = dynamics.geometry_model(g, "mixed", iters, adjoint=True)
        model.ctx.step(pre)
        model.ctx.synchronize()
        parts = {}
        for part, fn in (("K", lambda: model.ctx.set_atoms(model._rows(g.xyz + off))),
                         ("iterations", lambda: model.ctx.step(iters)), ("energy", lambda: model.ctx.energy()),
                         ("adjoint_forces", lambda: model.ctx.forces(L.FORCE_ADJOINT))):
            model.ctx.profile_begin()
            fn()
            model.ctx.synchronize()
            parts[part] = round(sum(v["ms"] for v in model.ctx.profile_end().values()), 3)
        x0, m = g.xyz + off, dynamics.masses_for(Z)
        t0 = time.perf_counter()
        if name.endswith("fire"):
            tr = dynamics.fire(model, x0, max_steps=n, masses=m)
        else:
            tr = dynamics.velocity_verlet(model, x0, np.zeros_like(x0), m, 0.5 * dynamics.FS, n)
        dt = time.perf_counter() - t0
        out[name] = {"grid": f"{g.NN}^3", "nuclei": len(Z), "domains": len(g.seeds), "iterations_per_step": iters,
                     "geometry_steps": len(tr.energies), "ms_per_geometry_step": dt / len(tr.energies) * 1e3,
                     "kernel_ms_of_one_evaluation": parts, "E_first": tr.energies[0], "E_last": tr.energies[-1]}
        model.ctx.close()
    return out


def caller_legs(a):
    """The other reference callers of the step, timed through their drop-ins (rank 0, context only):
    the recorded hairpin job of cloud/run_hairpin.py through RealQMSolver (its A100 time per step is
    in cloud/hairpin_results.json) and atom.js's physicsStep on the He page (atom_He.html) against
    the sequential restatement on one host core."""
    import torch
    from realmolecule_b200 import RealQMSolver
    from realmolecule_b200.shells import AtomShells
    out = {}
    with open(os.path.join(ROOT, "tests", "golden", "hairpin_config.json")) as f:
        cfg = json.load(f)
    with open(os.path.join(ROOT, "tests", "golden", "hairpin_golden.json")) as f:
        gold = json.load(f)
    s = RealQMSolver(cfg)
    s.set_fold_atoms(cfg["fold_atoms"])
    s.initialize()
    s.run(total_steps=100, report_interval=100)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.run(total_steps=1000, report_interval=1000)
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) / 1000 * 1e3
    out["hairpin"] = {"atoms": len(cfg["atoms"]), "grid": f"{cfg['gridN']}^3", "steps": 1000,
                      "ms_per_step": ms, "recorded_a100_ms_per_step": gold["snapshots"][-1]["ms_per_step"],
                      "timing": "host wall clock around RealQMSolver.run (dynamics on, forces every 500 steps)"}
    he = [{"ne": 1, "Rmax": 5.0, "Zeff": 2, "split": "halfspace", "halfIndex": 0, "fixedW": True},
          {"ne": 1, "Rmax": 5.0, "Zeff": 2, "split": "halfspace", "halfIndex": 1, "fixedW": True}]
    sh = AtomShells(100, 5.0, 2, he, d=0.15)
    sh.step(2)
    t0 = time.perf_counter()
    sh.step(100)
    gpu_ms = (time.perf_counter() - t0) / 100 * 1e3
    sh.close()
    cpu_ms = None
    if not a.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        o = orc.AtomShellsDriver(100, 5.0, 2, he, d=0.15)
        o.initialize()
        t0 = time.perf_counter()
        o.step()
        o.step()
        cpu_ms = (time.perf_counter() - t0) / 2 * 1e3
    out["atom_js_he"] = {"grid": "100^3", "shells": 2, "ms_per_step": gpu_ms,
                         "cpu_sequential_ms_per_step": cpu_ms, "cpu_cores": 1,
                         "cpu": "the oracle's sequential restatement of atom.js (2 steps)"}
    out["mol_fast_ch4"] = mol_fast_leg(a)
    out["realqm_rb_h2"] = realqm_rb_leg(a)
    out["molecule_js_lobpcg"] = lobpcg_leg(a)
    return out


def lobpcg_leg(a):
    """molecule.js's LOBPCG frames (doLOBPCGStep, the page's 'L' solver) on the water molecule of the
    C1 geometry (O with a 0.4-bohr core at the centre, H at (+-1.4305, 1.1078, 0) bohr; 64^3,
    h = 0.25 bohr): frames from the third on replay one CUDA graph each; the oracle's restatement
    of the same frames on the host cores beside them."""
    import torch
    from realmolecule_b200 import Context
    rows = [{"i": 32, "j": 32, "k": 32, "Z": 6, "Z_nuc": 6, "rc": 0.4},
            {"i": 37, "j": 36, "k": 32, "Z": 1, "Z_nuc": 1, "rc": 0.0},
            {"i": 26, "j": 36, "k": 32, "Z": 1, "Z_nuc": 1, "rc": 0.0}]
    ctx = Context(64, 16.0, rows, flavor="molecule.js", steps_per_frame=10, lobpcg=1)
    ctx.initialize()
    ctx.step(2)  # frame 0 (no search direction yet) eagerly, frame 1 captured
    torch.cuda.synchronize()
    frames, l0 = 50, ctx.kernel_launches
    t0 = time.perf_counter()
    ctx.step(frames)
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) / frames * 1e3
    launches = (ctx.kernel_launches - l0) / frames
    ctx.close()
    out = {"grid": "64^3", "domains": 3, "iterations_per_domain": 10, "ms_per_frame": ms,
           "launches_per_frame": launches,
           "timing": "host wall clock around 50 frames (one CUDA-graph replay each, synchronised)"}
    if not a.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        ref = orc.MoleculeJsDriver(64, 16.0, rows, steps_per_frame=10, lobpcg=True)
        ref.initialize()
        ref.step()
        t0 = time.perf_counter()
        ref.step()
        ref.step()
        out.update({"cpu_ms_per_frame": (time.perf_counter() - t0) / 2 * 1e3,
                    "cpu_cores": len(os.sched_getaffinity(0)),
                    "cpu": "the oracle's restatement of the frame, OpenMP, 2 frames"})
    return out


def realqm_rb_leg(a):
    """realqm_rb.js's direct H2 page (NN = 100, 2 electrons, 10-step frames) through the drop-in
    RealqmRb, against the oracle's restatement (the reference's per-electron passes) on the host."""
    from realmolecule_b200 import configs
    from realmolecule_b200.realqm_rb import RealqmRb
    cfg = configs.realqm_rb_h2_page()
    g = RealqmRb(**cfg)
    g.doSteps(100)
    steps = 3000
    t0 = time.perf_counter()
    g.doSteps(steps)
    ms = (time.perf_counter() - t0) / steps * 1e3
    E = g.computeEnergy()["E_tot"]
    g.close()
    out = {"grid": f"{cfg['NN']}^3", "electrons_fields": 2, "ms_per_step": ms, "steps": steps, "E_tot": E,
           "timing": "host wall clock around doSteps(3000) (one CUDA graph, synchronised)"}
    if not a.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        ref = orc.RealqmRbDriver(cfg["nuclei"], NN=cfg["NN"], screen=cfg["screen"], norm_targets=cfg["norm_targets"])
        ref.initialize()
        t0 = time.perf_counter()
        ref.do_steps(20)
        out.update({"cpu_ms_per_step": (time.perf_counter() - t0) / 20 * 1e3, "cpu_cores": 1,
                    "cpu": "the oracle's sequential restatement of the passes (20 steps)"})
    return out


def mol_fast_leg(a):
    """mol_fast.js's CH4 page (NN = 200, 5 electrons, 500-step frames with forces and nuclear
    moves) through the drop-in MolFast, against the oracle's restatement on the host cores."""
    from realmolecule_b200 import configs
    from realmolecule_b200.mol_fast import MolFast
    cfg = configs.mol_fast_ch4_page()
    mf = MolFast(**cfg)
    mf.frame()
    frames = 3
    t0 = time.perf_counter()
    for _ in range(frames):
        mf.frame()
    frame_ms = (time.perf_counter() - t0) / frames * 1e3
    launches = mf.kernel_launches
    mf.close()
    n, vox = len(cfg["nuclei"]), (cfg["NN"] - 1) ** 3
    upd_bytes = vox * (24 * n + 4)
    out = {"grid": f"{cfg['NN']}^3", "electrons_fields": n, "steps_per_frame": 500, "frame_ms": frame_ms,
           "ms_per_step": frame_ms / 500, "update_bytes_per_step": upd_bytes,
           "update_GBps_if_all_time": upd_bytes / (frame_ms / 500 * 1e-3) / 1e9,
           "timing": "host wall clock around frame() = doSteps(500) + computeForces + stepNuclei",
           "librq_launches_total": launches}
    if not a.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        ref = orc.MolFastDriver(cfg["nuclei"], NN=cfg["NN"], screen=cfg["screen"], norm_targets=cfg["norm_targets"])
        ref.initialize()
        steps = 10
        t0 = time.perf_counter()
        ref.do_steps(steps)
        cpu_ms = (time.perf_counter() - t0) / steps * 1e3
        out.update({"cpu_ms_per_step": cpu_ms, "cpu_cores": len(os.sched_getaffinity(0)),
                    "cpu": f"the oracle's restatement of the shaders, OpenMP, {steps} steps (one reduction)"})
    return out


def _glycine_forces(g, rows, c32, c64):
    """Mixed-vs-FP64 force errors on glycine: (1) the Hellmann-Feynman force of the converged mixed
    solve (fp32 fields) against that of the converged FP64 solve; (2) the adjoint through ADJ_STEPS
    warm-started steps from the converged FP64 state, fp32 fields against FP64."""
    from realmolecule_b200 import _lib as L
    n_nuc = len(g.elements)
    F64 = c64.forces(L.FORCE_HF)[:n_nuc]
    F32 = c32.forces(L.FORCE_HF)[:n_nuc]
    # the adjoint from one state, in the same schedule phase on both contexts
    st = c64.download(psi=True, label=True, P=True)
    adj = {}
    for name, c in (("fp64", c64), ("mixed", c32)):
        c.step((4 - c.info().steps_done % 4) % 4)
        c.set_adjoint_window(ADJ_STEPS)
        c.upload(psi=st["psi"], label=st["label"], P=st["P"])
        c.set_atoms(rows)
        c.step(ADJ_STEPS)
        adj[name] = c.adjoint()[0][:n_nuc]
    return {"hf_converged_fp32_vs_fp64_max_abs": float(np.abs(F32 - F64).max()),
            "adjoint_fp32_vs_fp64_max_abs": float(np.abs(adj["mixed"] - adj["fp64"]).max()),
            "max_abs_force": float(np.abs(F64).max()), "unit": "Ha/bohr", "adjoint_steps": ADJ_STEPS}


def converge_leg(stream, dist, rank, world):
    from realmolecule_b200 import Context, configs, _lib as L
    from realmolecule_b200.batch import Batch
    from realmolecule_b200 import shard
    out = {"criterion": f"|dE| < {TOL:g} Ha on {CHECKS} consecutive checks {CHECK} steps apart (a mixed solve "
                        "would finish in FP64 only below 1e-12 |E|)",
           "labels": f"level set for the first {LABEL_UNTIL} steps, then frozen",
           "timing": "CUDA events around initialise + solve on the solver stream (allocation excluded)"}

    # glycine 128^3, one context per precision (every rank solves it; rank 0 reports)
    g = configs.glycine128()
    rows = configs.to_domain_atoms(g)
    gly, keep = {}, {}
    for prec in ("mixed", "fp64"):
        c = Context(g.NN, g.screen, rows, flavor="new", precision=prec, label_until=LABEL_UNTIL,
                    converge_checks=CHECKS)
        c.set_stream(stream.cuda_stream)
        (steps, E), t = _timed(stream, lambda: (c.initialize(), c.solve(TOL, MAX_STEPS, CHECK))[1])
        gly[prec] = (_max_over_ranks(dist, t), int(steps), float(E), bool(c.fp64))
        keep[prec] = c
    forces = _glycine_forces(g, rows, keep["mixed"], keep["fp64"])
    for c in keep.values():
        c.close()
    n_int = (g.NN - 1) ** 3
    out["glycine128"] = {"electrons": int(g.charges.sum()), "grid": f"{g.NN}^3 h={g.h}",
                         "mixed_s": gly["mixed"][0], "fp64_s": gly["fp64"][0],
                         "gpts_mixed": gly["mixed"][1] * n_int / gly["mixed"][0] / 1e9,
                         "gpts_fp64": gly["fp64"][1] * n_int / gly["fp64"][0] / 1e9,
                         "speedup_vs_fp64": gly["fp64"][0] / gly["mixed"][0],
                         "steps_mixed": gly["mixed"][1], "steps_fp64": gly["fp64"][1],
                         "mixed_promoted_to_fp64": gly["mixed"][3],
                         "E_mixed": gly["mixed"][2], "E_fp64": gly["fp64"][2],
                         "abs_dE_Ha": abs(gly["mixed"][2] - gly["fp64"][2]), "forces": forces}

    # water 64^3 (the H2O configuration in the new flavour), one context per precision
    w = configs.h2o64()
    rows_w = configs.to_domain_atoms(w)
    wat = {}
    for prec in ("fp64", "mixed"):
        c = Context(w.NN, w.screen, rows_w, flavor="new", precision=prec, label_until=LABEL_UNTIL,
                    converge_checks=CHECKS)
        c.set_stream(stream.cuda_stream)
        (steps, E), t = _timed(stream, lambda: (c.initialize(), c.solve(TOL, MAX_STEPS, CHECK))[1])
        wat[prec] = (_max_over_ranks(dist, t), int(steps), float(E))
        c.close()
    n_w = (w.NN - 1) ** 3
    out["water64"] = {"electrons": int(w.charges.sum()), "grid": f"{w.NN}^3 h={w.h}",
                      "fp64_s": wat["fp64"][0], "mixed_s": wat["mixed"][0],
                      "steps_fp64": wat["fp64"][1], "steps_mixed": wat["mixed"][1],
                      "gpts_fp64": wat["fp64"][1] * n_w / wat["fp64"][0] / 1e9,
                      "gpts_mixed": wat["mixed"][1] * n_w / wat["mixed"][0] / 1e9,
                      "E_fp64": wat["fp64"][2], "abs_dE_Ha": abs(wat["fp64"][2] - wat["mixed"][2])}

    # 96 water clusters: this rank's cost share, mixed batch vs one FP64 context per instance
    geoms = configs.clusters96()
    inst = [{"NN": x.NN, "screen": x.screen, "atoms": configs.to_domain_atoms(x)} for x in geoms]
    share = [inst[q] for q in shard.my_share(inst, rank, world)]
    b = Batch(share, precision="mixed", label_until=LABEL_UNTIL, converge_checks=CHECKS)
    b.set_stream(stream.cuda_stream)
    tune, t_tune = None, 0.0
    if share:  # tuned once for this batch before the timed solve (a deployment keeps the choice)
        b.initialize()
        tune, t_tune = _timed(stream, b.autotune)
    (cb, Eb), tb = _timed(stream, lambda: (b.initialize(), b.solve(TOL, MAX_STEPS, CHECK))[1])
    pts = b.info()["interior_points"]
    b.close()

    def plain():
        E, steps = [], []
        for it in share:
            c = Context(it["NN"], it["screen"], it["atoms"], flavor="new", precision="fp64",
                        label_until=LABEL_UNTIL, converge_checks=CHECKS)
            c.set_stream(stream.cuda_stream)
            c.initialize()
            n, e = c.solve(TOL, MAX_STEPS, CHECK)
            c.close()
            E.append(e)
            steps.append(n)
        return np.array(E), np.array(steps)
    (Ep, sp), tp = _timed(stream, plain)
    tb, tp = _max_over_ranks(dist, tb), _max_over_ranks(dist, tp)
    dE = _max_over_ranks(dist, float(np.max(np.abs(Eb - Ep))) if len(share) else 0.0)
    out["clusters96"] = {"instances": len(inst), "ranks": world, "scaling": "strong",
                         "interior_points_rank0": pts,
                         "mixed_batched_s": tb, "fp64_plain_s": tp,
                         "autotune_rank0": {"s": t_tune, "config": tune["config"] if tune else None},
                         "solves_per_s_mixed_batched": len(inst) / tb, "solves_per_s_fp64_plain": len(inst) / tp,
                         "speedup_vs_fp64_plain": tp / tb, "max_abs_dE_Ha": dE,
                         "unconverged_rank0": {"mixed_batched": int((cb < 0).sum()) if len(share) else 0,
                                               "fp64_plain": int((sp >= MAX_STEPS).sum()) if len(share) else 0},
                         "steps_rank0": {"mixed_batched_max": int(cb.max()) if len(share) else 0,
                                         "fp64_plain_max": int(sp.max()) if len(share) else 0,
                                         "fp64_plain_sum": int(sp.sum()) if len(share) else 0}}
    return out


def main():
    a = parse()
    if a.leg:
        import torch
        torch.cuda.set_device(0)
        leg = {"molecule_js_lobpcg": lobpcg_leg, "mol_fast_ch4": mol_fast_leg, "realqm_rb_h2": realqm_rb_leg}[a.leg]
        print(json.dumps({a.leg: leg(a)}), flush=True)
        return
    if a.impl == "reference":
        run_reference_arm(a)
        return
    run_ours(a)


if __name__ == "__main__":
    main()
