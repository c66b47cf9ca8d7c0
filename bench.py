"""Benchmark of the RealQM solver step on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload glycine128]

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
``roofline`` the dominant kernel (fused ITP update, 20 algorithmic B per interior point)
           against the measured HBM copy bandwidth;
``cpu_baseline`` the reference's own cloud/solver.py kernels compiled for the host
           (oracle/_ref, OpenMP over all host cores) on a bounded sample of the same workload.

``--impl reference`` times that reference CPU implementation alone (the reference has no
GPU path that can run here: its kernels need CuPy, which is not installed).
Multi-GPU (torchrun): every rank runs an independent replica (the solve does not shard);
value = all ranks' updates / max-over-ranks time; scaling "weak".
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
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="glycine128")
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
    # each bench step is a bounded sample: 20 solver steps (a 1/5 period) of the same workload
    per = 20
    rate, threads, dt = cpu_reference_rate(cfg, per * a.steps, per * a.warmup)
    line = {"metric": METRIC, "value": rate, "unit": "Gpt/s", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": dt / a.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": desc, "step": f"{per} solver steps (bounded sample of the period)"},
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
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
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


def ncu_traffic():
    """DRAM bytes per launch of the update kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "update_sp_glycine128.md")
    try:
        with open(p) as f:
            for ln in f:
                if ln.startswith("traffic_bytes_per_launch:"):
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

    if rank == 0:
        peak, peak_kind = measured_peak()
        up = prof.get("update", {"ms": 0, "bytes": 0, "launches": 1})
        upd_ms = up["ms"] / max(1, up["launches"])
        upd_bytes = up["bytes"] / max(1, up["launches"])
        achieved = upd_bytes / (upd_ms * 1e-3) / 1e9 if upd_ms > 0 else None
        cpu = None
        if world == 1 and not a.no_cpu_baseline:
            try:
                rate, threads, dt = cpu_reference_rate(cfg, 40, 2)
                cpu = {"value": rate, "unit": "Gpt/s", "cores": threads, "kind": "reference",
                       "sample": f"40 solver steps of {a.workload} after 2 warm-up ({dt:.1f} s)"}
            except Exception as e:  # the reference build is missing: say so
                cpu = {"value": None, "unit": "Gpt/s", "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}
        line = {
            "metric": METRIC, "value": value, "unit": "Gpt/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc,
                       "step": f"one schedule period = {PERIOD} solver steps (one CUDA-graph replay)",
                       "l2": "flushed (256 MB write) before every timed period; flush not timed",
                       "parallelism": f"replicas x{world}"},
            "value_l2_flushed_every_solver_step": value_cold,
            "e2e": {"value": e2e, "unit": "Gpt/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if achieved else None, "traffic": ncu_traffic(),
                         "kernel": "k_update_sp (fused ITP update)", "bytes_per_launch": upd_bytes,
                         "peak_kind": peak_kind},
            "kernels": {k: {"launches": v["launches"], "ms": round(v["ms"], 4), "GB/s": round(v["gbs"], 1)}
                        for k, v in prof.items()},
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference_arm(a)
        return
    run_ours(a)


if __name__ == "__main__":
    main()
