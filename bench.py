"""Benchmark of the BB_PD hot path on B200: bond-updates/s of the fused
persistent time-step kernel (one bond-update = one undirected bond evaluated
in one time step).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
                    [--config c1|c2|c3] [--form fp64|fp32] [--no-cpu-baseline]

Default workload (N=1): the 1.28M-node beam (400 x 40 x 80 lattice at
dx = 1.25 mm, 74.5M bonds), trilinear softening, ADR, plain FP64; synthetic
inputs built like the reference's input scripts. A step is one time step of
the whole beam. `value` times K steps of one persistent-kernel launch on data
resident in HBM (CUDA events on the launching stream); `e2e` times the C-ABI
job from host buffers (upload and layout, K steps, download of the state).
With N > 1 (torchrun) every rank solves its own beam: independent replicas,
no collective on the data path, value = all ranks' bond-updates / max time.

`--impl reference` times the reference's CPU implementation of the path (its
compiled MEX routines from oracle/_ref driven by the oracle's loop, the
MATLAB-only pieces restated in C) on this host's cores, on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    "c1": ("config1", "beam 100x10x20 dx=5mm (20k nodes, 1.0M bonds)"),
    "c2": ("config2", "beam 400x40x80 dx=1.25mm (1.28M nodes, 74.5M bonds)"),
    "c3": ("config3", "notched beam 160x20x40 dx=2.5mm (128k nodes, 7.1M bonds), lognormal sc"),
}
# ADR displacement control: 1e-7 mm per step at the midspan top nodes (metres)
RATE = -1e-10


def law_for(cfg):
    return ("exponential", dict(law="exponential", s0=1e-4)) if cfg == "c3" else \
        ("trilinear", dict(law="trilinear", s0=1e-4, s1=3e-4, sc=2e-3))


def peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def fp64_per_step(cfg, form, node_order):
    """FP64 thread-instructions per time step of the step kernel from an ncu
    count of this workload (profiles/step_kernel_fp64_inst.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "step_kernel_fp64_inst.json")) as f:
            t = json.load(f)[cfg][form][node_order]
        return float(t["fp64_thread_inst_per_step"]), t.get("source")
    except Exception:
        return None, None


def fp64_peak():
    """Measured FP64 FMA lane-operations per second of this device
    (bbpd_selftest_fp64_peak: independent FMA chains, CUDA events)."""
    import ctypes as C
    from bb_pd_b200 import _native as N
    v = C.c_double()
    N.check(N.lib().bbpd_selftest_fp64_peak(0.3, C.byref(v)))
    return v.value


def measured_traffic(cfg, form, node_order):
    """DRAM bytes (read + write) per time step of the step kernel from an ncu
    capture of this workload (profiles/step_kernel_traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "step_kernel_traffic.json")) as f:
            t = json.load(f)[cfg][form][node_order]
        return float(t["dram_bytes_per_step"]), t.get("source")
    except Exception:
        return None, None


def batch_traffic(form, mixed, bonds):
    """DRAM bytes per step of the batch launches, from the bytes per
    bond-update of an ncu capture of a smaller batch of the same series
    (profiles/batch_kernel_traffic.json) times the run's bonds, or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "batch_kernel_traffic.json")) as f:
            t = json.load(f)[form]["mixed" if mixed else "per_law"]
        return float(t["dram_bytes_per_bond_update"]) * bonds, t.get("source")
    except Exception:
        return None, None


def max_over_ranks(x, dist, device=None):
    """The largest of every rank's x (every rank gets it); x itself without a
    process group. Timings of a multi-GPU run are the slowest rank's."""
    if not dist:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(bonds_per_rank, steps, world, seconds):
    """Whole-job bond-updates/s of `world` independent replicas, each evaluating
    bonds_per_rank bonds for `steps` steps, timed by the slowest rank."""
    return bonds_per_rank * steps * world / seconds


def algorithmic_bytes(nN, nB, per_bond_sc):
    """Bytes one time step must move: per directed bond entry 4 B of neighbour
    index + 8 B of damage state (+ 8 B of per-bond critical stretch), per node
    181 B (x0, u, v, F_prev read and written, mass, family count, flags)."""
    nD = 2 * nB
    return nD * 12 + (nD * 8 if per_bond_sc else 0) + nN * 181


class Clocks:
    """nvidia-smi samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_rate(inp, lawkw, budget_s, warmup, max_steps, kernels="reference"):
    """Time the CPU implementation on `inp`: returns (bond-updates/s, steps, seconds, kind, threads)."""
    from oracle import pyoracle as po
    kind = "reference" if (kernels == "reference" and po.ref_available()) else "port"
    run = po.Run(inp, scheme="adr", rate=RATE, kernels="reference" if kind == "reference" else "restated", **lawkw)
    for _ in range(warmup):
        run.step(1)
    t0 = time.perf_counter()
    run.step(1)
    t1 = time.perf_counter() - t0
    n = 1
    limit = max(1, min(max_steps, int(budget_s / max(t1, 1e-9))))
    while n < limit:
        run.step(1)
        n += 1
    dt = time.perf_counter() - t0
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)) if kind == "reference" else 1
    return inp["nBonds"] * n / dt, n, dt, kind, threads


def _batch_line(args, metric, unit, value, ms_step, config, extra):
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.form == "fp64" else "f32+f64", "data": "synthetic",
            "config": config}
    line.update(extra)
    print(json.dumps(line), flush=True)


def run_batch(args):
    """The size-effect series (geometrically similar beams, log-uniform depths
    50-400 mm, span/depth 5, width 50 mm, seeded lognormal sc, laws alternating
    linear/trilinear) stepped together by one persistent batch launch replayed
    from a CUDA graph, against the same beams stepped one at a time in plain
    FP64."""
    import bb_pd_b200 as bb
    from bb_pd_b200 import serving
    series = bb.beam.size_effect_series(args.members, dx=args.dx)
    mk = lambda i, law, prec: bb.Solver(i, scheme="adr", rate=RATE, precision=prec, **serving.LAWKW[law])
    # one beam's host arrays at a time: the full series (dx 2.5 mm) holds
    # billions of bonds, resident on the device but not at once on the host
    sol, nodes, bonds = [], [], []
    t_create = time.perf_counter()
    for sp, law in series:
        i = bb.beam.build(sp)
        nodes.append(i["nNodes"])
        bonds.append(i["nBonds"])
        sol.append(mk(i, law, args.form))
        del i
    t_create = time.perf_counter() - t_create
    tot_b = float(sum(bonds))
    batch = bb.Batch(args.form)
    if args.batch_mixed >= 0:
        batch.set_mixing(args.batch_mixed != 0)
    for s in sol:
        batch.add(s)
    if args.batch_schedule:   # a fixed schedule instead of the autotuner (profiling one kernel)
        bps, grab = (int(v) for v in args.batch_schedule.split(","))
        batch.set_schedule(bps, grab)
    else:
        bps, grab = batch.tune(max(1, args.warmup // 3))
    batch.step(args.warmup)
    clocks = Clocks(0)
    clocks.start()
    time.sleep(0.15)
    batch.step(args.steps)          # graph replays from the second launch of this length on
    batch.step(args.steps)
    clk = clocks.stop()
    ms = batch.last_kernel_ms()
    info = batch.info()
    batch.close()
    value = tot_b * args.steps / (ms / 1e3)
    # plain FP64, one beam at a time, same steps
    seq_ms = 0.0
    for s in sol:
        s.close()
    for sp, law in ([] if args.no_sequential else series):
        s = mk(bb.beam.build(sp), law, "fp64")
        s.step(args.warmup)
        s.step(args.steps)
        seq_ms += s.last_kernel_ms()
        s.close()
    seq = tot_b * args.steps / (seq_ms / 1e3) if seq_ms > 0 else None
    peak, kind = peak_hbm()
    alg = sum(algorithmic_bytes(n, b, True) for n, b in zip(nodes, bonds))
    ach = alg / (ms / args.steps / 1e3) / 1e9
    traffic, tsrc = batch_traffic(args.form, info["n_classes"] == 1 and len(set(l for _, l in series)) > 1, tot_b)
    config = {"workload": f"size-effect series: {args.members} beams, depth 50-400 mm log-uniform, span/depth 5, "
                          f"width 50 mm, dx {args.dx * 1e3:g} mm, linear/trilinear, lognormal sc, ADR, "
                          f"1e-7 mm/step", "nodes": int(sum(nodes)), "bonds": int(tot_b),
              "min_nodes": int(min(nodes)), "max_nodes": int(max(nodes)), "form": args.form,
              "l2": "inputs larger than L2", "parallelism": "1 GPU, one persistent batch launch",
              "steps_note": f"{args.steps} timed steps of the 10 000 the series names (time budget)",
              "create_s": round(t_create, 1), "classes": info["n_classes"]}
    _batch_line(args, "bond-updates/s", "bond-updates/s", value, ms / args.steps, config, {
        "sequential_plain_fp64": {"value": seq, "unit": "bond-updates/s",
                                  "ms_per_step": seq_ms / args.steps if seq else None},
        "speedup_vs_sequential_fp64": value / seq if seq else None,
        "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                     "peak_kind": peak_kind_str(kind), "traffic": traffic, "traffic_source": tsrc,
                     "per": "time step of the whole batch"},
        "schedule": {"blocks_per_sm": bps, "grab": grab, "graph": bool(info["graph"]),
                     "launches_per_replay": info["n_classes"],
                     "mixing": "fixed" if args.batch_mixed >= 0 else "autotuned"},
        "gpu_launches": info["n_classes"], "clocks": clk, "cpu_baseline": None, "e2e": None})


def peak_kind_str(kind):
    return f"{kind} (MEASURED_PEAKS.json hbm_gbs)" if kind == "measured" else kind


def run_serve(args):
    """A Poisson stream of beam solves (node counts log-uniform, dx from
    1.25/2.5/5 mm, law uniform over the four laws), each run until its load has
    dropped to 80 % of its peak or the step cap; continuous batching under a
    150 GB HBM budget against one plain FP64 solve at a time."""
    import bb_pd_b200 as bb
    from bb_pd_b200 import serving
    stream = bb.beam.serving_stream(args.requests, nodes_range=(1e4, args.max_nodes), rate_hz=args.arrival_hz)
    reqs = []
    for k, r in enumerate(stream):   # arrays built on admission: the full stream does not fit host memory
        c = bb.beam.count(r["spec"])
        reqs.append(serving.Request(k, r["arrival"], (lambda sp=r["spec"]: bb.beam.build(sp)), r["law"],
                                    args.serve_rate, args.max_steps, sizes=(c.n_nodes, c.n_bonds, False)))
    clocks = Clocks(0)
    clocks.start()
    res, st = serving.run_batched(reqs, precision=args.form, chunk=100)
    clk = clocks.stop()
    seq, sst = serving.run_sequential(reqs, precision="fp64", chunk=100)
    a, b = serving.summary(res, st), serving.summary(seq, sst)
    peaks = {r.id: r for r in res}
    peak_err = max((abs(peaks[r.id].peak - r.peak) / r.peak for r in seq if r.peak > 0), default=0.0)
    reached = sum(1 for r in res if r.steps < args.max_steps)
    config = {"workload": f"serving stream: {args.requests} Poisson arrivals at {args.arrival_hz} /s, nodes "
                          f"log-uniform 1e4-{args.max_nodes:.0e}, dx 1.25/2.5/5 mm, four laws, to 80 % post-peak "
                          f"load or {args.max_steps} steps, {abs(args.serve_rate) * 1e3:g} mm/step, HBM budget 150 GB",
              "form": args.form, "parallelism": "1 GPU, continuous batching"}
    _batch_line(args, "solves/h", "solves/h", a["solves_per_hour"], None, config, {
        "batched": a, "sequential_plain_fp64": b,
        "speedup_solves_per_hour": a["solves_per_hour"] / b["solves_per_hour"],
        "p50_latency_s": a["p50_latency_s"], "p99_latency_s": a["p99_latency_s"],
        "peak_load_rel_diff_vs_fp64_max": peak_err, "solves_past_peak": reached,
        "gpu_launches": st["launches"], "clocks": clk, "cpu_baseline": None, "e2e": None})


def run_precision(args):
    """Error of the FP32 form against plain FP64: (1) one step from the same
    FP64 state of the --config beam after --warmup steps: nodal force error
    relative to the largest nodal force, and whether the broken-bond set is
    the same; (2) the 500 x 100 x 50 mm beam (dx 5 mm) loaded at 1e-4 mm/step
    in both forms until its load has dropped to 80 % of the peak: peak load,
    its step, the largest load difference along the curve, and the broken-bond
    sets at the end."""
    import numpy as np
    import bb_pd_b200 as bb
    from bb_pd_b200 import serving
    fn, wname = CONFIGS[args.config]
    lawname, lawkw = law_for(args.config)
    inp = bb.beam.build(getattr(bb.beam, fn)())
    kw = dict(lawkw, scheme="adr", rate=RATE)
    a = bb.Solver(inp, precision="fp64", **kw)
    b = bb.Solver(inp, precision="fp32", **kw)
    a.step(args.warmup)
    b.restore(a.checkpoint())
    a.step(1)
    b.step(1)
    Fa, Fb = a.get("force"), b.get("force")
    ferr = float(np.abs(Fa - Fb).max() / np.abs(Fa).max())
    same_broken = bool(np.array_equal(a.get("bsf") == 1, b.get("bsf") == 1) and
                       np.array_equal(a.get("fail") == 0, b.get("fail") == 0))
    a.close()
    b.close()
    # load-displacement to 20 % post-peak on the 20 000-node beam
    inp1 = bb.beam.build(bb.beam.config1())
    curves, broken = {}, {}
    for form in ("fp64", "fp32"):
        s = bb.Solver(inp1, precision=form, scheme="adr", rate=-1e-7, **serving.LAWKW["trilinear"])
        tr = serving._Track(serving.Request(0, 0.0, inp1, "trilinear", -1e-7, 20000))
        while True:
            s.step(100)
            if tr.update(s.reaction(100)):
                break
        curves[form] = (np.concatenate(tr.hist), tr.peak, tr.peak_step)
        broken[form] = (s.get("bsf") == 1) | (s.get("fail") == 0)
        s.close()
    (ra, pa, sa), (rb, pb, sb) = curves["fp64"], curves["fp32"]
    n = min(len(ra), len(rb))
    line = {"metric": "fp32 nodal-force error vs fp64", "value": ferr, "unit": "max |dF| / max |F|",
            "n_gpus": 1, "steps": 1, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": f"{wname}, {lawname}, ADR: one step from the FP64 state after "
                                   f"{args.warmup} steps; load-displacement: 500x100x50 mm beam, dx 5 mm, "
                                   f"trilinear, 1e-4 mm/step, to 80 % post-peak load"},
            "broken_set_identical_one_step": same_broken,
            "load_displacement": {"peak_load_fp64": pa, "peak_load_fp32": pb,
                                  "peak_load_rel_diff": abs(pb - pa) / pa, "peak_step_fp64": sa,
                                  "peak_step_fp32": sb,
                                  "max_load_diff_rel_to_peak": float(np.abs(ra[:n] - rb[:n]).max() / pa),
                                  "steps_fp64": len(ra), "steps_fp32": len(rb),
                                  "broken_bonds_fp64": int(broken["fp64"].sum()),
                                  "broken_bonds_fp32": int(broken["fp32"].sum()),
                                  "broken_set_identical_at_end": bool(np.array_equal(broken["fp64"], broken["fp32"]))},
            "gpu_launches": None, "cpu_baseline": None, "e2e": None, "roofline": None}
    print(json.dumps(line), flush=True)


def serving_sample(requests=12, max_nodes=6e4, arrival_hz=6.0, rate=-1e-7, max_steps=4000, seed=20261203):
    """A short serving run (continuous batching vs one plain FP64 solve at a
    time) for the default bench line: a Poisson stream of `requests` beams of
    1e4 .. max_nodes nodes, the four laws, each to 80 % post-peak load or
    max_steps, at `rate` metres per step."""
    import bb_pd_b200 as bb
    from bb_pd_b200 import serving
    stream = bb.beam.serving_stream(requests, seed=seed, nodes_range=(1e4, max_nodes), rate_hz=arrival_hz,
                                    dx_choices=(2.5e-3, 5e-3))
    reqs = [serving.Request(k, r["arrival"], bb.beam.build(r["spec"]), r["law"], rate, max_steps)
            for k, r in enumerate(stream)]
    res, st = serving.run_batched(reqs, precision="fp64", chunk=100)
    seq, sst = serving.run_sequential(reqs, precision="fp64", chunk=100)
    a, b = serving.summary(res, st), serving.summary(seq, sst)
    peaks = {r.id: r for r in res}
    peak_err = max((abs(peaks[r.id].peak - r.peak) / r.peak for r in seq if r.peak > 0), default=0.0)
    return {"metric": "solves/h", "value": a["solves_per_hour"], "unit": "solves/h",
            "p50_latency_s": a["p50_latency_s"], "p99_latency_s": a["p99_latency_s"],
            "sequential_plain_fp64": {"solves_per_hour": b["solves_per_hour"], "p50_latency_s": b["p50_latency_s"],
                                      "p99_latency_s": b["p99_latency_s"]},
            "speedup_solves_per_hour": a["solves_per_hour"] / b["solves_per_hour"],
            "peak_load_rel_diff_vs_sequential_max": peak_err,
            "solves_past_peak": sum(1 for r in res if r.steps < max_steps),
            "config": {"workload": f"serving sample: {requests} Poisson arrivals at {arrival_hz:g}/s, nodes "
                                   f"log-uniform 1e4-{max_nodes:.0e}, dx 2.5/5 mm, four laws, to 80 % post-peak "
                                   f"load or {max_steps} steps, {abs(rate) * 1e3:g} mm/step, plain FP64, "
                                   "continuous batching vs one solve at a time"},
            "gpu_launches": st["launches"], "peak_members": st.get("peak_members")}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=list(CONFIGS))
    ap.add_argument("--form", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--node-order", default="input", choices=["input", "morton", "tiled", "lattice"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving sample of the default line")
    ap.add_argument("--workload", default="single", choices=["single", "batch", "serve", "precision"],
                    help="single: one beam (--config); batch: the size-effect series in one "
                         "persistent batch launch; serve: a Poisson stream of solves, continuous batching")
    ap.add_argument("--members", type=int, default=64, help="batch: beams in the size-effect series")
    ap.add_argument("--dx", type=float, default=2.5e-3, help="batch: lattice spacing of the series (m)")
    ap.add_argument("--batch-schedule", default="", help="batch: 'blocks_per_sm,grab' instead of autotuning")
    ap.add_argument("--batch-mixed", type=int, default=-1,
                    help="batch: 1 one launch for all laws, 0 one per law, -1 the autotuner chooses")
    ap.add_argument("--no-sequential", action="store_true", help="batch: skip the one-beam-at-a-time baseline")
    ap.add_argument("--requests", type=int, default=48, help="serve: number of requests")
    ap.add_argument("--max-nodes", type=float, default=3e5, help="serve: largest beam (nodes)")
    ap.add_argument("--arrival-hz", type=float, default=4.0, help="serve: Poisson arrival rate")
    ap.add_argument("--max-steps", type=int, default=6000, help="serve: step cap per solve")
    ap.add_argument("--serve-rate", type=float, default=-1e-7, help="serve: displacement per step (m)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.workload != "single" and args.impl == "ours":
        if int(os.environ.get("RANK", "0")) == 0:
            {"batch": run_batch, "serve": run_serve, "precision": run_precision}[args.workload](args)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if args.impl == "reference" and rank != 0:
        return                      # the CPU reference runs on rank 0 only
    if world > 1 and args.impl == "ours":
        import torch
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    import bb_pd_b200 as bb
    fn, wname = CONFIGS[args.config]
    lawname, lawkw = law_for(args.config)
    per_bond_sc = args.config == "c3"
    metric, unit = "bond-updates/s", "bond-updates/s"
    config = {"workload": f"{wname}, {lawname} law, ADR, 1e-7 mm/step midspan displacement control",
              "nodes": None, "bonds": None, "form": args.form, "node_order": args.node_order,
              "l2": "inputs larger than L2: every step streams the whole bond layout (GBs) through HBM",
              "parallelism": f"replicas x{args.gpus}" if args.gpus > 1 else "1 GPU"}

    if args.impl == "reference":
        if rank != 0:
            return
        inp = bb.beam.build(getattr(bb.beam, fn)())
        config.update(nodes=inp["nNodes"], bonds=inp["nBonds"])
        rate, n, dt, kind, threads = cpu_reference_rate(inp, lawkw, budget_s=120.0, warmup=args.warmup,
                                                        max_steps=args.steps)
        line = {"metric": metric, "value": rate, "unit": unit, "n_gpus": args.gpus, "steps": n,
                "warmup": args.warmup, "ms_per_step": 1e3 * dt / n, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
                "impl": "reference",
                "cpu_baseline": {"value": rate, "unit": unit, "cores": threads, "kind": kind,
                                 "sample": f"{n} of the requested {args.steps} time steps of the full beam"},
                "e2e": {"value": rate, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    dev = local
    torch.cuda.set_device(dev)
    inp = bb.beam.build(getattr(bb.beam, fn)())
    nN, nB = inp["nNodes"], inp["nBonds"]
    config.update(nodes=nN, bonds=nB)
    kw = dict(lawkw, scheme="adr", rate=RATE, precision=args.form, node_order=args.node_order)

    # ---- value: resident data, one persistent launch of K steps ----
    torch.cuda.synchronize()
    tc0 = time.perf_counter()
    s = bb.Solver(inp, device=dev, **kw)
    torch.cuda.synchronize()
    cold_create_s = time.perf_counter() - tc0
    info = s.info()
    s.step(args.warmup)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(dev)
    clocks.start()
    time.sleep(0.15)
    s.step_async(args.steps)
    s.sync()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(s.last_kernel_ms(), dist, "cuda")
    if dist:
        dist.barrier()
    ms_step = ms / args.steps
    value = replica_rate(nB, args.steps, world, ms / 1e3)
    s.close()
    del s

    # ---- e2e: the C-ABI job from host buffers ----
    e2e = None
    if not args.no_e2e:
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        s2 = bb.Solver(inp, device=dev, **kw)
        t1 = time.perf_counter()
        s2.step(args.steps)
        t2 = time.perf_counter()
        outs = [s2.get(f) for f in ("displacement", "force", "bsf", "flag", "fail")]
        torch.cuda.synchronize()
        te = time.perf_counter() - t0
        parts = {"create_s": t1 - t0, "steps_s": t2 - t1, "download_s": te - (t2 - t0)}
        s2.close()
        te = max_over_ranks(te, dist, "cuda")
        h2d = sum(inp[k].nbytes for k in ("undeformedCoordinates", "BONDLIST", "UNDEFORMEDLENGTH",
                                           "BONDSTIFFNESS", "VOLUMECORRECTIONFACTORS", "massVector",
                                           "CONSTRAINTFLAG", "BODYFORCEFLAG")) + (inp["sc"].nbytes if per_bond_sc else 0)
        d2h = sum(o.nbytes for o in outs)
        e2e = {"value": replica_rate(nB, args.steps, world, te), "unit": unit,
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "seconds": te, **{k: round(v, 4) for k, v in parts.items()},
               "cold_create_s": round(cold_create_s, 4),
               "includes": "upload of the reference arrays, layout build, K steps, download of state",
               "pool": "warm: the timed create is the second in the process, so the pinned staging slots "
                       "and the layout pool allocated by the first are reused (a resident service); "
                       "cold_create_s is the first create of the process"}

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return

    peak, peak_kind = peak_hbm()
    alg = algorithmic_bytes(nN, nB, per_bond_sc)
    achieved = alg / (ms_step / 1e3) / 1e9
    traffic, tsrc = measured_traffic(args.config, args.form, args.node_order)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind, "traffic": traffic, "traffic_source": tsrc, "per": "time step",
                "algorithmic_bytes_per_step": alg, "layout_bytes_per_step": info["bytes_per_step"]}
    f64, f64src = fp64_per_step(args.config, args.form, args.node_order)
    if f64 is not None:
        pk = fp64_peak()
        ach64 = f64 / (ms_step / 1e3)
        roofline["fp64"] = {"achieved": ach64, "peak": pk, "unit": "FP64 thread-instructions/s",
                            "frac": ach64 / pk, "inst_per_step": f64, "source": f64src,
                            "peak_kind": "measured now (bbpd_selftest_fp64_peak: FMA chains)"}

    cpu = None
    if not args.no_cpu_baseline and world == 1:
        rate, n, dt, kind, threads = cpu_reference_rate(inp, lawkw, budget_s=20.0, warmup=0, max_steps=50)
        cpu = {"value": rate, "unit": unit, "cores": threads, "kind": kind,
               "sample": f"{n} time steps of the same beam ({dt:.1f} s)"}

    serve = None
    if not args.no_serving and world == 1:
        t0 = time.perf_counter()
        serve = serving_sample()
        serve["seconds"] = round(time.perf_counter() - t0, 1)

    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.form == "fp64" else "f32+f64", "data": "synthetic",
            "config": config, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": 1,
            "clocks": clk, "solver": {"grid_blocks": info["grid_blocks"], "entries": info["n_entries"],
                                      "device_bytes": info["device_bytes"], "layout": info["layout"]},
            "serving": serve}
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
