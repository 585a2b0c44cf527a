"""Benchmark of the B200 likelihood engine (one JSON line on rank 0).

Workload (one "step"), on the 128-taxon x 100,000-site GTR+I+G4 alignment
(synthetic, seeded; GARLI-compressed to unique patterns):
  1. every CLA dirty and the branch lengths reset to their starting values,
  2. a full-tree rescore (126 CLA updates + root lnL),
  3. one all-branch Newton-Raphson pass (OptimizeAllBranches: d1/d2 per branch,
     the CLAs each move dirties recomputed on the way).
Metric: CLA site-updates per second (pattern x CLA update) over the whole step;
lnL evaluations per second (full scores + edge lnL/d1/d2 evaluations) beside it.
The headline form is the precision form (FP32 CLAs, power-of-two scalers,
FP64 P(t)/sums/Newton); the plain FP64 form is measured in the same run.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times GARLI's CPU path (the oracle restatement, built with
GARLI's -O3 -ffast-math flags, OpenMP over patterns on all host cores) on the
same workload and metric.  N > 1 runs N independent replicas (one per GPU, no
data-path collective); value = all replicas' site-updates / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "CLA site-updates/s (128x100k GTR+I+G4: full rescore + all-branch Newton pass)"
UNIT = "site-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ntax", type=int, default=128)
    ap.add_argument("--nsites", type=int, default=100_000)
    ap.add_argument("--precision", type=float, default=0.01, help="Newton optPrecision")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-sites", type=int, default=20_000)
    return ap.parse_args()


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.rows.append([x.strip() for x in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, n in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    """Per-launch DRAM bytes of the CLA kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "cla_kernel_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


def make_workload(args, seed):
    from garli_b200 import synth

    return synth.make_dna(args.ntax, args.nsites, seed, pinv_range=(0.05, 0.3),
                          name=f"dna_gtr_i_g4_{args.ntax}x{args.nsites}")


def one_step(tree, dlen0, prec, marks=None):
    """Reset, full rescore, all-branch Newton pass.

    Returns (lnL of the rescore, counters delta).  ``marks`` (optional) is a
    callable recording CUDA events between the phases."""
    c0 = tree.counters()
    for nd in range(1, len(dlen0)):
        tree.set_branch_length(nd, float(dlen0[nd]))
    tree.make_all_dirty()
    if marks:
        marks("start")
    lnl = tree.score(0)
    if marks:
        marks("scored")
    tree.optimize_all_branches(prec)
    if marks:
        marks("optimised")
    c1 = tree.counters()
    return lnl, {k: c1[k] - c0[k] for k in c0}


def run_form(w, args, mixed, device, steps, warmup, timing_pass=True):
    import torch

    from garli_b200 import engine

    inst, tree = engine.tree_engine(w.data, w.child3, w.dlen, w.model, device=device, mixed=mixed)
    stream = torch.cuda.ExternalStream(inst.stream_ptr(), device=f"cuda:{device}")
    for _ in range(warmup):
        one_step(tree, w.dlen, args.precision)
    inst.synchronize()
    l0 = inst.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    tot = {"cla_ops": 0, "pattern_updates": 0, "edge_evals": 0, "scores": 0, "rescale_retries": 0}
    torch.cuda.synchronize(device)
    e0.record(stream)
    lnl = None
    for _ in range(steps):
        lnl, d = one_step(tree, w.dlen, args.precision)
        for k in tot:
            tot[k] += d[k]
    e1.record(stream)
    inst.synchronize()
    torch.cuda.synchronize(device)
    ms = e0.elapsed_time(e1)
    launches = inst.launch_count() - l0
    kt = None
    phases = None
    if timing_pass:
        inst.set_kernel_timing(True)
        ev = {}

        def marks(name):
            e = torch.cuda.Event(enable_timing=True)
            e.record(stream)
            ev[name] = e

        one_step(tree, w.dlen, args.precision, marks)
        inst.synchronize()
        kt = inst.kernel_timing()
        inst.set_kernel_timing(False)
        phases = {"rescore_ms": ev["start"].elapsed_time(ev["scored"]),
                  "newton_pass_ms": ev["scored"].elapsed_time(ev["optimised"])}
    return {"ms": ms, "tot": tot, "lnl": lnl, "launches": launches, "kt": kt, "phases": phases, "inst": inst,
            "tree": tree}


def e2e_run(w, args, device, steps):
    """The same step through the C ABI from host buffers: tips, weights and model are
    uploaded every step and the site log-likelihoods and branch lengths read back."""
    import torch

    from garli_b200 import engine

    pd = w.data
    inst, tree = engine.tree_engine(pd, w.child3, w.dlen, w.model, device=device, mixed=True)
    tips = [np.ascontiguousarray(pd.tips[t]) for t in range(pd.ntax)]
    bi = sum(t.nbytes for t in tips) + pd.counts.nbytes + pd.const_states.nbytes + w.dlen.nbytes
    bo = 8 * pd.npat + w.dlen.nbytes
    one_step(tree, w.dlen, args.precision)
    t0 = time.perf_counter()
    updates = 0
    for _ in range(steps):
        inst.set_data(pd)
        tree.set_model(w.model)
        lnl, d = one_step(tree, w.dlen, args.precision)
        updates += d["pattern_updates"]
        inst.site_lnl()
        tree.branch_lengths()
    torch.cuda.synchronize(device)
    dt = time.perf_counter() - t0
    tree.close()
    inst.close()
    return updates / dt, bi, bo


def cpu_baseline(args, threads=None):
    """GARLI's CPU path (oracle restatement, GARLI's gcc flags) on a bounded sample:
    the same tree and model, the first ``cpu_sample_sites`` sites."""
    from oracle import oracle as orc

    wsamp = make_workload(argparse.Namespace(ntax=args.ntax, nsites=args.cpu_sample_sites), seed=1)
    cores = threads or os.cpu_count() or 1
    orc.set_threads(cores, fast=True)
    ot = orc.OracleTree(wsamp.data, wsamp.child3, wsamp.dlen, wsamp.model, fast=True)
    t0 = time.perf_counter()
    c0 = ot.counts()["cla"]
    ot.make_all_dirty()
    ot.score(0)
    ot.optimize_all_branches(args.precision)
    dt = time.perf_counter() - t0
    ops = ot.counts()["cla"] - c0
    ot.close()
    return {"value": ops * wsamp.data.npat / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{args.ntax} taxa x {args.cpu_sample_sites} sites ({wsamp.data.npat} patterns), "
                      f"1 step = rescore + all-branch Newton pass, {dt:.1f} s"}


def reference_arm(args, ws, rank):
    if rank != 0:
        return
    steps = max(1, args.steps)
    from oracle import oracle as orc

    cores = os.cpu_count() or 1
    wsamp = make_workload(args, seed=1)
    orc.set_threads(cores, fast=True)
    ot = orc.OracleTree(wsamp.data, wsamp.child3, wsamp.dlen, wsamp.model, fast=True)
    for _ in range(min(args.warmup, 1)):
        ot.make_all_dirty(); ot.score(0)
    t0 = time.perf_counter()
    c0 = ot.counts()["cla"]
    for _ in range(steps):
        for nd in range(1, len(wsamp.dlen)):
            ot.set_branch_length(nd, float(wsamp.dlen[nd]))
        ot.make_all_dirty()
        ot.score(0)
        ot.optimize_all_branches(args.precision)
    dt = time.perf_counter() - t0
    v = (ot.counts()["cla"] - c0) * wsamp.data.npat / dt
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": steps, "warmup": args.warmup, "ms_per_step": 1000 * dt / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wsamp.name, "ntax": args.ntax, "nsites": args.nsites, "npat": wsamp.data.npat,
                       "model": "GTR+I+G4", "form": "GARLI CPU path, FP64", "parallelism": "openmp-patterns"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{steps} step(s) of the full {args.ntax}x{args.nsites} workload"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        reference_arm(args, ws, rank)
        return
    import torch

    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    device = local if ws > 1 else 0
    torch.cuda.set_device(device)
    w = make_workload(args, seed=1 + rank)
    peak, peak_kind = peaks()

    # plain FP64 form (same workload, fewer steps)
    plain = run_form(w, args, mixed=False, device=device, steps=max(1, args.steps // 2), warmup=1)
    # precision form: the headline
    if pg:
        pg.barrier()
    with ClockSampler(device) as clk:
        mixed = run_form(w, args, mixed=True, device=device, steps=args.steps, warmup=args.warmup)
    ms = mixed["ms"]
    if pg:
        t = torch.tensor([ms], dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
        u = torch.tensor([float(mixed["tot"]["pattern_updates"])], dtype=torch.float64)
        pg.all_reduce(u)
        updates_all = float(u.item())
    else:
        updates_all = float(mixed["tot"]["pattern_updates"])
    value = updates_all / (ms / 1000.0)
    evals = mixed["tot"]["scores"] + mixed["tot"]["edge_evals"]
    plain_v = plain["tot"]["pattern_updates"] / (plain["ms"] / 1000.0)
    kt = mixed["kt"]
    achieved = kt["cla_bytes"] / (kt["cla_ms"] / 1000.0) / 1e9 if kt and kt["cla_ms"] > 0 else None
    traffic = profiled_traffic()
    e2e_v, bi, bo = e2e_run(w, args, device, max(1, args.steps // 2))
    if pg:
        t = torch.tensor([e2e_v], dtype=torch.float64)
        pg.all_reduce(t)
        e2e_v = float(t.item())
    # precision form vs plain FP64 on the same tree (the rescore at the starting lengths);
    # the oracle itself is checked in tests/
    dl = abs(mixed["lnl"] - plain["lnl"])
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32-cla/f64-sums", "data": "synthetic (seeded)",
            "config": {"workload": w.name, "ntax": args.ntax, "nsites": args.nsites, "npat": w.data.npat,
                       "model": "GTR+I+G4", "form": "precision (FP32 CLAs, pow2 scalers)",
                       "step": "reset + full rescore + all-branch Newton pass",
                       "l2": "working set > L2 (378 CLAs x 4.3 MB)", "parallelism": f"replicas{ws}"},
            "lnl_evals_per_s": evals * ws / (ms / 1000.0),
            "plain_fp64": {"value": plain_v, "unit": UNIT, "ms_per_step": plain["ms"] / max(1, args.steps // 2),
                           "lnl": plain["lnl"], "phases": plain["phases"]},
            "phases": mixed["phases"],
            "mixed_over_plain": value / ws / plain_v,
            "abs_dlnl_mixed_vs_plain_same_tree": dl,
            "gpu_launches": mixed["launches"],
            "e2e": {"value": e2e_v, "unit": UNIT, "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "traffic": traffic.get("bytes_per_launch") if traffic else None,
                         "kernel": "k_cla4<float,4> (CLA update)", "peak_kind": f"{peak_kind} hbm_gbs",
                         "cla_kernel_ms_per_step": kt["cla_ms"] if kt else None,
                         "edge_kernel_ms_per_step": kt["edge_ms"] if kt else None},
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    for f in (plain, mixed):
        f["tree"].close()
        f["inst"].close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
