"""Benchmark of the B200 likelihood engine (one JSON line on rank 0).

Headline workload (one "step" = one GA generation): 256 candidate trees, each a
64-taxon Yule base tree after one SPR/NNI move (radius ~ U{1..8}), DNA GTR+G4,
50,000 sites (seeded synthetic, GARLI-compressed to unique patterns).  Every
candidate is rescored (its dirty CLAs recomputed, every other CLA shared with
the base tree) and the three branches at its move's connector are optimised by
GARLI's Newton-Raphson (nd->left, nd, nd->right), then scored at the optimised
lengths.
  * batched precision form (the headline value): all candidates in one
    persistent kernel launch (FP32 CLAs, FP64 coefficients, sums and Newton);
  * plain FP64 per-tree path (measured in the same run): GARLI's way, one
    candidate after another, a host Newton loop per branch.
Metric: CLA site-updates per second (pattern x CLA update; the per-step
partials on the connector count as updates in both forms); lnL evaluations per
second (edge evaluations: Newton derivative evaluations + final scores) beside it.
The single-tree step of the 128-taxon x 100,000-site GTR+I+G4 alignment
(full rescore + all-branch Newton pass) is reported as a secondary object.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times GARLI's CPU path (the oracle restatement, built with
GARLI's -O3 -ffast-math flags, OpenMP over patterns on all host cores) on a
bounded sample of the same generation: per candidate the CLAs GARLI would
recompute after the move, the same three Newton optimisations and the final
score.  N > 1 runs N independent replicas (one per GPU, no data-path
collective); value = all replicas' site-updates / max-over-ranks time.
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

METRIC = ("CLA site-updates/s (GA generation: 256 SPR/NNI candidates of a 64-taxon tree, 50k sites, GTR+G4; "
          "rescore + 3-branch Newton each), batched precision form")
UNIT = "site-updates/s"
SINGLE_METRIC = "CLA site-updates/s (128x100k GTR+I+G4: full rescore + all-branch Newton pass)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ncand", type=int, default=256)
    ap.add_argument("--batch-ntax", type=int, default=64)
    ap.add_argument("--batch-nsites", type=int, default=50_000)
    ap.add_argument("--ntax", type=int, default=128, help="single-tree workload")
    ap.add_argument("--nsites", type=int, default=100_000, help="single-tree workload")
    ap.add_argument("--precision", type=float, default=0.01, help="Newton optPrecision")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-single", action="store_true", help="skip the single-tree secondary measurement")
    ap.add_argument("--batch-only", action="store_true",
                    help="profiling: only the batched form (no per-tree comparison, no e2e pass)")
    ap.add_argument("--nstate-only", action="store_true",
                    help="profiling: only the 20- and 61-state rescores (tensor cores, CUDA cores, plain)")
    ap.add_argument("--single-only", action="store_true",
                    help="profiling: only the 128x100k single-tree step (precision and plain forms)")
    ap.add_argument("--cpu-sample-cands", type=int, default=24, help="candidates in the CPU baseline sample")
    ap.add_argument("--cpu-repeats", type=int, default=16, help="timed repeats per sampled candidate")
    ap.add_argument("--ref-cands-per-step", type=int, default=2, help="candidates per --impl reference step")
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
    """Per-launch DRAM bytes of the batched pass kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "batch_kernel_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


def batch_workload(args, seed):
    from garli_b200 import synth

    return synth.batch_workload(seed=seed, ntax=args.batch_ntax, nsites=args.batch_nsites, ncand=args.ncand)


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


def run_batch(bw, args, device, mixed, sequential, steps, warmup, clocks=None):
    """Time `steps` generations (device-timed on the instance stream)."""
    import torch

    from garli_b200 import engine

    w, c3s, dls, conn = bw
    inst, pop = engine.population_engine(w.data, w.child3, w.dlen, w.model, len(conn), device=device, mixed=mixed)
    stream = torch.cuda.ExternalStream(inst.stream_ptr(), device=f"cuda:{device}")
    out = lens = None
    for _ in range(warmup):  # the first call computes the base tree's CLAs and autotunes
        out, lens = pop.score(c3s, dls, conn, args.precision, sequential=sequential)
    torch.cuda.synchronize(device)
    l0 = inst.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    updates = edges = 0
    ctx = clocks if clocks is not None else _Null()
    with ctx:
        e0.record(stream)
        for _ in range(steps):
            out, lens = pop.score(c3s, dls, conn, args.precision, sequential=sequential)
            cnt = pop.counters()
            updates += cnt["pattern_updates"]
            edges += cnt["edge_evals"]
        e1.record(stream)
        torch.cuda.synchronize(device)
    ms = e0.elapsed_time(e1)
    res = {"ms": ms, "updates": updates, "edges": edges, "launches": inst.launch_count() - l0, "out": out,
           "lens": lens, "counters": pop.counters(), "tuning": pop.tuning(), "inst": inst, "pop": pop}
    return res


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def batch_kernel_roofline(r, args, peak, peak_kind):
    """Achieved bandwidth of the batched pass (one CUDA graph per generation:
    k_level4m per CLA level, k_coef4m per step, k_batch4m for the Newton and
    score runs): its algorithmic bytes over its CUDA-event time on the
    instance stream (a few extra timed passes)."""
    import torch

    w_c3s = r["bw"]
    pop, inst = r["pop"], r["inst"]
    _, c3s, dls, conn = w_c3s
    inst.set_kernel_timing(True)
    t0 = pop.batch_timing()
    n = 5
    for _ in range(n):
        pop.score(c3s, dls, conn, args.precision)
    t1 = pop.batch_timing()
    inst.set_kernel_timing(False)
    torch.cuda.synchronize()
    ms = (t1["ms"] - t0["ms"]) / max(1, t1["launches"] - t0["launches"])
    alg = pop.counters()["alg_bytes"]
    achieved = alg / (ms / 1e3) / 1e9
    traffic = profiled_traffic()
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic.get("bytes_per_pass") if traffic else None,
            "kernel": "batched pass: k_level4m<4> per CLA level, k_coef4m<4> per step, k_batch4m<4> per "
                      "Newton run (one CUDA graph per generation)",
            "peak_kind": f"{peak_kind} hbm_gbs (burst copy)", "ms_per_pass": ms,
            "algorithmic_bytes_per_pass": alg,
            "traffic_note": traffic.get("note") if traffic else "no ncu capture committed"}


def e2e_batch(bw, args, device, steps):
    """The generation through the public call with host buffers: candidate
    topologies, lengths and connectors go in from pinned host memory, per-candidate
    lnL / improvement / evaluations and the optimised lengths come back."""
    import torch

    from garli_b200 import engine

    w, c3s, dls, conn = bw
    inst, pop = engine.population_engine(w.data, w.child3, w.dlen, w.model, len(conn), device=device, mixed=True)
    pin = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy() for a in (c3s, dls, conn)]
    pop.score(*pin, args.precision)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    updates = 0
    out = lens = None
    for _ in range(steps):
        out, lens = pop.score(*pin, args.precision)
        updates += pop.counters()["pattern_updates"]
    torch.cuda.synchronize(device)
    dt = time.perf_counter() - t0
    bi = sum(a.nbytes for a in pin)
    bo = out.nbytes + lens.nbytes
    pop.close()
    inst.close()
    return updates / dt, bi, bo


def single_tree(args, device, rank):
    """Secondary: the 128x100k single-tree step, precision and plain forms."""
    w = make_workload(args, seed=1 + rank)
    plain = run_form(w, args, mixed=False, device=device, steps=2, warmup=1)
    mixed = run_form(w, args, mixed=True, device=device, steps=4, warmup=2)
    kt = mixed["kt"]
    v = mixed["tot"]["pattern_updates"] / (mixed["ms"] / 1000.0)
    pv = plain["tot"]["pattern_updates"] / (plain["ms"] / 1000.0)
    res = {"metric": SINGLE_METRIC, "workload": w.name, "npat": w.data.npat, "value": v, "unit": UNIT,
           "ms_per_step": mixed["ms"] / 4, "phases": mixed["phases"],
           "lnl_evals_per_s": (mixed["tot"]["scores"] + mixed["tot"]["edge_evals"]) / (mixed["ms"] / 1000.0),
           "plain_fp64": {"value": pv, "ms_per_step": plain["ms"] / 2, "phases": plain["phases"]},
           "mixed_over_plain": v / pv, "abs_dlnl_mixed_vs_plain": abs(mixed["lnl"] - plain["lnl"]),
           "cla_kernel_gbs": (kt["cla_bytes"] / (kt["cla_ms"] / 1000.0) / 1e9) if kt and kt["cla_ms"] > 0 else None}
    for f in (plain, mixed):
        f["tree"].close()
        f["inst"].close()
    return res


def nstate_forms(kind, device, reps=3):
    """Secondary: full-tree rescore of the 20-state (64 taxa x 20,000 sites, +G4)
    or 61-state (32 taxa x 5,000 codons) alignment in the precision form with the
    tensor-core CLA update, the same form on CUDA cores, and the plain FP64 form;
    CLA site-updates/s (device-timed) and each form's lnL against plain FP64."""
    import torch

    from garli_b200 import engine, synth

    w = synth.aa() if kind == "aa" else synth.codon()
    out = {"workload": w.name, "npat": w.data.npat, "states": w.data.nstates, "categories": w.model.ncat}
    ref = None
    for name, mixed, tc in (("plain_fp64", False, False), ("precision_tensor_cores", True, True),
                            ("precision_cuda_cores", True, False)):
        inst, tree = engine.tree_engine(w.data, w.child3, w.dlen, w.model, device=device, mixed=mixed)
        if mixed:
            inst.set_tensor_cores(tc)
        stream = torch.cuda.ExternalStream(inst.stream_ptr(), device=f"cuda:{device}")
        tree.make_all_dirty()
        lnl = tree.score(0)
        c0 = tree.counters()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        e0.record(stream)
        for _ in range(reps):
            tree.make_all_dirty()
            tree.score(0)
        e1.record(stream)
        torch.cuda.synchronize(device)
        ms = e0.elapsed_time(e1)
        upd = tree.counters()["pattern_updates"] - c0["pattern_updates"]
        if ref is None:
            ref = lnl
        out[name] = {"site_updates_per_s": upd / (ms / 1000.0), "ms_per_rescore": ms / reps, "lnl": lnl,
                     "dlnl_vs_plain": lnl - ref}
        tree.close()
        inst.close()
    return out


def _oracle_candidate(w, c3, dl, X, prec, orc, repeats=1):
    """GARLI's CPU path for one candidate: the tree is built and scored (the
    parent's CLAs), the move's branches are touched so the CLAs GARLI would
    recompute are dirty (SweepDirtynessOverTree), then -- timed -- the rescore,
    the three Newton optimisations and the final score; ``repeats`` times from
    the same starting lengths.  Returns (seconds, CLA ops)."""
    ot = orc.OracleTree(w.data, c3, dl, w.model, fast=True)
    ot.score(0)
    order = [int(c3[X][0]), int(X), int(c3[X][2])]
    tt = 0.0
    ops = 0
    for _ in range(repeats):
        for nd in order:
            ot.set_branch_length(nd, float(dl[nd]))
        c0 = ot.counts()["cla"]
        t0 = time.perf_counter()
        ot.score(0)
        for nd in order:
            ot.optimize_branch(nd, prec)
        ot.make_all_dirty()
        ot.score(int(X))
        tt += time.perf_counter() - t0
        ops += ot.counts()["cla"] - c0
    ot.close()
    return tt, ops


def cpu_baseline(args, bw):
    """GARLI's CPU path (oracle restatement, GARLI's gcc flags, OpenMP over
    patterns on all cores) on a bounded sample of the generation."""
    from oracle import oracle as orc

    w, c3s, dls, conn = bw
    cores = os.cpu_count() or 1
    orc.set_threads(cores, fast=True)
    k = min(args.cpu_sample_cands, len(conn))
    tt = 0.0
    ops = 0
    reps = max(1, args.cpu_repeats)
    for i in range(k):
        dt, o = _oracle_candidate(w, c3s[i], dls[i], int(conn[i]), args.precision, orc, repeats=reps)
        tt += dt
        ops += o
    return {"value": ops * w.data.npat / tt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{k} of {len(conn)} candidates x {reps} repeats ({w.data.npat} patterns): dirty-CLA "
                      f"rescore + 3-branch Newton + final score each, {tt:.1f} s timed"}


def reference_arm(args, ws, rank):
    if rank != 0:
        return
    from oracle import oracle as orc

    bw = batch_workload(args, seed=4)
    w, c3s, dls, conn = bw
    cores = os.cpu_count() or 1
    orc.set_threads(cores, fast=True)
    per = max(1, args.ref_cands_per_step)
    nxt = 0

    def step():
        nonlocal nxt
        t = 0.0
        o = 0
        for _ in range(per):
            i = nxt % len(conn)
            nxt += 1
            dt, ops = _oracle_candidate(w, c3s[i], dls[i], int(conn[i]), args.precision, orc)
            t += dt
            o += ops
        return t, o

    for _ in range(args.warmup):
        step()
    tt = 0.0
    ops = 0
    for _ in range(max(1, args.steps)):
        dt, o = step()
        tt += dt
        ops += o
    v = ops * w.data.npat / tt
    steps = max(1, args.steps)
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": steps, "warmup": args.warmup, "ms_per_step": 1000 * tt / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": w.name, "ntax": args.batch_ntax, "nsites": args.batch_nsites,
                       "npat": w.data.npat, "candidates": len(conn), "model": "GTR+G4",
                       "form": "GARLI CPU path, FP64, one candidate at a time", "parallelism": "openmp-patterns"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{per} candidate(s) per step (cycling through the generation): dirty-CLA "
                                       "rescore + 3-branch Newton + final score each"},
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
    peak, peak_kind = peaks()
    if args.single_only:
        res = single_tree(args, device, rank)
        if rank == 0:
            print(json.dumps({"single_only": True, "single_tree": res}))
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return
    if args.nstate_only:
        res = {"aa_20_states": nstate_forms("aa", device), "codon_61_states": nstate_forms("codon", device)}
        if rank == 0:
            print(json.dumps({"nstate_only": True, "nstate": res}))
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return
    bw = batch_workload(args, seed=4 + rank)
    w, c3s, dls, conn = bw

    if args.batch_only:
        r = run_batch(bw, args, device, mixed=True, sequential=False, steps=args.steps, warmup=args.warmup)
        if rank == 0:
            print(json.dumps({"batch_only": True, "value": r["updates"] / (r["ms"] / 1000.0), "unit": UNIT,
                              "ms_per_step": r["ms"] / args.steps, "npat": w.data.npat,
                              "alg_bytes_per_launch": r["counters"]["alg_bytes"], "tuning": r["tuning"]}))
        r["pop"].close()
        r["inst"].close()
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return
    # plain FP64 per-tree path (GARLI's way), same generation
    plain = run_batch(bw, args, device, mixed=False, sequential=True, steps=max(1, args.steps // 20), warmup=1)
    # headline: batched precision form
    if pg:
        pg.barrier()
    torch.cuda.synchronize(device)
    clk = ClockSampler(device)
    mixed = run_batch(bw, args, device, mixed=True, sequential=False, steps=args.steps, warmup=args.warmup,
                      clocks=clk)
    torch.cuda.synchronize(device)
    if pg:
        pg.barrier()
    from garli_b200.replicas import aggregate

    ms, (updates, edges) = aggregate(pg, mixed["ms"], [mixed["updates"], mixed["edges"]])
    value = updates / (ms / 1000.0)
    plain_v = plain["updates"] / (plain["ms"] / 1000.0)
    mixed["bw"] = bw
    roof = batch_kernel_roofline(mixed, args, peak, peak_kind)
    d0 = float(np.abs(mixed["out"][:, 0] - plain["out"][:, 0]).max())
    d1 = float(np.abs(mixed["out"][:, 1] - plain["out"][:, 1]).max())
    dlen = float(np.max(np.abs(mixed["lens"] - plain["lens"]) / np.maximum(plain["lens"], 1e-8)))
    tuning = mixed["tuning"]
    cnt = mixed["counters"]
    for f in (plain, mixed):
        f["pop"].close()
        f["inst"].close()
    e2e_v, bi, bo = e2e_batch(bw, args, device, max(3, args.steps // 4))
    _, (e2e_v,) = aggregate(pg, 0.0, [e2e_v])
    single = None if args.no_single else single_tree(args, device, rank)
    nstate = None if args.no_single else {"aa_20_states": nstate_forms("aa", device),
                                          "codon_61_states": nstate_forms("codon", device)}
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args, bw)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32-cla/f64-coef-sums-newton",
            "data": "synthetic (seeded)",
            "config": {"workload": w.name, "ntax": args.batch_ntax, "nsites": args.batch_nsites,
                       "npat": w.data.npat, "candidates": len(conn), "moves": "SPR radius U{1..8} (1 = NNI)",
                       "model": "GTR+G4", "form": "batched precision (FP32 CLAs, pow2 scalers, FP64 Newton)",
                       "step": "one generation: dirty-CLA rescore + 3-branch Newton + final score per candidate",
                       "cla_updates_per_step": cnt["cla_ops"], "l2": "working set > L2 (coefficients 0.97 GB)",
                       "tuning": tuning, "parallelism": f"replicas{ws}"},
            "lnl_evals_per_s": edges / (ms / 1000.0),
            "plain_per_tree": {"value": plain_v, "unit": UNIT, "form": "plain FP64, per candidate, host Newton loop",
                               "ms_per_step": plain["ms"] / max(1, args.steps // 20),
                               "lnl_evals_per_s": plain["edges"] / (plain["ms"] / 1000.0)},
            "mixed_over_plain": (value / ws) / plain_v,
            "max_abs_dlnl_vs_plain": {"rescore": d0, "optimised": d1, "max_rel_dlen": dlen},
            "gpu_launches": mixed["launches"],
            "e2e": {"value": e2e_v, "unit": UNIT, "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo},
            "roofline": roof,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "single_tree": single,
            "nstate": nstate,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
