"""Benchmark of the B200 likelihood engine (one JSON line on rank 0).

Headline workload (one "step" = one GA generation): 256 candidate trees, each a
64-taxon Yule base tree after one SPR/NNI move (radius ~ U{1..8}), DNA GTR+G4,
50,000 sites (seeded synthetic, GARLI-compressed to unique patterns).  Every
candidate is rescored (its dirty CLAs recomputed, every other CLA shared with
the base tree) and the three branches at its move's connector are optimised by
GARLI's Newton-Raphson (nd->left, nd, nd->right), then scored at the optimised
lengths.  Three forms run on the same generation in the same process:
  * batched precision form (the headline value): the whole generation in one
    CUDA graph (FP32 CLAs, FP64 coefficients, sums and Newton);
  * plain FP64 batched: the whole generation in one pass with GARLI's FP64
    arithmetic;
  * plain FP64 per tree: GARLI's way, one candidate after another, a host
    Newton loop per branch.
The ratios of the first to the third (site-updates/s, lnL evaluations/s and
generation time) are the headline comparison; the second splits it into a
batching share and a precision share.
Metric: CLA site-updates per second (pattern x CLA update; the per-step
partials on the connector count as updates in both forms); lnL evaluations per
second (edge evaluations: Newton derivative evaluations + final scores) beside it.
Secondary objects: the 32-taxon x 2,000-site step (full rescore + all-branch
Newton pass), the 128-taxon x 100,000-site GTR+I+G4 step, and the 20- and
61-state rescores.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times GARLI's CPU path (the oracle restatement, built with
GARLI's -O3 -ffast-math flags, OpenMP over patterns on all host cores) on a
bounded sample of the same generation: per candidate the CLAs GARLI would
recompute after the move, the same three Newton optimisations and the score at
the connector; the engine's library is never loaded in that process.  N > 1
runs N independent replicas (one per GPU, no data-path collective); value = all
replicas' site-updates / max-over-ranks time.
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
    ap.add_argument("--tuning", default="",
                    help="profiling: fixed work-item sizes 'tiles,chunks' of the batched pass (no autotuning)")
    ap.add_argument("--batch-only", action="store_true",
                    help="profiling: only the batched form (no per-tree comparison, no e2e pass)")
    ap.add_argument("--nstate-only", action="store_true",
                    help="profiling: only the 20- and 61-state rescores (tensor cores, CUDA cores, plain)")
    ap.add_argument("--nstate-tile", type=int, default=0,
                    help="profiling: fixed pattern tile of the n-state CUDA-core CLA kernel (no autotuning; "
                         "a profiler's serialised launches would mislead the tile timing)")
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


def fp64_nominal_instr_per_s():
    """Nominal FP64 instruction rate of a B200 (no measured FP64 peak exists
    for this pool): 148 SMs x 64 FP64 lanes x the maximum SM clock; a fused
    multiply-add, a product or a sum is one instruction."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            mhz = float(json.load(f)["sm_max_mhz"])
    except Exception:
        mhz = 1965.0
    return 148 * 64 * mhz * 1e6


def profiled_traffic():
    """Per-launch DRAM bytes of the batched pass kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "batch_kernel_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return None


def batch_workload(args, seed, mathlib=None):
    from garli_b200 import synth

    return synth.batch_workload(seed=seed, ntax=args.batch_ntax, nsites=args.batch_nsites, ncand=args.ncand,
                                mathlib=mathlib)


def batch_config(args, w, ncand, ws):
    """The workload's config: identical in both arms (the implementation and its
    form are reported outside it)."""
    return {"workload": w.name, "ntax": args.batch_ntax, "nsites": args.batch_nsites, "npat": w.data.npat,
            "candidates": ncand, "moves": "SPR radius U{1..8} (1 = NNI)", "model": "GTR+G4",
            "step": "one generation: dirty-CLA rescore + 3-branch Newton + final score per candidate",
            "newton_precision": args.precision,
            "l2": "working set > L2 (CLAs 2.3 MB each, coefficients 0.97 GB)", "parallelism": f"replicas{ws}"}


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
    if args.tuning:
        pop.set_tuning(*[int(x) for x in args.tuning.split(",")])
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
    instance stream (a few extra timed passes), and the same per phase (every
    launch bracketed by its own events, launched without the graph)."""
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
    parts = pop.byte_counters()
    achieved = alg / (ms / 1e3) / 1e9
    # per phase
    pop.set_phase_timing(True)
    p0 = pop.phase_timing()
    for _ in range(n):
        pop.score(c3s, dls, conn, args.precision)
    p1 = pop.phase_timing()
    pop.set_phase_timing(False)
    kernels = {"levels": "k_level4m", "coefficients": "k_coef4m", "sweeps": "k_batch4m"}
    phases = {}
    for k, kname in kernels.items():
        pms = (p1[k]["ms"] - p0[k]["ms"]) / n
        nl = (p1[k]["launches"] - p0[k]["launches"]) / n
        ach = parts[k] / (pms / 1e3) / 1e9 if pms > 0 else None
        phases[k] = {"kernel": kname, "ms_per_pass": pms, "launches_per_pass": nl,
                     "algorithmic_bytes_per_pass": parts[k], "achieved": ach,
                     "frac": (ach / peak) if ach else None}
    traffic = profiled_traffic()
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic.get("bytes_per_pass") if traffic else None,
            "kernel": "batched pass: k_level4m<4> per CLA level, k_coef4m<4> per step, k_batch4m<4> per "
                      "Newton run (one CUDA graph per generation)",
            "peak_kind": f"{peak_kind} hbm_gbs (burst copy)", "ms_per_pass": ms,
            "algorithmic_bytes_per_pass": alg, "phases": phases,
            "traffic_note": traffic.get("note") if traffic else "no ncu capture committed"}


def e2e_batch(r, args, device, steps, clocks=None):
    """The generation through the public call with host buffers, on the
    headline's population right after its timed loop, for as many generations
    and with the same clock sampler running: candidate topologies, lengths and
    connectors go in from pinned host memory, per-candidate lnL / improvement /
    evaluations and the optimised lengths come back; wall-clock time."""
    import torch

    _, c3s, dls, conn = r["bw"]
    pop = r["pop"]
    pin = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy() for a in (c3s, dls, conn)]
    pop.score(*pin, args.precision)
    torch.cuda.synchronize(device)
    updates = 0
    out = lens = None
    ctx = clocks if clocks is not None else _Null()
    with ctx:
        t0 = time.perf_counter()
        for _ in range(steps):
            out, lens = pop.score(*pin, args.precision)
            updates += pop.counters()["pattern_updates"]
        torch.cuda.synchronize(device)
        dt = time.perf_counter() - t0
    bi = sum(a.nbytes for a in pin)
    bo = out.nbytes + lens.nbytes
    return updates / dt, bi, bo, 1000.0 * dt / steps


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


def nstate_forms(kind, device, reps=3, tile=0):
    """Secondary: full-tree rescore of the 20-state (64 taxa x 20,000 sites, +G4)
    or 61-state (32 taxa x 5,000 codons) alignment in the precision form with the
    tensor-core CLA update, the same form on CUDA cores, and the plain FP64 form;
    CLA site-updates/s (device-timed) and each form's lnL against plain FP64;
    then one all-branch Newton pass per form (device-timed)."""
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
        if tile > 0:
            inst.set_cla_tuning(-1, tile)
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
        # CLA kernels alone: algorithmic bytes (by op kind) over their CUDA-event time
        inst.set_kernel_timing(True)
        for _ in range(2):
            tree.make_all_dirty()
            tree.score(0)
        inst.synchronize()
        kt = inst.kernel_timing()
        inst.set_kernel_timing(False)
        gbs = kt["cla_bytes"] / (kt["cla_ms"] / 1000.0) / 1e9 if kt["cla_ms"] > 0 else None
        if ref is None:
            ref = lnl
        out[name] = {"site_updates_per_s": upd / (ms / 1000.0), "ms_per_rescore": ms / reps, "lnl": lnl,
                     "dlnl_vs_plain": lnl - ref, "cla_ms_per_rescore": kt["cla_ms"] / 2, "cla_kernel_gbs": gbs,
                     "cla_hbm_frac": gbs / peaks()[0] if gbs else None}
        if not tc and kt["cla_ms"] > 0:
            # the CUDA-core kernel is FP64-bound: its FP64 instruction rate against the nominal one
            ips = kt["cla_fp64_instr"] / (kt["cla_ms"] / 1000.0)
            out[name]["cla_fp64_instr_per_s"] = ips
            out[name]["cla_fp64_frac_of_nominal"] = ips / fp64_nominal_instr_per_s()
        # edge evaluation with first and second derivatives (the Newton step's
        # input), its kernels device-timed over 20 calls
        nd = w.data.ntax + 3
        tree.derivatives(nd)
        inst.set_kernel_timing(True)
        for _ in range(20):
            tree.derivatives(nd)
        inst.synchronize()
        kt = inst.kernel_timing()
        inst.set_kernel_timing(False)
        out[name]["edge_derivatives_us"] = kt["edge_ms"] * 1e3 / max(1, kt["edge_evals"])
        # one all-branch Newton pass (OptimizeAllBranches, GARLI's branch order and
        # precision 0.01) from the starting lengths, device-timed: CLA updates,
        # edge derivatives, Newton steps; the first pass (untimed) builds the
        # pass's device schedule
        for timed in (False, True):
            for nd in range(1, len(w.dlen)):
                tree.set_branch_length(nd, float(w.dlen[nd]))
            tree.make_all_dirty()
            tree.score(0)
            torch.cuda.synchronize(device)
            e0.record(stream)
            imp, lnl_after = tree.optimize_all_branches(0.01)
            e1.record(stream)
            torch.cuda.synchronize(device)
        out[name]["newton_pass_ms"] = e0.elapsed_time(e1)
        out[name]["newton_pass_lnl"] = lnl_after
        tree.close()
        inst.close()
    return out


def _oracle_candidate(w, c3, dl, X, prec, orc, model, repeats=1):
    """GARLI's CPU path for one candidate: the tree is built and scored (the
    parent's CLAs), the move's branches are touched so the CLAs GARLI would
    recompute are dirty (SweepDirtynessOverTree), then -- timed -- the rescore,
    the three Newton optimisations (nd->left, nd, nd->right) and the score at
    the optimised lengths (Tree::Score at the connector: only CLAs the
    optimisation left dirty are recomputed); ``repeats`` times from the same
    starting lengths.  Returns (seconds, CLA ops)."""
    ot = orc.OracleTree(w.data, c3, dl, model, fast=True)
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
        ot.score(int(X))
        tt += time.perf_counter() - t0
        ops += ot.counts()["cla"] - c0
    ot.close()
    return tt, ops


def _oracle_sample(w, c3s, dls, conn, prec, orc, model, cands, repeats, threads):
    """Candidates ``cands`` of the generation on ``threads`` host threads:
    (site-updates/s, candidates/s, seconds timed)."""
    orc.set_threads(threads, fast=True)
    tt = 0.0
    ops = 0
    for i in cands:
        dt, o = _oracle_candidate(w, c3s[i], dls[i], int(conn[i]), prec, orc, model, repeats=repeats)
        tt += dt
        ops += o
    return ops * w.data.npat / tt, len(cands) * repeats / tt, tt


def cpu_baseline(args, bw):
    """GARLI's CPU path (oracle restatement, GARLI's gcc flags) on a bounded
    sample of the generation: OpenMP over patterns on all host cores (GARLI's
    --enable-openmp build), and one thread (its default build).  The oracle's
    model is built with the oracle's own model math."""
    from oracle import oracle as orc

    w, c3s, dls, conn = bw
    model = w.model_with(orc)
    cores = os.cpu_count() or 1
    k = min(args.cpu_sample_cands, len(conn))
    reps = max(1, args.cpu_repeats)
    v, cps, tt = _oracle_sample(w, c3s, dls, conn, args.precision, orc, model, range(k), reps, cores)
    k1 = min(4, len(conn))
    v1, cps1, tt1 = _oracle_sample(w, c3s, dls, conn, args.precision, orc, model, range(k1), 2, 1)
    return {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "candidates_per_s": cps,
            "sample": f"{k} of {len(conn)} candidates x {reps} repeats ({w.data.npat} patterns): dirty-CLA "
                      f"rescore + 3-branch Newton + score at the connector each, {tt:.1f} s timed",
            "single_thread": {"value": v1, "unit": UNIT, "cores": 1, "candidates_per_s": cps1,
                              "sample": f"{k1} candidates x 2 repeats, {tt1:.1f} s timed"}}


def small_tree(args, device, orc_time=True):
    """The small single-tree step as a measured object: 32 taxa x 2,000 sites, GTR+G4,
    full-tree rescore + one all-branch Newton pass per step, plain FP64 and
    precision forms (device-timed); GARLI's CPU path on the same step beside
    them is timed by the caller."""
    from garli_b200 import synth

    w = synth.dna_small(seed=0)
    out = {"workload": w.name, "npat": w.data.npat}
    for name, mixed, steps in (("plain_fp64", False, 20), ("precision", True, 20)):
        f = run_form(w, args, mixed=mixed, device=device, steps=steps, warmup=3, timing_pass=False)
        secs = f["ms"] / 1000.0
        out[name] = {"ms_per_step": f["ms"] / steps, "site_updates_per_s": f["tot"]["pattern_updates"] / secs,
                     "lnl_evals_per_s": (f["tot"]["scores"] + f["tot"]["edge_evals"]) / secs, "lnl": f["lnl"],
                     "gpu_launches_per_step": f["launches"] / steps}
        f["tree"].close()
        f["inst"].close()
    return out, w


def small_tree_cpu(args, w):
    """GARLI's CPU path on the config-0 step (score + all-branch Newton pass)."""
    from oracle import oracle as orc

    model = w.model_with(orc)
    res = {}
    for label, threads in (("all_cores", os.cpu_count() or 1), ("single_thread", 1)):
        orc.set_threads(threads, fast=True)
        ot = orc.OracleTree(w.data, w.child3, w.dlen, model, fast=True)
        ot.score(0)
        n = 0
        c0 = ot.counts()
        t0 = time.perf_counter()
        while True:
            for nd in range(1, len(w.dlen)):
                ot.set_branch_length(nd, float(w.dlen[nd]))
            ot.make_all_dirty()
            ot.score(0)
            ot.optimize_all_branches(args.precision)
            n += 1
            if time.perf_counter() - t0 > 2.0:
                break
        dt = time.perf_counter() - t0
        c1 = ot.counts()
        ot.close()
        res[label] = {"cores": threads, "ms_per_step": 1000.0 * dt / n,
                      "site_updates_per_s": (c1["cla"] - c0["cla"]) * w.data.npat / dt,
                      "lnl_evals_per_s": (c1["derivs"] - c0["derivs"] + n) / dt}
    return res


def reference_arm(args, ws, rank):
    """GARLI's CPU path on the headline workload.  Nothing of the engine is
    loaded here: the workload's model is built with the oracle's own model math
    (the alignment, trees and candidates are the same arrays as the GPU arm's)."""
    if rank != 0:
        return
    from oracle import oracle as orc

    bw = batch_workload(args, seed=4, mathlib=orc)
    w, c3s, dls, conn = bw
    model = w.model
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
            dt, ops = _oracle_candidate(w, c3s[i], dls[i], int(conn[i]), args.precision, orc, model)
            t += dt
            o += ops
        return t, o

    for _ in range(args.warmup):
        step()
    tt = 0.0
    ops = 0
    steps = max(1, args.steps)
    for _ in range(steps):
        dt, o = step()
        tt += dt
        ops += o
    v = ops * w.data.npat / tt
    k1 = min(2, len(conn))
    v1, cps1, tt1 = _oracle_sample(w, c3s, dls, conn, args.precision, orc, model, range(k1), 1, 1)
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": steps, "warmup": args.warmup, "ms_per_step": 1000 * tt / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": batch_config(args, w, len(conn), ws),
            "form": "GARLI CPU path (oracle restatement, GARLI's -O3 -ffast-math flags), FP64, one candidate "
                    "at a time, OpenMP over patterns",
            "candidates_per_s": per * steps / tt,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{per} candidate(s) per step (cycling through the generation): dirty-CLA "
                                       "rescore + 3-branch Newton + score at the connector each",
                             "single_thread": {"value": v1, "unit": UNIT, "cores": 1, "candidates_per_s": cps1,
                                               "sample": f"{k1} candidates, {tt1:.1f} s timed"}},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "site_update_count": "CLA updates GARLI's path performs per candidate (its Newton loop re-dirties "
                                 "and recomputes CLAs), more than the batched engine's content-keyed plan does "
                                 "for the same candidates: candidates_per_s compares equal work"}
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
        res = {"aa_20_states": nstate_forms("aa", device, tile=args.nstate_tile),
               "codon_61_states": nstate_forms("codon", device, tile=args.nstate_tile)}
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
                              "alg_bytes_per_pass": r["counters"]["alg_bytes"], "tuning": r["tuning"],
                              "launches_per_step": r["launches"] / max(1, args.steps)}))
        r["pop"].close()
        r["inst"].close()
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return
    # plain FP64 per-tree path (GARLI's way: one candidate after another, host Newton loop)
    n_plain = max(3, args.steps // 10)
    plain = run_batch(bw, args, device, mixed=False, sequential=True, steps=n_plain, warmup=1)
    for k in ("pop", "inst"):
        plain.pop(k).close()
    # plain FP64 batched (k_batch4: the whole generation in one pass, GARLI's FP64 arithmetic)
    n_pb = max(3, args.steps // 4)
    pbatch = run_batch(bw, args, device, mixed=False, sequential=False, steps=n_pb, warmup=2)
    for k in ("pop", "inst"):
        pbatch.pop(k).close()
    # headline: batched precision form
    if pg:
        pg.barrier()
    torch.cuda.synchronize(device)
    clk = ClockSampler(device)
    with clk:
        mixed = run_batch(bw, args, device, mixed=True, sequential=False, steps=args.steps, warmup=args.warmup)
        torch.cuda.synchronize(device)
        if pg:
            pg.barrier()
        mixed["bw"] = bw
        # e2e: the same public call from pinned host buffers, same population, as many generations
        e2e_v, bi, bo, e2e_ms = e2e_batch(mixed, args, device, args.steps)
    from garli_b200.replicas import aggregate

    ms, (updates, edges, e2e_sum) = aggregate(pg, mixed["ms"], [mixed["updates"], mixed["edges"], e2e_v])
    value = updates / (ms / 1000.0)
    roof = batch_kernel_roofline(mixed, args, peak, peak_kind)

    def per_s(r, n):
        secs = r["ms"] / 1000.0
        return {"value": r["updates"] / secs, "unit": UNIT, "lnl_evals_per_s": r["edges"] / secs,
                "ms_per_step": r["ms"] / n, "generations_timed": n}

    mine = per_s(mixed, args.steps)
    pt = per_s(plain, n_plain)
    pb = per_s(pbatch, n_pb)

    def diffs(a, b):
        return {"rescore": float(np.abs(a["out"][:, 0] - b["out"][:, 0]).max()),
                "optimised": float(np.abs(a["out"][:, 1] - b["out"][:, 1]).max()),
                "max_rel_dlen": float(np.max(np.abs(a["lens"] - b["lens"]) / np.maximum(b["lens"], 1e-8)))}

    north = {
        "target": "batched precision form >= 10x the plain FP64 per-tree GPU path, |dlnL| <= 1e-4 per tree",
        "plain_per_tree": dict(pt, form="plain FP64, one candidate at a time, host Newton loop"),
        "plain_batched": dict(pb, form="plain FP64, whole generation batched (k_batch4)"),
        "ratio_site_updates": mine["value"] / pt["value"],
        "ratio_lnl_evals": mine["lnl_evals_per_s"] / pt["lnl_evals_per_s"],
        "ratio_generation_time": pt["ms_per_step"] / mine["ms_per_step"],
        "split_generation_time": {"batching (plain batched vs plain per tree)": pt["ms_per_step"] / pb["ms_per_step"],
                                  "precision form (batched precision vs plain batched)":
                                      pb["ms_per_step"] / mine["ms_per_step"]},
        "max_abs_dlnl_vs_plain_per_tree": diffs(mixed, plain),
        "max_abs_dlnl_plain_batched_vs_plain_per_tree": diffs(pbatch, plain),
    }
    tuning = mixed["tuning"]
    cnt = mixed["counters"]
    launches = mixed["launches"]
    for k in ("pop", "inst"):
        mixed.pop(k).close()
    c0, w0 = (None, None) if args.no_single else small_tree(args, device)
    single = None if args.no_single else single_tree(args, device, rank)
    nstate = None if args.no_single else {"aa_20_states": nstate_forms("aa", device),
                                          "codon_61_states": nstate_forms("codon", device)}
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args, bw)
        if c0 is not None:
            c0["cpu_oracle"] = small_tree_cpu(args, w0)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32-cla/f64-coef-sums-newton",
            "data": "synthetic (seeded)",
            "config": batch_config(args, w, len(conn), ws),
            "form": "batched precision (FP32 CLAs, pow2 scalers, FP64 coefficients, sums and Newton)",
            "cla_updates_per_step": cnt["cla_ops"], "tuning": tuning,
            "lnl_evals_per_s": edges / (ms / 1000.0),
            "candidates_per_s": len(conn) * ws * args.steps / (ms / 1000.0),
            "speedup_vs_plain": north,
            "gpu_launches": launches,
            "e2e": {"value": e2e_sum, "unit": UNIT, "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo,
                    "ms_per_step": e2e_ms, "generations_timed": args.steps},
            "roofline": roof,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "small_tree_32x2000": c0,
            "single_tree": single,
            "nstate": nstate,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
