"""Multi-process and CPU-side parts of the benchmark contract (no GPU).

* N > 1 runs independent replicas: the only exchange is the max-over-ranks time
  and the summed work (garli_b200.replicas.aggregate), checked with two gloo ranks.
* ``bench.py --impl reference`` times GARLI's CPU path (the oracle's GARLI-flag
  build) and prints the contract's JSON line.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from garli_b200.replicas import aggregate

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    ms, work = aggregate(dist, 10.0 * (rank + 1), [rank + 1.0, 2.0])
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, ms, work))


def test_two_replicas_take_max_time_and_sum_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, work in res:
        assert ms == 20.0 and work == [3.0, 4.0]


def test_single_process_aggregate_is_identity():
    sys.path.insert(0, ROOT)
    from garli_b200.replicas import aggregate

    assert aggregate(None, 5.0, [1, 2]) == (5.0, [1.0, 2.0])


REF_ARGS = ["--steps", "1", "--warmup", "0", "--ref-cands-per-step", "1", "--batch-nsites", "1500", "--ncand", "4"]


def test_reference_arm_prints_contract_line():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference"] + REF_ARGS,
                         capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "site-updates/s"
    assert line["e2e"]["value"] == line["value"] and line["cpu_baseline"]["kind"] == "port"
    assert line["higher_is_better"] is True and line["steps"] == 1
    assert line["cpu_baseline"]["single_thread"]["cores"] == 1


def test_reference_arm_loads_no_engine_library_and_shares_the_config():
    """The reference arm builds its model with the oracle's math: the engine's
    .so is never mapped in that process, and its config dict is the GPU arm's."""
    code = (
        "import sys, json, io, contextlib; sys.argv = ['bench.py', '--impl', 'reference'] + %r\n"
        "import bench\n"
        "buf = io.StringIO()\n"
        "with contextlib.redirect_stdout(buf): bench.main()\n"
        "line = json.loads(buf.getvalue().strip().splitlines()[-1])\n"
        "maps = open('/proc/self/maps').read()\n"
        "from garli_b200 import synth\n"
        "args = bench.parse()\n"
        "w = synth.batch_workload(seed=4, ntax=args.batch_ntax, nsites=args.batch_nsites, ncand=args.ncand)[0]\n"
        "print(json.dumps({'engine_mapped': 'libgarli_b200' in maps, 'oracle_mapped': 'liboracle' in maps,\n"
        "                  'same_config': line['config'] == json.loads(json.dumps(bench.batch_config(args, w, args.ncand, 1)))}))\n"
    ) % (REF_ARGS,)
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    res = json.loads(out.stdout.strip().splitlines()[-1])
    # the maps are read before the config check builds the workload with the engine's math
    assert not res["engine_mapped"] and res["oracle_mapped"] and res["same_config"]
