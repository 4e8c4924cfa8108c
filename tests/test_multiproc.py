"""The multi-GPU form of the bench is replicas (independent circuits per rank,
no data-path collective): its process-group plumbing -- barrier, max over
ranks of the timed region, rank 0 alone printing -- checked with gloo ranks
on the CPU."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import argparse

    import bench
    dist, r, w, _ = bench.dist_setup(argparse.Namespace(impl="reference"))
    got = bench.max_over_ranks(dist, float(10 * (r + 1)), "cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((r, w, got))


def test_max_over_ranks_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert res == [(0, 2, 20.0), (1, 2, 20.0)]


def test_reference_arm_under_torchrun_two_ranks():
    """`torchrun --nproc-per-node 2 bench.py --impl reference`: rank 0 prints
    one JSON line, the other rank exits 0 without work."""
    env = dict(os.environ, OMP_NUM_THREADS="1")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--ref-step-seconds", "0.5"]
    out = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2 and rec["value"] > 0
    assert rec["e2e"]["h2d_bytes_per_step"] == 0


def test_reference_arm_never_loads_the_product():
    """The reference arm times the oracle only: after a run, neither the
    product package nor its shared library is in the process, and the line
    names the gate mix, the threads and the physical cores."""
    code = (
        "import sys, json, argparse, io, contextlib\n"
        f"sys.path.insert(0, {ROOT!r})\n"
        "import bench\n"
        "buf = io.StringIO()\n"
        "args = argparse.Namespace(impl='reference', gpus=1, steps=1, warmup=1, ref_step_seconds=0.5)\n"
        "with contextlib.redirect_stdout(buf):\n"
        "    bench.run_reference(args)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'line': json.loads(buf.getvalue().strip().splitlines()[-1]),\n"
        "                  'lib': 'libpz_b200' in maps, 'oracle': 'liboracle_pz' in maps,\n"
        "                  'pkg': any(m.startswith('phantom-zone_b200') for m in sys.modules)}))\n")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    rec = json.loads(out.stdout.strip().splitlines()[-1])
    assert not rec["lib"] and not rec["pkg"] and rec["oracle"]
    cb = rec["line"]["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["physical_cores"] >= 1
    assert "gate mix" in cb["sample"] and "and " in cb["sample"]
