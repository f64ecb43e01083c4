"""Replica mode of bench.py on two gloo ranks (CPU), launched the way the multi-GPU bench is:
`torch.distributed.run --nnodes=1 --nproc-per-node 2 --master-addr 127.0.0.1`.

A channel does not shard, so N GPUs run N independent replicas. The process group carries
no data: only the barrier around the timed region and the max over ranks of its time. These
tests check that host logic (the rank environment, the barrier, the max over ranks, the
whole-job rate N * K / max time) and that the reference arm's ranks above 0 exit without work.
"""
import json
import os
import socket
import subprocess
import sys

from conftest import ROOT

RANK_SCRIPT = r'''
import importlib.util, json, os, sys, time
spec = importlib.util.spec_from_file_location("bench", os.path.join(sys.argv[1], "bench.py"))
bench = importlib.util.module_from_spec(spec)
spec.loader.exec_module(bench)
world, rank, local = bench.dist_setup(backend="gloo")
assert (world, rank, local) == (int(os.environ["WORLD_SIZE"]), int(os.environ["RANK"]), int(os.environ["LOCAL_RANK"]))
bench.barrier(world)
t0 = time.perf_counter()
time.sleep(0.05 * (rank + 1))                      # ranks of unequal speed
bench.barrier(world)
wall = time.perf_counter() - t0
ms = 100.0 * (rank + 1)                            # a stand-in device time per rank
ms_max = bench.max_over_ranks(ms, world)
rate = bench.replica_rate(world, 50, ms_max)
ref = bench.run_reference(None, world, rank) if rank > 0 else "rank0"
out = {"rank": rank, "world": world, "ms_max": ms_max, "rate": rate, "wall": wall, "ref": ref}
with open(os.path.join(sys.argv[2], f"rank{rank}.json"), "w") as f:
    json.dump(out, f)
import torch.distributed as dist
dist.destroy_process_group()
'''


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_replicas_two_gloo_ranks(tmp_path):
    script = tmp_path / "rank.py"
    script.write_text(RANK_SCRIPT)
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    env["CUDA_VISIBLE_DEVICES"] = ""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           str(script), ROOT, str(tmp_path)]
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=240)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    outs = [json.loads((tmp_path / f"rank{i}.json").read_text()) for i in range(2)]
    for o in outs:
        assert o["world"] == 2
        assert o["ms_max"] == 200.0                    # the slowest rank's time on every rank
        assert o["rate"] == 2 * 50 / 0.2               # N * K / max time
        assert o["wall"] >= 0.1 - 1e-3                 # the closing barrier waited for the slow rank
    assert outs[1]["ref"] is None                      # reference arm: rank 1 does no work


def test_single_rank_is_plain():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_single", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    saved = {k: os.environ.pop(k) for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK") if k in os.environ}
    try:
        assert bench.dist_setup(backend="gloo") == (1, 0, 0)
    finally:
        os.environ.update(saved)
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.replica_rate(1, 3000, 1840.8) == round(3000 / 1.8408, 3)
