"""The N > 1 launch path on CPU (world size 2, gloo): the path does not shard,
so bench.py runs one replica per rank and only reduces its timing, the
slowest rank's, with a max all-reduce; under torchrun the reference arm runs
on rank 0 alone and the other ranks exit 0 without work."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, values, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = bench.max_over_ranks(dist, values[rank], "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    values = [0.25, 0.75]
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(2, _free_port(), values, out), nprocs=2, join=True)
        assert dict(out) == {0: 0.75, 1: 0.75}


def test_max_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(None, 1.5, "cpu") == 1.5


def test_reference_arm_under_torchrun_prints_one_line():
    import oracle
    if not oracle.ref_available():
        pytest.skip("reference library not built here")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--gpus", "2", "--impl", "reference",
           "--workload", "c1", "--steps", "1", "--warmup", "3"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["iterations"] > 0 and line["value"] > 0
