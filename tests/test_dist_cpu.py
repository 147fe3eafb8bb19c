"""Multi-process paths of bench.py on CPU: two gloo ranks on 127.0.0.1.

The engine's multi-GPU mode is replicas (one independent solve or batch per GPU, no data-path
collective); the only cross-rank steps are the barrier around the timed region and the maximum of
the per-rank times.  These tests run exactly those helpers with world_size 2, check that every rank
draws its own seeded batch instances, and run the reference arm under torchrun, where rank 0 alone
works and prints the one JSON line."""
import json
import os
import socket
import subprocess
import sys
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import argparse
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_init(argparse.Namespace(impl="reference"))
    bench.barrier(w)
    m = bench.allmax(w, 1.5 + r)
    inst = bench.batch_instances(3, [6, 7], bench.SEED + r)
    with open(os.path.join(out_dir, f"r{r}.json"), "w") as f:
        json.dump({"world": w, "max": m, "first_h": float(inst[0][0].oei_a[0, 0])}, f)
    dist.destroy_process_group()


def test_replica_helpers_two_gloo_ranks():
    import torch.multiprocessing as mp
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(2, _free_port(), d), nprocs=2, start_method="spawn", join=True)
        res = [json.load(open(os.path.join(d, f"r{r}.json"))) for r in range(2)]
    assert all(x["world"] == 2 and x["max"] == 2.5 for x in res)
    # replicas: each rank solves its own seeded instances
    assert res[0]["first_h"] != res[1]["first_h"]


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun_prints_one_line():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(x) for x in p.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1 and lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2
    assert lines[0]["value"] > 0
