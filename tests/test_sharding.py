"""Multi-rank plumbing of batched problems, on the CPU with gloo (world size 2):
largest-first partition, no collective on the data path, a final gather."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from chronoslab_b200.sharding import gather_results, partition_largest_first


def test_partition_balances_and_covers():
    rng = np.random.default_rng(0)
    edges = rng.integers(16, 65, 64)
    w = [int(e) ** 3 * 7 for e in edges]
    for nr in (1, 2, 3, 8):
        parts = partition_largest_first(w, nr)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        loads = [sum(w[i] for i in p) for p in parts]
        # LPT bound: max load <= mean + largest item
        assert max(loads) <= sum(w) / nr + max(w)
        for p in parts:
            assert [w[i] for i in p] == sorted((w[i] for i in p), reverse=True)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, weights, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        parts = partition_largest_first(weights, world)
        # stand-in for each rank's batch solve: per-problem results
        local = {i: {"iters": 3 * i + 1, "rank": rank} for i in parts[rank]}
        merged = gather_results(local, world, dist)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"),
                np.array([[i, merged[i]["iters"], merged[i]["rank"]] for i in sorted(merged)]))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_partition_and_gather(tmp_path):
    weights = [5, 100, 30, 30, 7, 64, 1, 12]
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, weights, str(tmp_path)), nprocs=2,
                       start_method="spawn", join=True)
    r0 = np.load(tmp_path / "rank0.npy")
    r1 = np.load(tmp_path / "rank1.npy")
    assert np.array_equal(r0, r1)
    assert list(r0[:, 0]) == list(range(len(weights)))
    assert list(r0[:, 1]) == [3 * i + 1 for i in range(len(weights))]
    parts = partition_largest_first(weights, 2)
    for i, _, rank in r0:
        assert i in parts[rank]


def test_reference_arm_under_torchrun_two_ranks():
    """bench.py --impl reference launched as the driver launches it for N = 2
    (torchrun, one process per rank, rendezvous on 127.0.0.1): rank 0 alone
    runs the reference's CPU path and prints one JSON line, rank 1 exits 0."""
    import json
    import subprocess
    import sys
    from oracle import amg_oracle as O
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(root, "bench.py"), "--impl", "reference", "--gpus", "2", "--ne", "8",
           "--steps", "1", "--warmup", "3"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["steps"] == 1
    assert d["e2e"]["value"] == d["value"] and d["cpu_baseline"]["value"] == d["value"]
