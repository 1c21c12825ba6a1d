"""Multi-rank plumbing of batched problems and blocks of right-hand sides, on
the CPU with gloo (world size 2): largest-first partition of problems,
contiguous split of columns, no collective on the data path, a final gather;
the ranks run real AMG-PCG solves (the oracle's, on the CPU)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from chronoslab_b200.sharding import partition_largest_first, split_columns


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


def test_split_columns():
    assert split_columns(16, 1) == [(0, 16)]
    assert split_columns(16, 3) == [(0, 6), (6, 11), (11, 16)]
    assert split_columns(2, 4) == [(0, 1), (1, 2), (2, 2), (2, 2)]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class _CpuBatch:
    """CPU stand-in for the GPU Batch in multi-rank tests: each problem solved
    by the oracle's PCG_CJ (C, one thread) on the hierarchy built with the
    reference's FSAI/BAMG C++."""

    def __init__(self, As):
        from oracle import amg_oracle as O
        from oracle import c_oracle as CO
        prm = O.default_params()
        prm["tspace"]["ntv"] = 1
        self.H = [CO.CHierarchy(CO.reference_hierarchy(A, None, prm), threads=1) for A in As]

    def solve(self, bs, itmax=1000, tol=1e-8):
        xs, its, fls = [], [], []
        for H, b in zip(self.H, bs):
            x, it, _, flag = H.pcg(b, itmax=itmax, tol=tol)
            xs.append(x)
            its.append(it)
            fls.append(flag)
        return xs, its, fls, 0.0


def _problems():
    from chronoslab_b200 import problems as PB
    rng = np.random.default_rng(3)
    As, bs = [], []
    for p, e in enumerate(rng.integers(6, 13, 7)):
        A = PB.poisson7(int(e)) if p % 2 == 0 else PB.diffusion7(int(e), seed=p)[0]
        As.append(A)
        bs.append(PB.uniform_rhs(A.shape[0], seed=50 + p))
    return As, bs


def _run_sharded(world, rank, dist):
    from chronoslab_b200 import problems as PB
    from chronoslab_b200.sharding import ShardedBatch, ShardedBlock
    As, bs = _problems()
    sb = ShardedBatch(As, world, rank, dist, make_batch=_CpuBatch)
    res, times = sb.solve(bs)
    A = PB.diffusion7(10, seed=9)[0]
    B = PB.uniform_rhs(A.shape[0], seed=10, ncols=5)
    blk = ShardedBlock(A, B.shape[1], world, rank, dist, make_block=_CpuBlockOf)
    cres, ctimes = blk.solve(B)
    return sb.parts, res, times, blk.ranges, cres


class _CpuBlockOf(_CpuBatch):
    """CPU stand-in for a Hierarchy's pcg_block: the columns one by one."""

    def __init__(self, A):
        super().__init__([A])

    def pcg_block(self, B, itmax=1000, tol=1e-8):
        H = self.H[0]
        xs, its, fls = [], [], []
        for j in range(B.shape[1]):
            x, it, _, flag = H.pcg(B[:, j], itmax=itmax, tol=tol)
            xs.append(x)
            its.append(it)
            fls.append(flag)
        return np.stack(xs, axis=1), its, fls, 0.0


def _worker(rank, world, port, out_dir):
    import pickle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out = _run_sharded(world, rank, dist)
        with open(os.path.join(out_dir, f"rank{rank}.pkl"), "wb") as f:
            pickle.dump(out, f)
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_sharded_solves_match_one_rank(tmp_path):
    """A batch of 7 independent problems and a block of 5 right-hand sides,
    each solved for real (the oracle's AMG-PCG on the CPU), split over two
    gloo ranks: every rank ends with every unit's result, each rank solved
    only its share, and the merged results equal one rank's solving all."""
    import pickle
    from oracle import amg_oracle as O
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn",
                       join=True)
    outs = [pickle.load(open(tmp_path / f"rank{r}.pkl", "rb")) for r in range(2)]
    one = _run_sharded(1, 0, None)
    parts, res1, _, ranges, cres1 = one
    assert len(parts) == 1 and len(ranges) == 1
    for r, (parts2, res2, times2, ranges2, cres2) in enumerate(outs):
        assert sorted(times2) == [0, 1]
        assert sorted(i for p in parts2 for i in p) == list(range(len(res1)))
        assert ranges2 == [(0, 3), (3, 5)]
        for units1, units2 in ((res1, res2), (cres1, cres2)):
            assert sorted(units2) == sorted(units1)
            for i in units1:
                assert units2[i]["iters"] == units1[i]["iters"] and units2[i]["flag"] == 0
                assert np.array_equal(units2[i]["x"], units1[i]["x"])


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
