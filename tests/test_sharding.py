"""Multi-rank path on CPU: pairs sharded over 2 gloo ranks, per-rank
traversal (the CPU oracle stands in for the GPU kernel here), gathered rows
equal the unsharded result."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from kdop_b200 import scenes, sharding


def test_partition_covers_every_pair_once_and_balances():
    sc = scenes.config3(n_pairs=64, seed=5)
    tets = [m.n_tets for m in sc.meshes]
    for world in (1, 2, 3, 8):
        parts = sharding.partition(sc.pairs, tets, world)
        allp = np.sort(np.concatenate(parts))
        assert np.array_equal(allp, np.arange(len(sc.pairs)))
        cost = sharding.pair_costs(sc.pairs, tets)
        loads = np.array([cost[p].sum() for p in parts])
        # greedy LPT: no rank above the average by more than the largest pair
        assert loads.max() <= loads.mean() + cost.max()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out_dir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "bvh-tvcg18_b200")]
    import torch.distributed as dist

    from kdop_b200 import scenes, sharding
    from oracle.pyoracle import Oracle

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        sc = scenes.small_batch(n_pairs=10, n_lo=2, n_hi=5, seed=17)
        tets = [m.n_tets for m in sc.meshes]
        mine = sharding.shard(sc.pairs, tets, rank, world)
        O = Oracle()
        worlds = [O.rotate(sc.quat[i], sc.pos[i], m.xyz) for i, m in enumerate(sc.meshes)]
        rows, _, _ = O.run_pairs(sc.K, worlds, sc.meshes, sc.pairs[mine], threads=1)
        allrows = sharding.gather_rows(rows, mine)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), allrows)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_the_unsharded_result(tmp_path, oracle):
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    sc = scenes.small_batch(n_pairs=10, n_lo=2, n_hi=5, seed=17)
    worlds = [oracle.rotate(sc.quat[i], sc.pos[i], m.xyz) for i, m in enumerate(sc.meshes)]
    rows, _, _ = oracle.run_pairs(sc.K, worlds, sc.meshes, sc.pairs, threads=1)
    want = rows.astype(np.int64)
    want = want[np.lexsort((want[:, 2], want[:, 1], want[:, 0]))]
    for r in range(world):
        got = np.load(tmp_path / f"rank{r}.npy")
        assert np.array_equal(got, want)


def test_config3_keep_builds_the_same_pairs():
    """config3(keep=...) skips the other pairs' jitter draws without drawing
    them, so the kept pairs equal the whole scene's."""
    full = scenes.config3(n_pairs=24, seed=13, max_tets=2e4)
    keep = [20, 3, 11, 0]
    part = scenes.config3(n_pairs=24, seed=13, max_tets=2e4, keep=keep)
    assert np.array_equal(part.extra["pair_ids"], keep)
    for k, i in enumerate(keep):
        for s in range(2):
            a, b = full.meshes[full.pairs[i, s]], part.meshes[part.pairs[k, s]]
            assert np.array_equal(a.xyz, b.xyz) and np.array_equal(a.tets, b.tets) and np.array_equal(a.surf, b.surf)
            assert np.array_equal(full.quat[full.pairs[i, s]], part.quat[part.pairs[k, s]])
            assert np.array_equal(full.pos[full.pairs[i, s]], part.pos[part.pairs[k, s]])
    tets = np.array([full.meshes[a].n_tets + full.meshes[b].n_tets for a, b in full.pairs])
    assert np.array_equal(part.extra["pair_tets"], tets)


def _bench_rank_main(rank, world, port, out_dir):
    """One rank of the benchmark's partitioned workload (bench.workload), the
    oracle standing in for the GPU traversal; rows gathered with global pair
    indices."""
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "bvh-tvcg18_b200")]
    import argparse

    import torch.distributed as dist

    import bench
    from kdop_b200 import sharding
    from oracle.pyoracle import Oracle

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        args = argparse.Namespace(workload="config3", pairs=6)
        sc = bench.workload(args, rank, world)
        O = Oracle()
        worlds = [O.rotate(sc.quat[i], sc.pos[i], m.xyz) for i, m in enumerate(sc.meshes)]
        rows, tpp, _ = O.run_pairs(sc.K, worlds, sc.meshes, sc.pairs, threads=1)
        allrows = sharding.gather_rows(rows, sc.extra["pair_ids"])
        np.save(os.path.join(out_dir, f"bench_rank{rank}.npy"), allrows)
        np.save(os.path.join(out_dir, f"bench_ids{rank}.npy"), sc.extra["pair_ids"])
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_run_the_partitioned_benchmark_workload(tmp_path, oracle):
    """bench.py's multi-GPU layout on 2 gloo ranks: one workload of 6 pairs
    per rank x 2, split by estimated cost, every pair on exactly one rank,
    the gathered rows equal to the unsharded workload's."""
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_bench_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    ids = [np.load(tmp_path / f"bench_ids{r}.npy") for r in range(world)]
    assert np.array_equal(np.sort(np.concatenate(ids)), np.arange(12))
    sc = scenes.config3(n_pairs=12)
    worlds = [oracle.rotate(sc.quat[i], sc.pos[i], m.xyz) for i, m in enumerate(sc.meshes)]
    rows, _, _ = oracle.run_pairs(sc.K, worlds, sc.meshes, sc.pairs, threads=4)
    want = rows.astype(np.int64)
    want = want[np.lexsort((want[:, 2], want[:, 1], want[:, 0]))]
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / f"bench_rank{r}.npy"), want)


def _exchange_rank_main(rank, world, port, out_dir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "bvh-tvcg18_b200")]
    import torch
    import torch.distributed as dist

    from kdop_b200 import sharding

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        row_bytes, cap = 32, 16
        n = [5, 0, 11][rank]
        mine = torch.zeros(cap * row_bytes, dtype=torch.uint8)
        for i in range(n):  # row i of rank r: bytes (r, i, 7, 7, ...)
            mine[i * row_bytes: (i + 1) * row_bytes] = 7
            mine[i * row_bytes] = rank
            mine[i * row_bytes + 1] = i
        gathered = [torch.empty_like(mine) for _ in range(world)]
        out = torch.zeros(cap * row_bytes * world, dtype=torch.uint8)
        cnt = sharding.gather_row_buffers(mine, n, row_bytes, gathered, out, rank)
        np.save(os.path.join(out_dir, f"ex_cnt{rank}.npy"), np.array(cnt))
        if rank == 0:
            np.save(os.path.join(out_dir, "ex_out.npy"), out.numpy())
    finally:
        dist.destroy_process_group()


def test_three_gloo_ranks_exchange_sharded_rows(tmp_path):
    """The exchange step of the sharded traversal (bench.py --shard): each
    rank's variable number of fixed-size rows reaches rank 0 packed in rank
    order; every rank learns every rank's count."""
    world = 3
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_exchange_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for r in range(world):
        assert np.load(tmp_path / f"ex_cnt{r}.npy").tolist() == [5, 0, 11]
    out = np.load(tmp_path / "ex_out.npy").reshape(-1, 32)
    want = [(0, i) for i in range(5)] + [(2, i) for i in range(11)]
    assert [(int(a), int(b)) for a, b in out[:16, :2]] == want
    assert (out[:16, 2:] == 7).all() and (out[16:] == 0).all()
