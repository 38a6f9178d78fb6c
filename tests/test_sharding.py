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
