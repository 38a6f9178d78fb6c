"""Benchmark of the kDOP BVH collision step on B200.

Workload (default): the batched configuration -- 512 mesh pairs of uneven size
(1k-200k tets per mesh, log-uniform), jittered Kuhn lattices, random rigid
poses, k = 14.  One step = the reference's per-step hot path for all pairs:
rigid transform + kDOP refit of every mesh, tandem traversal of every pair
(one persistent launch), MOST_OPPOSING contact generation; captured in one
CUDA graph.  Metric: kDOP node-pair tests per second (the reference's
overlap_dop_dop calls, counted exactly as the reference counts them).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]

N > 1 runs under torch.distributed (one rank per GPU): one workload of
512 x N pairs (the same seeded generator) is split over the ranks by
estimated cost (kdop_b200.sharding.partition), so every GPU holds about one
headline batch (weak scaling) and no data crosses between GPUs on the data
path; the step time is the max over ranks.  --shard instead splits the
node-pair tree of the same pairs over the ranks (strong scaling) and
all-gathers the contact rows to rank 0 over NCCL.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "bvh-tvcg18_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "kDOP tandem-traversal node-pair tests/s, batched vs plain, % of HBM roofline"
UNIT = "node-pair tests/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["cuda", "reference"], default="cuda")
    ap.add_argument("--pairs", type=int, default=0, help="mesh pairs per GPU (config3: 512, config5: 256)")
    ap.add_argument("--workload", default="config3", choices=["config3", "config2", "config4", "config5", "config1"],
                    help="config3 is the headline; the others are the same step on the other configs")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="bounded CPU-baseline sample, seconds")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--opts", default="", help="traversal options key=value,... (skips the autotuner)")
    ap.add_argument("--shard", action="store_true",
                    help="strong scaling: every rank takes the same pairs and traverses its shard of their "
                         "node-pair tree (kdop_traverse_shard); contacts all-gathered to rank 0 each step")
    ap.add_argument("--frontier", type=int, default=16384, help="--shard: frontier node pairs before dealing")
    return ap.parse_args()


# ---- distributed plumbing -------------------------------------------------------
class Dist:
    def __init__(self, backend: str):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            if self.pg.get_backend() == "nccl":
                import torch
                self.pg.barrier(device_ids=[self.local])
                torch.cuda.synchronize()
            else:
                self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        dev = "cuda" if self.pg.get_backend() == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        dev = "cuda" if self.pg.get_backend() == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def gather(self, values) -> list:
        """Every rank's list of numbers, in rank order (all-gather)."""
        if not self.pg:
            return [list(values)]
        import torch
        dev = "cuda" if self.pg.get_backend() == "nccl" else "cpu"
        t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=dev)
        parts = [torch.empty_like(t) for _ in range(self.world)]
        self.pg.all_gather(parts, t)
        return [p.cpu().tolist() for p in parts]

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---- clocks during the timed region ----------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_ready(self, timeout: float = 5.0):
        """Block until nvidia-smi has printed its first sample (its start-up
        takes a few hundred ms), so that the samples cover the timed region."""
        t0 = time.time()
        while self.proc and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.01)

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def shape_key(opts) -> str:
    """The traversal launch shape (every autotuned knob) as one string."""
    o = opts.as_dict()
    return ",".join(f"{k}={o[k]}" for k in ("block_warps", "stack_cap", "init_chunk", "donate_min", "load_group",
                                            "wave_pairs", "smem_carveout"))


def traverse_dram_capture(workload: str, pairs: int, opts):
    """DRAM bytes per node-pair test and L1 data-pipe use of the traversal
    launch, from the ncu capture of the same launch shape on the same
    workload (profiles/traverse_dram.json, keyed by workload and pair count);
    None when no capture of this launch exists, so that no traffic is quoted
    for a launch nobody measured."""
    path = os.path.join(ROOT, "profiles", "traverse_dram.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    return d.get("captures", {}).get(f"{workload}:{pairs}", {}).get(shape_key(opts))


def workload(args, rank: int = 0, world: int = 1):
    """This rank's share of the workload.  The batched configurations are one
    workload of `pairs` per GPU x world pairs, split over the ranks by
    estimated cost (kdop_b200.sharding.partition: largest pair first onto the
    least-loaded rank), so every GPU holds about one headline batch (weak
    scaling).  The single-pair configurations run as replicas."""
    from kdop_b200 import scenes, sharding
    if args.workload == "config2":
        return scenes.config2()
    if args.workload == "config1":
        return scenes.config1()
    if args.workload == "config3":
        total = (args.pairs or 512) * world
        # sizes of every pair first (no mesh built), then only this rank's meshes
        sizes = scenes.config3(n_pairs=total, keep=[]).extra["pair_tets"]
        pairs = np.arange(2 * total, dtype=np.uint32).reshape(-1, 2)
        mine = sharding.partition(pairs, np.repeat(sizes // 2, 2), world)[rank]
        sc = scenes.config3(n_pairs=total, keep=mine)
    else:
        full = (scenes.config5(n_pairs=(args.pairs or 256) * world) if args.workload == "config5" else
                scenes.config4(n_pairs=(args.pairs or 64) * world))
        mine = sharding.partition(full.pairs, [m.n_tets for m in full.meshes], world)[rank]
        sc = scenes.subset(full, mine)
    sc.extra["pairs_total"] = int(len(sc.extra["pair_tets"]) if "pair_tets" in sc.extra else
                                  (args.pairs or (256 if args.workload == "config5" else 64)) * world)
    return sc


def cpu_sample(sc, tests_per_pair, budget_tests):
    """First pairs of the workload whose node-pair tests sum to the budget."""
    n, acc = 0, 0
    for t in tests_per_pair:
        if n > 0 and acc + t > budget_tests:
            break
        acc += int(t)
        n += 1
    return n, acc


def oracle_tests_per_pair(sc, threads=0):
    from oracle.pyoracle import Oracle
    O = Oracle()
    worlds = [O.rotate(sc.quat[i], sc.pos[i], m.xyz) for i, m in enumerate(sc.meshes)]
    _, tpp, _ = O.run_pairs(sc.K, worlds, sc.meshes, sc.pairs, threads=threads)
    return tpp


def reference_time(sc, n_pairs, threads, repeats=1):
    from oracle.pyoracle import RefTimer
    R = RefTimer()
    used = sorted(set(sc.pairs[:n_pairs].ravel().tolist()))
    remap = {m: i for i, m in enumerate(used)}
    meshes = [sc.meshes[m] for m in used]
    pairs = np.array([[remap[a], remap[b]] for a, b in sc.pairs[:n_pairs]], np.uint32)
    sec, contacts = R.time_pairs(sc.K, meshes, sc.quat[used], sc.pos[used], pairs, threads=threads,
                                 repeats=repeats)
    return sec, contacts


def reference_workload(args, world: int):
    """The first pairs of the CUDA arm's whole workload (all of it at one GPU),
    enough for the reference arm's bounded sample."""
    from kdop_b200 import scenes
    if args.workload == "config3":
        total = (args.pairs or 512) * world
        sc = scenes.config3(n_pairs=total, keep=range(min(total, args.pairs or 512)))
    elif args.workload in ("config4", "config5"):
        per = args.pairs or (256 if args.workload == "config5" else 64)
        full = (scenes.config5(n_pairs=per * world) if args.workload == "config5" else
                scenes.config4(n_pairs=per * world))
        sc = scenes.subset(full, range(per))
        total = per * world
    else:
        return workload(args)
    sc.extra["pairs_total"] = total
    return sc


# ---- reference arm ----------------------------------------------------------------
def run_reference(args):
    dist = Dist("gloo")
    if dist.rank != 0:
        dist.close()
        return
    from oracle import pyoracle
    if not pyoracle.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU path not built (oracle/_ref missing)"}))
        return
    threads = os.cpu_count() or 1
    sc = reference_workload(args, dist.world)
    tpp = oracle_tests_per_pair(sc, threads=threads)
    # per step: the workload's first pairs, all of them when they fit, sized
    # so that the whole run takes at most about 3 minutes on all threads (at
    # most 8 s a step)
    per_step_s = min(8.0, 180.0 / max(args.steps + args.warmup, 1))
    n, tests = cpu_sample(sc, tpp, budget_tests=per_step_s * 30e6 * threads)
    reps = args.warmup + max(args.steps, 1)
    secs, _ = reference_time(sc, n, threads, repeats=reps)
    times = (secs if isinstance(secs, list) else [secs])[args.warmup:]
    t = sum(times) / len(times)
    value = tests / t
    total = int(sc.extra.get("pairs_total", len(sc.pairs)))
    sample = (f"all {n} pairs per step" if n == total else f"first {n} of {total} pairs per step") + \
        f" ({tests} node-pair tests), one-chunk trees, pose + refit + tandem traversal with contacts"
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": sc.name, "pairs": total, "K": sc.K,
                       "sample_pairs": n, "threads": threads},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---- CUDA arm, sharded: one workload split over the ranks --------------------------------
def run_cuda_sharded(args):
    import torch

    import kdop_b200 as kd
    from kdop_b200 import sharding

    dist = Dist("nccl")
    torch.cuda.set_device(dist.local)
    sc = workload(args, 0)  # the same pairs on every rank
    ctx = kd.Context(dist.local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    full = ds.traverse_sync(sc.pairs, contacts=True)
    ds.reserve(candidates=int(full.n_candidates * 1.2) + 1024, contacts=int(full.n_contacts * 1.2) + 1024,
               queue=max(full.queue_used * 2, 1 << 20))
    opts = ds.default_opts()
    row_bytes = 32
    cap_rows = int(full.n_contacts * 1.2) + 1024
    mine = torch.empty(cap_rows * row_bytes, dtype=torch.uint8, device="cuda")
    gathered = [torch.empty_like(mine) for _ in range(dist.world)]
    host_rows = torch.empty(cap_rows * row_bytes * dist.world, dtype=torch.uint8).pin_memory()

    def step():
        # poses in from the host, refit, this rank's shard, contacts, then the
        # exchange: every rank's rows to rank 0
        ds.set_poses(sc.quat, sc.pos)
        ds.refit(kd.REFIT_POSE)
        ds.traverse_shard(sc.pairs, dist.rank, dist.world, args.frontier, opts)
        ds.contacts()
        st = ds.stats()
        n = ds.read_contacts_into(mine)
        with torch.cuda.stream(stream):
            cnt = sharding.gather_row_buffers(mine, n, row_bytes, gathered, host_rows, dist.rank)
            stream.synchronize()
        return st.n_tests, sum(cnt)

    for _ in range(args.warmup):
        step()
    ctx.synchronize()
    dist.barrier()
    clocks = ClockSampler(dist.local)
    clocks.start()
    clocks.wait_ready()
    times, tests, rows = [], 0, 0
    launches0 = ctx.launches
    for _ in range(args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        t, rows = step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        tests = t
    clk = clocks.stop()
    ms = sum(times) / len(times)
    ms_max = dist.max(ms)
    total_tests = dist.sum(tests)
    dist.barrier()
    if dist.rank == 0:
        value = total_tests / (ms_max * 1e-3)
        node_bytes = ds.info()["node_bytes"]
        peak, peak_kind = measured_peaks()
        alg = total_tests * 2 * node_bytes / dist.world
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": sc.name, "pairs": int(len(sc.pairs)), "K": sc.K,
                       "parallelism": f"node-pair tree sharded over {dist.world} rank(s) from a "
                                      f"{args.frontier}-pair frontier; contacts all-gathered to rank 0",
                       "tests_per_step": int(total_tests), "contacts": int(rows),
                       "step": "poses H2D, refit, traversal shard, contacts, contact all-gather + D2H"},
            "roofline": {"bound": "hbm", "achieved": alg / (ms_max * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (ms_max * 1e-3) / 1e9 / peak, "traffic": None, "peak_kind": peak_kind,
                         "kernel": "whole step per rank (algorithmic bytes of its share of the tests)"},
            "cpu_baseline": None,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": int(sc.quat.nbytes + sc.pos.nbytes),
                    "d2h_bytes_per_step": int(rows * row_bytes)},
            "gpu_launches": int(ctx.launches - launches0), "clocks": clk,
        }
        print(json.dumps(line))
    # buffers used on the library's stream go before the stream does
    del mine, gathered, host_rows
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    ds.close()
    ctx.close()
    dist.close()


# ---- CUDA arm -------------------------------------------------------------------------
def run_cuda(args):
    import torch

    import kdop_b200 as kd

    dist = Dist("nccl")
    torch.cuda.set_device(dist.local)
    sc = workload(args, dist.rank, dist.world)
    ctx = kd.Context(dist.local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    ds = kd.DeviceScene(ctx, sc.K, sc.meshes)
    info = ds.info()
    ds.set_poses(sc.quat, sc.pos)
    # config 4 deforms and moves every step (motion integrated inside the graph)
    deforming = args.workload == "config4"
    refit_mode = kd.REFIT_DEFORM if deforming else kd.REFIT_POSE
    if deforming:
        ex = sc.extra
        ds.set_deformation(ex["amp"], float(np.float32(2 * np.pi / ex["L"])), 0.0)
        ds.set_motion(ex["lin_vel"], ex["ang_vel"], ex["phase_rate"])
    ds.refit(refit_mode)
    st = ds.traverse_sync(sc.pairs, contacts=True)
    tuned = None
    if args.opts:
        opts = ds.opts(**{k: int(v) for k, v in (kv.split("=") for kv in args.opts.split(","))})
    else:
        if not args.no_autotune:
            tuned = ds.autotune(sc.pairs, repeats=2).as_dict()
        opts = ds.default_opts()
    st = ds.traverse_sync(sc.pairs, opts, contacts=True)
    tests_per_step = st.n_tests
    ds.reserve(candidates=int(st.n_candidates * 1.2) + 1024, contacts=int(st.n_contacts * 1.2) + 1024,
               queue=max(st.queue_used * 2, 1 << 20))

    # one step = pose refit + traversal + contacts in one CUDA graph (config 4:
    # motion update + deforming refit + traversal + contacts)
    ds.graph_capture(sc.pairs, refit_mode=refit_mode, opts=opts, motion=deforming)
    launches0 = ctx.launches
    for _ in range(args.warmup):
        ds.graph_launch()
    ctx.synchronize()
    dist.barrier()
    clocks = ClockSampler(dist.local)
    clocks.start()
    clocks.wait_ready()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ctx.synchronize()
    launches_before = ctx.launches
    if deforming:
        # the state moves every step: time each step, count its own tests
        total_ms, total_tests = 0.0, 0
        for _ in range(args.steps):
            e0.record(stream)
            ds.graph_launch()
            e1.record(stream)
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
            total_tests += ds.stats().n_tests
        ms = total_ms / args.steps
        tests_per_step = total_tests / args.steps
    else:
        e0.record(stream)
        for _ in range(args.steps):
            ds.graph_launch()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
    launches_timed = ctx.launches - launches_before
    clk = clocks.stop()
    dist.barrier()
    st2 = ds.stats()
    state_tests = st2.n_tests  # tests of the state the later timings traverse
    if not deforming:  # a fixed state makes the same tests every step
        assert state_tests == tests_per_step, (state_tests, tests_per_step)
    ms_max = dist.max(ms)
    total_tests = dist.sum(float(tests_per_step))
    value = total_tests / (ms_max * 1e-3)
    per_rank = dist.gather([len(sc.pairs), sc.n_tets, tests_per_step, ms])

    # dominant kernel: the batched traversal launch, timed alone
    reps = 5
    tt = []
    for _ in range(reps + 1):
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        ds.traverse(sc.pairs, opts)
        a1.record(stream)
        a1.synchronize()
        tt.append(a0.elapsed_time(a1))
    trav_ms = statistics.median(tt[1:])
    node_bytes = info["node_bytes"]
    alg_bytes = state_tests * 2 * node_bytes
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (trav_ms * 1e-3) / 1e9
    # DRAM bytes of this launch: the ncu capture of the same launch (shape
    # and workload), per node-pair test
    cap = (traverse_dram_capture(args.workload, int(sc.extra.get("pairs_total", len(sc.pairs))), opts)
           if dist.world == 1 else None)
    traffic = cap["dram_bytes_per_test"] * state_tests if cap else None

    # plain: one traversal launch per mesh pair, same trees and descent rule;
    # the faster of the default and the batched-tuned launch shape
    plain = None
    if not args.no_plain:
        best = None
        for name in ("default", "tuned"):
            if name == "default":
                popts = kd.TraverseOpts()
                ds.lib.kdop_traverse_opts_default(None, popts)
            else:
                popts = kd.TraverseOpts.from_buffer_copy(opts)
            popts.mode = kd.TRAVERSE_PLAIN
            ds.traverse_sync(sc.pairs, popts)
            pt = []
            for _ in range(2):
                a0 = torch.cuda.Event(enable_timing=True)
                a1 = torch.cuda.Event(enable_timing=True)
                a0.record(stream)
                ds.traverse(sc.pairs, popts)
                a1.record(stream)
                a1.synchronize()
                pt.append(a0.elapsed_time(a1))
            pst = ds.stats()
            assert pst.n_tests == state_tests
            if best is None or min(pt) < best[0]:
                best = (min(pt), name, popts.as_dict())
        plain_ms = best[0]
        plain = {"traversal_ms": plain_ms, "tests_per_s": state_tests / (plain_ms * 1e-3),
                 "batched_speedup": plain_ms / trav_ms, "launch_shape": best[1], "opts": best[2]}

    # e2e: through the public API with host buffers, two forms.  Rigid bodies
    # (the reference's narrow_update_kdop_bvh.h:146-171: pose, then refit):
    # per step the poses of all meshes and the pair list go host->device from
    # pinned memory (kdop_set_poses + kdop_refit(POSE)), then traversal and
    # contacts, and the contact rows and counters come back device->host.
    # Deformable bodies: the world positions of all meshes go host->device
    # instead (kdop_set_vertices + kdop_refit(VERTICES), 12 bytes a vertex).
    ds.set_poses(sc.quat, sc.pos)
    ds.refit(kd.REFIT_POSE)
    # the world positions of the posed meshes, as the library's pose refit
    # computes them (read back once, outside the timed region)
    world = ds.read_vertices()
    h_xyz = torch.empty((world.shape[0], 3), dtype=torch.float32, pin_memory=True)
    h_xyz.numpy()[:] = world
    h_quat = torch.empty((len(sc.quat), 4), dtype=torch.float32, pin_memory=True)
    h_quat.numpy()[:] = sc.quat
    h_pos = torch.empty((len(sc.pos), 3), dtype=torch.float32, pin_memory=True)
    h_pos.numpy()[:] = sc.pos
    h_pairs = torch.empty((len(sc.pairs), 2), dtype=torch.int32, pin_memory=True)
    h_pairs.numpy()[:] = sc.pairs.astype(np.int32)
    n_cont_cap = ds.stats().contact_capacity
    h_cont = torch.empty((n_cont_cap * 8,), dtype=torch.float32, pin_memory=True)
    import ctypes

    def e2e_step(vertices: bool):
        if vertices:
            ds.set_vertices(h_xyz.numpy())
            ds.refit(kd.REFIT_VERTICES)
        else:
            ds.set_poses(h_quat.numpy(), h_pos.numpy())
            ds.refit(kd.REFIT_POSE)
        ds.traverse(h_pairs.numpy().view(np.uint32), opts)
        ds.contacts()
        s = ds.stats()
        n = ctypes.c_int64()
        ds.ctx._check(ds.lib.kdop_read_contacts(ds.h, ctypes.c_void_p(h_cont.data_ptr()), n_cont_cap,
                                                ctypes.byref(n)))
        return s, n.value

    def e2e_time(vertices: bool):
        for _ in range(2):
            e2e_step(vertices)
        ctx.synchronize()
        dist.barrier()
        w0 = time.perf_counter()
        b0 = torch.cuda.Event(enable_timing=True)
        b1 = torch.cuda.Event(enable_timing=True)
        b0.record(stream)
        for _ in range(args.e2e_steps):
            s, ncont = e2e_step(vertices)
        b1.record(stream)
        b1.synchronize()
        ms = max(b0.elapsed_time(b1), (time.perf_counter() - w0) * 1e3) / args.e2e_steps
        if not deforming:
            assert s.n_tests == tests_per_step
        ms_max = dist.max(ms)
        # the end-to-end step traverses the rigidly posed meshes (config 4:
        # without its deformation), so it is rated by its own test count
        return dist.sum(float(s.n_tests)) / (ms_max * 1e-3), ms_max, ncont

    e2e_value, e2e_ms_max, ncont = e2e_time(False)
    h2d = h_quat.numpy().nbytes + h_pos.numpy().nbytes + sc.pairs.nbytes
    d2h = ncont * 32 + 128
    e2e_v_value, e2e_v_ms, ncont_v = e2e_time(True)
    h2d_v = world.nbytes + sc.pairs.nbytes

    # CPU baseline: the reference's own CPU path, one thread, bounded sample
    cpu = None
    if dist.rank == 0 and not args.no_cpu_baseline:
        from oracle import pyoracle
        if pyoracle.reference_available():
            tpp = oracle_tests_per_pair(sc)
            n, tests = cpu_sample(sc, tpp, budget_tests=args.cpu_seconds * 30e6)
            sec, _ = reference_time(sc, n, 1)
            cpu = {"value": tests / sec, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"first {n} of {len(sc.pairs)} pairs, one step ({tests} node-pair tests, "
                             f"{sec:.1f} s), rigid transform + refit + tandem traversal with contacts"}
        else:
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                   "sample": "unavailable: oracle/_ref not built"}

    if dist.rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": sc.name, "pairs_per_gpu": [int(r[0]) for r in per_rank],
                       "tets_per_gpu": [int(r[1]) for r in per_rank],
                       "pairs_total": int(sc.extra.get("pairs_total", len(sc.pairs))),
                       "K": sc.K, "node_bytes": node_bytes,
                       "parallelism": (f"{sc.extra.get('pairs_total', len(sc.pairs))} pairs partitioned by cost over "
                                       f"{dist.world} rank(s) (kdop_b200.sharding.partition), no collective on "
                                       f"the data path" if "pair_ids" in sc.extra else
                                       f"one pair, {dist.world} replica(s)"),
                       "tests_per_gpu": [int(r[2]) for r in per_rank],
                       "ms_per_step_per_gpu": [r[3] for r in per_rank],
                       "l2": (f"inputs larger than L2 (node records {info['n_nodes'] * node_bytes / 1e9:.2f} GB)"
                              if info['n_nodes'] * node_bytes > 126e6 else
                              f"inputs fit in L2 (node records {info['n_nodes'] * node_bytes / 1e6:.1f} MB), no flush"),
                       "step": "CUDA graph: pose transform + refit, batched traversal, contacts",
                       "candidates": int(st2.n_candidates),
                       "contacts": int(st2.n_contacts), "traverse_opts": opts.as_dict(), "autotuned": tuned},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "traverse_kernel (batched, one persistent launch)",
                         "launch_ms": trav_ms, "launch_shape": shape_key(opts),
                         "algorithmic_bytes_per_launch": alg_bytes,
                         # three readings side by side: `frac` counts every test's two node
                         # records (most are served by L1/L2: a cache-reuse figure, not HBM);
                         # dram_frac is the DRAM bytes this launch shape really moves (ncu)
                         # over the live launch time; l1_lsu_pct is the busiest unit, the L1
                         # data pipe, as a % of its peak in the same capture
                         "frac_kind": "algorithmic bytes (2 node records per test) / launch time / HBM peak",
                         "dram_gbs": (traffic / (trav_ms * 1e-3) / 1e9) if traffic else None,
                         "dram_frac": (traffic / (trav_ms * 1e-3) / 1e9 / peak) if traffic else None,
                         "l1_lsu_pct": cap["l1_lsu_pct"] if cap else None,
                         "l1_lsu_pct_source": cap.get("l1_lsu_pct_source") if cap else None,
                         "traffic_source": (cap["source"] if cap else
                                            "no ncu capture of this launch shape: traffic not quoted")},
            "plain": plain,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "ms_per_step": e2e_ms_max,
                    "inputs": "per step: poses of every mesh and the pair list H2D (kdop_set_poses, pinned), "
                              "contact rows and counters D2H"},
            "e2e_vertices": {"value": e2e_v_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d_v),
                             "d2h_bytes_per_step": int(ncont_v * 32 + 128), "ms_per_step": e2e_v_ms,
                             "inputs": "per step: world positions of every vertex and the pair list H2D "
                                       "(kdop_set_vertices, pinned), contact rows and counters D2H"},
            "gpu_launches": int(launches_timed),
            "clocks": clk,
        }
        print(json.dumps(line))
    ds.graph_release()
    ds.close()
    ctx.close()
    dist.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_cuda_sharded(args) if args.shard else run_cuda(args)


if __name__ == "__main__":
    main()
