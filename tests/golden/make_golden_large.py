"""Generate tests/golden/reference_large.json from the reference's own CPU code.

Full-size fixtures of the benchmark workloads, made by the reference itself
(oracle/_ref/libkdop_ref_record.so: Morton reorder, make_tree, tiny::rotate,
refit_tree and tandem_traversal with MOST_OPPOSING contact generation,
compiled from the reference's sources) and stored as digests, so that the
checked-in file stays a few kilobytes:

  config 2  one pair of 64^3-cell jittered lattices, k = 26
  config 3  512 uneven pairs (1k-200k tets), k = 14
  config 5  256 touching pairs of 20^3-cell lattices, k = 14
  config 4  64 pairs of 40^3-cell lattices at their initial rigid poses
            (the deforming benchmark's meshes before any step), k = 18

Per workload: node-pair tests (total and per pair), the number of candidate
tet pairs (leaf pairs reaching contact generation) with the sha256 of their
canonical list, and the number of FP32 contacts with the sha256 of their
canonical rows.  Canonical forms (shared with the tests, see canonical_*):

  candidates  uint32 rows (pair index, tet of A, tet of B), mesh-local tet
              numbering as given by the caller, sorted lexicographically
  contacts    uint32 rows (pair index, bit patterns of p.x p.y p.z n.x n.y
              n.z depth), sorted lexicographically

Run where the reference sources are present and the harness is built
(`make -C oracle ref`):

    python tests/golden/make_golden_large.py [--threads N]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
for _p in (ROOT, os.path.join(ROOT, "bvh-tvcg18_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

from kdop_b200 import scenes  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_large.json")


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def canonical_candidates(pair_idx, tet_a, tet_b) -> np.ndarray:
    rows = np.column_stack([np.asarray(pair_idx, np.uint32), np.asarray(tet_a, np.uint32),
                            np.asarray(tet_b, np.uint32)]).astype(np.uint32).reshape(-1, 3)
    return rows[np.lexsort((rows[:, 2], rows[:, 1], rows[:, 0]))]


def canonical_contacts(pair_idx, p, n, depth) -> np.ndarray:
    f = np.column_stack([np.asarray(p, np.float32).reshape(-1, 3), np.asarray(n, np.float32).reshape(-1, 3),
                         np.asarray(depth, np.float32).reshape(-1, 1)]).astype(np.float32)
    rows = np.column_stack([np.asarray(pair_idx, np.uint32).reshape(-1, 1), f.view(np.uint32)]).astype(np.uint32)
    return rows[np.lexsort(rows.T[::-1])]


WORKLOADS = {
    "config2": lambda: scenes.config2(),
    "config3": lambda: scenes.config3(),
    "config5": lambda: scenes.config5(),
    "config4": lambda: scenes.config4(),
}


def reference_run(R, sc, threads):
    """Every pair of the scene through the reference pipeline, in parallel
    (the harness's counters are thread-local)."""
    def one(i):
        a, b = (int(x) for x in sc.pairs[i])
        A, B = sc.meshes[a], sc.meshes[b]
        return R.traverse(sc.K, A.xyz, sc.quat[a], sc.pos[a], A.tets, B.xyz, sc.quat[b], sc.pos[b], B.tets)

    with ThreadPoolExecutor(max_workers=threads) as ex:
        res = list(ex.map(one, range(len(sc.pairs))))
    tests = np.array([r["tests"] for r in res], np.int64)
    cand = [canonical_candidates(np.full(len(r["pairs"]), i), r["pairs"][:, 0], r["pairs"][:, 1])
            for i, r in enumerate(res)]
    cont = [canonical_contacts(np.full(len(r["contacts"]), i), r["contacts"][:, 0:3], r["contacts"][:, 3:6],
                               r["contacts"][:, 6]) for i, r in enumerate(res)]
    cand = canonical_candidates(*np.concatenate(cand).T) if cand else np.zeros((0, 3), np.uint32)
    cont = np.concatenate(cont)
    cont = cont[np.lexsort(cont.T[::-1])]
    return summary(sc, tests, cand, cont)


def summary(sc, tests_per_pair, cand, cont) -> dict:
    return {"workload": sc.name, "K": int(sc.K), "pairs": int(len(sc.pairs)), "tets": int(sc.n_tets),
            "tests": int(np.sum(tests_per_pair)), "tests_per_pair": [int(t) for t in tests_per_pair],
            "candidates": int(len(cand)), "candidates_sha256": digest(cand),
            "contacts": int(len(cont)), "contacts_sha256": digest(cont)}


def main():
    from oracle.pyoracle import Reference
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--only", default="")
    args = ap.parse_args()
    R = Reference()
    out = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            out = json.load(f)
    for name, make in WORKLOADS.items():
        if args.only and name not in args.only.split(","):
            continue
        t0 = time.time()
        sc = make()
        out[name] = reference_run(R, sc, args.threads)
        print(f"{name}: {out[name]['tests']} tests, {out[name]['candidates']} candidates, "
              f"{out[name]['contacts']} contacts ({time.time() - t0:.1f} s)")
    out["generator"] = ("tests/golden/make_golden_large.py: the reference's CPU path compiled from its sources "
                        "(oracle/_ref/libkdop_ref_record.so), one-chunk trees on Morton-reordered meshes")
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
