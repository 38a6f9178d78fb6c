"""The C restatement (oracle/kdop_oracle.c) against the reference's own results
on the full-size benchmark workloads (tests/golden/reference_large.json, made
by tests/golden/make_golden_large.py from the compiled reference).

This closes the chain reference -> restatement at the sizes the benchmark
runs: node-pair tests per pair, the canonical candidate list and the FP32
contact rows of config 2 (one pair of 1.57 M-tet meshes, k = 26), config 3
(512 uneven pairs, k = 14), config 5 (256 touching pairs, 3.5 M contacts,
k = 14) and config 4's 64 pairs of 384 k-tet meshes at their initial rigid
poses (k = 18).  The GPU tests compare the CUDA library with the same digests.
"""
import os

import numpy as np
import pytest

from conftest import canonical_candidates, canonical_contacts, digest
from kdop_b200 import scenes

WORKLOADS = {"config2": scenes.config2, "config3": scenes.config3, "config5": scenes.config5,
             "config4": scenes.config4}


def oracle_summary(oracle, sc, contacts=True):
    worlds = [oracle.rotate(sc.quat[i], sc.pos[i], m.xyz) for i, m in enumerate(sc.meshes)]
    rows, tests_pp, _ = oracle.run_pairs(sc.K, worlds, sc.meshes, sc.pairs, threads=os.cpu_count() or 1)
    cand = canonical_candidates(rows[:, 0], rows[:, 1], rows[:, 2])
    cont = None
    if contacts:
        parts = []
        starts = np.searchsorted(cand[:, 0], np.arange(len(sc.pairs) + 1))
        for p, (a, b) in enumerate(sc.pairs):
            sel = cand[starts[p]:starts[p + 1], 1:]
            if len(sel) == 0:
                continue
            A, B = sc.meshes[a], sc.meshes[b]
            r, _ = oracle.contacts(worlds[a], A.tets, A.surf, worlds[b], B.tets, B.surf, sel, "f")
            parts.append(canonical_contacts(np.full(len(r), p), r[:, 0:3], r[:, 3:6], r[:, 6]))
        cont = np.concatenate(parts) if parts else np.zeros((0, 8), np.uint32)
        cont = cont[np.lexsort(cont.T[::-1])]
    return tests_pp, cand, cont


@pytest.mark.parametrize("name", list(WORKLOADS))
def test_restatement_reproduces_the_reference_at_full_size(oracle, golden_large, name):
    ref = golden_large[name]
    sc = WORKLOADS[name]()
    assert sc.name == ref["workload"] and len(sc.pairs) == ref["pairs"] and sc.n_tets == ref["tets"]
    tests_pp, cand, cont = oracle_summary(oracle, sc)
    assert [int(t) for t in tests_pp] == ref["tests_per_pair"]
    assert int(tests_pp.sum()) == ref["tests"]
    assert len(cand) == ref["candidates"]
    assert digest(cand) == ref["candidates_sha256"]
    assert len(cont) == ref["contacts"]
    assert digest(cont) == ref["contacts_sha256"]
