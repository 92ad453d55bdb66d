"""Generates tests/golden/large.json: oracle answers at the benchmark sizes.

The small fixtures (make_golden.py) come from the reference's own code and pin
the CPU restatement (oracle/gk_oracle.cpp) to it; at the benchmark sizes the
reference under the Kokkos-API shim would take hours, so these entries come
from the pinned restatement ("source": "port"), each cross-checked by a
second, independent CPU algorithm where one exists:

  * triangle counting on RMAT-24 seed 5 (and RMAT-18 seed 1, RMAT-20 seed 2):
    orc_tc_lower (the reference's masked Gustavson product, src/main.cpp:69-90)
    and orc_tc_merge (sorted-list merge) must agree;
  * k-truss k=5 on RMAT-20 seed 2 (src/main.cpp:94-141): edge-set hash, nnz,
    iteration count and nnz per iteration;
  * batched BC on RMAT-18 seed 3 with 512 sources drawn uniformly with seed 4
    (include/betweenness_centrality.h:406-506, FP64): the full score vector is
    2 MB, so the fixture keeps exact FP64 scores of 4,096 vertices drawn with
    seed 12345 plus the 64 highest-scoring vertices, four positive random
    projections sum_v w_v * bc[v] (weights seeds 900..903, summed with
    math.fsum), the number of exact zeros and a hash of their indices.

Usage:  python tests/golden/make_golden_large.py [--only tc|ktruss|bc]
"""
import argparse
import json
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import graphkokkos_b200 as gk  # noqa: E402
import oracle  # noqa: E402
from tests.golden.make_golden import edge_hash  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "large.json")

BC_SPOTS = 4096
BC_SPOT_SEED = 12345
BC_TOP = 64
BC_PROJ_SEEDS = (900, 901, 902, 903)


def bc_projection(bc, seed):
    """sum_v w_v * bc[v] with w uniform in [0, 1) from seed, summed exactly
    rounded (math.fsum)."""
    w = np.random.default_rng(seed).random(len(bc))
    return math.fsum((w * bc).tolist())


def index_hash(idx):
    idx = np.asarray(idx, dtype=np.int64)
    return int(np.bitwise_xor.reduce((idx * 2654435761 + 97) & 0xFFFFFFFF)) if len(idx) else 0


def tc_cases():
    cases = []
    for scale, seed in [(18, 1), (20, 2), (24, 5)]:
        t0 = time.time()
        A = gk.gen_rmat(scale, 16, seed=seed)
        L = gk.lower_host(A)
        nnz_sym = A.nnz
        del A
        t = oracle.tc_lower(L)
        t1 = time.time()
        tm = oracle.tc_merge(L)
        assert t == tm, (scale, seed, t, tm)
        cases.append(dict(scale=scale, edge_factor=16, seed=seed, vertices=L.m, nnz_sym=nnz_sym, nnz_lower=L.nnz,
                          triangles=t, source="port", cross_check="orc_tc_merge"))
        print(f"tc scale {scale} seed {seed}: {t} ({t1 - t0:.1f}s gustavson, {time.time() - t1:.1f}s merge)",
              flush=True)
    return cases


def ktruss_cases():
    t0 = time.time()
    A = gk.gen_rmat(20, 16, seed=2)
    rp, col, iters, per = oracle.ktruss(A, 5, record=256)
    print(f"ktruss 20 k=5: {iters} iterations, nnz {len(col)} ({time.time() - t0:.1f}s)", flush=True)
    return [dict(scale=20, edge_factor=16, seed=2, k=5, nnz_in=A.nnz, iterations=iters, nnz=int(len(col)),
                 xor_hash=edge_hash(rp, col), nnz_per_iteration=[int(x) for x in per], source="port")]


def bc_cases():
    t0 = time.time()
    A = gk.gen_rmat(18, 16, seed=3)
    src = np.random.default_rng(4).choice(A.m, size=512, replace=False)
    bc = oracle.bc_f64(A, src)
    spots = np.random.default_rng(BC_SPOT_SEED).choice(A.m, size=BC_SPOTS, replace=False)
    top = np.argsort(-bc, kind="stable")[:BC_TOP]
    idx = np.unique(np.concatenate([spots, top]))
    zeros = np.flatnonzero(bc == 0.0)
    print(f"bc 18 x 512: {time.time() - t0:.1f}s, max {bc.max():.6g}, zeros {len(zeros)}", flush=True)
    return [dict(scale=18, edge_factor=16, seed=3, nsrc=512, src_seed=4, vertices=A.m, nnz=A.nnz,
                 sources_hash=index_hash(src), spot_index=[int(i) for i in idx],
                 spot_value=[float(bc[i]) for i in idx],
                 projections=[dict(seed=s, value=bc_projection(bc, s)) for s in BC_PROJ_SEEDS],
                 zeros=int(len(zeros)), zeros_hash=index_hash(zeros), total=math.fsum(bc.tolist()),
                 source="port")]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=["tc", "ktruss", "bc"], default=None)
    args = ap.parse_args()
    oracle.build(ref=False)
    data = {"generator": "tests/golden/make_golden_large.py", "tc": [], "ktruss": [], "bc": []}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data.update(json.load(f))
    for name, fn in [("bc", bc_cases), ("ktruss", ktruss_cases), ("tc", tc_cases)]:
        if args.only in (None, name):
            data[name] = fn()
            with open(OUT, "w") as f:
                json.dump(data, f, indent=1)
            print("wrote", name, flush=True)


if __name__ == "__main__":
    main()
