"""Generates the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own code (GraphKokkos include/*.h compiled unmodified
against the Kokkos-API shim: oracle/_ref/libgk_ref.so, built by
`make -C oracle ref` where the reference sources are present) on seeded
inputs from the library's host graph builder, and records the outputs.
The large-configuration entries (marked "source": "port") come from the
CPU restatement, which the small entries pin to the reference.

Usage:  python tests/golden/make_golden.py [--large]
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import graphkokkos_b200 as gk  # noqa: E402
import oracle  # noqa: E402
from tests import graphs as G  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def edge_hash(rp, col):
    rows = np.repeat(np.arange(len(rp) - 1, dtype=np.int64), np.diff(rp))
    return int(np.bitwise_xor.reduce((col.astype(np.int64) * 2654435761 + rows) & 0xFFFFFFFF)) if len(col) else 0


def tc_cases(large):
    cases = []
    specs = [(8, 16, 1), (10, 16, 2), (12, 16, 3), (14, 16, 1)]
    for scale, ef, seed in specs:
        A = gk.gen_rmat(scale, ef, seed=seed)
        L = gk.lower_host(A)
        t = oracle.ref_tc(A, "msa")
        assert oracle.ref_tc(A, "mca") == t
        cases.append(dict(scale=scale, edge_factor=ef, seed=seed, nnz_sym=A.nnz, nnz_lower=L.nnz, triangles=t,
                          source="reference"))
        print("tc", scale, seed, t, flush=True)
    if large:
        for scale, seed in [(18, 1), (20, 2), (24, 5)]:
            t0 = time.time()
            A = gk.gen_rmat(scale, 16, seed=seed)
            L = gk.lower_host(A)
            del A
            t = oracle.tc_lower(L)
            cases.append(dict(scale=scale, edge_factor=16, seed=seed, nnz_sym=2 * L.nnz, nnz_lower=L.nnz,
                              triangles=t, source="port"))
            print("tc", scale, seed, t, f"{time.time() - t0:.1f}s", flush=True)
    return cases


def ktruss_cases(large):
    cases = []
    for scale, seed in [(9, 5), (11, 7)]:
        A = gk.gen_rmat(scale, 16, seed=seed)
        for k in (3, 4, 5, 6, 8):
            rp, col, iters = oracle.ref_ktruss(A, k)
            cases.append(dict(scale=scale, edge_factor=16, seed=seed, k=k, iterations=iters, nnz=int(len(col)),
                              xor_hash=edge_hash(rp, col), source="reference"))
            print("ktruss", scale, k, iters, len(col), flush=True)
    if large:
        A = gk.gen_rmat(20, 16, seed=2)
        t0 = time.time()
        rp, col, iters, per = oracle.ktruss(A, 5, record=256)
        cases.append(dict(scale=20, edge_factor=16, seed=2, k=5, iterations=iters, nnz=int(len(col)),
                          xor_hash=edge_hash(rp, col), nnz_per_iteration=[int(x) for x in per], source="port"))
        print("ktruss 20", iters, len(col), f"{time.time() - t0:.1f}s", flush=True)
    return cases


def mxmm_cases():
    cases = []
    for i, (m, k, n, da, db, dm) in enumerate([(50, 40, 60, .1, .1, .2), (200, 150, 180, .03, .05, .05),
                                               (64, 64, 64, .3, .3, .5)]):
        a = (m, k, da, 100 + i)
        b = (k, n, db, 200 + i)
        mm = (m, n, dm, 300 + i)
        A = G.random_csr(*a, values=True)
        B = G.random_csr(*b, values=True)
        M = G.random_csr(*mm)
        c = oracle.ref_mxmm(A, B, M, "msa").astype(np.int64)
        assert np.array_equal(c, oracle.ref_mxmm(A, B, M, "mca"))
        cases.append(dict(A=list(a), B=list(b), M=list(mm), sum=int(c.sum()),
                          weighted_sum=int((c * np.arange(1, len(c) + 1)).sum()), source="reference"))
    return cases


def bc_cases(large):
    cases = []
    for scale, ef, seed, b, sseed in [(8, 8, 3, 32, 4), (10, 8, 6, 64, 7)]:
        A = gk.gen_rmat(scale, ef, seed=seed)
        rng = np.random.default_rng(sseed)
        src = rng.choice(A.m, size=b, replace=False)
        R, perm = oracle.relabel_sources_first(A, src)
        ref = oracle.ref_bc_float(R, b)[perm]
        cases.append(dict(scale=scale, edge_factor=ef, seed=seed, sources=[int(s) for s in src],
                          bc_ref_float=[float(x) for x in ref], source="reference"))
        print("bc", scale, b, flush=True)
    return cases


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--large", action="store_true", help="also the full-size configurations (minutes)")
    args = ap.parse_args()
    if not oracle.ref_available():
        oracle.build(ref=True)
    for name, cases in [("tc.json", tc_cases(args.large)), ("ktruss.json", ktruss_cases(args.large)),
                        ("mxmm.json", mxmm_cases()), ("bc.json", bc_cases(args.large))]:
        with open(os.path.join(OUT, name), "w") as f:
            json.dump({"generator": "tests/golden/make_golden.py", "cases": cases}, f, indent=1)
        print("wrote", name)


if __name__ == "__main__":
    main()
