"""Parity at the benchmark configurations, against the oracle answers in
tests/golden/large.json (tests/golden/make_golden_large.py; the CPU
restatement, itself pinned to the reference on the smaller fixtures, with an
independent cross-check where one exists):

  * triangle counting on RMAT-24 seed 5 (src/main.cpp:69-90): the uint64 count
    bit-exact under both schedules (plus RMAT-18 seed 1 and RMAT-20 seed 2);
  * k-truss k=5 on RMAT-20 seed 2 (src/main.cpp:94-141): iteration count, nnz
    and an order-sensitive hash of the edge set bit-exact;
  * batched BC on RMAT-18 seed 3 with 512 sources drawn with seed 4
    (include/betweenness_centrality.h:406-506, FP64): 4,160 stored scores within
    1e-12 relative with no absolute term (exact zeros stay exact), the number
    and positions of all zero scores, four positive random projections of the
    whole score vector and its sum within 1e-12 relative.
"""
import json
import math
import os

import numpy as np
import pytest

from tests import graphs as G
from tests.golden.make_golden import edge_hash
from tests.golden.make_golden_large import BC_PROJ_SEEDS, bc_projection, index_hash

pytestmark = pytest.mark.gpu

LARGE = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "large.json")))
BC_RTOL = 1e-12


@pytest.mark.parametrize("case", LARGE["tc"], ids=lambda c: f"rmat{c['scale']}_seed{c['seed']}")
def test_tc_benchmark_graphs_match_oracle(gk, cuda, case):
    import torch
    from graphkokkos_b200 import sched
    A = gk.gen_rmat(case["scale"], case["edge_factor"], seed=case["seed"], device="cuda")
    assert A.nnz == case["nnz_sym"]
    L = gk.extract_lower(A)
    del A
    torch.cuda.empty_cache()
    assert L.nnz == case["nnz_lower"]
    assert gk.tc_count(L, sched="plain") == case["triangles"]
    sched.load_model()
    assert gk.tc_count(L, sched="learned") == case["triangles"]


def test_ktruss_rmat20_matches_oracle(gk, cuda):
    case = LARGE["ktruss"][0]
    A = gk.gen_rmat(case["scale"], case["edge_factor"], seed=case["seed"], device="cuda")
    assert A.nnz == case["nnz_in"]
    for sched in ("plain", "learned"):
        if sched == "learned":
            from graphkokkos_b200 import sched as s
            s.load_model()
        T, iters = gk.ktruss(A, case["k"], sched=sched)
        assert iters == case["iterations"]
        assert T.nnz == case["nnz"]
        rp = T.rowptr.cpu().numpy()
        col = T.col[:T.nnz].cpu().numpy()
        assert edge_hash(rp, col) == case["xor_hash"]


def test_bc_rmat18_512_sources_matches_oracle(gk, cuda):
    case = LARGE["bc"][0]
    A = gk.gen_rmat(case["scale"], case["edge_factor"], seed=case["seed"], device="cuda")
    assert A.nnz == case["nnz"]
    src = np.random.default_rng(case["src_seed"]).choice(A.m, size=case["nsrc"], replace=False)
    assert index_hash(src) == case["sources_hash"]
    from graphkokkos_b200 import sched
    sched.load_bc_model()
    for s in ("plain", "learned"):
        bc = gk.bc_batch(A, src, sched=s).cpu().numpy()
        idx = np.asarray(case["spot_index"])
        G.assert_bc_close(bc[idx], np.asarray(case["spot_value"]), BC_RTOL)
        zeros = np.flatnonzero(bc == 0.0)
        assert len(zeros) == case["zeros"] and index_hash(zeros) == case["zeros_hash"]
        for p, seed in zip(case["projections"], BC_PROJ_SEEDS):
            assert p["seed"] == seed
            got = bc_projection(bc, seed)
            assert abs(got - p["value"]) <= BC_RTOL * abs(p["value"]), (seed, got, p["value"])
        total = math.fsum(bc.tolist())
        assert abs(total - case["total"]) <= BC_RTOL * case["total"]
