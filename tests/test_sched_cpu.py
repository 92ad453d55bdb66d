"""What the trained scheduler gains over the plain heuristic, on the measured
sweep committed with the model (graphkokkos_b200/sched/sweep.npz): for every
bin of every sweep graph, the time of the variant each method picks, summed.
Runs on the CPU (numpy inference of the committed weights)."""
import os

import numpy as np
import pytest

from graphkokkos_b200 import sched


def have_model():
    return os.path.exists(sched.MODEL_PATH) and os.path.exists(sched.DATA_PATH)


def test_variant_rule_covers_plain_heuristic(gk):
    """Every variant the plain heuristic can pick is admissible for its bin,
    and every bin admits at least the universal variant."""
    nv, nf, nb = sched.dims()
    for b in range(nb):
        assert sched.allowed(b, 6)
        assert any(sched.allowed(b, v) for v in range(nv))


@pytest.mark.skipif(not have_model(), reason="no trained model committed")
def test_learned_beats_plain_on_the_sweep(gk):
    nv, nf, nb = sched.dims()
    w = np.load(sched.MODEL_PATH)["w"].astype(np.float64)
    recs = sched.load_dataset()
    X, Y, M = sched.to_dataset(recs)
    out = sched.forward_numpy(w, X.astype(np.float64), nf, nv)
    picks = sched.choose(out, recs)
    ev = sched.evaluate(recs, picks)
    # the model may not be perfect, but over the whole sweep it must not lose
    assert ev["learned_ms"] <= ev["plain_ms"] * 1.0001, ev
    # and per graph family: triangle counting and k-truss support
    for mode in (0, 1):
        sub = [(r, p) for r, p in zip(recs, picks) if r["mode"] == mode]
        if sub:
            e = sched.evaluate([r for r, _ in sub], [p for _, p in sub])
            assert e["learned_ms"] <= e["plain_ms"] * 1.02, (mode, e)


@pytest.mark.skipif(not have_model(), reason="no trained model committed")
def test_model_file_shape(gk):
    w = np.load(sched.MODEL_PATH)["w"]
    assert w.shape[0] == sched.model_size()
    assert np.all(np.isfinite(w))
    nv, nf, nb = sched.dims()
    assert np.all(w[-nf:] > 0)  # sigma
