"""Learned row-bin scheduler: autotuner sweep, MLP training on the GPU, model I/O.

The masked SpGEMM engine bins the rows of C<M> = A·B by (log2 nnz(M_i),
log2 mean nnz(B_k)) and runs every bin on one kernel variant (include/gk_b200.h,
graphkokkos_b200/csrc/gk_sched.cuh).  This module

  * sweeps: for every bin of a graph with enough work and every variant the
    bin admits, times that bin alone on that variant (gk_tune_run; CUDA events
    around the variant kernel);
  * builds the training set: per bin the 8 features the model reads
    (gk_sched_bins) and, per variant, log2 of nanoseconds per streamed B entry;
  * trains the MLP with the library's CUDA training kernel (gk_mlp_train);
  * saves / loads the model (graphkokkos_b200/sched/model.npz) and hands it to
    the library (gk_sched_set_model).

The model changes only which variant runs a bin; every variant computes the
same integer terms, so results stay bit-exact.

The same network (its outputs 0 and 1) also picks the forward-level shape of
batched BC, pull or push (graphkokkos_b200/csrc/bc.cu): the BC sweep times
every forward level of seeded runs both ways (gk_bc_tune) and the model is
trained on log2 microseconds per level, saved as sched/bc_model.npz and handed
to the library with gk_bc_set_model.

  python -m graphkokkos_b200.sched --train          # sweep the training graphs, train, save
  python -m graphkokkos_b200.sched --train-bc       # the same for the BC level shapes
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import re
import time

import numpy as np

from . import _lib
from ._lib import check

HERE = os.path.dirname(os.path.abspath(__file__))
MODEL_DIR = os.path.join(HERE, "sched")
MODEL_PATH = os.path.join(MODEL_DIR, "model.npz")
DATA_PATH = os.path.join(MODEL_DIR, "sweep.npz")
BC_MODEL_PATH = os.path.join(MODEL_DIR, "bc_model.npz")
BC_DATA_PATH = os.path.join(MODEL_DIR, "bc_sweep.npz")
BC_PULL, BC_PUSH = 0, 1

MLP_H = 32


def dims():
    lib = _lib.load()
    return int(lib.gk_sched_num_variants()), int(lib.gk_sched_num_features()), int(lib.gk_sched_num_bins())


def model_size():
    return int(_lib.load().gk_sched_model_size())


# ---------------------------------------------------------------------------
# model I/O
# ---------------------------------------------------------------------------
MODEL_MAGIC = b"GKMLP001"


def bin_path(npz_path):
    """The model file (gk_sched_load_model_file layout) beside a .npz model."""
    return os.path.splitext(npz_path)[0] + ".bin"


def write_model_bin(w, path):
    """Model file read by gk_sched_load_model_file / gk_bc_load_model_file:
    magic, little-endian uint32 count, little-endian float32 weights."""
    w = np.ascontiguousarray(w, dtype="<f4")
    with open(path, "wb") as f:
        f.write(MODEL_MAGIC + np.uint32(w.shape[0]).astype("<u4").tobytes() + w.tobytes())


def read_model_bin(path):
    raw = open(path, "rb").read()
    if raw[:8] != MODEL_MAGIC:
        raise ValueError(f"{path} is not a scheduler model file")
    n = int(np.frombuffer(raw[8:12], dtype="<u4")[0])
    return np.frombuffer(raw[12:12 + 4 * n], dtype="<f4").astype(np.float32)


def widen_outputs(w, nv_old, nv_new, bias, nf=8, h=32):
    """A model of nv_old outputs as one of nv_new: the new outputs get zero
    weights and the given bias (a large bias: a variant predicted never to
    win, so that the widened model keeps the old choices until it is
    retrained with timings of the new variants)."""
    w = np.asarray(w, dtype=np.float32)
    o = h * nf + h + h * h + h
    W3 = w[o:o + nv_old * h].reshape(nv_old, h)
    b3 = w[o + nv_old * h:o + nv_old * h + nv_old]
    tail = w[o + nv_old * h + nv_old:]
    assert tail.shape[0] == 2 * nf
    W3n = np.concatenate([W3, np.zeros((nv_new - nv_old, h), dtype=np.float32)])
    b3n = np.concatenate([b3, np.full(nv_new - nv_old, bias, dtype=np.float32)])
    return np.concatenate([w[:o], W3n.ravel(), b3n, tail]).astype(np.float32)


def load_model(path=MODEL_PATH):
    """Loads the learned row-bin model through the library's file loader (the
    call a C or C++ host makes); `path` may name the .npz or the .bin."""
    path = bin_path(path)
    check(_lib.load().gk_sched_load_model_file(path.encode()))
    return read_model_bin(path)


def load_bc_model(path=BC_MODEL_PATH):
    """Loads the learned BC forward-shape model (gk_bc_load_model_file)."""
    path = bin_path(path)
    check(_lib.load().gk_bc_load_model_file(path.encode()))
    return read_model_bin(path)


def save_model(w, path=MODEL_PATH, **meta):
    """Writes the model as .npz (weights and training metadata) and as the
    .bin model file the library loads."""
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez(path, w=np.asarray(w, dtype=np.float32), meta=json.dumps(meta))
    write_model_bin(w, bin_path(path))


# ---------------------------------------------------------------------------
# bins and the sweep
# ---------------------------------------------------------------------------
def bins(G, mode):
    """Per-bin statistics (rows, sum_m, sum_a, sum_work, max_b), plain choice and
    features of C<G> = G·G (mode 0: triangle counting on L; mode 1: k-truss support)."""
    lib = _lib.load()
    nv, nf, nb = dims()
    stats = np.zeros((nb, 5), dtype=np.int64)
    plain = np.zeros(nb, dtype=np.int32)
    feats = np.zeros((nb, nf), dtype=np.float32)
    g = G.as_gk()
    check(lib.gk_sched_bins(ctypes.byref(g), mode, stats.ctypes.data, plain.ctypes.data, None, feats.ctypes.data,
                            _stream(G)))
    return stats, plain, feats


def learned_choice(G, mode):
    lib = _lib.load()
    nv, nf, nb = dims()
    stats = np.zeros((nb, 5), dtype=np.int64)
    learned = np.zeros(nb, dtype=np.int32)
    g = G.as_gk()
    check(lib.gk_sched_bins(ctypes.byref(g), mode, stats.ctypes.data, None, learned.ctypes.data, None, _stream(G)))
    return learned


def allowed(b, v):
    return bool(_lib.load().gk_sched_variant_allowed(int(b), int(v)))


def _stream(G):
    try:
        import torch
        if G.is_cuda:
            return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    except Exception:
        pass
    return ctypes.c_void_p(0)


def time_bin(G, mode, b, v, reps=2):
    """Best-of-reps CUDA-event time (ms) of bin b's rows on variant v."""
    lib = _lib.load()
    nv, nf, nb = dims()
    table = np.full(nb, -1, dtype=np.int32)
    table[b] = v
    ms = np.zeros(nv, dtype=np.float32)
    g = G.as_gk()
    best = float("inf")
    for _ in range(reps):
        check(lib.gk_tune_run(ctypes.byref(g), mode, table.ctypes.data, ms.ctypes.data, None, _stream(G)))
        best = min(best, float(ms[v]))
    return best


def sweep(G, mode, name, min_work=1 << 20, reps=2, log=print):
    """Times every admissible (bin, variant) pair of a graph; returns a list of
    records {graph, mode, bin, features, rows, work, plain, ms: {variant: ms}}."""
    nv, nf, nb = dims()
    stats, plain, feats = bins(G, mode)
    recs = []
    t0 = time.time()
    for b in range(nb):
        rows, _, _, work, _ = stats[b]
        if rows == 0 or work < min_work:
            continue
        ms = {}
        for v in range(nv):
            if allowed(b, v):
                ms[v] = time_bin(G, mode, b, v, reps)
        recs.append(dict(graph=name, mode=mode, bin=b, features=feats[b].tolist(), rows=int(rows), work=int(work),
                         plain=int(plain[b]), ms={int(k): float(x) for k, x in ms.items()}))
        best = min(ms, key=ms.get)
        log(f"  {name} bin {b:3d} (qm {b // 16:2d} qb {b % 16:2d}) rows {rows:9d} work {work:.3e}  plain v{plain[b]} "
            f"{ms.get(int(plain[b]), float('nan')):8.3f} ms  best v{best} {ms[best]:8.3f} ms")
    log(f"  {name}: {len(recs)} bins in {time.time() - t0:.1f} s")
    return recs


def to_dataset(recs):
    nv, nf, nb = dims()
    X = np.zeros((len(recs), nf), dtype=np.float32)
    Y = np.zeros((len(recs), nv), dtype=np.float32)
    M = np.zeros((len(recs), nv), dtype=np.float32)
    for i, r in enumerate(recs):
        X[i] = r["features"]
        for v, ms in r["ms"].items():
            Y[i, v] = np.log2(max(ms, 1e-4) * 1e6 / r["work"])  # log2 ns per streamed B entry
            M[i, v] = 1.0
    return X, Y, M


# ---------------------------------------------------------------------------
# model
# ---------------------------------------------------------------------------
def init_weights(X, seed=0):
    nv, nf, nb = dims()
    rng = np.random.default_rng(seed)
    parts = [
        rng.normal(0, np.sqrt(2.0 / nf), (MLP_H, nf)), np.zeros(MLP_H),
        rng.normal(0, np.sqrt(2.0 / MLP_H), (MLP_H, MLP_H)), np.zeros(MLP_H),
        rng.normal(0, np.sqrt(1.0 / MLP_H), (nv, MLP_H)), np.zeros(nv),
        X.mean(axis=0), np.maximum(X.std(axis=0), 1e-3),
    ]
    w = np.concatenate([np.ravel(p) for p in parts]).astype(np.float32)
    assert w.shape[0] == model_size()
    return w


def mean_target(Y, M):
    """Output bias initialised to the mean measured cost of each variant."""
    s = (Y * M).sum(axis=0)
    c = M.sum(axis=0)
    return np.where(c > 0, s / np.maximum(c, 1), 0.0)


def train(X, Y, M, epochs=4000, lr=3e-3, seed=0):
    lib = _lib.load()
    nv, nf, nb = dims()
    w = init_weights(X, seed)
    w[-(2 * nf + nv):-2 * nf] = mean_target(Y, M)
    trace = np.zeros(epochs, dtype=np.float32)
    X, Y, M = (np.ascontiguousarray(a, dtype=np.float32) for a in (X, Y, M))
    check(lib.gk_mlp_train(w.ctypes.data, X.ctypes.data, Y.ctypes.data, M.ctypes.data, X.shape[0], epochs,
                           ctypes.c_float(lr), trace.ctypes.data, None))
    return w, trace


def train_best(X, Y, M, recs, epochs, seeds, evaluate_fn):
    """Trains from `seeds` initialisations and keeps the network whose choices
    take the least measured time on the sweep (the MLP's argmin is sensitive to
    small prediction errors between close variants)."""
    best = None
    for seed in range(seeds):
        w, trace = train(X, Y, M, epochs=epochs, seed=seed)
        ev = evaluate_fn(w)
        if best is None or ev["learned_ms"] < best[2]["learned_ms"]:
            best = (w, trace, ev)
    return best


def forward_gpu(w, X):
    lib = _lib.load()
    nv, nf, nb = dims()
    X = np.ascontiguousarray(X, dtype=np.float32)
    out = np.zeros((X.shape[0], nv), dtype=np.float32)
    check(lib.gk_mlp_forward(np.ascontiguousarray(w, dtype=np.float32).ctypes.data, X.ctypes.data, X.shape[0],
                             out.ctypes.data, None))
    return out


def forward_numpy(w, X, nf, nv):
    """The network in numpy (same layout as the CUDA kernels)."""
    h = MLP_H
    o = 0
    W1 = w[o:o + h * nf].reshape(h, nf); o += h * nf
    b1 = w[o:o + h]; o += h
    W2 = w[o:o + h * h].reshape(h, h); o += h * h
    b2 = w[o:o + h]; o += h
    W3 = w[o:o + nv * h].reshape(nv, h); o += nv * h
    b3 = w[o:o + nv]; o += nv
    mu = w[o:o + nf]; o += nf
    sg = w[o:o + nf]
    x = (X - mu) / sg
    h1 = np.maximum(x @ W1.T + b1, 0)
    h2 = np.maximum(h1 @ W2.T + b2, 0)
    return h2 @ W3.T + b3


# log2(1.1): the model must predict >= 10% gain over the plain pick.  The row-bin
# scheduler's margin follows GK_LEARNED_MARGIN as the library's does; the BC
# level chooser's is fixed.
BC_LEARNED_MARGIN = 0.1375


def _margin_from_env(text, default=BC_LEARNED_MARGIN):
    """The library's parse of GK_LEARNED_MARGIN (csrc/sched.cu, learned_margin):
    C atof (the longest leading decimal number, 0.0 when there is none), and
    the default for an unset, non-finite or negative value."""
    if text is None:
        return default
    mt = re.match(r"\s*([+-]?(?:inf(?:inity)?|nan|(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?))", text, re.IGNORECASE)
    v = float(mt.group(1)) if mt else 0.0
    return v if math.isfinite(v) and v >= 0.0 else default


LEARNED_MARGIN = _margin_from_env(os.environ.get("GK_LEARNED_MARGIN"))


def choose(out, recs):
    """As the device inference does: argmin over the bin's admissible
    variants, kept only where it is predicted LEARNED_MARGIN (log2) faster
    than the plain heuristic's variant."""
    picks = []
    for i, r in enumerate(recs):
        cand = [v for v in range(out.shape[1]) if allowed(r["bin"], v)]
        best = min(cand, key=lambda v: out[i, v])
        p = r["plain"]
        picks.append(best if out[i, p] - out[i, best] >= LEARNED_MARGIN else p)
    return picks


def evaluate(recs, picks):
    """Measured time of the plain heuristic's, the model's and the best choices,
    summed over the bins (a pick without a measurement counts as the bin's
    slowest measured time)."""
    plain = learned = best = 0.0
    for r, p in zip(recs, picks):
        ms = r["ms"]
        worst = max(ms.values())
        plain += ms.get(r["plain"], worst)
        learned += ms.get(p, worst)
        best += min(ms.values())
    return dict(plain_ms=plain, learned_ms=learned, best_ms=best)


def save_dataset(recs, path=DATA_PATH):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez_compressed(path, records=json.dumps(recs))


def load_dataset(path=DATA_PATH):
    recs = json.loads(str(np.load(path)["records"]))
    for r in recs:  # JSON object keys are strings
        r["ms"] = {int(k): float(v) for k, v in r["ms"].items()}
    return recs


# ---------------------------------------------------------------------------
# batched BC: per-level forward shape (pull or push)
# ---------------------------------------------------------------------------
def bc_tune(A, sources, shape, max_levels=512):
    """One BC run with every forward level on `shape` (0 pull, 1 push, -1 the
    plain rule), levels driven from the host; returns (per-level ms, per-level
    features, bc)."""
    from . import api
    lib = _lib.load()
    nv, nf, nb = dims()
    src = np.ascontiguousarray(np.asarray(sources, dtype=np.int32))
    if A.is_cuda:
        import torch
        src = torch.as_tensor(src).to(A.rowptr.device)
    out = api._empty_like_space(A.rowptr, (A.m,), np.float64)
    ms = np.zeros(max_levels, dtype=np.float32)
    feat = np.zeros((max_levels, nf), dtype=np.float32)
    n = ctypes.c_int(0)
    g = A.as_gk()
    check(lib.gk_bc_tune(ctypes.byref(g), api._ptr(src), len(sources), int(shape), api._ptr(out), ms.ctypes.data,
                         feat.ctypes.data, max_levels, ctypes.byref(n), _stream(A)))
    k = min(n.value, max_levels)
    return ms[:k].copy(), feat[:k].copy(), out


def bc_plain_shape(f):
    """The plain rule of the device (bc.cu, bc_plain_shape) from a level's features."""
    nf_, ef, mu, m = (2.0 ** f[0] - 1, 2.0 ** f[1] - 1, 2.0 ** f[3] - 1, 2.0 ** f[4] - 1)
    if ef * 14.0 < mu:
        return BC_PUSH
    if nf_ * 24.0 < m:
        return BC_PUSH
    return BC_PULL


def bc_sweep(A, sources, name, reps=2, log=print):
    """Times every forward level of a BC run as pull and as push (best of
    reps); returns one record per level."""
    best = {}
    feats = None
    for shape in (BC_PULL, BC_PUSH):
        for _ in range(reps):
            ms, f, _ = bc_tune(A, sources, shape)
            if feats is None:
                feats = f
            t = best.setdefault(shape, ms.copy())
            np.minimum(t, ms, out=t)
    recs = []
    for i in range(len(feats)):
        ms = {BC_PULL: float(best[BC_PULL][i]), BC_PUSH: float(best[BC_PUSH][i])}
        recs.append(dict(graph=name, level=i + 1, features=feats[i].tolist(), ms=ms,
                         plain=bc_plain_shape(feats[i])))
        log(f"  {name} level {i + 1:3d}  pull {ms[0]:8.3f} ms  push {ms[1]:8.3f} ms  plain "
            f"{'push' if recs[-1]['plain'] else 'pull'}")
    return recs


def bc_dataset(recs):
    nv, nf, nb = dims()
    X = np.zeros((len(recs), nf), dtype=np.float32)
    Y = np.zeros((len(recs), nv), dtype=np.float32)
    M = np.zeros((len(recs), nv), dtype=np.float32)
    for i, r in enumerate(recs):
        X[i] = r["features"]
        for v, ms in r["ms"].items():
            Y[i, v] = np.log2(max(ms, 1e-4) * 1e3)  # log2 microseconds of the level
            M[i, v] = 1.0
    return X, Y, M


def bc_choose(out, recs):
    """The plain rule's shape unless the model predicts the other one
    BC_LEARNED_MARGIN (log2) faster (as k_bc_choose does)."""
    picks = []
    for o, r in zip(out, recs):
        p = r["plain"]
        picks.append(1 - p if o[p] - o[1 - p] >= BC_LEARNED_MARGIN else p)
    return picks


def bc_evaluate(recs, picks):
    plain = learned = best = 0.0
    for r, p in zip(recs, picks):
        ms = r["ms"]
        plain += ms[r["plain"]]
        learned += ms[p]
        best += min(ms.values())
    return dict(plain_ms=plain, learned_ms=learned, best_ms=best)


def load_bc_dataset(path=BC_DATA_PATH):
    recs = json.loads(str(np.load(path)["records"]))
    for r in recs:
        r["ms"] = {int(k): float(v) for k, v in r["ms"].items()}
    return recs


def bc_sources(m, n, seed):
    rng = np.random.default_rng(seed)
    return rng.choice(m, size=min(n, m), replace=False)


# ---------------------------------------------------------------------------
# training graphs (seeds differ from the benchmark graphs')
# ---------------------------------------------------------------------------
TRAIN_GRAPHS = [
    ("rmat16-s11", dict(kind="rmat", scale=16, seed=11)),
    ("rmat18-s12", dict(kind="rmat", scale=18, seed=12)),
    ("rmat20-s13", dict(kind="rmat", scale=20, seed=13)),
    ("rmat22-s14", dict(kind="rmat", scale=22, seed=14)),
    ("rmat24-s15", dict(kind="rmat", scale=24, seed=15)),
    ("er1m-d16-s16", dict(kind="er", n=1 << 20, nedges=8 << 20, seed=16)),
    ("er4m-d32-s17", dict(kind="er", n=1 << 22, nedges=64 << 20, seed=17)),
    ("batch512-s5000", dict(kind="batch", ngraphs=512, seed0=5000)),
    ("batch1024-s7000", dict(kind="batch", ngraphs=1024, seed0=7000)),
]
KTRUSS_GRAPHS = [
    ("rmat18-s18", dict(kind="rmat", scale=18, seed=18)),
    ("rmat20-s19", dict(kind="rmat", scale=20, seed=19)),
]


BC_GRAPHS = [
    ("rmat16-s21-b512", dict(kind="rmat", scale=16, seed=21), 512, 31),
    ("rmat18-s22-b512", dict(kind="rmat", scale=18, seed=22), 512, 32),
    ("rmat18-s23-b128", dict(kind="rmat", scale=18, seed=23), 128, 33),
    ("rmat19-s24-b512", dict(kind="rmat", scale=19, seed=24), 512, 34),
    ("rmat20-s25-b256", dict(kind="rmat", scale=20, seed=25), 256, 35),
    ("er256k-d16-s26-b512", dict(kind="er", n=1 << 18, nedges=1 << 21, seed=26), 512, 36),
    ("er128k-d8-s27-b256", dict(kind="er", n=1 << 17, nedges=1 << 19, seed=27), 256, 37),
]


def build_graph(spec):
    from . import api
    if spec["kind"] == "batch":  # an uneven many-graph batch as one block-diagonal graph
        return api.disjoint_union([api.gen_spec(g) for g in api.uneven_batch_specs(spec["ngraphs"], spec["seed0"])])
    if spec["kind"] == "rmat":
        return api.gen_rmat(spec["scale"], 16, seed=spec["seed"], device="cuda")
    return api.gen_er(spec["n"], spec["nedges"], seed=spec["seed"], device="cuda")


def add_variants(recs, variants, reps=2, log=print):
    """Times `variants` on the bins of the saved sweep records (where the bin
    admits them), re-building each record's graph, and merges the timings in
    place: a variant added to the catalogue joins the training data without
    re-measuring the others."""
    import torch
    from . import api
    specs = dict(TRAIN_GRAPHS)
    specs.update({name + "-ktruss": spec for name, spec in KTRUSS_GRAPHS})
    for name in dict.fromkeys(r["graph"] for r in recs):
        mine = [r for r in recs if r["graph"] == name]
        spec = specs[name]
        G = build_graph(spec)
        mode = mine[0]["mode"]
        if mode == 0:
            L = api.extract_lower(G)
            del G
            G = L
        t0 = time.time()
        for r in mine:
            for v in variants:
                if allowed(r["bin"], v):
                    r["ms"][v] = time_bin(G, mode, r["bin"], v, reps)
            best = min(r["ms"], key=r["ms"].get)
            log(f"  {name} bin {r['bin']:3d} " + " ".join(f"v{v} {r['ms'].get(v, float('nan')):8.3f}" for v in variants)
                + f"  plain v{r['plain']} {r['ms'].get(r['plain'], float('nan')):8.3f}  best v{best} {r['ms'][best]:8.3f}")
        log(f"  {name}: {len(mine)} bins in {time.time() - t0:.1f} s")
        del G
        torch.cuda.empty_cache()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", action="store_true", help="sweep the training graphs, train and save the model")
    ap.add_argument("--retrain", action="store_true", help="train from the saved sweep without re-measuring")
    ap.add_argument("--epochs", type=int, default=4000)
    ap.add_argument("--seeds", type=int, default=6, help="initialisations to train; the best on the sweep is kept")
    ap.add_argument("--max-scale", type=int, default=24)
    ap.add_argument("--out", default=MODEL_DIR, help="directory for model.npz (and sweep.npz with --train)")
    ap.add_argument("--data", default=DATA_PATH, help="sweep to train from with --retrain")
    ap.add_argument("--add-variants", default="",
                    help="comma-separated variant ids: time them on every bin of the saved sweep (re-building "
                         "its graphs), merge the timings into the sweep, then train")
    ap.add_argument("--train-bc", action="store_true", help="sweep the BC graphs, train and save the BC model")
    ap.add_argument("--retrain-bc", action="store_true", help="train the BC model from the saved BC sweep")
    args = ap.parse_args()
    if args.train_bc or args.retrain_bc:
        return main_bc(args)
    model_path = os.path.join(args.out, "model.npz")
    data_path = os.path.join(args.out, "sweep.npz") if args.train else args.data
    import torch
    from . import api
    torch.cuda.set_device(0)
    if args.train:
        recs = []
        for name, spec in TRAIN_GRAPHS:
            if spec.get("scale", 0) > args.max_scale:
                continue
            A = build_graph(spec)
            L = api.extract_lower(A)
            del A
            recs += sweep(L, 0, name)
            del L
            torch.cuda.empty_cache()
        for name, spec in KTRUSS_GRAPHS:
            A = build_graph(spec)
            recs += sweep(A, 1, name + "-ktruss")
            del A
            torch.cuda.empty_cache()
        save_dataset(recs, data_path)
    if args.add_variants:
        data_path = os.path.join(args.out, "sweep.npz")
        recs = load_dataset(args.data)
        add_variants(recs, [int(v) for v in args.add_variants.split(",")])
        save_dataset(recs, data_path)
    recs = load_dataset(data_path)
    X, Y, M = to_dataset(recs)
    w, trace, ev = train_best(X, Y, M, recs, args.epochs, args.seeds,
                              lambda w_: evaluate(recs, choose(forward_gpu(w_, X), recs)))
    print(json.dumps({"samples": len(recs), "loss_first": float(trace[0]), "loss_last": float(trace[-1]), **ev}))
    save_model(w, model_path, samples=len(recs), epochs=args.epochs, final_loss=float(trace[-1]), **ev)


def main_bc(args):
    import torch
    torch.cuda.set_device(0)
    model_path = os.path.join(args.out, "bc_model.npz")
    data_path = os.path.join(args.out, "bc_sweep.npz") if args.train_bc else BC_DATA_PATH
    if args.train_bc:
        recs = []
        for name, spec, nsrc, sseed in BC_GRAPHS:
            A = build_graph(spec)
            recs += bc_sweep(A, bc_sources(A.m, nsrc, sseed), name)
            del A
            torch.cuda.empty_cache()
        save_dataset(recs, data_path)
    recs = load_bc_dataset(data_path)
    X, Y, M = bc_dataset(recs)
    w, trace, ev = train_best(X, Y, M, recs, args.epochs, args.seeds,
                              lambda w_: bc_evaluate(recs, bc_choose(forward_gpu(w_, X), recs)))
    print(json.dumps({"samples": len(recs), "loss_first": float(trace[0]), "loss_last": float(trace[-1]), **ev}))
    save_model(w, model_path, samples=len(recs), epochs=args.epochs, final_loss=float(trace[-1]), **ev)


if __name__ == "__main__":
    main()
