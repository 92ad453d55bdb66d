"""Per-variant triangle-counting runs, for CUDA-event timing and for ncu.

  python -m graphkokkos_b200.profile_tc --scale 20 --seed 2 --variant 5 --reps 3

Builds the seeded RMAT graph on the device, takes its strict lower triangle L
and calls gk_tc_count (or, with --variant, gk_tc_count_variant: every row on
one kernel variant) --reps times after --warmup calls, printing one JSON line
with the per-call CUDA-event time and the per-variant profile (gk_prof_*) of
one extra call.  Nothing else runs on the GPU, so an ncu capture of this
command sees only the masked SpGEMM pipeline.  With --batch N it builds the
uneven many-graph batch of N graphs (seeds --seed0 ..) instead and calls
gk_tc_count_batched.
"""
import argparse
import ctypes
import json

import torch

import graphkokkos_b200 as gk
from graphkokkos_b200._lib import GkProfRec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=int, default=20)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--variant", type=int, default=-1)
    ap.add_argument("--sched", default="plain")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--batch", type=int, default=0, help="many-graph batch of this many graphs")
    ap.add_argument("--seed0", type=int, default=100)
    args = ap.parse_args()
    torch.cuda.set_device(0)
    lib = gk.load()
    if args.sched == "learned":
        from graphkokkos_b200 import sched
        sched.load_model()
    if args.batch > 0:
        Ls = []
        for spec in gk.api.uneven_batch_specs(args.batch, args.seed0):
            Lg = gk.extract_lower(gk.api.gen_spec(spec))
            Lg.col = Lg.col[:Lg.nnz].clone()
            Ls.append(Lg)
        L = gk.Csr(0, 0, None, None, None, sum(Lg.nnz for Lg in Ls))  # totals only
    else:
        A = gk.gen_rmat(args.scale, 16, seed=args.seed, device="cuda")
        L = gk.extract_lower(A)
        del A
    torch.cuda.synchronize()

    def call():
        if args.batch > 0:
            return int(gk.tc_count_batched(Ls, sched=args.sched).sum())
        if args.variant >= 0:
            return gk.tc_count_variant(L, args.variant)
        return gk.tc_count(L, sched=args.sched)

    for _ in range(args.warmup):
        count = call()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(args.reps):
        count = call()
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.reps
    lib.gk_prof_enable(1)
    call()
    rec = GkProfRec()
    prof = []
    for i in range(lib.gk_prof_count()):
        lib.gk_prof_get(i, ctypes.byref(rec))
        if rec.rows:
            prof.append({"variant": rec.variant, "ms": round(rec.ms, 3), "rows": rec.rows, "work": rec.sum_work,
                         "gprobe_per_s": round(rec.sum_work / (rec.ms * 1e6), 1) if rec.ms > 0 else None})
    lib.gk_prof_enable(0)
    print(json.dumps({"scale": args.scale, "seed": args.seed, "batch": args.batch, "variant": args.variant,
                      "nnz_lower": L.nnz,
                      "triangles": count, "ms_per_call": round(ms, 3), "profile": prof}))


if __name__ == "__main__":
    main()
