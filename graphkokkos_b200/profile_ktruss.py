"""k-truss runs for CUDA-event timing and for ncu.

  python -m graphkokkos_b200.profile_ktruss --scale 20 --seed 2 --k 5 --reps 2

Builds the seeded RMAT graph on the device and calls gk_ktruss --reps times
after --warmup calls, printing one JSON line with the per-call CUDA-event time
and the per-variant profile (gk_prof_*) of one extra call.  With
--host-passes the pass loop is driven from the host (library profiling mode
2), so that every kernel of every pass is a separate launch an ncu capture can
select; without it the passes run as one CUDA graph.
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
    ap.add_argument("--k", type=int, default=5)
    ap.add_argument("--sched", default="plain")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--host-passes", action="store_true")
    args = ap.parse_args()
    torch.cuda.set_device(0)
    lib = gk.load()
    if args.sched == "learned":
        from graphkokkos_b200 import sched
        sched.load_model()
    A = gk.gen_rmat(args.scale, 16, seed=args.seed, device="cuda")
    if args.host_passes:
        lib.gk_prof_enable(2)
    for _ in range(args.warmup):
        T, it = gk.ktruss(A, args.k, sched=args.sched)
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(args.reps):
        T, it = gk.ktruss(A, args.k, sched=args.sched)
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(args.reps, 1)
    lib.gk_prof_enable(1)
    gk.ktruss(A, args.k, sched=args.sched)
    rec = GkProfRec()
    per = {}
    for i in range(lib.gk_prof_count()):
        lib.gk_prof_get(i, ctypes.byref(rec))
        if rec.rows:
            d = per.setdefault(rec.variant, [0.0, 0])
            d[0] += rec.ms
            d[1] += rec.sum_work
    lib.gk_prof_enable(0)
    print(json.dumps({"scale": args.scale, "seed": args.seed, "k": args.k, "sched": args.sched,
                      "host_passes": args.host_passes, "iterations": it, "truss_nnz": T.nnz,
                      "ms_per_call": round(ms, 3),
                      "variants": {str(v): {"ms": round(x[0], 3), "work": x[1],
                                            "gprobe_per_s": round(x[1] / (x[0] * 1e6), 1) if x[0] > 0 else None}
                                   for v, x in sorted(per.items())}}))


if __name__ == "__main__":
    main()
