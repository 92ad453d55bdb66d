"""Batched BC runs for CUDA-event timing and for ncu.

  python -m graphkokkos_b200.profile_bc --scale 18 --seed 3 --nsrc 512 --src-seed 4 --reps 2

Builds the seeded RMAT graph on the device and calls gk_bc_batch --reps times
after --warmup calls, printing one JSON line with the per-call CUDA-event
time.  With --host-levels the level loops are driven from the host (library
profiling mode 2), so that every level kernel is a separate launch an ncu
launch list can see; without it they run as CUDA graphs.
"""
import argparse
import json

import numpy as np
import torch

import graphkokkos_b200 as gk


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=int, default=18)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--nsrc", type=int, default=512)
    ap.add_argument("--src-seed", type=int, default=4)
    ap.add_argument("--sched", default="plain")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--host-levels", action="store_true")
    args = ap.parse_args()
    torch.cuda.set_device(0)
    lib = gk.load()
    if args.sched == "learned":
        from graphkokkos_b200 import sched
        sched.load_bc_model()
    A = gk.gen_rmat(args.scale, 16, seed=args.seed, device="cuda")
    src = np.random.default_rng(args.src_seed).choice(A.m, size=args.nsrc, replace=False)
    if args.host_levels:
        lib.gk_prof_enable(2)
    for _ in range(args.warmup):
        bc = gk.bc_batch(A, src, sched=args.sched)
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(args.reps):
        bc = gk.bc_batch(A, src, sched=args.sched)
    e1.record(s)
    torch.cuda.synchronize()
    lib.gk_prof_enable(0)
    print(json.dumps({"scale": args.scale, "seed": args.seed, "nsrc": args.nsrc, "sched": args.sched,
                      "host_levels": args.host_levels, "ms_per_call": round(e0.elapsed_time(e1) / args.reps, 3),
                      "bc_sum": float(bc.sum().item())}))


if __name__ == "__main__":
    main()
