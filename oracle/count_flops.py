"""Algorithmic flops of the narrowphase per collision pass, counted in the
reference's FP64 build (oracle/flop_count.cpp, constants in oracle/flops.h),
on the benchmark's own workload and pass window. TEST INFRASTRUCTURE: it
writes the summary the benchmark reads for its narrowphase roofline.

    python oracle/count_flops.py [--workload mixed] [--out profiles/narrowphase_flops_mixed65536.md]

The run follows the benchmark: the 65,536-body mixed world (same seed, cube,
wall-reflected motion and centres of mass), a creation pass, the warm-up and
graph-capture passes untimed, then the timed window, whose passes are counted.
"""
import argparse
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=20, help="passes counted (the benchmark's timed window)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--out", default=os.path.join(ROOT, "profiles", "narrowphase_flops_mixed65536.md"))
    args = ap.parse_args()

    import bench
    from bounce_b200 import scene as S
    from oracle import oracle as O

    S.NATIVE_HULLS = False
    sc = bench.build_scene(bench.N_BODIES, bench.SEED)
    walls = bench.scene_half(sc)
    rw = O.RefWorld(sc, precision=64)
    rw.set_local_centers(sc.local_center)
    drv = S.KinematicDriver(sc, walls=walls)
    rw.first_pass()
    for _ in range(args.warmup + bench.GRAPH_PASSES):
        drv.advance()
        rw.set_sweeps(drv.sweeps14())
        rw.step_pass()
    O.flop_counts(reset=True)
    per_pass = []
    t0 = time.time()
    for _ in range(args.steps):
        drv.advance()
        rw.set_sweeps(drv.sweeps14())
        rw.step_pass()
        c = O.flop_counts(reset=True)
        c["contacts"] = rw.contact_count()
        c["touching"] = rw.touching()[0]
        per_pass.append(c)
    secs = time.time() - t0
    rw.close()
    keys = list(per_pass[0].keys())
    mean = {k: float(np.mean([p[k] for p in per_pass])) for k in keys}
    lo = min(p["flops"] for p in per_pass)
    hi = max(p["flops"] for p in per_pass)
    cmd = "python oracle/count_flops.py" + (f" --steps {args.steps}" if args.steps != 20 else "") + (
        f" --warmup {args.warmup}" if args.warmup != 5 else "")
    lines = [
        "# Narrowphase algorithmic flops: mixed 65,536-body world",
        "",
        f"Command: `{cmd}` (the reference's FP64 build with its narrowphase loop-trip",
        "counters, oracle/flop_count.cpp; flops per trip in oracle/flops.h).",
        "",
        f"Workload: {bench.WORKLOAD}; passes {1 + args.warmup + bench.GRAPH_PASSES}-"
        f"{args.warmup + bench.GRAPH_PASSES + args.steps} of the motion (the benchmark's timed window), counted one by one.",
        "",
        "A flop is one add, subtract, multiply, divide or square root. Counted: the",
        "b3Collide* calls per routine with their closed-form parts, the face and edge",
        "queries of the SAT (every (plane, vertex) trip; every edge pair and those past",
        "the Gauss-map test), feature-cache reads, GJK iterations with their support",
        "searches, side-plane clipping (vertices and crossings per plane) and polygon",
        "reduction. Estimated, not counted: the simplex solve of a GJK iteration.",
        "",
        f"flops per pass: {lo:.0f} - {hi:.0f} over the window",
        "",
        "| counter | mean per pass |",
        "|---|---|",
    ]
    for k in keys:
        lines.append(f"| {k} | {mean[k]:.1f} |")
    lines += ["", f"flops_per_pass_mean | {mean['flops']:.0f}", "",
              f"({args.steps} FP64 reference passes in {secs:.1f} s on the host.)", ""]
    with open(args.out, "w") as f:
        f.write("\n".join(lines))
    print("\n".join(lines))


if __name__ == "__main__":
    main()
