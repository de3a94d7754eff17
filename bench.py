"""Benchmark: one collision pass per step of the 65,536-body mixed world.

Workload: one world of 65,536 bodies (40 % spheres r ~ U[0.2, 1] m, 30 %
capsules r ~ U[0.1, 0.5] m, half-height ~ U[0.2, 1] m, 30 % quickhull-style
hulls of 8-32 points on ellipsoids with semi-axes ~ U[0.3, 1.2] m) in a 49 m
cube, linear velocities N(0, 1) m/s, angular N(0, 1) rad/s, seeded; bodies
move kinematically between passes (dt = 1/60 s). A step is one collision pass:
fat-AABB update, broadphase, contact begin/end, narrowphase manifolds (the
"Find New Pairs" block and UpdateContacts of b3World::Step).

Metric: manifolds/s = manifolds with at least one point produced per second.
`value` times passes with the body state already in HBM; `e2e` times the same
through the C ABI with host buffers (host->device copy of the pinned state,
device->host contact list and packed touching manifolds every step, the
copies of one step overlapping the next step's pass). Other workloads:
--workload pile (hull pile over a mesh), batched (1,024 worlds), serving
(request stream), queries (ray casts), shapecast (shape casts), toi (time
of impact of sweep pairs) and constraints (the solver's contact constraints
built from the pass's manifolds). The reference arm
(--impl reference) runs the reference's own CPU pipeline (oracle/_ref, the
unmodified Bounce sources) on the same scene and body motion.

Multi-GPU: replicas only (independent worlds per GPU, no collective); value is
the sum over ranks divided by the max time over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_BODIES = 65536
SIDE = 49.0
SEED = 2
WORKLOAD = ("one world, 65,536 mixed bodies (40% sphere, 30% capsule, 30% convex hull of 8-32 points on ellipsoids, "
            "built by this project's incremental hull builder, not the reference's quickhull), 49 m cube, "
            "kinematic motion reflected at the cube faces")
PILE_SEED = 9
# Untimed passes after the warm-up in which the device arm captures its CUDA
# graphs (one per contact-buffer parity); both arms skip them.
GRAPH_PASSES = 2
PILE_WORKLOAD = ("hull-heavy pile: 262,144 distinct hulls (quickhulls of 12-64 points on ellipsoids, semi-axes "
                 "U[0.3, 1.0] m) in 512 columns of 512 with 1e-3 m vertical gaps, over a static mesh ground of "
                 "512 x 512 vertices at 0.5 m (4 seeded sines, 2 m total amplitude); the pile settles kinematically")
PILE_SAMPLE = ("4 of the 512 columns (2,048 hulls) over a 64 x 64-vertex patch of the same terrain: a bounded "
               "sample, as the reference arm builds its hulls with the pure-Python builder, which would take minutes "
               "for the full pile's 262,144")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--bodies", type=int, default=N_BODIES)
    ap.add_argument("--e2e-steps", type=int, default=60)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-steps", type=int, default=30,
                    help="passes after the timed ones, with per-stage CUDA events (not part of value)")
    ap.add_argument("--no-graph", action="store_true", help="launch each pass kernel by kernel")
    ap.add_argument("--workload", default="mixed", choices=["mixed", "pile", "batched", "serving", "queries",
                                                             "constraints", "shapecast", "toi"])
    ap.add_argument("--rates", default="1000,5000,10000,20000,50000",
                    help="serving: arrival rates (worlds/s) of the sweep")
    ap.add_argument("--serve-seconds", type=float, default=1.0, help="serving: arrival window per rate")
    ap.add_argument("--worlds", type=int, default=1024)
    ap.add_argument("--autotune", dest="autotune", action="store_true", default=None,
                    help="measure the launch shapes (b3g_autotune) before the timed passes")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the default launch shapes")
    ap.add_argument("--max-contacts", type=int, default=0, help="contact capacity (0: sized from the workload)")
    args = ap.parse_args()
    if args.autotune is None:
        # The autotuner times each kernel alone; in a single world's pass the
        # convex and hull-hull branches run at the same time, and the shapes
        # it picks there measured slower than the default table (0.80 against
        # 0.77 ms per pass), so only the batched pass and the hull pile (its
        # narrowphase is the hull-hull branch alone) use it by default.
        args.autotune = args.workload in ("batched", "pile")
    if args.workload in ("batched", "pile"):
        # The batched and pile workloads are quoted on 30 steps.
        if "--steps" not in sys.argv:
            args.steps = 30
        if "--warmup" not in sys.argv:
            args.warmup = 3
    if args.workload == "pile":
        if "--e2e-steps" not in sys.argv:
            args.e2e_steps = 10
        if "--profile-steps" not in sys.argv:
            args.profile_steps = 10
    return args


def dist_init(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl" if args.impl == "ours" else "gloo",
                                timeout=__import__("datetime").timedelta(seconds=600))
    return rank, world, local, dist


def replica_totals(dist, device, seconds, work):
    """Replicas: the slowest rank's time and the work of all ranks
    (max / sum all-reduce; device is "cuda:i" under NCCL, "cpu" under gloo)."""
    if dist is None:
        return seconds, work
    import torch

    t = torch.tensor([seconds, float(work)], device=device, dtype=torch.float64)
    tmax = t.clone()
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    tsum = t.clone()
    dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
    return float(tmax[0]), float(tsum[1])


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {
            "sm_mhz": float(np.median(sm)) if sm else None,
            "sm_max_mhz": float(max(mx)) if mx else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def scene_half(scene):
    """Half-size of the cube the bodies start in; the driver reflects centres of
    mass off its faces so the contact density stays constant over long runs."""
    return float(np.abs(scene.body_pos).max())


def build_scene(n, seed):
    from bounce_b200 import scene as S

    return S.mixed_scene(seed=seed, n=n, side=SIDE * (n / N_BODIES) ** (1.0 / 3.0)).finalize()


def workload_scene(args, seed, sample=False):
    """(scene, walls) of the single-world workload; sample: the bounded case
    the reference's CPU pass is timed on when the full one cannot be built
    on the host (the pile's ground mesh)."""
    from bounce_b200 import scene as S

    if args.workload == "pile":
        sc = S.pile_scene(seed=seed, columns=4, grid=64) if sample else S.pile_scene(seed=seed)
        return sc.finalize(), None
    sc = build_scene(args.bodies, seed)
    return sc, scene_half(sc)


def config_dict(args, extra=None):
    pile = args.workload == "pile"
    bodies = 512 * 512 if pile else args.bodies
    d = {"workload": PILE_WORKLOAD if pile else WORKLOAD, "bodies": bodies, "proxies": bodies + (1 if pile else 0),
         "dt": 1.0 / 60.0,
         "passes_timed": args.steps, "warmup_passes": args.warmup,
         "l2": "inputs larger than L2: per-pass contact state (two 320 B manifolds per contact) exceeds 126 MB",
         "parallelism": f"replicas x{args.gpus}"}
    if extra:
        d.update(extra)
    return d


# ---------------------------------------------------------------------------
# Reference CPU pipeline (oracle/_ref): the CPU baseline leg and --impl reference.


def reference_run(scene, passes, seconds_cap=None, warmup=0, walls=None):
    """Runs the reference's collision pass on the CPU: creation pass, `warmup`
    untimed passes, then up to `passes` timed passes (stopping early once
    seconds_cap of measured time is spent). Returns (manifolds, seconds, passes)."""
    from bounce_b200 import scene as S
    from oracle import oracle as O

    if not O.available(32):
        raise RuntimeError("oracle/_ref/libb3ref32.so not built")
    rw = O.RefWorld(scene)
    # Both arms move the bodies with the scene's own centres of mass, so the
    # reference sees the transforms the device pass sees.
    rw.set_local_centers(scene.local_center)
    drv = S.KinematicDriver(scene, walls=walls)
    rw.first_pass()
    for _ in range(warmup):
        drv.advance()
        rw.set_sweeps(drv.sweeps14())
        rw.step_pass()
    total_m, total_t, done = 0, 0.0, 0
    for _ in range(passes):
        drv.advance()
        rw.set_sweeps(drv.sweeps14())
        t = rw.step_pass()
        total_t += float(t[0] + t[1])
        total_m += rw.touching()[1]
        done += 1
        if seconds_cap is not None and total_t >= seconds_cap:
            break
    rw.close()
    return total_m, total_t, done


def run_reference_arm(args, rank, world, dist):
    if rank != 0:
        return
    # Scenes are built with the pure-Python hull builder here, so this process
    # maps no library of this project: only the reference build in oracle/_ref.
    from bounce_b200 import scene as S

    S.NATIVE_HULLS = False
    if args.workload == "toi":
        sc, q = toi_setup(SEED)
        _, t = toi_reference(sc, q[:TOI_CPU_COUNT])
        v = TOI_CPU_COUNT / t
        print(json.dumps({
            "metric": "time-of-impact queries/s", "value": v, "unit": "queries/s", "n_gpus": args.gpus,
            "steps": 1, "warmup": 0, "ms_per_step": 1000.0 * t, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": TOI_WORKLOAD, "queries_per_step": TOI_CPU_COUNT},
            "cpu_baseline": {"value": v, "unit": "queries/s", "cores": 1, "kind": "reference",
                             "sample": f"{TOI_CPU_COUNT} queries through b3TimeOfImpact on 1 host core"},
            "e2e": {"value": v, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    if args.workload == "shapecast":
        scene, walls = workload_scene(args, SEED)
        casts = make_casts(scene, SEED + 300, CAST_CPU_COUNT, scene_half(scene))
        _, _, t = cast_reference(scene, walls, casts)
        v = len(casts) / t
        print(json.dumps({
            "metric": "shape casts/s", "value": v, "unit": "casts/s", "n_gpus": args.gpus, "steps": 1, "warmup": 0,
            "ms_per_step": 1000.0 * t, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": CAST_WORKLOAD, "casts_per_step": len(casts)},
            "cpu_baseline": {"value": v, "unit": "casts/s", "cores": 1, "kind": "reference",
                             "sample": f"{len(casts)} casts through b3World::ShapeCastSingle on 1 host core"},
            "e2e": {"value": v, "unit": "casts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    if args.workload == "constraints":
        scene, walls = workload_scene(args, SEED)
        rc, rm, t = constraint_reference(scene, walls, SEED + 200)
        v = rc / t
        print(json.dumps({
            "metric": "contact constraints/s", "value": v, "unit": "constraints/s", "n_gpus": args.gpus,
            "steps": 1, "warmup": 0, "ms_per_step": 1000.0 * t, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": CONSTRAINT_WORKLOAD, "constraints_per_step": rc, "manifolds_per_step": rm},
            "cpu_baseline": {"value": v, "unit": "constraints/s", "cores": 1, "kind": "reference",
                             "sample": f"the whole step ({rc} constraints) through b3ContactSolver's constructor "
                                       "and InitializeVelocityConstraints on 1 host core"},
            "e2e": {"value": v, "unit": "constraints/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    if args.workload == "queries":
        scene, walls = workload_scene(args, SEED)
        rays = make_rays(SEED + 100, QUERY_CPU_RAYS, scene_half(scene))
        _, t = query_reference(scene, walls, rays)
        v = len(rays) / t
        print(json.dumps({
            "metric": "rays/s", "value": v, "unit": "rays/s", "n_gpus": args.gpus, "steps": 1, "warmup": 0,
            "ms_per_step": 1000.0 * t, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": QUERY_WORKLOAD, "rays_per_step": len(rays)},
            "cpu_baseline": {"value": v, "unit": "rays/s", "cores": 1, "kind": "reference",
                             "sample": f"{len(rays)} rays through b3World::RayCastSingle on 1 host core"},
            "e2e": {"value": v, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    pile = args.workload == "pile"
    scene, walls = workload_scene(args, PILE_SEED if pile else SEED, sample=pile)
    # The same pass window as the device arm: creation pass, W warm-up passes
    # and the 2 passes that capture its graphs untimed, then K timed passes.
    m, t, done = reference_run(scene, args.steps, warmup=args.warmup + GRAPH_PASSES, walls=walls)
    v = m / t if t > 0 else 0.0
    sample = (f"{done} passes of {PILE_SAMPLE}" if pile else
              f"{done} passes of the full workload")
    line = {
        "metric": "manifolds/s", "value": v, "unit": "manifolds/s", "n_gpus": args.gpus, "steps": done,
        "warmup": args.warmup, "ms_per_step": 1000.0 * t / max(done, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": config_dict(args), "impl": "reference",
        "cpu_baseline": {"value": v, "unit": "manifolds/s", "cores": 1, "kind": "reference",
                         "sample": f"{sample} on 1 host core (the reference is single-threaded)"},
        "e2e": {"value": v, "unit": "manifolds/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# GPU arm.


def algorithmic_bytes(scene, counts):
    """Algorithmic HBM bytes of one pass's broadphase front end (the sync
    stage): per proxy the body state (68 B), fixture record (60 B), old and new
    fat AABB (2 x 32 B) and moved flag, plus each hull's local vertices once
    (16 B each, float4)."""
    ha = scene.hull_arrays
    desc = ha["desc"].reshape(-1, 6)
    hull_fix = scene.fix_type == 3
    hv = desc[scene.fix_hull[hull_fix], 1].sum() * 16
    return int(scene.n_fixtures * (68 + 60 + 64 + 1) + hv)


def broadphase_bytes(scene, counts):
    """Algorithmic HBM bytes of one pass's broadphase (sync, sort, build,
    traversal, contact begin/end), by the formula
        N (2 x 28 [xf0, xf1] + 24 [old fat AABB] + 24 [new fat AABB] + 1 [moved])
      + 12 per hull vertex of the hull fixtures (read once)
      + 2 N 12 [sort keys and ids, one read and one write]
      + (2N - 1) 32 [tree nodes written: box 24 + two child ids]
      + 8 P [contacts out] + 8 P_prev [previous contacts looked up]
      + 8 (P_begin + P_end) [begun and ended lists]
    with N proxies and P the contacts of the pass (P_prev = P - begun + ended)."""
    n = scene.n_fixtures
    ha = scene.hull_arrays
    desc = ha["desc"].reshape(-1, 6)
    hull_fix = scene.fix_type == 3
    hv = int(desc[scene.fix_hull[hull_fix], 1].sum())
    p = counts["contacts"]
    p_prev = p - counts["begun"] + counts["ended"]
    return int(n * (2 * 28 + 24 + 24 + 1) + 12 * hv + 2 * n * 12 + (2 * n - 1) * 32 + 8 * p + 8 * p_prev
               + 8 * (counts["begun"] + counts["ended"]))


def committed_flops(args):
    """Mean algorithmic narrowphase flops per pass of the timed window, as
    counted in the reference's FP64 build on this workload (written by
    oracle/count_flops.py to profiles/narrowphase_flops_mixed65536.md)."""
    if args.workload != "mixed" or args.bodies != N_BODIES:
        return None
    try:
        for line in open(os.path.join(ROOT, "profiles", "narrowphase_flops_mixed65536.md")):
            if line.startswith("flops_per_pass_mean |"):
                return float(line.split("|")[1])
    except (OSError, ValueError):
        pass
    return None


def committed_traffic(kernel, args, label="mixed 65,536"):
    """DRAM bytes per launch of `kernel` from the committed ncu summary
    (profiles/roofline_traffic.md), for the workload it was captured on."""
    if args.workload not in ("mixed", "constraints") or args.bodies != N_BODIES:
        return None
    try:
        for line in open(os.path.join(ROOT, "profiles", "roofline_traffic.md")):
            cells = [c.strip() for c in line.strip().strip("|").split("|")]
            if len(cells) == 3 and cells[0] == kernel and cells[1] == label:
                return int(cells[2])
    except (OSError, ValueError):
        pass
    return None


def run_ours(args, rank, world, local, dist):
    import torch

    from bounce_b200.pipeline import CollisionPipeline
    from bounce_b200 import scene as S

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pile = args.workload == "pile"
    scene, walls = workload_scene(args, (PILE_SEED if pile else SEED) + rank)
    drv = S.KinematicDriver(scene, walls=walls)
    # states: creation + warm-up, 2 passes that capture the tuned graphs, timed, profiled
    t0_k = 1 + args.warmup + GRAPH_PASSES
    n_dev = t0_k + args.steps + args.profile_steps
    e2e_warm = 2  # untimed host-state passes: they capture the pinned-state graphs
    total = n_dev + e2e_warm + args.e2e_steps
    nb = scene.n_bodies
    states = np.empty((total, 17 * nb), np.float32)
    states[0] = drv.state17()
    for k in range(1, total):
        drv.advance()
        states[k] = drv.state17()
    d_states = torch.from_numpy(states[:n_dev]).to(dev)
    max_contacts = args.max_contacts or (4 * nb if pile else max(2_000_000, 40 * nb))
    pipe = CollisionPipeline(scene, max_contacts=max_contacts, device=local, graph=not args.no_graph)
    stream = torch.cuda.Stream(device=dev)
    sptr = stream.cuda_stream
    row = 17 * nb * 4
    base = d_states.data_ptr()

    # creation pass + warm-up (the first steady-state passes capture the graphs)
    with torch.cuda.stream(stream):
        for k in range(0, 1 + args.warmup):
            pipe.collide(base + k * row, on_device=True, stream=sptr)
    stream.synchronize()
    c = pipe.counts()
    assert c["status"] == 0, c
    tuning = pipe.autotune(reps=5, stream=sptr).tolist() if args.autotune else pipe.tuning().tolist()
    # Two passes (one per contact-buffer parity) capture the graphs with the
    # tuned launch shapes before the timed region.
    with torch.cuda.stream(stream):
        for k in range(1 + args.warmup, t0_k):
            pipe.collide(base + k * row, on_device=True, stream=sptr)
    stream.synchronize()
    pipe.totals(reset=True)

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.2)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for k in range(t0_k, t0_k + args.steps):
        pipe.collide(base + k * row, on_device=True, stream=sptr)
    ev1.record(stream)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    tot = pipe.totals()
    c = pipe.counts()
    assert c["status"] == 0, c

    # Stage times: further passes with CUDA events between the stages
    # (launched kernel by kernel; not part of the timed value).
    prof = {}
    if args.profile_steps > 0:
        pipe.set_profiling(True)
        k0 = t0_k + args.steps
        for k in range(k0, k0 + args.profile_steps):
            pipe.collide(base + k * row, on_device=True, stream=sptr)
        prof = pipe.profile()
        pipe.set_profiling(False)
        assert pipe.counts()["status"] == 0

    pass_stats = pipe.pass_stats()
    ms_max, manifolds_all = replica_totals(dist, dev, ms, tot["manifolds"])
    value = manifolds_all / (ms_max / 1000.0)

    # e2e through the C ABI with host buffers (pinned), continuing the motion.
    nmax = pipe.max_contacts
    h_contacts = torch.empty((nmax, 3), dtype=torch.int32, pin_memory=True)
    h_index = torch.empty(nmax, dtype=torch.int32, pin_memory=True)
    h_man = torch.empty((nmax, 80), dtype=torch.int32, pin_memory=True)  # packed records fit in nmax * 320 bytes
    # The e2e steps' inputs sit in pinned host memory before the timed region
    # (the solver would write them there); each step copies its own.
    h_states = torch.from_numpy(states[n_dev:n_dev + e2e_warm + args.e2e_steps]).pin_memory()
    import ctypes

    lib = pipe.lib
    e2e_m, e2e_h2d, e2e_d2h = 0, 0, 0
    for k in range(e2e_warm):
        pipe.collide(h_states[k].numpy())
    pipe.counts()
    k0 = n_dev + e2e_warm
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    # Each step: host state in, contact list and touching manifolds out
    # (b3g_fetch_results_packed_async: manifolds packed to their points, the
    # copies of step k travel while step k + 1 runs; the host takes step k's
    # results before it starts step k + 2).
    from bounce_b200 import _native as N

    pending = False
    host_s = [0.0, 0.0, 0.0]  # host seconds in collide, waiting for copies, fetch (waits for the pass)
    for k in range(k0, k0 + args.e2e_steps):
        ta = time.perf_counter()
        pipe.collide(h_states[k - n_dev].numpy())
        tb = time.perf_counter()
        if pending:
            pipe.wait_results()
        tc = time.perf_counter()
        cnt = N.Counts()
        pipe._check(lib.b3g_fetch_results_packed_async(pipe.ctx, ctypes.c_void_p(h_contacts.data_ptr()), nmax,
                                                       ctypes.c_void_p(h_index.data_ptr()),
                                                       ctypes.c_void_p(h_man.data_ptr()), nmax, 320 * nmax,
                                                       ctypes.byref(cnt)))
        td = time.perf_counter()
        host_s[0] += tb - ta
        host_s[1] += tc - tb
        host_s[2] += td - tc
        pending = True
        nc, nt = cnt.contacts, cnt.manifolds
        e2e_m += nt
        e2e_h2d += 17 * 4 * nb
        e2e_d2h += nc * 12 + nt * (4 + 32) + 72 * cnt.points
    pipe.wait_results()
    t1 = time.perf_counter()
    e2e_s = t1 - t0
    e2e_value = e2e_m / e2e_s
    if dist is not None:
        e2e_max, e2e_all = replica_totals(dist, dev, e2e_s, e2e_m)
        e2e_value = e2e_all / e2e_max

    # Rooflines. The narrowphase (its kernels are most of a pass) is bound by
    # the FP32 pipe: algorithmic flops of the pass (counted in the reference's
    # FP64 build on this workload) over the narrowphase stages' time, against
    # one FP32 operation per lane per clock (multiplies and adds are separate
    # instructions here: -fmad=false keeps the reference's rounding), at the
    # SM clock sampled during the timed region. The broadphase is bound by HBM:
    # its algorithmic bytes over the time of its stages.
    roof = roof_bp = roof_sync = None
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    hbm_src = "MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks else "fallback 6650 GB/s"
    stage_ms = {k: v[0] / max(v[1], 1) for k, v in prof.items()}
    if stage_ms:
        props = torch.cuda.get_device_properties(dev)
        mhz = float(clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0) if isinstance(clocks, dict) else 1965.0
        fp32_peak = props.multi_processor_count * 128 * mhz * 1e6 / 1e12
        narrow_ms = sum(stage_ms.get(k, 0.0) for k in ("bucket", "narrow_hulls", "narrow_convex", "narrow_mesh"))
        fl = committed_flops(args)
        if fl and narrow_ms > 0:
            ach = fl / (narrow_ms / 1000.0) / 1e12
            roof = {"kernel": "narrowphase: k_bucket, k_hulls_probe, k_hulls_sat, k_hull_triangle, k_apart, k_convex<0-6>, "
                              "sensor/inactive (profiled passes, one stream)",
                    "bound": "fp32", "achieved": ach, "peak": fp32_peak, "unit": "TFLOP/s", "frac": ach / fp32_peak,
                    "traffic": None, "flops_per_pass": fl, "narrow_ms_per_pass": narrow_ms,
                    "peak_source": f"{props.multi_processor_count} SMs x 128 FP32 lanes x {mhz:.0f} MHz (sampled SM clock); "
                                   "an FMA-counted peak is twice this",
                    "flops_source": "profiles/narrowphase_flops_mixed65536.md (oracle/count_flops.py)"}
        bp_ms = sum(stage_ms.get(k, 0.0) for k in ("sync", "sort", "build", "traverse", "diff"))
        bb = broadphase_bytes(scene, c)
        if bp_ms > 0:
            ach = bb / (bp_ms / 1000.0) / 1e9
            roof_bp = {"kernel": "broadphase: k_sync, bounds/Morton/one-sweep sort, k_build/k_leaves/k_refit, "
                                 "k_traverse_count/emit/overflow, hash diff and list-order layout",
                       "bound": "hbm", "achieved": ach, "peak": hbm_peak, "unit": "GB/s", "frac": ach / hbm_peak,
                       "traffic": None, "algorithmic_bytes_per_pass": bb, "ms_per_pass": bp_ms, "peak_source": hbm_src}
        sync_ms = stage_ms.get("sync", 0.0)
        sb = algorithmic_bytes(scene, c)
        if sync_ms > 0:
            ach = sb / (sync_ms / 1000.0) / 1e9
            roof_sync = {"kernel": "k_sync (fat-AABB update)", "bound": "hbm", "achieved": ach, "peak": hbm_peak,
                         "unit": "GB/s", "frac": ach / hbm_peak, "traffic": committed_traffic("k_sync", args),
                         "algorithmic_bytes_per_launch": sb, "peak_source": hbm_src}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            ref_scene, ref_walls = workload_scene(args, PILE_SEED if pile else SEED, sample=pile)
            m, t, done = reference_run(ref_scene, 50, seconds_cap=args.cpu_seconds,
                                       warmup=args.warmup + GRAPH_PASSES, walls=ref_walls)
            what = PILE_SAMPLE if pile else "the same workload"
            cpu = {"value": m / t, "unit": "manifolds/s", "cores": 1, "kind": "reference",
                   "sample": f"{done} passes of {what} (creation pass excluded) on 1 host core; "
                             "the reference is single-threaded"}
        except Exception as e:  # the GPU number stands on its own
            cpu = {"value": None, "unit": "manifolds/s", "cores": 1, "kind": "reference", "sample": f"failed: {e}"}

    if rank == 0:
        line = {
            "metric": "manifolds/s", "value": value, "unit": "manifolds/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": config_dict(args),
            "counts_last_pass": {"contacts": c["contacts"], "touching": c["touching"], "points": c["points"]},
            "e2e": {"value": e2e_value, "unit": "manifolds/s", "h2d_bytes_per_step": e2e_h2d // max(args.e2e_steps, 1),
                    "d2h_bytes_per_step": e2e_d2h // max(args.e2e_steps, 1), "steps": args.e2e_steps,
                    "host_ms_per_step": {"collide": 1e3 * host_s[0] / args.e2e_steps,
                                         "wait_copies": 1e3 * host_s[1] / args.e2e_steps,
                                         "fetch": 1e3 * host_s[2] / args.e2e_steps}},
            "gpu_launches": tot["launches"],
            "graph_passes": tot["graph_passes"],
            "launch_shapes": tuning,
            "pairs_per_s": tot["contacts"] / (ms / 1000.0),
            "points_per_s": tot["points"] / (ms / 1000.0),
            "stage_ms": stage_ms,
            "pass_stats": pass_stats,
            "roofline": roof,
            "roofline_broadphase": roof_bp,
            "roofline_sync": roof_sync,
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line))
    pipe.close()


# ---------------------------------------------------------------------------
# Batched worlds (config 3): one context for all worlds against one context
# per world, run world by world.

BATCHED_WORKLOAD = ("1,024 independent worlds, body count per world log-uniform in [16, 4096], "
                    "unit boxes (b3Hull half-extent 0.5 m) and spheres r = 0.5 m in equal numbers over a "
                    "static ground box per world, positions in a cube scaled to keep the plain-scene density, "
                    "kinematic motion")


def batched_cpu_worker(job):
    """One host process: the reference's pass on a share of the worlds
    (creation pass + `passes` timed passes each) until `budget` seconds of
    measured pass time are spent. Returns (manifolds, seconds, worlds, passes)."""
    scenes, passes, budget = job
    sys.path.insert(0, ROOT)
    from bounce_b200 import scene as S
    from oracle import oracle as O

    m, t, nw, npass = 0, 0.0, 0, 0
    for sub in scenes:
        rw = O.RefWorld(sub)
        sub.set_local_centers(rw.local_centers())
        drv = S.KinematicDriver(sub)
        rw.first_pass()
        for _ in range(passes):
            drv.advance()
            rw.set_sweeps(drv.sweeps14())
            tt = rw.step_pass()
            t += float(tt[0] + tt[1])
            m += rw.touching()[1]
            npass += 1
        rw.close()
        nw += 1
        if t >= budget:
            break
    return m, t, nw, npass


def batched_cpu_baseline(sc, n_worlds, seconds):
    """The reference's CPU pass on all host cores, one process per core, each
    on its own share of the worlds (a bounded sample: each process stops after
    about `seconds` of pass time)."""
    import multiprocessing as mp

    cores = os.cpu_count() or 1
    shares = [[] for _ in range(cores)]
    for w in range(n_worlds):
        shares[w % cores].append(sc.world_subset(w)[0])
    jobs = [(sh, 5, seconds) for sh in shares if sh]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(len(jobs)) as pool:
        res = pool.map(batched_cpu_worker, jobs)
    wall = time.perf_counter() - t0
    m = sum(r[0] for r in res)
    busy = max(r[1] for r in res)
    worlds = sum(r[2] for r in res)
    passes = sum(r[3] for r in res)
    return {"value": m / busy if busy > 0 else None, "unit": "manifolds/s", "cores": len(jobs), "kind": "reference",
            "sample": f"{worlds} of the {n_worlds} worlds, 5 passes each after the creation pass, one reference "
                      f"process per host core ({passes} passes in all; throughput = manifolds / the longest "
                      f"process's pass time; wall {wall:.1f} s including process start)"}


def run_batched(args, rank, world, local, dist):
    import torch

    from bounce_b200.pipeline import CollisionPipeline
    from bounce_b200 import scene as S

    sc, counts = S.batched_scene(seed=3 + rank, n_worlds=args.worlds, lo=16, hi=4096, cube=20.0)
    sc.finalize()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # Host processes first (spawned before this process touches the GPU).
        try:
            cpu = batched_cpu_baseline(sc, args.worlds, args.cpu_seconds)
        except Exception as e:
            cpu = {"value": None, "unit": "manifolds/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {e}"}
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    drv = S.KinematicDriver(sc)
    nb = sc.n_bodies
    t0_k = 1 + args.warmup + 2
    n_states = t0_k + args.steps
    states = np.empty((n_states, 17 * nb), np.float32)
    states[0] = drv.state17()
    for k in range(1, n_states):
        drv.advance()
        states[k] = drv.state17()
    d_states = torch.from_numpy(states).to(dev)
    base = d_states.data_ptr()
    row = 17 * nb * 4
    stream = torch.cuda.Stream(device=dev)
    sptr = stream.cuda_stream

    # Batched: one context, all worlds, graph replay, autotuned shapes.
    pipe = CollisionPipeline(sc, device=local, graph=not args.no_graph)
    for k in range(0, 1 + args.warmup):
        pipe.collide(base + k * row, on_device=True, stream=sptr)
    stream.synchronize()
    assert pipe.counts()["status"] == 0
    tuning = pipe.autotune(reps=5, stream=sptr).tolist() if args.autotune else pipe.tuning().tolist()
    for k in range(1 + args.warmup, t0_k):
        pipe.collide(base + k * row, on_device=True, stream=sptr)
    stream.synchronize()
    pipe.totals(reset=True)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.2)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for k in range(t0_k, t0_k + args.steps):
        pipe.collide(base + k * row, on_device=True, stream=sptr)
    ev1.record(stream)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    tot = pipe.totals()
    cb = pipe.counts()
    assert cb["status"] == 0, cb
    pipe.close()

    # World by world: one context per world, the plain pass launched kernel by
    # kernel for each world in turn, on the same states (a world's bodies are
    # contiguous, so its state is a slice of the batched state).
    # First body of each world (worlds were built one after the other).
    starts = np.searchsorted(sc.body_world, np.arange(args.worlds))
    pipes = [CollisionPipeline(sc.world_subset(w)[0], device=local) for w in range(args.worlds)]
    for k in range(0, t0_k):
        for w, p in enumerate(pipes):
            p.collide(base + k * row + int(starts[w]) * 68, on_device=True, stream=sptr)
    stream.synchronize()
    for p in pipes:
        p.totals(reset=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for k in range(t0_k, t0_k + args.steps):
        for w, p in enumerate(pipes):
            p.collide(base + k * row + int(starts[w]) * 68, on_device=True, stream=sptr)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms_wbw = ev0.elapsed_time(ev1)
    m_wbw = sum(p.totals()["manifolds"] for p in pipes)
    c_wbw = sum(p.counts()["contacts"] for p in pipes)
    for p in pipes:
        p.close()

    ms_max, m_all = ms, float(tot["manifolds"])
    if dist is not None:
        t = torch.tensor([ms, m_all], device=dev, dtype=torch.float64)
        tmax, tsum = t.clone(), t.clone()
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
        ms_max, m_all = float(tmax[0]), float(tsum[1])
    value = m_all / (ms_max / 1000.0)
    v_wbw = m_wbw / (ms_wbw / 1000.0)
    if rank == 0:
        line = {
            "metric": "manifolds/s", "value": value, "unit": "manifolds/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": BATCHED_WORKLOAD, "worlds": args.worlds, "bodies": int(nb),
                       "proxies": int(sc.n_fixtures), "passes_timed": args.steps,
                       "l2": "inputs larger than L2 (contact state of ~0.75 M bodies)",
                       "parallelism": f"replicas x{world}", "graph": not args.no_graph},
            "gpu_launches": tot["launches"], "graph_passes": tot["graph_passes"], "launch_shapes": tuning,
            "world_by_world": {"value": v_wbw, "unit": "manifolds/s", "ms_per_step": ms_wbw / args.steps,
                               "contacts_last_pass": c_wbw},
            "speedup_vs_world_by_world": value / v_wbw if v_wbw > 0 else None,
            "same_contact_count": c_wbw == cb["contacts"],
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line))


# ---------------------------------------------------------------------------
# Serving (config 5): continuous batching of world requests.

SERVING_WORKLOAD = ("Poisson stream of world requests, each 32-8,192 bodies (log-uniform; config-1 mix of unit "
                    "boxes and spheres over a static ground box), K ~ U{1..16} collision passes on device-resident "
                    "state; continuous batching in one context, admission under a 160 GB budget")


def run_serving(args, rank, world, local, dist):
    import torch

    from bounce_b200 import serving as SV

    if rank != 0:
        return  # one GPU serves; other ranks idle
    torch.cuda.set_device(local)
    eng = SV.ServingEngine(capacity=1 << 20, max_worlds=4096, budget_bytes=160 << 30, device=local)
    tmpls = SV.make_templates(eng, 256, seed=11)
    # warm-up: capture the graphs, touch the code paths
    SV.run_stream(eng, tmpls, rate=2000.0, duration=0.2, seed=99)
    sampler = ClockSampler(local)
    sampler.start()
    sweep = []
    for i, rate in enumerate(float(x) for x in args.rates.split(",")):
        s0 = eng.step_index
        done, wall, arrived = SV.run_stream(eng, tmpls, rate=rate, duration=args.serve_seconds, seed=100 + i)
        lat = np.array([r.t_done - r.arrival for r in done]) * 1e3
        last = max((r.t_done for r in done), default=0.0)
        first = min((r.arrival for r in done), default=0.0)
        sweep.append({
            "rate": rate, "arrived": arrived, "completed": len(done),
            "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
            "throughput_worlds_per_s": len(done) / (last - first) if last > first else None,
            "passes": eng.step_index - s0, "mean_pass_ms": 1e3 * wall / max(eng.step_index - s0, 1),
        })
    clocks = sampler.stop()
    assert eng.counts()["status"] == 0
    at20 = next((x for x in sweep if x["rate"] == 20000.0), sweep[-1])
    line = {
        "metric": "served p99 latency", "value": at20["p99_ms"], "unit": "ms", "n_gpus": 1,
        "steps": sum(x["passes"] for x in sweep), "warmup": 1, "ms_per_step": None, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": SERVING_WORKLOAD, "rate_of_value": at20["rate"], "capacity_fixtures": eng.capacity,
                   "max_resident_worlds": eng.max_worlds,
                   "context_bytes": int(eng.context_bytes), "budget_bytes": 160 << 30,
                   "arrival_seconds_per_rate": args.serve_seconds, "templates": len(tmpls),
                   "l2": "resident contact state larger than L2 at the higher rates"},
        "sweep": sweep,
        "clocks": clocks,
    }
    print(json.dumps(line))
    eng.close()


# ---------------------------------------------------------------------------
# World queries: b3World::RayCastSingle on the device LBVH of the mixed world.

QUERY_RAYS = 1 << 20
QUERY_CPU_RAYS = 1 << 16
QUERY_WORKLOAD = ("b3World::RayCastSingle over the 65,536-body mixed world after 3 collision passes: "
                  "1,048,576 rays per step, start uniform in the cube, direction uniform, length 10 m")


def make_rays(seed, n, half, length=10.0):
    rng = np.random.default_rng(seed)
    p1 = rng.uniform(-half, half, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.ascontiguousarray(np.concatenate([p1, p1 + length * d], axis=1), np.float32)


def query_reference(scene, walls, rays):
    """The reference's RayCastSingle on the same world after the same 3 passes:
    (fixtures, seconds) on 1 host core."""
    from bounce_b200 import scene as S
    from oracle import oracle as O

    rw = O.RefWorld(scene)
    scene.set_local_centers(rw.local_centers())
    drv = S.KinematicDriver(scene, walls=walls)
    rw.first_pass()
    for _ in range(2):
        drv.advance()
        rw.set_sweeps(drv.sweeps14())
        rw.step_pass()
    fix, t = rw.ray_cast_single_batch(rays)
    rw.close()
    return fix, t


def run_queries(args, rank, world, local, dist):
    import ctypes

    import torch

    from bounce_b200.pipeline import CollisionPipeline
    from bounce_b200 import scene as S

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    scene, walls = workload_scene(args, SEED + rank)
    drv = S.KinematicDriver(scene, walls=walls)
    nb = scene.n_bodies
    pipe = CollisionPipeline(scene, max_contacts=max(2_000_000, 40 * nb), device=local)
    for k in range(3):
        if k:
            drv.advance()
        pipe.collide(drv.state17())
    assert pipe.counts()["status"] == 0
    n = QUERY_RAYS
    rays = make_rays(SEED + 100 + rank, n, scene_half(scene))
    d_rays = torch.from_numpy(rays).to(dev)
    d_fix = torch.empty(n, dtype=torch.int32, device=dev)
    d_hit = torch.empty((n, 7), dtype=torch.float32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    lib = pipe.lib

    def cast():
        pipe._check(lib.b3g_ray_cast_single_device(pipe.ctx, n, ctypes.c_void_p(d_rays.data_ptr()), None,
                                                    ctypes.c_void_p(d_fix.data_ptr()),
                                                    ctypes.c_void_p(d_hit.data_ptr()), sptr))

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            cast()
    stream.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.2)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ms = 0.0
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            flush.zero_()  # L2 flushed between steps (outside the events)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            cast()
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = sampler.stop()
    hits = int((d_fix != -1).sum().item())
    ms_max = ms
    if dist is not None:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t[0])
    value = world * n * args.steps / (ms_max / 1000.0)

    # e2e: the host-buffer entry point (rays copied in, results copied out).
    e2e_steps = max(1, min(args.e2e_steps, 5))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        fix_h, _ = pipe.ray_cast_single(rays)
    e2e_s = time.perf_counter() - t0
    e2e_value = n * e2e_steps / e2e_s
    if dist is not None:
        t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_value = world * n * e2e_steps / float(t[0])

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    algo = n * (24 + 4 + 28)
    achieved = algo / (ms / args.steps / 1000.0) / 1e9
    roof = {"kernel": "k_ray_cast<2> (RayCastSingle)", "bound": "hbm", "achieved": achieved, "peak": hbm_peak,
            "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": None, "algorithmic_bytes_per_launch": algo,
            "note": "rays in (24 B) and results out (32 B) per ray; the tree walk is latency bound",
            "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650 GB/s"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            ref_scene, ref_walls = workload_scene(args, SEED)
            sample = rays[:QUERY_CPU_RAYS]
            rfix, rt = query_reference(ref_scene, ref_walls, sample)
            agree = float(np.mean(rfix == fix_h[:QUERY_CPU_RAYS]))
            cpu = {"value": len(sample) / rt, "unit": "rays/s", "cores": 1, "kind": "reference",
                   "sample": f"{len(sample)} of the step's rays through b3World::RayCastSingle on 1 host core",
                   "same_fixture_as_gpu": agree}
        except Exception as e:
            cpu = {"value": None, "unit": "rays/s", "cores": 1, "kind": "reference", "sample": f"failed: {e}"}

    if rank == 0:
        line = {
            "metric": "rays/s", "value": value, "unit": "rays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": QUERY_WORKLOAD, "rays_per_step": n, "bodies": nb, "hit_fraction": hits / n,
                       "l2": "flushed between steps (256 MB write outside the timed events)",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_value, "unit": "rays/s", "h2d_bytes_per_step": 24 * n, "d2h_bytes_per_step": 32 * n,
                    "steps": e2e_steps},
            "gpu_launches": args.steps,
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line))
    pipe.close()


CAST_COUNT = 1 << 17
CAST_CPU_COUNT = 1 << 13
CAST_WORKLOAD = ("b3World::ShapeCastSingle over the 65,536-body mixed world after 3 collision passes: the world's "
                 "own sphere, capsule and hull shapes at uniform positions in the body cube and uniform rotations, "
                 "swept 1-4 m in uniform directions")


def make_casts(scene, seed, n, half):
    """Seeded shape casts of the scene's own convex shapes (b3g_shape_cast_input records)."""
    from bounce_b200 import _native as N

    rng = np.random.default_rng(seed)
    params = scene.fix_params.reshape(-1, 12)
    pool = np.nonzero(np.isin(scene.fix_type, [0, 1, 3]))[0]
    pick = rng.choice(pool, n)
    c = np.zeros(n, N.SHAPE_CAST_DTYPE)
    c["type"] = scene.fix_type[pick]
    c["hull"] = np.where(scene.fix_type[pick] == 3, scene.fix_hull[pick], 0)
    c["params"] = params[pick]
    c["position"] = rng.uniform(-half, half, (n, 3))
    q = rng.normal(size=(n, 4))
    c["rotation"] = q / np.linalg.norm(q, axis=1, keepdims=True)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    c["displacement"] = d * rng.uniform(1.0, 4.0, (n, 1))
    return c


def cast_reference(scene, walls, casts):
    """The reference's ShapeCastSingle on the same world after the same 3
    passes: (fixtures, seconds) on 1 host core."""
    from bounce_b200 import scene as S
    from oracle import oracle as O

    rw = O.RefWorld(scene)
    scene.set_local_centers(rw.local_centers())
    drv = S.KinematicDriver(scene, walls=walls)
    rw.first_pass()
    for _ in range(2):
        drv.advance()
        rw.set_sweeps(drv.sweeps14())
        rw.step_pass()
    fix, frac, t = rw.shape_cast_single_batch(casts.view(np.float32).reshape(-1, 28))
    rw.close()
    return fix, frac, t


def run_shapecast(args, rank, world, local, dist):
    import ctypes

    import torch

    from bounce_b200.pipeline import CollisionPipeline
    from bounce_b200 import scene as S

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    scene, walls = workload_scene(args, SEED + rank)
    drv = S.KinematicDriver(scene, walls=walls)
    nb = scene.n_bodies
    pipe = CollisionPipeline(scene, max_contacts=max(2_000_000, 40 * nb), device=local)
    for k in range(3):
        if k:
            drv.advance()
        pipe.collide(drv.state17())
    assert pipe.counts()["status"] == 0
    n = CAST_COUNT
    casts = make_casts(scene, SEED + 300 + rank, n, scene_half(scene))
    d_casts = torch.from_numpy(casts.view(np.uint8).copy()).to(dev)
    d_fix = torch.empty((n, 2), dtype=torch.int32, device=dev)
    d_hit = torch.empty((n, 7), dtype=torch.float32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    lib = pipe.lib

    def cast():
        pipe._check(lib.b3g_shape_cast_single_device(pipe.ctx, n, ctypes.c_void_p(d_casts.data_ptr()),
                                                      ctypes.c_void_p(d_fix.data_ptr()),
                                                      ctypes.c_void_p(d_hit.data_ptr()), sptr))

    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            cast()
    stream.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.2)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ms = 0.0
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            flush.zero_()  # L2 flushed between steps (outside the events)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            cast()
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = sampler.stop()
    hits = int((d_fix[:, 0] != -1).sum().item())
    secs, work = replica_totals(dist, dev, ms / 1000.0, n * args.steps)
    value = work / secs

    # e2e: the host-buffer entry point (casts copied in, results copied out)
    # with the caller's buffers allocated once in pinned host memory.
    e2e_steps = max(1, min(args.e2e_steps, 5))
    h_casts = torch.from_numpy(casts.view(np.uint8).copy()).pin_memory()
    h_fix = torch.empty((n, 2), dtype=torch.int32).pin_memory()
    h_hit = torch.empty((n, 7), dtype=torch.float32).pin_memory()

    def cast_host():
        pipe._check(lib.b3g_shape_cast_single(
            pipe.ctx, n, ctypes.c_void_p(h_casts.data_ptr()),
            ctypes.cast(ctypes.c_void_p(h_fix.data_ptr()), ctypes.POINTER(ctypes.c_uint32)),
            ctypes.cast(ctypes.c_void_p(h_hit.data_ptr()), ctypes.POINTER(ctypes.c_float))))

    cast_host()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        cast_host()
    e2e_s, e2e_work = replica_totals(dist, dev, time.perf_counter() - t0, n * e2e_steps)
    e2e_value = e2e_work / e2e_s
    fix_h, hit_h = h_fix.numpy().view(np.uint32), h_hit.numpy()

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    algo = n * (112 + 8 + 28)
    achieved = algo / (ms / args.steps / 1000.0) / 1e9
    roof = {"kernel": "k_shape_cast<2> (ShapeCastSingle)", "bound": "hbm", "achieved": achieved, "peak": hbm_peak,
            "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": None, "algorithmic_bytes_per_launch": algo,
            "note": "casts in (112 B) and results out (36 B) per cast; the tree walk and the GJK iterations of "
                    "each candidate's time of impact are latency and compute bound",
            "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650 GB/s"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            ref_scene, ref_walls = workload_scene(args, SEED)
            sample = casts[:CAST_CPU_COUNT]
            rfix, rfrac, rt = cast_reference(ref_scene, ref_walls, sample)
            k = CAST_CPU_COUNT
            cpu = {"value": len(sample) / rt, "unit": "casts/s", "cores": 1, "kind": "reference",
                   "sample": f"{len(sample)} of the step's casts through b3World::ShapeCastSingle on 1 host core",
                   "same_fraction_as_gpu": float(np.mean(rfrac == hit_h[:k, 6])),
                   "same_fixture_as_gpu": float(np.mean(rfix == fix_h[:k, 0])),
                   "note": "fixtures differ where several hits share the smallest fraction exactly (most often "
                           "0, casts that start touching several bodies): the reference keeps the first its "
                           "tree meets, the device the smallest fixture index"}
        except Exception as e:
            cpu = {"value": None, "unit": "casts/s", "cores": 1, "kind": "reference", "sample": f"failed: {e}"}

    if rank == 0:
        line = {
            "metric": "shape casts/s", "value": value, "unit": "casts/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": CAST_WORKLOAD, "casts_per_step": n, "bodies": nb, "hit_fraction": hits / n,
                       "l2": "flushed between steps (256 MB write outside the timed events)",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_value, "unit": "casts/s", "h2d_bytes_per_step": 112 * n,
                    "d2h_bytes_per_step": 36 * n, "steps": e2e_steps, "host_buffers": "pinned, allocated once"},
            "gpu_launches": args.steps,
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line))
    pipe.close()


TOI_COUNT = 1 << 20
TOI_CPU_COUNT = 1 << 16
TOI_WORKLOAD = ("b3TimeOfImpact(b3TOIInput) on 1,048,576 seeded sweep pairs of spheres, capsules, triangles and "
                "hulls (the hull pool of a 4,096-body mixed world): shape A sweeps toward the middle while "
                "rotating, shape B drifts near it, tMax = 1")


def toi_setup(seed):
    from bounce_b200 import scene as S

    sc = S.mixed_scene(seed=seed, n=4096, side=SIDE * (4096 / N_BODIES) ** (1.0 / 3.0)).finalize()
    q = S.toi_queries(np.random.default_rng(seed + 400), TOI_COUNT, len(sc.hull_arrays["desc"]) // 6)
    return sc, q


def toi_reference(sc, q):
    """The reference's b3TimeOfImpact over the queries on 1 host core: (states, seconds)."""
    from oracle import oracle as O

    hulls = O.RefHulls(sc.hull_arrays)
    raw = q.view(np.float32).reshape(-1, 68)
    t0 = time.perf_counter()
    out = hulls.time_of_impact(raw)
    return out, time.perf_counter() - t0


def run_toi(args, rank, world, local, dist):
    import ctypes

    import torch

    from bounce_b200.pipeline import CollisionPipeline

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    sc, q = toi_setup(SEED + rank)
    pipe = CollisionPipeline(sc, device=local)
    n = len(q)
    d_q = torch.from_numpy(q.view(np.uint8).copy()).to(dev)
    d_out = torch.empty((n, 4), dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    lib = pipe.lib

    def run():
        pipe._check(lib.b3g_time_of_impact_device(pipe.ctx, n, ctypes.c_void_p(d_q.data_ptr()),
                                                   ctypes.c_void_p(d_out.data_ptr()), sptr))

    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            run()
    stream.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.2)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ms = 0.0
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            flush.zero_()  # L2 flushed between steps (outside the events)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run()
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = sampler.stop()
    states = np.bincount(d_out[:, 0].cpu().numpy(), minlength=5).tolist()
    secs, work = replica_totals(dist, dev, ms / 1000.0, n * args.steps)
    value = work / secs

    # e2e: the host-buffer entry point (queries copied in, results copied
    # out) with the caller's buffers allocated once in pinned host memory.
    e2e_steps = max(1, min(args.e2e_steps, 5))
    h_q = torch.from_numpy(q.view(np.uint8).copy()).pin_memory()
    h_out = torch.empty((n, 4), dtype=torch.int32).pin_memory()

    def run_host():
        pipe._check(lib.b3g_time_of_impact(pipe.ctx, n, ctypes.c_void_p(h_q.data_ptr()),
                                           ctypes.cast(ctypes.c_void_p(h_out.data_ptr()),
                                                       ctypes.POINTER(ctypes.c_uint32))))

    run_host()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        run_host()
    e2e_s, e2e_work = replica_totals(dist, dev, time.perf_counter() - t0, n * e2e_steps)
    out_h = h_out.numpy().view(np.uint32)

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    algo = n * (272 + 16)
    achieved = algo / (ms / args.steps / 1000.0) / 1e9
    roof = {"kernel": "k_toi_sweeps (b3TimeOfImpact)", "bound": "hbm", "achieved": achieved, "peak": hbm_peak,
            "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": None, "algorithmic_bytes_per_launch": algo,
            "note": "queries in (272 B) and results out (16 B) per query; the conservative advancement and GJK "
                    "iterations are compute and divergence bound",
            "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650 GB/s"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            k = TOI_CPU_COUNT
            ref, rt = toi_reference(sc, q[:k])
            cpu = {"value": k / rt, "unit": "queries/s", "cores": 1, "kind": "reference",
                   "sample": f"{k} of the step's queries through b3TimeOfImpact on 1 host core",
                   "identical_to_gpu": float(np.mean(np.all(ref == out_h[:k], axis=1)))}
        except Exception as e:
            cpu = {"value": None, "unit": "queries/s", "cores": 1, "kind": "reference", "sample": f"failed: {e}"}
    if rank == 0:
        print(json.dumps({
            "metric": "time-of-impact queries/s", "value": value, "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": TOI_WORKLOAD, "queries_per_step": n,
                       "states_unknown_failed_overlapped_touching_separated": states,
                       "l2": "flushed between steps (256 MB write outside the timed events)",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_work / e2e_s, "unit": "queries/s", "h2d_bytes_per_step": 272 * n,
                    "d2h_bytes_per_step": 16 * n, "steps": e2e_steps, "host_buffers": "pinned, allocated once"},
            "gpu_launches": args.steps,
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clocks,
        }))
    pipe.close()


CONSTRAINT_WORKLOAD = ("b3ContactSolver constructor + InitializeVelocityConstraints over the 65,536-body mixed "
                       "world after 3 collision passes: every touching non-sensor contact, seeded body velocities "
                       "N(0, 1), inverse masses 1/U(0.5, 5) kg, world inverse inertias R diag(1/U(0.05, 2)) R^T, "
                       "friction U(0.2, 0.8) and restitution U(0, 0.5) per fixture")


def constraint_inputs(scene, drv, seed):
    """Seeded solver inputs: one b3g_solver_body per body (the pass's centre
    of mass and orientation, synthetic velocities and mass data) and the
    fixtures' friction and restitution."""
    from bounce_b200 import _native as N

    rng = np.random.default_rng(seed)
    sw = drv.sweeps14().reshape(-1, 14)
    n = len(sw)
    b = np.zeros(n, N.SOLVER_BODY_DTYPE)
    b["x"], b["q"] = sw[:, 7:10], sw[:, 10:14]
    b["v"] = rng.normal(0.0, 1.0, (n, 3))
    b["w"] = rng.normal(0.0, 1.0, (n, 3))
    b["localCenter"] = np.asarray(scene.local_center, np.float32).reshape(-1, 3)
    dyn = scene.body_type == 2
    b["invMass"] = np.where(dyn, 1.0 / rng.uniform(0.5, 5.0, n), 0.0)
    q = sw[:, 10:14].astype(np.float64)
    x, y, z, s = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    R = np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - s * z), 2 * (x * z + s * y)], -1),
                  np.stack([2 * (x * y + s * z), 1 - 2 * (x * x + z * z), 2 * (y * z - s * x)], -1),
                  np.stack([2 * (x * z - s * y), 2 * (y * z + s * x), 1 - 2 * (x * x + y * y)], -1)], 1)
    d = 1.0 / rng.uniform(0.05, 2.0, (n, 3))
    inv_i = np.einsum("nij,nj,nkj->nik", R, d, R) * dyn[:, None, None]
    b["invI"] = inv_i.transpose(0, 2, 1).reshape(n, 9)  # columns x, y, z
    nf = scene.n_fixtures
    fr = rng.uniform(0.2, 0.8, nf).astype(np.float32)
    re = rng.uniform(0.0, 0.5, nf).astype(np.float32)
    return b, fr, re


def constraint_reference(scene, walls, seed):
    """The reference's b3ContactSolver constructor and
    InitializeVelocityConstraints on the same world after the same 3 passes,
    on 1 host core: (constraints, manifolds, seconds)."""
    from bounce_b200 import scene as S
    from oracle import oracle as O

    rw = O.RefWorld(scene)
    drv = S.KinematicDriver(scene, walls=walls)
    rw.first_pass()
    for _ in range(2):
        drv.advance()
        rw.set_sweeps(drv.sweeps14())
        rw.step_pass()
    b, fr, re = constraint_inputs(scene, drv, seed)
    con, man, t = rw.contact_solver(b.view(np.float32).reshape(-1, 28), fr, re, timed=True)
    rw.close()
    return len(con), len(man), t


def run_constraints(args, rank, world, local, dist):
    import ctypes

    import torch

    from bounce_b200.pipeline import CollisionPipeline
    from bounce_b200 import scene as S

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    scene, walls = workload_scene(args, SEED + rank)
    drv = S.KinematicDriver(scene, walls=walls)
    nb, nf = scene.n_bodies, scene.n_fixtures
    pipe = CollisionPipeline(scene, max_contacts=max(2_000_000, 40 * nb), device=local)
    for k in range(3):
        if k:
            drv.advance()
        pipe.collide(drv.state17())
    counts = pipe.counts()
    assert counts["status"] == 0
    bodies, fr, re = constraint_inputs(scene, drv, SEED + 200 + rank)
    pipe.set_materials(fr, re)
    con_h, man_h = pipe.contact_constraints(bodies)
    nc, nm = len(con_h), len(man_h)
    d_bodies = torch.from_numpy(bodies.view(np.uint8).copy()).to(dev)
    d_con = torch.empty(max(nc, 1) * 128, dtype=torch.uint8, device=dev)
    d_man = torch.empty(max(nm, 1) * 464, dtype=torch.uint8, device=dev)
    d_counts = torch.zeros(2, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    lib = pipe.lib

    def build():
        pipe._check(lib.b3g_contact_constraints_device(
            pipe.ctx, 0, None, ctypes.c_void_p(d_bodies.data_ptr()), 1.0, 1, ctypes.c_void_p(d_con.data_ptr()), nc,
            ctypes.c_void_p(d_man.data_ptr()), nm, ctypes.c_void_p(d_counts.data_ptr()), sptr))

    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            build()
    stream.synchronize()
    assert d_counts.cpu().numpy().tolist() == [nc, nm]
    same = bool(np.array_equal(d_man.cpu().numpy().view(np.uint32), man_h.view(np.uint32).reshape(-1)))
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.2)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ms = 0.0
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            flush.zero_()  # L2 flushed between steps (outside the events)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            build()
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = sampler.stop()
    secs, work = replica_totals(dist, dev, ms / 1000.0, nc * args.steps)
    value = work / secs

    # e2e: the host-buffer entry point (bodies copied in, records copied out)
    # with the caller's buffers allocated once in pinned host memory.
    e2e_steps = max(1, min(args.e2e_steps, 10))
    h_bodies = torch.from_numpy(bodies.view(np.uint8).copy()).pin_memory()
    h_con = torch.empty(max(nc, 1) * 128, dtype=torch.uint8).pin_memory()
    h_man = torch.empty(max(nm, 1) * 464, dtype=torch.uint8).pin_memory()
    h_counts = np.zeros(2, np.uint32)
    u32p = ctypes.POINTER(ctypes.c_uint32)

    def build_host():
        return pipe._check(lib.b3g_contact_constraints(
            pipe.ctx, 0, None, ctypes.c_void_p(h_bodies.data_ptr()), 1.0, 1, ctypes.c_void_p(h_con.data_ptr()), nc,
            ctypes.c_void_p(h_man.data_ptr()), nm, h_counts.ctypes.data_as(u32p)))

    build_host()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        build_host()
    e2e_s, e2e_work = replica_totals(dist, dev, time.perf_counter() - t0, nc * e2e_steps)
    e2e_value = e2e_work / e2e_s
    e2e_same = bool(np.array_equal(h_man.numpy().view(np.uint32), man_h.view(np.uint32).reshape(-1)))

    # The island graph's edges of the same pass (b3g_fetch_fixture_contacts:
    # every fixture's contact list, device sort and copy to the host), timed
    # by wall clock through the host entry point.
    pipe.fixture_contacts()
    t0 = time.perf_counter()
    for _ in range(5):
        offsets, edges = pipe.fixture_contacts()
    edge_ms = (time.perf_counter() - t0) / 5 * 1000.0

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    # Algorithmic bytes of one launch, each byte once: per contact its state
    # and fixtures (12 B); per fixture flags, body, type, radius and material
    # (24 B); per body its b3g_solver_body (112 B); per manifold its header
    # and points as read (24 + 40 per point); the records written.
    points = int(man_h["pointCount"].sum())
    algo = (12 * counts["contacts"] + 24 * nf + 112 * nb + 24 * nm + 40 * points + 128 * nc + 464 * nm)
    achieved = algo / (ms / args.steps / 1000.0) / 1e9
    roof = {"kernel": "k_contact_constraints (b3g_contact_constraints_device)", "bound": "hbm",
            "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
            "traffic": committed_traffic("k_contact_constraints", args, "constraints 65,536"),
            "algorithmic_bytes_per_launch": algo,
            "note": "one launch per step after two small memsets (tile states, counts); achieved over the whole call",
            "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650 GB/s"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            ref_scene, ref_walls = workload_scene(args, SEED)
            rc, rm, rt = constraint_reference(ref_scene, ref_walls, SEED + 200)
            cpu = {"value": rc / rt, "unit": "constraints/s", "cores": 1, "kind": "reference",
                   "sample": f"the whole step ({rc} constraints, {rm} manifolds) through the reference's "
                             "b3ContactSolver constructor and InitializeVelocityConstraints on 1 host core"}
        except Exception as e:
            cpu = {"value": None, "unit": "constraints/s", "cores": 1, "kind": "reference", "sample": f"failed: {e}"}

    if rank == 0:
        line = {
            "metric": "contact constraints/s", "value": value, "unit": "constraints/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": CONSTRAINT_WORKLOAD, "bodies": nb, "contacts": counts["contacts"],
                       "constraints_per_step": nc, "manifolds_per_step": nm, "points_per_step": points,
                       "device_records_equal_host_entry": same and e2e_same,
                       "fixture_edges": {"edges": int(len(edges)), "ms_host_entry": edge_ms},
                       "l2": "flushed between steps (256 MB write outside the timed events)",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_value, "unit": "constraints/s", "h2d_bytes_per_step": 112 * nb,
                    "d2h_bytes_per_step": 128 * nc + 464 * nm + 8, "steps": e2e_steps,
                    "host_buffers": "pinned, allocated once"},
            "gpu_launches": args.steps,
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line))
    pipe.close()


def main():
    args = parse()
    rank, world, local, dist = dist_init(args)
    try:
        if args.impl == "reference":
            run_reference_arm(args, rank, world, dist)
        elif args.workload == "batched":
            run_batched(args, rank, world, local, dist)
        elif args.workload == "serving":
            run_serving(args, rank, world, local, dist)
        elif args.workload == "queries":
            run_queries(args, rank, world, local, dist)
        elif args.workload == "constraints":
            run_constraints(args, rank, world, local, dist)
        elif args.workload == "shapecast":
            run_shapecast(args, rank, world, local, dist)
        elif args.workload == "toi":
            run_toi(args, rank, world, local, dist)
        else:
            run_ours(args, rank, world, local, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
