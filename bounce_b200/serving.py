"""Serving: a continuous-batching request loop over one collision context.

Each request is a world (bodies + fixtures + initial motion) asking for K
collision passes. All resident worlds share one context and go through one
pass per step (one captured graph). Between steps the loop retires the worlds
that finished and admits waiting ones into free fixture ranges, as device
memory (the admission budget) and world ids allow; the other worlds keep
their proxies, contacts, feature caches and manifolds on the device
(b3g_update_scene). Body motion between passes is a kinematic integrator on
the device (elementwise float32, so a world moves the same alone or in the
mix). Per step, per-world counts (touching contacts, manifolds, points) are
reduced on the device and copied back asynchronously; a request completes
when the copy of its K-th step has landed on the host.

The reference has no counterpart (one b3World per request, stepped on the
CPU); the collision results of a world in the mix equal those of the world
alone (tests/test_gpu_serving.py).
"""
import collections
import ctypes
import time

import numpy as np

from . import _native as N
from . import scene as S

F = np.float32
u32 = ctypes.c_uint32


class RangeAllocator:
    """First-fit allocation of contiguous index ranges in [0, capacity)."""

    def __init__(self, capacity):
        self.capacity = capacity
        self.free = [(0, capacity)]  # sorted, coalesced (start, length)
        self.used = {}

    def alloc(self, n):
        for i, (s, ln) in enumerate(self.free):
            if ln >= n:
                if ln == n:
                    self.free.pop(i)
                else:
                    self.free[i] = (s + n, ln - n)
                self.used[s] = n
                return s
        return None

    def release(self, s):
        n = self.used.pop(s)
        self.free.append((s, n))
        self.free.sort()
        merged = []
        for a, ln in self.free:
            if merged and merged[-1][0] + merged[-1][1] == a:
                merged[-1] = (merged[-1][0], merged[-1][1] + ln)
            else:
                merged.append((a, ln))
        self.free = merged

    def high_water(self):
        return max((s + n for s, n in self.used.items()), default=0)


class WorldTemplate:
    """One world's arrays (local indices): the config-1 mix of unit boxes and
    spheres over a static ground box, scaled to the plain-scene density."""

    def __init__(self, seed, n, box_hull, ground_hull, hull_arrays):
        sc = S.Scene()
        side = max(20.0 * (n / 2000.0) ** (1.0 / 3.0), 4.0)
        S.plain_scene(seed=seed, n_boxes=n // 2, n_spheres=n - n // 2, cube=side, scene=sc, box_hull=box_hull,
                      ground_hull=ground_hull)
        sc.finalize(hull_arrays=hull_arrays)
        self.n = sc.n_bodies
        self.lc = sc.local_center.copy()
        self.body_type = sc.body_type.copy()
        self.fix_body = sc.fix_body.copy()
        self.fix_type = sc.fix_type.copy()
        self.fix_hull = sc.fix_hull.copy()
        self.fix_params = sc.fix_params.reshape(-1, 12).copy()
        self.fix_flags = sc.fix_flags.copy()
        self.pos = sc.body_pos.copy()
        self.quat = sc.body_quat.copy()
        self.lin = sc.body_lin.copy()
        self.ang = sc.body_ang.copy()
        self.scene = sc


class Request:
    __slots__ = ("rid", "tmpl", "k", "arrival", "start", "world", "steps_done", "done_step", "t_done", "counts")

    def __init__(self, rid, tmpl, k, arrival):
        self.rid, self.tmpl, self.k, self.arrival = rid, tmpl, k, arrival
        self.start = self.world = None
        self.steps_done = 0
        self.done_step = None
        self.t_done = None
        self.counts = None


class ServingEngine:
    """The request loop's device side: one context of `capacity` fixtures
    (one body per fixture), at most `max_worlds` resident worlds, admission
    while the resident bodies' estimated memory stays within budget_bytes."""

    def __init__(self, capacity=1 << 20, max_worlds=4096, budget_bytes=160 << 30, contacts_per_body=16, device=0,
                 graph=True, dt=1.0 / 60.0, active_quantum=16384, ring=4):
        import torch

        self.torch = torch
        self.lib = N.load()
        self.capacity = capacity
        self.max_worlds = max_worlds
        self.dt = F(dt)
        self.quantum = active_quantum
        self.dev = torch.device("cuda", device)
        torch.cuda.set_device(self.dev)
        free0 = torch.cuda.mem_get_info(self.dev)[0]
        pool = S.HullPool()
        self.box_hull = pool.add_box(0.5, 0.5, 0.5)
        self.ground_hull = pool.add_box(50.0, 0.5, 50.0)
        self.hull_arrays = pool.arrays()
        cfg = N.Config(max_proxies=capacity, max_contacts=contacts_per_body * capacity, max_hull_data=0,
                       flags=N.FLAG_WARM_STARTING | N.FLAG_CONVEX_CACHE | (N.FLAG_GRAPH if graph else 0),
                       device=device)
        h = ctypes.c_void_p()
        rc = self.lib.b3g_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != 0:
            raise N.B3GError(rc, "b3g_create failed")
        self.ctx = h
        ha = self.hull_arrays
        self._check(self.lib.b3g_set_hulls(self.ctx, len(ha["desc"]) // 6, N.ptr(ha["desc"], u32),
                                           N.ptr(ha["verts"], ctypes.c_float), N.ptr(ha["edges"], u32),
                                           N.ptr(ha["faces"], u32), N.ptr(ha["planes"], ctypes.c_float),
                                           N.ptr(ha["centroids"], ctypes.c_float)))
        # Placeholder scene: every slot a sphere on its own body; world ids
        # cover [0, max_worlds) so the world bits fit every admitted world.
        world = (np.arange(capacity) % max_worlds).astype(np.uint32)
        btype = np.full(capacity, N.BODY_DYNAMIC, np.uint32)
        awake = np.ones(capacity, np.uint8)
        self._check(self.lib.b3g_set_bodies(self.ctx, capacity, N.ptr(world, u32), N.ptr(btype, u32),
                                            N.ptr(awake, ctypes.c_uint8)))
        params = np.zeros((capacity, 12), F)
        params[:, 3] = 0.5
        ftype = np.zeros(capacity, np.uint32)
        zeros = np.zeros(capacity, np.uint32)
        body = np.arange(capacity, dtype=np.uint32)
        self._check(self.lib.b3g_set_fixtures(self.ctx, capacity, N.ptr(body, u32), N.ptr(ftype, u32),
                                              N.ptr(zeros, u32), N.ptr(params, ctypes.c_float), N.ptr(zeros, u32),
                                              None))
        # device state: the 17-float pass input and the 17-float motion record
        # (b3g_kinematic_step) of every body slot
        f32 = torch.float32
        self.state = torch.zeros((capacity, 17), dtype=f32, device=self.dev)
        self.state[:, 6] = 1.0
        self.state[:, 13] = 1.0
        self.motion = torch.zeros((capacity, 17), dtype=f32, device=self.dev)
        self.motion[:, 6] = 1.0
        self.counts_dev = torch.zeros((ring, max_worlds, 3), dtype=torch.int32, device=self.dev)
        self.counts_host = torch.zeros((ring, max_worlds, 3), dtype=torch.int32, pin_memory=True)
        self.ring = ring
        self._keep = None
        self.events = collections.deque()  # (step, ring slot, event, finished requests)
        self.stream = torch.cuda.Stream(device=self.dev)
        self.sptr = self.stream.cuda_stream
        self.alloc = RangeAllocator(capacity)
        self.world_ids = list(range(max_worlds - 1, -1, -1))
        self.resident = {}
        self.pending_retire = []
        self.pending_admit = []
        self.step_index = 0
        self.budget = budget_bytes
        # Device memory of the context and its state, per body slot: the
        # admission budget is counted in these units.
        self.context_bytes = max(free0 - torch.cuda.mem_get_info(self.dev)[0], 1)
        self.bytes_per_body = self.context_bytes / capacity
        self.resident_bodies = 0
        self.active = 0
        self.slot = 0
        with torch.cuda.stream(self.stream):
            self._check(self.lib.b3g_update_scene(self.ctx, 0, None, None, None, None, 0, None, None, None, None,
                                                  None, None, capacity, N.ptr(body, u32), ctypes.c_void_p(self.sptr)))
        self._set_active(self.quantum)

    def _check(self, rc):
        if rc < 0:
            msg = self.lib.b3g_last_error(self.ctx)
            raise N.B3GError(rc, msg.decode() if msg else "")
        return rc

    def close(self):
        if self.ctx:
            self.stream.synchronize()
            self.lib.b3g_destroy(self.ctx)
            self.ctx = None

    def _set_active(self, n):
        """Processed prefix: grows at once to cover the allocated ranges,
        shrinks only when two quanta are unused (a change drops the captured
        graphs)."""
        need = min(self.capacity, max(self.quantum, -(-n // self.quantum) * self.quantum))
        if need > self.active or need + 2 * self.quantum <= self.active:
            self._check(self.lib.b3g_set_active(self.ctx, need, need))
            self.active = need

    # -- admission -----------------------------------------------------------

    def fits(self, tmpl):
        return (bool(self.world_ids) and self.resident_bodies + tmpl.n <= self.budget / self.bytes_per_body)

    def admit(self, req):
        """Reserve a range and a world id for req; False if it does not fit now."""
        if not self.fits(req.tmpl):
            return False
        start = self.alloc.alloc(req.tmpl.n)
        if start is None:
            return False
        req.start = start
        req.world = self.world_ids.pop()
        self.resident[req.rid] = req
        self.resident_bodies += req.tmpl.n
        self.pending_admit.append(req)
        return True

    def load_templates(self, templates):
        """Stages the worlds requests may ask for in device memory (a request's
        payload is uploaded once; admission copies it into its slot on the
        device)."""
        torch = self.torch
        off = 0
        rows = []
        for t in templates:
            t.offset = off
            off += t.n
            center = S.xf_apply(t.pos, t.quat, t.lc).astype(F)
            st = np.concatenate([t.pos, t.quat, center, t.quat, t.lc], axis=1)
            mo = np.concatenate([center, t.quat, t.lc, t.lin, t.ang,
                                 (t.body_type == N.BODY_DYNAMIC).astype(F)[:, None]], axis=1)
            rows.append((t, st, mo))
        cat = lambda xs, dt: torch.from_numpy(np.ascontiguousarray(np.concatenate(xs), dt)).to(self.dev)
        self.st_btype = cat([t.body_type for t, _, _ in rows], np.int32)
        self.st_fbody = cat([t.fix_body for t, _, _ in rows], np.int32)
        self.st_ftype = cat([t.fix_type for t, _, _ in rows], np.int32)
        self.st_fhull = cat([t.fix_hull for t, _, _ in rows], np.int32)
        self.st_fflags = cat([t.fix_flags for t, _, _ in rows], np.int32)
        self.st_params = cat([t.fix_params for t, _, _ in rows], F)
        self.st_state = cat([st for _, st, _ in rows], F)
        self.st_motion = cat([mo for _, _, mo in rows], F)
        return templates

    def _expand(self, starts, counts, offsets=None):
        """Device index vectors of the ranges (start_i, count_i): for each
        element its destination, its source (offset_i + local) and its range."""
        torch = self.torch
        total = int(sum(counts))
        c = torch.tensor(counts, dtype=torch.int64).to(self.dev, non_blocking=True)
        st = torch.tensor(starts, dtype=torch.int64).to(self.dev, non_blocking=True)
        rep = torch.repeat_interleave(torch.arange(len(counts), device=self.dev), c, output_size=total)
        base = torch.cumsum(c, 0) - c
        local = torch.arange(total, device=self.dev) - base[rep]
        dst = st[rep] + local
        src = None
        if offsets is not None:
            src = torch.tensor(offsets, dtype=torch.int64).to(self.dev, non_blocking=True)[rep] + local
        return dst, src, rep, st

    def _flush_updates(self):
        torch = self.torch
        adm = self.pending_admit
        ret = self.pending_retire
        if not adm and not ret:
            return
        with torch.cuda.stream(self.stream):
            keep = []
            nb = nr = 0
            z = self.st_btype[:0]
            bidx = world = btype = fbody = ftype = fhull = fflags = rix = z
            params = self.st_params[:0]
            if adm:
                dst, src, rep, st = self._expand([r.start for r in adm], [r.tmpl.n for r in adm],
                                                 [r.tmpl.offset for r in adm])
                wids = torch.tensor([r.world for r in adm], dtype=torch.int32).to(self.dev, non_blocking=True)
                bidx = dst.to(torch.int32)
                world = wids[rep]
                btype = self.st_btype[src]
                fbody = (st[rep] + self.st_fbody[src]).to(torch.int32)
                ftype = self.st_ftype[src]
                fhull = self.st_fhull[src]
                fflags = self.st_fflags[src]
                params = self.st_params[src].contiguous()
                self.state.index_copy_(0, dst, self.st_state[src])
                self.motion.index_copy_(0, dst, self.st_motion[src])
                nb = len(bidx)
            if ret:
                rdst, _, _, _ = self._expand([a for a, _ in ret], [n for _, n in ret])
                rix = rdst.to(torch.int32)
                nr = len(rix)
            keep = [bidx, world, btype, fbody, ftype, fhull, fflags, params, rix]
            p = lambda t: ctypes.c_void_p(t.data_ptr()) if t.numel() else None
            self._check(self.lib.b3g_update_scene_device(
                self.ctx, nb, p(bidx), p(world), p(btype), nb, p(bidx), p(fbody), p(ftype), p(fhull), p(params),
                p(fflags), nr, p(rix), ctypes.c_void_p(self.sptr)))
            self._keep = keep  # alive until the next update (stream order covers their use)
        self.pending_admit = []
        self.pending_retire = []

    def _integrate(self, n):
        """One kinematic step of body slots [0, n) (b3g_kinematic_step)."""
        self._check(self.lib.b3g_kinematic_step(ctypes.c_void_p(self.state.data_ptr()),
                                                ctypes.c_void_p(self.motion.data_ptr()), n, self.dt,
                                                ctypes.c_void_p(self.sptr)))

    def step(self):
        """One pass over every resident world (admissions and retirements of
        the previous step applied first). Returns the step index."""
        torch = self.torch
        self._flush_updates()
        self._set_active(self.alloc.high_water())
        with torch.cuda.stream(self.stream):
            if self.step_index > 0 or self.resident:
                self._integrate(self.active)
            self._check(self.lib.b3g_collide(self.ctx, ctypes.cast(self.state.data_ptr(), ctypes.POINTER(ctypes.c_float)),
                                             1, ctypes.c_void_p(self.sptr)))
            slot = self.slot
            self.slot = (self.slot + 1) % self.ring
            cd = self.counts_dev[slot]
            self._check(self.lib.b3g_world_counts(self.ctx, self.max_worlds, ctypes.c_void_p(cd.data_ptr()),
                                                  ctypes.c_void_p(self.sptr)))
            self.counts_host[slot].copy_(cd, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.stream)
        finished = []
        for r in list(self.resident.values()):
            if r.done_step is None:
                r.steps_done += 1
                if r.steps_done == r.k:
                    r.done_step = self.step_index
                    finished.append(r)
        for r in finished:
            # Retired before the next pass; the range is free for admissions
            # of the same update (retirement applies first).
            del self.resident[r.rid]
            self.resident_bodies -= r.tmpl.n
            self.world_ids.append(r.world)
            self.alloc.release(r.start)
            self.pending_retire.append((r.start, r.tmpl.n))
        self.events.append((self.step_index, slot, ev, finished))
        self.step_index += 1
        return self.step_index - 1

    def poll(self, block=False):
        """Completes requests whose last step's counts reached the host.
        Returns the completed requests."""
        done = []
        while self.events:
            step, slot, ev, finished = self.events[0]
            if not (block or ev.query()):
                break
            ev.synchronize()
            now = time.perf_counter()
            counts = self.counts_host[slot].numpy()
            for r in finished:
                r.t_done = now
                r.counts = counts[r.world].copy()
            done.extend(finished)
            self.events.popleft()
            block = False
        return done

    def in_flight(self):
        return len(self.events)

    # -- results of the last pass (synchronous; tests and inspection) --------

    def counts(self):
        self.stream.synchronize()
        c = N.Counts()
        self._check(self.lib.b3g_get_counts(self.ctx, ctypes.byref(c)))
        return c.as_dict()

    def world_results(self, req):
        """Contacts (fixtures as indices local to the world), manifolds and
        feature caches of req's world after the last pass, in list order."""
        n = self.counts()["contacts"]
        con = np.zeros((max(n, 1), 3), np.uint32)
        man = np.zeros(max(n, 1), N.MANIFOLD_DTYPE)
        cache = np.zeros((max(n, 1), 4), np.uint32)
        self._check(self.lib.b3g_fetch_contacts(self.ctx, N.ptr(con, u32), n))
        self._check(self.lib.b3g_fetch_manifolds(self.ctx, ctypes.c_void_p(man.ctypes.data), n))
        self._check(self.lib.b3g_fetch_caches(self.ctx, N.ptr(cache, u32), n))
        con, man, cache = con[:n], man[:n], cache[:n]
        lo, hi = req.start, req.start + req.tmpl.n
        sel = (con[:, 0] >= lo) & (con[:, 0] < hi)
        c = con[sel].copy()
        c[:, 0] -= lo
        c[:, 1] -= lo
        return c, man[sel], cache[sel]


def make_templates(engine, n_templates, seed, lo=32, hi=8192):
    """World templates with body counts log-uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_templates):
        n = int(round(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
        out.append(WorldTemplate(int(rng.integers(1 << 31)), n, engine.box_hull, engine.ground_hull,
                                 engine.hull_arrays))
    return engine.load_templates(out)


def run_stream(engine, templates, rate, duration, seed, max_in_flight=2, kmax=16, drain=5.0):
    """Poisson arrivals at `rate` worlds/s for `duration` seconds, each a
    random template asking for K ~ U{1..kmax} passes. Returns the completed
    requests (latency = completion - arrival, wall clock) and the run time;
    the run stops `drain` seconds after the last arrival, so an overloaded
    rate returns fewer requests than arrived."""
    rng = np.random.default_rng(seed)
    n = max(1, int(rng.poisson(rate * duration)))
    arrivals = np.sort(rng.uniform(0.0, duration, n))
    reqs = [Request(i, templates[int(rng.integers(len(templates)))], int(rng.integers(1, kmax + 1)), float(a))
            for i, a in enumerate(arrivals)]
    queue = collections.deque()
    done = []
    nxt = 0
    t0 = time.perf_counter()
    for r in reqs:
        r.arrival += t0
    stop = t0 + duration + drain
    while len(done) < len(reqs):
        now = time.perf_counter()
        if now > stop:
            break
        while nxt < len(reqs) and reqs[nxt].arrival <= now:
            queue.append(reqs[nxt])
            nxt += 1
        while queue and engine.admit(queue[0]):
            queue.popleft()
        if engine.resident:
            while engine.in_flight() >= max_in_flight:
                done.extend(engine.poll(block=True))
            engine.step()
        else:
            if engine.in_flight():
                done.extend(engine.poll(block=True))
            elif nxt < len(reqs):
                time.sleep(max(0.0, min(reqs[nxt].arrival - time.perf_counter(), 0.001)))
        done.extend(engine.poll())
    while engine.in_flight():
        done.extend(engine.poll(block=True))
    t1 = time.perf_counter()
    return done, t1 - t0, len(reqs)
