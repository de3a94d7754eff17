"""Comparison helpers: pipeline results vs reference dumps (test infrastructure)."""
import numpy as np


def keys(a, b):
    return (np.asarray(a, np.uint64) << np.uint64(32)) | np.asarray(b, np.uint64)


def compare_contacts(pipe, rw, label="", check_cache=True):
    """Contact set, touching flags, manifolds and hull feature caches must be
    identical (bit for bit) between the pipeline and the FP32 reference."""
    g = pipe.contacts()
    r = rw.pairs()
    gk, rk = keys(g[:, 0], g[:, 1]), keys(r[:, 0], r[:, 1])
    gs, rs = np.sort(gk), np.sort(rk)
    if not np.array_equal(gs, rs):
        only_g = np.setdiff1d(gs, rs)
        only_r = np.setdiff1d(rs, gs)
        raise AssertionError(
            f"{label}: contact sets differ: gpu {len(gs)} ref {len(rs)}; "
            f"gpu-only {[(int(k >> 32), int(k & 0xFFFFFFFF)) for k in only_g[:5]]} "
            f"ref-only {[(int(k >> 32), int(k & 0xFFFFFFFF)) for k in only_r[:5]]}"
        )
    gi = np.argsort(gk)
    rc = rw.contacts()
    ri = np.argsort(keys(rc["fixtureA"], rc["fixtureB"]))
    gt = g[gi, 2] & 1
    rt = rc["flags"][ri] & 1
    bad = np.nonzero(gt != rt)[0]
    assert len(bad) == 0, f"{label}: touching flags differ at {len(bad)} contacts, e.g. {gk[gi][bad[:3]]}"
    gm = pipe.manifolds()[gi]
    rm = rc["manifolds"][ri, 0]
    rcount = rc["manifoldCount"][ri]
    gcount = (g[gi, 2] >> 8) & 0xFF
    assert np.array_equal(gcount, rcount), f"{label}: manifold counts differ"
    gpc = np.where(gcount > 0, gm["pointCount"], 0)
    rpc = np.where(rcount > 0, rm["pointCount"], 0)
    badpc = np.nonzero(gpc != rpc)[0]
    assert len(badpc) == 0, (
        f"{label}: point counts differ at {len(badpc)} of {len(gpc)} contacts; first "
        f"{[(int(gk[gi][i] >> 32), int(gk[gi][i] & 0xFFFFFFFF), int(gpc[i]), int(rpc[i])) for i in badpc[:5]]}"
    )
    _compare_points(gm, rm, gpc, label)
    if np.any(rcount > 1):
        ref_of_gpu = np.empty(len(gi), np.int64)
        ref_of_gpu[gi] = ri
        compare_all_manifolds(pipe, rc, ref_of_gpu, label)
    if check_cache:
        gc = pipe.caches()[gi]
        rcache = rc["cache"][ri]
        hh = rcache[:, 0] != 0xFFFFFFFF
        # An e_empty cache (type 0) leaves its other fields unset in the
        # reference (sat.h:69): only the type is compared there.
        empty = rcache[:, 0] == 0
        same = np.where(empty[:, None], gc[:, :1] == rcache[:, :1], gc == rcache)
        bad = np.nonzero(~np.all(same[hh], axis=1))[0]
        assert len(bad) == 0, f"{label}: feature caches differ at {len(bad)}: {gc[hh][bad[:3]]} vs {rcache[hh][bad[:3]]}"
    return dict(contacts=len(gs), touching=int(gt.sum()), points=int(gpc.sum()))


def _compare_points(gm, rm, gpc, label):
    """Points of manifolds gm (pipeline) and rm (reference), pointCount gpc each."""
    mask = np.arange(4)[None, :] < gpc[:, None]
    for f in ("n", "p1", "p2"):
        a = gm["points"][f][mask]
        b = rm["points"][f][mask].astype(np.float32)
        bad = np.nonzero(~np.all(a == b, axis=-1))[0]
        assert len(bad) == 0, f"{label}: manifold field {f} differs at {len(bad)} points; e.g. {a[bad[:2]]} vs {b[bad[:2]]}"
    assert np.array_equal(gm["points"]["key"][mask], rm["points"]["key"][mask]), f"{label}: feature ids differ"
    assert np.array_equal(gm["points"]["triangleKey"][mask], rm["points"]["triangleKey"][mask])
    assert np.array_equal(gm["points"]["edgeContact"][mask], rm["points"]["edgeContact"][mask].astype(np.uint8))
    assert np.array_equal(gm["points"]["persisting"][mask], rm["points"]["persisting"][mask].astype(np.uint8)), (
        f"{label}: persisting flags differ"
    )
    assert np.array_equal(gm["points"]["normalImpulse"][mask], rm["points"]["normalImpulse"][mask].astype(np.float32)), (
        f"{label}: normal impulses differ"
    )
    has = gpc > 0
    assert np.array_equal(gm["tangentImpulse"][has], rm["tangentImpulse"][has].astype(np.float32)), (
        f"{label}: tangent impulses differ"
    )
    assert np.array_equal(gm["motorImpulse"][has], rm["motorImpulse"][has].astype(np.float32)), (
        f"{label}: motor impulses differ"
    )


def compare_all_manifolds(pipe, rc, ref_of_gpu, label=""):
    """Every manifold with points (manifolds 1 and 2 of mesh contacts too), in
    contact and manifold order, against the reference's b3Contact::m_manifolds."""
    idx, man = pipe.touching()
    exp_idx, exp_man = [], []
    for c, r in enumerate(ref_of_gpu):
        for k in range(int(rc["manifoldCount"][r])):
            m = rc["manifolds"][r, k]
            if m["pointCount"] > 0:
                exp_idx.append(c)
                exp_man.append(m)
    exp_idx = np.asarray(exp_idx, np.uint32)
    assert np.array_equal(idx, exp_idx), (
        f"{label}: manifolds with points differ: gpu {len(idx)} ref {len(exp_idx)}"
    )
    if len(exp_man) == 0:
        return
    rm = np.stack(exp_man)
    gpc = man["pointCount"]
    assert np.array_equal(gpc, rm["pointCount"]), f"{label}: point counts of all manifolds differ"
    _compare_points(man, rm, gpc, label + " (all manifolds)")


def compare_fat_aabbs(pipe, rw, label=""):
    a = pipe.fat_aabbs()
    b = rw.fat_aabbs()
    bad = np.nonzero(~np.all(a == b, axis=1))[0]
    assert len(bad) == 0, f"{label}: fat AABBs differ at {len(bad)} proxies, e.g. {a[bad[:2]]} vs {b[bad[:2]]}"


class BatchedPass:
    """One pass's results of a many-world pipeline, fetched once, from which
    WorldView gives each world's part in the shape of a one-world pipeline."""

    def __init__(self, pipe, scene):
        self.c = pipe.contacts()
        self.m = pipe.manifolds()
        self.cache = pipe.caches()
        self.fat = pipe.fat_aabbs()
        self.end = pipe.ended()
        self.fix_world = scene.body_world[scene.fix_body]
        self.n_fixtures = scene.n_fixtures


class WorldView:
    """World w of a BatchedPass with fixture indices local to the world (the
    indices of world_subset(w)), in the world's own list order."""

    def __init__(self, bp, w, fixtures):
        local = np.full(bp.n_fixtures, -1, np.int64)
        local[fixtures] = np.arange(len(fixtures))
        sel = bp.fix_world[bp.c[:, 0]] == w
        c = bp.c[sel].astype(np.int64)
        c[:, 0] = local[c[:, 0]]
        c[:, 1] = local[c[:, 1]]
        self._c = c.astype(np.uint32)
        self._m = bp.m[sel]
        self._cache = bp.cache[sel]
        self._fat = bp.fat[fixtures]
        if len(bp.end):
            e = bp.end[bp.fix_world[bp.end[:, 0]] == w].astype(np.int64)
            e[:, 0] = local[e[:, 0]]
            e[:, 1] = local[e[:, 1]]
        else:
            e = np.zeros((0, 3), np.int64)
        self._e = e.astype(np.uint32)

    def contacts(self):
        return self._c

    def manifolds(self):
        return self._m

    def caches(self):
        return self._cache

    def fat_aabbs(self):
        return self._fat

    def ended(self):
        return self._e


def compare_order(pipe, rw, label):
    """The contact arrays follow the reference's contact list exactly:
    fixtures, touching flag and manifold count per position."""
    g = pipe.contacts()
    r = rw.pairs()
    assert len(g) == len(r), f"{label}: {len(g)} contacts vs {len(r)}"
    bad = np.nonzero(np.any(g[:, :2] != r[:, :2], axis=1))[0]
    assert len(bad) == 0, f"{label}: list order differs at {len(bad)} positions, first {bad[:5]}: {g[bad[:3]]} vs {r[bad[:3]]}"
    assert np.array_equal(g[:, 2] & 0xFF01, r[:, 2] & 0xFF01), f"{label}: flags differ in list order"


def compare_ended(pipe, prev, cur, label):
    """The contacts destroyed by the pass, in the previous list's order, with
    their touching flags (prev, cur: the reference's lists before and after)."""
    ck = set(map(tuple, cur[:, :2].tolist()))
    want = np.array([r for r in prev.tolist() if (r[0], r[1]) not in ck], np.uint32).reshape(-1, 3)
    got = pipe.ended()
    assert np.array_equal(got[:, :2], want[:, :2]), f"{label}: ended list"
    assert np.array_equal(got[:, 2] & 1, want[:, 2] & 1), f"{label}: ended touching flags"
