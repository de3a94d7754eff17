"""CPU check of the list-order layout and of the wake-up replay the pass
implements (bounce_b200/csrc/order.cu), written here as a plain model of the
kernels' logic and run against the reference's own sequential walk of its
contact list (oracle/_ref, FP32 build):

* new contacts first, in descending (smaller proxy key, larger proxy key)
  order, then the previous contacts in their previous order;
* a previous contact whose pair stopped overlapping is destroyed only if one
  of its bodies is active when the walk reaches it, else kept unchanged;
* wake-ups: a contact that starts or stops touching and a destroyed contact
  with points wake both bodies, for the contacts after it; the model finds
  them as the device does, by rounds of activation against the earliest
  position that woke each body, and must end with the reference's list and
  awake flags.

The narrowphase result of a contact the model activates is taken from the
reference's state after the pass; a contact the model activates that the
reference destroyed (or the reverse) shows up as a list mismatch.
"""
import numpy as np

from bounce_b200 import _native as N
from bounce_b200 import scene as S

INF = np.iinfo(np.int64).max


def model_pass(prev, prev_pc, raw, rank, awake0, body_type, fix_body, fix_flags, ref_final):
    """prev: (np, 3) contacts before the pass (A, B, touching | manifolds << 8);
    prev_pc: their point counts; raw: overlapping pairs (A, B) of this pass;
    ref_final: (A, B) -> flags of the reference after the pass.
    Returns (list of pairs, ended pairs, awake flags, counts of retained
    contacts, late destructions and activation rounds)."""
    prev_index = {(int(a), int(b)): p for p, (a, b) in enumerate(prev[:, :2])}
    raw = [(int(a), int(b)) for a, b in raw]
    new = [pr for pr in raw if pr not in prev_index]
    found = {pr for pr in raw if pr in prev_index}
    new.sort(key=lambda ab: (min(rank[ab[0]], rank[ab[1]]), max(rank[ab[0]], rank[ab[1]])), reverse=True)
    num_new = len(new)

    def active0(b):
        return awake0[b] != 0 and body_type[b] != N.BODY_STATIC

    def sensor(pr):
        return ((fix_flags[pr[0]] | fix_flags[pr[1]]) & N.FIXTURE_SENSOR) != 0

    # entries: [pair, position, previous index, stale]
    entries = [[pr, t, -1, False] for t, pr in enumerate(new)]
    ended = []
    for p, (a, b, _) in enumerate(prev):
        pr = (int(a), int(b))
        if pr in found:
            entries.append([pr, num_new + p, p, False])
        elif active0(fix_body[pr[0]]) or active0(fix_body[pr[1]]):
            ended.append(p)
        else:
            entries.append([pr, num_new + p, p, True])

    t_wake = {}

    def wake(body, pos):
        if not awake0[body]:
            t_wake[body] = min(t_wake.get(body, INF), pos)

    def update(e):
        # The contact is updated: its touching flag is the reference's result.
        pr, pos, p, _ = e
        was = 0 if p < 0 else int(prev[p, 2]) & 1
        now = int(ref_final[pr]) & 1
        if not sensor(pr) and now != was:
            wake(fix_body[pr[0]], pos)
            wake(fix_body[pr[1]], pos)

    def had_points(p):
        return ((int(prev[p, 2]) >> 8) & 0xFF) > 0 and prev_pc[p] > 0

    inactive = []
    for e in entries:
        pr = e[0]
        if active0(fix_body[pr[0]]) or active0(fix_body[pr[1]]):
            update(e)
        else:
            inactive.append(e)
    for p in ended:
        pr = (int(prev[p, 0]), int(prev[p, 1]))
        if had_points(p) and not sensor(pr):
            wake(fix_body[pr[0]], num_new + p)
            wake(fix_body[pr[1]], num_new + p)

    late = set()
    done = [False] * len(inactive)
    rounds = 0
    while True:
        # One device round: decisions against the wake positions known at its start.
        snapshot = dict(t_wake)
        batch = []
        for i, e in enumerate(inactive):
            if done[i]:
                continue
            pr, pos = e[0], e[1]
            ba, bb = fix_body[pr[0]], fix_body[pr[1]]
            if any(body_type[x] != N.BODY_STATIC and snapshot.get(x, INF) < pos for x in (ba, bb)):
                done[i] = True
                batch.append(e)
        if not batch:
            break
        rounds += 1
        for e in batch:
            pr, pos, p, stale = e
            if stale:
                late.add(p)
                if had_points(p) and not sensor(pr):
                    wake(fix_body[pr[0]], pos)
                    wake(fix_body[pr[1]], pos)
            else:
                update(e)
    final = [e[0] for e in entries if not (e[3] and e[2] in late)]
    ended_all = sorted(ended + list(late))
    awake = np.array([1 if (awake0[b] or b in t_wake) else 0 for b in range(len(awake0))], np.uint8)
    info = dict(retained=sum(1 for e in entries if e[3]), late=len(late), rounds=rounds)
    return final, ended_all, awake, info


def run_model(O, sc, passes, seed, sleep_frac):
    rw = O.RefWorld(sc)
    sc.set_local_centers(rw.local_centers())
    drv = S.KinematicDriver(sc)
    rng = np.random.default_rng(seed)
    keys = rw.proxy_ids()
    rank = np.empty(len(keys), np.int64)
    rank[np.argsort(keys, kind="stable")] = np.arange(len(keys))
    rw.first_pass()
    moved = rw.awake()
    stats = dict(woken=0, ended=0, retained=0, late=0, rounds=0, max_rounds=0)
    for k in range(1, passes):
        prev = rw.pairs()
        rc = rw.contacts()
        prev_pc = np.where((prev[:, 2] >> 8) & 0xFF, rc["manifolds"][:, 0]["pointCount"], 0)
        drv.advance(moved)
        awake0 = moved & (rng.random(sc.n_bodies) > sleep_frac).astype(np.uint8)
        rw.set_sweeps(drv.sweeps14())
        rw.step_pass_sleep(moved, awake0)
        fat = rw.fat_aabbs()
        raw = O.restate_pairs(sc, fat, keys=keys)
        cur = rw.pairs()
        ref_final = {(int(a), int(b)): int(f) for a, b, f in cur}
        final, ended, awake, info = model_pass(prev, prev_pc, raw, rank, awake0, sc.body_type, sc.fix_body,
                                         sc.fix_flags, ref_final)
        got = np.array(final, np.uint32).reshape(-1, 2)
        assert len(got) == len(cur), f"pass {k}: {len(got)} contacts vs reference {len(cur)}"
        bad = np.nonzero(np.any(got != cur[:, :2], axis=1))[0]
        assert len(bad) == 0, f"pass {k}: list order differs at {len(bad)} positions, first {bad[:5]}"
        ref_awake = rw.awake()
        badw = np.nonzero(awake != ref_awake)[0]
        assert len(badw) == 0, f"pass {k}: awake flags differ at bodies {badw[:5]}"
        cur_set = {(int(a), int(b)) for a, b in cur[:, :2]}
        want_ended = [p for p in range(len(prev)) if (int(prev[p, 0]), int(prev[p, 1])) not in cur_set]
        assert ended == want_ended, f"pass {k}: destroyed contacts differ"
        stats["woken"] += int(np.count_nonzero((awake != 0) & (awake0 == 0) & (sc.body_type != N.BODY_STATIC)))
        stats["ended"] += len(ended)
        for key in ("retained", "late", "rounds"):
            stats[key] += info[key]
        stats["max_rounds"] = max(stats["max_rounds"], info["rounds"])
        moved = ref_awake
    rw.close()
    return stats


def test_model_sleeping(oracle_mod):
    sc = S.mixed_scene(seed=9, n=1500, side=14.0, static_frac=0.1, sensor_frac=0.05).finalize()
    st = run_model(oracle_mod, sc, 8, seed=100, sleep_frac=0.3)
    # wake-ups, destroyed and retained contacts, late destructions, several rounds
    assert st["woken"] > 0 and st["ended"] > 0 and st["retained"] > 0 and st["late"] > 0, st
    assert st["max_rounds"] >= 2, st


def test_model_mostly_sleeping(oracle_mod):
    sc = S.mixed_scene(seed=13, n=2500, side=15.0, static_frac=0.05, sensor_frac=0.03).finalize()
    st = run_model(oracle_mod, sc, 8, seed=7, sleep_frac=0.8)
    assert st["woken"] > 0 and st["max_rounds"] >= 3, st


def test_model_all_awake(oracle_mod):
    sc = S.mixed_scene(seed=21, n=1500, side=14.0).finalize()
    st = run_model(oracle_mod, sc, 6, seed=1, sleep_frac=0.0)
    assert st["woken"] == 0 and st["ended"] > 0 and st["rounds"] == 0, st
