"""Serving: a world's collision results are the same alone and in the mix.

The mix admits and retires worlds around the world under test (it lands in a
range another world held before, next to worlds still running); the world
alone runs in a context of its own. Its contact list (order included, with
fixture indices local to the world), manifolds, feature caches and per-world
counts must be identical, bit for bit.
"""
import numpy as np
import pytest

from bounce_b200 import serving as SV

pytestmark = pytest.mark.gpu


def results_equal(a, b, label):
    ca, ma, ka = a
    cb, mb, kb = b
    assert np.array_equal(ca, cb), f"{label}: contact lists differ ({len(ca)} vs {len(cb)})"
    pc = np.where((ca[:, 2] >> 8) & 0xFF, ma["pointCount"], 0)
    pcb = np.where((cb[:, 2] >> 8) & 0xFF, mb["pointCount"], 0)
    assert np.array_equal(pc, pcb), f"{label}: point counts differ"
    mask = np.arange(4)[None, :] < pc[:, None]
    for f in ("n", "p1", "p2", "key", "normalImpulse", "persisting"):
        assert np.array_equal(ma["points"][f][mask], mb["points"][f][mask]), f"{label}: {f} differ"
    hh = ka[:, 0] != 0xFFFFFFFF
    assert np.array_equal(ka[hh], kb[hh]), f"{label}: caches differ"


def test_world_alone_equals_in_mix():
    mix = SV.ServingEngine(capacity=1 << 16, max_worlds=64, active_quantum=4096)
    tmpls = sorted(SV.make_templates(mix, 6, seed=4, lo=64, hi=1500), key=lambda t: t.n)
    # Steps 0-2: three worlds; the middle one (the largest template, K=2)
    # finishes at step 1, and its range is reused by the target (the second
    # largest), admitted at step 3 with K = 6.
    target = tmpls[4]
    r = [SV.Request(i, tmpls[j], k, 0.0) for i, (j, k) in enumerate(((0, 8), (5, 2), (1, 10)))]
    for q in r:
        assert mix.admit(q)
    mix.step()
    mix.step()
    mix.step()
    t = SV.Request(10, target, 6, 0.0)
    assert mix.admit(t)
    assert t.start == r[1].start, "the target reuses the finished world's range"
    late = SV.Request(11, tmpls[2], 5, 0.0)
    assert mix.admit(late)
    got = None
    for _ in range(6):
        mix.step()
        if t.done_step is not None and got is None:
            got = mix.world_results(t)
    mix.poll(block=True)
    assert got is not None and t.counts is not None
    assert mix.counts()["status"] == 0
    mix.close()

    alone = SV.ServingEngine(capacity=1 << 16, max_worlds=64, active_quantum=4096)
    alone.load_templates(tmpls)
    a = SV.Request(0, target, 6, 0.0)
    assert alone.admit(a) and a.start == 0
    ref = None
    for _ in range(6):
        alone.step()
        if a.done_step is not None and ref is None:
            ref = alone.world_results(a)
    alone.poll(block=True)
    alone.close()
    results_equal(got, ref, "target world")
    assert np.array_equal(t.counts, a.counts)
    assert int(a.counts[0]) > 0, "the world has touching contacts"


def test_stream_completes_every_request():
    eng = SV.ServingEngine(capacity=1 << 17, max_worlds=256, active_quantum=8192)
    tmpls = SV.make_templates(eng, 16, seed=9, lo=32, hi=2048)
    done, wall, arrived = SV.run_stream(eng, tmpls, rate=2000.0, duration=0.25, seed=1)
    assert len(done) == arrived
    assert all(r.t_done is not None and r.t_done >= r.arrival for r in done)
    assert len({r.rid for r in done}) == len(done)
    lat = np.array([r.t_done - r.arrival for r in done]) * 1e3
    print(f"{len(done)} requests, p50 {np.percentile(lat, 50):.2f} ms, p99 {np.percentile(lat, 99):.2f} ms")
    assert eng.counts()["status"] == 0
    eng.close()
