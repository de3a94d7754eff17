"""The pair search that allocates nothing (b3g_find_pairs_static).

It exists for callers that cannot allocate device memory themselves (an
engine that owns all GPU memory through its own arena, code running inside a
CUDA graph capture, a thread that must not wait on the allocator). Its scratch
is a fixed file-scope device array, so it handles at most
B3G_STATIC_MAX_PROXIES proxies. Here its pairs are checked, through the C ABI,
against the contact set of the main entry point b3g_collide for the same fat
AABBs, on two calls in a row. Collected last so a failure here comes after
every other test has run.
"""
import ctypes

import numpy as np
import pytest

from bounce_b200 import _native as N
from bounce_b200 import scene as S
from bounce_b200.pipeline import CollisionPipeline

MAX_STATIC = 16384


def test_rejects_more_than_the_static_capacity():
    lib = N.load()
    count = ctypes.c_void_p(0)
    # Rejected on the host before any device work.
    assert lib.b3g_find_pairs_static(None, MAX_STATIC + 1, None, 0, count, None) == N.B3G_E_CAPACITY


@pytest.mark.gpu
def test_static_pairs_match_the_pipeline_twice():
    import torch

    lib = N.load()
    # One fixture per dynamic body of registered shape types: the pipeline's
    # contact set is then exactly the set of overlapping fat-AABB pairs.
    sc = S.mixed_scene(seed=21, n=4000, side=20.0).finalize()
    assert sc.n_fixtures <= MAX_STATIC
    drv = S.KinematicDriver(sc)
    pipe = CollisionPipeline(sc)
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    for call in range(2):
        if call:
            for _ in range(3):
                drv.advance()
                pipe.collide(drv.state17())
        else:
            pipe.collide(drv.state17())
        assert pipe.counts()["status"] == 0
        contacts = pipe.contacts()
        want = np.unique(np.stack([np.minimum(contacts[:, 0], contacts[:, 1]),
                                   np.maximum(contacts[:, 0], contacts[:, 1])], axis=1), axis=0)
        aabbs = torch.from_numpy(pipe.fat_aabbs().reshape(-1)).to(dev)
        cap = len(want) + 1024
        pairs = torch.full((cap, 2), -1, dtype=torch.int32, device=dev)
        count = torch.zeros(1, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        rc = lib.b3g_find_pairs_static(
            ctypes.c_void_p(aabbs.data_ptr()), sc.n_fixtures, ctypes.c_void_p(pairs.data_ptr()), cap,
            ctypes.c_void_p(count.data_ptr()), None)
        assert rc == 0
        torch.cuda.synchronize()
        n = int(count.item())
        assert n == len(want), f"call {call}: {n} pairs vs {len(want)} contacts"
        got = np.unique(pairs[:n].cpu().numpy().astype(np.uint32), axis=0)
        assert np.array_equal(got, want), f"call {call}: pair sets differ"
    pipe.close()


def _brute_pairs(aabbs):
    """Every (i, j), i < j, whose closed boxes overlap (b3TestOverlap), by rows."""
    a = aabbs.reshape(-1, 6)
    out = []
    for i0 in range(0, len(a), 512):
        blk = a[i0:i0 + 512]
        ov = ~((blk[:, None, 3] < a[None, :, 0]) | (blk[:, None, 0] > a[None, :, 3]) |
               (blk[:, None, 4] < a[None, :, 1]) | (blk[:, None, 1] > a[None, :, 4]) |
               (blk[:, None, 5] < a[None, :, 2]) | (blk[:, None, 2] > a[None, :, 5]))
        i, j = np.nonzero(ov)
        i = i + i0
        keep = i < j
        out.append(np.stack([i[keep], j[keep]], axis=1))
    return np.concatenate(out).astype(np.uint32)


def _call(lib, torch, aabbs_np, cap):
    dev = torch.device("cuda", 0)
    n = len(aabbs_np) // 6
    aabbs = torch.from_numpy(np.ascontiguousarray(aabbs_np, np.float32)).to(dev) if n else None
    pairs = torch.full((max(cap, 1), 2), -1, dtype=torch.int32, device=dev)
    count = torch.full((1,), 12345, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    rc = lib.b3g_find_pairs_static(ctypes.c_void_p(aabbs.data_ptr() if n else 0), n,
                                   ctypes.c_void_p(pairs.data_ptr()), cap, ctypes.c_void_p(count.data_ptr()), None)
    torch.cuda.synchronize()
    return rc, int(count.item()), pairs.cpu().numpy().astype(np.uint32)


def _boxes(rng, n, side, size):
    lo = rng.uniform(-side / 2, side / 2, (n, 3)).astype(np.float32)
    hi = (lo + rng.uniform(0.1, size, (n, 3))).astype(np.float32)
    return np.ascontiguousarray(np.concatenate([lo, hi], axis=1).reshape(-1))


@pytest.mark.gpu
def test_static_pairs_small_and_clipped():
    """Fewer than two proxies give no pairs; a capacity below the pair count
    keeps the true count and fills the capacity with valid pairs."""
    import torch

    lib = N.load()
    rng = np.random.default_rng(3)
    for n in (0, 1):
        rc, cnt, _ = _call(lib, torch, _boxes(rng, n, 4.0, 1.0), 8)
        assert rc == 0 and cnt == 0, (n, rc, cnt)
    boxes = _boxes(rng, 3000, 10.0, 1.5)
    want = _brute_pairs(boxes)
    assert len(want) > 200
    want_set = set(map(tuple, want.tolist()))
    for cap in (0, 1, 100, len(want) - 1):
        rc, cnt, got = _call(lib, torch, boxes, cap)
        assert rc == 0 and cnt == len(want), (cap, cnt, len(want))
        got = got[:cap]
        assert len(set(map(tuple, got.tolist()))) == cap, cap  # distinct pairs
        assert set(map(tuple, got.tolist())) <= want_set, cap


@pytest.mark.gpu
def test_static_pairs_at_the_static_capacity():
    """n = B3G_STATIC_MAX_PROXIES (the sort's 128 KB of shared memory) against
    a brute-force overlap set."""
    import torch

    lib = N.load()
    rng = np.random.default_rng(4)
    boxes = _boxes(rng, MAX_STATIC, 40.0, 1.2)
    want = _brute_pairs(boxes)
    assert len(want) > 1000
    rc, cnt, got = _call(lib, torch, boxes, len(want) + 16)
    assert rc == 0 and cnt == len(want), (cnt, len(want))
    got = np.unique(got[:cnt], axis=0)
    assert np.array_equal(got, np.unique(want, axis=0))
