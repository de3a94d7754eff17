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
