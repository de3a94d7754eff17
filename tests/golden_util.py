"""Loading the golden fixtures of tests/golden (test infrastructure)."""
import os

import numpy as np

from bounce_b200 import scene as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SCENES = ("plain_small", "mixed_small")
PASSES = 3


def load(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def scene_from(d):
    """Rebuild the Scene the fixture was made from (arrays as stored)."""
    sc = S.Scene()
    sc.hull_arrays = {k: np.ascontiguousarray(d[f"hull_{k}"]) for k in
                      ("desc", "verts", "edges", "faces", "planes", "centroids")}
    for k in ("body_world", "body_type", "body_pose", "body_lin", "body_ang", "fix_body", "fix_type", "fix_hull",
              "fix_params", "fix_flags", "local_center"):
        setattr(sc, k, np.ascontiguousarray(d[k]))
    sc.body_pos = np.ascontiguousarray(sc.body_pose[:, :3])
    sc.body_quat = np.ascontiguousarray(sc.body_pose[:, 3:])
    return sc


def contact_keys(pairs):
    return (pairs[:, 0].astype(np.uint64) << 32) | pairs[:, 1]
