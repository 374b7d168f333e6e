"""Loads the golden fixtures made by tests/golden/gen_golden.py from the reference's proto/interp.py, and rebuilds
each scene's input pair from the seeded generator (checked against the stored digest)."""
import hashlib
import os

import numpy as np

import workloads

HERE = os.path.dirname(os.path.abspath(__file__))
_G = None


def golden():
    global _G
    if _G is None:
        _G = dict(np.load(os.path.join(HERE, "golden", "v1_golden.npz")))
    return _G


def scene_inputs(name):
    """The scene's (prev, curr) RGBA8, regenerated exactly as gen_golden.py made them."""
    if name == "pan640x360":
        p, c = workloads.pan_pair()
    elif name.startswith("pan"):
        W, H = map(int, name[3:].split("x"))
        p, c = workloads.pan_pair(W, H, seed=W)
    elif name.startswith("flow_"):
        kind = name[5:].split("320")[0]
        p, c, _ = workloads.flow_pair(320, 180, seed=7, kind=kind)
    elif name.startswith("hardcut"):
        p, c = workloads.contrast_pair(160, 96, seed=5, kind="cut")
    else:
        raise KeyError(name)
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(p).tobytes())
    h.update(np.ascontiguousarray(c).tobytes())
    assert np.array_equal(np.frombuffer(h.digest(), np.uint8), golden()[f"{name}/in_sha"]), \
        f"{name}: the workload generator no longer makes the fixture's inputs"
    return p, c


def sha(a):
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), np.uint8)


def scene_names():
    return [str(s) for s in golden()["scenes"]]


def times():
    return [float(t) for t in golden()["ts"]]
