"""Live check of the oracle against the reference's proto/interp.py on more seeded scenes. Runs only where FGR_REF names
a checkout of the reference (the directory that holds proto/interp.py); skipped otherwise."""
import hashlib
import os
import sys

import numpy as np
import pytest

import oracle
import workloads

REF = os.environ.get("FGR_REF")
PIN = "b5f5c7000221002e31a1f4c2b2883878eeab4ffd83760c4080facad527904315"


@pytest.fixture(scope="module")
def interp():
    if not REF:
        pytest.skip("FGR_REF is not set")
    path = os.path.join(REF, "proto", "interp.py")
    if not os.path.isfile(path):
        pytest.skip("reference checkout not present at FGR_REF")
    pytest.importorskip("cv2")
    assert hashlib.sha256(open(path, "rb").read()).hexdigest() == PIN
    sys.path.insert(0, os.path.dirname(path))
    import interp as m
    return m


@pytest.mark.parametrize("W,H,seed,kind", [(64, 48, 1, "normal"), (97, 61, 2, "fresh"), (250, 140, 3, "normal"),
                                           (96, 96, 4, "cut"), (203, 117, 5, "normal")])
def test_random_scenes(interp, W, H, seed, kind):
    p, c, _ = workloads.flow_pair(W, H, seed=seed, kind=kind)
    a, cc = p[..., [2, 1, 0]].copy(), c[..., [2, 1, 0]].copy()
    ei, eo = interp.estimate(a, cc), oracle.estimate(a, cc, order="bgr", trace=False)
    assert ei["sad"] == eo["sad"]
    if ei["pf"] is not None:
        assert np.array_equal(ei["pf"], eo["pf"])
    for t in (0.5, 0.25, float(np.float32(0.6)), float(np.float32(1 / 3))):
        oi, wi = interp.synth(a, cc, ei, t, why=True)
        oo, wo = oracle.synth(a, cc, eo, t, order="bgr")
        assert wi == wo and np.array_equal(oi, oo)
