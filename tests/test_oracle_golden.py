"""The oracle (oracle/fg_oracle.c) against the golden vectors of the reference's own proto/interp.py: every stage
bit-exact, every decision identical. This pins the checker that the CUDA parity tests use."""
import numpy as np
import pytest

import oracle
from golden_io import golden, scene_inputs, scene_names, sha, times

WHY = {None: 0, "cut": 1, "untrusted": 2}


@pytest.mark.parametrize("name", scene_names())
def test_estimate_stages(name):
    g = golden()
    p, c = scene_inputs(name)
    bgr = lambda x: np.ascontiguousarray(x[..., [2, 1, 0]])
    est = oracle.estimate(bgr(p), bgr(c), order="bgr")
    n = len(est["layout"].levels)
    for l in range(n):
        assert np.array_equal(est["fields"][l][0], g[f"{name}/search{l}"]), f"search level {l}"
        assert np.array_equal(est["fields"][l][1], g[f"{name}/median{l}"]), f"median3 level {l}"
    assert f"{name}/search{n}" not in g, "pyramid depth differs"
    for k in range(2):
        assert np.array_equal(est["sub"][k], g[f"{name}/sub{k}"]), f"subpixel step {k}"
    assert np.array_equal(est["sads"], g[f"{name}/sads"])
    assert est["sad"] == float(g[f"{name}/sad"][0])
    if f"{name}/pf" in g:
        assert not est["cut"]
        assert np.array_equal(est["pf"], g[f"{name}/pf"])
    else:
        assert est["cut"]


@pytest.mark.parametrize("name", scene_names())
def test_synth_frames(name):
    g = golden()
    p, c = scene_inputs(name)
    est = oracle.estimate(p, c, trace=False)   # RGBA order: the same arithmetic, channels re-addressed
    for k, t in enumerate(times()):
        out, why = oracle.synth(p, c, est, t)
        assert WHY[why] == int(g[f"{name}/why_t{k}"][0]), f"decision at t={t}"
        bgr = np.ascontiguousarray(out[..., [2, 1, 0]])
        if f"{name}/out_t{k}" in g:
            ref = g[f"{name}/out_t{k}"]
            assert np.array_equal(bgr, ref), f"t={t}: {np.count_nonzero(bgr != ref)} bytes differ"
        else:
            assert np.array_equal(sha(bgr), g[f"{name}/outsha_t{k}"]), f"t={t}: frame digest differs"
        assert np.all(out[..., 3] == (p if t <= 0.5 else c)[..., 3]), "alpha is the nearer frame's"


def test_pairwise_mean_matches_numpy():
    rng = np.random.default_rng(0)
    for n in (1, 7, 8, 9, 127, 128, 129, 1000, 32400, 129600):
        a = (rng.integers(0, 255 * 4096, n) / 4096).astype(np.float32)
        assert oracle.mean_f32(a) == float(a.mean())


def test_layout_matches_reference_sizes():
    """interp.pyramid level sizes (rint half-even, stop when min // 2 < 48) for the standard frame sizes."""
    exp = {(640, 360): [(320, 180), (160, 90)],
           (1920, 1080): [(960, 540), (480, 270), (240, 135), (120, 68)],
           (3840, 2160): [(1920, 1080), (960, 540), (480, 270), (240, 135), (120, 68)],
           (2560, 1440): [(1280, 720), (640, 360), (320, 180), (160, 90)]}
    for (W, H), lv in exp.items():
        L = oracle.layout(W, H)
        assert [(w, h) for w, h, _, _ in L.levels] == lv
