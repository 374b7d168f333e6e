"""Motion blur without a GPU: the oracle's blur (oracle.synth_blur) against the reference's own definition of
recordSynthBlur, and the library's host-side sample plan against the oracle's.

The reference checks its blur (gpu/blurtest.cpp:757-806) against the double-precision weighted average of the
recordSynth sub-frames, rounded half up, allowing 1 level, for N = 2..8, the windows [.5, 1], [.25, .75], [0, 1],
[.1, .4], [.6, .9], both weights, and with the scene cut and the whole-frame flick forced. The oracle fixes the
rounding (weights in units of 2^-16); here it must meet that same bar, and equal the double model exactly where the
weights are exact in both (even weights, N a power of two).
"""
import math

import numpy as np
import pytest

import framegen as fg
import oracle
import workloads

WINDOWS = [(0.5, 1.0), (0.25, 0.75), (0.0, 1.0), (0.1, 0.4), (0.6, 0.9)]


@pytest.fixture(scope="module", autouse=True)
def built():
    import build
    build.build()


def reference_model(subs, n, gaussian):
    """gpu/blurtest.cpp:610-620 + 793-797: weights normalised in double, sum_k w_k v_k, floor(a + 0.5)"""
    g = []
    for k in range(n):
        x = (2.0 * k + 1 - n) / n
        g.append(math.exp(-2.0 * x * x) if gaussian else 1.0)
    s = sum(g)
    a = np.zeros(np.shape(subs[0]), np.float64)
    for wk, f in zip(g, subs):
        a += (wk / s) * f.astype(np.float64)
    return np.floor(a + 0.5).astype(np.int64)


def test_plan_library_equals_oracle():
    cases = [(n, g, t0, t1) for n in (0, 1, 2, 3, 4, 5, 6, 7, 8, 11, 16) for g in (0, 1)
             for t0, t1 in WINDOWS + [(0.3, 0.3), (0.0, 0.0), (1.0, 1.0), (0.9999999, 1.0), (0.0, 1e-7)]]
    for n, g, t0, t1 in cases:
        lib_plan = fg.blur_plan(n, g, t0, t1)
        ref_plan = oracle.blur_plan(n, g, t0, t1)
        assert lib_plan is not None and ref_plan is not None
        assert np.array_equal(lib_plan[0], ref_plan[0]), (n, g, t0, t1)
        assert lib_plan[1] == ref_plan[1], (n, g, t0, t1)
        assert sum(ref_plan[1]) == 65536
        assert all(np.float32(t0) <= t <= np.float32(t1) for t in ref_plan[0])
    for bad in [(4, 0, 0.6, 0.5), (4, 0, -0.1, 0.5), (4, 0, 0.2, 1.5), (4, 0, float("nan"), 0.5)]:
        assert fg.blur_plan(*bad) is None and oracle.blur_plan(*bad) is None


def test_plan_midpoints_and_weights():
    t, q = oracle.blur_plan(4, False, 0.0, 1.0)
    assert t.tolist() == [0.125, 0.375, 0.625, 0.875] and q == [16384] * 4
    t, q = oracle.blur_plan(3, True, 0.25, 0.75)
    assert q[0] == q[2] or abs(q[0] - q[2]) == 1
    assert q[1] > q[0]
    # blur off: one instant at the window's END
    t, q = oracle.blur_plan(1, True, 0.2, 0.6)
    assert t.tolist() == [np.float32(0.6)] and q == [65536]


@pytest.fixture(scope="module")
def pair():
    p, c, _ = workloads.flow_pair(192, 108, seed=7)
    return p, c


@pytest.mark.parametrize("variant", [("default", 30.0, 0.15), ("cut forced", 0.5, 0.15),
                                     ("flick forced", 30.0, 0.001), ("flick on some samples", 30.0, 0.0323),
                                     ("flick on more samples", 30.0, 0.0321)])
def test_oracle_blur_meets_the_reference_bar(pair, variant):
    """(this pair's syntheses leave 659..678 of 20,736 pixels untrusted, more at small t: a flick threshold of
    0.0323 / 0.0321 falls back on the earlier samples of a window only)"""
    name, cut, flick = variant
    p, c = pair
    s = oracle.Settings(sceneCutSad=cut, globalFallback=flick)
    est = oracle.estimate(p, c, settings=s, trace=False)
    worst, off = 0, 0
    ns = range(2, 9) if name == "default" else (3, 4, 7)
    for n in ns:
        for t0, t1 in WINDOWS:
            for gaussian in (False, True):
                subs = oracle.blur_subframes(p, c, est, t0, t1, n, gaussian, s)
                got = ((sum(q * f.astype(np.int64) for _, q, f in subs) + 32768) >> 16)
                assert np.array_equal(got.astype(np.uint8), oracle.synth_blur(p, c, est, t0, t1, n, gaussian, s))
                want = reference_model([f for _, _, f in subs], n, gaussian)
                d = np.abs(got - want)
                worst = max(worst, int(d.max()))
                off += int((d > 0).sum())
                if not gaussian and n in (2, 4, 8):
                    assert not d.any(), f"{name}: N={n} [{t0},{t1}] even weights must be exact"
    assert worst <= 1, f"{name}: the oracle differs from the double-precision average by {worst} levels"


def test_oracle_blur_instants(pair):
    p, c = pair
    est = oracle.estimate(p, c, trace=False)
    mid, _ = oracle.synth(p, c, est, 0.3)
    assert np.array_equal(oracle.synth_blur(p, c, est, 0.3, 0.3, 8, True), mid)      # t0 == t1
    assert np.array_equal(oracle.synth_blur(p, c, est, 0.1, 0.3, 1, True), mid)      # blur off: t1
    assert np.array_equal(oracle.synth_blur(p, c, est, 1.0, 1.0, 4, False), c)       # a real-frame instant
    assert np.array_equal(oracle.synth_blur(p, c, est, 0.0, 0.0, 4, False), p)
    assert oracle.synth_blur(p, c, est, 0.7, 0.2, 4, False) is None


@pytest.mark.parametrize("fmt", ["rgb10", "f16", "nv12", "p010"])
def test_oracle_blur_formats(fmt):
    """the other formats: instants are synth_fmt's frames; the average stays between the sub-frames' extremes and,
    for the integer formats, within 1 code of the double-precision weighted mean of their codes"""
    spec = {"rgb10": oracle.FormatSpec("rgb10"), "f16": oracle.FormatSpec("f16", linear=True, white=80.0),
            "nv12": oracle.FormatSpec("nv12", matrix="bt709"), "p010": oracle.FormatSpec("p010", matrix="bt2020")}[fmt]
    p8, c8, _ = workloads.flow_pair(96, 64, seed=23)
    conv = {"rgb10": workloads.to_rgb10, "f16": lambda f: workloads.to_f16(f, linear=True),
            "nv12": lambda f: workloads.to_yuv(f, 8, "bt709"), "p010": lambda f: workloads.to_yuv(f, 10, "bt2020")}[fmt]
    a, c = conv(p8), conv(c8)
    est = oracle.estimate_fmt(a, c, spec, trace=False)
    planes = lambda f: list(f) if isinstance(f, tuple) else [f]
    s30 = oracle.synth_fmt(a, c, est, float(np.float32(0.3)), spec)[0]
    for got in (oracle.synth_blur_fmt(a, c, est, 0.3, 0.3, 8, True, spec),
                oracle.synth_blur_fmt(a, c, est, 0.1, 0.3, 1, True, spec)):
        assert all(np.array_equal(x, y) for x, y in zip(planes(got), planes(s30)))
    assert all(np.array_equal(x, y) for x, y in zip(planes(oracle.synth_blur_fmt(a, c, est, 1.0, 1.0, 4, False, spec)),
                                                    planes(c)))
    assert oracle.synth_blur_fmt(a, c, est, 0.7, 0.2, 4, False, spec) is None
    n, gaussian = 5, True
    times, q = oracle.blur_plan(n, gaussian, 0.1, 0.9)
    subs = [oracle.synth_fmt(a, c, est, float(t), spec)[0] for t in times.tolist()]
    got = oracle.synth_blur_fmt(a, c, est, 0.1, 0.9, n, gaussian, spec)
    for k, gp in enumerate(planes(got)):
        sp = [planes(f)[k] for f in subs]
        if fmt == "f16":
            v = np.stack([x.astype(np.float64) for x in sp])
            g = gp.astype(np.float64)
            assert np.all(g >= v.min(0) - 1e-3 * np.abs(v.min(0))) and np.all(g <= v.max(0) + 1e-3 * np.abs(v.max(0)))
            continue
        shift = 6 if fmt == "p010" else 0
        fields = [(0, 1023), (10, 1023), (20, 1023)] if fmt == "rgb10" else [(0, (1 << 16) - 1)]
        for pos, mask in fields:
            codes = np.stack([((x.astype(np.int64) >> shift) >> pos) & mask for x in sp])
            want = np.tensordot(np.array(q, np.float64) / 65536.0, codes.astype(np.float64), axes=1)
            gc = ((gp.astype(np.int64) >> shift) >> pos) & mask
            assert np.abs(gc - want).max() <= 1.0
