"""The oracle's restatement of the other frame formats (oracle/fg_oracle_fmt.c): its float helpers against numpy and
float64 mathematics, its luma against an independent numpy statement of the same rules, and known answers (a still
pair comes back unchanged in every format, an integer pan is found). CPU only."""
import math

import numpy as np
import pytest

import oracle
import workloads

SPECS = {
    "rgb10": oracle.FormatSpec("rgb10"),
    "rgb10_rhigh": oracle.FormatSpec("rgb10", r_high=True),
    "f16_linear": oracle.FormatSpec("f16", linear=True),
    "f16_encoded": oracle.FormatSpec("f16"),
    "nv12": oracle.FormatSpec("nv12"),
    "nv12_full": oracle.FormatSpec("nv12", matrix="bt601", full_range=True),
    "p010": oracle.FormatSpec("p010", matrix="bt2020"),
}
CONV = {
    "rgb10": lambda f: workloads.to_rgb10(f),
    "rgb10_rhigh": lambda f: workloads.to_rgb10(f, r_high=True),
    "f16_linear": lambda f: workloads.to_f16(f, True),
    "f16_encoded": lambda f: workloads.to_f16(f, False),
    "nv12": lambda f: workloads.to_yuv(f, 8, "bt709"),
    "nv12_full": lambda f: workloads.to_yuv(f, 8, "bt601", True),
    "p010": lambda f: workloads.to_yuv(f, 10, "bt2020"),
}


def pq_ref(v, white=80.0):
    """SMPTE ST 2084 inverse EOTF in float64, times 255"""
    y = min(max(v * white / 10000.0, 0.0), 1.0)
    m1, m2, c1, c2, c3 = 0.1593017578125, 78.84375, 0.8359375, 18.8515625, 18.6875
    p = y ** m1
    return ((c1 + c2 * p) / (1 + c3 * p)) ** m2 * 255.0


def test_pq_against_float64():
    rng = np.random.default_rng(0)
    vs = np.concatenate([np.exp(rng.uniform(np.log(1e-5), np.log(300.0), 4000)), [0.0, 1e-30, 125.0, 1e6, -3.0]])
    for white in (80.0, 203.0, 10000.0):
        err = max(abs(oracle.pq255(float(np.float32(v)), white) - pq_ref(float(np.float32(v)), white)) for v in vs)
        assert err < 0.01, (white, err)   # levels; a level is the metric's unit


def test_log2_exp2_series():
    rng = np.random.default_rng(1)
    xs = np.exp(rng.uniform(-80.0, 5.0, 3000)).astype(np.float32)
    assert max(abs(oracle.log2(x) - math.log2(x)) / max(abs(math.log2(x)), 1e-3) for x in xs) < 1e-6
    es = rng.uniform(-120.0, 10.0, 3000).astype(np.float32)
    assert max(abs(oracle.exp2(x) - 2.0 ** float(x)) / 2.0 ** float(x) for x in es) < 1e-6
    assert oracle.exp2(-127.0) == 0.0 and oracle.exp2(0.0) == pytest.approx(1.0, rel=1e-7)


def test_half_conversions_match_numpy():
    rng = np.random.default_rng(2)
    fs = np.concatenate([rng.standard_normal(20000).astype(np.float32) * np.float32(3000),
                         (rng.standard_normal(20000) * 1e-5).astype(np.float32),
                         np.array([65504, 65519.99, 65520, 1e-8, 2 ** -24, 2 ** -25, 3 * 2 ** -26, 2 ** -14, -0.0,
                                   np.inf, -np.inf], np.float32)])
    with np.errstate(over="ignore"):
        ref = fs.astype(np.float16).view(np.uint16)
    assert np.array_equal(np.array([oracle.f2h(float(v)) for v in fs], np.uint16), ref)
    hs = np.arange(0, 65536, 7, dtype=np.uint16)
    got = np.array([oracle.h2f(int(h)) for h in hs], np.float32)
    want = hs.view(np.float16).astype(np.float32)
    assert np.array_equal(got[~np.isnan(want)], want[~np.isnan(want)])


def test_yuv_constants_match_the_reference_formula():
    """gpu/framegen.cpp:1518-1533: R' = ys dY + rcr dCr, G' = ys dY + gcb dCb + gcr dCr, B' = ys dY + bcb dCb"""
    for matrix, (kr, kb) in {"bt601": (0.299, 0.114), "bt709": (0.2126, 0.0722), "bt2020": (0.2627, 0.0593)}.items():
        for full in (False, True):
            f = oracle.fmt_struct(oracle.FormatSpec("nv12", matrix=matrix, full_range=full))
            kg = 1 - kr - kb
            sy, sc = (1.0, 1.0) if full else (255 / 219, 255 / 224)
            assert f.ys == np.float32(sy) and f.black == (0.0 if full else 16.0)
            assert f.rcr == np.float32(sc * 2 * (1 - kr)) and f.bcb == np.float32(sc * 2 * (1 - kb))
            assert f.gcb == np.float32(-sc * 2 * (1 - kb) * kb / kg) and f.gcr == np.float32(-sc * 2 * (1 - kr) * kr / kg)


def luma_numpy(frame, spec, fs):
    """level-0 luma of the restatement, stated again with numpy float32 (luma.comp:9-27, format.glsl fgLuma)"""
    f32 = np.float32
    if spec.format == "rgb10":
        sh = (20, 10, 0) if spec.r_high else (0, 10, 20)
        lv = [((frame >> s) & 1023).astype(f32) * f32(255.0 / 1023.0) for s in sh]
    elif spec.format == "f16":
        v = frame[..., :3].astype(f32)
        if spec.linear:
            lv = [np.vectorize(lambda x: np.float32(oracle.pq255(float(x), spec.white)))(v[..., k]).astype(f32)
                  for k in range(3)]
        else:
            lv = [v[..., k] * f32(255.0) for k in range(3)]
    if spec.format in ("rgb10", "f16"):
        d = f32(4899.0) * lv[0]
        d = d + f32(9617.0) * lv[1]
        d = d + f32(1868.0) * lv[2]
        y = d * f32(1.0 / 16384.0)
    else:
        f = oracle.fmt_struct(spec)
        lev = frame[0].astype(f32) * (f32(1.0) if spec.format == "nv12" else f32(2.0 ** -8))
        y = (lev - f32(f.black)) * f32(f.ys)
    q = np.rint(np.clip(y, 0, 255) * f32(4.0)).astype(np.int64)
    H, W = q.shape
    fh, fw = int(np.rint(H / fs)), int(np.rint(W / fs))
    out = np.zeros((fh, fw), np.float32)
    for yy in range(fh):
        for xx in range(fw):
            cell = q[yy * fs:yy * fs + fs, xx * fs:xx * fs + fs]
            num, n = 4 * int(cell.sum()), cell.size
            qq, r = divmod(num, n)
            if 2 * r > n or (2 * r == n and qq % 2):
                qq += 1
            out[yy, xx] = qq / 16.0
    return out


@pytest.mark.parametrize("name", list(SPECS))
@pytest.mark.parametrize("fs", [2, 4])
def test_luma_restatement(name, fs):
    p, _ = workloads.pan_pair(45, 33, seed=3)
    a = CONV[name](p)
    est = oracle.estimate_fmt(a, a, SPECS[name], settings=oracle.Settings(flowScale=fs, pyramidMinSide=16))
    assert np.array_equal(est["luma"][0][0], luma_numpy(a, SPECS[name], fs))
    for l, (la, _) in enumerate(est["luma"]):   # the grids every exactness argument rests on
        g = 16.0 if l == 0 else 1024.0
        assert np.array_equal(la * g, np.rint(la * g)), f"level {l} off its grid"


@pytest.mark.parametrize("name", list(SPECS))
def test_still_pair_comes_back_unchanged(name):
    """a == c: zero vectors everywhere and every output sample (chroma included) equal to the input's"""
    p, _ = workloads.pan_pair(64, 48, seed=5)
    a = CONV[name](p)
    spec = SPECS[name]
    est = oracle.estimate_fmt(a, a, spec)
    assert not est["pf"].any() and est["sad"] == 0.0
    for t in (0.5, 0.25, 0.75):
        out, why = oracle.synth_fmt(a, a, est, t, spec)
        assert why is None
        if isinstance(a, tuple):
            assert all(np.array_equal(o, i) for o, i in zip(out, a)), t
        else:
            assert np.array_equal(out.view(np.uint8), a.view(np.uint8)), t


@pytest.mark.parametrize("name", ["rgb10", "f16_linear", "nv12", "p010"])
def test_integer_pan_is_found(name):
    """curr = prev shifted by (+4, -2) px: the interior blocks' half-vectors are (2, -1) at level 0 (flowScale 2 ->
    flow pixels: (+2, -1) shift, half-vector (1, -0.5))"""
    rng = np.random.default_rng(7)
    tex = workloads.value_noise(200, 260, rng, octaves=4, base=24.0)
    big = workloads._to_rgba(tex)
    prev, curr = big[8:168, 8:248], big[10:170, 4:244]   # content moved by (+4, -2)
    spec = SPECS[name]
    est = oracle.estimate_fmt(CONV[name](np.ascontiguousarray(prev)), CONV[name](np.ascontiguousarray(curr)), spec)
    v = est["sub"][1][2:-2, 2:-2]
    frac = np.mean(np.all(v == np.array([1.0, -0.5], np.float32), axis=-1))
    assert frac > 0.9, frac
