"""Parity of the CUDA path with the oracle for the frame formats other than 8-bit RGBA (framegen::Format Rgb10,
RgbaF16, Nv12, P010), through the C ABI.

proto/interp.py is 8-bit BGR only; for these formats the oracle restates the reference's shader math
(gpu/shaders/format.glsl, luma.comp, motion_v1.glsl, resolve.comp; oracle/fg_oracle_fmt.c). Bar: every intermediate
of the estimate, the scene-cut mean and every whole-frame decision bit-exact; output samples within TOL = 1 code
(10-bit codes for Rgb10 / P010, 8-bit codes for Nv12, 1 PQ level for linear RgbaF16, 1 level for encoded RgbaF16);
the kernels are designed to be exact, which the tests also assert.
"""
import numpy as np
import pytest
import torch

import framegen as fg
import oracle
import workloads
from gpu_util import assert_estimate_equal, decision

pytestmark = pytest.mark.gpu
TOL = 1
T23 = float(np.float32(2 / 3))

# (name, view format, oracle spec, converter of an 8-bit RGBA frame, InitInfo extras)
SPECS = [
    ("rgb10_abgr", fg.VK_A2B10G10R10_UNORM, oracle.FormatSpec("rgb10"), lambda f: workloads.to_rgb10(f), {}),
    ("rgb10_argb", fg.VK_A2R10G10B10_UNORM, oracle.FormatSpec("rgb10", r_high=True),
     lambda f: workloads.to_rgb10(f, r_high=True), {}),
    ("f16_linear", fg.VK_R16G16B16A16_SFLOAT, oracle.FormatSpec("f16", linear=True, white=80.0),
     lambda f: workloads.to_f16(f, linear=True), {"transfer": 1, "linear_white_nits": 80.0}),
    ("f16_linear_203", fg.VK_R16G16B16A16_SFLOAT, oracle.FormatSpec("f16", linear=True, white=203.0),
     lambda f: workloads.to_f16(f, linear=True), {"transfer": 1, "linear_white_nits": 203.0}),
    ("f16_encoded", fg.VK_R16G16B16A16_SFLOAT, oracle.FormatSpec("f16", linear=False),
     lambda f: workloads.to_f16(f, linear=False), {"transfer": 0}),
    ("nv12_709_limited", fg.VK_R8_UNORM, oracle.FormatSpec("nv12", matrix="bt709"),
     lambda f: workloads.to_yuv(f, 8, "bt709"), {"yuv_matrix": 1, "yuv_full_range": False}),
    ("nv12_601_full", fg.VK_R8_UNORM, oracle.FormatSpec("nv12", matrix="bt601", full_range=True),
     lambda f: workloads.to_yuv(f, 8, "bt601", True), {"yuv_matrix": 0, "yuv_full_range": True}),
    ("p010_2020_limited", fg.VK_R16_UNORM, oracle.FormatSpec("p010", matrix="bt2020"),
     lambda f: workloads.to_yuv(f, 10, "bt2020"), {"yuv_matrix": 2, "yuv_full_range": False}),
    ("p010_709_full", fg.VK_R16_UNORM, oracle.FormatSpec("p010", matrix="bt709", full_range=True),
     lambda f: workloads.to_yuv(f, 10, "bt709", True), {"yuv_matrix": 1, "yuv_full_range": True}),
]
SPEC = {s[0]: s for s in SPECS}


@pytest.fixture(scope="module", autouse=True)
def built():
    import build
    build.build()


def _plane_dev(a, pad):
    """numpy plane -> CUDA tensor (uint32 / uint16 viewed as int32 / int16); pad adds unused elements per row."""
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    elif a.dtype == np.uint16:
        a = a.view(np.int16)
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    if not pad:
        return t
    buf = torch.zeros((a.shape[0], a.shape[1] + pad) + a.shape[2:], dtype=t.dtype, device="cuda")
    buf[:, :a.shape[1]] = t
    return buf[:, :a.shape[1]]


def to_dev(frame, pad=0):
    if isinstance(frame, tuple):
        return (_plane_dev(frame[0], pad), _plane_dev(frame[1], pad))
    return _plane_dev(frame, pad)


def new_out(dev, pad=0):
    if isinstance(dev, tuple):
        return tuple(new_out(d, pad) for d in dev)
    buf = torch.zeros((dev.shape[0], dev.shape[1] + pad) + tuple(dev.shape[2:]), dtype=dev.dtype, device="cuda")
    return buf[:, :dev.shape[1]]


def to_host(dev, like):
    if isinstance(dev, tuple):
        return tuple(to_host(d, l) for d, l in zip(dev, like))
    return dev.cpu().numpy().view(like.dtype)


def sample_diff(name, got, ref, spec):
    """max difference in the test's unit (codes / PQ levels / levels), and the number of samples that differ"""
    if isinstance(got, tuple):
        res = [sample_diff(name, g, r, spec) for g, r in zip(got, ref)]
        return max(r[0] for r in res), sum(r[1] for r in res)
    if spec.format == "rgb10":
        sh = [0, 10, 20, 30]
        d = max(int(np.abs(((got >> s) & m).astype(np.int64) - ((ref >> s) & m).astype(np.int64)).max())
                for s, m in zip(sh, [1023, 1023, 1023, 3]))
        return d, int(np.count_nonzero(got != ref))
    if spec.format == "f16":
        g, r = got.astype(np.float32), ref.astype(np.float32)
        if spec.linear:   # in PQ levels, the unit of the mismatch metric
            pq = np.vectorize(lambda v: oracle.pq255(v, spec.white))
            nd = got != ref
            d = float(np.abs(pq(g[nd]) - pq(r[nd])).max()) if nd.any() else 0.0
        else:
            d = float(np.abs(g - r).max() * 255.0)
        return d, int(np.count_nonzero(got.view(np.uint16) != ref.view(np.uint16)))
    shift = 6 if spec.format == "p010" else 0
    d = int(np.abs((got >> shift).astype(np.int64) - (ref >> shift).astype(np.int64)).max())
    return d, int(np.count_nonzero(got != ref))


def check(name, prev8, curr8, ts, settings=None, pad=0):
    conv = SPEC[name][3]
    check_frames(name, conv(prev8), conv(curr8), ts, settings, pad)


def check_frames(name, a, c, ts, settings=None, pad=0):
    _, vk, spec, _, extra = SPEC[name]
    W, H = oracle.frame_size(a, spec)
    s = settings or oracle.Settings()
    fs = fg.Settings(**{k: getattr(s, k) for k in oracle.Settings.__dataclass_fields__})
    I = fg.Interpolator()
    assert I.init(W, H, vk, settings=fs, **extra), I.init_error()
    assert I.format() == {"rgb10": "Rgb10", "f16": "RgbaF16", "nv12": "Nv12", "p010": "P010"}[spec.format]
    da, dc = to_dev(a, pad), to_dev(c, pad)
    cnt = torch.zeros(2, dtype=torch.int32, device="cuda")
    I.begin_frame()
    assert I.record_estimate(da, dc), I.last_error()
    tr = fg.read_trace(I)
    est = oracle.estimate_fmt(a, c, spec, settings=s)
    if not s.subpixel:
        est.pop("sub")
    assert_estimate_equal(tr, est)
    for t in ts:
        o = new_out(da, pad)
        assert I.record_synth(da, dc, o, t), I.last_error()
        assert I.record_debug_counters(cnt)
        torch.cuda.synchronize()
        got = to_host(o, a)
        ref = oracle.synth_fmt(a, c, est, t, spec, settings=s, trace=True)
        assert decision(tr["cut"], int(cnt[0]), W, H, s.globalFallback) == ref["reason"], f"decision at t={t}"
        if not tr["cut"]:
            assert int(cnt[0]) == ref["untrusted"], f"untrusted count at t={t}"
        mx, nd = sample_diff(name, got, ref["out"], spec)
        assert mx <= TOL, f"{name} t={t}: max diff {mx}, {nd} samples differ"
        assert nd == 0, f"{name} t={t}: {nd} samples differ (max {mx})"
    I.close()


@pytest.mark.parametrize("name", [s[0] for s in SPECS])
def test_format_flow(name):
    p, c, _ = workloads.flow_pair(320, 180, seed=11)
    check(name, p, c, [0.5, 0.25, T23])


@pytest.mark.parametrize("name", ["rgb10_abgr", "f16_linear", "nv12_709_limited", "p010_2020_limited"])
def test_format_odd_size_padded(name):
    """odd width and height (a chroma plane of ceil(W / 2) x ceil(H / 2)), rows with unused padding"""
    p, c = workloads.pan_pair(131, 97, seed=4)
    check(name, p, c, [0.5, 0.75], pad=3)


@pytest.mark.parametrize("name", ["rgb10_argb", "f16_encoded", "nv12_601_full", "p010_709_full"])
def test_format_fallbacks(name):
    """a scene cut and a pair with fresh content: the whole-frame decisions in each format"""
    p, c = workloads.contrast_pair(160, 96, seed=2, kind="cut")
    check(name, p, c, [0.25, 0.5])
    p, c, _ = workloads.flow_pair(320, 180, seed=8, kind="fresh")
    check(name, p, c, [0.5])


@pytest.mark.parametrize("fs", [1, 4])
@pytest.mark.parametrize("name", ["rgb10_abgr", "p010_2020_limited"])
def test_format_flow_scales(name, fs):
    p, c, _ = workloads.flow_pair(256, 192, seed=13)
    check(name, p, c, [0.5, 0.25], settings=oracle.Settings(flowScale=fs))


@pytest.mark.parametrize("name", ["rgb10_abgr", "f16_linear", "nv12_709_limited", "p010_709_full"])
def test_format_1080p(name):
    """1080p: four pyramid levels, the 2^-10 rounding of the coarse levels in play"""
    p, c, _ = workloads.flow_pair(1920, 1080, seed=21)
    check(name, p, c, [0.5, 0.25])


def test_hdr_4k_f16_linear():
    """The 4K HDR workload: 3840x2160 RgbaF16 linear scRGB (80 nits), t = 1/3 and 2/3; every channel log-uniform in 1e-3..10 with
    4-octave correlation, a global pan of up to +-16 px and 3 rigid sprites of 128-384 px moving up to +-32 px
    (workloads_gpu.hdr_pair, generated on the device)"""
    import workloads_gpu
    gen = torch.Generator(device="cuda")
    gen.manual_seed(2 * 10 ** 6)
    a, c = (x.cpu().numpy() for x in workloads_gpu.hdr_pair(3840, 2160, gen))
    check_frames("f16_linear", a, c, [float(np.float32(1 / 3)), T23])


@pytest.mark.parametrize("frac", [0.3, 1.0])
def test_p010_off_grid_low_bits(frac):
    """P010 samples whose low 6 bits are not zero (off the 10-bit code grid) in a share of the luma and chroma samples:
    the synthesis filters a tap group of on-grid samples with integer arithmetic and any other group with the float
    taps, and both must give the oracle's values"""
    p, c, _ = workloads.flow_pair(200, 120, seed=17)
    rng = np.random.default_rng(5)
    frames = []
    for f in (p, c):
        y, uv = workloads.to_yuv(f, 10, "bt709", True)
        for q in (y, uv):
            hit = rng.random(q.shape) < frac
            q[hit] |= rng.integers(1, 64, size=int(hit.sum())).astype(q.dtype)
        frames.append((y, uv))
    check_frames("p010_709_full", frames[0], frames[1], [0.5, 0.25])


def test_format_refusals():
    """YUV frames need their CbCr plane; a bad YUV matrix is refused at init"""
    p, c, _ = workloads.flow_pair(64, 48, seed=1)
    y, uv = workloads.to_yuv(p, 8)
    I = fg.Interpolator()
    assert not I.init(64, 48, fg.VK_R8_UNORM, yuv_matrix=7)
    assert "yuvMatrix" in I.init_error()
    assert I.init(64, 48, fg.VK_R8_UNORM)
    dy = torch.from_numpy(y).cuda()
    I.begin_frame()
    assert not I.record_estimate(dy, dy)   # no chroma plane
    d = (dy, torch.from_numpy(uv).cuda())
    assert I.record_estimate(d, d)
    assert not I.resize(64, 48, fg.VK_R8G8B8A8_UNORM)   # another Format
    I.close()
