"""Static-UI protection, CrosshairV2, in the Rgb10, RgbaF16 (encoded and linear), Nv12 and P010 formats on the GPU,
through the C ABI. The state machine sees the shaders' 8-bit-equivalent levels of each format (gpu/shaders/format.glsl
FG_STILL / fgStillYuv, as gpu/shaders/ui_v2_update.comp's pixAt reads them; YUV's contrast gate on the R'G'B'
difference); the estimate fill uses the format's luma; the synthesis rejects warp taps on the UI of their own frame
(YUV: the chroma-texel footprint, and the block-centre chroma on its own positions) and the real curr pixels are
pasted back (colour channels, alpha kept; YUV chroma texels by their strongest pixel). Parity is against the oracle's
restatement (oracle/ui_v2.py levels_fmt / yuv_diff_max / patch_fmt, oracle/fg_oracle_fmt.c ui_fill_fmt and
fgo_synth_fmt_ui): every state word, mask byte and output sample equal, over the 12-frame sequence of
test_ui_v2_gpu.py converted to each format.
"""
import numpy as np
import pytest
import torch

import framegen as fg
import oracle
import ui_v2
import workloads
from gpu_util import assert_estimate_equal
from test_ui_v2_gpu import grain_scene, oracle_settings, oracle_words, v2_settings

pytestmark = pytest.mark.gpu

# (name, view format, oracle spec, converter of an 8-bit RGBA frame, InitInfo extras)
SPECS = {
    "rgb10": (fg.VK_A2B10G10R10_UNORM, oracle.FormatSpec("rgb10"), lambda f: workloads.to_rgb10(f), {}),
    "rgb10_argb": (fg.VK_A2R10G10B10_UNORM, oracle.FormatSpec("rgb10", r_high=True),
                   lambda f: workloads.to_rgb10(f, r_high=True), {}),
    "f16_linear": (fg.VK_R16G16B16A16_SFLOAT, oracle.FormatSpec("f16", linear=True, white=80.0),
                   lambda f: workloads.to_f16(f, linear=True), {"transfer": 1, "linear_white_nits": 80.0}),
    "f16_encoded": (fg.VK_R16G16B16A16_SFLOAT, oracle.FormatSpec("f16", linear=False),
                    lambda f: workloads.to_f16(f, linear=False), {"transfer": 0}),
    "nv12": (fg.VK_R8_UNORM, oracle.FormatSpec("nv12", matrix="bt709"), lambda f: workloads.to_yuv(f, 8, "bt709"),
             {"yuv_matrix": 1, "yuv_full_range": False}),
    "p010": (fg.VK_R16_UNORM, oracle.FormatSpec("p010", matrix="bt2020"), lambda f: workloads.to_yuv(f, 10, "bt2020"),
             {"yuv_matrix": 2, "yuv_full_range": False}),
}
FMT_NAME = {"rgb10": "Rgb10", "f16": "RgbaF16", "nv12": "Nv12", "p010": "P010"}


@pytest.fixture(scope="module", autouse=True)
def built():
    import build
    build.build()


def dev(frame):
    if isinstance(frame, tuple):
        return tuple(dev(p) for p in frame)
    a = frame.view(np.int32) if frame.dtype == np.uint32 else frame.view(np.int16) if frame.dtype == np.uint16 else frame
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t, like):
    if isinstance(t, tuple):
        return tuple(host(x, l) for x, l in zip(t, like))
    return t.cpu().numpy().view(like.dtype)


def empty_like(d):
    return tuple(torch.empty_like(x) for x in d) if isinstance(d, tuple) else torch.empty_like(d)


def same(a, b):
    if isinstance(a, tuple):
        return all(same(x, y) for x, y in zip(a, b))
    return np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("case", ["defaults", "estimate_fill", "offset_box_fs1"])
@pytest.mark.parametrize("name", list(SPECS))
def test_state_and_outputs_match_the_oracle(name, case):
    vk, spec, conv, extra = SPECS[name]
    W, H = 320, 192   # large enough that the pair does not fall back as a whole: the rejection shows in the output
    kw = {"defaults": {}, "estimate_fill": dict(uiEstimateFill=True, uiBoxWidth=20, uiBoxHeight=18),
          "offset_box_fs1": dict(uiBoxWidth=24, uiBoxHeight=20, uiBoxOffsetX=-9, uiBoxOffsetY=5, flowScale=1,
                                 uiEstimateFill=True)}[case]
    s = v2_settings(**kw)
    assert fg.settings_error(s, FMT_NAME[spec.format]) is None
    rgba, _ = grain_scene(W, H, 12)
    rgba[6] = rgba[6].copy()   # a flash over the plus: the leave counter runs
    rgba[6][H // 2 - 4:H // 2 + 4, W // 2 - 4:W // 2 + 4, :3] = 255
    frames = [conv(f) for f in rgba]
    I = fg.Interpolator()
    assert I.init(W, H, vk, settings=s, **extra), I.init_error()
    st = ui_v2.State(s, W, H)
    d = [dev(f) for f in frames]
    masks = {}
    for k in range(len(frames)):
        assert I.record_observe(d[k])
        st.update(frames[k], spec=spec)
        masks[k] = st.mask()
        got = fg.read_ui(I, d[k], s, W, H)
        for wname, want in zip(("w0", "w1", "w2"), oracle_words(st)):
            assert np.array_equal(got[wname], want), f"frame {k}: state word {wname} differs"
        assert np.array_equal(got["mask"], masks[k]), f"frame {k}: mask differs"
    assert (masks[11] == 255).sum() > 0, "the plus was never detected"
    I.begin_frame()
    assert I.record_estimate(d[10], d[11])
    rect = st.work
    os_ = oracle_settings(s)
    fill = ((masks[10], rect), (masks[11], rect)) if s.uiEstimateFill else None
    est = oracle.estimate_fmt(frames[10], frames[11], spec, settings=os_, trace=True, ui_fill=fill)
    assert_estimate_equal(fg.read_trace(I), est)
    ui = ((masks[10], rect), (masks[11], rect))
    for t in (0.5, 0.25, float(np.float32(2 / 3))):
        o = empty_like(d[0])
        assert I.record_synth(d[10], d[11], o, t), I.last_error()
        torch.cuda.synchronize()
        ref, _ = oracle.synth_fmt(frames[10], frames[11], est, t, spec, settings=os_, ui=ui)
        ui_v2.patch_fmt(ref, frames[11], masks[11], rect, spec)
        assert same(host(o, ref), ref), f"t={t}: outputs differ"
    I.close()


@pytest.mark.parametrize("name", ["rgb10", "f16_linear", "nv12"])
def test_blur_with_the_protection(name):
    """recordSynthBlur with CrosshairV2 in the format: every synthesized sample with the tap rejection, the average,
    then the paste-back"""
    vk, spec, conv, extra = SPECS[name]
    W, H = 320, 192
    s = v2_settings(blurSamples=3)
    rgba, _ = grain_scene(W, H, 10)
    frames = [conv(f) for f in rgba]
    I = fg.Interpolator()
    assert I.init(W, H, vk, settings=s, **extra), I.init_error()
    st = ui_v2.State(s, W, H)
    d = [dev(f) for f in frames]
    keep = {}
    for k in range(len(frames)):
        assert I.record_observe(d[k])
        st.update(frames[k], spec=spec)
        keep[k] = st.mask()
    rect = st.work
    I.begin_frame()
    assert I.record_estimate(d[8], d[9])
    os_ = oracle_settings(s)
    est = oracle.estimate_fmt(frames[8], frames[9], spec, settings=os_, trace=False)
    o = empty_like(d[0])
    assert I.record_synth_blur(d[8], d[9], o, 0.25, 0.75), I.last_error()
    torch.cuda.synchronize()
    ref = oracle.synth_blur_fmt(frames[8], frames[9], est, 0.25, 0.75, 3, s.blurWeights == 1, spec, settings=os_,
                                ui=((keep[8], rect), (keep[9], rect)))
    ui_v2.patch_fmt(ref, frames[9], keep[9], rect, spec)
    assert same(host(o, ref), ref)
    I.close()


@pytest.mark.parametrize("name", ["rgb10", "f16_encoded"])
def test_off_and_never_detected_are_byte_identical(name):
    vk, spec, conv, extra = SPECS[name]
    W, H = 160, 96
    rgba, _ = grain_scene(W, H, 8)
    frames = [conv(f) for f in rgba]
    outs = []
    for s in (fg.Settings(), v2_settings(uiStillFrames=200, uiReentryFrames=0)):
        I = fg.Interpolator()
        assert I.init(W, H, vk, settings=s, **extra), I.init_error()
        d = [dev(f) for f in frames]
        for x in d:
            assert I.record_observe(x)
        I.begin_frame()
        assert I.record_estimate(d[-2], d[-1])
        o = torch.empty_like(d[0])
        assert I.record_synth(d[-2], d[-1], o, 0.25)
        torch.cuda.synchronize()
        outs.append(o.cpu().numpy())
        I.close()
    assert np.array_equal(outs[0], outs[1])


def test_every_format_is_accepted():
    for fmt in ("Rgba8", "Rgb10", "RgbaF16", "Nv12", "P010"):
        assert fg.settings_error(v2_settings(uiEstimateFill=True), fmt) is None
