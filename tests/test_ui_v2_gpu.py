"""Static-UI protection in its CrosshairV2 mode (Settings::uiProtection = CrosshairV2) on the GPU, through the C ABI.

The reference has this mode only as Vulkan shaders, so parity is against the oracle's restatement of them
(oracle/ui_v2.py: the per-pixel state machine, the mask with its 1 px grow and pair gate, the paste-back;
oracle/fg_oracle.c fgo_synth_ui: the warp-tap rejection inside the synthesis): every state word, every mask byte and
every output byte equal. Beside that, the reference's own gates for the mode (gpu/formattest.cpp:611-690,
1100-1111): on a grain background panning (14, 6) px per frame with a small static plus, the unprotected run copies the
plus along the pan (the "doubled crosshair"), CrosshairV2 pastes the plus pixel-exact and leaves few artifact pixels
around it; and the lifecycle of gpu/framegen.h:576-691 (Off is byte-identical, explicit and implicit observe,
recordTrack, eviction).
"""
import numpy as np
import pytest
import torch

import framegen as fg
import oracle
import ui_v2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def built():
    import build
    build.build()


def grain_scene(W, H, n, pan=(14, 6), seed=0, plus=True, plus_size=12):
    """n RGBA8 frames: a background of value noise with per-pixel grain, panned by `pan` px per frame (integer shifts
    of one big image, so consecutive frames are exact translations), and a static opaque cyan plus of plus_size px
    (arms 2 px thick, on even coordinates) at the frame centre. Returns (frames, ui) with ui the plus's pixels."""
    rng = np.random.default_rng(seed)
    dx, dy = pan
    BW, BH = W + abs(dx) * n + 8, H + abs(dy) * n + 8
    gy, gx = np.mgrid[0:BH, 0:BW].astype(np.float64)
    base = np.zeros((BH, BW, 3))
    for period, amp in ((24.0, 120.0), (5.0, 40.0)):
        grid = rng.random((int(BH / period) + 3, int(BW / period) + 3, 3))
        fy, fx = gy / period, gx / period
        y0, x0 = np.floor(fy).astype(int), np.floor(fx).astype(int)
        ty, tx = (fy - y0)[..., None], (fx - x0)[..., None]
        v = (grid[y0, x0] * (1 - tx) + grid[y0, x0 + 1] * tx) * (1 - ty) + \
            (grid[y0 + 1, x0] * (1 - tx) + grid[y0 + 1, x0 + 1] * tx) * ty
        base += amp * v
    base += 60.0 + (rng.random((BH, BW, 3)) - 0.5) * 70.0
    base[..., 2] *= 0.8
    bg = np.clip(base, 0, 255).astype(np.uint8)
    cx, cy = (W // 2) & ~1, (H // 2) & ~1
    ui = np.zeros((H, W), bool)
    if plus:
        h = plus_size // 2
        for y in range(cy - h, cy + h):
            for x in range(cx - h, cx + h):
                ui[y, x] = (cx <= x < cx + 2) or (cy <= y < cy + 2)
    frames = []
    ox, oy = (abs(dx) * n if dx < 0 else 0) + 4, (abs(dy) * n if dy < 0 else 0) + 4
    for k in range(n):
        x0, y0 = ox + k * dx, oy + k * dy
        f = np.empty((H, W, 4), np.uint8)
        f[..., :3] = bg[y0:y0 + H, x0:x0 + W]
        f[..., 3] = 255
        f[ui, 0], f[ui, 1], f[ui, 2] = 0, 255, 255
        frames.append(f)
    return frames, ui


def v2_settings(**kw):
    d = dict(uiProtection=3, uiBoxWidth=16, uiBoxHeight=16)
    d.update(kw)
    return fg.Settings(**d)


def oracle_words(st):
    """the oracle's unpacked state as the kernels' three state words"""
    pack = lambda c: (c[..., 0] | (c[..., 1] << 8) | (c[..., 2] << 16)).astype(np.uint32)
    w0 = pack(st.prev) | (st.cnt.astype(np.uint32) << 24)
    w1 = pack(st.stored) | (st.flags.astype(np.uint32) << 24)
    w2 = (st.leave | (st.match << 8)).astype(np.uint32)
    return w0, w1, w2


def oracle_settings(s):
    return oracle.Settings(**{k: getattr(s, k) for k in oracle.Settings.__dataclass_fields__})


def run_sequence(frames, s, ts=(0.5, 0.25), observe=True, blur=None):
    """observe every frame (or rely on the implicit observe), then estimate the last pair and synthesize at ts (and
    a blurred output over `blur`); returns the outputs (host), the Interpolator and the device frames"""
    H, W = frames[0].shape[:2]
    I = fg.Interpolator()
    assert I.init(W, H, fg.VK_R8G8B8A8_UNORM, settings=s), I.init_error()
    dev = [torch.from_numpy(f).cuda() for f in frames]
    if observe:
        for d in dev:
            assert I.record_observe(d)
    I.begin_frame()
    assert I.record_estimate(dev[-2], dev[-1])
    outs = []
    for t in ts:
        o = torch.empty_like(dev[0])
        assert I.record_synth(dev[-2], dev[-1], o, t), I.last_error()
        outs.append(o)
    if blur is not None:
        o = torch.empty_like(dev[0])
        assert I.record_synth_blur(dev[-2], dev[-1], o, *blur), I.last_error()
        outs.append(o)
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in outs], I, dev


@pytest.mark.parametrize("case", ["defaults", "fast_reentry_off", "no_contrast_gate", "offset_box", "estimate_fill",
                                  "estimate_fill_fs1"])
def test_state_and_outputs_match_the_oracle(case):
    W, H = 160, 96
    kw = {"defaults": {}, "fast_reentry_off": dict(uiReentryFrames=0, uiLeaveFrames=1),
          "no_contrast_gate": dict(uiContrastThreshold=0.0, uiStillFrames=3),
          "offset_box": dict(uiBoxWidth=24, uiBoxHeight=20, uiBoxOffsetX=-9, uiBoxOffsetY=5),
          "estimate_fill": dict(uiEstimateFill=True, uiBoxWidth=20, uiBoxHeight=18),
          "estimate_fill_fs1": dict(uiEstimateFill=True, flowScale=1)}[case]
    s = v2_settings(**kw)
    frames, _ = grain_scene(W, H, 12)
    # a disturbance: frame 6 flashes a square over the plus (the leave counter runs, the plus may leave and re-enter)
    frames[6] = frames[6].copy()
    frames[6][H // 2 - 4:H // 2 + 4, W // 2 - 4:W // 2 + 4, :3] = 255
    I = fg.Interpolator()
    assert I.init(W, H, fg.VK_R8G8B8A8_UNORM, settings=s), I.init_error()
    st = ui_v2.State(s, W, H)
    assert fg.work_rect(s, W, H) == st.work
    dev = [torch.from_numpy(f).cuda() for f in frames]
    masks = {}
    for k, d in enumerate(dev):
        assert I.record_observe(d)
        st.update(frames[k])
        masks[k] = st.mask()
        got = fg.read_ui(I, d, s, W, H)
        for name, want in zip(("w0", "w1", "w2"), oracle_words(st)):
            assert np.array_equal(got[name], want), f"frame {k}: state word {name} differs"
        assert np.array_equal(got["mask"], masks[k]), f"frame {k}: mask differs"
        wx, wy, ww, wh = st.work
        assert tuple(int(v) for v in got["header"][1:]) == (wx | (wy << 16), ww | (wh << 16), (ww + 3) // 4)
    assert (masks[11] == 255).sum() > 0, "the plus was never detected"
    # the last pair: (the estimate fill,) rejection + paste, against the oracle
    I.begin_frame()
    assert I.record_estimate(dev[10], dev[11])
    rect = st.work
    fill = ((masks[10], rect), (masks[11], rect)) if s.uiEstimateFill else None
    est = oracle.estimate(frames[10], frames[11], settings=oracle_settings(s), trace=True, ui_fill=fill)
    from gpu_util import assert_estimate_equal
    assert_estimate_equal(fg.read_trace(I), est)
    for t in (0.5, 0.25, float(np.float32(2 / 3))):
        o = torch.empty_like(dev[0])
        assert I.record_synth(dev[10], dev[11], o, t)
        torch.cuda.synchronize()
        ref, _ = oracle.synth(frames[10], frames[11], est, t, settings=oracle_settings(s),
                              ui=((masks[10], rect), (masks[11], rect)))
        ui_v2.patch(ref, frames[11], masks[11], rect)
        got = o.cpu().numpy()
        assert np.array_equal(got, ref), f"t={t}: {np.count_nonzero(got != ref)} bytes differ"
    I.close()


def test_off_and_never_detected_are_byte_identical():
    """gpu/framegen.h:218: Off = byte-identical to a library without the protection; a CrosshairV2 run that never
    masks anything (uiStillFrames above the sequence length, re-entry off) is byte-identical to Off as well, blurred
    output included"""
    frames, _ = grain_scene(160, 96, 10)
    never, I1, _ = run_sequence(frames, v2_settings(uiStillFrames=200, uiReentryFrames=0, blurSamples=3),
                                blur=(0.25, 0.75))
    off3, I2, _ = run_sequence(frames, fg.Settings(blurSamples=3), blur=(0.25, 0.75))
    for a, b in zip(off3, never):
        assert np.array_equal(a, b)
    for I in (I1, I2):
        I.close()


def artifacts(ui, out, ref, cx, cy, r=40, tol=24):
    """the reference's count of doubled-crosshair pixels: not-UI pixels within r px of the plus that differ by more
    than tol levels from the run on the scene without the plus"""
    H, W = ui.shape
    d = np.abs(out[..., :3].astype(int) - ref[..., :3].astype(int)).max(axis=2)
    ys, xs = np.mgrid[0:H, 0:W]
    near = (np.abs(xs - cx) <= r) & (np.abs(ys - cy) <= r) & ~ui
    return int(np.count_nonzero(near & (d > tol)))


def test_doubled_crosshair_gates():
    """gpu/formattest.cpp:611-690, 1100-1111: a grain background panning (14, 6) px per frame, a static 12x12 cyan
    plus. Off copies the plus along the pan (>= 15 artifact pixels: the check has teeth); CrosshairV2 with the estimate
    fill (as the reference measures it) pastes the plus pixel-exact at t = 0.5 and leaves at most 8 artifact pixels
    around it, at t = 0.5 and in the blurred output. The count without the fill is printed beside it."""
    W, H = 320, 192
    frames, ui = grain_scene(W, H, 12)
    clean, _ = grain_scene(W, H, 12, plus=False)
    cx, cy = (W // 2) & ~1, (H // 2) & ~1
    blur = (0.3, 0.7)
    ref, Ir, _ = run_sequence(clean, fg.Settings(blurSamples=3), ts=(0.5,), blur=blur)
    off, Io, _ = run_sequence(frames, fg.Settings(blurSamples=3), ts=(0.5,), blur=blur)
    v2, Iv, _ = run_sequence(frames, v2_settings(blurSamples=3, uiEstimateFill=True), ts=(0.5,), blur=blur)
    nofill, In, _ = run_sequence(frames, v2_settings(blurSamples=3), ts=(0.5,), blur=blur)
    a_off = [artifacts(ui, o, r, cx, cy) for o, r in zip(off, ref)]
    a_v2 = [artifacts(ui, o, r, cx, cy) for o, r in zip(v2, ref)]
    a_nf = [artifacts(ui, o, r, cx, cy) for o, r in zip(nofill, ref)]
    plus_bad = int(np.count_nonzero(np.abs(v2[0][..., :3].astype(int) - frames[-1][..., :3].astype(int)).max(axis=2)[ui] > 1))
    print(f"artifact px around the plus (t = 0.5 / blurred): Off {a_off}, CrosshairV2 + fill {a_v2}, without the fill "
          f"{a_nf}; plus pixels wrong {plus_bad}")
    assert min(a_off) >= 15
    assert plus_bad == 0
    assert max(a_v2) <= 8
    for I in (Ir, Io, Iv, In):
        I.close()


def test_lifecycle():
    W, H = 96, 64
    frames, _ = grain_scene(W, H, 8)
    s = v2_settings()
    I = fg.Interpolator()
    assert I.init(W, H, fg.VK_R8G8B8A8_UNORM, settings=s), I.init_error()
    dev = [torch.from_numpy(f).cuda() for f in frames]
    o = torch.empty_like(dev[0])
    # implicit observe: estimates alone keep the pair's entries (prev if not kept, curr if not the latest observed)
    for k in range(1, 5):
        I.begin_frame()
        assert I.record_estimate(dev[k - 1], dev[k])
        assert I.record_synth(dev[k - 1], dev[k], o, 0.5)
    assert fg.read_ui(I, dev[4], s, W, H)["header"][3] != 0   # frame 4 is kept
    # explicit observe: observing 3 more frames evicts the estimate's entries (uiHistory = 3): the synth refuses
    I.begin_frame()
    assert I.record_observe(dev[4]) and I.record_observe(dev[5])
    assert I.record_estimate(dev[4], dev[5]) and I.record_synth(dev[4], dev[5], o, 0.5)
    for k in (6, 7):
        assert I.record_observe(dev[k])
    assert I.record_observe(dev[0])
    assert not I.record_synth(dev[4], dev[5], o, 0.5)
    # recordTrack forgets the entry of the frame it tracks (its pixels are new): a pair with it is unprotected
    assert I.record_track(dev[7])
    assert fg.read_ui(I, dev[7], s, W, H)["header"][3] == 0
    I.begin_frame()
    assert I.record_estimate(dev[6], dev[7]) and I.record_synth(dev[6], dev[7], o, 0.5)
    # a change of the box restarts the protection and drops the estimate
    assert I.set_settings(v2_settings(uiBoxWidth=20))
    assert not I.record_synth(dev[6], dev[7], o, 0.5)
    # off: observe / track return true and record nothing
    assert I.set_settings(fg.Settings())
    assert I.record_observe(dev[0]) and I.record_track(dev[0])
    I.close()
