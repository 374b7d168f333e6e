"""CPU checks of the oracle's CrosshairV2 restatement for the formats other than 8-bit RGBA (oracle/ui_v2.py
levels_fmt, yuv_diff_max, patch_fmt; oracle/fg_oracle_fmt.c fgo_synth_fmt_ui), the checker the GPU tests in
test_ui_v2_fmt_gpu.py compare the kernels with. They pin the restatement to independent statements of the shaders'
formulas (gpu/shaders/format.glsl FG_STILL / fgStillYuv / fgYuvDiff, gpu/shaders/ui_patch_chroma.comp)."""
import numpy as np
import pytest

import oracle
import ui_v2
import workloads


def test_levels_of_8bit_content_round_trip():
    """8-bit content carried in Rgb10 codes or encoded RgbaF16 halves comes back as its own 8-bit levels"""
    p, _, _ = workloads.flow_pair(96, 64, seed=3)
    rgb = p[..., :3].astype(np.int32)
    for spec, conv in ((oracle.FormatSpec("rgb10"), workloads.to_rgb10),
                       (oracle.FormatSpec("rgb10", r_high=True), lambda f: workloads.to_rgb10(f, r_high=True)),
                       (oracle.FormatSpec("f16", linear=False), lambda f: workloads.to_f16(f, linear=False))):
        assert np.array_equal(ui_v2.levels_fmt(conv(p), spec), rgb), spec


def test_yuv_levels():
    """Nv12: the bytes of the pixel and of its chroma texel; P010: floor(s / 256 + 0.5) of each 16-bit sample"""
    rng = np.random.default_rng(1)
    H, W = 10, 14
    y8 = rng.integers(0, 256, (H, W), dtype=np.uint8)
    c8 = rng.integers(0, 256, (H // 2, W // 2, 2), dtype=np.uint8)
    lv = ui_v2.levels_fmt((y8, c8), oracle.FormatSpec("nv12"))
    ys, xs = np.mgrid[0:H, 0:W]
    assert np.array_equal(lv[..., 0], y8) and np.array_equal(lv[..., 1:], c8[ys // 2, xs // 2])
    y16 = rng.integers(0, 65536, (H, W), dtype=np.uint16)
    c16 = rng.integers(0, 65536, (H // 2, W // 2, 2), dtype=np.uint16)
    lv = ui_v2.levels_fmt((y16, c16), oracle.FormatSpec("p010"))
    want_y = np.minimum((y16.astype(np.int64) + 128) >> 8, 255)
    want_c = np.minimum((c16.astype(np.int64) + 128) >> 8, 255)[ys // 2, xs // 2]
    assert np.array_equal(lv[..., 0], want_y) and np.array_equal(lv[..., 1:], want_c)


def test_f16_levels_clamp_non_finite_and_out_of_range():
    f = np.zeros((1, 4, 4), np.float16)
    f[0, :, 0] = [np.nan, np.inf, -np.inf, 2.0]
    f[0, :, 1] = [-1.0, 0.5, 1.0, 0.001]
    lv = ui_v2.levels_fmt(f, oracle.FormatSpec("f16", linear=False))
    assert lv[0, :, 0].tolist() == [0, 255, 0, 255]
    assert lv[0, :, 1].tolist() == [0, 128, 255, 0]


@pytest.mark.parametrize("matrix", ["bt601", "bt709", "bt2020"])
def test_yuv_contrast_difference_is_the_rgb_difference(matrix):
    """fgYuvDiff: the R'G'B' difference a (Y, Cb, Cr) level difference stands for, the largest channel: compared with
    a float64 statement of the same limited-range matrix"""
    spec = oracle.FormatSpec("nv12", matrix=matrix)
    f = oracle.fmt_struct(spec)
    rng = np.random.default_rng(2)
    for _ in range(200):
        d = rng.integers(-60, 61, 3)
        dy, db, dr = (float(v) for v in d)
        y = f.ys * dy
        want = max(abs(y + f.rcr * dr), abs(y + f.gcb * db + f.gcr * dr), abs(y + f.bcb * db))
        assert abs(ui_v2.yuv_diff_max(d, spec) - want) <= 1e-4 * max(1.0, want)


def test_yuv_patch_takes_the_strongest_pixel_of_each_chroma_texel():
    H, W = 8, 8
    rect = (1, 1, 5, 5)
    mask = np.zeros((5, 5), np.uint8)
    mask[0, 0] = 255   # pixel (1, 1): texel (0, 0)
    mask[2, 2] = 64    # pixel (3, 3): texel (1, 1), changed only: not pasted
    mask[3, 3] = 255   # pixel (4, 4): texel (2, 2)
    out = (np.zeros((H, W), np.uint8), np.zeros((H // 2, W // 2, 2), np.uint8))
    cur = (np.full((H, W), 9, np.uint8), np.full((H // 2, W // 2, 2), 7, np.uint8))
    ui_v2.patch_fmt(out, cur, mask, rect, oracle.FormatSpec("nv12"))
    assert out[0][1, 1] == 9 and out[0][4, 4] == 9 and out[0][3, 3] == 0 and int(out[0].sum()) == 18
    texels = {(ty, tx) for ty in range(4) for tx in range(4) if out[1][ty, tx, 0] == 7}
    assert texels == {(0, 0), (2, 2)}


def test_rejection_only_changes_pixels_whose_taps_touch_the_mask():
    """fgo_synth_fmt_ui with a mask of one frame only: the output differs from the plain synthesis only where a tap of
    that frame could read a masked pixel"""
    p, c, _ = workloads.flow_pair(160, 96, seed=5)
    spec = oracle.FormatSpec("rgb10")
    a, b = workloads.to_rgb10(p), workloads.to_rgb10(c)
    s = oracle.Settings(globalFallback=1.0)
    est = oracle.estimate_fmt(a, b, spec, settings=s, trace=False)
    rect = (70, 40, 12, 10)
    mask = np.full((10, 12), 255, np.uint8)
    plain, _ = oracle.synth_fmt(a, b, est, 0.5, spec, settings=s)
    rej, _ = oracle.synth_fmt(a, b, est, 0.5, spec, settings=s, ui=((mask, rect), None))
    ys, xs = np.nonzero(plain != rej)
    assert len(ys) > 0
    # the half-vectors at t = 1/2 are below 16 px here: a pixel far from the rectangle cannot have touched it
    assert (np.abs(xs - 76) < 40).all() and (np.abs(ys - 45) < 40).all()
