"""The C ABI without a GPU: the library loads, exports every symbol include/framegen_c.h declares, and its host-only
logic (defaults, validate, settingsError, formatOf, init's refusals) behaves like gpu/framegen.h / framegen.cpp."""
import ctypes
import math
import os
import re

import pytest

import framegen as fg

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "framegen_c.h")


@pytest.fixture(scope="module", autouse=True)
def built():
    import build
    build.build()


def declared():
    src = open(HDR).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fg_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported_and_bound():
    names = declared()
    assert len(names) >= 30
    L = fg.lib()
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(fg.SIGNATURES), "the Python binding covers exactly the header"


def test_struct_sizes_match_header():
    assert ctypes.sizeof(fg.CSettings) == 4 * (17 + 15)   # the V1 fields, then the 15 static-UI protection fields
    assert ctypes.sizeof(fg.CFrame) == 32
    ii = fg.CInitInfo()
    fg.lib().fg_default_init_info(ctypes.byref(ii))
    assert ii.size == ctypes.sizeof(fg.CInitInfo)
    assert ii.settings.size == ctypes.sizeof(fg.CSettings)


def test_defaults_are_interp_constants():
    c = fg.CSettings()
    fg.lib().fg_default_settings(ctypes.byref(c))
    s = fg.Settings.from_c(c)
    assert s == fg.Settings.from_c(fg.Settings().to_c())
    # proto/interp.py:43-61 / gpu/framegen.h:167-409
    assert (s.trustLow, s.trustHigh, s.globalFallback, s.sceneCutSad) == (12.0, 40.0, pytest.approx(0.15), 30.0)
    assert (s.hudBonus, s.smoothBonus, s.searchPenalty) == (1.0, 0.5, 0.5)
    assert (s.searchRadius, s.searchRadiusTop, s.subpixel, s.flowScale, s.pyramidMinSide) == (2, 6, True, 2, 48)
    # gpu/framegen.h:220-305: the static-UI protection defaults
    assert (s.uiProtection, s.uiHistory, s.uiBoxWidth, s.uiBoxHeight, s.uiBoxOffsetX, s.uiBoxOffsetY) == (0, 3, 0, 0, 0, 0)
    assert (s.uiBoxHeightFrac, s.uiCrosshairArea) == (pytest.approx(0.025), pytest.approx(0.03))
    assert (s.uiStillFrames, s.uiStillThreshold, s.uiContrastThreshold, s.uiLeaveFrames, s.uiReentryFrames) == \
        (8, 3.5, 20.0, 4, 2)
    assert (s.uiInpaintReach, s.uiMaxStillFraction, s.uiEstimateFill) == (12, 0.75, False)
    ii = fg.CInitInfo()
    fg.lib().fg_default_init_info(ctypes.byref(ii))
    assert ii.view_format == fg.VK_B8G8R8A8_UNORM and ii.linear_white_nits == 80.0 and ii.device == -1


@pytest.mark.parametrize("field,value,ok", [
    ("trustLow", 0.0, True), ("trustLow", -0.5, False), ("trustLow", 39.5, False), ("trustHigh", 255.0, True),
    ("trustHigh", 256.0, False), ("globalFallback", 0.0, False), ("globalFallback", 1.0, True),
    ("sceneCutSad", 0.0, False), ("sceneCutSad", 255.0, True), ("hudBonus", math.nan, False),
    ("smoothBonus", math.inf, False), ("searchPenalty", 255.0, True), ("searchRadius", 0, False),
    ("searchRadius", 12, True), ("searchRadiusTop", 13, False), ("flowScale", 3, False), ("flowScale", 4, True),
    ("flowScale", 1, True), ("pyramidMinSide", 15, False), ("pyramidMinSide", 256, True), ("blurSamples", 17, False),
    ("uiProtection", 4, False), ("motionVersion", 4, False)])
def test_validate_ranges(field, value, ok):
    s = fg.Settings()
    setattr(s, field, value)
    assert fg.validate(s) is ok
    err = fg.settings_error(s)
    assert (err is None) is ok or (ok and err is not None)
    if not ok:
        assert err.startswith("invalid settings")


def test_settings_error_names_unbuilt_parts():
    s = fg.Settings(motionVersion=1)
    assert fg.validate(s) and "V1 only" in fg.settings_error(s)
    for mode in (1, 2):   # Crosshair, WholeScreen
        s = fg.Settings(uiProtection=mode)
        assert fg.validate(s) and "only CrosshairV2" in fg.settings_error(s)
    s = fg.Settings(uiProtection=3)   # CrosshairV2: built for every frame format, with or without the fill
    assert fg.validate(s) and fg.settings_error(s) is None
    for fmt in ("Rgba8", "Rgb10", "RgbaF16", "Nv12", "P010"):
        assert fg.settings_error(s, fmt=fmt) is None
        assert fg.settings_error(fg.Settings(uiProtection=3, uiEstimateFill=True), fmt=fmt) is None


def test_box_geometry():
    """Interpolator::boxSize / boxRect / boxMargin / workRect against gpu/framegen.cpp:1041-1075, restated in
    oracle/ui_v2.py"""
    import ui_v2
    cases = [fg.Settings(uiProtection=3), fg.Settings(uiProtection=3, uiBoxWidth=40, uiBoxHeight=6),
             fg.Settings(uiProtection=3, uiBoxOffsetX=5000, uiBoxOffsetY=-7), fg.Settings(uiProtection=3, uiBoxHeightFrac=0.0),
             fg.Settings(uiProtection=0), fg.Settings(uiProtection=1, uiBoxHeightFrac=0.3)]
    for s in cases:
        for W, H in ((3840, 2160), (640, 360), (17, 16), (101, 999)):
            assert fg.box_rect(s, W, H) == ui_v2.box_rect(s, W, H), (s, W, H)
            m = {0: 0, 1: 2, 2: 0, 3: 1}[s.uiProtection]
            assert fg.box_margin(s) == m
            assert fg.work_rect(s, W, H) == ui_v2.work_rect(s, W, H, m), (s, W, H)
    assert fg.box_rect(fg.Settings(), 3840, 2160) == (1893, 1053, 54, 54)   # round(2160 * 0.025) = 54


def test_format_of():
    assert fg.format_of(fg.VK_R8G8B8A8_UNORM) == "Rgba8" and fg.format_of(fg.VK_B8G8R8A8_UNORM) == "Rgba8"
    assert fg.format_of(fg.VK_A2B10G10R10_UNORM) == "Rgb10" and fg.format_of(fg.VK_R16G16B16A16_SFLOAT) == "RgbaF16"
    assert fg.format_of(fg.VK_R8_UNORM) == "Nv12" and fg.format_of(fg.VK_R16_UNORM) == "P010"
    assert fg.format_of(12345) is None


def test_init_refusals_without_recording():
    I = fg.Interpolator()
    assert not I.init(8, 8) and "kMinSize" in I.init_error()
    assert not I.init(64, 64, view_format=12345) and "viewFormat" in I.init_error()
    assert not I.init(64, 64, settings=fg.Settings(flowScale=3))
    # no estimate / not initialised: every record is refused and nothing is launched
    assert I.size_error(64, 64) == "not initialised"
    assert I.read_timings() is None
    assert I.read_costs() is None
    I.release_unused_ui()        # gpu/framegen.h:693, 700: nothing is ever unused here (V1 only, no UI memory)
    I.release_unused_motion()
    I.close()


NULL_PROBE = r"""
import ctypes, sys
sys.path[:0] = [sys.argv[1]]
import framegen as fg
L = fg.lib()
for name in sorted(fg.SIGNATURES):
    res, args = fg.SIGNATURES[name]
    vals = [0.0 if a in (ctypes.c_float, ctypes.c_double) else
            0 if a in (ctypes.c_int, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int64) else None for a in args]
    print(name, flush=True)
    getattr(L, name)(*vals)
print("all returned", flush=True)
"""


def test_null_arguments_never_crash():
    """every exported function called with null handles / pointers and zero sizes returns (the reference's API never
    throws; a null object is 'not initialised', not a crash), run in a child process so a crash names the function"""
    import subprocess
    import sys
    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "frame-gen-ritz_b200")
    r = subprocess.run([sys.executable, "-c", NULL_PROBE, pkg], capture_output=True, text=True, timeout=120)
    last = r.stdout.strip().splitlines()[-1] if r.stdout.strip() else "(nothing)"
    assert r.returncode == 0 and last == "all returned", f"crashed in {last}: {r.stderr[-500:]}"


def test_noalloc_frame_span_limit():
    """fg_record_synth_noalloc refuses a frame whose first plane spans more than 2^34 bytes ((height - 1) * pitch + the
    row's bytes; the 8-bit kernels address it in 32-bit words) and takes one that spans exactly 2^34. The pointers are
    stand-ins that are never dereferenced: the frame checks and the null field refuse each call before CUDA is used."""
    W = H = 16
    limit = 1 << 34
    at = (limit - 4 * W) // (H - 1)
    assert at % 4 == 0 and (H - 1) * at + 4 * W == limit

    def call(pitch, field=None):
        f = fg.CFrame()
        f.data, f.pitch = 1 << 20, pitch
        err = ctypes.c_char_p()
        ok = fg.lib().fg_record_synth_noalloc(None, fg.VK_R8G8B8A8_UNORM, W, H, ctypes.byref(f), ctypes.byref(f),
                                              ctypes.byref(f), field, 0, 0.5, ctypes.byref(fg.Settings().to_c()),
                                              ctypes.byref(err))
        return ok, err.value.decode()

    ok, msg = call(at)
    assert not ok and "field is null" in msg, msg   # the frames passed
    for pitch in (at + 4, limit + 4 * W, 1 << 62):
        ok, msg = call(pitch)
        assert not ok and "2^34" in msg, (pitch, msg)
    # the field is read as float pairs: a 4-byte aligned stand-in pointer is refused before CUDA is used
    ok, msg = call(at, field=(1 << 20) + 4)
    assert not ok and "8-byte aligned" in msg, msg


def test_batch_shape_round_trip():
    """Batch::Shape through the C ABI (no slots, no device needed): the default is the forked per-synthesis shape,
    fg_batch_set_shape_merged keeps mergeEstimates (1..8 groups), fg_batch_set_shape resets it, and shapes outside the
    ranges are refused without changing the current one"""
    B = fg.Batch()
    assert B.shape() == (0, 0, 8, 0)
    assert B.set_shape(0, 0, 8, 4) and B.shape() == (0, 0, 8, 4)
    assert B.set_shape(3, 1, 8) and B.shape() == (3, 1, 8, 0)
    for bad in ((0, 0, 0), (5, 0, 8), (0, 2, 8), (0, 0, 9), (0, 0, 8, 9)):
        assert not B.set_shape(*bad), bad
    assert B.shape() == (3, 1, 8, 0)
    B.close()
