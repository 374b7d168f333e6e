"""Python binding of the B200 framegen library's C ABI (include/framegen_c.h), by ctypes.

It mirrors framegen::Interpolator of frame-gen-ritz's gpu/framegen.h (init, resize, setSettings, reconfigure,
beginFrame, recordEstimate, recordSynth, record, setProfiling, readTimings, recordDebugCounters, debugMapLayout,
recordDebugMaps) with the same argument meaning and the same bool / error-string behaviour. Frames are CUDA tensors
(uint8, (H, W, 4), rows may be padded: pitch = stride(0)); streams are torch.cuda.Stream or raw handles.

The library is the only compute path: there is no CPU fallback. Loading fails loudly if libframegen_b200.so is
missing (build it with frame-gen-ritz_b200/build.py).
"""
import ctypes
import os
from dataclasses import dataclass, fields

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libframegen_b200.so")

# framegen::Format and the VkFormat numbers of include/framegen.h
FORMAT = {"Rgba8": 0, "Rgb10": 1, "RgbaF16": 2, "Nv12": 3, "P010": 4}
VK_R8G8B8A8_UNORM, VK_B8G8R8A8_UNORM = 37, 44
VK_A2R10G10B10_UNORM, VK_A2B10G10R10_UNORM = 58, 64
VK_R16G16B16A16_SFLOAT, VK_R8_UNORM, VK_R16_UNORM = 97, 9, 70
SET_RING, MIN_SIZE = 32, 16


class CSettings(ctypes.Structure):
    _fields_ = [("size", ctypes.c_uint32)] + \
               [(n, ctypes.c_float) for n in ("trustLow", "trustHigh", "globalFallback", "sceneCutSad", "hudBonus",
                                              "smoothBonus", "searchPenalty")] + \
               [(n, ctypes.c_uint32) for n in ("searchRadius", "searchRadiusTop", "subpixel", "uiProtection",
                                               "blurSamples", "blurWeights", "motionVersion", "flowScale",
                                               "pyramidMinSide")] + \
               [("uiHistory", ctypes.c_uint32), ("uiBoxHeightFrac", ctypes.c_float), ("uiBoxWidth", ctypes.c_uint32),
                ("uiBoxHeight", ctypes.c_uint32), ("uiCrosshairArea", ctypes.c_float), ("uiBoxOffsetX", ctypes.c_int32),
                ("uiBoxOffsetY", ctypes.c_int32), ("uiStillFrames", ctypes.c_uint32), ("uiStillThreshold", ctypes.c_float),
                ("uiInpaintReach", ctypes.c_uint32), ("uiMaxStillFraction", ctypes.c_float),
                ("uiContrastThreshold", ctypes.c_float), ("uiLeaveFrames", ctypes.c_uint32),
                ("uiReentryFrames", ctypes.c_uint32), ("uiEstimateFill", ctypes.c_uint32)]


class CFrame(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("pitch", ctypes.c_uint64), ("chroma", ctypes.c_void_p),
                ("chroma_pitch", ctypes.c_uint64)]


class CInitInfo(ctypes.Structure):
    _fields_ = [("size", ctypes.c_uint32), ("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("view_format", ctypes.c_uint32), ("transfer", ctypes.c_uint32), ("linear_white_nits", ctypes.c_float),
                ("yuv_matrix", ctypes.c_uint32), ("yuv_full_range", ctypes.c_uint32), ("device", ctypes.c_int32),
                ("settings", CSettings)]


class CDebugMapLayout(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("W", "H", "fw", "fh", "bw", "bh", "fscale", "eStride")] + \
               [(n, ctypes.c_uint64) for n in ("blockOff", "pixOff", "eOff", "size")]


class CTraceLayout(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("nLevels", "fw", "fh")] + \
               [(n, ctypes.c_uint32 * 16) for n in ("lw", "lh", "bw", "bh")] + \
               [(n, ctypes.c_uint64) for n in ("lumaOff", "lumaBytes", "fieldOff", "fieldBytes", "medOff", "sadOff",
                                               "pfOff", "stateOff", "size")] + \
               [("seedLevel", ctypes.c_uint32), ("seedOff", ctypes.c_uint64)]


# every symbol include/framegen_c.h declares, with (restype, argtypes)
_P, _U32, _I, _F, _S = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_float, ctypes.c_char_p


class CCosts(ctypes.Structure):
    _fields_ = [("estimate_ms", ctypes.c_float), ("synth_ms", ctypes.c_float), ("seq", ctypes.c_uint32),
                ("synths", ctypes.c_uint32)]
SIGNATURES = {
    "fg_abi_version": (_U32, []),
    "fg_default_settings": (None, [ctypes.POINTER(CSettings)]),
    "fg_default_init_info": (None, [ctypes.POINTER(CInitInfo)]),
    "fg_format_of": (_I, [_U32, ctypes.POINTER(_U32)]),
    "fg_create": (_P, []),
    "fg_destroy": (None, [_P]),
    "fg_init": (_I, [_P, ctypes.POINTER(CInitInfo)]),
    "fg_init_error": (_S, [_P]),
    "fg_format": (_U32, [_P]),
    "fg_resize": (_I, [_P, _U32, _U32, _U32]),
    "fg_validate": (_I, [ctypes.POINTER(CSettings)]),
    "fg_settings_error_format": (_S, [ctypes.POINTER(CSettings), _U32]),
    "fg_settings_error": (_S, [_P, ctypes.POINTER(CSettings)]),
    "fg_size_error": (_S, [_P, _U32, _U32]),
    "fg_set_settings": (_I, [_P, ctypes.POINTER(CSettings)]),
    "fg_reconfigure": (_I, [_P, ctypes.POINTER(CSettings)]),
    "fg_get_settings": (None, [_P, ctypes.POINTER(CSettings)]),
    "fg_begin_frame": (None, [_P]),
    "fg_release_unused_ui": (None, [_P]),
    "fg_release_unused_motion": (None, [_P]),
    "fg_record_estimate": (_I, [_P, _P, ctypes.POINTER(CFrame), ctypes.POINTER(CFrame)]),
    "fg_record_observe": (_I, [_P, _P, ctypes.POINTER(CFrame)]),
    "fg_record_track": (_I, [_P, _P, ctypes.POINTER(CFrame)]),
    "fg_box_size": (None, [ctypes.POINTER(CSettings), _U32, _U32, ctypes.POINTER(_U32), ctypes.POINTER(_U32)]),
    "fg_box_rect": (None, [ctypes.POINTER(CSettings), _U32, _U32, ctypes.POINTER(ctypes.c_int32)]),
    "fg_box_margin": (_U32, [ctypes.POINTER(CSettings)]),
    "fg_work_rect": (None, [ctypes.POINTER(CSettings), _U32, _U32, ctypes.POINTER(ctypes.c_int32)]),
    "fg_ui_trace_bytes": (ctypes.c_uint64, [_P]),
    "fg_ui_trace": (_I, [_P, _P, _P, _P]),
    "fg_record_synth": (_I, [_P, _P, ctypes.POINTER(CFrame), ctypes.POINTER(CFrame), ctypes.POINTER(CFrame), _F]),
    "fg_record": (_I, [_P, _P, ctypes.POINTER(CFrame), ctypes.POINTER(CFrame), ctypes.POINTER(CFrame), _F]),
    "fg_record_synth_blur": (_I, [_P, _P, ctypes.POINTER(CFrame), ctypes.POINTER(CFrame), ctypes.POINTER(CFrame), _F,
                                  _F]),
    "fg_blur_plan": (_U32, [_U32, _U32, _F, _F, _P, _P]),
    "fg_set_profiling": (_I, [_P, _I]),
    "fg_read_costs": (_I, [_P, _P]),
    "fg_read_timings": (_I, [_P, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_uint64), _U32,
                             ctypes.POINTER(_U32)]),
    "fg_record_debug_counters": (_I, [_P, _P, _P]),
    "fg_debug_sad_blocks": (_U32, [_P]),
    "fg_get_debug_map_layout": (_I, [_P, ctypes.POINTER(CDebugMapLayout)]),
    "fg_record_debug_maps": (_I, [_P, _P, _P]),
    "fg_set_debug_capture": (_I, [_P, _I]),
    "fg_get_trace_layout": (_I, [_P, ctypes.POINTER(CTraceLayout)]),
    "fg_record_trace": (_I, [_P, _P, _P]),
    "fg_last_error": (_S, [_P]),
    "fg_record_synth_noalloc": (_I, [_P, _U32, _U32, _U32, ctypes.POINTER(CFrame), ctypes.POINTER(CFrame),
                                     ctypes.POINTER(CFrame), _P, _I, _F, ctypes.POINTER(CSettings),
                                     ctypes.POINTER(ctypes.c_char_p)]),
    "fg_batch_create": (_P, []),
    "fg_batch_destroy": (None, [_P]),
    "fg_batch_add": (_I, [_P, ctypes.POINTER(CInitInfo), _U32]),
    "fg_batch_error": (_S, [_P]),
    "fg_batch_slots": (_U32, [_P]),
    "fg_batch_record": (_I, [_P, _P, _P, _P, _P]),
    "fg_batch_tune": (_I, [_P, _P, _P, _P, _P, _U32]),
    "fg_batch_get_shape": (None, [_P, ctypes.POINTER(_U32), ctypes.POINTER(_U32), ctypes.POINTER(_U32)]),
    "fg_batch_set_shape": (_I, [_P, _U32, _U32, _U32]),
    "fg_batch_set_shape_merged": (_I, [_P, _U32, _U32, _U32, _U32]),
    "fg_batch_merge_estimates": (_U32, [_P]),
    "fg_batch_trace_layout": (_I, [_P, _U32, ctypes.POINTER(CTraceLayout)]),
    "fg_batch_trace": (_I, [_P, _U32, _P, _P]),
    "fg_set_seed_net": (_I, [_P, _P, _U32]),
    "fg_seed_net_level": (_U32, [_P]),
    "fg_seednet_param_count": (_U32, []),
    "fg_seednet_create": (_P, [_I, _I, _I, _I]),
    "fg_seednet_destroy": (None, [_P]),
    "fg_seednet_error": (_S, [_P]),
    "fg_seednet_set_params": (_I, [_P, _P]),
    "fg_seednet_get_params": (_I, [_P, _P]),
    "fg_seednet_get_grads": (_I, [_P, _P]),
    "fg_seednet_pack": (_I, [_P, _P, _P, _I, _P]),
    "fg_seednet_forward": (_I, [_P, _P, _P, _I, _I, _I, _P]),
    "fg_seednet_forward_luma": (_I, [_P, _P, _P, _P, _I, _I, _I, _P]),
    "fg_seednet_forward_fused": (_I, [_P, _P, _P, _P, _I, _I, _I, _P]),
    "fg_seednet_fused_errors": (_U32, [_P]),
    "fg_seednet_backward": (_I, [_P, _P, _P, _I, _I, _I, _P, _P]),
    "fg_seednet_zero_grads": (_I, [_P, _P]),
    "fg_seednet_adam": (_I, [_P, _P, _F]),
    "fg_seednet_adam_scaled": (_I, [_P, _P, _F, _F]),
    "fg_seednet_grad_buffer": (_P, [_P]),
}

_lib = None


def lib():
    """Load libframegen_b200.so (no fallback: a missing library is an error)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with frame-gen-ritz_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _lib = L
    return _lib


@dataclass
class Settings:
    """framegen::Settings (the V1 fields), defaults = the tuned constants of proto/interp.py."""
    trustLow: float = 12.0
    trustHigh: float = 40.0
    globalFallback: float = 0.15
    sceneCutSad: float = 30.0
    hudBonus: float = 1.0
    smoothBonus: float = 0.5
    searchPenalty: float = 0.5
    searchRadius: int = 2
    searchRadiusTop: int = 6
    subpixel: bool = True
    uiProtection: int = 0
    blurSamples: int = 0
    blurWeights: int = 1
    motionVersion: int = 0
    flowScale: int = 2
    pyramidMinSide: int = 48
    uiHistory: int = 3
    uiBoxHeightFrac: float = 0.025
    uiBoxWidth: int = 0
    uiBoxHeight: int = 0
    uiCrosshairArea: float = 0.03
    uiBoxOffsetX: int = 0
    uiBoxOffsetY: int = 0
    uiStillFrames: int = 8
    uiStillThreshold: float = 3.5
    uiInpaintReach: int = 12
    uiMaxStillFraction: float = 0.75
    uiContrastThreshold: float = 20.0
    uiLeaveFrames: int = 4
    uiReentryFrames: int = 2
    uiEstimateFill: bool = False

    def to_c(self):
        c = CSettings()
        c.size = ctypes.sizeof(CSettings)
        for f in fields(self):
            setattr(c, f.name, int(getattr(self, f.name)) if f.type in (int, bool) else getattr(self, f.name))
        return c

    @staticmethod
    def from_c(c):
        s = Settings()
        for f in fields(s):
            v = getattr(c, f.name)
            setattr(s, f.name, bool(v) if f.type is bool else v)
        return s


def _s(b):
    return None if b is None else b.decode()


def frame_of(t, chroma=None):
    """A CFrame for a CUDA tensor (pitch = the row stride in bytes): (H, W, 4) uint8 for Rgba8, (H, W) int32 words
    for Rgb10, (H, W, 4) float16 for RgbaF16; Nv12 / P010 frames are (Y plane, CbCr plane) tuples or pass chroma."""
    if t is None:
        return None
    if isinstance(t, tuple):
        t, chroma = t
    f = CFrame()
    f.data = t.data_ptr()
    f.pitch = t.stride(0) * t.element_size()
    if chroma is not None:
        f.chroma = chroma.data_ptr()
        f.chroma_pitch = chroma.stride(0) * chroma.element_size()
    return f


def _stream(s):
    if s is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return s if isinstance(s, int) else s.cuda_stream


def validate(settings):
    return bool(lib().fg_validate(ctypes.byref(settings.to_c())))


def settings_error(settings, fmt="Rgba8"):
    return _s(lib().fg_settings_error_format(ctypes.byref(settings.to_c()), FORMAT[fmt]))


def format_of(view_format):
    out = ctypes.c_uint32()
    return {v: k for k, v in FORMAT.items()}[out.value] if lib().fg_format_of(view_format, ctypes.byref(out)) else None


class Interpolator:
    """framegen::Interpolator through the C ABI."""

    def __init__(self):
        self._h = lib().fg_create()

    def close(self):
        if self._h and _lib is not None:   # (at interpreter exit the module's globals may already be gone)
            _lib.fg_destroy(self._h)
        self._h = None

    __del__ = close

    def init(self, width, height, view_format=VK_R8G8B8A8_UNORM, settings=None, device=-1, transfer=0,
             linear_white_nits=80.0, yuv_matrix=1, yuv_full_range=False):
        ii = CInitInfo()
        lib().fg_default_init_info(ctypes.byref(ii))
        ii.width, ii.height, ii.view_format, ii.device = width, height, view_format, device
        ii.transfer, ii.linear_white_nits, ii.yuv_matrix, ii.yuv_full_range = transfer, linear_white_nits, yuv_matrix, int(yuv_full_range)
        ii.settings = (settings or Settings()).to_c()
        return bool(lib().fg_init(self._h, ctypes.byref(ii)))

    def init_error(self):
        return _s(lib().fg_init_error(self._h))

    def format(self):
        return {v: k for k, v in FORMAT.items()}[lib().fg_format(self._h)]

    def resize(self, w, h, view_format=VK_R8G8B8A8_UNORM):
        return bool(lib().fg_resize(self._h, w, h, view_format))

    def settings_error(self, settings):
        return _s(lib().fg_settings_error(self._h, ctypes.byref(settings.to_c())))

    def size_error(self, w, h):
        return _s(lib().fg_size_error(self._h, w, h))

    def set_settings(self, settings):
        return bool(lib().fg_set_settings(self._h, ctypes.byref(settings.to_c())))

    def reconfigure(self, settings):
        return bool(lib().fg_reconfigure(self._h, ctypes.byref(settings.to_c())))

    def settings(self):
        c = CSettings()
        lib().fg_get_settings(self._h, ctypes.byref(c))
        return Settings.from_c(c)

    def begin_frame(self):
        lib().fg_begin_frame(self._h)

    def release_unused_ui(self):
        lib().fg_release_unused_ui(self._h)

    def release_unused_motion(self):
        lib().fg_release_unused_motion(self._h)

    def record_observe(self, frame, stream=None):
        """recordObserve: static-UI protection (CrosshairV2) advances its state with this real frame and keeps its mask"""
        return bool(lib().fg_record_observe(self._h, _stream(stream), ctypes.byref(frame_of(frame))))

    def record_track(self, frame, stream=None):
        """recordTrack: the state update only, for a real frame passed through without generating"""
        return bool(lib().fg_record_track(self._h, _stream(stream), ctypes.byref(frame_of(frame))))

    def record_estimate(self, prev, curr, stream=None):
        return bool(lib().fg_record_estimate(self._h, _stream(stream), ctypes.byref(frame_of(prev)),
                                             ctypes.byref(frame_of(curr))))

    def record_synth(self, prev, curr, out, t, stream=None):
        return bool(lib().fg_record_synth(self._h, _stream(stream), ctypes.byref(frame_of(prev)),
                                          ctypes.byref(frame_of(curr)), ctypes.byref(frame_of(out)), float(t)))

    def record(self, prev, curr, out, t=0.5, stream=None):
        return bool(lib().fg_record(self._h, _stream(stream), ctypes.byref(frame_of(prev)),
                                    ctypes.byref(frame_of(curr)), ctypes.byref(frame_of(out)), float(t)))

    def record_synth_blur(self, prev, curr, out, t0, t1, stream=None):
        """recordSynthBlur: the weighted average of settings.blurSamples sub-frames over [t0, t1]"""
        return bool(lib().fg_record_synth_blur(self._h, _stream(stream), ctypes.byref(frame_of(prev)),
                                               ctypes.byref(frame_of(curr)), ctypes.byref(frame_of(out)), float(t0),
                                               float(t1)))

    def set_profiling(self, on):
        return bool(lib().fg_set_profiling(self._h, int(on)))

    def read_timings(self):
        n = 64
        names = (ctypes.c_char_p * n)()
        ns = (ctypes.c_uint64 * n)()
        cnt = ctypes.c_uint32()
        if not lib().fg_read_timings(self._h, names, ns, n, ctypes.byref(cnt)):
            return None
        return [(names[i].decode(), int(ns[i])) for i in range(min(cnt.value, n))]

    def read_costs(self):
        """readCosts: {estimate_ms, synth_ms, seq, synths} of the last profile (the pacer's cost-guard inputs), or None"""
        c = CCosts()
        if not lib().fg_read_costs(self._h, ctypes.byref(c)):
            return None
        return {"estimate_ms": c.estimate_ms, "synth_ms": c.synth_ms, "seq": c.seq, "synths": c.synths}

    def record_debug_counters(self, dst, stream=None):
        return bool(lib().fg_record_debug_counters(self._h, _stream(stream), dst.data_ptr()))

    def debug_sad_blocks(self):
        return int(lib().fg_debug_sad_blocks(self._h))

    def debug_map_layout(self):
        l = CDebugMapLayout()
        return l if lib().fg_get_debug_map_layout(self._h, ctypes.byref(l)) else None

    def record_debug_maps(self, dst, stream=None):
        return bool(lib().fg_record_debug_maps(self._h, _stream(stream), dst.data_ptr()))

    def set_debug_capture(self, on):
        return bool(lib().fg_set_debug_capture(self._h, int(on)))

    def trace_layout(self):
        l = CTraceLayout()
        return l if lib().fg_get_trace_layout(self._h, ctypes.byref(l)) else None

    def record_trace(self, dst, stream=None):
        return bool(lib().fg_record_trace(self._h, _stream(stream), dst.data_ptr()))

    def last_error(self):
        return _s(lib().fg_last_error(self._h))

    def set_seed_net(self, params, level=1):
        """Interpolator::setSeedNet: CNN-seeded estimates from `level` with these flat float32 parameters (None: off)"""
        if params is None:
            return bool(lib().fg_set_seed_net(self._h, None, 0))
        p = np.ascontiguousarray(params, np.float32)
        return bool(lib().fg_set_seed_net(self._h, p.ctypes.data, int(level)))

    def seed_net_level(self):
        v = int(lib().fg_seed_net_level(self._h))
        return None if v == 0xFFFFFFFF else v


# ---------------------------------------------------------------------------------------------- debug wire formats
# What the reference's test harness writes for its tooling (gpu/fgtest.cpp:25-33, 777-789; read by gpu/fgmaps.py and
# bench/score): an .fgmaps file = a 64-byte header then Interpolator::recordDebugMaps' bytes, and one STATS line per
# pair = recordDebugCounters' two counts with the block count and the pixel count.
FGMAPS_MAGIC, FGMAPS_VERSION = 0x504D4746, 5   # 'FGMP'


def fgmaps_header(layout, settings):
    """the 64-byte fgmaps header: uint32 magic, version, W, H, fw, fh, bw, bh, fscale, eStride, float32 trustLow,
    trustHigh, smoothBonus, hudBonus, uint32 motionVersion, v2Mode (0 here: V1 has no mode)"""
    h = np.zeros(16, np.uint32)
    h[:10] = [FGMAPS_MAGIC, FGMAPS_VERSION, layout.W, layout.H, layout.fw, layout.fh, layout.bw, layout.bh,
              layout.fscale, layout.eStride]
    h[10:14] = np.array([settings.trustLow, settings.trustHigh, settings.smoothBonus, settings.hudBonus],
                        np.float32).view(np.uint32)
    h[14] = settings.motionVersion
    return h.tobytes()


def fgmaps_bytes(fg, stream=None):
    """an fgmaps file's bytes for the latest records of Interpolator fg (header + recordDebugMaps: the block field,
    the per-pixel half-vector field, the packed mismatch of the latest synth recorded with setDebugCapture on)"""
    import torch
    l = fg.debug_map_layout()
    if l is None:
        raise RuntimeError("not initialised")
    buf = torch.zeros(int(l.size), dtype=torch.uint8, device="cuda")
    if not fg.record_debug_maps(buf, stream=stream):
        raise RuntimeError("recordDebugMaps failed")
    (stream or torch.cuda.current_stream()).synchronize()
    return fgmaps_header(l, fg.settings()) + buf.cpu().numpy().tobytes()


def write_fgmaps(fg, path, stream=None):
    with open(path, "wb") as f:
        f.write(fgmaps_bytes(fg, stream))


def stats_line(fg, pair, stream=None):
    """'STATS <pair> <untrusted px> <SAD sum x256> <SAD blocks> <W*H>': the whole-frame decision inputs of the latest
    synth (recordDebugCounters), as the reference harness prints them for its scoring scripts"""
    import torch
    cnt = torch.zeros(2, dtype=torch.int32, device="cuda")
    if not fg.record_debug_counters(cnt, stream=stream):
        raise RuntimeError("recordDebugCounters failed")
    (stream or torch.cuda.current_stream()).synchronize()
    u, s = (int(v) & 0xFFFFFFFF for v in cnt.cpu().tolist())
    l = fg.debug_map_layout()
    return f"STATS {pair} {u} {s} {fg.debug_sad_blocks()} {l.W * l.H}"


def read_trace(fg, stream=None):
    """Copy the latest estimate's intermediates to the host: a dict in the oracle's trace layout."""
    import torch
    l = fg.trace_layout()
    buf = torch.empty(l.size, dtype=torch.uint8, device="cuda")
    assert fg.record_trace(buf, stream)
    torch.cuda.synchronize()
    h = buf.cpu().numpy()
    f32 = lambda off, n: h[off:off + 4 * n].view(np.float32)
    n = l.nLevels
    luma, fld, o, of = [], [], l.lumaOff, l.fieldOff
    for i in range(n):
        w, hh, bw, bh = l.lw[i], l.lh[i], l.bw[i], l.bh[i]
        luma.append((f32(o, w * hh).reshape(hh, w), f32(o + 4 * w * hh, w * hh).reshape(hh, w)))
        o += 8 * w * hh
        fld.append((f32(of, 2 * bw * bh).reshape(bh, bw, 2), f32(of + 8 * bw * bh, 2 * bw * bh).reshape(bh, bw, 2)))
        of += 16 * bw * bh
    bw0, bh0 = l.bw[0], l.bh[0]
    sub = [f32(of, 2 * bw0 * bh0).reshape(bh0, bw0, 2), f32(of + 8 * bw0 * bh0, 2 * bw0 * bh0).reshape(bh0, bw0, 2)]
    st = h[l.stateOff:l.stateOff + 16].view(np.uint32)
    seed = None
    if l.seedLevel != 0xFFFFFFFF:
        k = l.seedLevel
        seed = f32(l.seedOff, 8 * l.bw[k] * l.bh[k]).reshape(l.bh[k], l.bw[k], 8)
    return {"seed_level": None if seed is None else int(l.seedLevel), "seed": seed,"luma": luma, "fields": fld, "sub": sub, "meds": f32(l.medOff, 2 * n).reshape(n, 2),
            "sads": f32(l.sadOff, bw0 * bh0).reshape(bh0, bw0), "pf": f32(l.pfOff, 2 * l.fw * l.fh).reshape(l.fh, l.fw, 2),
            "cut": bool(st[0]), "sad": float(st[1:2].view(np.float32)[0]), "sadSum256": int(st[2]), "err": int(st[3])}


def blur_plan(samples, gaussian, t0, t1):
    """Interpolator::blurPlan: ([t_k as float32], [q_k in units of 2^-16]) of a blur, or None if refused"""
    times = (ctypes.c_float * 16)()
    q = (ctypes.c_uint32 * 16)()
    n = lib().fg_blur_plan(int(samples), int(bool(gaussian)), float(t0), float(t1), ctypes.addressof(times),
                           ctypes.addressof(q))
    if n == 0:
        return None
    return np.array(times[:n], np.float32), [int(v) for v in q[:n]]


def record_synth_noalloc(prev, curr, out, field, cut, t, settings=None, view_format=VK_R8G8B8A8_UNORM, stream=None):
    """fg_record_synth_noalloc: the synthesis without an Interpolator and without allocating (the per-pixel field and the
    scene-cut decision come from the caller). Returns (ok, error message or None)."""
    err = ctypes.c_char_p()
    H, W = prev.shape[:2]
    ok = lib().fg_record_synth_noalloc(_stream(stream), view_format, W, H, ctypes.byref(frame_of(prev)),
                                       ctypes.byref(frame_of(curr)), ctypes.byref(frame_of(out)), field.data_ptr(),
                                       int(cut), float(t), ctypes.byref((settings or Settings()).to_c()),
                                       ctypes.byref(err))
    return bool(ok), (err.value.decode() if err.value else None)


class SeedNet:
    """The seed proposer (fg_seednet_*): parameters, forward pass and training step on the GPU. Inputs are CUDA
    tensors: x (B, h, w, 2) bfloat16 from pack(), targets (B, ceil(h/8), ceil(w/8), 6) float32."""

    N_OUT, N_TGT = 8, 6

    def __init__(self, max_batch, max_h, max_w, device=-1):
        self._h = lib().fg_seednet_create(device, max_batch, max_h, max_w)
        if not self._h:
            raise RuntimeError("fg_seednet_create failed")
        self.n_params = int(lib().fg_seednet_param_count())

    def close(self):
        if self._h and _lib is not None:
            _lib.fg_seednet_destroy(self._h)
        self._h = None

    __del__ = close

    def _ok(self, r):
        if not r:
            raise RuntimeError(f"seed net call failed: {_s(lib().fg_seednet_error(self._h))}")

    def set_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == self.n_params
        self._ok(lib().fg_seednet_set_params(self._h, p.ctypes.data))

    def params(self):
        p = np.zeros(self.n_params, np.float32)
        self._ok(lib().fg_seednet_get_params(self._h, p.ctypes.data))
        return p

    def grads(self):
        g = np.zeros(self.n_params, np.float32)
        self._ok(lib().fg_seednet_get_grads(self._h, g.ctypes.data))
        return g

    @staticmethod
    def pack(luma_prev, luma_curr, stream=None):
        """(..., h, w) float32 CUDA luma pair -> (..., h, w, 2) bfloat16 net input"""
        import torch
        x = torch.empty(tuple(luma_prev.shape) + (2,), dtype=torch.bfloat16, device=luma_prev.device)
        assert lib().fg_seednet_pack(_stream(stream), luma_prev.data_ptr(), luma_curr.data_ptr(), luma_prev.numel(),
                                     x.data_ptr())
        return x

    def forward(self, x, out=None, stream=None):
        import torch
        B, h, w = x.shape[:3]
        if out is None:
            out = torch.empty((B, (h + 7) // 8, (w + 7) // 8, self.N_OUT), dtype=torch.float32, device=x.device)
        self._ok(lib().fg_seednet_forward(self._h, _stream(stream), x.data_ptr(), B, h, w, out.data_ptr()))
        return out

    def forward_luma(self, luma_prev, luma_curr, out=None, stream=None):
        """the forward pass straight from (B, h, w) float32 luma planes (the first layer packs them)"""
        import torch
        B, h, w = luma_prev.shape
        if out is None:
            out = torch.empty((B, (h + 7) // 8, (w + 7) // 8, self.N_OUT), dtype=torch.float32, device=luma_prev.device)
        self._ok(lib().fg_seednet_forward_luma(self._h, _stream(stream), luma_prev.data_ptr(), luma_curr.data_ptr(), B,
                                               h, w, out.data_ptr()))
        return out

    def forward_fused(self, luma_prev, luma_curr, out=None, stream=None):
        """the fused tensor-core forward (two launches; the Interpolator's) from (B, h, w) float32 luma planes"""
        import torch
        B, h, w = luma_prev.shape
        if out is None:
            out = torch.empty((B, (h + 7) // 8, (w + 7) // 8, self.N_OUT), dtype=torch.float32, device=luma_prev.device)
        self._ok(lib().fg_seednet_forward_fused(self._h, _stream(stream), luma_prev.data_ptr(), luma_curr.data_ptr(),
                                                B, h, w, out.data_ptr()))
        return out

    def fused_errors(self):
        """the fused forward's sticky error bits (4: a tensor-core wait gave up); synchronous"""
        return int(lib().fg_seednet_fused_errors(self._h))

    def backward(self, x, targets, loss=None, stream=None):
        B, h, w = x.shape[:3]
        self._ok(lib().fg_seednet_backward(self._h, _stream(stream), x.data_ptr(), B, h, w, targets.data_ptr(),
                                           None if loss is None else loss.data_ptr()))

    def zero_grads(self, stream=None):
        self._ok(lib().fg_seednet_zero_grads(self._h, _stream(stream)))

    def adam(self, lr, grad_scale=1.0, stream=None):
        """one Adam step on the gradient times grad_scale (1 / ranks after a data-parallel all-reduce sum)"""
        if grad_scale == 1.0:
            self._ok(lib().fg_seednet_adam(self._h, _stream(stream), float(lr)))
        else:
            self._ok(lib().fg_seednet_adam_scaled(self._h, _stream(stream), float(lr), float(grad_scale)))

    def grad_buffer(self):
        """the float32 gradient accumulator as a CUDA tensor view (no copy; valid while the net lives), for an
        in-place all-reduce between backward() and adam()"""
        import torch
        ptr = lib().fg_seednet_grad_buffer(self._h)
        if not ptr:
            raise RuntimeError("fg_seednet_grad_buffer failed")

        class _View:
            __cuda_array_interface__ = {"shape": (self.n_params,), "typestr": "<f4", "data": (ptr, False),
                                        "version": 3, "strides": None}
        return torch.as_tensor(_View(), device=torch.device("cuda", torch.cuda.current_device()))


class Batch:
    """framegen::Batch through the C ABI: many frame pairs (slots) of any sizes and formats recorded together; the
    8-bit RGBA syntheses of all slots run in one persistent launch. Frames as for Interpolator (tuples for YUV)."""

    def __init__(self):
        self._h = lib().fg_batch_create()
        self.mult = []

    def close(self):
        if self._h and _lib is not None:
            _lib.fg_batch_destroy(self._h)
        self._h = None

    __del__ = close

    def add(self, width, height, view_format=VK_R8G8B8A8_UNORM, multiplier=2, settings=None, device=-1, transfer=0,
            linear_white_nits=80.0, yuv_matrix=1, yuv_full_range=False):
        ii = CInitInfo()
        lib().fg_default_init_info(ctypes.byref(ii))
        ii.width, ii.height, ii.view_format, ii.device = width, height, view_format, device
        ii.transfer, ii.linear_white_nits, ii.yuv_matrix, ii.yuv_full_range = transfer, linear_white_nits, yuv_matrix, int(yuv_full_range)
        ii.settings = (settings or Settings()).to_c()
        i = lib().fg_batch_add(self._h, ctypes.byref(ii), int(multiplier))
        if i >= 0:
            self.mult.append(int(multiplier))
        return i

    def error(self):
        return _s(lib().fg_batch_error(self._h))

    @staticmethod
    def times(multiplier):
        import numpy as np
        return [float(np.float32(k) / np.float32(multiplier)) for k in range(1, multiplier)]

    def _frames(self, prev, curr, outs):
        p = (CFrame * len(prev))(*[frame_of(f) for f in prev])
        c = (CFrame * len(curr))(*[frame_of(f) for f in curr])
        o = (CFrame * len(outs))(*[frame_of(f) for f in outs])
        return p, c, o

    def record(self, prev, curr, outs, stream=None):
        """prev, curr: one frame per slot; outs: every slot's multiplier - 1 output frames, slots in order"""
        p, c, o = self._frames(prev, curr, outs)
        return bool(lib().fg_batch_record(self._h, _stream(stream), p, c, o))

    def tune(self, prev, curr, outs, reps=3, stream=None):
        p, c, o = self._frames(prev, curr, outs)
        return int(lib().fg_batch_tune(self._h, _stream(stream), p, c, o, int(reps)))

    def shape(self):
        """(ctasPerSm, order, streams, mergeEstimates)"""
        a, b, c = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        lib().fg_batch_get_shape(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return a.value, b.value, c.value, int(lib().fg_batch_merge_estimates(self._h))

    def set_shape(self, ctas_per_sm, order, streams=8, merge_estimates=0):
        return bool(lib().fg_batch_set_shape_merged(self._h, int(ctas_per_sm), int(order), int(streams),
                                                    int(merge_estimates)))


def box_rect(settings, W, H):
    """Interpolator::boxRect: (x, y, w, h) of the static-UI box of a W x H frame"""
    r = (ctypes.c_int32 * 4)()
    lib().fg_box_rect(ctypes.byref(settings.to_c()), W, H, r)
    return tuple(r)


def work_rect(settings, W, H):
    """Interpolator::workRect: the box grown by boxMargin, clamped to the frame"""
    r = (ctypes.c_int32 * 4)()
    lib().fg_work_rect(ctypes.byref(settings.to_c()), W, H, r)
    return tuple(r)


def box_margin(settings):
    return int(lib().fg_box_margin(ctypes.byref(settings.to_c())))


def read_ui(I, frame, settings, W, H, stream=None):
    """the CrosshairV2 state of an Interpolator and the kept mask of `frame` (a CUDA tensor; its data pointer is the
    key): dict with w0, w1, w2 ((wh, ww) uint32 each), mask ((wh, ww) uint8), header (4 words), rect"""
    import numpy as np
    import torch
    n = int(lib().fg_ui_trace_bytes(I._h))
    if not n:
        return None
    buf = torch.empty(n, dtype=torch.uint8, device="cuda")
    key = frame[0].data_ptr() if isinstance(frame, tuple) else frame.data_ptr()
    assert lib().fg_ui_trace(I._h, _stream(stream), key, buf.data_ptr())
    torch.cuda.synchronize()
    raw = buf.cpu().numpy()
    wx, wy, ww, wh = work_rect(settings, W, H)
    st = raw[:ww * wh * 16].view(np.uint32).reshape(wh, ww, 4)
    mk = raw[ww * wh * 16:].view(np.uint32)
    stride = (ww + 3) // 4
    mask = mk[4:4 + stride * wh].view(np.uint8).reshape(wh, stride * 4)[:, :ww]
    return {"w0": st[..., 0], "w1": st[..., 1], "w2": st[..., 2], "mask": mask, "header": mk[:4].copy(),
            "rect": (wx, wy, ww, wh)}
