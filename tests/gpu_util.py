"""Helpers of the GPU tests: run the CUDA path through the C ABI and compare it with the oracle."""
import numpy as np
import torch

import framegen as fg
import oracle

ORDER_VK = {"rgba": fg.VK_R8G8B8A8_UNORM, "bgra": fg.VK_B8G8R8A8_UNORM}


def to_dev(a, pad=0):
    """(H, W, 4) uint8 -> a CUDA tensor; pad > 0 adds that many unused pixels per row (pitch > W * 4)."""
    t = torch.from_numpy(np.ascontiguousarray(a))
    if not pad:
        return t.cuda()
    H, W, C = a.shape
    buf = torch.zeros((H, W + pad, C), dtype=torch.uint8, device="cuda")
    buf[:, :W] = t.cuda()
    return buf[:, :W]


def new_out(like, pad=0):
    H, W, C = like.shape
    buf = torch.full((H, W + pad, C), 7, dtype=torch.uint8, device="cuda")
    return buf[:, :W]


def run_gpu(prev, curr, ts, settings=None, order="rgba", pad=0, capture=False):
    """One estimate + one synth per t on the GPU: returns (trace, outputs, untrusted counts, interpolator)."""
    H, W = prev.shape[:2]
    I = fg.Interpolator()
    assert I.init(W, H, ORDER_VK[order], settings=settings), I.init_error()
    a, c = to_dev(prev, pad), to_dev(curr, pad)
    if capture:
        I.set_debug_capture(True)
    I.begin_frame()
    assert I.record_estimate(a, c), I.last_error()
    tr = fg.read_trace(I)
    outs, unt, emaps = [], [], []
    cnt = torch.zeros(2, dtype=torch.int32, device="cuda")
    for t in ts:
        o = new_out(a, pad)
        assert I.record_synth(a, c, o, t), I.last_error()
        assert I.record_debug_counters(cnt)
        if capture:
            l = I.debug_map_layout()
            buf = torch.zeros(l.size, dtype=torch.uint8, device="cuda")
            assert I.record_debug_maps(buf)
            torch.cuda.synchronize()
            e = buf[l.eOff:l.eOff + l.eStride * 4 * l.H].view(l.H, l.eStride * 4)[:, :W].cpu().numpy()
            emaps.append(e)
        torch.cuda.synchronize()
        outs.append(o.cpu().numpy())
        unt.append(int(cnt[0]))
    return tr, outs, unt, emaps, I


def decision(cut, unt, W, H, frac=0.15):
    """The whole-frame decision the GPU took: its cut flag, else its untrusted share against globalFallback (a float)."""
    if cut:
        return "cut"
    return "untrusted" if unt / (W * H) > float(np.float32(frac)) else None


def assert_estimate_equal(tr, est, check_luma=True):
    """Every intermediate of the GPU estimate equals the oracle's (bit-exact)."""
    n = len(est["layout"].levels)
    assert len(tr["fields"]) == n
    for l in range(n):
        if check_luma:
            for k in range(2):
                assert np.array_equal(tr["luma"][l][k], est["luma"][l][k]), f"luma level {l}"
        assert np.array_equal(tr["fields"][l][0], est["fields"][l][0]), \
            f"search level {l}: {np.count_nonzero((tr['fields'][l][0] != est['fields'][l][0]).any(-1))} blocks differ"
        assert np.array_equal(tr["fields"][l][1], est["fields"][l][1]), f"median3 level {l}"
        assert np.array_equal(tr["meds"][l], est["meds"][l]), f"global median of level {l}"
    if "sub" in est:
        for k in range(2):
            assert np.array_equal(tr["sub"][k], est["sub"][k]), f"subpixel step {k}"
    assert np.array_equal(tr["sads"], est["sads"]), "block SADs"
    assert tr["sad"] == est["sad"], ("scene-cut mean", tr["sad"], est["sad"])
    assert tr["cut"] == est["cut"]
    assert tr["err"] == 0
    assert np.array_equal(tr["pf"], est["pf"]), f"pixel field: {np.count_nonzero((tr['pf'] != est['pf']).any(-1))} px differ"


def frame_diff(a, b):
    d = np.abs(a.astype(np.int16) - b.astype(np.int16))
    return int(d.max()), float(d.mean()), int(np.count_nonzero(d))
