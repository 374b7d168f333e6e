"""The debug wire formats of the reference's test harness (gpu/fgtest.cpp:25-33, 777-789), which its tooling reads
(gpu/fgmaps.py: the .fgmaps maps; bench/score: the STATS lines): the header and the map layout, written by this
library's Python helpers (framegen.fgmaps_bytes / write_fgmaps / stats_line). The parser here restates the layout the
reference documents: a 64-byte header, then the block field (bw*bh vec2 f32), the per-pixel half-vector field (fw*fh
vec2 f32) and the packed mismatch (eStride*H uint32, 4 pixels per word, low byte first), back to back."""
import numpy as np
import pytest

import framegen as fg


def load_fgmaps(raw):
    h = np.frombuffer(raw[:64], np.uint32)
    hf = np.frombuffer(raw[40:56], np.float32)
    assert h[0] == 0x504D4746 and h[1] == 5
    W, H, fw, fh, bw, bh, fscale, es = (int(x) for x in h[2:10])
    o = 64
    block = np.frombuffer(raw, np.float32, bw * bh * 2, o).reshape(bh, bw, 2)
    o += bw * bh * 8
    pf = np.frombuffer(raw, np.float32, fw * fh * 2, o).reshape(fh, fw, 2)
    o += fw * fh * 8
    ew = np.frombuffer(raw, np.uint32, es * H, o).reshape(H, es)
    o += es * H * 4
    assert o == len(raw), "nothing after the packed mismatch"
    e = np.stack([(ew >> (8 * i)) & 255 for i in range(4)], -1).reshape(H, es * 4)[:, :W].astype(np.uint8)
    return dict(W=W, H=H, fw=fw, fh=fh, bw=bw, bh=bh, fscale=fscale, block=block, pf=pf, e=e, trust=tuple(hf[:2]),
                bonus=tuple(hf[2:4]), motion=int(h[14]), mode=int(h[15]))


def test_fgmaps_header_fields():
    l = fg.CDebugMapLayout()
    l.W, l.H, l.fw, l.fh, l.bw, l.bh, l.fscale, l.eStride = 321, 203, 161, 102, 21, 13, 2, 81
    s = fg.Settings(trustLow=10.0, trustHigh=44.5, smoothBonus=0.25, hudBonus=2.0)
    h = fg.fgmaps_header(l, s)
    assert len(h) == 64
    w = np.frombuffer(h, np.uint32)
    assert w[0] == 0x504D4746 and bytes(h[:4]) == b"FGMP" and w[1] == 5
    assert list(w[2:10]) == [321, 203, 161, 102, 21, 13, 2, 81]
    assert list(np.frombuffer(h[40:56], np.float32)) == [10.0, 44.5, 0.25, 2.0]
    assert w[14] == 0 and w[15] == 0


@pytest.mark.gpu
def test_fgmaps_file_and_stats_line(tmp_path):
    import build
    import oracle
    import torch
    import workloads
    from gpu_util import run_gpu
    build.build()
    p, c, _ = workloads.flow_pair(203, 117, seed=41, kind="fresh")
    tr, outs, unt, emaps, I = run_gpu(p, c, [0.5, 0.25], capture=True)
    l = I.debug_map_layout()
    assert (l.blockOff, l.pixOff, l.eOff) == (0, l.bw * l.bh * 8, l.bw * l.bh * 8 + l.fw * l.fh * 8)
    assert l.size == l.eOff + l.eStride * 4 * l.H
    path = tmp_path / "pair_0000.fgmaps"
    fg.write_fgmaps(I, str(path))
    d = load_fgmaps(path.read_bytes())
    assert (d["W"], d["H"], d["fw"], d["fh"], d["bw"], d["bh"], d["fscale"]) == (203, 117, l.fw, l.fh, l.bw, l.bh, 2)
    assert d["trust"] == (12.0, 40.0) and d["motion"] == 0
    assert np.array_equal(d["block"], tr["sub"][1]), "block field: the finest level after sub-pixel refinement"
    assert np.array_equal(d["pf"], tr["pf"])
    est = oracle.estimate(p, c)
    assert np.array_equal(d["e"], oracle.synth(p, c, est, 0.25, trace=True)["e"]), "mismatch of the latest synth"
    line = fg.stats_line(I, 7).split()
    assert line[0] == "STATS" and int(line[1]) == 7 and int(line[2]) == unt[-1]
    assert int(line[3]) == tr["sadSum256"] and int(line[4]) == I.debug_sad_blocks() and int(line[5]) == 203 * 117
    I.close()
