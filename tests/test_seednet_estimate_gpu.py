"""CNN-seeded estimates (Interpolator::setSeedNet) against the oracle.

With the seed net on at level k the library runs the net on level k's luma, seeds that level's integer search with the
net's candidates and skips the levels above it. The net computes in bf16 (checked against float64 in
test_seednet_gpu.py); everything from its output on is exact, so the oracle, given the GPU net's output
(oracle.estimate(..., seed_net=(k, output))), must reproduce every later stage and output byte bit for bit.
"""
import os

import numpy as np
import pytest
import torch

import framegen as fg
import oracle
import seednet_ref as ref
import workloads
from gpu_util import decision, frame_diff, new_out, to_dev

pytestmark = pytest.mark.gpu
WEIGHTS = os.path.join(os.path.dirname(fg.__file__), "seednet_l1.bin")


@pytest.fixture(scope="module", autouse=True)
def built():
    import build
    build.build()


def net_params():
    """the trained weights when they ship, else a seeded random net (the exactness argument does not need training)"""
    if os.path.exists(WEIGHTS):
        return np.fromfile(WEIGHTS, np.float32)
    return ref.init_params(3)


def run(prev, curr, params, level, ts):
    H, W = prev.shape[:2]
    I = fg.Interpolator()
    assert I.init(W, H, fg.VK_R8G8B8A8_UNORM), I.init_error()
    assert I.set_seed_net(params, level)
    k = I.seed_net_level()
    a, c = to_dev(prev), to_dev(curr)
    I.begin_frame()
    assert I.record_estimate(a, c), I.last_error()
    tr = fg.read_trace(I)
    outs, unt = [], []
    cnt = torch.zeros(2, dtype=torch.int32, device="cuda")
    for t in ts:
        o = new_out(a)
        assert I.record_synth(a, c, o, t), I.last_error()
        assert I.record_debug_counters(cnt)
        torch.cuda.synchronize()
        outs.append(o.cpu().numpy())
        unt.append(int(cnt[0]))
    return I, k, tr, outs, unt


@pytest.mark.parametrize("size,level", [((640, 360), 1), ((1280, 720), 1), ((1280, 720), 0), ((321, 203), 5)])
def test_seeded_estimate_matches_oracle(size, level):
    W, H = size
    prev, curr, _ = workloads.flow_pair(W, H, seed=41)
    ts = [0.5, 0.25]
    I, k, tr, outs, unt = run(prev, curr, net_params(), level, ts)
    assert tr["seed_level"] == k and k <= level
    est = oracle.estimate(prev, curr, seed_net=(k, tr["seed"]))
    for l in range(k + 1):
        for j in range(2):
            assert np.array_equal(tr["luma"][l][j], est["luma"][l][j]), f"luma level {l}"
            assert np.array_equal(tr["fields"][l][j], est["fields"][l][j]), f"field {j} level {l}"
    for l in range(k):
        assert np.array_equal(tr["meds"][l], est["meds"][l]), f"global median of level {l}"
    for j in range(2):
        assert np.array_equal(tr["sub"][j], est["sub"][j]), f"subpixel step {j}"
    assert np.array_equal(tr["sads"], est["sads"]) and tr["sad"] == est["sad"] and tr["cut"] == est["cut"]
    assert tr["err"] == 0
    assert np.array_equal(tr["pf"], est["pf"])
    for t, o, u in zip(ts, outs, unt):
        r = oracle.synth(prev, curr, est, t, trace=True)
        assert decision(tr["cut"], u, W, H) == r["reason"]
        assert frame_diff(o, r["out"])[2] == 0, f"t={t}"
    # the net itself on the level's luma, against float64 (the seeds above depend on it only through rounding)
    la, lc = tr["luma"][k]
    want = ref.forward(ref.unflatten(net_params()), ref.pack(la[None], lc[None])).detach().numpy()[0]
    err, scale = np.abs(tr["seed"] - want).max(), np.abs(want).max()
    assert err <= 0.03 * max(1.0, scale), f"logit error {err:.4g} at scale {scale:.3g}"
    I.close()


def test_switching_the_net_off_restores_the_plain_path():
    prev, curr, _ = workloads.flow_pair(640, 360, seed=42)
    I = fg.Interpolator()
    assert I.init(640, 360, fg.VK_R8G8B8A8_UNORM)
    assert I.set_seed_net(net_params(), 1) and I.seed_net_level() == 1
    assert I.set_seed_net(None) and I.seed_net_level() is None
    a, c = to_dev(prev), to_dev(curr)
    I.begin_frame()
    assert I.record_estimate(a, c)
    tr = fg.read_trace(I)
    est = oracle.estimate(prev, curr)
    assert tr["seed_level"] is None
    assert np.array_equal(tr["pf"], est["pf"]) and tr["sad"] == est["sad"]
    I.close()
