#!/usr/bin/env python3
"""Generates the golden fixtures of the V1 path by running the reference's own proto/interp.py.

Run with FGR_REF set to a checkout of the reference (read-only); interp.py is imported from
there, never copied, and its sha256 is pinned. Writes tests/golden/v1_golden.npz:

  per scene <name>:
    <name>/in_sha       sha256 of the regenerated input pair (the generator in frame-gen-ritz_b200/workloads.py is
                        seeded; the fixture stores only the digest so a drifting generator is caught)
    <name>/search<l>, <name>/median<l>   block fields per pyramid level (interp.search / interp.median3)
    <name>/sub0, sub1   the finest level after the 0.5 and 0.25 px steps
    <name>/sads, sad    the per-block SADs of the scene-cut test and their float32 mean
    <name>/pf           the per-pixel half-vector field (interp.pixel_field), absent for a cut
    <name>/out_t<k>     the synthesised frame (B,G,R uint8) for the k-th time of TS (small scenes), or
    <name>/outsha_t<k>  its sha256 (large scenes); <name>/why_t<k>: 0 none, 1 cut, 2 untrusted

Times TS are float32 values (the C API takes t as a float), passed to interp.synth as the Python floats they round to.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "frame-gen-ritz_b200"))
import workloads  # noqa: E402

INTERP_SHA256 = "b5f5c7000221002e31a1f4c2b2883878eeab4ffd83760c4080facad527904315"
TS = [0.5, 0.25, 0.75, float(np.float32(1 / 3)), float(np.float32(2 / 3))]
WHY = {None: 0, "cut": 1, "untrusted": 2}


def scenes():
    """(name, prev RGBA, curr RGBA, store full outputs?)"""
    p, c = workloads.pan_pair()
    yield "pan640x360", p, c, False
    for W, H in [(45, 33), (131, 97), (17, 16), (200, 120)]:
        p, c = workloads.pan_pair(W, H, seed=W)
        yield f"pan{W}x{H}", p, c, True
    for kind in ("normal", "fresh", "cut"):
        p, c, _ = workloads.flow_pair(320, 180, seed=7, kind=kind)
        yield f"flow_{kind}320x180", p, c, False
    p, c = workloads.contrast_pair(160, 96, seed=5, kind="cut")
    yield "hardcut160x96", p, c, True


def sha(*arrs):
    h = hashlib.sha256()
    for a in arrs:
        h.update(np.ascontiguousarray(a).tobytes())
    return np.frombuffer(h.digest(), np.uint8)


def load_interp():
    ref = os.environ.get("FGR_REF")
    if not ref:
        raise SystemExit("set FGR_REF to a checkout of the reference (the directory that holds proto/interp.py)")
    path = os.path.join(ref, "proto", "interp.py")
    digest = hashlib.sha256(open(path, "rb").read()).hexdigest()
    if digest != INTERP_SHA256:
        raise SystemExit(f"{path}: sha256 {digest} is not the pinned {INTERP_SHA256}")
    sys.path.insert(0, os.path.dirname(path))
    import interp
    return interp


def trace(interp, cv2, a, c):
    """interp.flow(a, c), keeping each level's search and median3 output and the two sub-pixel steps."""
    s = 1 / interp.FLOW_SCALE
    ya = cv2.resize(interp.luma(a), None, fx=s, fy=s, interpolation=cv2.INTER_AREA)
    yc = cv2.resize(interp.luma(c), None, fx=s, fy=s, interpolation=cv2.INTER_AREA)
    pa, pc = interp.pyramid(ya), interp.pyramid(yc)
    v, out = None, {}
    n = len(pa)
    for i, (la, lc) in enumerate(zip(reversed(pa), reversed(pc))):
        lvl = n - 1 - i
        la, lc = interp.pad_to_block(la), interp.pad_to_block(lc)
        bh, bw = la.shape[0] // interp.BLOCK, la.shape[1] // interp.BLOCK
        seed = np.zeros((bh, bw, 2), np.float32) if v is None else interp.seed_from(v, la, lc, bh, bw)
        vs, sad = interp.search(la, lc, seed, interp.TOP_RADIUS if v is None else interp.RADIUS, 1.0)
        v = interp.median3(vs)
        out[f"search{lvl}"], out[f"median{lvl}"] = vs, v
    for k, step in enumerate(interp.SUBPIX):
        v, sad = interp.search(la, lc, v, 1, step)
        out[f"sub{k}"] = v
    out["sads"] = sad
    return out


def main():
    import cv2
    interp = load_interp()
    data = {"ts": np.array(TS, np.float64), "interp_sha": np.frombuffer(bytes.fromhex(INTERP_SHA256), np.uint8),
            "cv2_version": np.frombuffer(cv2.__version__.encode(), np.uint8)}
    names = []
    for name, p, c, full in scenes():
        names.append(name)
        a, cc = np.ascontiguousarray(p[..., [2, 1, 0]]), np.ascontiguousarray(c[..., [2, 1, 0]])
        data[f"{name}/in_sha"] = sha(p, c)
        data[f"{name}/shape"] = np.array(p.shape[:2], np.int32)
        tr = trace(interp, cv2, a, cc)
        for k, v in tr.items():
            data[f"{name}/{k}"] = v
        est = interp.estimate(a, cc)
        data[f"{name}/sad"] = np.array([est["sad"]], np.float64)
        if est["pf"] is not None:
            data[f"{name}/pf"] = est["pf"]
        for k, t in enumerate(TS):
            o, why = interp.synth(a, cc, est, t, why=True)
            data[f"{name}/why_t{k}"] = np.array([WHY[why]], np.int32)
            if full:
                data[f"{name}/out_t{k}"] = o
            else:
                data[f"{name}/outsha_t{k}"] = sha(o)
        print(f"{name}: sad {est['sad']:.4f}, decisions",
              [int(data[f'{name}/why_t{k}'][0]) for k in range(len(TS))], flush=True)
    data["scenes"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "v1_golden.npz"), **data)


if __name__ == "__main__":
    main()
