"""Parity at the benchmark configurations' sizes: the engine's single-pair path
(hbp_run_pair, no post stage) against the CPU oracle, bit for bit, at
720x496 D128 (the quarter-scale batch's first pair, FP32 and FP16 messages),
1080x744 D192 (a size of the uneven batch) and 1440x992 D256 with 40 segments
(the precision workload, FP32 and FP16). These sizes reach the deep pyramids,
the warp-per-node select path and CRTrees on graphs of 357k to 1.4M nodes.

The oracle's disparity hashes come from tests/golden/make_large_oracle.py
(large_oracle.json). When this machine's scene or the oracle's sources differ
from the ones the fixture was made with, the oracle runs here instead.
The served mix at the end puts a 720x496 D128 request beside smaller ones and
compares each result with hbp_run_pair's."""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_large_oracle as G  # noqa: E402


@pytest.fixture(scope="module")
def eng():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hbp_b200 as E
    ctx = E.Context(0)
    yield E, ctx
    ctx.close()


def fixtures():
    path = os.path.join(HERE, "golden", "large_oracle.json")
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f)


@pytest.mark.parametrize("name", list(G.CASES))
def test_engine_matches_oracle_at_config_size(eng, name):
    E, ctx = eng
    case = G.CASES[name]
    W, H, D, seed, nseg, fp16 = case
    s = G.scene_of(case)
    disp = ctx.run_pair(s.left, s.right, D, E.default_params(post=0, msg_fp16=int(fp16)))
    fx = fixtures().get(name)
    stored = (fx is not None and fx["input_sha"] == G.sha_arrays(s.left, s.right)
              and fx["oracle_sha"] == G.oracle_source_sha())
    if stored and G.sha_arrays(disp) == fx["disp_sha"]:
        return
    ref = G.oracle_disp(case, s)  # no usable fixture, or a mismatch to report
    diff = float(np.mean(disp.view(np.uint32) != ref.view(np.uint32)))
    assert diff == 0.0, f"{name}: {diff:.4%} of pixels differ from the oracle (fixture used: {stored})"


def test_served_mix_with_headline_size_equals_run_pair(eng):
    """A 720x496 D128 request served beside 450x375 D64 and 160x120 D48 ones
    (FP16 messages, post 1): each result equals hbp_run_pair's bit for bit."""
    E, ctx = eng
    from scenes import make_scene
    mix = [(720, 496, 128, 1000), (450, 375, 64, 1001), (160, 120, 48, 1002), (720, 496, 128, 1003),
           (450, 375, 64, 1004)]
    scenes = [make_scene(W, H, D, sd) for W, H, D, sd in mix]
    prm = E.default_params(post=1, msg_fp16=1)
    want = [ctx.run_pair(s.left, s.right, m[2], prm) for s, m in zip(scenes, mix)]
    srv = E.Server(0, budget_bytes=24 << 30, prep_lanes=3, params=prm)
    try:
        ids = [srv.submit(s.left, s.right, m[2]) for s, m in zip(scenes, mix)]
        for rid, w, m in zip(ids, want, mix):
            got, _ = srv.wait(rid)
            assert np.array_equal(got.view(np.uint32), w.view(np.uint32)), m
    finally:
        srv.close()
