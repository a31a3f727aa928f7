"""The AD cost path (StereoCost::compute_stereo_cost("AD"), stereo_cost.cu:
421-429): float grey images, the truncated absolute-difference volume of both
views and HBP on it, bit for bit against the oracle. Requires a GPU."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [(96, 64, 32, 7), (160, 120, 48, 11), (203, 77, 40, 3)]  # W, H, D, seed (ragged tiles included)


@pytest.fixture(scope="module")
def eng():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hbp_b200 as E
    ctx = E.Context(0)
    yield E, ctx, torch
    ctx.close()


def run_ad(E, ctx, torch, L, R, D):
    H, W = L.shape[:2]
    cuda = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    nv = E.volume_f32_bytes(W, H, D) // 4
    # filled with NaN: every float, overhanging tile entries included, must be written
    vol, volR = (torch.full((nv,), float("nan"), device="cuda") for _ in range(2))
    wta, wtaR, gL, gR = (torch.full((H * W,), float("nan"), device="cuda") for _ in range(4))
    ctx.cost_ad_d(cuda(L), cuda(R), W, H, D, gL, gR, vol, wta, volR, wtaR)
    torch.cuda.synchronize()
    out = dict(vol_d=vol, wta_d=wta, volR_d=volR, wtaR_d=wtaR)
    for k, v in (("vol", vol), ("volR", volR)):
        a = v.cpu().numpy()
        assert not np.isnan(a).any(), "tile overhang left unwritten"
        out[k] = E.volume_f32_to_dhw(a, W, H, D)
    for k, v in (("wta", wta), ("wtaR", wtaR), ("greyL", gL), ("greyR", gR)):
        out[k] = v.cpu().numpy().reshape(H, W)
    return out


def test_grey_every_colour(eng):
    """The float grey image of all 2^24 colours equals the oracle's (the
    reference's double expression stored as float)."""
    import pyoracle as O
    E, ctx, torch = eng
    c = np.arange(1 << 24, dtype=np.uint32)
    img = np.stack([c & 255, (c >> 8) & 255, c >> 16], axis=1).astype(np.uint8).reshape(4096, 4096, 3)
    g = run_ad(E, ctx, torch, img, img, 2)
    want = O.grey_f32(img)
    assert np.array_equal(g["greyL"].view(np.uint32), want.view(np.uint32))
    assert np.array_equal(g["greyR"].view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("W,H,D,seed", CASES)
def test_ad_volume_bit_exact(eng, W, H, D, seed):
    import pyoracle as O
    from scenes import make_scene
    E, ctx, torch = eng
    s = make_scene(W, H, D, seed)
    g = run_ad(E, ctx, torch, s.left, s.right, D)
    for right, vk, wk in ((False, "vol", "wta"), (True, "volR", "wtaR")):
        ov, ow, ogL, ogR = O.cost_ad(s.left, s.right, D, right=right)
        assert np.array_equal(g[vk].view(np.uint32), ov.view(np.uint32)), vk
        assert np.array_equal(g[wk].view(np.uint32), ow.view(np.uint32)), wk
    assert np.array_equal(g["greyL"].view(np.uint32), ogL.view(np.uint32))
    assert np.array_equal(g["greyR"].view(np.uint32), ogR.view(np.uint32))


@pytest.mark.parametrize("right", [False, True])
def test_ad_hbp_bit_exact(eng, right):
    """HBP on the AD volume (tau 30), left and right view, equals the oracle's
    bit for bit."""
    import pyoracle as O
    from scenes import make_scene
    E, ctx, torch = eng
    W, H, D = 160, 120, 48
    s = make_scene(W, H, D, 11)
    g = run_ad(E, ctx, torch, s.left, s.right, D)
    ctx.segment_d(torch.from_numpy(np.ascontiguousarray(s.right if right else s.left)).cuda(), W, H)
    disp = torch.zeros(H * W, device="cuda")
    plane = torch.zeros(H * W * 3, device="cuda")
    vol, wta = (g["volR_d"], g["wtaR_d"]) if right else (g["vol_d"], g["wta_d"])
    ctx.infer_f32_d(vol, wta, D, 30.0, E.default_params(), disp, plane)
    ref = O.pipeline_ad(s.left, s.right, D, right_view=right)
    got = disp.cpu().numpy().reshape(H, W)
    assert np.array_equal(got.view(np.uint32), ref["disp"].view(np.uint32)), float(np.mean(got != ref["disp"]))
    assert np.array_equal(plane.cpu().numpy().reshape(H, W, 3).view(np.uint32), ref["plane"].view(np.uint32))
