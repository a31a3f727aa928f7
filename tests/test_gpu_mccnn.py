"""The MC-CNN cost path (a float matching-cost volume, read from im0.acrt by
the reference: main_bench_middv3.cu:73-108 with cost "MC-CNN"): the engine's
volume ingest and HBP on the float volume, bit for bit against the oracle.
Requires a GPU. The volumes are seeded synthetic stand-ins for a network's
output (scenes.mccnn_like_volume)."""
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


def ingest(E, ctx, torch, src, tau):
    D, H, W = src.shape
    s = torch.from_numpy(np.ascontiguousarray(src)).cuda()
    # filled with NaN: every float, overhanging tile entries included, must be written
    vol = torch.full((E.volume_f32_bytes(W, H, D) // 4,), float("nan"), dtype=torch.float32, device="cuda")
    wta = torch.full((H * W,), float("nan"), dtype=torch.float32, device="cuda")
    ctx.cost_f32_d(s, W, H, D, tau, vol, wta)
    torch.cuda.synchronize()
    v = vol.cpu().numpy()
    assert not np.isnan(v).any(), "tile overhang left unwritten"
    return vol, wta, E.volume_f32_to_dhw(v, W, H, D), wta.cpu().numpy().reshape(H, W)


@pytest.mark.parametrize("W,H,D,seed", CASES)
def test_ingest_bit_exact(eng, W, H, D, seed):
    import pyoracle as O
    from scenes import make_scene, mccnn_like_volume
    E, ctx, torch = eng
    src = mccnn_like_volume(make_scene(W, H, D, seed), D, seed + 1)
    _, _, vol, wta = ingest(E, ctx, torch, src, 0.5)
    ovol, owta = O.cost_f32(src, 0.5)
    assert np.array_equal(vol.view(np.uint32), ovol.view(np.uint32))
    assert np.array_equal(wta.view(np.uint32), owta.view(np.uint32))


@pytest.mark.parametrize("fp16", [0, 1])
@pytest.mark.parametrize("W,H,D,seed", CASES[:2])
def test_hbp_f32_bit_exact(eng, W, H, D, seed, fp16):
    """Same pyramid, float volume and WTA in (MC-CNN parameters: alpha 1.3,
    tau 0.5, tau_smooth 0.6): disparity and planes equal the oracle's bit for
    bit, with FP32 and with FP16 message storage."""
    import pyoracle as O
    from scenes import make_scene, mccnn_like_volume
    E, ctx, torch = eng
    sc = make_scene(W, H, D, seed)
    src = mccnn_like_volume(sc, D, seed + 1)
    vol_d, wta_d, vol, wta = ingest(E, ctx, torch, src, 0.5)
    ctx.segment_d(torch.from_numpy(np.ascontiguousarray(sc.left)).cuda(), W, H)
    pyr = ctx.pyramid()
    disp = torch.zeros(H * W, dtype=torch.float32, device="cuda")
    plane = torch.zeros(H * W * 3, dtype=torch.float32, device="cuda")
    prm = E.default_params(alpha=1.3, msg_fp16=fp16)
    ctx.infer_f32_d(vol_d, wta_d, D, 0.5, prm, disp, plane)
    torch.cuda.synchronize()
    od, op = O.hbp_f32(pyr, vol, wta, W, H, D, tau=0.5, alpha=1.3, fp16_msg=bool(fp16))
    gd = disp.cpu().numpy().reshape(H, W)
    gp = plane.cpu().numpy().reshape(H, W, 3)
    assert np.array_equal(gd.view(np.uint32), od.view(np.uint32)), float(np.mean(gd != od))
    assert np.array_equal(gp.view(np.uint32), op.view(np.uint32))


@pytest.mark.parametrize("W,H,D,seed", CASES)
def test_ingest_right_view_bit_exact(eng, W, H, D, seed):
    """Both views in one call: the right view equals the oracle's cost_to_right."""
    import pyoracle as O
    from scenes import make_scene, mccnn_like_volume
    E, ctx, torch = eng
    src = mccnn_like_volume(make_scene(W, H, D, seed), D, seed + 1)
    s = torch.from_numpy(src).cuda()
    nv = E.volume_f32_bytes(W, H, D) // 4
    vol, volR = (torch.full((nv,), float("nan"), device="cuda") for _ in range(2))
    wta, wtaR = (torch.full((H * W,), float("nan"), device="cuda") for _ in range(2))
    ctx.cost_f32_d(s, W, H, D, 0.5, vol, wta, volR, wtaR)
    torch.cuda.synchronize()
    for v, w, right in ((vol, wta, False), (volR, wtaR, True)):
        ov, ow = O.cost_f32(src, 0.5, right=right)
        got = E.volume_f32_to_dhw(v.cpu().numpy(), W, H, D)
        assert np.array_equal(got.view(np.uint32), ov.view(np.uint32))
        assert np.array_equal(w.cpu().numpy().reshape(H, W).view(np.uint32), ow.view(np.uint32))


def test_right_view_hbp_bit_exact(eng):
    """The right view's HBP (right image's pyramid, cost_to_right volume)
    equals the oracle's bit for bit."""
    import pyoracle as O
    from scenes import make_scene, mccnn_like_volume
    E, ctx, torch = eng
    W, H, D, seed = 160, 120, 48, 11
    sc = make_scene(W, H, D, seed)
    src = mccnn_like_volume(sc, D, seed + 1)
    nv = E.volume_f32_bytes(W, H, D) // 4
    volR = torch.zeros(nv, device="cuda")
    wtaR = torch.zeros(H * W, device="cuda")
    ctx.cost_f32_d(torch.from_numpy(src).cuda(), W, H, D, 0.5, None, None, volR, wtaR)
    ctx.segment_d(torch.from_numpy(np.ascontiguousarray(sc.right)).cuda(), W, H)
    disp = torch.zeros(H * W, device="cuda")
    ctx.infer_f32_d(volR, wtaR, D, 0.5, E.default_params(alpha=1.3), disp)
    ref = O.pipeline_f32(sc.left, src, R=sc.right)
    got = disp.cpu().numpy().reshape(H, W)
    assert np.array_equal(got.view(np.uint32), ref["disp"].view(np.uint32)), float(np.mean(got != ref["disp"]))


def test_mccnn_path_accuracy(eng):
    """On the synthetic MC-CNN-like volume the float path recovers the scene:
    bad-2.0 below 5% of non-occluded pixels (450x375, D 64)."""
    from scenes import make_scene, mccnn_like_volume
    E, ctx, torch = eng
    W, H, D = 450, 375, 64
    sc = make_scene(W, H, D, 1000)
    src = mccnn_like_volume(sc, D, 1001)
    vol_d, wta_d, _, _ = ingest(E, ctx, torch, src, 0.5)
    ctx.segment_d(torch.from_numpy(np.ascontiguousarray(sc.left)).cuda(), W, H)
    disp = torch.zeros(H * W, dtype=torch.float32, device="cuda")
    ctx.infer_f32_d(vol_d, wta_d, D, 0.5, E.default_params(alpha=1.3), disp)
    d = disp.cpu().numpy().reshape(H, W)
    bad = 100.0 * float(np.mean(np.abs(d - sc.gt)[sc.nonocc] > 2.0))
    assert bad < 5.0, bad
