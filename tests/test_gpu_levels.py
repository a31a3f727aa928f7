"""Per-level outputs (HBP_ISP::run_ms_vis, hbp_isp.cu:1348-1383, without its
superpixel drawing): every level's map from the top level down to min_level,
bit for bit against the oracle, on the Census and on a float volume.
Requires a GPU."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hbp_b200 as E
    ctx = E.Context(0)
    yield E, ctx, torch
    ctx.close()


def _levels(E, ctx, torch, s, D, vol, volf, wta, tau, prm):
    W, H = s.left.shape[1], s.left.shape[0]
    L = ctx.segment_d(torch.from_numpy(np.ascontiguousarray(s.left)).cuda(), W, H)
    n_max = L - prm.min_level
    dl = torch.full((n_max * H * W,), float("nan"), device="cuda")
    pl = torch.full((n_max * H * W * 3,), float("nan"), device="cuda")
    n = ctx.infer_levels_d(vol, volf, wta, D, tau, prm, n_max, dl, pl)
    assert n == n_max
    torch.cuda.synchronize()
    return ctx.pyramid(), dl.cpu().numpy().reshape(n, H, W), pl.cpu().numpy().reshape(n, H, W, 3)


@pytest.mark.parametrize("min_level", [2, 0])
def test_levels_census_bit_exact(eng, min_level):
    import pyoracle as O
    from scenes import make_scene
    E, ctx, torch = eng
    W, H, D = 160, 120, 48
    s = make_scene(W, H, D, 11)
    cuda = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    vol = torch.zeros(E.volume_bytes(W, H, D), dtype=torch.uint8, device="cuda")
    wta = torch.zeros(H * W, device="cuda")
    cL, cR = (torch.zeros(H * W, dtype=torch.int32, device="cuda") for _ in range(2))
    ctx.cost_census_d(cuda(s.left), cuda(s.right), W, H, D, cL, cR, vol, wta, None, None)
    prm = E.default_params(min_level=min_level)
    pyr, gd, gp = _levels(E, ctx, torch, s, D, vol, None, wta, 25.0, prm)
    cs = O.cost_stage(s.left, s.right, D)
    od, op = O.hbp_levels(pyr, cs["vol"], cs["wta"], W, H, D, min_level=min_level)
    assert gd.shape == od.shape and gd.shape[0] == len(pyr["level_sizes"]) - min_level
    assert np.array_equal(gd.view(np.uint32), od.view(np.uint32)), [float(np.mean(a != b)) for a, b in zip(gd, od)]
    assert np.array_equal(gp.view(np.uint32), op.view(np.uint32))
    assert not gd[0].any()  # top level: planes never written
    # the last map is the ordinary result
    disp = torch.zeros(H * W, device="cuda")
    ctx.infer_d(vol, wta, D, prm, disp)
    assert np.array_equal(disp.cpu().numpy().reshape(H, W).view(np.uint32), gd[-1].view(np.uint32))


def test_levels_float_volume_bit_exact(eng):
    import pyoracle as O
    from scenes import make_scene, mccnn_like_volume
    E, ctx, torch = eng
    W, H, D = 160, 120, 48
    s = make_scene(W, H, D, 11)
    src = mccnn_like_volume(s, D, 12)
    volf = torch.zeros(E.volume_f32_bytes(W, H, D) // 4, device="cuda")
    wta = torch.zeros(H * W, device="cuda")
    ctx.cost_f32_d(torch.from_numpy(src).cuda(), W, H, D, 0.5, volf, wta)
    prm = E.default_params(alpha=1.3, msg_fp16=1)
    pyr, gd, gp = _levels(E, ctx, torch, s, D, None, volf, wta, 0.5, prm)
    ov, ow = O.cost_f32(src, 0.5)
    od, op = O.hbp_levels(pyr, None, ow, W, H, D, volf=ov, tau=0.5, alpha=1.3, fp16_msg=True)
    assert np.array_equal(gd.view(np.uint32), od.view(np.uint32))
    assert np.array_equal(gp.view(np.uint32), op.view(np.uint32))
