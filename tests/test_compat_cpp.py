"""The reference-interface C++ classes (include/hbp_isp/): they compile
without a GPU, and the reference's two driver flows written against them give
the engine's results bit for bit (GPU)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "compat", "compat_pipeline.cpp")
LIBDIR = os.path.join(ROOT, "hbp-isp_b200", "lib")


def _compile(out, syntax_only=False):
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), SRC]
    if syntax_only:
        cmd += ["-fsyntax-only"]
    else:
        cmd += ["-L", LIBDIR, "-lhbp_b200", f"-Wl,-rpath,{LIBDIR}", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "warning" not in r.stderr, r.stderr


def test_headers_compile():
    _compile(None, syntax_only=True)


def test_cv_mat_conversions(tmp_path):
    """With an OpenCV core header on the include path (here the project's
    stand-in), hbp_isp::Mat wraps a cv::Mat without copying, converts back by
    copy, and refuses unsupported or non-continuous images. Host only."""
    exe = str(tmp_path / "cvmat_check")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "tests", "compat", "cv"), os.path.join(ROOT, "tests", "compat", "cvmat_check.cpp"),
           "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", (r.returncode, r.stdout, r.stderr)


def _run_driver(tmp_path, s, W, H, D, src=None):
    exe = str(tmp_path / "compat_pipeline")
    _compile(exe)
    (tmp_path / "l.bgr").write_bytes(np.ascontiguousarray(s.left).tobytes())
    (tmp_path / "r.bgr").write_bytes(np.ascontiguousarray(s.right).tobytes())
    args = [exe, str(tmp_path / "l.bgr"), str(tmp_path / "r.bgr"), str(W), str(H), str(D), str(tmp_path / "o_")]
    if src is not None:
        (tmp_path / "im0.acrt").write_bytes(np.ascontiguousarray(src, np.float32).tobytes())
        args.append(str(tmp_path / "im0.acrt"))
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

    def read(name):  # one H x W map, or [levels][H][W] for "*_levels"
        a = np.fromfile(tmp_path / f"o_{name}.f32", np.float32).reshape(-1, H, W)
        return a if name.endswith("levels") else a[0]
    return read


def _flows_via_stages(E, ctx, torch, s, D, vols, tau, alpha):
    """Both driver flows through the engine's stage entry points on float
    volumes (vol, wta, volR, wtaR): (single with the driver median, lr)."""
    W, H = s.left.shape[1], s.left.shape[0]
    n = W * H
    cuda = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    f = lambda k=1: torch.zeros(k * n, dtype=torch.float32, device="cuda")
    vol, wta, volR, wtaR = vols
    prm = E.default_params(alpha=alpha)
    dL, pL, dR, pR = f(), f(3), f(), f(3)
    ctx.segment_d(cuda(s.left), W, H)
    ctx.infer_f32_d(vol, wta, D, tau, prm, dL, pL)
    single = dL.clone()
    ctx.driver_median_d(single, W, H)
    ctx.segment_d(cuda(s.right), W, H)
    ctx.infer_f32_d(volR, wtaR, D, tau, prm, dR, pR)
    fail = torch.zeros(n, dtype=torch.uint8, device="cuda")
    dout = f()
    ctx.lr_check_d(dL, dR, pL, fail, dout, W, H)
    ctx.weighted_median_d(cuda(s.left), fail, pL, dout, W, H)
    torch.cuda.synchronize()
    return single.cpu().numpy().reshape(H, W), dout.cpu().numpy().reshape(H, W)


def _same(a, b):
    return np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.gpu
def test_driver_flows_match_the_engine(tmp_path):
    """Census and AD, both driver flows: the Census ones against hbp_run_pair,
    the AD ones against the engine's stage entry points, bit for bit."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hbp_b200 as E
    from scenes import make_scene
    W, H, D = 160, 120, 48
    s = make_scene(W, H, D, 77)
    out = _run_driver(tmp_path, s, W, H, D)
    ctx = E.Context(0)
    try:
        want1 = ctx.run_pair(s.left, s.right, D, E.default_params(post=1))
        want2 = ctx.run_pair(s.left, s.right, D, E.default_params(post=2))
        cuda = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        nv = E.volume_f32_bytes(W, H, D) // 4
        vols = [torch.zeros(k, dtype=torch.float32, device="cuda") for k in (nv, W * H, nv, W * H)]
        gL, gR = (torch.zeros(W * H, dtype=torch.float32, device="cuda") for _ in range(2))
        ctx.cost_ad_d(cuda(s.left), cuda(s.right), W, H, D, gL, gR, *vols)
        ad1, ad2 = _flows_via_stages(E, ctx, torch, s, D, vols, 30.0, 1000.1)
        # run_ms_vis of the Census flow against the engine's per-level entry point
        cL, cR = (torch.zeros(W * H, dtype=torch.int32, device="cuda") for _ in range(2))
        vol = torch.zeros(E.volume_bytes(W, H, D), dtype=torch.uint8, device="cuda")
        wta = torch.zeros(W * H, device="cuda")
        ctx.cost_census_d(cuda(s.left), cuda(s.right), W, H, D, cL, cR, vol, wta, None, None)
        L = ctx.segment_d(cuda(s.left), W, H)
        lv = torch.zeros((L - 2) * W * H, device="cuda")
        n = ctx.infer_levels_d(vol, None, wta, D, 25.0, E.default_params(), L - 2, lv)
        levels = lv.cpu().numpy().reshape(n, H, W)
        # the Census LR flow with the GPU variant of the weighted median
        n2 = W * H
        f = lambda k=1: torch.zeros(k * n2, dtype=torch.float32, device="cuda")
        dL, pL, dR, pR = f(), f(3), f(), f(3)
        volR = torch.zeros(E.volume_bytes(W, H, D), dtype=torch.uint8, device="cuda")
        wtaR = torch.zeros(W * H, device="cuda")
        ctx.cost_census_d(cuda(s.left), cuda(s.right), W, H, D, cL, cR, vol, wta, volR, wtaR)
        ctx.segment_d(cuda(s.left), W, H)
        ctx.infer_d(vol, wta, D, E.default_params(), dL, pL)
        ctx.segment_d(cuda(s.right), W, H)
        ctx.infer_d(volR, wtaR, D, E.default_params(), dR, pR)
        fail = torch.zeros(n2, dtype=torch.uint8, device="cuda")
        dout = f()
        ctx.lr_check_d(dL, dR, pL, fail, dout, W, H)
        ctx.weighted_median_gpu_d(cuda(s.left), fail, pL, dout, W, H)
        torch.cuda.synchronize()
        lr_gpu = dout.cpu().numpy().reshape(H, W)
    finally:
        ctx.close()
    _check_seg_pictures(tmp_path, s, W, H)
    assert _same(out("census_single"), want1) and _same(out("census_lr"), want2)
    assert _same(out("census_levels"), levels)
    assert _same(out("census_lr_gpu"), lr_gpu)
    assert _same(out("ad_single"), ad1) and _same(out("ad_lr"), ad2)


def _draw(labels, bgr, fmt):
    """draw_segmentation's pictures (segment.cu:213-292) of a 0-based label
    image, restated in numpy: "int" label+1; "u3" label+1 as B,G,R bytes, low
    byte first; "bd" the image with pixels unlike their left or upper
    neighbour set to (0,0,255)."""
    c = labels.astype(np.int64) + 1
    if fmt == "int":
        return c.astype(np.int32)
    if fmt == "u3":
        return np.stack([c & 255, (c >> 8) & 255, (c >> 16) & 255], -1).astype(np.uint8)
    edge = np.zeros(labels.shape, bool)
    edge[:, 1:] |= labels[:, 1:] != labels[:, :-1]
    edge[1:, :] |= labels[1:, :] != labels[:-1, :]
    out = bgr.copy()
    out[edge] = (0, 0, 255)
    return out


def _check_seg_pictures(tmp_path, s, W, H):
    """SegHAC::run_ms(&segs) in each picture format (Ward, 8 neighbours) against
    the engine's label image of every level (target 1) or of the 60
    superpixels, drawn by the reference's rules."""
    import hbp_b200 as E
    import torch
    ctx = E.Context(0)
    try:
        img = torch.from_numpy(np.ascontiguousarray(s.left)).cuda()
        for target in (1, 60):
            L = ctx.segment_target_d(img, W, H, 3, 8, 0.0, target)
            levels = range(L) if target == 1 else [L - 1]
            labels = []
            for lv in levels:
                t = torch.zeros(W * H, dtype=torch.int32, device="cuda")
                k = ctx.segment_labels_d(t, lv)
                lab = t.cpu().numpy().reshape(H, W)
                assert np.array_equal(np.unique(lab), np.arange(k))
                labels.append(lab)
            assert target == 1 or len(np.unique(labels[0])) == target
            for fmt, dt, ch in (("int", np.int32, 1), ("u3", np.uint8, 3), ("bd", np.uint8, 3)):
                got = np.fromfile(tmp_path / f"o_seg_{fmt}_t{target}.bin", dt)
                want = np.concatenate([_draw(lab, s.left, fmt).ravel() for lab in labels])
                assert got.shape == want.shape, (fmt, target)
                assert np.array_equal(got, want), (fmt, target)
    finally:
        ctx.close()


@pytest.mark.gpu
def test_mccnn_driver_flows_match_the_engine(tmp_path):
    """Both driver flows with the MC-CNN cost (volume read from an
    im0.acrt-style raw file by StereoCost) against the engine's stage entry
    points on the same volume, bit for bit."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hbp_b200 as E
    from scenes import make_scene, mccnn_like_volume
    W, H, D = 160, 120, 48
    s = make_scene(W, H, D, 78)
    src = mccnn_like_volume(s, D, 79)
    out = _run_driver(tmp_path, s, W, H, D, src)
    ctx = E.Context(0)
    try:
        nv = E.volume_f32_bytes(W, H, D) // 4
        vols = [torch.zeros(k, dtype=torch.float32, device="cuda") for k in (nv, W * H, nv, W * H)]
        ctx.cost_f32_d(torch.from_numpy(src).cuda(), W, H, D, 0.5, *vols)
        want1, want2 = _flows_via_stages(E, ctx, torch, s, D, vols, 0.5, 1.3)
    finally:
        ctx.close()
    assert _same(out("mccnn_single"), want1) and _same(out("mccnn_lr"), want2)
