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


@pytest.mark.gpu
def test_driver_flows_match_the_engine(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import hbp_b200 as E
    from scenes import make_scene
    exe = str(tmp_path / "compat_pipeline")
    _compile(exe)
    W, H, D = 160, 120, 48
    s = make_scene(W, H, D, 77)
    (tmp_path / "l.bgr").write_bytes(np.ascontiguousarray(s.left).tobytes())
    (tmp_path / "r.bgr").write_bytes(np.ascontiguousarray(s.right).tobytes())
    r = subprocess.run([exe, str(tmp_path / "l.bgr"), str(tmp_path / "r.bgr"), str(W), str(H), str(D),
                        str(tmp_path / "single.f32"), str(tmp_path / "lr.f32")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    single = np.fromfile(tmp_path / "single.f32", np.float32).reshape(H, W)
    lr = np.fromfile(tmp_path / "lr.f32", np.float32).reshape(H, W)
    ctx = E.Context(0)
    try:
        want1 = ctx.run_pair(s.left, s.right, D, E.default_params(post=1))
        want2 = ctx.run_pair(s.left, s.right, D, E.default_params(post=2))
    finally:
        ctx.close()
    assert np.array_equal(single.view(np.uint32), want1.view(np.uint32))
    assert np.array_equal(lr.view(np.uint32), want2.view(np.uint32))


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
    exe = str(tmp_path / "compat_pipeline")
    _compile(exe)
    W, H, D = 160, 120, 48
    s = make_scene(W, H, D, 78)
    src = mccnn_like_volume(s, D, 79)
    (tmp_path / "l.bgr").write_bytes(np.ascontiguousarray(s.left).tobytes())
    (tmp_path / "r.bgr").write_bytes(np.ascontiguousarray(s.right).tobytes())
    (tmp_path / "im0.acrt").write_bytes(src.tobytes())
    outs = [str(tmp_path / n) for n in ("c1.f32", "c2.f32", "m1.f32", "m2.f32")]
    r = subprocess.run([exe, str(tmp_path / "l.bgr"), str(tmp_path / "r.bgr"), str(W), str(H), str(D),
                        outs[0], outs[1], str(tmp_path / "im0.acrt"), outs[2], outs[3]],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    single = np.fromfile(outs[2], np.float32).reshape(H, W)
    lr = np.fromfile(outs[3], np.float32).reshape(H, W)

    ctx = E.Context(0)
    try:
        cuda = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        n = H * W
        f = lambda k=1: torch.zeros(k * n, dtype=torch.float32, device="cuda")
        nv = E.volume_f32_bytes(W, H, D) // 4
        vol, volR = (torch.zeros(nv, dtype=torch.float32, device="cuda") for _ in range(2))
        wta, wtaR = f(), f()
        ctx.cost_f32_d(cuda(src), W, H, D, 0.5, vol, wta, volR, wtaR)
        prm = E.default_params(alpha=1.3)
        dL, pL, dR, pR = f(), f(3), f(), f(3)
        ctx.segment_d(cuda(s.left), W, H)
        ctx.infer_f32_d(vol, wta, D, 0.5, prm, dL, pL)
        want1 = dL.clone()
        ctx.driver_median_d(want1, W, H)
        ctx.segment_d(cuda(s.right), W, H)
        ctx.infer_f32_d(volR, wtaR, D, 0.5, prm, dR, pR)
        fail = torch.zeros(n, dtype=torch.uint8, device="cuda")
        dout = f()
        ctx.lr_check_d(dL, dR, pL, fail, dout, W, H)
        ctx.weighted_median_d(cuda(s.left), fail, pL, dout, W, H)
        torch.cuda.synchronize()
        want1 = want1.cpu().numpy().reshape(H, W)
        want2 = dout.cpu().numpy().reshape(H, W)
    finally:
        ctx.close()
    assert np.array_equal(single.view(np.uint32), want1.view(np.uint32))
    assert np.array_equal(lr.view(np.uint32), want2.view(np.uint32))
