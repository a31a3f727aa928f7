"""PFM files and bad-pixel rates (include/hbp_isp/io.hpp): the C++ writer and
reader round-trip 1- and 3-channel images, read a PFM written here, and the
evaluator's all / nonocc / occ rates equal a numpy restatement of
Evaluator.h:49-79. CPU only."""
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def write_pfm(path, img):
    """PFM as the format defines it: header, little endian (negative scale), rows bottom-up."""
    h, w = img.shape[:2]
    ch = 1 if img.ndim == 2 else img.shape[2]
    with open(path, "wb") as f:
        f.write(f"{'Pf' if ch == 1 else 'PF'}\n{w} {h}\n-1.0\n".encode())
        f.write(np.ascontiguousarray(img[::-1], dtype="<f4").tobytes())


def read_pfm(path):
    with open(path, "rb") as f:
        tag = f.readline().strip()
        w, h = map(int, f.readline().split())
        scale = float(f.readline())
        data = np.frombuffer(f.read(), dtype="<f4" if scale < 0 else ">f4")
    ch = 1 if tag == b"Pf" else 3
    img = data.reshape(h, w, ch) if ch == 3 else data.reshape(h, w)
    return img[::-1]


def bad_rates(disp, gt, nonocc, t):
    valid = (gt > 0) & np.isfinite(gt)
    good = np.abs(disp - gt) <= t
    occ = valid & ~nonocc
    r = lambda m: 100.0 * (1.0 - np.count_nonzero(good & m) / np.count_nonzero(m))
    return r(valid), r(nonocc), r(occ)


def test_pfm_and_evaluator(tmp_path):
    from scenes import make_scene
    W, H = 96, 64
    s = make_scene(W, H, 32, 3)
    rng = np.random.default_rng(0)
    disp = (s.gt + rng.normal(0, 1.5, s.gt.shape)).astype(np.float32)
    gt = s.gt.copy()
    gt[0, :5] = 0.0          # invalid ground truth
    gt[1, :3] = np.inf
    (tmp_path / "disp.f32").write_bytes(disp.tobytes())
    (tmp_path / "gt.f32").write_bytes(gt.astype(np.float32).tobytes())
    (tmp_path / "nonocc.u8").write_bytes((s.nonocc.astype(np.uint8) * 255).tobytes())
    write_pfm(tmp_path / "py.pfm", disp)
    exe = str(tmp_path / "io_check")
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "compat", "io_check.cpp"), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0 and "warning" not in r.stderr, r.stderr
    r = subprocess.run([exe, str(tmp_path), str(W), str(H)], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stderr)
    lines = r.stdout.split("\n")
    for line, t in zip(lines[:2], (1.0, 2.0)):
        got = [float(v) for v in line.split()]
        want = bad_rates(disp, gt, s.nonocc, t)
        assert np.allclose(got, want, rtol=0, atol=1e-9), (got, want)
    assert float(lines[2]) == round(float(disp[0, 0]), 6)
    assert np.array_equal(read_pfm(tmp_path / "cpp1.pfm"), disp)
    three = read_pfm(tmp_path / "cpp3.pfm")
    assert three.shape == (H, W, 3) and np.array_equal(three[..., 2], disp + 2)
