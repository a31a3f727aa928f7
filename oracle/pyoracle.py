"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE: a CPU restatement of the reference HBP-ISP stereo path
used to check the B200 engine. Only tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline / reference legs import this module; the engine never
does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
P = C.c_void_p


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
    return LIB_PATH


def _p(a):
    return None if a is None else a.ctypes.data_as(P)


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _lib.orc_crtrees.restype = C.c_int
        _lib.orc_crtrees_literal.restype = C.c_int
        _lib.orc_segment.restype = C.c_int
        _lib.orc_segment_cfg.restype = C.c_int
        _lib.orc_segment_target.restype = C.c_int
        _lib.orc_lab_sigma.argtypes = [P, C.c_int, C.c_int, C.c_double, P]
        _lib.orc_hbp.restype = C.c_int
        _lib.orc_hbp.argtypes = [P, C.c_int, P, P, P, P, P, P, C.c_int, C.c_int, C.c_int, C.c_float,
                                 C.c_float, C.c_int, C.c_int, C.c_long, P, P, P, P]
        _lib.orc_hbp_lockstep.restype = C.c_int
        _lib.orc_hbp_lockstep.argtypes = [P, C.c_int, P, P, P, P, P, P, C.c_int, C.c_int, C.c_int, C.c_float,
                                          C.c_float, C.c_int, C.c_int, C.c_int, P, P]
        _lib.orc_hbp_f32.restype = C.c_int
        _lib.orc_hbp_f32.argtypes = [P, C.c_int, P, P, P, P, P, P, C.c_int, C.c_int, C.c_int, C.c_float,
                                     C.c_float, C.c_float, C.c_int, C.c_int, C.c_long, P, P, P, P]
        _lib.orc_hbp_levels.restype = C.c_int
        _lib.orc_hbp_levels.argtypes = [P, C.c_int, P, P, P, P, P, P, P, C.c_int, C.c_int, C.c_int, C.c_float,
                                        C.c_float, C.c_float, C.c_int, C.c_int, P, P]
        _lib.orc_cost_f32.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_float, P, P]
        _lib.orc_cost_f32_right.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_float, P, P]
        _lib.orc_grey_f32.argtypes = [P, C.c_int, P]
        _lib.orc_cost_ad.argtypes = [P, P, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, P, P]
        _load_lab_overrides()
    return _lib


# The colours whose LAB differs between the host's pow and the device's (found by
# an exhaustive sweep against the reference build, tests/golden/make_golden.py
# --only lab_sweep); the oracle returns the reference's values there.
LAB_OVERRIDES = os.path.join(os.path.dirname(HERE), "tests", "golden", "lab_overrides.npz")


def _load_lab_overrides():
    if os.path.exists(LAB_OVERRIDES):
        z = np.load(LAB_OVERRIDES)
        set_lab_overrides(z["keys"], z["vals"])


def grey_u8(bgr: np.ndarray) -> np.ndarray:
    bgr = np.ascontiguousarray(bgr, np.uint8)
    out = np.zeros(bgr.shape[:2], np.uint8)
    lib().orc_grey_u8(_p(bgr), int(bgr.shape[0] * bgr.shape[1]), _p(out))
    return out


def census(grey: np.ndarray) -> np.ndarray:
    grey = np.ascontiguousarray(grey, np.uint8)
    H, W = grey.shape
    out = np.zeros((H, W), np.uint32)
    lib().orc_census(_p(grey), W, H, _p(out))
    return out


def cost_volume(cL, cR, D):
    H, W = cL.shape
    vol = np.zeros((D, H * W), np.uint8)
    wta = np.zeros((H, W), np.float32)
    lib().orc_cost_volume(_p(np.ascontiguousarray(cL)), _p(np.ascontiguousarray(cR)), W, H, D, _p(vol), _p(wta))
    return vol, wta


def cost_to_right(volL, W, H, D):
    volR = np.zeros_like(volL)
    wta = np.zeros((H, W), np.float32)
    lib().orc_cost_to_right(_p(np.ascontiguousarray(volL)), W, H, D, _p(volR), _p(wta))
    return volR, wta


def set_lab_overrides(keys: np.ndarray, vals: np.ndarray):
    keys = np.ascontiguousarray(keys, np.uint32)
    vals = np.ascontiguousarray(vals, np.float32)
    order = np.argsort(keys)
    keys, vals = keys[order], vals[order]
    global _lab_keep
    _lab_keep = (keys, vals)
    lib().orc_lab_set_overrides(_p(keys), _p(vals), int(len(keys)))


def lab(bgr: np.ndarray) -> np.ndarray:
    bgr = np.ascontiguousarray(bgr, np.uint8)
    H, W = bgr.shape[:2]
    out = np.zeros((H, W, 4), np.float32)
    lib().orc_lab(_p(bgr), H * W, _p(out))
    return out


def nn_grid(lab4: np.ndarray):
    lab4 = np.ascontiguousarray(lab4, np.float32)
    H, W = lab4.shape[:2]
    nn = np.zeros(H * W, np.int32)
    dmin = np.zeros(H * W, np.float32)
    bd = np.zeros((H * W * 4, 2), np.int32)
    lib().orc_nn_grid(_p(lab4), W, H, _p(nn), _p(dmin), _p(bd))
    return nn, dmin, bd


def crtrees(nn: np.ndarray, literal: bool = False):
    nn = np.ascontiguousarray(nn, np.int32)
    out = np.zeros_like(nn)
    f = lib().orc_crtrees_literal if literal else lib().orc_crtrees
    n = f(_p(nn), len(nn), _p(out))
    return out, n


def lab_sigma(bgr: np.ndarray, sigma: float) -> np.ndarray:
    """LAB of the image blurred with sigma (SegHAC::img_CPU_to_GPU)."""
    bgr = np.ascontiguousarray(bgr, np.uint8)
    H, W = bgr.shape[:2]
    out = np.zeros((H, W, 4), np.float32)
    lib().orc_lab_sigma(_p(bgr), W, H, float(sigma), _p(out))
    return out


def segment(lab4: np.ndarray, link: int = 2, num_nb: int = 4) -> dict:
    """SegHAC pyramid of a LAB image; link 0 Min, 1 Max, 2 Centroid, 3 Ward."""
    lab4 = np.ascontiguousarray(lab4, np.float32)
    H, W = lab4.shape[:2]
    n = H * W
    sizes = np.zeros(2 * 64, np.int32)
    clus = np.zeros(2 * n, np.int32)
    mean = np.zeros(12 * n, np.float32)
    bd = np.zeros(4 * num_nb * n, np.int32)
    bdl = np.zeros(2 * num_nb * n, np.int32)
    L = lib().orc_segment_cfg(_p(lab4), W, H, link, num_nb, 64, _p(sizes), _p(clus), _p(mean), _p(bd), _p(bdl))
    if L < 1:
        raise ValueError("orc_segment_cfg rejected its input")
    sizes = sizes[: 2 * L].reshape(L, 2)
    tc, tb = int(sizes[:, 0].sum()), int(sizes[:, 1].sum())
    return dict(level_sizes=sizes, clus=clus[:tc], mean=mean[: 6 * tc], bd=bd[: 2 * tb].reshape(tb, 2), bdl=bdl[:tb])


def segment_target(lab4: np.ndarray, target: int, link: int = 2, num_nb: int = 4) -> dict:
    """SegHAC with target_clus (the superpixel mode): the pyramid up to the
    level whose clus maps onto exactly `target` superpixels, and the label
    image (each pixel's superpixel)."""
    H, W = lab4.shape[:2]
    N0 = W * H
    sizes = np.zeros((64, 2), np.int32)
    clus = np.zeros(2 * N0, np.int32)
    mean = np.zeros(12 * N0, np.float32)
    bd = np.zeros((4 * num_nb * N0,), np.int32)
    bdl = np.zeros(2 * num_nb * N0, np.int32)
    L = lib().orc_segment_target(_p(np.ascontiguousarray(lab4, np.float32)), W, H, link, num_nb, target, 64,
                                 _p(sizes), _p(clus), _p(mean), _p(bd), _p(bdl))
    if L < 1:
        raise ValueError("oracle segmentation rejected its input")
    sizes = sizes[:L].copy()
    tn, te = int(sizes[:, 0].sum()), int(sizes[:, 1].sum())
    labels = np.arange(N0, dtype=np.int64)
    off = 0
    for l in range(L):
        labels = clus[off + labels]
        off += int(sizes[l, 0])
    return dict(level_sizes=sizes, clus=clus[:tn].copy(), mean=mean[:6 * tn].copy(),
                bd=bd[:2 * te].reshape(te, 2).copy(), bdl=bdl[:te].copy(),
                labels=labels.astype(np.int32).reshape(H, W))


def round_fp16(x: np.ndarray) -> np.ndarray:
    """The oracle's FP16 store: nearest FP16 value, back to float32."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty_like(x)
    lib().orc_round_fp16(_p(x), _p(out), C.c_long(x.size))
    return out


def hbp(seg: dict, vol, wta, W, H, D, alpha=1000.1, tau_smooth=0.6, min_level=2, fp64=False,
        max_steps=-1, fp16_msg=False):
    """Returns (disparity HxW, plane HxWx3, steps, belief KxN, plane KxNx4).
    fp64 selects the FP64 oracle; fp16_msg the float path with FP16 message
    storage (min-normalised), as the engine's msg_fp16."""
    sizes = np.ascontiguousarray(seg["level_sizes"], np.int32)
    L = sizes.shape[0]
    disp = np.zeros((H, W), np.float32)
    plane = np.zeros((H, W, 3), np.float32)
    nmax = int(sizes[:, 0].max())
    sb = np.zeros(12 * nmax, np.float32)
    sp = np.zeros(12 * nmax * 4, np.float32)
    mean = np.ascontiguousarray(seg["mean"], np.float32).copy()
    steps = lib().orc_hbp(_p(sizes), L, _p(np.ascontiguousarray(seg["clus"], np.int32)), _p(mean),
                          _p(np.ascontiguousarray(seg["bd"], np.int32)),
                          _p(np.ascontiguousarray(seg["bdl"], np.int32)),
                          _p(np.ascontiguousarray(vol, np.uint8)), _p(np.ascontiguousarray(wta, np.float32)),
                          W, H, D, alpha, tau_smooth, min_level, 2 if fp16_msg else int(fp64), int(max_steps), _p(disp),
                          _p(plane), _p(sb), _p(sp))
    if steps < 0:
        raise ValueError("oracle hbp rejected its input")
    return disp, plane, steps, sb, sp


def hbp_lockstep(seg: dict, vol, wta, W, H, D, fp16_msg=False, shadow_fp64=True, alpha=1000.1,
                 tau_smooth=0.6, min_level=2):
    """The float run (the engine's arithmetic; FP16 message storage with
    fp16_msg) with a lock-step shadow that takes the same candidate planes
    and kept slots but carries costs, beliefs and messages in FP64
    (shadow_fp64=False: in float, which must repeat the run exactly).
    Returns (disparity, stats): over every message value of every BP step,
    each message minus its own minimum in both runs (a per-message constant
    changes no decision), msg_err_max / msg_err_mean of the difference and
    msg_ref_mean / msg_ref_max of the FP64 values; msg_raw_err_max / _mean of
    the stored values (each run normalised by its mode); values compared."""
    sizes = np.ascontiguousarray(seg["level_sizes"], np.int32)
    L = sizes.shape[0]
    disp = np.zeros((H, W), np.float32)
    st = np.zeros(7, np.float64)
    mean = np.ascontiguousarray(seg["mean"], np.float32).copy()
    steps = lib().orc_hbp_lockstep(_p(sizes), L, _p(np.ascontiguousarray(seg["clus"], np.int32)), _p(mean),
                                   _p(np.ascontiguousarray(seg["bd"], np.int32)),
                                   _p(np.ascontiguousarray(seg["bdl"], np.int32)),
                                   _p(np.ascontiguousarray(vol, np.uint8)),
                                   _p(np.ascontiguousarray(wta, np.float32)), W, H, D, alpha, tau_smooth,
                                   min_level, 2 if fp16_msg else 0, int(shadow_fp64), _p(disp), _p(st))
    if steps < 0:
        raise ValueError("oracle lock-step rejected its input")
    return disp, {"msg_err_max": float(st[0]), "msg_err_mean": float(st[1]), "msg_ref_mean": float(st[2]),
                  "msg_ref_max": float(st[6]), "msg_raw_err_max": float(st[4]),
                  "msg_raw_err_mean": float(st[5]), "values": int(st[3]), "steps": int(steps)}


def pipeline_lockstep(L, R, D, fp16_msg=False, shadow_fp64=True):
    """pipeline() with the lock-step FP64 shadow of hbp_lockstep."""
    H, W = L.shape[:2]
    cs = cost_stage(L, R, D)
    seg = segment(lab(L))
    return hbp_lockstep(seg, cs["vol"], cs["wta"], W, H, D, fp16_msg, shadow_fp64)


def lr_check(dispL, dispR, planeL):
    H, W = dispL.shape
    pl = np.ascontiguousarray(planeL, np.float32).copy()
    fail = np.zeros((H, W), np.uint8)
    lib().orc_lr_check(_p(np.ascontiguousarray(dispL, np.float32)), _p(np.ascontiguousarray(dispR, np.float32)),
                       _p(pl), W, H, _p(fail))
    return pl, fail


def plane_to_disp(plane):
    H, W = plane.shape[:2]
    d = np.zeros((H, W), np.float32)
    lib().orc_plane_to_disp(_p(np.ascontiguousarray(plane, np.float32)), W, H, _p(d))
    return d


def weighted_median(bgr, fail, plane, stable=True):
    H, W = fail.shape
    pl = np.ascontiguousarray(plane, np.float32).copy()
    lib().orc_weighted_median(_p(np.ascontiguousarray(bgr, np.uint8)), _p(np.ascontiguousarray(fail, np.uint8)),
                              _p(pl), W, H, int(stable))
    return pl


def weighted_median_gpu(bgr, fail, plane, wtab, z_mode=0):
    """PostProcess::median_filter_gpu (the reference's GPU variant); wtab holds the
    766 device patch weights expf(-k / 10)."""
    H, W = fail.shape
    pl = np.ascontiguousarray(plane, np.float32).copy()
    lib().orc_weighted_median_gpu(_p(np.ascontiguousarray(bgr, np.uint8)), _p(np.ascontiguousarray(fail, np.uint8)),
                                  _p(pl), W, H, _p(np.ascontiguousarray(wtab, np.float32)), int(z_mode))
    return pl


def driver_median(disp):
    d = np.ascontiguousarray(disp, np.float32).copy()
    H, W = d.shape
    lib().orc_driver_median(_p(d), W, H)
    return d


def cost_stage(L, R, D):
    """grey -> census -> volume/WTA for a BGR pair (the StereoCost Census path)."""
    gL, gR = grey_u8(L), grey_u8(R)
    cL, cR = census(gL), census(gR)
    vol, wta = cost_volume(cL, cR, D)
    return dict(greyL=gL, greyR=gR, censusL=cL, censusR=cR, vol=vol, wta=wta)


def cost_f32(src, tau=0.5, right=False):
    """The MC-CNN cost path on a float volume src [D][H][W]: (vol [D][H*W], wta HxW);
    right: the volume after cost_to_right."""
    src = np.ascontiguousarray(src, np.float32)
    D, H, W = src.shape
    vol = np.zeros((D, H * W), np.float32)
    wta = np.zeros((H, W), np.float32)
    f = lib().orc_cost_f32_right if right else lib().orc_cost_f32
    f(_p(src), W, H, D, tau, _p(vol), _p(wta))
    return vol, wta


def hbp_levels(seg, vol, wta, W, H, D, volf=None, tau=25.0, alpha=1000.1, tau_smooth=0.6, min_level=2,
               fp16_msg=False):
    """HBP_ISP::run_ms_vis without its superpixel image: (disp [L-m][H][W],
    plane [L-m][H][W][3]) from the top level down to min_level. vol is the
    uint8 volume [D][H*W], or None with volf the float one."""
    sizes = np.ascontiguousarray(seg["level_sizes"], np.int32)
    L = sizes.shape[0]
    n = L - min_level
    disp = np.zeros((n, H, W), np.float32)
    plane = np.zeros((n, H, W, 3), np.float32)
    vb = None if vol is None else np.ascontiguousarray(vol, np.uint8)
    vf = None if volf is None else np.ascontiguousarray(volf, np.float32)
    steps = lib().orc_hbp_levels(_p(sizes), L, _p(np.ascontiguousarray(seg["clus"], np.int32)),
                                 _p(np.ascontiguousarray(seg["mean"], np.float32)),
                                 _p(np.ascontiguousarray(seg["bd"], np.int32)),
                                 _p(np.ascontiguousarray(seg["bdl"], np.int32)), _p(vb), _p(vf),
                                 _p(np.ascontiguousarray(wta, np.float32)), W, H, D, tau, alpha, tau_smooth,
                                 min_level, 2 if fp16_msg else 0, _p(disp), _p(plane))
    if steps < 0:
        raise ValueError("orc_hbp_levels rejected its input")
    return disp, plane


def grey_f32(bgr):
    """img_BGR_to_grey: float grey image of a BGR uint8 image."""
    bgr = np.ascontiguousarray(bgr, np.uint8)
    out = np.zeros(bgr.shape[:-1], np.float32)
    lib().orc_grey_f32(_p(bgr), int(out.size), _p(out))
    return out


def cost_ad(L, R, D, tau=30.0, right=False):
    """The AD cost: (vol [D][H*W], wta HxW, greyL, greyR); right: after cost_to_right."""
    gL, gR = grey_f32(L), grey_f32(R)
    H, W = gL.shape
    vol = np.zeros((D, H * W), np.float32)
    wta = np.zeros((H, W), np.float32)
    lib().orc_cost_ad(_p(gL), _p(gR), W, H, D, tau, int(right), _p(vol), _p(wta))
    return vol, wta, gL, gR


def pipeline_ad(L, R, D, alpha=1000.1, tau_smooth=0.6, min_level=2, right_view=False):
    """The AD single-view path: AD cost, pyramid of the view's image, HBP (tau 30)."""
    H, W = L.shape[:2]
    vol, wta, _, _ = cost_ad(L, R, D, right=right_view)
    seg = segment(lab(R if right_view else L))
    disp, plane = hbp_f32(seg, vol, wta, W, H, D, 30.0, alpha, tau_smooth, min_level)
    return dict(disp=disp, plane=plane, vol=vol, wta=wta, seg=seg)


def hbp_f32(seg, volf, wta, W, H, D, tau=0.5, alpha=1.3, tau_smooth=0.6, min_level=2, fp64=False,
            fp16_msg=False):
    """HBP on a float cost volume [D][H*W] (the MC-CNN path): (disparity, plane)."""
    sizes = np.ascontiguousarray(seg["level_sizes"], np.int32)
    L = sizes.shape[0]
    disp = np.zeros((H, W), np.float32)
    plane = np.zeros((H, W, 3), np.float32)
    mean = np.ascontiguousarray(seg["mean"], np.float32)
    steps = lib().orc_hbp_f32(_p(sizes), L, _p(np.ascontiguousarray(seg["clus"], np.int32)), _p(mean),
                              _p(np.ascontiguousarray(seg["bd"], np.int32)),
                              _p(np.ascontiguousarray(seg["bdl"], np.int32)),
                              _p(np.ascontiguousarray(volf, np.float32)), _p(np.ascontiguousarray(wta, np.float32)),
                              W, H, D, tau, alpha, tau_smooth, min_level, 2 if fp16_msg else int(fp64), -1,
                              _p(disp), _p(plane), None, None)
    if steps < 0:
        raise ValueError("orc_hbp_f32 rejected its input")
    return disp, plane


def pipeline_f32(L, src, tau=0.5, alpha=1.3, tau_smooth=0.6, min_level=2, R=None):
    """The reference's MC-CNN single-view path (main_bench_middv3.cu:73-108 with
    cost "MC-CNN"): the volume ingest, the left image's pyramid and HBP. With
    the right image R: its right view (main_bench_middv3.cu:189-203)."""
    D, H, W = np.asarray(src).shape
    vol, wta = cost_f32(src, tau, right=R is not None)
    seg = segment(lab(L if R is None else R))
    disp, plane = hbp_f32(seg, vol, wta, W, H, D, tau, alpha, tau_smooth, min_level)
    return dict(disp=disp, plane=plane, vol=vol, wta=wta, seg=seg)


def pipeline(L, R, D, alpha=1000.1, tau_smooth=0.6, min_level=2, fp64=False, right_view=False,
             fp16_msg=False, link=2, num_nb=4, sigma=0.0, lab_image=None):
    """The single-pair path of main_stereo_hbp_isp.cu:33-72 (without the driver
    median); right_view selects the right-view path of main_bench_middv3.cu:189-203.
    link / num_nb / sigma: the SegHAC configuration; lab_image replaces the
    oracle's LAB of the segmented view (e.g. the engine's blurred LAB)."""
    H, W = L.shape[:2]
    cs = cost_stage(L, R, D)
    vol, wta = cs["vol"], cs["wta"]
    if right_view:
        vol, wta = cost_to_right(vol, W, H, D)
    img = R if right_view else L
    if lab_image is None:
        lab_image = lab(img) if sigma == 0 else lab_sigma(img, sigma)
    seg = segment(lab_image, link, num_nb)
    disp, plane, steps, _, _ = hbp(seg, vol, wta, W, H, D, alpha, tau_smooth, min_level, fp64,
                                   fp16_msg=fp16_msg)
    return dict(disp=disp, plane=plane, steps=steps, seg=seg, wta=wta, vol=vol)
