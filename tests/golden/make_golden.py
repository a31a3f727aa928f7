"""Generate the golden fixtures in tests/golden/ by running the reference's own
CUDA build (oracle/_ref/libhbpref.so, made by ``make -C oracle/ref``) on seeded
synthetic scenes. It needs a GPU; run it on a B200 box:

    python tests/golden/make_golden.py --out <dir> [--only census|mccnn|ad|seg|target|post_gpu|post_c1|lab_sweep]

and copy ``<dir>/*.npz`` into tests/golden/. The fixtures hold the reference's
outputs for every stage of the stereo path at small sizes (full arrays) and at
the 450x375, D=64 single-pair configuration (hashes, WTA, level-1 labels,
disparity). The reference library is only read here and by the GPU parity
tests; the product never loads it.
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "hbp-isp_b200"))
from scenes import make_scene, mccnn_like_volume  # noqa: E402

P = C.c_void_p


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(P)


class RefLib:
    """ctypes binding of oracle/ref/ref_harness.cu."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(ROOT, "oracle", "_ref", "libhbpref.so")
        self.lib = C.CDLL(path)
        for name in ("ref_grey", "ref_lab", "ref_1nn_grid", "ref_crtrees", "ref_cost",
                     "ref_segment", "ref_hbp_pair", "ref_post", "ref_hbp_f32", "ref_hbp_ad", "ref_lab_sigma",
                     "ref_segment_cfg", "ref_segment_target"):
            getattr(self.lib, name).restype = C.c_int
        self.lib.ref_hbp_pair.argtypes = [P, P, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                          C.c_int, C.c_int, P, P]
        self.lib.ref_lab_sigma.argtypes = [P, C.c_int, C.c_int, C.c_double, P]
        self.lib.ref_segment_cfg.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, P, P, P,
                                             P, P]
        self.lib.ref_segment_target.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                                P, P, P, P, P]
        self.lib.ref_hbp_ad.argtypes = [P, P, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int,
                                        P, P, P, P, P, P]
        self.lib.ref_hbp_f32.argtypes = [P, P, P, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int,
                                         C.c_int, P, P, P, P]

    def grey(self, bgr):
        H, W, _ = bgr.shape
        f = np.zeros((H, W), np.float32)
        u = np.zeros((H, W), np.uint8)
        rc = self.lib.ref_grey(ptr(bgr), W, H, ptr(f), ptr(u))
        assert rc == 0, rc
        return f, u

    def lab(self, bgr):
        H, W, _ = bgr.shape
        out = np.zeros((H, W, 4), np.float32)
        rc = self.lib.ref_lab(ptr(bgr), W, H, ptr(out))
        assert rc == 0, rc
        return out

    def nn_grid(self, lab4):
        H, W, _ = lab4.shape
        nn = np.zeros(H * W, np.int32)
        dmin = np.zeros(H * W, np.float32)
        d4 = np.full(H * W * 4, np.nan, np.float32)
        rc = self.lib.ref_1nn_grid(ptr(np.ascontiguousarray(lab4)), W, H, ptr(nn), ptr(dmin), ptr(d4))
        assert rc == 0, rc
        return nn, dmin, d4.reshape(H * W, 4)

    def crtrees(self, nn):
        nn = np.ascontiguousarray(nn, np.int32)
        clus = np.zeros_like(nn)
        n = self.lib.ref_crtrees(ptr(nn), len(nn), ptr(clus))
        assert n >= 0, n
        return clus, n

    def cost(self, L, R, D, to_right=False):
        H, W, _ = L.shape
        Da = (D + 31) // 32 * 32
        out = dict(
            greyL=np.zeros((H, W), np.uint8), greyR=np.zeros((H, W), np.uint8),
            censusL=np.zeros((H, W), np.uint32), censusR=np.zeros((H, W), np.uint32),
            vol_u8=np.zeros((H * W, Da), np.uint8), vol_f32=np.zeros((D, H * W), np.float32),
            wta=np.zeros((H, W), np.float32))
        rc = self.lib.ref_cost(ptr(L), ptr(R), W, H, D, int(to_right), ptr(out["greyL"]),
                               ptr(out["greyR"]), ptr(out["censusL"]), ptr(out["censusR"]),
                               ptr(out["vol_u8"]), ptr(out["vol_f32"]), ptr(out["wta"]))
        assert rc == 0, rc
        return out

    def segment(self, bgr):
        H, W, _ = bgr.shape
        n = H * W
        sizes = np.zeros(2 * 64, np.int32)
        clus = np.zeros(2 * n, np.int32)
        mean = np.zeros(12 * n, np.float32)
        bd = np.zeros(16 * n, np.int32)
        bdl = np.zeros(8 * n, np.int32)
        L = self.lib.ref_segment(ptr(bgr), W, H, 64, ptr(sizes), ptr(clus), ptr(mean), ptr(bd), ptr(bdl))
        assert L > 0, L
        sizes = sizes[: 2 * L].reshape(L, 2)
        tc, tb = int(sizes[:, 0].sum()), int(sizes[:, 1].sum())
        return dict(level_sizes=sizes, clus=clus[:tc], mean=mean[: 6 * tc], bd=bd[: 2 * tb].reshape(tb, 2),
                    bdl=bdl[:tb])

    def hbp_pair(self, L, R, D, alpha=1000.1, tau_smooth=0.6, min_level=2, right_view=False):
        H, W, _ = L.shape
        disp = np.zeros((H, W), np.float32)
        plane = np.zeros((H, W, 3), np.float32)
        levels = self.lib.ref_hbp_pair(ptr(L), ptr(R), W, H, D, alpha, tau_smooth, min_level,
                                       int(right_view), ptr(disp), ptr(plane))
        assert levels > 0, levels
        return disp, plane, levels

    def hbp_f32(self, L, R, src, alpha=1.3, tau_smooth=0.6, min_level=2, right_view=False):
        D, H, W = src.shape
        vol = np.zeros((D, H * W), np.float32)
        wta = np.zeros((H, W), np.float32)
        disp = np.zeros((H, W), np.float32)
        plane = np.zeros((H, W, 3), np.float32)
        levels = self.lib.ref_hbp_f32(ptr(L), ptr(R), ptr(np.ascontiguousarray(src, np.float32)), W, H, D,
                                      alpha, tau_smooth, min_level, int(right_view), ptr(vol), ptr(wta), ptr(disp),
                                      ptr(plane))
        assert levels > 0, levels
        return vol, wta, disp, plane, levels

    def hbp_ad(self, L, R, D, alpha=1000.1, tau_smooth=0.6, min_level=2, right_view=False):
        H, W, _ = L.shape
        out = dict(greyL=np.zeros((H, W), np.float32), greyR=np.zeros((H, W), np.float32),
                   vol=np.zeros((D, H * W), np.float32), wta=np.zeros((H, W), np.float32),
                   disp=np.zeros((H, W), np.float32), plane=np.zeros((H, W, 3), np.float32))
        levels = self.lib.ref_hbp_ad(ptr(L), ptr(R), W, H, D, alpha, tau_smooth, min_level, int(right_view),
                                     *(ptr(out[k]) for k in ("greyL", "greyR", "vol", "wta", "disp", "plane")))
        assert levels > 0, levels
        out["levels"] = levels
        return out

    def lab_sigma(self, bgr, sigma):
        H, W, _ = bgr.shape
        out = np.zeros((H, W, 4), np.float32)
        rc = self.lib.ref_lab_sigma(ptr(bgr), W, H, sigma, ptr(out))
        assert rc == 0, rc
        return out

    def segment_cfg(self, bgr, link, num_nb, sigma, target=1):
        H, W, _ = bgr.shape
        n = H * W
        sizes = np.zeros(2 * 64, np.int32)
        clus = np.zeros(2 * n, np.int32)
        mean = np.zeros(12 * n, np.float32)
        bd = np.zeros(4 * num_nb * n, np.int32)
        bdl = np.zeros(2 * num_nb * n, np.int32)
        L = self.lib.ref_segment_target(ptr(bgr), W, H, link, num_nb, sigma, target, 64, ptr(sizes), ptr(clus),
                                        ptr(mean), ptr(bd), ptr(bdl))
        assert L > 0, L
        sizes = sizes[: 2 * L].reshape(L, 2)
        tc, tb = int(sizes[:, 0].sum()), int(sizes[:, 1].sum())
        return dict(level_sizes=sizes, clus=clus[:tc], mean=mean[: 6 * tc], bd=bd[: 2 * tb].reshape(tb, 2),
                    bdl=bdl[:tb])

    def post(self, L, R, dispL, planeL, dispR, planeR, median=True):
        """LR check + fill; median: False none, True (1) the CPU weighted median,
        2 the GPU variant (median_filter_gpu)."""
        H, W, _ = L.shape
        dL, pL = dispL.copy(), planeL.copy()
        rc = self.lib.ref_post(ptr(L), ptr(R), W, H, ptr(dL), ptr(pL), ptr(np.ascontiguousarray(dispR)),
                               ptr(np.ascontiguousarray(planeR)), int(median))
        assert rc == 0, rc
        return dL, pL


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def random_graphs(seed: int = 4242):
    """Functional graphs (every node has exactly one successor) of several shapes."""
    rng = np.random.Generator(np.random.PCG64(seed))
    graphs = []
    for N in (1, 2, 3, 5, 8, 17, 64, 257, 1000, 4096):
        graphs.append(rng.integers(0, N, N).astype(np.int32))  # uniform successor
    for N in (10, 100, 1000):
        g = np.arange(1, N + 1, dtype=np.int32)  # one long chain ending in a self-loop
        g[-1] = N - 1
        graphs.append(g)
        graphs.append(np.zeros(N, np.int32))  # star into node 0
        perm = rng.permutation(N).astype(np.int32)  # a permutation: cycles only
        graphs.append(perm)
    for N in (500, 3000):
        # 1-NN graph of random points on a line with mutual-pair cycles and trees
        x = np.sort(rng.uniform(0, 1, N))
        left = np.r_[np.inf, np.diff(x)]
        right = np.r_[np.diff(x), np.inf]
        idx = np.arange(N)
        graphs.append(np.where(left < right, idx - 1, idx + 1).astype(np.int32))
    for N in (300, 2000):
        # random trees hanging on a few cycles of length 1..6
        g = np.empty(N, np.int32)
        k = 0
        while k < N:
            L = int(rng.integers(1, 7))
            L = min(L, N - k)
            g[k:k + L] = np.r_[np.arange(k + 1, k + L), k]
            k += L
            if k < N:
                m = min(int(rng.integers(5, 40)), N - k)
                g[k:k + m] = rng.integers(0, k, m)
                k += m
        graphs.append(g)
    return graphs


def random_lab(seed: int = 99) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    lab_rand = np.zeros((128, 192, 4), np.float32)
    lab_rand[..., 0] = rng.uniform(0, 100, (128, 192))
    lab_rand[..., 1:3] = rng.uniform(-90, 90, (128, 192, 2))
    lab_rand[..., 3] = 1
    lab_rand[40:60, 40:60, :3] = np.round(lab_rand[40:60, 40:60, :3])  # exact ties
    return lab_rand


def scene_record(ref: RefLib, W, H, D, seed, full: bool):
    s = make_scene(W, H, D, seed)
    L, R = s.left, s.right
    rec = dict(W=W, H=H, D=D, seed=seed, left=L, right=R)
    cost = ref.cost(L, R, D)
    costR = ref.cost(L, R, D, to_right=True)
    lab = ref.lab(L)
    nn, dmin, d4 = ref.nn_grid(lab)
    seg = ref.segment(L)
    n1 = int(seg["level_sizes"][0, 0])
    clus1 = seg["clus"][:n1]
    disp, plane, levels = ref.hbp_pair(L, R, D)
    dispR, planeR, levelsR = ref.hbp_pair(L, R, D, right_view=True)
    post_d, post_p = ref.post(L, R, disp, plane, dispR, planeR, median=True)
    lr_d, lr_p = ref.post(L, R, disp, plane, dispR, planeR, median=False)
    rec.update(
        sha_greyL=sha(cost["greyL"]), sha_greyR=sha(cost["greyR"]),
        sha_censusL=sha(cost["censusL"]), sha_censusR=sha(cost["censusR"]),
        sha_vol_u8=sha(cost["vol_u8"]), sha_vol_f32=sha(cost["vol_f32"]),
        sha_lab=sha(lab), sha_nn=sha(nn),
        wta=cost["wta"].astype(np.uint16), wta_right=costR["wta"].astype(np.uint16),
        sha_vol_right=sha(costR["vol_f32"]),
        level_sizes=seg["level_sizes"], clus1=clus1, sha_clus1=sha(clus1),
        disp=disp, disp_right=dispR, levels=levels, levels_right=levelsR,
        post_disp=post_d, lr_disp=lr_d,
    )
    if full:
        rec.update(
            greyL=cost["greyL"], greyR=cost["greyR"], censusL=cost["censusL"], censusR=cost["censusR"],
            lab=lab, nn=nn, dist_min=dmin,
            dist4=d4, seg_clus=seg["clus"], seg_mean=seg["mean"], seg_bd=seg["bd"], seg_bdl=seg["bdl"],
            plane=plane, plane_right=planeR, post_plane=post_p, lr_plane=lr_p,
        )
    return rec


MCCNN_CASES = [(96, 64, 32, 7, "mccnn_96x64_d32_s7"), (160, 120, 48, 11, "mccnn_160x120_d48_s11")]


def mccnn_record(ref: RefLib, W, H, D, seed):
    """The MC-CNN path on a seeded synthetic float volume (scenes.mccnn_like_volume
    with seed + 1; the tests regenerate it and check its hash)."""
    s = make_scene(W, H, D, seed)
    src = mccnn_like_volume(s, D, seed + 1)
    vol, wta, disp, plane, levels = ref.hbp_f32(s.left, s.right, src)
    volR, wtaR, dispR, planeR, levelsR = ref.hbp_f32(s.left, s.right, src, right_view=True)
    return dict(W=W, H=H, D=D, seed=seed, sha_src=sha(src), sha_vol_f32=sha(vol),
                wta=wta.astype(np.uint16), disp=disp, plane=plane, levels=levels,
                sha_vol_right=sha(volR), wta_right=wtaR.astype(np.uint16), disp_right=dispR,
                plane_right=planeR, levels_right=levelsR)


AD_CASES = [(96, 64, 32, 7, "ad_96x64_d32_s7"), (160, 120, 48, 11, "ad_160x120_d48_s11")]


def ad_record(ref: RefLib, W, H, D, seed):
    """The AD cost path on a seeded synthetic scene, both views."""
    s = make_scene(W, H, D, seed)
    a = ref.hbp_ad(s.left, s.right, D)
    b = ref.hbp_ad(s.left, s.right, D, right_view=True)
    return dict(W=W, H=H, D=D, seed=seed, sha_greyL=sha(a["greyL"]), sha_greyR=sha(a["greyR"]),
                sha_vol_f32=sha(a["vol"]), wta=a["wta"].astype(np.uint16), disp=a["disp"], plane=a["plane"],
                sha_vol_right=sha(b["vol"]), wta_right=b["wta"].astype(np.uint16), disp_right=b["disp"],
                levels=a["levels"], levels_right=b["levels"])


# (linkage, num_nb, sigma) of the segmentation variants; 0 Min, 1 Max,
# 2 Centroid, 3 Ward (segment.hpp:8-16)
SEG_CFGS = [(0, 4, 0.0), (1, 4, 0.0), (3, 4, 0.0), (2, 8, 0.0), (0, 8, 0.0), (2, 4, 1.0), (3, 8, 0.7)]


def seg_record(ref: RefLib, W, H, seed):
    """The segmentation variants on one seeded scene: every configuration's
    pyramid (full arrays) and the blurred LAB images."""
    s = make_scene(W, H, 32, seed)
    rec = dict(W=W, H=H, seed=seed, left=s.left, cfgs=np.array(SEG_CFGS, np.float64))
    for i, (link, nb, sigma) in enumerate(SEG_CFGS):
        seg = ref.segment_cfg(s.left, link, nb, sigma)
        for k, v in seg.items():
            rec[f"c{i}_{k}"] = v
    for sigma in sorted({c[2] for c in SEG_CFGS if c[2] > 0}):
        rec[f"lab_sigma_{sigma:g}"] = ref.lab_sigma(s.left, sigma)
    return rec


# SegHAC's superpixel mode: (linkage, num_nb, target_clus) on the seg scenes
TARGET_CFGS = [(2, 4, 7), (2, 4, 50), (2, 4, 300), (2, 4, 2000), (3, 8, 120), (0, 4, 40)]


def target_record(ref: RefLib, W, H, seed):
    """target_clus > 1: the pyramid (level sizes, the last level's clus) and
    the label image of each configuration."""
    s = make_scene(W, H, 32, seed)
    rec = dict(W=W, H=H, seed=seed, left=s.left, cfgs=np.array(TARGET_CFGS, np.int32))
    for i, (link, nb, target) in enumerate(TARGET_CFGS):
        seg = ref.segment_cfg(s.left, link, nb, 0.0, target)
        sizes = seg["level_sizes"]
        labels = np.arange(W * H)
        off = 0
        for l in range(sizes.shape[0]):
            labels = seg["clus"][off + labels]
            off += int(sizes[l, 0])
        rec[f"t{i}_level_sizes"] = sizes
        rec[f"t{i}_clus"] = seg["clus"]
        rec[f"t{i}_labels"] = labels.astype(np.int32).reshape(H, W)
    return rec


def post_c1_record(ref: RefLib):
    """Post-processing at the single-pair size (450x375, D 64, seed 1000): the
    reference's own HBP results of both views, then its LR check + fill, its
    weighted median (CPU variant) and its GPU variant, so that the tie order of
    the median is pinned on many failed pixels."""
    W, H, D, seed = 450, 375, 64, 1000
    s = make_scene(W, H, D, seed)
    L, R = s.left, s.right
    disp, plane, _ = ref.hbp_pair(L, R, D)
    dispR, planeR, _ = ref.hbp_pair(L, R, D, right_view=True)
    post_d, post_p = ref.post(L, R, disp, plane, dispR, planeR, median=True)
    lr_d, lr_p = ref.post(L, R, disp, plane, dispR, planeR, median=False)
    gpu_d, gpu_p = ref.post(L, R, disp, plane, dispR, planeR, median=2)
    return dict(W=W, H=H, D=D, seed=seed, left=L, right=R, disp=disp, plane=plane.astype(np.float32),
                disp_right=dispR, plane_right=planeR.astype(np.float32), lr_disp=lr_d, post_disp=post_d,
                post_gpu_disp=gpu_d, post_gpu_plane=gpu_p.astype(np.float32))


def post_gpu_record(ref: RefLib, golden_dir: str):
    """median_filter_gpu on the reference's own HBP results stored in the small
    fixtures (both views' disparities and planes), and the device patch weights."""
    w = np.zeros(766, np.float32)
    assert ref.lib.ref_patch_weights(ptr(w)) == 0
    rec = dict(patch_weights=w)
    for name in ("tiny_96x64_d32_s7", "small_160x120_d48_s11"):
        z = np.load(os.path.join(golden_dir, name + ".npz"))
        d, p = ref.post(z["left"], z["right"], z["disp"], z["plane"].astype(np.float32), z["disp_right"],
                        z["plane_right"].astype(np.float32), median=2)
        rec[name + "_disp"] = d
        rec[name + "_plane"] = p
    return rec


def all_colours() -> np.ndarray:
    """A 4096x4096 BGR image holding every 24-bit colour once (key = B | G << 8 | R << 16)."""
    c = np.arange(1 << 24, dtype=np.uint32)
    return np.stack([c & 255, (c >> 8) & 255, c >> 16], axis=1).astype(np.uint8).reshape(4096, 4096, 3)


def lab_sweep_record(ref: RefLib):
    """The reference build's LAB of all 2^24 colours: its hash, and the colours where
    the CPU oracle's LAB (the host's pow) differs, with the reference's values there
    (the oracle takes them as overrides)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O
    O.set_lab_overrides(np.zeros(0, np.uint32), np.zeros((0, 3), np.float32))  # the plain host pow
    img = all_colours()
    lab = ref.lab(img)
    mine = O.lab(img)
    diff = np.nonzero(np.any(lab.view(np.uint32) != mine.view(np.uint32), axis=2).ravel())[0]
    return dict(sha_lab_all=sha(lab), keys=diff.astype(np.uint32), vals=lab.reshape(-1, 4)[diff, :3].copy())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--lib", default=None)
    ap.add_argument("--only", choices=["census", "mccnn", "ad", "seg", "target", "post_gpu", "post_c1", "lab_sweep"],
                    default=None)
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    ref = RefLib(args.lib)

    if args.only in (None, "mccnn"):
        for (W, H, D, seed, name) in MCCNN_CASES:
            rec = mccnn_record(ref, W, H, D, seed)
            np.savez_compressed(os.path.join(args.out, name + ".npz"), **rec)
            print(name, "levels", rec["levels"])
    if args.only in (None, "ad"):
        for (W, H, D, seed, name) in AD_CASES:
            rec = ad_record(ref, W, H, D, seed)
            np.savez_compressed(os.path.join(args.out, name + ".npz"), **rec)
            print(name, "levels", rec["levels"])
    if args.only in (None, "seg"):
        # sizes a multiple of 16: the reference's blur races at a ragged edge
        for (W, H, seed, name) in [(96, 64, 7, "seg_96x64_s7"), (160, 112, 11, "seg_160x112_s11")]:
            rec = seg_record(ref, W, H, seed)
            np.savez_compressed(os.path.join(args.out, name + ".npz"), **rec)
            print(name, [int(rec[f"c{i}_level_sizes"].shape[0]) for i in range(len(SEG_CFGS))])
    if args.only in (None, "target"):
        for (W, H, seed, name) in [(96, 64, 7, "target_96x64_s7"), (160, 112, 11, "target_160x112_s11")]:
            rec = target_record(ref, W, H, seed)
            np.savez_compressed(os.path.join(args.out, name + ".npz"), **rec)
            print(name, [int(rec[f"t{i}_level_sizes"].shape[0]) for i in range(len(TARGET_CFGS))])
    if args.only in (None, "post_c1"):
        np.savez_compressed(os.path.join(args.out, "post_450x375_d64_s1000.npz"), **post_c1_record(ref))
        print("post_c1")
    if args.only in (None, "post_gpu"):
        # inputs: the reference's HBP results in the committed census fixtures
        src = os.path.dirname(os.path.abspath(__file__))
        np.savez_compressed(os.path.join(args.out, "post_gpu.npz"), **post_gpu_record(ref, src))
        print("post_gpu")
    if args.only in (None, "lab_sweep"):
        rec = lab_sweep_record(ref)
        np.savez_compressed(os.path.join(args.out, "lab_overrides.npz"), **rec)
        print("lab_sweep: colours where the host pow differs:", len(rec["keys"]))
    if args.only in ("mccnn", "ad", "seg", "target", "post_gpu", "post_c1", "lab_sweep"):
        return

    for (W, H, D, seed, full, name) in [
        (96, 64, 32, 7, True, "tiny_96x64_d32_s7"),
        (160, 120, 48, 11, True, "small_160x120_d48_s11"),
        (450, 375, 64, 1000, False, "c1_450x375_d64_s1000"),
    ]:
        rec = scene_record(ref, W, H, D, seed, full)
        np.savez_compressed(os.path.join(args.out, name + ".npz"), **rec)
        print(name, "levels", rec["levels"], rec["levels_right"], "sizes", rec["level_sizes"][:, 0].tolist())

    graphs = random_graphs()
    outs, nums = [], []
    for g in graphs:
        c, n = ref.crtrees(g)
        outs.append(c)
        nums.append(n)
    np.savez_compressed(os.path.join(args.out, "crtrees_graphs.npz"),
                        **{f"g{i}": g for i, g in enumerate(graphs)},
                        **{f"c{i}": c for i, c in enumerate(outs)}, nums=np.array(nums, np.int32))
    print("crtrees graphs", len(graphs), "clusters", nums)

    # Random LAB images exercise the pixel 1-NN distance arithmetic over a wide
    # range of values (used to pin the floating-point evaluation order).
    nn, dmin, d4 = ref.nn_grid(random_lab())
    # the random LAB image is regenerated from its seed by the tests
    np.savez_compressed(os.path.join(args.out, "nn_grid_random.npz"), nn=nn, dist_min=dmin, dist4=d4)
    print("done")


if __name__ == "__main__":
    main()
