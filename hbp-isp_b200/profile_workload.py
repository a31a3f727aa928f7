"""Workloads for kernel profiles: each runs one stage family of the engine on
seeded synthetic scenes, so that a profiler (ncu -k <kernel> -c 1) captures a
launch of every kernel at a stated size. Nothing is timed or checked here.

    python hbp-isp_b200/profile_workload.py --workload pair --W 720 --H 496 --D 128
    python hbp-isp_b200/profile_workload.py --workload pair_lr ...     # + right view, LR check, weighted median
    python hbp-isp_b200/profile_workload.py --workload median_gpu ...  # median_filter_gpu variant
    python hbp-isp_b200/profile_workload.py --workload mccnn --W 1440 --H 992 --D 144
    python hbp-isp_b200/profile_workload.py --workload ad ...
    python hbp-isp_b200/profile_workload.py --workload segvar ...
    python hbp-isp_b200/profile_workload.py --workload noalloc ...

pair:        hbp_run_pair (post 1): grey/census/Hamming, LAB, 1-NN grid,
             CRTrees, the pyramid levels (radix sorts, scans, sums, 1-NN),
             BP setup, every BP kernel, the driver median.
pair_lr:     hbp_run_pair (post 2): the above for both views, then the LR
             check and fill and the weighted median (CPU order).
median_gpu:  the weighted median's GPU variant on the LR result of a pair.
mccnn:       the MC-CNN volume ingest (a synthetic float volume) and HBP on it.
ad:          the AD cost (float grey, AD volume) and HBP on it.
segvar:      SegHAC's other configurations on the left image: Min linkage,
             the 8-neighbour grid, the sigma = 1 pre-blur and 300 superpixels
             (target mode), then its label image and boundary picture.
noalloc:     the no-allocation driver median on a disparity map.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", required=True, choices=["pair", "pair_lr", "median_gpu", "mccnn", "ad", "segvar", "noalloc"])
    ap.add_argument("--W", type=int, default=720)
    ap.add_argument("--H", type=int, default=496)
    ap.add_argument("--D", type=int, default=128)
    ap.add_argument("--fp16", type=int, default=1)
    ap.add_argument("--seed", type=int, default=1000)
    a = ap.parse_args()
    import hbp_b200 as E
    from scenes import make_scene, mccnn_like_volume

    W, H, D = a.W, a.H, a.D
    s = make_scene(W, H, D, a.seed)
    ctx = E.Context(0, W * H, D)
    try:
        if a.workload in ("pair", "pair_lr"):
            prm = E.default_params(post=1 if a.workload == "pair" else 2, msg_fp16=a.fp16)
            ctx.run_pair(s.left, s.right, D, prm)
            return
        import torch
        dev = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
        prm = E.default_params(post=0, msg_fp16=a.fp16)
        if a.workload == "median_gpu":
            dL, dR = dev(s.left), dev(s.right)
            dispL = torch.zeros((H, W), device="cuda")
            dispR = torch.zeros_like(dispL)
            planeL = torch.zeros((H, W, 3), device="cuda")
            planeR = torch.zeros_like(planeL)
            cL = torch.zeros(H * W, dtype=torch.int32, device="cuda")
            cR = torch.zeros_like(cL)
            vol = torch.zeros(E.volume_bytes(W, H, D), dtype=torch.uint8, device="cuda")
            volR = torch.zeros_like(vol)
            wta = torch.zeros(H * W, device="cuda")
            wtaR = torch.zeros_like(wta)
            ctx.cost_census_d(dL, dR, W, H, D, cL, cR, vol, wta, volR, wtaR)
            ctx.segment_d(dL, W, H)
            ctx.infer_d(vol, wta, D, prm, dispL, planeL)
            ctx.segment_d(dR, W, H)
            ctx.infer_d(volR, wtaR, D, prm, dispR, planeR)
            fail = torch.zeros((H, W), dtype=torch.uint8, device="cuda")
            out = torch.zeros((H, W), device="cuda")
            ctx.lr_check_d(dispL, dispR, planeL, fail, out, W, H)
            ctx.weighted_median_gpu_d(dL, fail, planeL, out, W, H)
        elif a.workload == "segvar":
            img = dev(s.left)
            ctx.segment_target_d(img, W, H, 0, 8, 1.0, 300)
            labels = torch.zeros(H * W, dtype=torch.int32, device="cuda")
            ctx.segment_labels_d(labels)
            pic = torch.zeros(H * W * 3, dtype=torch.uint8, device="cuda")
            ctx.segment_draw_d(pic, 2, bgr=img)
        elif a.workload == "noalloc":
            disp = dev((np.random.default_rng(a.seed).random((H, W)) * D).astype(np.float32))
            E.driver_median_noalloc_d(disp, W, H)
        elif a.workload == "mccnn":
            src = dev(mccnn_like_volume(s, D, a.seed + 1).astype(np.float32))
            vol = torch.zeros(E.volume_f32_bytes(W, H, D) // 4, device="cuda")
            wta = torch.zeros(H * W, device="cuda")
            ctx.cost_f32_d(src, W, H, D, 0.5, vol, wta)
            ctx.segment_d(dev(s.left), W, H)
            disp = torch.zeros((H, W), device="cuda")
            p13 = E.default_params(post=0, msg_fp16=a.fp16, alpha=1.3)
            ctx.infer_f32_d(vol, wta, D, 0.5, p13, disp)
        else:  # ad
            dL, dR = dev(s.left), dev(s.right)
            gL = torch.zeros(H * W, device="cuda")
            gR = torch.zeros_like(gL)
            vol = torch.zeros(E.volume_f32_bytes(W, H, D) // 4, device="cuda")
            wta = torch.zeros(H * W, device="cuda")
            ctx.cost_ad_d(dL, dR, W, H, D, gL, gR, vol, wta)
            ctx.segment_d(dL, W, H)
            disp = torch.zeros((H, W), device="cuda")
            ctx.infer_f32_d(vol, wta, D, 30.0, prm, disp)
        torch.cuda.synchronize()
    finally:
        ctx.close()


if __name__ == "__main__":
    main()
