"""Seeded synthetic rectified stereo pairs (piecewise-planar Voronoi scenes).

The reference benchmarks on Middlebury V3 pairs (bench_MiddV3_train.sh:14-18,
main_bench_middv3.cu:50-130), which are not available here. These scenes stand
in for them with the same image sizes and a known ground truth:

* ``n_seg`` Voronoi sites drawn uniformly in the image; every pixel belongs to
  its nearest site (ties go to the lower site index).
* Each segment carries a disparity plane ``d = a*x + b*y + c`` with
  ``a, b ~ U[-0.05, 0.05]`` and ``c`` chosen so that the disparity at the site
  is ``U[lo, hi]``; disparities are clipped to ``[lo, hi] = [4, D - 4]``.
* Texture per segment: a base colour ``U[0, 255]^3``, Gaussian noise with
  sigma 8 per channel, and one sinusoid of amplitude 20 with a random
  orientation and a period ``U[4, 32]`` pixels; clamped to uint8, stored BGR
  (the reference reads ``.x`` as blue, imutil.cu:11-13, :129).
* The right image is a z-buffered forward warp of the left one
  (``xR = round(xL - d)``, the larger disparity wins); pixels of the right
  image that receive nothing are filled with uniform noise.
* Ground truth is the left disparity (float32) with a non-occlusion mask
  (left pixels that won the z-buffer of their target column).

All randomness comes from numpy's PCG64 generator seeded with ``seed``; the
conventional seeds are ``1000 + i`` for the i-th pair of a configuration.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

__all__ = ["Scene", "make_scene", "default_segments"]


@dataclass
class Scene:
    left: np.ndarray  # (H, W, 3) uint8, BGR
    right: np.ndarray  # (H, W, 3) uint8, BGR
    gt: np.ndarray  # (H, W) float32, left-view disparity
    nonocc: np.ndarray  # (H, W) bool, True where the left pixel is visible in the right view
    D: int
    seed: int

    @property
    def W(self) -> int:
        return self.left.shape[1]

    @property
    def H(self) -> int:
        return self.left.shape[0]


def default_segments(W: int, H: int) -> int:
    """Voronoi cell count per image size: 16 at 450x375, 24 up to 1080x744, 40 above."""
    if W * H <= 450 * 375:
        return 16
    if W * H <= 1080 * 744:
        return 24
    return 40


def _voronoi_labels(W: int, H: int, sites: np.ndarray) -> np.ndarray:
    ys, xs = np.mgrid[0:H, 0:W]
    best = np.full((H, W), np.inf, dtype=np.float64)
    lab = np.zeros((H, W), dtype=np.int32)
    for i, (sx, sy) in enumerate(sites):
        d2 = (xs - sx) ** 2 + (ys - sy) ** 2
        closer = d2 < best
        best[closer] = d2[closer]
        lab[closer] = i
    return lab


def make_scene(W: int, H: int, D: int, seed: int, n_seg: int | None = None) -> Scene:
    """Generate one synthetic pair of size ``W x H`` with disparity range ``D``."""
    if W < 16 or H < 16 or D < 16:
        raise ValueError("scene must be at least 16x16 with D >= 16")
    rng = np.random.Generator(np.random.PCG64(seed))
    n = default_segments(W, H) if n_seg is None else n_seg
    lo, hi = 4.0, float(D - 4)

    sites = np.stack([rng.uniform(0, W, n), rng.uniform(0, H, n)], axis=1)
    lab = _voronoi_labels(W, H, sites)

    a = rng.uniform(-0.05, 0.05, n)
    b = rng.uniform(-0.05, 0.05, n)
    d_site = rng.uniform(lo, hi, n)
    c = d_site - a * sites[:, 0] - b * sites[:, 1]
    base = rng.uniform(0, 255, (n, 3))
    theta = rng.uniform(0, np.pi, n)
    period = rng.uniform(4, 32, n)
    phase = rng.uniform(0, 2 * np.pi, n)

    ys, xs = np.mgrid[0:H, 0:W].astype(np.float64)
    gt = np.clip(a[lab] * xs + b[lab] * ys + c[lab], lo, hi)

    wave = 20.0 * np.sin(
        2 * np.pi * (xs * np.cos(theta[lab]) + ys * np.sin(theta[lab])) / period[lab] + phase[lab]
    )
    noise = rng.normal(0.0, 8.0, (H, W, 3))
    left_f = base[lab] + noise + wave[..., None]
    left = np.clip(np.rint(left_f), 0, 255).astype(np.uint8)

    # z-buffered forward warp: the larger disparity wins each right-image pixel.
    xr = np.rint(xs - gt).astype(np.int64)
    valid = (xr >= 0) & (xr < W)
    key = (ys.astype(np.int64) * W + xr)[valid]
    dval = gt[valid]
    src = np.flatnonzero(valid.ravel())
    zbuf = np.full(W * H, -np.inf)
    np.maximum.at(zbuf, key, dval)
    win = dval == zbuf[key]
    # among equal disparities the lower source index wins (deterministic)
    order = np.lexsort((src[win], key[win]))
    k_sorted = key[win][order]
    s_sorted = src[win][order]
    first = np.ones(k_sorted.size, dtype=bool)
    first[1:] = k_sorted[1:] != k_sorted[:-1]
    k_win, s_win = k_sorted[first], s_sorted[first]

    right = rng.integers(0, 256, (H * W, 3), dtype=np.uint8)
    right[k_win] = left.reshape(-1, 3)[s_win]
    nonocc = np.zeros(H * W, dtype=bool)
    nonocc[s_win] = True

    return Scene(
        left=np.ascontiguousarray(left),
        right=np.ascontiguousarray(right.reshape(H, W, 3)),
        gt=gt.astype(np.float32),
        nonocc=nonocc.reshape(H, W),
        D=D,
        seed=seed,
    )


def mccnn_like_volume(scene: Scene, D: int, seed: int) -> np.ndarray:
    """A float matching-cost volume [D][H][W] in [0, 1] standing in for an
    MC-CNN output (im0.acrt): the 5x5 mean of |grey_L(x) - grey_R(x - d)|
    (column 0 where x - d < 0) scaled by 1/48, plus Gaussian noise sigma 0.02,
    clipped to [0, 1]; seeded."""
    rng = np.random.Generator(np.random.PCG64(seed))
    w = np.array([0.114, 0.587, 0.299])
    gl = scene.left.astype(np.float64) @ w
    gr = scene.right.astype(np.float64) @ w
    H, W = gl.shape
    xs = np.arange(W)
    out = np.empty((D, H, W), np.float32)
    k = np.ones(5) / 5.0
    for d in range(D):
        diff = np.abs(gl - gr[:, np.maximum(xs - d, 0)])
        diff = np.apply_along_axis(lambda r: np.convolve(r, k, mode="same"), 1, diff)
        diff = np.apply_along_axis(lambda c: np.convolve(c, k, mode="same"), 0, diff)
        out[d] = diff / 48.0
    out += rng.normal(0.0, 0.02, out.shape)
    return np.clip(out, 0.0, 1.0).astype(np.float32)
