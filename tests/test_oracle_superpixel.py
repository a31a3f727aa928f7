"""The oracle's restatement of SegHAC's superpixel mode (target_clus > 1,
get_target_clus, segment.cu:1016-1041) on the CPU; the GPU tests compare the
engine with it bit for bit and with the reference build's fixtures."""
import numpy as np
import pytest


@pytest.mark.parametrize("target", [2, 7, 50, 300, 5000, 19199])
def test_superpixel_mode_restatement(target):
    """The oracle's get_target_clus: exactly `target` superpixels labelled
    0..target-1 at the pyramid's last level, the level before it holds more
    than `target` clusters, and target 1 is the full pyramid."""
    import pyoracle as O
    from scenes import make_scene
    lab = O.lab(make_scene(160, 120, 48, 11).left)
    r = O.segment_target(lab, target)
    assert np.array_equal(np.unique(r["labels"]), np.arange(target))
    sizes = r["level_sizes"]
    assert sizes[-1, 0] > target
    top = r["clus"][int(sizes[:-1, 0].sum()):]
    assert top.max() == target - 1 and np.unique(top).size == target
    if target == 2:
        full, one = O.segment(lab), O.segment_target(lab, 1)
        for k in ("level_sizes", "clus", "mean", "bd", "bdl"):
            assert np.array_equal(full[k], one[k]), k


@pytest.mark.parametrize("name", ["target_96x64_s7", "target_160x112_s11"])
def test_superpixel_mode_against_reference(golden_dir, name):
    """The reference build's superpixels (make_golden.py --only target): the
    same level sizes and the same clus below the last level; at the last level
    the reference hands labels out with atomicSub in no fixed order, so the
    label images are compared as partitions (each oracle superpixel's majority
    reference superpixel) and must agree on >= 98% of the pixels."""
    import os
    import pyoracle as O
    z = dict(np.load(os.path.join(golden_dir, name + ".npz")))
    lab = O.lab(z["left"])
    for i, (link, nb, target) in enumerate(z["cfgs"].tolist()):
        o = O.segment_target(lab, target, link, nb)
        sizes = z[f"t{i}_level_sizes"]
        assert np.array_equal(o["level_sizes"], sizes), (name, i)
        n_last = int(sizes[-1, 0])
        assert np.array_equal(o["clus"][:-n_last], z[f"t{i}_clus"][:-n_last]), (name, i)
        ref = z[f"t{i}_labels"]
        pairs = o["labels"].astype(np.int64).ravel() * target + ref.astype(np.int64).ravel()
        cnt = np.bincount(pairs, minlength=target * target).reshape(target, target)
        assert cnt.max(axis=1).sum() / ref.size >= 0.98, (name, i)
