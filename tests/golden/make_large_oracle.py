"""Oracle fixtures at the benchmark configurations' sizes (CPU only):

    python tests/golden/make_large_oracle.py [--only NAME ...]

For each case it generates the seeded synthetic scene, runs the CPU oracle's
single-pair path (cost volume, pyramid, HBP at min_level 2, no post stage) in
the case's message mode, and records in ``tests/golden/large_oracle.json``:

* ``input_sha``: SHA-256 of the left and right images, so that a machine whose
  numpy produces a different scene (another SIMD path for sin/exp) is noticed;
* ``oracle_sha``: SHA-256 of the oracle's sources (oracle/*.cpp, *.h), so that
  a fixture made by an older oracle is noticed;
* ``disp_sha`` and a few summary figures of the oracle's disparity.

The GPU parity test (tests/test_gpu_large.py) compares the engine's disparity
hash with ``disp_sha`` when both input and oracle hashes match, and otherwise
runs the oracle itself. The oracle at 1440x992 takes minutes, which is why its
result is stored.
"""
from __future__ import annotations

import argparse
import glob
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "hbp-isp_b200"), os.path.join(ROOT, "oracle")]
OUT = os.path.join(HERE, "large_oracle.json")

# name: (W, H, D, seed, segments or None, fp16 messages)
CASES = {
    "c2_720x496_d128_s1000_fp32": (720, 496, 128, 1000, None, False),
    "c2_720x496_d128_s1000_fp16": (720, 496, 128, 1000, None, True),
    "c3_1080x744_d192_s1500_fp32": (1080, 744, 192, 1500, None, False),
    "c4_1440x992_d256_s4000_fp16": (1440, 992, 256, 4000, 40, True),
    "c4_1440x992_d256_s4000_fp32": (1440, 992, 256, 4000, 40, False),
}


def sha_arrays(*arrs) -> str:
    h = hashlib.sha256()
    for a in arrs:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def oracle_source_sha() -> str:
    h = hashlib.sha256()
    for f in sorted(glob.glob(os.path.join(ROOT, "oracle", "*.cpp")) +
                    glob.glob(os.path.join(ROOT, "oracle", "*.h"))):
        with open(f, "rb") as fh:
            h.update(os.path.basename(f).encode())
            h.update(fh.read())
    return h.hexdigest()


def scene_of(case):
    from scenes import make_scene
    W, H, D, seed, nseg, _ = case
    return make_scene(W, H, D, seed, nseg)


def oracle_disp(case, s):
    import pyoracle as O
    W, H, D, seed, nseg, fp16 = case
    return O.pipeline(s.left, s.right, D, fp16_msg=fp16)["disp"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*")
    a = ap.parse_args()
    table = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            table = json.load(f)
    src = oracle_source_sha()
    for name, case in CASES.items():
        if a.only and name not in a.only:
            continue
        s = scene_of(case)
        t0 = time.time()
        disp = oracle_disp(case, s)
        el = time.time() - t0
        table[name] = {"W": case[0], "H": case[1], "D": case[2], "seed": case[3], "segments": case[4],
                       "fp16": case[5], "input_sha": sha_arrays(s.left, s.right), "oracle_sha": src,
                       "disp_sha": sha_arrays(disp), "disp_mean": float(disp.mean()),
                       "disp_min": float(disp.min()), "disp_max": float(disp.max()),
                       "oracle_seconds": round(el, 1), "threads": os.cpu_count()}
        print(name, f"{el:.1f} s", table[name]["disp_mean"], flush=True)
        with open(OUT, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
