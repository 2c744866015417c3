"""Writes tests/golden/ca_params.npz: the track and vertex products of the
reference's own serial chain (oracle/ref checker build) with each
non-default switch of the CA module (CAHitNtupletGeneratorOnGPU.cc:46-58) on
one seeded PU10 event.  Needs the reference tree; run from the repository
root:

    python tests/golden/make_golden_ca_params.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "pixeltrack-standalone_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import build  # noqa: E402
import pixgpu  # noqa: E402
import oracle  # noqa: E402

EVENT = (pixgpu.BASE_SEED + 431, 10)  # (seed, pile-up)
PRODUCTS = ("nCells", "nTuples", "tupleOff", "tupleHits", "quality", "pt", "chi2", "nVertices", "zv")
# name -> the switches that differ from the reference's configuration
VARIANTS = {
    "quadruplets": {"min_hits_per_ntuplet": 4},
    "no_jumping": {"include_jumping_forward_doublets": 0},
    "late_fishbone": {"early_fishbone": 0, "late_fishbone": 1},
    "real_conditions": {"ideal_conditions": 0},
    "no_cluster_cut": {"do_cluster_cut": 0},
    "no_z0_cut": {"do_z0_cut": 0},
    "no_pt_cut": {"do_pt_cut": 0},
}


def main():
    build.build_synth()
    if build.build_ref() is None:
        raise SystemExit("the reference sources are needed to regenerate the fixture")
    det = pixgpu.Detector()
    d = tempfile.mkdtemp()
    det.write(d)
    raw = det.event(*EVENT)
    arrays = {"event": np.array(EVENT, dtype=np.float64)}
    for name, ca in VARIANTS.items():
        p = oracle.Reference(d, ca=ca).process(raw, names=list(PRODUCTS))
        n = int(p["tupleOff"][min(int(p["nTuples"]), len(p["tupleOff"]) - 1)])
        for k in PRODUCTS:
            v = np.asarray(p[k])
            if k == "tupleHits":
                v = v[:n]
            elif k in ("tupleOff",):
                v = v[:int(p["nTuples"]) + 1]
            elif k in ("quality", "pt", "chi2"):
                v = v[:int(p["nTuples"])]
            arrays[name + "_" + k] = v
    np.savez_compressed(os.path.join(HERE, "ca_params.npz"), **arrays)


if __name__ == "__main__":
    main()
