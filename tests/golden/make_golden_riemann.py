"""Writes tests/golden/riemann_fits.npz: the reference's own Riemann fit
(plugin-PixelTriplets/RiemannFit.h, compiled from its sources by
oracle/ref/Makefile with the linear-algebra subset of pixeltrack-standalone_b200/framework/compat/eigen) on
seeded synthetic 3-, 4- and 5-hit tuples (5-hit tuples are fitted on their
first 4 hits, as fit5as4 does).  Needs the reference tree; run from the
repository root:

    python tests/golden/make_golden_riemann.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "pixeltrack-standalone_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import build  # noqa: E402
import pixgpu  # noqa: E402
import oracle  # noqa: E402

CASES = [(3, 3, 9103), (4, 4, 9104), (5, 4, 9105)]  # (hits per tuple, hits fitted, seed)
PER_CASE = 128


def main():
    build.build_synth()
    if build.build_ref() is None:
        raise SystemExit("the reference sources are needed to regenerate the fixture")
    arrays = {}
    for nh, N, seed in CASES:
        hits, ge, _ = pixgpu.fit_tuples(seed, PER_CASE, nh)
        out = oracle.ref_fit_riemann(N, hits, ge)
        key = "h%d" % nh
        arrays[key + "_hits"] = hits
        arrays[key + "_ge"] = ge
        for k, v in out.items():
            arrays[key + "_" + k] = v
    np.savez_compressed(os.path.join(HERE, "riemann_fits.npz"), **arrays)


if __name__ == "__main__":
    main()
