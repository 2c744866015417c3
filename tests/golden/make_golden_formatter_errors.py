"""Writes tests/golden/formatter_errors.npz: the digi and error products of
the reference's own serial chain (oracle/ref checker build) with the
ErrorChecker recording its framing errors, on one seeded PU2 event edited by
tests/faults.py (a framing fault on eight FEDs, RawToDigi error words of types
25-31 on two).  Needs the reference tree; run from the repository root:

    python tests/golden/make_golden_formatter_errors.py
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "pixeltrack-standalone_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(HERE))
import build  # noqa: E402
import pixgpu  # noqa: E402
import oracle  # noqa: E402
import faults  # noqa: E402

EVENT = (pixgpu.BASE_SEED + 461, 2)  # (seed, pile-up)
PRODUCTS = ("formatterErrors", "errors", "nDigis", "xx", "yy", "adc", "moduleInd", "rawIdArr", "nClusters",
            "nHits", "nTuples", "nVertices")


def main():
    build.build_synth()
    if build.build_ref() is None:
        raise SystemExit("the reference sources are needed to regenerate the fixture")
    det = pixgpu.Detector()
    d = tempfile.mkdtemp()
    det.write(d)
    raw = faults.faulted_event(det, *EVENT)
    p = oracle.Reference(d, formatter_errors=True).process(raw, names=list(PRODUCTS))
    arrays = {"event": np.array(EVENT, dtype=np.float64)}
    for k in PRODUCTS:
        arrays[k] = np.asarray(p[k])
    np.savez_compressed(os.path.join(HERE, "formatter_errors.npz"), **arrays)


if __name__ == "__main__":
    main()
