"""Writes the golden fixtures of tests/: the reference's own serial chain
(compiled from its sources by oracle/ref/Makefile) run on small seeded
synthetic events.  Needs the reference tree; run from the repository root:

    python tests/golden/make_golden.py

Outputs tests/golden/events.json (event recipes and raw-record digests) and
one compressed .npz of products per event.
"""
import hashlib
import json
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

# (name, detector seed, dead column fraction, bad ROC fraction, event seed, pile-up, error words)
EVENTS = [
    ("pu3", pixgpu.BASE_SEED, 0.0, 0.0, pixgpu.BASE_SEED + 0, 3, 0),
    ("pu8", pixgpu.BASE_SEED, 0.0, 0.0, pixgpu.BASE_SEED + 1, 8, 0),
    ("pu5_errors", pixgpu.BASE_SEED, 0.0, 0.0, pixgpu.BASE_SEED + 2, 5, 14),
    ("pu5_deadcols", pixgpu.BASE_SEED + 7, 0.002, 0.003, pixgpu.BASE_SEED + 3, 5, 0),
]


def main():
    build.build_synth()
    if build.build_ref() is None:
        raise SystemExit("the reference sources are needed to regenerate the fixtures")
    meta = []
    dets = {}
    for name, dseed, dead, badroc, seed, pu, nerr in EVENTS:
        key = (dseed, dead, badroc)
        if key not in dets:
            det = pixgpu.Detector(dseed, dead, badroc)
            d = tempfile.mkdtemp()
            det.write(d)
            dets[key] = (det, oracle.Reference(d))
        det, ref = dets[key]
        raw = det.event(seed, pu, inject_errors=nerr)
        prods = ref.process(raw)
        arrays = {k: (np.asarray(v) if not isinstance(v, int) else np.array(v, dtype=np.int64)) for k, v in prods.items()}
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
        meta.append({"name": name, "detector_seed": dseed, "dead_column_frac": dead, "bad_roc_frac": badroc,
                     "event_seed": seed, "pu": pu, "inject_errors": nerr,
                     "raw_sha256": hashlib.sha256(raw).hexdigest(), "raw_bytes": len(raw),
                     "es_sha256": [hashlib.sha256(b).hexdigest() for b in det.es],
                     "counts": {k: int(prods[k]) for k in oracle.PRODUCTS if isinstance(prods.get(k), int)}})
        print(name, meta[-1]["counts"])
    with open(os.path.join(HERE, "events.json"), "w") as f:
        json.dump(meta, f, indent=1)


if __name__ == "__main__":
    main()
