import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "pixeltrack-standalone_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def golden_meta():
    with open(os.path.join(GOLDEN, "events.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def detectors():
    import pixgpu
    cache = {}

    def get(seed, dead, badroc):
        key = (seed, dead, badroc)
        if key not in cache:
            cache[key] = pixgpu.Detector(seed, dead, badroc)
        return cache[key]
    return get


@pytest.fixture(scope="session")
def default_detector(detectors):
    import pixgpu
    return detectors(pixgpu.BASE_SEED, 0.0, 0.0)


def load_golden(name):
    import pixgpu
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    out = {k: (int(d[k]) if d[k].ndim == 0 else d[k]) for k in d.files}
    # the fixtures come from the reference's configuration, whose ErrorChecker
    # records no formatter errors
    out.setdefault("formatterErrors", np.zeros(0, dtype=pixgpu.FORMATTER_ERROR_DTYPE))
    return out


def golden_event(meta_entry, detectors):
    det = detectors(meta_entry["detector_seed"], meta_entry["dead_column_frac"], meta_entry["bad_roc_frac"])
    raw = det.event(meta_entry["event_seed"], meta_entry["pu"], inject_errors=meta_entry["inject_errors"])
    return det, raw
