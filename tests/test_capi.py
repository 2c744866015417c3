"""The C-ABI libraries load on a CPU-only host and export every entry point
their headers declare (no device calls)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(p[gs]_[a-z_]+)\s*\(", text)))


@pytest.mark.parametrize("header,lib", [("pixgpu.h", "libpixgpu.so"), ("pixsynth.h", "libpixsynth.so")])
def test_exports(header, lib):
    import build
    path = os.path.join(ROOT, "pixeltrack-standalone_b200", "lib", lib)
    if not os.path.exists(path):
        build.build_all(gpu=(lib == "libpixgpu.so"))
    so = ctypes.CDLL(path)
    names = declared(header)
    assert len(names) >= 5
    missing = [n for n in names if not hasattr(so, n)]
    assert missing == []


@pytest.mark.gpu
@pytest.mark.parametrize("seed,pu,errors", [(7, 5, 3), (11, 50, 0)])
def test_unpack_matches_oracle_word_stream(default_detector, seed, pu, errors):
    """pg_unpack_raw (the product's host FED scan, called through the C ABI)
    gives the oracle FED loop's word stream and per-pair FED indices, on a
    clean PU50 event and on an event with injected raw-data errors.  A
    context needs a device, so this runs on the GPU box."""
    import ctypes
    import numpy as np
    import oracle
    import pixgpu
    raw = default_detector.event(seed, pu, inject_errors=errors)
    want = oracle.Oracle(default_detector.es)
    want.process(raw)
    ww = want._products(["fedWords", "fedWordFedIds"])
    c = pixgpu.Chain(default_detector.es, max_events=1, max_words_per_batch=300000)
    try:
        cap = 300000
        words = np.zeros(cap, np.uint32)
        fed = np.zeros(cap // 2 + 2, np.uint8)
        n = ctypes.c_uint32()
        rc = pixgpu.gpu_lib().pg_unpack_raw(c._h, raw, len(raw), words.ctypes.data, fed.ctypes.data, cap,
                                            ctypes.byref(n))
        assert rc == 0
    finally:
        c.close()
    assert n.value == len(ww["fedWords"]) > 0
    assert np.array_equal(words[:n.value], ww["fedWords"])
    assert np.array_equal(fed[:(n.value + 1) // 2], ww["fedWordFedIds"])
