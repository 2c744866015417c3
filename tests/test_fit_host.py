"""The device Riemann-fit code compiled for the host (tests/host/fit_host.cc)
against the oracle: the FP64 kernel arithmetic restates the reference
operation by operation, so on the host, where both use the same math
library, the two agree to the last bit.  On the device only the
transcendental functions differ (tests/test_gpu_riemann.py).  The
mixed-precision variant is checked for finite results on tuples where
single-precision intermediates used to cancel."""
import ctypes
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = ("state", "cov", "pt", "eta", "chi2")


@pytest.fixture(scope="module")
def host_lib():
    out = os.path.join(tempfile.mkdtemp(), "libfithost.so")
    subprocess.run(["g++", "-std=c++17", "-O2", "-w", "-shared", "-fPIC", "-I",
                    os.path.join(ROOT, "pixeltrack-standalone_b200", "csrc"),
                    os.path.join(ROOT, "tests", "host", "fit_host.cc"), "-o", out], check=True)
    lib = ctypes.CDLL(out)
    lib.hf_fit_riemann.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint32] + [ctypes.c_void_p] * 2 + \
        [ctypes.c_double] + [ctypes.c_void_p] * 5
    return lib


def host_fit(lib, N, hits, ge, mixed):
    n = hits.shape[0]
    h = np.ascontiguousarray(hits[:, :N, :], dtype=np.float64)
    g = np.ascontiguousarray(ge[:, :N, :], dtype=np.float32)
    out = {"state": np.zeros((n, 5), np.float32), "cov": np.zeros((n, 15), np.float32),
           "pt": np.zeros(n, np.float32), "eta": np.zeros(n, np.float32), "chi2": np.zeros(n, np.float32)}
    assert lib.hf_fit_riemann(N, int(mixed), n, h.ctypes.data, g.ctypes.data, 0.0114256972711507,
                              *[out[k].ctypes.data for k in KEYS]) == 0
    return out


@pytest.mark.parametrize("nh,N", [(3, 3), (4, 4), (5, 4)])
def test_device_riemann_arithmetic_equals_oracle(host_lib, default_detector, nh, N):
    import pixgpu
    hits, ge, _ = pixgpu.fit_tuples(51 + nh, 20000, nh)
    got = host_fit(host_lib, N, hits, ge, False)
    want = oracle.Oracle(default_detector.es).fit(N, hits, ge, riemann=True)
    for k in KEYS:
        a, b = got[k], want[k]
        assert np.all((a == b) | (np.isnan(a) & np.isnan(b))), k


@pytest.mark.parametrize("nh,N,index", [(3, 3, 139459), (5, 4, 102442), (5, 4, 126818)])
def test_mixed_riemann_stays_finite_where_single_precision_cancels(host_lib, nh, N, index):
    """Tuples of the seeded sets of the mixed-precision test whose radial hit
    variance cancels to ~1e-16 in double precision (0 in single precision)."""
    import pixgpu
    hits, ge, _ = pixgpu.fit_tuples(4242 + nh, index + 1, nh)
    got = host_fit(host_lib, N, hits[index:], ge[index:], True)
    assert np.isfinite(got["state"]).all() and np.isfinite(got["pt"]).all()
