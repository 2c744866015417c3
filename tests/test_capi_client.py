"""include/pixgpu.h and include/pixsynth.h as an integrator uses them: a C
client (tests/host/capi_client.c) is compiled as C99 and as C++17 against
the headers and linked against libpixgpu.so and libpixsynth.so.  On the CPU
it checks the calls that need no device; on the GPU it runs a seeded event
through the synchronous and the asynchronous API, and its counts must equal
the oracle's."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "pixeltrack-standalone_b200", "lib")


@pytest.fixture(scope="module", params=["c99", "c++17"])
def client(request, tmp_path_factory):
    import build
    for lib in ("libpixgpu.so", "libpixsynth.so"):
        if not os.path.exists(os.path.join(LIB, lib)):
            build.build_all(gpu=True)
    out = str(tmp_path_factory.mktemp("client") / "capi_client")
    src = os.path.join(ROOT, "tests", "host", "capi_client.c")
    if request.param == "c99":
        cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-Wno-missing-field-initializers"]
    else:
        cmd = ["g++", "-std=c++17", "-x", "c++", "-Wall", "-Werror"]
    cmd += ["-I", os.path.join(ROOT, "include"), src, "-x", "none", "-L", LIB, "-lpixgpu", "-lpixsynth",
            "-Wl,-rpath," + LIB, "-o", out]
    subprocess.run(cmd, check=True)
    return out


def test_client_cpu_calls(client):
    r = subprocess.run([client, "cpu"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith("cpu ok")


@pytest.mark.gpu
def test_client_runs_an_event(client, default_detector):
    import oracle
    import pixgpu
    r = subprocess.run([client, "gpu", "20"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    words, hits, cells, tuples, vertices, loose = map(int, r.stdout.split())
    raw = default_detector.event(pixgpu.BASE_SEED, 20)
    want = oracle.Oracle(default_detector.es).process(raw)
    assert (hits, cells, tuples, vertices) == (want["nHits"], want["nCells"], want["nTuples"], want["nVertices"])
    assert loose == int((want["quality"][:want["nTuples"]] >= 2).sum())
