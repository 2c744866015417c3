"""The allocation-free vertex entry point, for callers that cannot allocate
device memory where they need vertices (a per-event module inside a
framework that owns all device memory, where cudaFree would synchronise the
device).

pg_vertices_noalloc, given the chain's own track SoA, must return the
chain's vertices (pg_process_batch products), and on a track set of more
than 5500 vertex tracks -- large enough for the vertex kernel to work in the
static scratch instead of shared memory -- the serial vertex finder's
result.  Everything runs twice in a row, since every call reuses the same
static scratch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
RTOL = 1e-5
NAMES = ["tupleOff", "quality", "pt", "state", "cov", "idv", "zv", "wv", "vchi2", "ptv2", "ndof", "sortInd",
         "nVertices"]


@pytest.fixture(scope="module")
def chain_products(default_detector):
    import pixgpu
    events = [default_detector.event(900, 50), default_detector.event(901, 30)]
    c = pixgpu.Chain(default_detector.es, max_events=1, max_words_per_batch=300000)
    out = []
    try:
        for raw in events:
            c.process([raw])
            out.append({n: c.product(0, n) for n in NAMES})
    finally:
        c.close()
    return out


@pytest.fixture(scope="module")
def large_track_set(default_detector):
    """6000 four-hit loose tracks from 60 vertices, with the serial vertex finder's result."""
    import oracle
    rng = np.random.default_rng(5)
    n = 6000
    vz = rng.normal(0, 3.5, 60)
    z = (vz[rng.integers(0, 60, n)] + rng.normal(0, 0.004, n)).astype(np.float32)
    st = np.zeros((n, 5), np.float32)
    st[:, 4] = z
    cv = np.zeros((n, 15), np.float32)
    cv[:, 14] = (rng.uniform(0.002, 0.012, n) ** 2).astype(np.float32)
    tracks = {"tupleOff": (np.arange(n + 1) * 4).astype(np.uint32), "quality": np.full(n, 2, np.uint8),
              "pt": (0.5 + rng.exponential(1.0, n)).astype(np.float32), "state": st.ravel(), "cov": cv.ravel()}
    want = oracle.Oracle(default_detector.es).vertices(tracks["tupleOff"], tracks["quality"], tracks["pt"],
                                                       tracks["state"], tracks["cov"])
    want.update(tracks)
    return want


def _run(want):
    import torch
    import pixgpu
    dev = torch.device("cuda", 0)
    n = len(want["quality"])
    t = {k: torch.from_numpy(np.ascontiguousarray(want[k]).view(np.int32 if want[k].dtype == np.uint32
                                                                else want[k].dtype)).to(dev)
         for k in ("tupleOff", "quality", "pt", "state", "cov")}
    idv = torch.full((max(n, 1),), 12345, dtype=torch.int16, device=dev)
    out = {k: torch.zeros(1024, dtype=dt, device=dev) for k, dt in
           (("zv", torch.float32), ("wv", torch.float32), ("vchi2", torch.float32), ("ptv2", torch.float32),
            ("ndof", torch.int32))}
    sort_ind = torch.zeros(1024, dtype=torch.int16, device=dev)
    nv, _ = pixgpu.vertices_noalloc(t["tupleOff"], t["quality"], t["pt"], t["state"], t["cov"], idv, out["zv"],
                                   out["wv"], out["vchi2"], out["ptv2"], out["ndof"], sort_ind)
    assert nv == want["nVertices"], (nv, want["nVertices"])
    assert np.array_equal(idv.cpu().numpy()[:n], want["idv"])
    assert np.array_equal(out["ndof"].cpu().numpy()[:nv], want["ndof"])
    assert np.array_equal(sort_ind.cpu().numpy().view(np.uint16)[:nv], want["sortInd"])
    for k in ("zv", "wv", "vchi2", "ptv2"):
        np.testing.assert_allclose(out[k].cpu().numpy()[:nv], want[k], rtol=RTOL, atol=0, err_msg=k)


def test_noalloc_vertices_equal_chain_vertices_twice(chain_products):
    for call in range(2):
        for want in chain_products:
            _run(want)


def test_noalloc_large_track_set_twice(large_track_set):
    nh = np.diff(large_track_set["tupleOff"].astype(np.int64))
    assert int((nh >= 4).sum()) > 5500  # beyond the kernel's shared-memory size: the static scratch is used
    for call in range(2):
        _run(large_track_set)


def test_noalloc_rejects_too_many_tuples():
    """The C entry point refuses more tuples than its static scratch holds,
    and so does the Python wrapper, before any call."""
    import ctypes
    import torch
    import pixgpu
    dev = torch.device("cuda", 0)
    n = 32768
    z = lambda k, dt: torch.zeros(k, dtype=dt, device=dev)  # noqa: E731
    args = [z(n + 1, torch.int32), z(n, torch.uint8), z(n, torch.float32), z(5 * n, torch.float32),
            z(15 * n, torch.float32), z(n, torch.int16), z(1024, torch.float32), z(1024, torch.float32),
            z(1024, torch.float32), z(1024, torch.float32), z(1024, torch.int32), z(1024, torch.int16)]
    with pytest.raises(ValueError, match="32767"):
        pixgpu.vertices_noalloc(*args)
    nv, fl = ctypes.c_uint32(), ctypes.c_uint32()
    msg = ctypes.create_string_buffer(256)
    ptrs = [t.data_ptr() for t in args]
    rc = pixgpu.gpu_lib().pg_vertices_noalloc(*ptrs[:5], n, *ptrs[5:], ctypes.addressof(nv), ctypes.addressof(fl),
                                               torch.cuda.current_stream(dev).cuda_stream, msg, len(msg))
    assert rc != 0 and b"32767" in msg.value


def test_noalloc_wrapper_checks_its_tensors():
    """Short outputs, wrong dtypes and host tensors are refused before the call."""
    import torch
    import pixgpu
    dev = torch.device("cuda", 0)
    n = 10
    z = lambda k, dt, d=dev: torch.zeros(k, dtype=dt, device=d)  # noqa: E731
    good = [z(n + 1, torch.int32), z(n, torch.uint8), z(n, torch.float32), z(5 * n, torch.float32),
            z(15 * n, torch.float32), z(n, torch.int16), z(1024, torch.float32), z(1024, torch.float32),
            z(1024, torch.float32), z(1024, torch.float32), z(1024, torch.int32), z(1024, torch.int16)]
    for k, bad in ((6, z(100, torch.float32)), (0, z(n, torch.int32)), (5, z(n - 1, torch.int16)),
                   (2, z(n, torch.float64)), (3, z(5 * n, torch.float32, "cpu"))):
        args = list(good)
        args[k] = bad
        with pytest.raises(ValueError):
            pixgpu.vertices_noalloc(*args)
