"""Asynchronous batches, the device-resident pool and the serving loop.

The compact per-event result (loose tracks, their fits and vertex
assignment, vertices) must be identical whether an event is processed alone,
inside a batch, through the pool, or inside the continuous-batching serving
loop mixed with events of other pileup.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ["n_tracks", "n_loose_all", "n_vertices", "n_hits", "n_tuples", "n_digis", "n_cells", "flags", "tuple_index",
        "track_n_hits", "quality", "state", "cov", "pt", "eta", "chi2", "hits", "vertex", "zv", "wv", "vchi2", "ptv2",
        "ndof", "sort_ind"]


def same(a, b):
    bad = []
    for k in KEYS:
        x, y = a[k], b[k]
        if isinstance(x, np.ndarray):
            if x.shape != y.shape or not np.array_equal(x.view(np.uint8), y.view(np.uint8)):
                bad.append(k)
        elif x != y:
            bad.append(k)
    return bad


@pytest.fixture(scope="module")
def events(default_detector):
    pus = [50, 5, 30, 80, 20, 1, 60, 40]
    return [default_detector.event(500 + k, pu) for k, pu in enumerate(pus)]


@pytest.fixture(scope="module")
def alone(default_detector, events):
    """Per-event results, each event alone in a batch of one (plain launches, no graph)."""
    import pixgpu
    c = pixgpu.Chain(default_detector.es, max_events=1, max_words_per_batch=300000, use_graphs=False)
    out = []
    try:
        for r in events:
            s = c.submit([r])
            c.wait(s)
            out.append(c.result(s, 0))
            c.release(s)
    finally:
        c.close()
    return out


def test_result_matches_full_products(default_detector, events):
    """The packed result is the loose subset of the full track and vertex products."""
    import pixgpu
    c = pixgpu.Chain(default_detector.es, max_events=1, max_words_per_batch=300000)
    try:
        c.process([events[0]])
        full = {n: c.product(0, n) for n in ["quality", "state", "pt", "tupleOff", "tupleHits", "idv", "zv"]}
        s = c.submit([events[0]])
        c.wait(s)
        res = c.result(s, 0)
        c.release(s)
    finally:
        c.close()
    loose = np.nonzero(full["quality"] >= 2)[0]
    assert res["n_loose_all"] == len(loose)
    assert np.array_equal(res["tuple_index"], loose[:res["n_tracks"]])
    st = full["state"].reshape(-1, 5)
    assert np.array_equal(res["state"], st[loose])
    assert np.array_equal(res["pt"], full["pt"][loose])
    assert np.array_equal(res["vertex"], full["idv"][loose])
    assert np.array_equal(res["zv"], full["zv"])
    off = full["tupleOff"]
    for j, t in enumerate(loose[:50]):
        h = full["tupleHits"][off[t]:off[t + 1]]
        assert np.array_equal(res["hits"][j, :len(h)], h)


def test_batched_graph_equals_alone(default_detector, events, alone):
    import pixgpu
    c = pixgpu.Chain(default_detector.es, max_events=8, max_words_per_batch=8 * 300000, slots=2)
    try:
        s0 = c.submit(events[:5])
        s1 = c.submit(events[5:])
        assert s0 is not None and s1 is not None and s0 != s1
        assert c.submit(events[:1]) is None  # both slots busy
        c.wait(s1)
        c.wait(s0)
        for k in range(5):
            assert same(c.result(s0, k), alone[k]) == [], k
        for k in range(3):
            assert same(c.result(s1, k), alone[5 + k]) == [], k
        c.release(s0)
        c.release(s1)
    finally:
        c.close()


def test_pool_admission_and_gather(default_detector, events, alone):
    import pixgpu
    pool_words = 300000  # the smallest pool: room for a few events only
    c = pixgpu.Chain(default_detector.es, max_events=16, max_words_per_batch=16 * 300000, pool_words=pool_words)
    try:
        handles, refused = [], 0
        for j in range(16):
            k = j % len(events)
            h = c.pool_put(events[k])
            if h is None:
                refused += 1
            else:
                handles.append((k, h))
        assert refused > 0, "a 300k-word pool must refuse some of 16 events"
        info = c.pool_info()
        assert info["live_events"] == len(handles)
        s = c.submit_pooled([h for _, h in handles])
        c.wait(s)
        for j, (k, _) in enumerate(handles):
            assert same(c.result(s, j), alone[k]) == [], k
        c.release(s)
        info = c.pool_info()
        assert info["live_events"] == 0 and info["free_words"] == info["cap_words"]
        # a released handle cannot be submitted again
        with pytest.raises(RuntimeError):
            c.submit_pooled([handles[0][1]])
        h = c.pool_put(events[1])
        c.pool_release(h)
        assert c.pool_info()["live_events"] == 0
    finally:
        c.close()


def test_serving_abort_gives_back_the_pool(default_detector):
    """A request larger than a batch slot aborts the serving loop with
    PG_ERR_CAPACITY; the events admitted before it (waiting in the ready
    queue or refused with their batch) must leave the pool, so that the
    context stays usable."""
    import pixgpu
    small = [default_detector.event(700 + k, 3) for k in range(4)]
    big = default_detector.event(710, 50)
    assert len(big) // 4 > 40000 > max(len(r) for r in small) // 4
    c = pixgpu.Chain(default_detector.es, max_events=4, max_words_per_batch=40000, pool_words=600000)
    try:
        raws = small + [big]
        with pytest.raises(RuntimeError, match="larger than a batch slot"):
            c.serve(raws, n_requests=40, arrivals=np.linspace(0.0, 0.002, 40),
                    request_event=[k % 4 if k < 30 else 4 for k in range(40)])
        info = c.pool_info()
        assert info["live_events"] == 0 and info["free_words"] == info["cap_words"], info
        # the context serves again afterwards
        stats, lat = c.serve(small, n_requests=20, rate_hz=5000.0)
        assert stats["completed"] == 20
        info = c.pool_info()
        assert info["live_events"] == 0 and info["free_words"] == info["cap_words"], info
    finally:
        c.close()


@pytest.mark.parametrize("rate_hz", [2000.0, 200000.0])
def test_serving_results_same_alone_and_in_the_mix(default_detector, events, alone, rate_hz):
    """Continuous batching: results delivered by the serving loop equal the
    events processed alone, at a low rate (small batches) and a rate far above
    throughput (full batches, admission waits)."""
    import pixgpu
    c = pixgpu.Chain(default_detector.es, max_events=16, max_words_per_batch=16 * 300000, slots=3,
                     pool_words=4 * 1000 * 1000)
    n = 96
    rng = np.random.default_rng(7)
    req_event = rng.integers(0, len(events), n)
    got = {}

    def on_result(req, ev, res):
        got[req] = (ev, res)
    try:
        stats, lat = c.serve(events, n, rate_hz=rate_hz, request_event=req_event, on_result=on_result, seed=3)
    finally:
        c.close()
    assert stats["completed"] == n and len(got) == n
    for req, (ev, res) in got.items():
        assert ev == req_event[req]
        assert same(res, alone[ev]) == [], (req, ev)
    assert np.all(lat > 0)
    assert stats["p50_ms"] <= stats["p99_ms"] <= stats["max_ms"]
    assert stats["mean_batch"] >= 1.0
    if rate_hz > 100000:
        assert stats["max_batch_seen"] > 1


def test_mixed_pileup_batch_equals_alone(default_detector):
    """A batch of uneven events with pileup from 20 to 200 (the capacities
    saturate above ~PU80 and the events carry overflow flags): every event's
    result is the same inside the batch as alone."""
    import pixgpu
    pus = [20, 200, 120, 60, 180, 35, 90, 150]
    raws = [default_detector.event(700 + k, pu) for k, pu in enumerate(pus)]
    c1 = pixgpu.Chain(default_detector.es, max_events=1, max_words_per_batch=300000, use_graphs=False)
    alone = []
    try:
        for r in raws:
            s = c1.submit([r])
            c1.wait(s)
            alone.append(c1.result(s, 0))
            c1.release(s)
    finally:
        c1.close()
    c = pixgpu.Chain(default_detector.es, max_events=8, max_words_per_batch=8 * 300000)
    try:
        s = c.submit(raws)
        c.wait(s)
        for k in range(len(raws)):
            assert same(c.result(s, k), alone[k]) == [], (k, pus[k])
        assert any(c.result(s, k)["flags"] for k in range(len(raws)))  # the dense events do overflow
        c.release(s)
    finally:
        c.close()
