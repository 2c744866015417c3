"""The B200 chain with the non-default vertex clusterers of
PixelVertexProducerCUDA (pg_config.vertex_algo: 1 useDBSCAN, 2 useIterative)
against the oracle configured the same way, and against the reference's own
results (tests/golden/vertex_algos.npz).  Integers exact, floats within 1e-5
relative."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
RTOL = 1e-5
HERE = os.path.dirname(os.path.abspath(__file__))
VERTEX_PRODUCTS = ["nVertices", "zv", "wv", "vchi2", "ptv2", "ndof", "sortInd", "idv"]


def _run(det, raws, algo, max_events):
    import pixgpu
    c = pixgpu.Chain(det.es, max_events=max_events, max_words_per_batch=max_events * 300000, vertex_algo=algo)
    try:
        c.process(raws)
        return [c.products(k) for k in range(len(raws))]
    finally:
        c.close()


@pytest.mark.parametrize("algo", [1, 2])
def test_vertex_algo_chain_matches_oracle(default_detector, algo):
    import oracle
    raws = [default_detector.event(421 + k, pu) for k, pu in enumerate([20, 50, 35])]
    got = _run(default_detector, raws, algo, 4)
    orc = oracle.Oracle(default_detector.es, vertex_algo=algo)
    for k, raw in enumerate(raws):
        diffs = oracle.compare(orc.process(raw), got[k], rtol=RTOL)
        assert diffs == [], "event %d: %s" % (k, diffs[:3])


@pytest.mark.parametrize("algo,name", [(1, "dbscan"), (2, "iterative")])
def test_vertex_algo_chain_matches_reference_fixture(default_detector, algo, name):
    import oracle
    z = np.load(os.path.join(HERE, "golden", "vertex_algos.npz"))
    seed, pu = z["event"]
    got = _run(default_detector, [default_detector.event(int(seed), float(pu))], algo, 1)[0]
    want = {k: (int(z[name + "_" + k]) if z[name + "_" + k].ndim == 0 else z[name + "_" + k]) for k in VERTEX_PRODUCTS}
    assert oracle.compare(want, got, names=VERTEX_PRODUCTS, rtol=RTOL) == []


def test_vertex_algo_out_of_range_is_refused(default_detector):
    import pixgpu
    with pytest.raises(RuntimeError):
        pixgpu.Chain(default_detector.es, max_events=1, max_words_per_batch=300000, vertex_algo=3)
