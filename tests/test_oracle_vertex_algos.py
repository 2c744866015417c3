"""The non-default vertex clusterers of PixelVertexProducerCUDA (useDBSCAN,
useIterative; gpuClusterTracksDBSCAN.h, gpuClusterTracksIterative.h) in the
oracle, against the reference's own serial chain configured the same way: the
committed fixture (tests/golden/make_golden_vertex_algos.py) and, where the
reference tree is present, fresh events."""
import os
import tempfile

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
VERTEX_PRODUCTS = ["nVertices", "zv", "wv", "vchi2", "ptv2", "ndof", "sortInd", "idv"]


@pytest.mark.parametrize("algo,name", [(1, "dbscan"), (2, "iterative")])
def test_vertex_algo_oracle_matches_reference_fixture(default_detector, algo, name):
    z = np.load(os.path.join(HERE, "golden", "vertex_algos.npz"))
    seed, pu = z["event"]
    raw = default_detector.event(int(seed), float(pu))
    got = oracle.Oracle(default_detector.es, vertex_algo=algo).process(raw, names=VERTEX_PRODUCTS)
    want = {k: (int(z[name + "_" + k]) if z[name + "_" + k].ndim == 0 else z[name + "_" + k])
            for k in VERTEX_PRODUCTS}
    assert oracle.compare(want, got, names=VERTEX_PRODUCTS, rtol=0.0) == []
    assert want["nVertices"] > 10


@pytest.mark.skipif(not oracle.ref_available(), reason="checker build of the reference not present")
@pytest.mark.parametrize("algo", [1, 2])
@pytest.mark.parametrize("seed,pu", [(411, 20), (412, 60)])
def test_vertex_algo_oracle_equals_reference(default_detector, algo, seed, pu):
    d = tempfile.mkdtemp()
    default_detector.write(d)
    raw = default_detector.event(seed, pu)
    want = oracle.Reference(d, vertex_algo=algo).process(raw)
    got = oracle.Oracle(default_detector.es, vertex_algo=algo).process(raw)
    assert oracle.compare(want, got, rtol=0.0) == []


def test_the_three_clusterers_differ(default_detector):
    raw = default_detector.event(413, 60)
    n = [oracle.Oracle(default_detector.es, vertex_algo=a).process(raw, names=["nVertices", "zv"]) for a in (0, 1, 2)]
    assert n[0]["nVertices"] != n[1]["nVertices"] or not np.array_equal(n[0]["zv"], n[1]["zv"])
