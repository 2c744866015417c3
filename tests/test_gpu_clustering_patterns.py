"""The B200 clusterizer (pg_cluster_digis: countModules, findClus and
clusterChargeCut on given digis) on the reference's own clustering test
patterns (src/serial/test/gpuClustering_t.h, tests/clustering_patterns.py)
and on the capacity edges of a module: every output equal to the oracle's,
and the reference test's checks hold.

Capacity edges (gpuClustering.h:88-92, gpuClusterChargeCut.h:46-59): a
module of more than 4000 pixels is clustered on its first 4000 (its
remaining pixels keep their initial index, which the cluster-count cap then
invalidates), and a module of more than 1024 clusters keeps the pixels of
its first 1024, the others set invalid."""
import numpy as np
import pytest

import clustering_patterns as cp

pytestmark = pytest.mark.gpu
FIELDS = ("moduleInd", "clus", "clusInModule", "moduleId", "moduleStart", "nModules")


@pytest.fixture(scope="module")
def chain(default_detector):
    import pixgpu
    c = pixgpu.Chain(default_detector.es, max_events=1, max_words_per_batch=600000)
    yield c
    c.close()


def _equal(want, got):
    for k in FIELDS:
        assert np.array_equal(np.asarray(want[k]), np.asarray(got[k])), k


@pytest.mark.parametrize("kn", range(5))
def test_reference_clustering_patterns(chain, default_detector, kn):
    import oracle
    ids, x, y, adc, _ = cp.patterns(kn)
    got = chain.cluster_digis(ids, x, y, adc)
    cp.reference_checks(ids, got)
    _equal(oracle.Oracle(default_detector.es).cluster_digis(ids, x, y, adc), got)
    assert got["flags"] == 0


def _isolated(module, n, charge=5000):
    rows, cols = np.meshgrid(np.arange(0, 160, 2), np.arange(0, 416, 2), indexing="ij")
    r, c = rows.ravel()[:n], cols.ravel()[:n]
    return (np.full(n, module, np.uint16), r.astype(np.uint16), c.astype(np.uint16), np.full(n, charge, np.uint16))


@pytest.mark.parametrize("n", [1100, 4500])
def test_module_capacity_edges(chain, default_detector, n):
    """n isolated pixels of charge above the threshold in one module, between
    two ordinary modules: 1100 clusters (the 1024-cluster cap) and 4500
    pixels (the 4000-pixel cap, then the cluster cap)."""
    import oracle
    import pixgpu
    parts = [_isolated(120, 30), _isolated(300, n), _isolated(500, 40)]
    ids, x, y, adc = (np.concatenate([p[i] for p in parts]) for i in range(4))
    got = chain.cluster_digis(ids, x, y, adc)
    _equal(oracle.Oracle(default_detector.es).cluster_digis(ids, x, y, adc), got)
    # the first 1024 clusters keep their pixels; the count itself is left as
    # found when every kept cluster passes the charge threshold (the charge
    # cut only renumbers when it removes one)
    kept = got["moduleInd"] == 300
    assert len(set(got["clus"][kept].tolist())) == 1024
    assert got["clusInModule"][300] == min(n, 4000)
    assert got["clusInModule"][120] == 30 and got["clusInModule"][500] == 40
    assert got["flags"] & pixgpu.PG_FLAG_MODULE_TOO_BIG  # both caps are reported
