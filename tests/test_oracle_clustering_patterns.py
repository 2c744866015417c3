"""The oracle's clustering on the reference's own clustering test patterns
(tests/clustering_patterns.py, from src/serial/test/gpuClustering_t.h):
the test's checks after the charge cut hold for every variant."""
import pytest

import clustering_patterns as cp


@pytest.mark.parametrize("kn", range(5))
def test_oracle_passes_the_reference_clustering_checks(kn, default_detector):
    import oracle
    ids, x, y, adc, ncl = cp.patterns(kn)
    res = oracle.Oracle(default_detector.es).cluster_digis(ids, x, y, adc)
    cp.reference_checks(ids, res)
    # every generated cluster exists before the cut; after it the low ones are gone
    assert 0 < int(res["clusInModule"].sum()) <= ncl
