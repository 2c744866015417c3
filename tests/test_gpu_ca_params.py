"""The B200 chain with each non-default switch of the CA module
(pg_config: min_hits_per_ntuplet, include_jumping_forward_doublets,
early/late_fishbone, ideal_conditions, do_cluster_cut, do_z0_cut, do_pt_cut;
CAHitNtupletGeneratorOnGPU.cc:46-58) against the oracle configured the same
way, and against the reference's own results (tests/golden/ca_params.npz).
Integers exact, floats within 1e-5 relative."""
import numpy as np
import pytest

from test_oracle_ca_params import PRODUCTS, VARIANTS, fixture_products, trimmed

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _run(det, raws, ca, max_events):
    import pixgpu
    c = pixgpu.Chain(det.es, max_events=max_events, max_words_per_batch=max_events * 300000, ca=ca)
    try:
        c.process(raws)
        return [c.products(k) for k in range(len(raws))]
    finally:
        c.close()


@pytest.mark.parametrize("name", sorted(VARIANTS) + ["late_on_early"])
def test_ca_params_chain_matches_oracle(default_detector, name):
    import oracle
    ca = VARIANTS.get(name, {"late_fishbone": 1})
    raws = [default_detector.event(441 + k, pu) for k, pu in enumerate([20, 50, 5])]
    got = _run(default_detector, raws, ca, 4)
    orc = oracle.Oracle(default_detector.es, ca=ca)
    for k, raw in enumerate(raws):
        diffs = oracle.compare(orc.process(raw), got[k], rtol=RTOL)
        assert diffs == [], "%s event %d: %s" % (name, k, diffs[:3])


@pytest.mark.parametrize("name", sorted(VARIANTS))
def test_ca_params_chain_matches_reference_fixture(default_detector, name):
    import oracle
    (seed, pu), want = fixture_products(name)
    got = _run(default_detector, [default_detector.event(seed, pu)], VARIANTS[name], 1)[0]
    assert oracle.compare(want, trimmed(got), names=list(PRODUCTS), rtol=RTOL) == []


@pytest.mark.parametrize("ca", [{"min_hits_per_ntuplet": 2}, {"min_hits_per_ntuplet": 5}, {"minhits": 4}])
def test_ca_params_out_of_range_are_refused(default_detector, ca):
    import pixgpu
    with pytest.raises((RuntimeError, ValueError)):
        pixgpu.Chain(default_detector.es, max_events=1, max_words_per_batch=300000, ca=ca)
