"""High-pileup events (the uneven-pileup batched and serving workloads reach
PU 200 and 250) through the chain with widened container capacities,
against the oracle with the same capacities: integers and orderings
identical, floats within 1e-5 relative, and no capacity flag on any event.
The reference treats its capacities as compile-time constants
(CAConstants.h:18-40); at its own values it truncates or overflows these
events."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
RTOL = 1e-5


@pytest.fixture(scope="module")
def wide_chain(default_detector):
    import pixgpu
    c = pixgpu.Chain(default_detector.es, max_events=2, max_words_per_batch=2 * 400000, caps=pixgpu.WIDE_CAPS)
    yield c
    c.close()


@pytest.mark.parametrize("pu", [100, 150, 200, 250])
def test_high_pileup_matches_wide_oracle(wide_chain, default_detector, pu):
    import oracle
    import pixgpu
    raw = default_detector.event(20261203 + 1000 + pu, pu, model="calibrated")
    want = oracle.Oracle(default_detector.es, caps=pixgpu.WIDE_CAPS).process(raw)
    wide_chain.process([raw])
    assert wide_chain.counts(0)["flags"] == 0
    got = wide_chain.products(0)
    diffs = oracle.compare(want, got, rtol=RTOL)
    assert diffs == [], "\n".join("%s: %s" % d for d in diffs)
    assert want["nTuples"] > 0 and want["nVertices"] > 0


def test_mixed_pileup_batch_with_wide_caps(wide_chain, default_detector):
    """Two events of very different pileup in one batch: each equals its own
    run alone (per-event offsets, no cross-talk through the wide strides)."""
    raws = [default_detector.event(501, 30, model="calibrated"), default_detector.event(502, 220, model="calibrated")]
    alone = []
    for r in raws:
        wide_chain.process([r])
        alone.append(wide_chain.products(0))
    wide_chain.process(raws)
    import oracle
    for k in range(2):
        diffs = oracle.compare(alone[k], wide_chain.products(k), rtol=0)
        assert diffs == [], (k, diffs[:3])
        assert wide_chain.counts(k)["flags"] == 0
