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


def test_tuple_overflow_keeps_the_serial_prefix(default_detector):
    """An event with more tuples than the reference's 32768: with a tuple
    capacity that holds them all the chain equals the oracle (the n-tuplet
    write copies the tuples its count pass staged); at the reference's
    capacity the event overflows (the write searches a second time instead)
    and its stored tuples are the oracle's first 32767, as the reference
    keeps them (HistoContainer.h:193-204, bulkFinalizeFill)."""
    import oracle
    import pixgpu
    caps = {"tuples": 1 << 17, "multiplicity": 1 << 17, "hit_to_tuple": 1 << 20}
    raw = default_detector.event(20261203 + 7055, 55)  # dense model: ~412k doublets, ~34k tuples
    want = oracle.Oracle(default_detector.es, caps=caps).process(raw)
    assert want["nTuples"] > 32768 and want["nCells"] < 458752
    for ch_caps in (caps, None):
        ch = pixgpu.Chain(default_detector.es, max_events=1, max_words_per_batch=400000, caps=ch_caps)
        try:
            ch.process([raw])
            flags = ch.counts(0)["flags"]
            got = ch.products(0)
        finally:
            ch.close()
        if ch_caps:
            assert flags == 0
            diffs = oracle.compare(want, got, rtol=RTOL)
            assert diffs == [], "\n".join("%s: %s" % d for d in diffs)
        else:
            assert flags & pixgpu.PG_FLAG_TUPLE_OVERFLOW
            off = np.asarray(got["tupleOff"], np.int64)
            assert len(off) == 32768
            np.testing.assert_array_equal(off, np.asarray(want["tupleOff"], np.int64)[:32768])
            np.testing.assert_array_equal(np.asarray(got["tupleHits"])[:off[-1]],
                                          np.asarray(want["tupleHits"])[:off[-1]])
