"""The B200 chain (libpixgpu.so through its C ABI) against the golden
fixtures of the reference and against the CPU oracle.

Integers, indices and orderings (digis, clusters, hits sizes and iphi, phi
histogram, doublets, CA links, tuples, track lists, qualities, vertex
assignments) must be identical; floating-point products must agree within
1e-5 relative (the tolerance the fits and vertices are specified with).
"""
import numpy as np
import pytest

from conftest import golden_event, load_golden

pytestmark = pytest.mark.gpu
RTOL = 1e-5


@pytest.fixture(scope="module")
def chain(default_detector):
    import pixgpu
    c = pixgpu.Chain(default_detector.es, max_events=8, max_words_per_batch=8 * 200000)
    yield c
    c.close()


def _report(diffs):
    return "\n".join("%s: %s" % d for d in diffs)


@pytest.mark.parametrize("name", ["pu3", "pu8", "pu5_errors", "pu5_deadcols"])
def test_matches_reference_fixture(name, golden_meta, detectors):
    import oracle
    import pixgpu
    m = [x for x in golden_meta if x["name"] == name][0]
    det, raw = golden_event(m, detectors)
    c = pixgpu.Chain(det.es, max_events=1, max_words_per_batch=300000)
    try:
        c.process([raw])
        got = c.products(0)
    finally:
        c.close()
    diffs = oracle.compare(load_golden(name), got, rtol=RTOL)
    assert diffs == [], _report(diffs)


@pytest.mark.parametrize("seed,pu", [(11, 20), (12, 50), (13, 50)])
def test_matches_oracle(chain, default_detector, seed, pu):
    import oracle
    raw = default_detector.event(seed, pu)
    want = oracle.Oracle(default_detector.es).process(raw)
    chain.process([raw])
    got = chain.products(0)
    diffs = oracle.compare(want, got, rtol=RTOL)
    assert diffs == [], _report(diffs)


def test_matches_oracle_at_saturation(chain, default_detector):
    """This PU 75 event fills the 458752-doublet capacity and the 32768-tuple
    container; the last tuple is written and joins its cells' track lists
    before the finalize empties its bin, as in the reference."""
    import oracle
    raw = default_detector.event(105, 75)
    want = oracle.Oracle(default_detector.es).process(raw)
    assert want["nCells"] == 458752 and want["nTuples"] == 32767
    chain.process([raw])
    got = chain.products(0)
    diffs = oracle.compare(want, got, rtol=RTOL)
    assert diffs == [], _report(diffs)


def test_batch_results_equal_single_event_results(chain, default_detector):
    """Each event's products are the same alone and inside a mixed-PU batch."""
    import oracle
    raws = [default_detector.event(30 + k, pu) for k, pu in enumerate([5, 50, 20, 80, 1, 35])]
    chain.process(raws)
    mixed = [chain.products(k) for k in range(len(raws))]
    for k, raw in enumerate(raws):
        chain.process([raw])
        alone = chain.products(0)
        diffs = oracle.compare(alone, mixed[k], rtol=0.0)
        assert diffs == [], "event %d: %s" % (k, _report(diffs))


def test_empty_and_tiny_events(chain, default_detector):
    import oracle
    raws = [default_detector.event(50, 0), default_detector.event(51, 1)]
    chain.process(raws)
    orc = oracle.Oracle(default_detector.es)
    for k, raw in enumerate(raws):
        diffs = oracle.compare(orc.process(raw), chain.products(k), rtol=RTOL)
        assert diffs == [], _report(diffs)


@pytest.mark.parametrize("nhits,N", [(3, 3), (4, 4), (5, 4)])
def test_broken_line_fit_matches_oracle(chain, nhits, N):
    import oracle
    import pixgpu
    hits, ge, _ = pixgpu.fit_tuples(777 + nhits, 4096, nhits)
    want = oracle.Oracle(pixgpu.Detector().es).fit(N, hits, ge)
    got = chain.fit(N, hits, ge)
    for k in want:
        a, b = want[k].astype(np.float64), got[k].astype(np.float64)
        den = np.maximum(np.maximum(np.abs(a), np.abs(b)), 1e-30)
        rel = np.abs(a - b) / den
        assert rel.max() <= RTOL, (k, float(rel.max()))


def test_cut_margin_counts_match_oracle(default_detector):
    """Cut decisions on their float boundary (within four single-precision
    ulps), counted per event by the GPU chain and by the oracle over the same
    decisions: doublet cuts, CA cuts and classification cuts.  40 dense PU50
    events, one batch; the oracle finds 21 such decisions in them."""
    import oracle
    import pixgpu
    raws = [default_detector.event(pixgpu.BASE_SEED + 5000 + k, 50) for k in range(40)]
    c = pixgpu.Chain(default_detector.es, max_events=40, max_words_per_batch=sum(len(r) // 4 for r in raws) + 1024)
    try:
        c.process(raws)
        got = [c.counts(k) for k in range(len(raws))]
    finally:
        c.close()
    orc = oracle.Oracle(default_detector.es)
    total = 0
    for k, r in enumerate(raws):
        w = orc.process(r, list(oracle.CUT_MARGIN_COUNTS))
        want = (w["nCutMarginDoublets"], w["nCutMarginCA"], w["nCutMarginQuality"])
        have = (got[k]["n_cut_margin_doublets"], got[k]["n_cut_margin_ca"], got[k]["n_cut_margin_quality"])
        assert have == want, (k, have, want)
        total += sum(want)
    assert total > 0
