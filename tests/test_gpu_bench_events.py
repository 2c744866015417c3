"""The benchmark's own PU50 events, checked against the oracle: 64 of the 576
events bench.py times (every ninth), processed as one 64-event batch the way
the batched leg runs them.  Integers and orderings identical, floats within
1e-5 relative."""
import pytest

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def test_bench_events_match_oracle(default_detector):
    import concurrent.futures as cf
    import oracle
    import pixgpu
    ks = list(range(0, 576, 9))
    assert len(ks) == 64
    raws = [default_detector.event(pixgpu.BENCH_SEED_BASE + k, 50, model=pixgpu.BENCH_MODEL) for k in ks]
    c = pixgpu.Chain(default_detector.es, max_events=64, max_words_per_batch=sum(len(r) // 4 for r in raws) + 1024)
    try:
        c.process(raws)
        got = [c.products(j) for j in range(len(raws))]
        flags = [c.counts(j)["flags"] for j in range(len(raws))]
    finally:
        c.close()
    assert flags == [0] * len(raws)

    def check(j):
        want = oracle.Oracle(default_detector.es).process(raws[j])
        return j, oracle.compare(want, got[j], rtol=RTOL)
    with cf.ThreadPoolExecutor(max_workers=8) as ex:
        bad = [(ks[j], d[:3]) for j, d in ex.map(check, range(len(raws))) if d]
    assert bad == [], bad
