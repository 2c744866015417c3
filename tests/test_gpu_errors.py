"""The B200 chain on the raw-data error paths, with the FED scan on the host
and on the device (pg_config.fed_scan): the FED loop's framing errors
(pg_config.formatter_errors: the ErrorChecker's includeErrors) and RawToDigi's
error words against the oracle and the reference's fixture
(tests/golden/formatter_errors.npz); the device scan against the host scan on
plain batches; and the product's defined behaviour where the reference's is
undefined.  Integers exact, floats within 1e-5 relative."""
import numpy as np
import pytest

import faults
import rawedit
from test_oracle_errors import fixture

pytestmark = pytest.mark.gpu
RTOL = 1e-5
SCANS = ["host", "device"]


def _run(det, raws, max_events=4, **kw):
    import pixgpu
    c = pixgpu.Chain(det.es, max_events=max_events, max_words_per_batch=max_events * 300000, **kw)
    try:
        c.process(raws)
        return [c.products(k) for k in range(len(raws))], [c.counts(k) for k in range(len(raws))]
    finally:
        c.close()


@pytest.mark.parametrize("scan", SCANS)
@pytest.mark.parametrize("formatter_errors", [False, True])
def test_faulted_events_match_oracle(default_detector, scan, formatter_errors):
    import oracle
    raws = [faults.faulted_event(default_detector, 471, 10), faults.faulted_event(default_detector, 472, 40)]
    got, _ = _run(default_detector, raws, fed_scan=scan, formatter_errors=formatter_errors)
    orc = oracle.Oracle(default_detector.es, formatter_errors=formatter_errors)
    for k, raw in enumerate(raws):
        want = orc.process(raw)
        assert len(want["formatterErrors"]) == (6 if formatter_errors else 0)
        diffs = oracle.compare(want, got[k], rtol=RTOL)
        assert diffs == [], "event %d: %s" % (k, diffs[:3])


@pytest.mark.parametrize("scan", SCANS)
def test_faulted_event_matches_reference_fixture(default_detector, scan):
    import oracle
    (seed, pu), want = fixture()
    got, _ = _run(default_detector, [faults.faulted_event(default_detector, seed, pu)], max_events=1, fed_scan=scan,
                  formatter_errors=True)
    assert oracle.compare(want, got[0], names=list(want), rtol=RTOL) == []


def test_device_scan_equals_host_scan(default_detector):
    """Bit-identical products over a mixed batch with an empty record and an
    event without pixel FEDs."""
    import oracle
    raws = [default_detector.event(473 + k, pu) for k, pu in enumerate([50, 1, 20, 80])]
    raws += [b"\x00\x00\x00\x00", default_detector.event(478, 35)]
    host, _ = _run(default_detector, raws, max_events=8, fed_scan="host")
    dev, _ = _run(default_detector, raws, max_events=8, fed_scan="device")
    for k in range(len(raws)):
        assert oracle.compare(host[k], dev[k], rtol=0.0) == [], "event %d" % k
    assert host[4]["nDigis"] == 0


@pytest.mark.parametrize("scan", SCANS)
def test_inputs_undefined_in_the_reference(default_detector, scan):
    """A payload word of link 0 reads as padding (flagged PG_FLAG_BAD_INPUT);
    a FED whose trailer search reaches its header contributes no words.  The
    products equal the oracle's on the event with that word zeroed and that
    FED left out."""
    import oracle
    import pixgpu
    feds = rawedit.parse(default_detector.event(479, 8))
    w9 = list(feds[9][1])
    bad = (0 << 26) | (1 << 21) | (5 << 8) | 7
    rawedit.append_payload(w9, [bad, 0])
    w12 = list(feds[12][1])
    w12 = [w12[0], w12[-1] | (1 << 3), w12[-1] | (1 << 3)]
    raw = rawedit.build([(f, w9 if i == 9 else w12 if i == 12 else w) for i, (f, w) in enumerate(feds)])
    w9z = list(feds[9][1])
    rawedit.append_payload(w9z, [0, 0])
    ref_raw = rawedit.build([(f, w9z if i == 9 else w) for i, (f, w) in enumerate(feds) if i != 12])
    got, counts = _run(default_detector, [raw], max_events=1, fed_scan=scan)
    want = oracle.Oracle(default_detector.es).process(ref_raw)
    assert oracle.compare(want, got[0], rtol=RTOL) == []
    assert counts[0]["flags"] & pixgpu.PG_FLAG_BAD_INPUT


@pytest.mark.parametrize("scan", SCANS)
def test_split_module_keeps_its_first_run(default_detector, scan):
    """A module whose digis come in two runs: the later run reads as padding
    and the event is flagged PG_FLAG_SPLIT_MODULE; the products equal the
    oracle's on the event with that word zeroed."""
    import oracle
    import pixgpu
    from test_oracle_errors import split_module_word
    feds = rawedit.parse(default_detector.event(482, 8))
    w = list(feds[9][1])
    rawedit.append_payload(w, [split_module_word(w), 0])
    raw = rawedit.build([(f, w if i == 9 else ws) for i, (f, ws) in enumerate(feds)])
    wz = list(feds[9][1])
    rawedit.append_payload(wz, [0, 0])
    ref_raw = rawedit.build([(f, wz if i == 9 else ws) for i, (f, ws) in enumerate(feds)])
    got, counts = _run(default_detector, [raw], max_events=1, fed_scan=scan)
    assert oracle.compare(oracle.Oracle(default_detector.es).process(ref_raw), got[0], rtol=RTOL) == []
    assert counts[0]["flags"] & pixgpu.PG_FLAG_SPLIT_MODULE


def test_device_scan_refusals(default_detector):
    import pixgpu
    with pytest.raises(RuntimeError):  # the input pool stages on the host
        pixgpu.Chain(default_detector.es, max_events=1, max_words_per_batch=300000, fed_scan="device",
                     pool_words=1 << 20)
    c = pixgpu.Chain(default_detector.es, max_events=2, max_words_per_batch=100000, fed_scan="device")
    try:
        raws = [default_detector.event(480, 50), default_detector.event(481, 50)]
        with pytest.raises(RuntimeError):  # more words than the batch holds
            c.process(raws)
        c.process(raws[:1])
        assert c.product(0, "nDigis") > 0
    finally:
        c.close()
