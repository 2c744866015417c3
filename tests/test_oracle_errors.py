"""The error paths of the raw-data unpacking in the oracle: the FED loop's
framing checks with the ErrorChecker recording them (PixelFormatterErrors:
CRC-modified, source id, trailer marker, fragment length; ErrorChecker.cc:38-91)
and RawToDigi's error words (types 25-31, 30 with state 1 as 40;
SiPixelRawToClusterGPUKernel.cc:188-339), against the reference's own serial
chain: the committed fixture (tests/golden/make_golden_formatter_errors.py)
and, where the reference tree is present, fresh events, bit for bit."""
import os
import tempfile

import numpy as np
import pytest

import faults
import oracle
import rawedit

HERE = os.path.dirname(os.path.abspath(__file__))


def fixture():
    z = np.load(os.path.join(HERE, "golden", "formatter_errors.npz"))
    seed, pu = z["event"]
    want = {k: (int(z[k]) if z[k].ndim == 0 else z[k]) for k in z.files if k != "event"}
    return (int(seed), float(pu)), want


def test_oracle_matches_reference_fixture(default_detector):
    (seed, pu), want = fixture()
    raw = faults.faulted_event(default_detector, seed, pu)
    got = oracle.Oracle(default_detector.es, formatter_errors=True).process(raw, names=list(want))
    assert oracle.compare(want, got, names=list(want), rtol=0.0) == []
    assert sorted(set(want["formatterErrors"]["errorType"].tolist())) == [32, 33, 34, 39]
    assert {25, 26, 27, 28, 29, 30, 31, 40} <= set(want["errors"]["errorType"].tolist())


def test_recording_changes_nothing_else(default_detector):
    raw = faults.faulted_event(default_detector, 462, 10)
    a = oracle.Oracle(default_detector.es).process(raw)
    b = oracle.Oracle(default_detector.es, formatter_errors=True).process(raw)
    assert len(a["formatterErrors"]) == 0 and len(b["formatterErrors"]) == 6
    a.pop("formatterErrors")
    b.pop("formatterErrors")
    assert oracle.compare(a, b, rtol=0.0) == []


def test_crc_modified_fed_is_dropped(default_detector):
    """A FED whose trailer has the CRC-modified bit contributes no words."""
    raw = default_detector.event(463, 5)
    feds = rawedit.parse(raw)
    w = list(feds[5][1])
    rawedit.crc_modified(w)
    edited = rawedit.build([(f, w if i == 5 else ws) for i, (f, ws) in enumerate(feds)])
    dropped = rawedit.build([(f, ws) for i, (f, ws) in enumerate(feds) if i != 5])
    orc = oracle.Oracle(default_detector.es)
    a = orc.process(edited)
    b = orc.process(dropped)
    assert a["nDigis"] < orc.process(raw)["nDigis"]
    assert oracle.compare(a, b, rtol=0.0) == []


def split_module_word(words):
    """A copy of the FED's first pixel word, to append after its other modules."""
    return next(x for x in rawedit.payload32(words) if x and (x >> 26) & 0x3f and ((x >> 21) & 0x1f) < 8)


@pytest.mark.parametrize("edit", ["overlap", "link0", "split"])
def test_oracle_refuses_undefined_reference_behaviour(default_detector, edit):
    """A FED whose trailer search runs into its header (negative payload
    length), a payload word of link 0 (a cabling index below the tables) and
    a module whose digis come in two runs (cluster counts and hit slots
    overwritten in loop order) are undefined in the reference; the oracle
    reports them."""
    feds = rawedit.parse(default_detector.event(464, 3))
    w = list(feds[9][1])
    if edit == "overlap":
        w = [w[0], w[-1] | (1 << 3), w[-1] | (1 << 3)]
    elif edit == "link0":
        rawedit.append_payload(w, [(0 << 26) | (1 << 21) | (5 << 8) | 7])
    else:
        rawedit.append_payload(w, [split_module_word(w)])
    raw = rawedit.build([(f, w if i == 9 else ws) for i, (f, ws) in enumerate(feds)])
    with pytest.raises(RuntimeError):
        oracle.Oracle(default_detector.es).process(raw)


@pytest.mark.skipif(not oracle.ref_available(), reason="checker build of the reference not present")
@pytest.mark.parametrize("formatter_errors", [False, True])
@pytest.mark.parametrize("seed,pu", [(465, 10), (466, 40)])
def test_oracle_equals_reference_on_faulted_events(default_detector, formatter_errors, seed, pu):
    d = tempfile.mkdtemp()
    default_detector.write(d)
    raw = faults.faulted_event(default_detector, seed, pu)
    want = oracle.Reference(d, formatter_errors=formatter_errors).process(raw)
    got = oracle.Oracle(default_detector.es, formatter_errors=formatter_errors).process(raw)
    assert oracle.compare(want, got, rtol=0.0) == []
