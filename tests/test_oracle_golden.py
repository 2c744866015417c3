"""The CPU oracle against the golden fixtures made by the reference's own
serial chain (tests/golden/make_golden.py), and the generator's determinism."""
import hashlib

import pytest

from conftest import golden_event, load_golden


def test_generator_is_deterministic(golden_meta, detectors):
    for m in golden_meta:
        det, raw = golden_event(m, detectors)
        assert hashlib.sha256(raw).hexdigest() == m["raw_sha256"], m["name"]
        assert [hashlib.sha256(b).hexdigest() for b in det.es] == m["es_sha256"], m["name"]


@pytest.mark.parametrize("name", ["pu3", "pu8", "pu5_errors", "pu5_deadcols"])
def test_oracle_matches_reference_fixture(name, golden_meta, detectors):
    import oracle
    m = [x for x in golden_meta if x["name"] == name][0]
    det, raw = golden_event(m, detectors)
    got = oracle.Oracle(det.es).process(raw)
    want = load_golden(name)
    # the oracle restates the serial arithmetic operation by operation: exact
    assert oracle.compare(want, got, rtol=0.0) == []


def test_fixtures_cover_the_error_and_calibration_paths(golden_meta):
    assert len(load_golden("pu5_errors")["errors"]) == 14
    assert any(m["dead_column_frac"] > 0 for m in golden_meta)
    q = load_golden("pu8")["quality"]
    assert set(q.tolist()) == {0, 1, 2}
