"""The CPU oracle against the reference's serial chain compiled from its own
sources (oracle/_ref), on fresh seeded events.  Skipped where the reference
tree (and so the checker build) is absent."""
import os
import tempfile

import pytest

import oracle

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="checker build of the reference not present")


@pytest.fixture(scope="module")
def both(default_detector):
    d = tempfile.mkdtemp()
    default_detector.write(d)
    return oracle.Oracle(default_detector.es), oracle.Reference(d)


@pytest.mark.parametrize("seed,pu", [(101, 1), (102, 20), (103, 50)])
def test_oracle_equals_reference(both, default_detector, seed, pu):
    orc, ref = both
    raw = default_detector.event(seed, pu)
    assert oracle.compare(ref.process(raw), orc.process(raw), rtol=0.0) == []


def test_oracle_equals_reference_at_saturation(both, default_detector):
    """This PU 75 event fills the 458752-doublet capacity and the 32768-tuple
    container: the truncation order must match."""
    orc, ref = both
    raw = default_detector.event(105, 75)
    r = ref.process(raw)
    assert r["nCells"] == 458752 and r["nTuples"] == 32767
    assert oracle.compare(r, orc.process(raw), rtol=0.0) == []


def test_oracle_refuses_undefined_reference_behaviour(both, default_detector):
    """Seed 104 at PU 80 overflows the reference's TupleMultiplicity storage
    (a write past its bins, undefined behaviour); the oracle reports it."""
    orc, _ = both
    with pytest.raises(RuntimeError):
        orc.process(default_detector.event(104, 80))
