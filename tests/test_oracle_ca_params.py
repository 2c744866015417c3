"""The CA module's non-default switches (CAHitNtupletGeneratorOnGPU.cc:46-58:
minHitsPerNtuplet, includeJumpingForwardDoublets, early/lateFishbone with the
fishbone cleaner, idealConditions, doClusterCut, doZ0Cut, doPtCut) in the
oracle, against the reference's own serial chain configured the same way: the
committed fixture (tests/golden/make_golden_ca_params.py) and, where the
reference tree is present, fresh events, bit for bit."""
import os
import tempfile

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "ca_params.npz")
PRODUCTS = ("nCells", "nTuples", "tupleOff", "tupleHits", "quality", "pt", "chi2", "nVertices", "zv")
VARIANTS = {
    "quadruplets": {"min_hits_per_ntuplet": 4},
    "no_jumping": {"include_jumping_forward_doublets": 0},
    "late_fishbone": {"early_fishbone": 0, "late_fishbone": 1},
    "real_conditions": {"ideal_conditions": 0},
    "no_cluster_cut": {"do_cluster_cut": 0},
    "no_z0_cut": {"do_z0_cut": 0},
    "no_pt_cut": {"do_pt_cut": 0},
}


def fixture_products(name):
    z = np.load(GOLDEN)
    out = {}
    for k in PRODUCTS:
        v = z[name + "_" + k]
        out[k] = int(v) if v.ndim == 0 else v
    return (int(z["event"][0]), float(z["event"][1])), out


def trimmed(p):
    """The fixture's view of a product set: the filled part of each tuple array."""
    nt = int(p["nTuples"])
    q = dict(p)
    q["tupleOff"] = p["tupleOff"][:nt + 1]
    q["tupleHits"] = p["tupleHits"][:int(q["tupleOff"][-1])]
    for k in ("quality", "pt", "chi2"):
        q[k] = p[k][:nt]
    return q


@pytest.mark.parametrize("name", sorted(VARIANTS))
def test_ca_params_oracle_matches_reference_fixture(default_detector, name):
    (seed, pu), want = fixture_products(name)
    got = oracle.Oracle(default_detector.es, ca=VARIANTS[name]).process(default_detector.event(seed, pu),
                                                                        names=list(PRODUCTS))
    assert oracle.compare(want, trimmed(got), names=list(PRODUCTS), rtol=0.0) == []


@pytest.mark.parametrize("name", sorted(VARIANTS))
def test_each_switch_changes_the_tracks(default_detector, name):
    (seed, pu), want = fixture_products(name)
    base = trimmed(oracle.Oracle(default_detector.es).process(default_detector.event(seed, pu), names=list(PRODUCTS)))
    assert oracle.compare(want, base, names=list(PRODUCTS), rtol=0.0) != []


def test_late_fishbone_marks_tracks_bad(default_detector):
    """Without the early fishbone, the late one kills cells after the n-tuplet
    search and the cleaner turns their tracks bad: the n-tuplets are those of
    no fishbone at all, with fewer good tracks.  On top of the early fishbone
    it finds nothing more to kill (its comparisons are a subset)."""
    raw = default_detector.event(433, 30)
    names = ["nTuples", "tupleHits", "quality"]
    none = oracle.Oracle(default_detector.es, ca={"early_fishbone": 0}).process(raw, names=names)
    late = oracle.Oracle(default_detector.es, ca={"early_fishbone": 0, "late_fishbone": 1}).process(raw, names=names)
    assert none["nTuples"] == late["nTuples"] and np.array_equal(none["tupleHits"], late["tupleHits"])
    assert int(np.count_nonzero(late["quality"] > 1)) < int(np.count_nonzero(none["quality"] > 1))
    early = oracle.Oracle(default_detector.es).process(raw, names=names)
    both = oracle.Oracle(default_detector.es, ca={"late_fishbone": 1}).process(raw, names=names)
    assert oracle.compare(early, both, names=names, rtol=0.0) == []


def test_invalid_ca_params_are_refused(default_detector):
    with pytest.raises(ValueError):
        oracle.Oracle(default_detector.es, ca={"min_hits_per_ntuplet": 5})
    with pytest.raises(ValueError):
        oracle.Oracle(default_detector.es, ca={"min_hits": 4})


@pytest.mark.skipif(not oracle.ref_available(), reason="checker build of the reference not present")
@pytest.mark.parametrize("name", sorted(VARIANTS) + ["late_on_early"])
@pytest.mark.parametrize("seed,pu", [(434, 20), (435, 50)])
def test_ca_params_oracle_equals_reference(default_detector, name, seed, pu):
    ca = VARIANTS.get(name, {"late_fishbone": 1})
    d = tempfile.mkdtemp()
    default_detector.write(d)
    raw = default_detector.event(seed, pu)
    want = oracle.Reference(d, ca=ca).process(raw)
    got = oracle.Oracle(default_detector.es, ca=ca).process(raw)
    assert oracle.compare(want, got, rtol=0.0) == []
