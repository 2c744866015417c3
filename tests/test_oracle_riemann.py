"""The Riemann-fit restatement of the oracle against the reference's own
Riemann fit: the committed fixture (tests/golden/make_golden_riemann.py) and,
where the reference tree is present, fresh seeded tuples through the checker
build.  Both sides take their 3x3 eigen-decompositions from the closed-form
solver of oracle/sym_eigen.h (the reference's comes from its un-vendored
linear-algebra dependency), so the pin covers every step but that one."""
import os

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
KEYS = ("state", "cov", "pt", "eta", "chi2")


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


@pytest.fixture(scope="module")
def orc(default_detector):
    return oracle.Oracle(default_detector.es)


@pytest.mark.parametrize("nh,N", [(3, 3), (4, 4), (5, 4)])
def test_riemann_oracle_matches_reference_fixture(orc, nh, N):
    z = np.load(os.path.join(HERE, "golden", "riemann_fits.npz"))
    key = "h%d" % nh
    got = orc.fit(N, z[key + "_hits"], z[key + "_ge"], riemann=True)
    for k in KEYS:
        assert _same(got[k], z[key + "_" + k]), k


@pytest.mark.skipif(not oracle.ref_available(), reason="checker build of the reference not present")
@pytest.mark.parametrize("nh,N,seed", [(3, 3, 31), (4, 4, 32), (5, 4, 33)])
def test_riemann_oracle_equals_reference(orc, nh, N, seed):
    import pixgpu
    hits, ge, _ = pixgpu.fit_tuples(seed, 5000, nh)
    got = orc.fit(N, hits, ge, riemann=True)
    want = oracle.ref_fit_riemann(N, hits, ge)
    for k in KEYS:
        assert _same(got[k], want[k]), k


def test_riemann_and_broken_line_agree_on_the_helix(orc):
    """Two fits of the same quadruplets: same helix within the errors."""
    import pixgpu
    hits, ge, _ = pixgpu.fit_tuples(34, 4000, 4)
    r = orc.fit(4, hits, ge, riemann=True)
    b = orc.fit(4, hits, ge)
    assert np.isfinite(r["state"]).all() and np.isfinite(r["cov"]).all()
    d = r["state"].astype(np.float64) - b["state"]
    sig = np.sqrt(r["cov"][:, [0, 5, 9, 12, 14]].astype(np.float64))
    assert np.median(np.abs(d) / sig, axis=0).max() < 0.5


@pytest.mark.skipif(not oracle.ref_available(), reason="checker build of the reference not present")
@pytest.mark.parametrize("seed,pu", [(201, 20), (202, 50)])
def test_riemann_chain_oracle_equals_reference(default_detector, seed, pu):
    """The whole chain with useRiemannFit: tracks and vertices of the oracle
    equal the reference's own serial chain configured the same way."""
    import tempfile
    d = tempfile.mkdtemp()
    default_detector.write(d)
    orc = oracle.Oracle(default_detector.es, riemann_fit=True)
    ref = oracle.Reference(d, riemann_fit=True)
    raw = default_detector.event(seed, pu)
    want = ref.process(raw)
    got = orc.process(raw)
    assert oracle.compare(want, got, rtol=0.0) == []
    # the fit choice reached both chains: the broken-line tracks differ
    bl = oracle.Oracle(default_detector.es).process(raw)
    assert not np.array_equal(bl["state"], got["state"])
