"""The B200 Riemann fit (pg_fit_riemann) against the oracle's Riemann fit
and the reference's own results (tests/golden/riemann_fits.npz).

Tolerance: 1e-5 relative on every output.  The device and the host differ
only in the last bits of their transcendental functions; the single-precision
rounding inside the numerical eigenvector Jacobian (RiemannFit.h:328-334)
could turn such a difference into a relative change of ~1e-3 of a circle
covariance term, with a probability of ~1e-7 per tuple, so a covariance term
is allowed to differ beyond 1e-5 in at most one tuple in 10^4.

For a triplet the circle passes through the three points and its chi2 is
the rounding residue of a zero eigenvalue (below 5e-8 on these tuples, on
host and device alike), so the chi2 of a triplet fit is compared at 1e-5
relative or 2e-7 absolute."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
RTOL = 1e-5


@pytest.fixture(scope="module")
def chain(default_detector):
    import pixgpu
    c = pixgpu.Chain(default_detector.es, max_events=1, max_words_per_batch=300000)
    yield c
    c.close()


def _rel(a, b):
    a, b = a.astype(np.float64), b.astype(np.float64)
    both_nan = np.isnan(a) & np.isnan(b)
    den = np.maximum(np.maximum(np.abs(a), np.abs(b)), 1e-30)
    return np.where(both_nan, 0.0, np.abs(a - b) / den)


def _check(got, want, n, N):
    for k in ("state", "pt", "eta", "chi2"):
        r = _rel(got[k], want[k])
        if k == "chi2" and N == 3:
            r = np.where(np.abs(got[k].astype(np.float64) - want[k]) <= 2e-7, 0.0, r)
        assert np.nanmax(r) <= RTOL, (k, float(np.nanmax(r)))
    # covariance: relative to the diagonal scale of its row and column
    c, w = got["cov"].astype(np.float64), want["cov"].astype(np.float64)
    diag = [0, 5, 9, 12, 14]
    idx = [(i, j) for i in range(5) for j in range(i, 5)]
    scale = np.zeros_like(w)
    for k, (i, j) in enumerate(idx):
        scale[:, k] = np.sqrt(np.abs(w[:, diag[i]] * w[:, diag[j]]))
    r = np.abs(c - w) / np.maximum(scale, 1e-30)
    bad = (r > RTOL).any(axis=1).sum()
    assert bad <= max(1, n // 10000), (int(bad), float(r.max()))


@pytest.mark.parametrize("nhits,N", [(3, 3), (4, 4), (5, 4)])
def test_riemann_fit_matches_oracle(chain, default_detector, nhits, N):
    import oracle
    import pixgpu
    hits, ge, _ = pixgpu.fit_tuples(4711 + nhits, 8192, nhits)
    want = oracle.Oracle(default_detector.es).fit(N, hits, ge, riemann=True)
    got = chain.fit(N, hits, ge, riemann=True)
    _check(got, want, len(hits), N)


@pytest.mark.parametrize("nhits,N", [(3, 3), (4, 4), (5, 4)])
def test_riemann_fit_matches_reference_fixture(chain, nhits, N):
    z = np.load(os.path.join(HERE, "golden", "riemann_fits.npz"))
    key = "h%d" % nhits
    got = chain.fit(N, z[key + "_hits"], z[key + "_ge"], riemann=True)
    want = {k: z[key + "_" + k] for k in ("state", "cov", "pt", "eta", "chi2")}
    _check(got, want, len(z[key + "_pt"]), N)


def test_riemann_fit_rejects_other_multiplicities(chain):
    import pixgpu
    hits, ge, _ = pixgpu.fit_tuples(5, 16, 5)
    with pytest.raises(RuntimeError):
        chain.fit(5, hits, ge, riemann=True)


# Mixed-precision Riemann fit against the FP64 one on the same tuples.
# Measured on 200k seeded tuples per multiplicity (maxima unless rms):
# triplets |d(1/pT)| 0, |d phi| 0, |d d0| 2e-9 cm (the circle through three
# points is the FP64 one), cot(theta) rms 2e-5, z0 rms 2e-4 cm; quadruplets
# |d(1/pT)| 1.2e-6 /GeV, |d phi| 2.4e-7, |d d0| 4e-8 cm, cot(theta) rms 4e-6,
# z0 rms 1.1e-5 cm.  The bounds leave a margin of ~10.
MIXED_BOUNDS = {  # nhits: (max |d 1/pT|, max |d phi|, max |d d0|, rms d cot, rms d z0)
    3: (1e-6, 1e-6, 1e-6, 5e-4, 5e-3),
    4: (2e-5, 5e-6, 1e-6, 5e-5, 2e-4),
    5: (2e-5, 5e-6, 1e-6, 5e-5, 2e-4),
}


@pytest.mark.parametrize("nhits,N", [(3, 3), (4, 4), (5, 4)])
def test_mixed_riemann_fit_within_bounds_of_fp64(chain, nhits, N):
    import pixgpu
    hits, ge, _ = pixgpu.fit_tuples(4343 + nhits, 20000, nhits)
    a = chain.fit(N, hits, ge, riemann=True)
    b = chain.fit(N, hits, ge, mixed=True, riemann=True)
    sa, sb = a["state"].astype(np.float64), b["state"].astype(np.float64)
    assert np.isfinite(sb).all() and np.isfinite(b["pt"]).all()
    dk = np.abs(1.0 / b["pt"].astype(np.float64) - 1.0 / a["pt"].astype(np.float64))
    d = np.abs(sb - sa)
    mk, mphi, md0, rcot, rz0 = MIXED_BOUNDS[nhits]
    assert dk.max() < mk, dk.max()
    assert d[:, 0].max() < mphi, d[:, 0].max()
    assert d[:, 1].max() < md0, d[:, 1].max()
    assert np.sqrt((d[:, 3] ** 2).mean()) < rcot
    assert np.sqrt((d[:, 4] ** 2).mean()) < rz0


def _d0_cancellation(p):
    """Per track, var(R) / var(d0): the transverse impact parameter of the
    Riemann fit is |centre| - R (FitUtils.h:198-214), so its variance is the
    difference of terms of the size of var(R); for a stiff track (R of
    10^3-10^5 cm) FP64 keeps only eps * var(R) / var(d0) of it."""
    nt = p["nTuples"]
    st = p["state"].reshape(-1, 5)[:nt].astype(np.float64)
    cov = p["cov"].reshape(-1, 15)[:nt].astype(np.float64)
    with np.errstate(all="ignore"):
        pt = 1.0 / np.abs(st[:, 2])
        k = cov[:, 9] * pt ** 4 / 0.0114256972711507 ** 2 / np.abs(cov[:, 5])
    return np.nan_to_num(k, nan=0.0, posinf=1e300)


@pytest.mark.parametrize("seed,pu", [(211, 20), (212, 50)])
def test_riemann_chain_matches_oracle(default_detector, seed, pu):
    """The whole chain configured with useRiemannFit (pg_config.riemann_fit)
    against the oracle chain configured the same way: integer products
    exact, floating-point ones within 1e-5 relative.  A track's covariance
    and chi2 may also differ by 8 eps times its d0 cancellation factor
    (_d0_cancellation): on these events every difference beyond 1e-5 sits in
    a stiff triplet with a factor above 1e10 and stays below 3 eps times it,
    the last bits of FP64 terms that cancel, where the device and host
    transcendental functions round differently."""
    import oracle
    import pixgpu
    raw = default_detector.event(seed, pu)
    want = oracle.Oracle(default_detector.es, riemann_fit=True).process(raw)
    c = pixgpu.Chain(default_detector.es, max_events=1, max_words_per_batch=300000, riemann_fit=True)
    try:
        c.process([raw])
        got = c.products(0)
    finally:
        c.close()
    names = [n for n in oracle.PRODUCTS if n not in ("chi2", "cov")]
    diffs = oracle.compare(want, got, names=names, rtol=RTOL)
    assert diffs == [], "\n".join("%s: %s" % d for d in diffs)
    nt = want["nTuples"]
    tol = RTOL + 8 * 2.220446e-16 * _d0_cancellation(want)
    for name, width in (("cov", 15), ("chi2", 1)):
        a = want[name].reshape(-1, width)[:nt].astype(np.float64)
        b = got[name].reshape(-1, width)[:nt].astype(np.float64)
        both_nan = np.isnan(a) & np.isnan(b)
        bad = (np.abs(a - b) > tol[:, None] * np.maximum(np.abs(a), np.abs(b))) & ~both_nan
        if name == "chi2":
            bad &= np.abs(a - b) > 2e-7
        assert not bad.any(), (name, np.nonzero(bad.any(axis=1))[0][:10].tolist())
