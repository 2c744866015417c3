"""Mixed-precision broken-line fit (FP32 arithmetic; FP64 for the reference
circle, the arc lengths and radial residuals measured from it, the Cholesky
solves and the covariance propagation) against the FP64 fit on the same
tuples.

The FP64 fit equals the oracle within 1e-5 (test_gpu_parity.py); here the
deviation of the variant is bounded, absolutely and in units of the FP64
fit's own uncertainty.  Measured on 1M seeded tuples per multiplicity
(maxima, 3 / 4 hits): |d(1/pT)| 1.6e-5 / 2.4e-6 /GeV, |d phi| 1.4e-6 / 4.8e-7,
|d d0| 4.6e-6 / 1.6e-6 cm, |d cot(theta)| 1.9e-5 / 1.4e-5, |d z0| 2.1e-4 /
2.3e-4 cm; at most 0.07 sigma of the FP64 fit for any parameter.

Against the 1e-5 relative specification: 1/pT, phi, cot(theta) and z0 meet
it for at least 98.5 % of the tuples (99.5 % for the broken-line fit), and d0
(of order 1e-4 cm, so compared absolutely) as well; that every tuple meets it
is a known
exceedance (strict xfail below: the FP32 multiple-scattering and band-matrix
arithmetic moves a tail of tuples by up to ~1e-4 relative).  In the chain
(pg_config mixed_fit) the variant changes only fit products and what follows
from them; the quality codes and vertex assignments that flip against the
FP64 chain are bounded below.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BOUNDS = {  # nhits: (max |d 1/pT|, max |d phi|, max |d d0|, max |d cot|, max |d z0|)
    3: (1e-4, 1e-5, 5e-5, 2e-4, 2e-3),
    4: (5e-5, 1e-5, 5e-5, 2e-4, 2e-3),
    5: (5e-5, 1e-5, 5e-5, 2e-4, 2e-3),
}
MAX_PULL = 0.5  # max |mixed - FP64| / sigma(FP64) over the five parameters
SPEC = 1e-5     # relative (absolute in cm for d0)
DIAG = [0, 2, 5, 9, 14]  # diagonal of the packed 5x5 covariance


@pytest.fixture(scope="module")
def chain(default_detector):
    import pixgpu
    c = pixgpu.Chain(default_detector.es, max_events=1, max_words_per_batch=300000)
    yield c
    c.close()


@pytest.mark.parametrize("nhits,N", [(3, 3), (4, 4), (5, 4)])
def test_mixed_fit_within_bounds_of_fp64(chain, nhits, N):
    import pixgpu
    hits, ge, _ = pixgpu.fit_tuples(4242 + nhits, 20000, nhits)
    a = chain.fit(N, hits, ge)
    b = chain.fit(N, hits, ge, mixed=True)
    sa, sb = a["state"].astype(np.float64), b["state"].astype(np.float64)
    assert np.isfinite(sb).all() and np.isfinite(b["pt"]).all()
    dk = np.abs(1.0 / b["pt"].astype(np.float64) - 1.0 / a["pt"].astype(np.float64))
    d = np.abs(sb - sa)
    mk, mphi, md0, mcot, mz0 = BOUNDS[nhits]
    assert dk.max() < mk, dk.max()
    assert d[:, 0].max() < mphi, d[:, 0].max()
    assert d[:, 1].max() < md0, d[:, 1].max()
    assert d[:, 3].max() < mcot, d[:, 3].max()
    assert d[:, 4].max() < mz0, d[:, 4].max()
    sig = np.sqrt(np.maximum(a["cov"].astype(np.float64).reshape(-1, 15)[:, DIAG], 0.0))
    ok = (sig > 0).all(axis=1)
    pull = (d[ok] / sig[ok]).max()
    assert pull < MAX_PULL, pull


def _spec_fractions(a, b):
    """Per parameter, the fraction of tuples within SPEC of the FP64 fit."""
    sa, sb = a["state"].astype(np.float64), b["state"].astype(np.float64)
    ka, kb = 1.0 / a["pt"].astype(np.float64), 1.0 / b["pt"].astype(np.float64)
    rel = lambda x, y: np.abs(x - y) / np.maximum(np.abs(x), 1e-30)  # noqa: E731
    return {"inv_pt": (rel(ka, kb) <= SPEC).mean(), "phi": (rel(sa[:, 0], sb[:, 0]) <= SPEC).mean(),
            "d0": (np.abs(sa[:, 1] - sb[:, 1]) <= SPEC).mean(),
            "cot_theta": (rel(sa[:, 3], sb[:, 3]) <= SPEC).mean(), "z0": (rel(sa[:, 4], sb[:, 4]) <= SPEC).mean()}


@pytest.mark.parametrize("riemann", [False, True])
@pytest.mark.parametrize("nhits,N", [(3, 3), (4, 4)])
def test_mixed_fit_meets_the_spec_for_most_tuples(chain, nhits, N, riemann):
    import pixgpu
    hits, ge, _ = pixgpu.fit_tuples(4343 + nhits, 20000, nhits)
    a = chain.fit(N, hits, ge, riemann=riemann)
    b = chain.fit(N, hits, ge, mixed=True, riemann=riemann)
    fr = _spec_fractions(a, b)
    # measured: every fraction >= 0.995 for the broken-line fit; the Riemann
    # fit's z0 reaches 0.9896 for 4-hit tuples
    assert min(fr.values()) >= 0.985, fr


@pytest.mark.xfail(strict=True, reason="known exceedance of the 1e-5 specification: a tail of tuples (<1 %) "
                                       "deviates by up to ~1e-4 relative in the mixed-precision fits")
@pytest.mark.parametrize("riemann", [False, True])
def test_mixed_fit_every_tuple_within_the_spec(chain, riemann):
    import pixgpu
    hits, ge, _ = pixgpu.fit_tuples(4444, 20000, 4)
    a = chain.fit(4, hits, ge, riemann=riemann)
    b = chain.fit(4, hits, ge, mixed=True, riemann=riemann)
    assert min(_spec_fractions(a, b).values()) == 1.0


def test_mixed_fit_in_the_chain(default_detector):
    """The chain with pg_config mixed_fit against the FP64 chain on 16 PU50
    events: identical up to the tuples, fits within the spec for most
    tuples, and few quality codes and vertex assignments flipped."""
    import pixgpu
    raws = [default_detector.event(pixgpu.BENCH_SEED_BASE + 2000 + k, 50, model=pixgpu.BENCH_MODEL)
            for k in range(16)]
    words = sum(len(r) // 4 for r in raws) + 1024
    got = {}
    for mixed in (False, True):
        c = pixgpu.Chain(default_detector.es, max_events=16, max_words_per_batch=words, mixed_fit=mixed)
        try:
            c.process(raws)
            got[mixed] = [c.products(k) for k in range(len(raws))]
        finally:
            c.close()
    ntup = nq = nidv = nvtx_diff = 0
    for a, b in zip(got[False], got[True]):
        for n in ("nHits", "nCells", "nTuples"):
            assert a[n] == b[n], n
        for n in ("cellNbr", "tupleHits", "tupleOff"):
            assert np.array_equal(a[n], b[n]), n
        ntup += a["nTuples"]
        nq += int((a["quality"] != b["quality"]).sum())
        m = min(len(a["idv"]), len(b["idv"]))
        nidv += int((a["idv"][:m] != b["idv"][:m]).sum())
        nvtx_diff = max(nvtx_diff, abs(a["nVertices"] - b["nVertices"]))
    # flips: quality codes of at most 0.5 % of the tuples, vertex counts within one per event
    assert nq <= 0.005 * ntup, (nq, ntup)
    assert nvtx_diff <= 1, nvtx_diff
    assert nidv <= 0.02 * ntup, (nidv, ntup)
