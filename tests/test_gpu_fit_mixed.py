"""Mixed-precision broken-line fit (FP32 arithmetic; FP64 for the reference
circle, the arc lengths and radial residuals measured from it, the Cholesky
solves and the covariance propagation) against the FP64 fit on the same
tuples.

The FP64 fit equals the oracle within 1e-5 (test_gpu_parity.py); here the
deviation of the variant is bounded, absolutely and in units of the FP64
fit's own uncertainty.  Measured on 1M seeded tuples per multiplicity
(maxima, 3 / 4 hits): |d(1/pT)| 1.6e-5 / 2.4e-6 /GeV, |d phi| 1.4e-6 / 4.8e-7,
|d d0| 4.6e-6 / 1.6e-6 cm, |d cot(theta)| 1.9e-5 / 1.4e-5, |d z0| 2.1e-4 /
2.3e-4 cm; at most 0.07 sigma of the FP64 fit for any parameter.  The bounds
below leave a margin of ~5-10.
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
