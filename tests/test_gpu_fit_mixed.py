"""Mixed-precision broken-line fit (FP32 arithmetic; FP64 for the reference
circle, the radial residuals, the Cholesky solves and the covariance
propagation) against the FP64 fit on the same tuples.

The FP64 fit equals the oracle within 1e-5 (test_gpu_parity.py); here the
deviation of the variant is bounded.  Measured on 200k seeded tuples per
multiplicity (maxima): |d(1/pT)| 4e-6 /GeV, |d phi| 5e-7, |d d0| 2e-6 cm for
every multiplicity; cot(theta) and z0 rms 5e-5 and 8e-4 cm for triplets,
5e-7 and 5e-6 cm for quadruplets.  The bounds below leave a margin of ~10.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BOUNDS = {  # nhits: (max |d 1/pT|, max |d phi|, max |d d0|, rms d cot, rms d z0)
    3: (5e-5, 1e-5, 5e-5, 1e-3, 1e-2),
    4: (5e-5, 1e-5, 5e-5, 1e-5, 1e-4),
    5: (5e-5, 1e-5, 5e-5, 1e-5, 1e-4),
}


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
    mk, mphi, md0, rcot, rz0 = BOUNDS[nhits]
    assert dk.max() < mk, dk.max()
    assert d[:, 0].max() < mphi, d[:, 0].max()
    assert d[:, 1].max() < md0, d[:, 1].max()
    assert np.sqrt((d[:, 3] ** 2).mean()) < rcot
    assert np.sqrt((d[:, 4] ** 2).mean()) < rz0
