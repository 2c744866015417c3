"""Launch-shape tuning (pg_tune_*, pg_autotune): the grid scales change the
speed of the chain, never its results; the tuner runs, and its cache file
round-trips."""
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_results_do_not_depend_on_launch_shapes(default_detector):
    import oracle
    import pixgpu
    raws = [default_detector.event(491 + k, pu) for k, pu in enumerate([50, 5, 80, 20])]
    c = pixgpu.Chain(default_detector.es, max_events=4, max_words_per_batch=4 * 300000)
    try:
        c.process(raws)
        base = [c.products(k) for k in range(len(raws))]
        rng = np.random.default_rng(5)
        for trial in range(2):
            for name in pixgpu.tune_kernel_names():
                c.tune_set(len(raws), name, int(rng.integers(-3, 4)))
            c.process(raws)
            for k in range(len(raws)):
                assert oracle.compare(base[k], c.products(k), rtol=0.0) == [], (trial, k)
    finally:
        c.close()


def test_autotune_and_cache_round_trip(default_detector):
    import pixgpu
    raws = [default_detector.event(495 + k, 50) for k in range(8)]
    c = pixgpu.Chain(default_detector.es, max_events=8, max_words_per_batch=8 * 200000, slots=1)
    try:
        gain = c.autotune(raws, repeats=1)
        assert gain >= 0.0
        table = c.tune_table(8)
        assert set(table) == set(pixgpu.tune_kernel_names())
        assert all(-3 <= v <= 3 for v in table.values())
        path = os.path.join(tempfile.mkdtemp(), "tune.txt")
        c.tune_save(path)
        c2 = pixgpu.Chain(default_detector.es, max_events=8, max_words_per_batch=8 * 200000, slots=1)
        try:
            assert c2.tune_load(path) == len(table)
            assert c2.tune_table(8) == table
            assert c2.tune_table(16) == table  # larger batches fall back to the largest tuned size
            assert c2.tune_table(4) == {k: 0 for k in table}
        finally:
            c2.close()
        with pytest.raises(RuntimeError):
            c.tune_set(8, "kNotAKernel", 1)
        with pytest.raises(RuntimeError):
            c.tune_set(8, "kConnect", 4)
    finally:
        c.close()
