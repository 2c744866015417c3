"""The oracle's container capacities (oracle::Caps).

At the reference's capacities the oracle equals the reference build bit for
bit (test_oracle_reference.py).  Wider capacities must change nothing on
events whose containers the reference's capacities already hold, and must
let events of higher pileup through in full, where the reference's
capacities either truncate (hits, doublets) or overflow
(TupleMultiplicity, HitToTuple: undefined behaviour in the reference, which
the oracle refuses)."""
import pytest

import oracle


def _wide():
    import pixgpu
    return dict(pixgpu.WIDE_CAPS)


@pytest.mark.parametrize("seed,pu,model", [(31, 20, "dense"), (32, 50, "calibrated"), (33, 80, "calibrated")])
def test_wide_caps_change_nothing_below_the_reference_caps(default_detector, seed, pu, model):
    raw = default_detector.event(seed, pu, model=model)
    narrow = oracle.Oracle(default_detector.es).process(raw)
    wide = oracle.Oracle(default_detector.es, caps=_wide()).process(raw)
    assert narrow["nHits"] < 49152 and narrow["nCells"] < 458752
    assert oracle.compare(narrow, wide, rtol=0) == []


def test_wide_caps_hold_pileup_150(default_detector):
    raw = default_detector.event(20261203 + 7, 150, model="calibrated")
    wide = oracle.Oracle(default_detector.es, caps=_wide()).process(raw)
    # the reference's 49152 hits and 458752 doublets are exceeded ...
    assert wide["nHits"] > 49152 and wide["nCells"] > 458752
    assert wide["nTuples"] > 32768
    # ... where its own capacities truncate the event
    try:
        narrow = oracle.Oracle(default_detector.es).process(raw)
    except RuntimeError:
        return  # refused: a container of the reference overflows (undefined there)
    assert narrow["nHits"] == 49152 and narrow["nCells"] == 458752


def test_caps_below_the_reference_are_refused(default_detector):
    with pytest.raises(ValueError):
        oracle.Oracle(default_detector.es, caps={"hits": 1000})
    with pytest.raises(ValueError):
        oracle.Oracle(default_detector.es, caps={"bogus": 1})


def test_capi_refuses_caps_below_the_reference(default_detector):
    """pg_create checks the capacities before touching a device."""
    import ctypes
    import pixgpu
    lib = pixgpu.gpu_lib()
    keep = list(default_detector.es)
    img = pixgpu.ESImages(*[x for b in keep for x in (b, len(b))])
    cfg = pixgpu.Config()
    lib.pg_default_config(ctypes.byref(cfg))
    cfg.cap_hits = 1000
    h = ctypes.c_void_p()
    assert lib.pg_create(ctypes.byref(img), ctypes.byref(cfg), ctypes.byref(h)) == -1  # PG_ERR_ARG
    cfg.cap_hits = 0
    cfg.cap_tuples = 1 << 20  # the multiplicity fill counts bins in 20-bit fields
    assert lib.pg_create(ctypes.byref(img), ctypes.byref(cfg), ctypes.byref(h)) == -1
    cfg.cap_tuples = 0
    cfg.cap_hits = (1 << 21) + 1  # hit indices are packed into 21 bits
    assert lib.pg_create(ctypes.byref(img), ctypes.byref(cfg), ctypes.byref(h)) == -1
