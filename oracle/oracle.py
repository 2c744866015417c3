"""Checker-side Python access to the CPU oracle (liboracle.so) and to the
checker build of the reference's serial sources (oracle/_ref/libpixref.so).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, never by the product path.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "pixeltrack-standalone_b200"))
import build as _build  # noqa: E402
from pixgpu import ERROR_DTYPE, FORMATTER_ERROR_DTYPE, SCALARS, _TYPES  # noqa: E402

# the CA module's switches (CAHitNtupletGeneratorOnGPU.cc:46-58) with the
# reference's defaults; the same names as the product's pg_config fields
CA_DEFAULTS = {"min_hits_per_ntuplet": 3, "include_jumping_forward_doublets": 1, "early_fishbone": 1,
               "late_fishbone": 0, "ideal_conditions": 1, "do_cluster_cut": 1, "do_z0_cut": 1, "do_pt_cut": 1}


def _ca_args(ca):
    p = dict(CA_DEFAULTS)
    for k, v in (ca or {}).items():
        if k not in p:
            raise ValueError("unknown CA parameter %s" % k)
        p[k] = int(v)
    return [p[k] for k in CA_DEFAULTS]

# container capacities, in the order of or_set_caps (oracle::Caps)
CAPS_FIELDS = ["fed_words", "hits", "doublets", "lists", "tuples", "multiplicity", "hit_to_tuple"]

# the per-event counts of cut decisions on their float boundary (oracle and
# GPU chain; the reference's own code has no such counter)
CUT_MARGIN_COUNTS = ("nCutMarginDoublets", "nCutMarginCA", "nCutMarginQuality")

PRODUCTS = ["nDigis", "nModules", "xx", "yy", "adc", "moduleInd", "clus", "pdigi", "rawIdArr", "errors",
            "formatterErrors", "nClusters",
            "moduleStart", "clusInModule", "moduleId", "clusModuleStart", "nHits", "xl", "yl", "xerr", "yerr", "xg",
            "yg", "zg", "rg", "charge", "iphi", "xsize", "ysize", "detInd", "hitsLayerStart", "phiOff", "phiBins",
            "nCells", "cellInner", "cellOuter", "cellLayerPair", "cellDoubletId", "cellUsed", "cellNbrOff",
            "cellNbr", "cellTrkOff", "cellTrk", "outerHitOff", "outerHitCells", "nNbrLists", "nTrkLists", "nTuples",
            "nCutMarginDoublets", "nCutMarginCA", "nCutMarginQuality",
            "tupleOff", "tupleHits", "tupleDet", "quality", "state", "cov", "pt", "eta", "chi2", "nVertices", "zv",
            "wv", "vchi2", "ptv2", "ndof", "sortInd", "idv"]


def _decode(buf, name, elem):
    if name == "errors":
        return np.frombuffer(buf, dtype=ERROR_DTYPE).copy()
    if name == "formatterErrors":
        return np.frombuffer(buf, dtype=FORMATTER_ERROR_DTYPE).copy()
    if name in SCALARS:
        return int(np.frombuffer(buf, dtype=np.uint32)[0])
    dt = _TYPES.get(name)
    if dt is None or np.dtype(dt).itemsize != elem:
        dt = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[elem]
    return np.frombuffer(buf, dtype=dt).copy()


class _Named:
    _get = None

    def _products(self, names):
        out = {}
        for n in names:
            d = ctypes.c_void_p()
            c = ctypes.c_size_t()
            e = ctypes.c_int()
            if self._get(self._h, n.encode(), ctypes.byref(d), ctypes.byref(c), ctypes.byref(e)) != 0:
                continue
            out[n] = _decode(ctypes.string_at(d, c.value * e.value), n, e.value)
        return out


class Oracle(_Named):
    """Sequential restatement of the serial chain (oracle/*.cc)."""

    def __init__(self, es_images, riemann_fit=False, vertex_algo=0, ca=None, formatter_errors=False, caps=None):
        """caps: container capacities (CAPS_FIELDS names) above the reference's."""
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            _build.build_oracle()
        self.lib = ctypes.CDLL(path)
        self.lib.or_create.restype = ctypes.c_void_p
        self.lib.or_create.argtypes = [ctypes.c_char_p, ctypes.c_size_t] * 5
        self.lib.or_process.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
        self.lib.or_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p),
                                    ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int)]
        self.lib.or_last_seconds.argtypes = [ctypes.c_void_p]
        self.lib.or_last_seconds.restype = ctypes.c_double
        self.lib.or_time_events.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_char_p),
                                            ctypes.POINTER(ctypes.c_size_t), ctypes.c_int, ctypes.c_int,
                                            ctypes.c_void_p]
        self.lib.or_time_events.restype = ctypes.c_double
        self.lib.or_fit.argtypes = [ctypes.c_int, ctypes.c_uint32] + [ctypes.c_void_p] * 2 + [ctypes.c_double] + \
            [ctypes.c_void_p] * 5
        self.lib.or_fit_riemann.argtypes = self.lib.or_fit.argtypes
        self.lib.or_destroy.argtypes = [ctypes.c_void_p]
        self.lib.or_set_riemann.argtypes = [ctypes.c_void_p, ctypes.c_int]
        self._keep = list(es_images)
        args = []
        for b in self._keep:
            args += [b, len(b)]
        self._h = ctypes.c_void_p(self.lib.or_create(*args))
        if not self._h.value:
            raise RuntimeError("oracle: malformed ES images")
        self._get = self.lib.or_get
        self.lib.or_set_riemann(self._h, 1 if riemann_fit else 0)
        self.lib.or_set_vertex_algo.argtypes = [ctypes.c_void_p, ctypes.c_int]
        if self.lib.or_set_vertex_algo(self._h, int(vertex_algo)) != 0:
            raise ValueError("vertex_algo: 0 density, 1 DBSCAN, 2 iterative")
        self.lib.or_set_ca_params.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 8
        if self.lib.or_set_ca_params(self._h, *_ca_args(ca)) != 0:
            raise ValueError("min_hits_per_ntuplet: 3 or 4")
        self.lib.or_set_formatter_errors.argtypes = [ctypes.c_void_p, ctypes.c_int]
        self.lib.or_set_formatter_errors(self._h, 1 if formatter_errors else 0)
        if caps:
            self.lib.or_set_caps.argtypes = [ctypes.c_void_p] + [ctypes.c_uint32] * len(CAPS_FIELDS)
            unknown = set(caps) - set(CAPS_FIELDS)
            if unknown:
                raise ValueError("unknown capacities %s" % sorted(unknown))
            if self.lib.or_set_caps(self._h, *[int(caps.get(k, 0)) for k in CAPS_FIELDS]) != 0:
                raise ValueError("capacities below the reference's")

    def process(self, raw, names=None):
        if self.lib.or_process(self._h, raw, len(raw)) != 0:
            raise RuntimeError("oracle failed on this event")
        return self._products(names or PRODUCTS)

    def last_seconds(self):
        return self.lib.or_last_seconds(self._h)

    def time_events(self, raws, threads=1):
        """Wall seconds and per-event seconds for the chain over raws on `threads` host threads."""
        n = len(raws)
        ptrs = (ctypes.c_char_p * n)(*raws)
        sizes = (ctypes.c_size_t * n)(*[len(r) for r in raws])
        lat = np.zeros(n, dtype=np.float64)
        wall = self.lib.or_time_events(self._h, ptrs, sizes, n, threads, lat.ctypes.data)
        if wall < 0:
            raise RuntimeError("oracle failed while timing")
        return wall, lat

    def fit(self, N, hits, ge, B=0.0114256972711507, riemann=False):
        n = hits.shape[0]
        h = np.ascontiguousarray(hits[:, :N, :], dtype=np.float64)
        g = np.ascontiguousarray(ge[:, :N, :], dtype=np.float32)
        out = {"state": np.zeros((n, 5), np.float32), "cov": np.zeros((n, 15), np.float32),
               "pt": np.zeros(n, np.float32), "eta": np.zeros(n, np.float32), "chi2": np.zeros(n, np.float32)}
        fn = self.lib.or_fit_riemann if riemann else self.lib.or_fit
        rc = fn(N, n, h.ctypes.data, g.ctypes.data, B, out["state"].ctypes.data, out["cov"].ctypes.data,
                             out["pt"].ctypes.data, out["eta"].ctypes.data, out["chi2"].ctypes.data)
        if rc != 0:
            raise RuntimeError("oracle fit failed")
        return out

    def cluster_digis(self, module_ind, xx, yy, adc):
        """countModules, findClus and clusterChargeCut on given digis (calibrated charges)."""
        return _cluster_digis(self.lib.or_cluster_digis, module_ind, xx, yy, adc)

    def vertices(self, tupleOff, quality, pt, state, cov):
        """The serial vertex finder on a given track SoA (n tuples)."""
        n = len(quality)
        out = {"idv": np.zeros(max(n, 1), np.int16), "zv": np.zeros(1024, np.float32),
               "wv": np.zeros(1024, np.float32), "vchi2": np.zeros(1024, np.float32),
               "ptv2": np.zeros(1024, np.float32), "ndof": np.zeros(1024, np.int32),
               "sortInd": np.zeros(1024, np.uint16)}
        nv = ctypes.c_uint32()
        args = [np.ascontiguousarray(a) for a in (tupleOff, quality, pt, state, cov)]
        self.lib.or_vertices.argtypes = [ctypes.c_uint32] + [ctypes.c_void_p] * 13
        rc = self.lib.or_vertices(n, *[a.ctypes.data for a in args],
                                  *[out[k].ctypes.data for k in ("idv", "zv", "wv", "vchi2", "ptv2", "ndof",
                                                                 "sortInd")], ctypes.addressof(nv))
        if rc != 0:
            raise RuntimeError("oracle vertexing failed")
        k = nv.value
        return {"nVertices": k, "idv": out["idv"][:n], "zv": out["zv"][:k], "wv": out["wv"][:k],
                "vchi2": out["vchi2"][:k], "ptv2": out["ptv2"][:k], "ndof": out["ndof"][:k],
                "sortInd": out["sortInd"][:k]}

    def __del__(self):
        try:
            self.lib.or_destroy(self._h)
        except Exception:
            pass


REF_LIB = os.path.join(HERE, "_ref", "libpixref.so")


def _cluster_digis(fn, module_ind, xx, yy, adc):
    """or_cluster_digis on host arrays; returns a dict of arrays."""
    n = len(module_ind)
    arrs = [np.ascontiguousarray(a, dtype=np.uint16) for a in (module_ind, xx, yy, adc)]
    out = {"moduleInd": np.zeros(n, np.uint16), "clus": np.zeros(n, np.int32),
           "clusInModule": np.zeros(2000, np.uint32), "moduleId": np.zeros(2000, np.uint32),
           "moduleStart": np.zeros(2001, np.uint32)}
    nm = ctypes.c_uint32()
    fn.argtypes = [ctypes.c_uint32] + [ctypes.c_void_p] * 10
    rc = fn(n, *[a.ctypes.data for a in arrs],
            *[out[k].ctypes.data for k in ("moduleInd", "clus", "clusInModule", "moduleId", "moduleStart")],
            ctypes.byref(nm))
    if rc != 0:
        raise RuntimeError("oracle: clustering undefined for these digis")
    out["nModules"] = nm.value
    return out


def ref_available():
    return os.path.exists(REF_LIB)


class Reference(_Named):
    """The reference's own serial chain, compiled from its sources (checker build)."""

    def __init__(self, datadir, riemann_fit=False, vertex_algo=0, ca=None, formatter_errors=False):
        self.lib = ctypes.CDLL(REF_LIB)
        self.lib.pr_create.restype = ctypes.c_void_p
        self.lib.pr_create.argtypes = [ctypes.c_char_p]
        self.lib.pr_process.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_int]
        self.lib.pr_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p),
                                    ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int)]
        self.lib.pr_last_seconds.argtypes = [ctypes.c_void_p]
        self.lib.pr_last_seconds.restype = ctypes.c_double
        self._h = ctypes.c_void_p(self.lib.pr_create(datadir.encode()))
        self._get = self.lib.pr_get
        self.lib.pr_set_riemann.argtypes = [ctypes.c_void_p, ctypes.c_int]
        self.lib.pr_set_riemann(self._h, 1 if riemann_fit else 0)
        self.lib.pr_set_vertex_algo.argtypes = [ctypes.c_void_p, ctypes.c_int]
        if self.lib.pr_set_vertex_algo(self._h, int(vertex_algo)) != 0:
            raise ValueError("vertex_algo: 0 density, 1 DBSCAN, 2 iterative")
        self.lib.pr_set_formatter_errors.argtypes = [ctypes.c_void_p, ctypes.c_int]
        self.lib.pr_set_formatter_errors(self._h, 1 if formatter_errors else 0)
        if ca:
            self.lib.pr_set_ca_params.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 8
            if self.lib.pr_set_ca_params(self._h, *_ca_args(ca)) != 0:
                raise ValueError("min_hits_per_ntuplet: 3 or 4")

    def process(self, raw, names=None, internals=True):
        if self.lib.pr_process(self._h, raw, len(raw), 1 if internals else 0) != 0:
            raise RuntimeError("reference chain failed")
        return self._products(names or PRODUCTS)

    def last_seconds(self):
        return self.lib.pr_last_seconds(self._h)


def ref_fit_riemann(N, hits, ge, B=0.0114256972711507):
    """The reference's own Riemann fit (RiemannFit.h through the checker
    build) on standalone tuples, in the layout of Oracle.fit."""
    lib = ctypes.CDLL(REF_LIB)
    lib.pr_fit_riemann.argtypes = [ctypes.c_int, ctypes.c_uint32] + [ctypes.c_void_p] * 2 + [ctypes.c_double] + \
        [ctypes.c_void_p] * 5
    n = hits.shape[0]
    h = np.ascontiguousarray(hits[:, :N, :], dtype=np.float64)
    g = np.ascontiguousarray(ge[:, :N, :], dtype=np.float32)
    out = {"state": np.zeros((n, 5), np.float32), "cov": np.zeros((n, 15), np.float32),
           "pt": np.zeros(n, np.float32), "eta": np.zeros(n, np.float32), "chi2": np.zeros(n, np.float32)}
    if lib.pr_fit_riemann(N, n, h.ctypes.data, g.ctypes.data, B, out["state"].ctypes.data, out["cov"].ctypes.data,
                          out["pt"].ctypes.data, out["eta"].ctypes.data, out["chi2"].ctypes.data) != 0:
        raise RuntimeError("reference Riemann fit failed")
    return out


def ref_time_events(datadir, raws, threads=1):
    """The reference serial chain over raws on `threads` host threads, one
    chain instance per thread: (wall seconds, per-event chain seconds)."""
    lib = ctypes.CDLL(REF_LIB)
    lib.pr_time_events.restype = ctypes.c_double
    lib.pr_time_events.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_size_t),
                                   ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    n = len(raws)
    ptrs = (ctypes.c_char_p * n)(*raws)
    sizes = (ctypes.c_size_t * n)(*[len(r) for r in raws])
    lat = np.zeros(n, dtype=np.float64)
    wall = lib.pr_time_events(datadir.encode(), ptrs, sizes, n, threads, lat.ctypes.data)
    if wall < 0:
        raise RuntimeError("reference chain failed while timing")
    return wall, lat


def compare(a, b, names=None, rtol=1e-5, atol=None):
    """Differences between two product dicts: integers exactly, floats within
    rtol relative.  atol is an absolute floor for values that are pure
    cancellation residue (a fitted cot(theta) of 1e-16 where the exact value is
    0): float32 outputs of O(1) quantities carry no information below it.  It
    defaults to 1e-12, or to 0 for an exact comparison (rtol == 0)."""
    if atol is None:
        atol = 1e-12 if rtol > 0 else 0.0
    diffs = []
    for n in names or PRODUCTS:
        if n not in a and n not in b:
            continue
        if n in CUT_MARGIN_COUNTS and (n not in a or n not in b):
            continue  # the reference build and its fixtures do not count cut margins
        if (n in a) != (n in b):
            diffs.append((n, "missing on one side"))
            continue
        x, y = a[n], b[n]
        if isinstance(x, int) or isinstance(y, int):
            if int(x) != int(y):
                diffs.append((n, "value %d != %d" % (x, y)))
            continue
        if x.shape != y.shape:
            diffs.append((n, "shape %s != %s" % (x.shape, y.shape)))
            continue
        if n == "errors":
            for f in ("rawId", "word", "errorType", "fedId"):
                if not np.array_equal(x[f], y[f]):
                    diffs.append((n, "error records differ in %s" % f))
            continue
        if x.dtype.kind == "f":
            xd, yd = x.astype(np.float64), y.astype(np.float64)
            both_nan = np.isnan(xd) & np.isnan(yd)
            den = np.maximum(np.abs(xd), np.abs(yd))
            ad = np.abs(xd - yd)
            rel = np.where(both_nan, 0.0, ad / np.where(den > 0, den, 1.0))
            bad = (rel > rtol) & (ad > atol) & ~both_nan
            if bad.any():
                i = int(np.nonzero(bad)[0][0])
                diffs.append((n, "%d values beyond rtol %g (max rel %.3g; first at %d: %r vs %r)"
                              % (int(bad.sum()), rtol, float(rel[bad].max()), i, float(xd[i]), float(yd[i]))))
        elif not np.array_equal(x, y):
            i = np.nonzero(x != y)[0]
            diffs.append((n, "%d entries differ, first at %d: %s vs %s" % (len(i), i[0], x[i[0]], y[i[0]])))
    return diffs
