"""Python access to the B200 pixel chain (include/pixgpu.h), the synthetic
event generator (include/pixsynth.h) and, for tests only, the CPU oracle and
the checker build of the reference.

The product path is libpixgpu.so; this module only marshals buffers.  If the
library is missing it is built (nvcc cross-compiles without a GPU); a context
cannot be created without a CUDA device, and every failure raises.
"""
import ctypes
import os
import sys

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB = os.path.join(PKG, "lib")
sys.path.insert(0, PKG)
import build as _build  # noqa: E402

U8P = ctypes.POINTER(ctypes.c_uint8)

# products and their element types (names follow the reference's SoA members)
_TYPES = {
    "xx": np.uint16, "yy": np.uint16, "adc": np.uint16, "moduleInd": np.uint16, "clus": np.int32,
    "pdigi": np.uint32, "rawIdArr": np.uint32, "moduleStart": np.uint32, "clusInModule": np.uint32,
    "moduleId": np.uint32, "clusModuleStart": np.uint32, "xl": np.float32, "yl": np.float32,
    "xerr": np.float32, "yerr": np.float32, "xg": np.float32, "yg": np.float32, "zg": np.float32,
    "rg": np.float32, "charge": np.int32, "iphi": np.int16, "xsize": np.int16, "ysize": np.int16,
    "detInd": np.uint16, "hitsLayerStart": np.uint32, "phiOff": np.uint32, "phiBins": np.uint32,
    "agcLadderR": np.float32, "cellInner": np.uint32, "cellOuter": np.uint32, "cellLayerPair": np.int16,
    "cellDoubletId": np.int32, "cellUsed": np.uint16, "cellNbrOff": np.uint32, "cellNbr": np.uint32,
    "cellTrkOff": np.uint32, "cellTrk": np.uint32, "outerHitOff": np.uint32, "outerHitCells": np.uint32,
    "tupleOff": np.uint32, "tupleHits": np.uint32, "tupleDet": np.uint16, "quality": np.uint8,
    "state": np.float32, "cov": np.float32, "pt": np.float32, "eta": np.float32, "chi2": np.float32,
    "zv": np.float32, "wv": np.float32, "vchi2": np.float32, "ptv2": np.float32, "ndof": np.int32,
    "sortInd": np.uint16, "idv": np.int16,
    "outerHitOffRaw": np.uint32, "outerHitCellsRaw": np.uint32, "cellNbrOffRaw": np.uint32,
    "cellNbrRaw": np.uint32, "cellTrkOffRaw": np.uint32, "cellTrkRaw": np.uint32,
}
SCALARS = ["nDigis", "nModules", "nClusters", "nHits", "nCells", "nTuples", "nVertices", "nNbrLists",
           "nTrkLists", "nCutMarginDoublets", "nCutMarginCA", "nCutMarginQuality"]
ERROR_DTYPE = np.dtype([("rawId", "<u4"), ("word", "<u4"), ("errorType", "u1"), ("fedId", "u1"),
                        ("pad", "u1", 2)])
# PfFormatterError: the 64-bit header/trailer word, the error type, the full FED id
FORMATTER_ERROR_DTYPE = np.dtype([("word64", "<u8"), ("errorType", "<u4"), ("fedId", "<u4")])
FLOAT_PRODUCTS = {"xl", "yl", "xerr", "yerr", "xg", "yg", "zg", "rg", "agcLadderR", "state", "cov", "pt", "eta",
                  "chi2", "zv", "wv", "vchi2", "ptv2"}
B_FIELD = 0.0114256972711507


def _as_array(buf, name, elem):
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


def _load(path, builder):
    if not os.path.exists(path):
        builder()
    return ctypes.CDLL(path)


# --------------------------------------------------------------------- generator
_synth = None


def synth():
    global _synth
    if _synth is None:
        _synth = _load(os.path.join(LIB, "libpixsynth.so"), _build.build_synth)
        _synth.ps_event_generate.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double, ctypes.c_void_p,
                                             ctypes.POINTER(ctypes.c_void_p)]
        _synth.ps_event_raw.argtypes = [ctypes.c_void_p, ctypes.POINTER(U8P), ctypes.POINTER(ctypes.c_size_t)]
        _synth.ps_event_destroy.argtypes = [ctypes.c_void_p]
        _synth.ps_detector_es.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(U8P),
                                          ctypes.POINTER(ctypes.c_size_t)]
        _synth.ps_detector_write.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        _synth.ps_detector_destroy.argtypes = [ctypes.c_void_p]
        _synth.ps_calibrated_event_config.argtypes = [ctypes.c_void_p]
        _synth.ps_default_event_config.argtypes = [ctypes.c_void_p]
        _synth.ps_fit_tuples.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p]
    return _synth


class DetectorConfig(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("dead_column_frac", ctypes.c_double), ("bad_roc_frac", ctypes.c_double)]


class EventConfig(ctypes.Structure):
    _fields_ = [("tracks_per_vertex", ctypes.c_double), ("pt_min", ctypes.c_double), ("pt_index", ctypes.c_double),
                ("eta_max", ctypes.c_double), ("noise_frac", ctypes.c_double), ("inject_errors", ctypes.c_int),
                ("fixed_pu", ctypes.c_int), ("soft_per_vertex", ctypes.c_double), ("soft_pt_min", ctypes.c_double),
                ("soft_pt_mean", ctypes.c_double), ("secondary_frac", ctypes.c_double)]


class Truth(ctypes.Structure):
    _fields_ = [("n_vertices", ctypes.c_uint32), ("n_tracks", ctypes.c_uint32), ("n_sim_hits", ctypes.c_uint32),
                ("n_digis", ctypes.c_uint32), ("vertex_z", ctypes.c_void_p), ("track_pt", ctypes.c_void_p),
                ("track_eta", ctypes.c_void_p), ("track_phi", ctypes.c_void_p), ("track_q", ctypes.c_void_p),
                ("track_vertex", ctypes.c_void_p), ("track_nhits", ctypes.c_void_p)]


ES_NAMES = ["cablingMap.bin", "gain.bin", "cpefast.bin", "beamspot.bin", "fedIds.bin"]
BASE_SEED = 20261203
# the benchmark's PU50 events: event k is seed BENCH_SEED_BASE + k of the
# calibrated event model
BENCH_SEED_BASE = BASE_SEED + 100000
BENCH_MODEL = "calibrated"
# pg_flag bits (include/pixgpu.h)
PG_FLAG_MODULE_TOO_BIG = 1 << 0
PG_FLAG_TUPLE_OVERFLOW = 1 << 5
PG_FLAG_CELL_OVERFLOW = 1 << 6
PG_FLAG_TOO_MANY_WORDS = 1 << 9
PG_FLAG_BAD_INPUT = 1 << 15
PG_FLAG_SPLIT_MODULE = 1 << 17


class Detector:
    """Seeded synthetic Phase-1 detector: ES file images and raw events."""

    def __init__(self, seed=BASE_SEED, dead_column_frac=0.0, bad_roc_frac=0.0):
        lib = synth()
        cfg = DetectorConfig(seed, dead_column_frac, bad_roc_frac)
        self._h = ctypes.c_void_p()
        if lib.ps_detector_create(ctypes.byref(cfg), ctypes.byref(self._h)) != 0:
            raise RuntimeError("ps_detector_create failed")
        self.es = []
        for k in range(5):
            p = U8P()
            n = ctypes.c_size_t()
            lib.ps_detector_es(self._h, k, ctypes.byref(p), ctypes.byref(n))
            self.es.append(ctypes.string_at(p, n.value))

    def write(self, directory):
        os.makedirs(directory, exist_ok=True)
        if synth().ps_detector_write(self._h, directory.encode()) != 0:
            raise RuntimeError("ps_detector_write failed")

    def event(self, seed, pu, tracks_per_vertex=None, inject_errors=0, noise_frac=None, fixed_pu=True,
              with_truth=False, model="dense"):
        """One raw.bin record.  model: "dense" (every track prompt and above 0.5 GeV,
        ps_default_event_config) or "calibrated" (ps_calibrated_event_config: a soft,
        mostly displaced component; PU50 gives ~57k digis, ~18k hits, ~1.6k loose tracks)."""
        lib = synth()
        cfg = EventConfig()
        if model == "dense":
            lib.ps_default_event_config(ctypes.byref(cfg))
        elif model == "calibrated":
            lib.ps_calibrated_event_config(ctypes.byref(cfg))
        else:
            raise ValueError("model: 'dense' or 'calibrated'")
        if tracks_per_vertex is not None:
            cfg.tracks_per_vertex = tracks_per_vertex
        if noise_frac is not None:
            cfg.noise_frac = noise_frac
        cfg.inject_errors = inject_errors
        cfg.fixed_pu = 1 if fixed_pu else 0
        ev = ctypes.c_void_p()
        if lib.ps_event_generate(self._h, seed, float(pu), ctypes.byref(cfg), ctypes.byref(ev)) != 0:
            raise RuntimeError("ps_event_generate failed")
        try:
            p = U8P()
            n = ctypes.c_size_t()
            lib.ps_event_raw(ev, ctypes.byref(p), ctypes.byref(n))
            raw = ctypes.string_at(p, n.value)
            truth = None
            if with_truth:
                t = Truth()
                lib.ps_event_truth(ev, ctypes.byref(t))
                truth = {"n_vertices": t.n_vertices, "n_tracks": t.n_tracks, "n_sim_hits": t.n_sim_hits,
                         "n_digis": t.n_digis}
        finally:
            lib.ps_event_destroy(ev)
        return (raw, truth) if with_truth else raw

    def __del__(self):
        try:
            synth().ps_detector_destroy(self._h)
        except Exception:
            pass


def fit_tuples(seed, n, nhits):
    """Seeded n tuples of nhits hits (MS-smeared helices) for the fit workload."""
    hits = np.zeros((n, nhits, 3), dtype=np.float64)
    ge = np.zeros((n, nhits, 6), dtype=np.float32)
    truth = np.zeros((n, 5), dtype=np.float64)
    rc = synth().ps_fit_tuples(seed, n, nhits, hits.ctypes.data, ge.ctypes.data, truth.ctypes.data)
    if rc != 0:
        raise RuntimeError("ps_fit_tuples failed")
    return hits, ge, truth


# --------------------------------------------------------------------- GPU chain
_gpu = None


class ESImages(ctypes.Structure):
    _fields_ = [("cabling", ctypes.c_char_p), ("cabling_size", ctypes.c_size_t), ("gain", ctypes.c_char_p),
                ("gain_size", ctypes.c_size_t), ("cpe", ctypes.c_char_p), ("cpe_size", ctypes.c_size_t),
                ("beamspot", ctypes.c_char_p), ("beamspot_size", ctypes.c_size_t), ("fedids", ctypes.c_char_p),
                ("fedids_size", ctypes.c_size_t)]


CA_FIELDS = ("min_hits_per_ntuplet", "include_jumping_forward_doublets", "early_fishbone", "late_fishbone",
             "ideal_conditions", "do_cluster_cut", "do_z0_cut", "do_pt_cut")


# per-event container capacities (pg_config cap_* fields); 0 keeps the reference's value
CAPS_FIELDS = ("fed_words", "hits", "doublets", "lists", "tuples", "multiplicity", "hit_to_tuple")
# capacities for events up to pileup 250 of the calibrated generator (PU250:
# ~86k hits, ~4.3M doublets, ~0.93M cells with tracks, ~0.61M tuples)
WIDE_CAPS = {"fed_words": 400000, "hits": 131072, "doublets": 6 << 20, "lists": 2 << 20, "tuples": (1 << 20) - 1,
             "multiplicity": (1 << 20) - 1, "hit_to_tuple": 1 << 20}


class Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("max_events", ctypes.c_uint32), ("max_words_per_batch", ctypes.c_uint32),
                ("slots", ctypes.c_uint32), ("use_graphs", ctypes.c_uint32), ("pool_words", ctypes.c_uint64),
                ("hbm_fraction", ctypes.c_double), ("riemann_fit", ctypes.c_uint32), ("vertex_algo", ctypes.c_uint32)] + \
        [(n, ctypes.c_uint32) for n in CA_FIELDS] + [("formatter_errors", ctypes.c_uint32), ("fed_scan", ctypes.c_uint32),
                                                      ("mixed_fit", ctypes.c_uint32)] + \
        [("cap_" + n, ctypes.c_uint32) for n in CAPS_FIELDS]


def tune_kernel_names():
    """The kernels whose launch shape the tuner sets."""
    out, i = [], 0
    while True:
        n = gpu_lib().pg_tune_kernel_name(i)
        if not n:
            return out
        out.append(n.decode())
        i += 1


def default_config():
    """pg_default_config as a dict (the reference's configuration)."""
    cfg = Config()
    gpu_lib().pg_default_config(ctypes.byref(cfg))
    return {n: getattr(cfg, n) for n, _ in Config._fields_}


class ResultView(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("n_tracks", "n_loose_all", "n_vertices", "n_hits", "n_tuples",
                                                "n_digis", "n_cells", "flags")] + \
        [(n, ctypes.c_void_p) for n in ("tuple_index", "track_n_hits", "quality", "state", "cov", "pt", "eta", "chi2",
                                        "hits", "vertex", "zv", "wv", "vchi2", "ptv2", "ndof", "sort_ind")]


class ServeConfig(ctypes.Structure):
    _fields_ = [("n_requests", ctypes.c_uint32), ("rate_hz", ctypes.c_double), ("seed", ctypes.c_uint64),
                ("max_batch", ctypes.c_uint32), ("upload_threads", ctypes.c_uint32)]


class ServeStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("completed", "batches", "max_batch_seen", "admission_waits")] + \
        [(n, ctypes.c_double) for n in ("wall_s", "events_per_s", "mean_batch", "offered_hz", "p50_ms", "p90_ms",
                                        "p99_ms", "mean_ms", "max_ms")]


class BatchSummary(ctypes.Structure):
    _fields_ = [("n_events", ctypes.c_uint32), ("flags", ctypes.c_uint32)] + \
        [(n, ctypes.c_uint64) for n in ("n_tracks", "n_vertices", "result_bytes", "n_digis", "n_modules", "n_hits",
                                        "n_cells", "n_edges", "n_tuples", "n_tuple_hits", "n_cut_margin",
                                        "n_flagged_events")]


class ProbeEntry(ctypes.Structure):
    _fields_ = [("kernel", ctypes.c_char_p), ("ms", ctypes.c_float)]


RESULT_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(ResultView))

# (field, dtype, elements per track / vertex)
_TRACK_FIELDS = [("tuple_index", np.uint32, 1), ("track_n_hits", np.uint8, 1), ("quality", np.uint8, 1),
                 ("state", np.float32, 5), ("cov", np.float32, 15), ("pt", np.float32, 1), ("eta", np.float32, 1),
                 ("chi2", np.float32, 1), ("hits", np.uint32, 5), ("vertex", np.int16, 1)]
_VERTEX_FIELDS = [("zv", np.float32), ("wv", np.float32), ("vchi2", np.float32), ("ptv2", np.float32),
                  ("ndof", np.int32), ("sort_ind", np.uint16)]


def result_from_view(v):
    """Copies a pg_result_view into numpy arrays."""
    out = {n: getattr(v, n) for n in ("n_tracks", "n_loose_all", "n_vertices", "n_hits", "n_tuples", "n_digis",
                                       "n_cells", "flags")}
    nt, nv = v.n_tracks, v.n_vertices
    for name, dt, k in _TRACK_FIELDS:
        nb = nt * k * np.dtype(dt).itemsize
        a = np.frombuffer(ctypes.string_at(getattr(v, name), nb), dtype=dt) if nb else np.zeros(0, dt)
        out[name] = a.reshape(nt, k) if k > 1 else a
    for name, dt in _VERTEX_FIELDS:
        nb = nv * np.dtype(dt).itemsize
        out[name] = np.frombuffer(ctypes.string_at(getattr(v, name), nb), dtype=dt) if nb else np.zeros(0, dt)
    return out


class EventCounts(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("n_words", "n_modules", "n_digi_errors", "n_hits", "n_cells",
                                                "n_tuples", "n_loose", "n_vertices", "flags", "n_cut_margin_doublets",
                                                "n_cut_margin_ca", "n_cut_margin_quality")]


def gpu_lib():
    """libpixgpu.so (built if missing)."""
    global _gpu
    if _gpu is None:
        _gpu = _load(os.path.join(LIB, "libpixgpu.so"), _build.build_gpu)
        _gpu.pg_create.argtypes = [ctypes.POINTER(ESImages), ctypes.POINTER(Config), ctypes.POINTER(ctypes.c_void_p)]
        _gpu.pg_destroy.argtypes = [ctypes.c_void_p]
        _gpu.pg_last_error.argtypes = [ctypes.c_void_p]
        _gpu.pg_last_error.restype = ctypes.c_char_p
        _gpu.pg_slot_bytes.argtypes = [ctypes.c_void_p]
        _gpu.pg_slot_bytes.restype = ctypes.c_size_t
        _gpu.pg_process_batch.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_char_p),
                                          ctypes.POINTER(ctypes.c_size_t)]
        _gpu.pg_stage_batch.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                                        ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_size_t)]
        _gpu.pg_run_staged.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        _gpu.pg_sync.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        _gpu.pg_slot_stream.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        _gpu.pg_slot_stream.restype = ctypes.c_void_p
        _gpu.pg_event_counts_get.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(EventCounts)]
        _gpu.pg_get_product.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_char_p, ctypes.c_void_p,
                                        ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int)]
        _gpu.pg_unpack_raw.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]
        _gpu.pg_fit_broken_line.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32] + [ctypes.c_void_p] * 2 + \
            [ctypes.c_double] + [ctypes.c_void_p] * 6
        _gpu.pg_fit_broken_line_mixed.argtypes = _gpu.pg_fit_broken_line.argtypes
        _gpu.pg_fit_riemann.argtypes = _gpu.pg_fit_broken_line.argtypes
        _gpu.pg_fit_riemann_mixed.argtypes = _gpu.pg_fit_broken_line.argtypes
        _gpu.pg_get_config.argtypes = [ctypes.c_void_p, ctypes.POINTER(Config)]
        _gpu.pg_default_config.argtypes = [ctypes.POINTER(Config)]
        _gpu.pg_submit.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_char_p),
                                   ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_uint32)]
        for f in ("pg_query", "pg_wait", "pg_release"):
            getattr(_gpu, f).argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        _gpu.pg_result.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(ResultView)]
        _gpu.pg_pool_put.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint32)]
        _gpu.pg_pool_release.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        _gpu.pg_pool_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                      ctypes.POINTER(ctypes.c_uint32)]
        _gpu.pg_submit_pooled.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32),
                                          ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]
        _gpu.pg_set_probe.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        _gpu.pg_tune_kernel_name.restype = ctypes.c_char_p
        _gpu.pg_tune_kernel_name.argtypes = [ctypes.c_uint32]
        _gpu.pg_tune_set.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_char_p, ctypes.c_int]
        _gpu.pg_tune_get.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
        _gpu.pg_autotune.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_char_p),
                                     ctypes.POINTER(ctypes.c_size_t), ctypes.c_uint32, ctypes.POINTER(ctypes.c_double)]
        _gpu.pg_tune_save.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        _gpu.pg_tune_load.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        _gpu.pg_batch_summary_get.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(BatchSummary)]
        _gpu.pg_probe_read.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(ProbeEntry),
                                       ctypes.POINTER(ctypes.c_uint32)]
        _gpu.pg_prepare.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        _gpu.pg_default_serve_config.argtypes = [ctypes.POINTER(ServeConfig)]
        _gpu.pg_serve.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_char_p),
                                  ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ServeConfig), ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.POINTER(ServeStats), ctypes.c_void_p, RESULT_FN,
                                  ctypes.c_void_p]
        _gpu.pg_vertices_noalloc.argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_uint32] + [ctypes.c_void_p] * 10 + \
            [ctypes.c_char_p, ctypes.c_size_t]
    return _gpu


NOALLOC_MAX_TUPLES = 32767   # pg_vertices_noalloc's static scratch limit
NOALLOC_VERTEX_SLOTS = 1024  # entries of the per-vertex outputs (ZVertexSoA::MAXVTX)


def vertices_noalloc(tuple_off, quality, pt, state, cov, idv, zv, wv, chi2, ptv2, ndof, sort_ind, stream=None):
    """pg_vertices_noalloc on device tensors (torch): one event's track SoA in,
    the vertices out; returns (n_vertices, flags).  Allocates nothing on the
    device; raises with the library's message on failure.

    Every tensor must be a contiguous CUDA tensor on the same device, with the
    dtype and length the C entry point reads or writes: n = quality.numel()
    tuples, tuple_off >= n + 1 (uint32 as int32), pt >= n, state >= 5n,
    cov >= 15n, idv >= n (int16), and the per-vertex outputs at least 1024
    entries.  The call runs on `stream` (a CUDA stream handle), by default on
    torch's current stream of that device."""
    import torch
    n = int(quality.numel())
    if n > NOALLOC_MAX_TUPLES:
        raise ValueError("vertices_noalloc: %d tuples above the limit of %d" % (n, NOALLOC_MAX_TUPLES))
    spec = (("tuple_off", tuple_off, (torch.int32,), n + 1), ("quality", quality, (torch.uint8,), n),
            ("pt", pt, (torch.float32,), n), ("state", state, (torch.float32,), 5 * n),
            ("cov", cov, (torch.float32,), 15 * n), ("idv", idv, (torch.int16,), n),
            ("zv", zv, (torch.float32,), NOALLOC_VERTEX_SLOTS), ("wv", wv, (torch.float32,), NOALLOC_VERTEX_SLOTS),
            ("chi2", chi2, (torch.float32,), NOALLOC_VERTEX_SLOTS),
            ("ptv2", ptv2, (torch.float32,), NOALLOC_VERTEX_SLOTS),
            ("ndof", ndof, (torch.int32,), NOALLOC_VERTEX_SLOTS),
            ("sort_ind", sort_ind, (torch.int16, torch.uint16), NOALLOC_VERTEX_SLOTS))
    dev = quality.device
    if dev.type != "cuda":
        raise ValueError("vertices_noalloc: tensors must be on a CUDA device")
    for name, t, dtypes, need in spec:
        if t.device != dev:
            raise ValueError("vertices_noalloc: %s is on %s, quality on %s" % (name, t.device, dev))
        if t.dtype not in dtypes:
            raise ValueError("vertices_noalloc: %s has dtype %s, expected %s" % (name, t.dtype, dtypes[0]))
        if not t.is_contiguous():
            raise ValueError("vertices_noalloc: %s is not contiguous" % name)
        if t.numel() < need:
            raise ValueError("vertices_noalloc: %s has %d entries, needs %d" % (name, t.numel(), need))
    nv = ctypes.c_uint32()
    fl = ctypes.c_uint32()
    msg = ctypes.create_string_buffer(256)
    with torch.cuda.device(dev):
        if stream is None:
            stream = torch.cuda.current_stream(dev).cuda_stream
        rc = gpu_lib().pg_vertices_noalloc(tuple_off.data_ptr(), quality.data_ptr(), pt.data_ptr(),
                                           state.data_ptr(), cov.data_ptr(), n, idv.data_ptr(), zv.data_ptr(),
                                           wv.data_ptr(), chi2.data_ptr(), ptv2.data_ptr(), ndof.data_ptr(),
                                           sort_ind.data_ptr(), ctypes.addressof(nv), ctypes.addressof(fl), stream,
                                           msg, len(msg))
    if rc != 0:
        raise RuntimeError("pg_vertices_noalloc failed (%d): %s" % (rc, msg.value.decode()))
    return nv.value, fl.value


def _raw_arrays(raws):
    n = len(raws)
    ptrs = (ctypes.c_char_p * n)(*raws)
    sizes = (ctypes.c_size_t * n)(*[len(r) for r in raws])
    return ptrs, sizes


class Chain:
    """A device context: resident conditions plus batch slots."""

    def __init__(self, es_images, max_events=64, max_words_per_batch=None, slots=1, device=0, use_graphs=True,
                 pool_words=0, hbm_fraction=0.5, riemann_fit=False, vertex_algo=0, ca=None, formatter_errors=False,
                 fed_scan="host", caps=None, mixed_fit=False):
        """ca: CAHitNtupletGeneratorOnGPU parameters overriding the reference's (pg_config field
        names: min_hits_per_ntuplet, include_jumping_forward_doublets, early_fishbone, late_fishbone,
        ideal_conditions, do_cluster_cut, do_z0_cut, do_pt_cut).  formatter_errors: record the FED
        loop's framing errors ("formatterErrors").  fed_scan: "host", or "device" for the header and
        trailer checks and the word concatenation on the GPU.  caps: per-event container capacities
        (CAPS_FIELDS names, e.g. WIDE_CAPS) above the reference's.  mixed_fit: the chain's fit in its
        mixed-precision variant (FP32 with FP64 Cholesky solves and covariance) instead of FP64."""
        lib = gpu_lib()
        self._keep = list(es_images)
        img = ESImages(*[x for b in self._keep for x in (b, len(b))])
        if max_words_per_batch is None:
            max_words_per_batch = max_events * 160000
        cfg = Config()
        lib.pg_default_config(ctypes.byref(cfg))
        cfg.device, cfg.max_events, cfg.max_words_per_batch, cfg.slots = device, max_events, max_words_per_batch, slots
        cfg.use_graphs, cfg.pool_words, cfg.hbm_fraction = 1 if use_graphs else 0, pool_words, hbm_fraction
        cfg.riemann_fit, cfg.vertex_algo = 1 if riemann_fit else 0, int(vertex_algo)
        cfg.formatter_errors = 1 if formatter_errors else 0
        cfg.mixed_fit = 1 if mixed_fit else 0
        if fed_scan not in ("host", "device"):
            raise ValueError("fed_scan: 'host' or 'device'")
        cfg.fed_scan = 1 if fed_scan == "device" else 0
        for k, v in (ca or {}).items():
            if k not in CA_FIELDS:
                raise ValueError("unknown CA parameter %s" % k)
            setattr(cfg, k, int(v))
        for k, v in (caps or {}).items():
            if k not in CAPS_FIELDS:
                raise ValueError("unknown capacity %s" % k)
            setattr(cfg, "cap_" + k, int(v))
        self._h = ctypes.c_void_p()
        rc = lib.pg_create(ctypes.byref(img), ctypes.byref(cfg), ctypes.byref(self._h))
        if rc != 0:
            raise RuntimeError("pg_create failed with status %d" % rc)
        got = Config()
        lib.pg_get_config(self._h, ctypes.byref(got))
        self.max_events = max_events
        self.slots = got.slots

    def _check(self, rc, what):
        if rc != 0:
            msg = gpu_lib().pg_last_error(self._h)
            raise RuntimeError("%s failed (%d): %s" % (what, rc, msg.decode() if msg else ""))

    def process(self, raws):
        ptrs, sizes = _raw_arrays(raws)
        self._check(gpu_lib().pg_process_batch(self._h, len(raws), ptrs, sizes), "pg_process_batch")

    def stage(self, raws, slot=0):
        ptrs, sizes = _raw_arrays(raws)
        self._check(gpu_lib().pg_stage_batch(self._h, slot, len(raws), ptrs, sizes), "pg_stage_batch")

    def run_staged(self, slot=0):
        self._check(gpu_lib().pg_run_staged(self._h, slot), "pg_run_staged")

    def sync(self, slot=0):
        self._check(gpu_lib().pg_sync(self._h, slot), "pg_sync")

    def stream(self, slot=0):
        return gpu_lib().pg_slot_stream(self._h, slot)

    def counts(self, k):
        c = EventCounts()
        self._check(gpu_lib().pg_event_counts_get(self._h, k, ctypes.byref(c)), "pg_event_counts_get")
        return {n: getattr(c, n) for n, _ in EventCounts._fields_}

    def product(self, k, name):
        lib = gpu_lib()
        count = ctypes.c_size_t()
        elem = ctypes.c_int()
        self._check(lib.pg_get_product(self._h, k, name.encode(), None, 0, ctypes.byref(count), ctypes.byref(elem)),
                    "pg_get_product(%s)" % name)
        buf = ctypes.create_string_buffer(max(1, count.value * elem.value))
        self._check(lib.pg_get_product(self._h, k, name.encode(), buf, len(buf), ctypes.byref(count),
                                       ctypes.byref(elem)), "pg_get_product(%s)" % name)
        return _as_array(buf.raw[:count.value * elem.value], name, elem.value)

    def products(self, k):
        """All products of event k in the oracle's naming, CA lists capped as in the reference."""
        out = {}
        for n in SCALARS:
            out[n] = self.product(k, n)
        for n in ["xx", "yy", "adc", "moduleInd", "clus", "pdigi", "rawIdArr", "errors", "formatterErrors", "moduleStart",
                  "clusInModule",
                  "moduleId", "clusModuleStart", "xl", "yl", "xerr", "yerr", "xg", "yg", "zg", "rg", "charge", "iphi",
                  "xsize", "ysize", "detInd", "cellInner", "cellOuter", "cellLayerPair", "cellDoubletId", "cellUsed",
                  "tupleOff", "tupleHits", "tupleDet", "quality", "state", "cov", "pt", "eta", "chi2", "zv", "wv",
                  "vchi2", "ptv2", "ndof", "sortInd", "idv"]:
            out[n] = self.product(k, n)
        if out["nHits"]:
            for n in ["hitsLayerStart", "phiOff", "phiBins"]:
                out[n] = self.product(k, n)
        out["cellLayerPair"] = out["cellLayerPair"].view(np.uint8).astype(np.int16)
        out["cellUsed"] = out["cellUsed"].view(np.uint8).astype(np.uint16)
        # CSR lists with the reference's per-object capacities
        def capped(off, val, cap):
            off = off.astype(np.int64)
            sizes = np.minimum(np.diff(off), cap)
            newoff = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
            # source position of every kept entry: its segment's start plus its rank
            pos = np.arange(newoff[-1]) - np.repeat(newoff[:-1] - off[:-1], sizes)
            return newoff.astype(np.uint32), val[pos].astype(val.dtype)
        out["outerHitOff"], out["outerHitCells"] = capped(self.product(k, "outerHitOffRaw"),
                                                          self.product(k, "outerHitCellsRaw"), 128)
        if out["nHits"] == 0:
            out["outerHitOff"] = np.zeros(1, np.uint32)
        out["cellNbrOff"], out["cellNbr"] = capped(self.product(k, "cellNbrOffRaw"), self.product(k, "cellNbrRaw"), 36)
        out["cellTrkOff"], out["cellTrk"] = capped(self.product(k, "cellTrkOffRaw"), self.product(k, "cellTrkRaw"), 48)
        return out

    # ------------------------------------------------------------ asynchronous batches
    def submit(self, raws):
        """Launches a batch on a free slot and returns the slot (None when all are busy)."""
        ptrs, sizes = _raw_arrays(raws)
        slot = ctypes.c_uint32()
        rc = gpu_lib().pg_submit(self._h, len(raws), ptrs, sizes, ctypes.byref(slot))
        if rc == -5:
            return None
        self._check(rc, "pg_submit")
        return slot.value

    def query(self, slot):
        rc = gpu_lib().pg_query(self._h, slot)
        if rc == -5:
            return False
        self._check(rc, "pg_query")
        return True

    def wait(self, slot):
        self._check(gpu_lib().pg_wait(self._h, slot), "pg_wait")

    def result(self, slot, k):
        v = ResultView()
        self._check(gpu_lib().pg_result(self._h, slot, k, ctypes.byref(v)), "pg_result")
        return result_from_view(v)

    def summary(self, slot):
        """Totals over the finished batch on `slot` (result bytes, event counts)."""
        b = BatchSummary()
        self._check(gpu_lib().pg_batch_summary_get(self._h, slot, ctypes.byref(b)), "pg_batch_summary_get")
        return {n: getattr(b, n) for n, _ in BatchSummary._fields_}

    def release(self, slot):
        self._check(gpu_lib().pg_release(self._h, slot), "pg_release")

    # ------------------------------------------------------------ device-resident pool
    def pool_put(self, raw):
        """Admits one event into the pool; None when the pool has no room now."""
        h = ctypes.c_uint32()
        rc = gpu_lib().pg_pool_put(self._h, raw, len(raw), ctypes.byref(h))
        if rc in (-5, -6):
            return None
        self._check(rc, "pg_pool_put")
        return h.value

    def pool_release(self, handle):
        self._check(gpu_lib().pg_pool_release(self._h, handle), "pg_pool_release")

    def pool_info(self):
        cap, free, live = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint32()
        self._check(gpu_lib().pg_pool_info(self._h, ctypes.byref(cap), ctypes.byref(free), ctypes.byref(live)),
                    "pg_pool_info")
        return {"cap_words": cap.value, "free_words": free.value, "live_events": live.value}

    def submit_pooled(self, handles, keep=False):
        """Gathers pooled events into a free slot and launches; None when all slots are busy.
        keep=True leaves the events resident for later batches."""
        arr = (ctypes.c_uint32 * len(handles))(*handles)
        slot = ctypes.c_uint32()
        rc = gpu_lib().pg_submit_pooled(self._h, len(handles), arr, 1 if keep else 0, ctypes.byref(slot))
        if rc == -5:
            return None
        self._check(rc, "pg_submit_pooled")
        return slot.value

    def set_probe(self, kernel):
        """Times every launch of `kernel` ("*" = all kernels, None = off) from now on."""
        self._check(gpu_lib().pg_set_probe(self._h, kernel.encode() if kernel else None), "pg_set_probe")

    def probe_read(self, slot):
        """[(kernel, ms)] of the timed launches of the last finished batch on `slot`."""
        buf = (ProbeEntry * 256)()
        n = ctypes.c_uint32()
        self._check(gpu_lib().pg_probe_read(self._h, slot, 256, buf, ctypes.byref(n)), "pg_probe_read")
        return [(buf[i].kernel.decode(), buf[i].ms) for i in range(n.value)]

    def tune_set(self, n_events, kernel, scale):
        """Grid scale of one tunable kernel for batches of n_events (default grid x 2^scale)."""
        self._check(gpu_lib().pg_tune_set(self._h, n_events, kernel.encode(), int(scale)), "pg_tune_set")

    def tune_table(self, n_events):
        """{kernel: scale} in force for batches of n_events."""
        out = {}
        for name in tune_kernel_names():
            v = ctypes.c_int()
            self._check(gpu_lib().pg_tune_get(self._h, n_events, name.encode(), ctypes.byref(v)), "pg_tune_get")
            out[name] = v.value
        return out

    def autotune(self, raws, repeats=3):
        """Tunes the launches for batches of len(raws) events; returns the saving per batch in ms."""
        ptrs, sizes = _raw_arrays(raws)
        gain = ctypes.c_double()
        self._check(gpu_lib().pg_autotune(self._h, len(raws), ptrs, sizes, repeats, ctypes.byref(gain)),
                    "pg_autotune")
        return gain.value

    def tune_save(self, path):
        self._check(gpu_lib().pg_tune_save(self._h, path.encode()), "pg_tune_save")

    def tune_load(self, path):
        """Applies the cache entries of this device; returns how many."""
        n = gpu_lib().pg_tune_load(self._h, path.encode())
        if n < 0:
            self._check(n, "pg_tune_load")
        return n

    def prepare(self, max_batch=0):
        self._check(gpu_lib().pg_prepare(self._h, max_batch), "pg_prepare")

    def serve(self, raws, n_requests, rate_hz=None, arrivals=None, request_event=None, max_batch=0, seed=1,
              upload_threads=2, on_result=None):
        """Runs the serving loop; returns (stats dict, per-request latency seconds)."""
        lib = gpu_lib()
        ptrs, sizes = _raw_arrays(raws)
        cfg = ServeConfig()
        lib.pg_default_serve_config(ctypes.byref(cfg))
        cfg.n_requests = n_requests
        if rate_hz is not None:
            cfg.rate_hz = rate_hz
        cfg.seed = seed
        cfg.max_batch = max_batch
        cfg.upload_threads = upload_threads
        arr = None
        if arrivals is not None:
            arr = np.ascontiguousarray(arrivals, dtype=np.float64)
            assert arr.shape == (n_requests,)
        rev = None
        if request_event is not None:
            rev = np.ascontiguousarray(request_event, dtype=np.uint32)
            assert rev.shape == (n_requests,)
        lat = np.zeros(n_requests, dtype=np.float64)
        st = ServeStats()
        fn = RESULT_FN(0)
        if on_result is not None:
            fn = RESULT_FN(lambda user, req, ev, view: on_result(req, ev, result_from_view(view.contents)))
        rc = lib.pg_serve(self._h, len(raws), ptrs, sizes, ctypes.byref(cfg),
                          arr.ctypes.data if arr is not None else None, rev.ctypes.data if rev is not None else None,
                          ctypes.byref(st), lat.ctypes.data, fn, None)
        self._check(rc, "pg_serve")
        return {n: getattr(st, n) for n, _ in ServeStats._fields_}, lat

    def fit(self, N, hits, ge, B=B_FIELD, mixed=False, riemann=False):
        """Broken-line fit of host arrays hits[n, N, 3] (f64), ge[n, N, 6] (f32) on the device;
        mixed=True runs the FP32 variant with FP64 Cholesky solves and covariance propagation;
        riemann=True runs the Riemann fit instead (with mixed=True, its mixed-precision variant)."""
        import torch
        n = hits.shape[0]
        dh = torch.from_numpy(np.ascontiguousarray(hits[:, :N, :])).cuda()
        dg = torch.from_numpy(np.ascontiguousarray(ge[:, :N, :])).cuda()
        st = torch.empty((n, 5), dtype=torch.float32, device="cuda")
        cv = torch.empty((n, 15), dtype=torch.float32, device="cuda")
        pt = torch.empty(n, dtype=torch.float32, device="cuda")
        eta = torch.empty(n, dtype=torch.float32, device="cuda")
        chi2 = torch.empty(n, dtype=torch.float32, device="cuda")
        s = torch.cuda.current_stream().cuda_stream
        if riemann and mixed:
            fn, name = gpu_lib().pg_fit_riemann_mixed, "pg_fit_riemann_mixed"
        elif riemann:
            fn, name = gpu_lib().pg_fit_riemann, "pg_fit_riemann"
        elif mixed:
            fn, name = gpu_lib().pg_fit_broken_line_mixed, "pg_fit_broken_line_mixed"
        else:
            fn, name = gpu_lib().pg_fit_broken_line, "pg_fit_broken_line"
        self._check(fn(self._h, N, n, dh.data_ptr(), dg.data_ptr(), B, st.data_ptr(), cv.data_ptr(), pt.data_ptr(),
                       eta.data_ptr(), chi2.data_ptr(), s), name)
        torch.cuda.synchronize()
        return {"state": st.cpu().numpy(), "cov": cv.cpu().numpy(), "pt": pt.cpu().numpy(), "eta": eta.cpu().numpy(),
                "chi2": chi2.cpu().numpy()}

    def cluster_digis(self, module_ind, xx, yy, adc):
        """pg_cluster_digis: countModules, findClus and clusterChargeCut on given digis
        (module index, row, column, calibrated charge); returns a dict of arrays."""
        lib = gpu_lib()
        n = len(module_ind)
        arrs = [np.ascontiguousarray(a, dtype=np.uint16) for a in (module_ind, xx, yy, adc)]
        out = {"moduleInd": np.zeros(n, np.uint16), "clus": np.zeros(n, np.int32),
               "clusInModule": np.zeros(2000, np.uint32), "moduleId": np.zeros(2000, np.uint32),
               "moduleStart": np.zeros(2001, np.uint32)}
        nm, fl = ctypes.c_uint32(), ctypes.c_uint32()
        lib.pg_cluster_digis.argtypes = [ctypes.c_void_p, ctypes.c_uint32] + [ctypes.c_void_p] * 11
        self._check(lib.pg_cluster_digis(self._h, n, *[a.ctypes.data for a in arrs],
                                         *[out[k].ctypes.data for k in ("moduleInd", "clus", "clusInModule",
                                                                        "moduleId", "moduleStart")],
                                         ctypes.byref(nm), ctypes.byref(fl)), "pg_cluster_digis")
        out["nModules"], out["flags"] = nm.value, fl.value
        return out

    def slot_bytes(self):
        """Device bytes of one batch slot (pg_slot_bytes)."""
        return int(gpu_lib().pg_slot_bytes(self._h))

    def close(self):
        if self._h:
            gpu_lib().pg_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
