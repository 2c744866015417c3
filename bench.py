#!/usr/bin/env python
"""Throughput and latency of the B200 pixel reconstruction chain at PU50.

One JSON line (rank 0):
  value      events/s of the batched chain (64 events per launch sequence,
             captured CUDA graph), inputs resident in a device pool when the
             timed region starts, results packed into mapped host memory;
  e2e        the same through the public C ABI (pg_submit) from host raw
             records: FED scan on the host, H2D of the words, chain, results
             written to host memory, every step inside the timed region;
  per_event  the plain one-event-per-launch chain (no graph), for the
             batched-vs-per-event ratio, with its per-event latency p50/p99;
  serving    the continuous-batching serving loop (pg_serve): Poisson
             arrivals swept over the offered load, p50/p99 latency from
             arrival to completion, and the highest sustained rate whose p99
             stays under 5 ms (over 6, 4 and 3 batches in flight) against the
             best per-event rate;
  batched_mixed_pu, serving_mixed_pu
             the uneven-pileup configurations (PU uniform 20-200 per 64-event
             batch; PU log-uniform 30-250 served at 10-100 kHz) with the
             container capacities widened for them, and their capacity flags;
  dense_pu50 the batched rate on the denser event model (every track prompt
             and above 0.5 GeV: ~3x the doublets of the calibrated one);
  roofline   the dominant kernel (largest share of device time, found by a
             timed census of every kernel) against the measured HBM copy
             bandwidth, its duration measured with timing events captured
             into the graphs of the timed region;
  cpu_baseline  the reference's serial chain (checker build of its own
             sources, or the oracle port when that build is absent) on the
             host cores.

`--impl reference` times the reference's CPU implementation of the chain on
the same workload and prints the same line with "impl": "reference".

Multi-GPU (torchrun): replicas, one process per GPU, each running the same
per-GPU workload; value = all events / max-over-ranks time ("scaling": "weak").
"""
import argparse
import collections
import concurrent.futures as cf
import json
import os
import shutil
import struct
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "pixeltrack-standalone_b200")
TUNE_CACHE = os.path.join(PKG, "tuning", "launch_tuning.txt")
sys.path.insert(0, PKG)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import replicas  # noqa: E402

METRIC = "events/s and p50/p99 latency at PU50: batched serving vs per-event chain, one B200"
DATA = ("synthetic: seeded Phase-1 pixel events (1856 modules, 108 FEDs, helices in 3.8 T, Landau charge; "
        "calibrated event model: prompt power-law tracks above 0.5 GeV plus a soft, mostly displaced component), "
        "PU50 ~57k digis, ~18k hits, ~1.6k loose tracks per event, packed into FED words through the generated "
        "cabling map")
PU = 50
SEED0 = 20261203

# Algorithmic bytes per unit of each kernel (each column read once by the
# consuming stage and written once at its declared width; ES tables resident
# and excluded).  Units: W digis (FED words), H hits, C doublets, E CA links,
# Sh hits over tuples, N tuples, M active modules.
KERNEL_BYTES = {
    "kRawToDigi": lambda u: 50.5 * u["W"],            # raw-to-digi 38.5*W + calibration 12*W (fused)
    "kModuleBoundaries": lambda u: 6.0 * u["W"],
    "kFindClusters": lambda u: 24.0 * u["W"],         # findClus 10*W + charge cut 14*W (fused)
    "kGetHits": lambda u: 12.0 * u["W"] + 44.0 * u["H"] + 112.0 * u["M"],
    # doublets: the count pass reads each hit's packed record and writes each
    # doublet's outer hit once (staged); the write pass the doublet columns
    "kDoubletCount": lambda u: 16.0 * u["H"] + 4.0 * u["C"],
    "kDoubletWrite": lambda u: 14.0 * u["H"] + 44.0 * u["C"],
    "kConnect": lambda u: 40.0 * u["C"] + 8.0 * u["E"],
    "kFishbone": lambda u: 16.0 * u["C"],
    "kNtupletWrite": lambda u: 2.0 * u["Sh"] + 9.0 * u["N"],
    "kBLFit": lambda u: 68.0 * u["Sh"] + 92.0 * u["N"],
    "kVertices": lambda u: 16.0 * u["N"],
    # list ordering: read + write of every ordered entry (cells by outer hit,
    # CA links, tracks per cell, tuples per hit)
    "kSortSegments": lambda u: 2 * (4.0 * u["C"] + 4.0 * u["E"] + 2.0 * u["Sh"] + 2.0 * u["Sh"]),
}


# DRAM bytes per event of a kernel (dram__bytes_read.sum + dram__bytes_write.sum
# of one ncu capture on 16 PU50 events, divided by 16; traffic scales with the
# events of a launch), from the full-set captures of these kernels
NCU_DRAM_BYTES_PER_EVENT = {"kConnect": 4.39e6, "kDoubletCount": 0.46e6, "kFishbone": 2.51e6, "kNtupletCount": 1.83e6}


def chain_bytes(u):
    """Whole-chain algorithmic bytes: 92.5 W + 64 H + 100 C + 8 E + 76 Sh + 42 N + 92 T (T = N fitted)."""
    return 92.5 * u["W"] + 64 * u["H"] + 100 * u["C"] + 8 * u["E"] + 76 * u["Sh"] + 42 * u["N"] + 92 * u["N"]


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--batch", type=int, default=64, help="events per launch sequence")
    p.add_argument("--events", type=int, default=1000, help="distinct PU50 events (inputs > L2)")
    p.add_argument("--slots", type=int, default=4, help="batches in flight")
    p.add_argument("--per-event", type=int, default=256, help="events for the one-event-per-launch leg")
    p.add_argument("--serve", type=int, default=4000, help="requests for the serving leg (0: skip)")
    p.add_argument("--serve-batch", type=int, default=32, help="max events per serving batch")
    p.add_argument("--serve-slots", type=int, default=6, help="batches in flight in the serving loop")
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="target length of the CPU baseline sample")
    p.add_argument("--serve-mixed", type=int, default=2000, help="requests per uneven-pileup serving point (0: skip)")
    p.add_argument("--mixed-batches", type=int, default=3,
                   help="distinct 64-event batches with PU uniform in [20, 200] (0: skip that leg)")
    p.add_argument("--tune-out", default="", help="where to write the table --autotune finds")
    p.add_argument("--autotune", action="store_true",
                   help="tune the launch shapes now (else load the committed cache) and write the table")
    return p.parse_args()


# ----------------------------------------------------------------------------- helpers
def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


def make_events(det, n, pu=PU, base=SEED0 + 100000, model="calibrated"):
    """n distinct seeded events, generated on all host cores."""
    with cf.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        return list(ex.map(lambda k: det.event(base + k, pu, model=model), range(n)))


class Clocks:
    """nvidia-smi samples during a timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.out.close()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


# capacities for the 64-event batches of PU uniform in [20, 200] (calibrated
# model, PU200: ~68k hits, ~2.8M doublets, ~0.5M cells with tracks, ~0.33M tuples)
PU200_CAPS = {"fed_words": 300000, "hits": 98304, "doublets": 4 << 20, "lists": 1 << 20, "tuples": 512 * 1024,
              "multiplicity": 512 * 1024, "hit_to_tuple": 1 << 19}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def units_of(summary):
    return {"W": summary["n_digis"], "H": summary["n_hits"], "C": summary["n_cells"], "E": summary["n_edges"],
            "Sh": summary["n_tuple_hits"], "N": summary["n_tuples"], "M": summary["n_modules"]}


# ----------------------------------------------------------------------------- reference arm
def run_reference(a):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle
    import pixgpu
    det = pixgpu.Detector()
    cores = os.cpu_count() or 1
    n_distinct = 64
    raws = make_events(det, n_distinct)
    if oracle.ref_available():
        kind = "reference"
        d = tempfile.mkdtemp()
        det.write(d)
        timer = lambda evs: oracle.ref_time_events(d, evs, cores)[0]  # noqa: E731
    else:
        kind = "port"
        orc = oracle.Oracle(det.es)
        timer = lambda evs: orc.time_events(evs, cores)[0]  # noqa: E731
    # pilot: size each step so that the whole run stays within a few minutes
    pilot = timer(raws[:min(len(raws), 2 * cores)])
    rate = min(len(raws), 2 * cores) / pilot
    per_step = int(max(cores, min(n_distinct, rate * 120.0 / max(1, a.steps + a.warmup))))
    for i in range(a.warmup):
        timer([raws[(i * per_step + k) % n_distinct] for k in range(per_step)])
    tot = 0.0
    for i in range(a.steps):
        tot += timer([raws[(i * per_step + k) % n_distinct] for k in range(per_step)])
    value = a.steps * per_step / tot
    line = {"metric": METRIC, "value": value, "unit": "events/s", "impl": "reference", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * tot / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u16/u32 int, f32 hits and cuts, f64 fits",
            "data": DATA,
            "config": {"workload": "PU50 pixel chain, events processed on host threads (one chain instance "
                                   "per thread, the reference's event-level concurrency)",
                       "pu": PU, "events_per_step": per_step, "distinct_events": n_distinct},
            "cpu_baseline": {"value": value, "unit": "events/s", "cores": cores, "kind": kind,
                             "sample": "%d PU50 events per step x %d steps" % (per_step, a.steps)},
            "e2e": {"value": value, "unit": "events/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- our arm
def pipeline(chain, torch, n_steps, submit, on_done):
    """Runs n_steps submissions over the chain's slots, keeping every slot busy;
    returns device milliseconds between a start event joined into every slot
    stream and an end event joined from all of them."""
    streams = [torch.cuda.ExternalStream(chain.stream(s)) for s in range(chain.slots)]
    side = torch.cuda.Stream()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record(side)
    for s in streams:
        s.wait_event(start)
    inflight = collections.deque()
    for i in range(n_steps):
        while True:
            slot = submit(i)
            if slot is not None:
                break
            s0 = inflight.popleft()
            chain.wait(s0)
            on_done(s0)
            chain.release(s0)
        inflight.append(slot)
    while inflight:
        s0 = inflight.popleft()
        chain.wait(s0)
        on_done(s0)
        chain.release(s0)
    for s in streams:
        e = torch.cuda.Event()
        e.record(s)
        side.wait_event(e)
    end.record(side)
    end.synchronize()
    return start.elapsed_time(end)


def fit_leg(det, dev, torch, n=1000000):
    """1M seeded MS-smeared tuples of 3 and of 4 hits: broken-line and Riemann
    fits per second in FP64 (the reference's precision) and in their
    mixed-precision variants, and each variant's deviation from its FP64
    result (max and rms over the tuples)."""
    import pixgpu
    c = pixgpu.Chain(det.es, max_events=1, max_words_per_batch=300000, device=dev)
    lib = pixgpu.gpu_lib()
    methods = {"broken_line": (lib.pg_fit_broken_line, lib.pg_fit_broken_line_mixed),
               "riemann": (lib.pg_fit_riemann, lib.pg_fit_riemann_mixed)}
    res = {}
    for nh in (3, 4):
        hits, ge, _ = pixgpu.fit_tuples(20261203 + nh, n, nh)
        dh = torch.from_numpy(np.ascontiguousarray(hits)).cuda()
        dg = torch.from_numpy(np.ascontiguousarray(ge)).cuda()
        per = {}
        for method, fns in methods.items():
            outs = {}
            rates = {}
            for label, fn in zip(("fp64", "mixed"), fns):
                o = [torch.empty(n * k, dtype=torch.float32, device="cuda") for k in (5, 15, 1, 1, 1)]
                st = torch.cuda.current_stream().cuda_stream
                args = (c._h, nh, n, dh.data_ptr(), dg.data_ptr(), pixgpu.B_FIELD, *[x.data_ptr() for x in o], st)
                for _ in range(2):
                    if fn(*args) != 0:
                        raise RuntimeError("fit launch failed")
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record()
                for _ in range(5):
                    fn(*args)
                e1.record()
                e1.synchronize()
                rates[label] = n / (e0.elapsed_time(e1) / 5 / 1e3)
                outs[label] = [x.cpu().numpy().astype(np.float64) for x in o]
            sa, sb = outs["fp64"][0].reshape(n, 5), outs["mixed"][0].reshape(n, 5)
            cov = outs["fp64"][1].reshape(n, 15)
            fin = np.isfinite(sa).all(axis=1) & np.isfinite(sb).all(axis=1)
            dk = np.abs(1 / outs["mixed"][2] - 1 / outs["fp64"][2])[fin]
            vk = np.abs(1 / outs["fp64"][2])[fin]
            d = np.abs(sb - sa)[fin]
            # packed symmetric 5x5 covariance: diagonal entries 0, 2, 5, 9, 14
            sig = np.sqrt(np.maximum(cov[fin][:, [0, 2, 5, 9, 14]], 0.0))
            err = {"inv_pt_per_gev": (dk, vk, sig[:, 2]), "phi": (d[:, 0], np.abs(sa[fin][:, 0]), sig[:, 0]),
                   "d0_cm": (d[:, 1], np.abs(sa[fin][:, 1]), sig[:, 1]),
                   "cot_theta": (d[:, 3], np.abs(sa[fin][:, 3]), sig[:, 3]),
                   "z0_cm": (d[:, 4], np.abs(sa[fin][:, 4]), sig[:, 4])}

            def stats(v, ref, sg):
                rel = v / np.maximum(ref, 1e-30)
                pull = v / np.maximum(sg, 1e-30)
                return {"max": float(v.max()), "rms": float(np.sqrt((v ** 2).mean())),
                        "frac_rel_over_1e-5": float((rel > 1e-5).mean()),
                        "rel_p999": float(np.quantile(rel, 0.999)),
                        "max_over_fp64_sigma": float(pull.max()), "p9999_over_fp64_sigma": float(np.quantile(pull, 0.9999))}
            per[method] = {"fits_per_s": rates, "both_finite": int(fin.sum()),
                           "mixed_vs_fp64": {k: stats(*v) for k, v in err.items()}}
        res["%d_hits" % nh] = per
    c.close()
    return {"tuples": n, "per_multiplicity": res,
            "mixed": {"broken_line": "FP32 arithmetic; FP64 for the reference circle, radial residuals, Cholesky "
                                     "solves and covariance propagation",
                      "riemann": "FP32 for the multiple-scattering models, the s-z projection and the "
                                 "single-precision eigen-solves of the numerical Jacobian; FP64 for the prefit "
                                 "circle, the radiation-length path lengths, the Riemann matrix and its smallest "
                                 "eigenvector, the Cholesky solves and the covariance propagation"}}


def run_ours(a):
    import torch
    import pixgpu
    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)
    dev = local
    B = a.batch
    det = pixgpu.Detector()
    # each rank its own distinct events (replicas, weak scaling)
    raws = make_events(det, a.events, base=replicas.shard_seeds(rank, world, a.events, SEED0 + 100000)[0])
    nw = [len(r) // 4 for r in raws]  # upper bound of FED words per event
    max_words = int(max(nw)) * B + 1024
    input_bytes = sum(len(r) for r in raws)

    # ------------------------------------------------------------ batched, device-resident
    chain = pixgpu.Chain(det.es, max_events=B, max_words_per_batch=max_words, slots=a.slots, device=dev,
                         pool_words=sum(nw) + 64 * len(nw) + 4096)
    tuning = apply_tuning(chain, B, raws, a)
    handles = []
    for r in raws:
        h = chain.pool_put(r)
        while h is None:  # staging buffers in flight
            time.sleep(0.001)
            h = chain.pool_put(r)
        handles.append(h)
    nb = len(handles) // B
    batches = [handles[(i % nb) * B:(i % nb) * B + B] for i in range(max(nb, 1))]

    # census: every kernel timed once, to find the dominant one
    chain.set_probe("*")
    s = chain.submit_pooled(batches[0], keep=True)
    chain.wait(s)
    census = collections.defaultdict(float)
    launches = collections.Counter()
    for name, ms in chain.probe_read(s):
        census[name] += ms
        launches[name] += 1
    sums = chain.summary(s)
    chain.release(s)
    launches_per_batch = sum(launches.values()) + 1  # + the pool gather
    total_ms = sum(census.values())
    top = max(census, key=census.get)
    chain.set_probe(top)
    chain.prepare(B)

    probe_ms = []
    units = collections.Counter()
    result_bytes = [0]

    margins = collections.Counter()

    def done(slot):
        probe_ms.extend(ms for _, ms in chain.probe_read(slot))
        sm = chain.summary(slot)
        units.update(units_of(sm))
        result_bytes[0] += sm["result_bytes"]
        margins.update({"cut_decisions_on_boundary": sm["n_cut_margin"], "flagged_events": sm["n_flagged_events"]})

    sub = lambda i: chain.submit_pooled(batches[i % len(batches)], keep=True)  # noqa: E731
    pipeline(chain, torch, a.warmup, sub, lambda s: None)
    probe_ms.clear()
    with Clocks(dev) as clk:
        ms = pipeline(chain, torch, a.steps, sub, done)
    clocks = clk.summary()
    events = a.steps * B
    value, ms = replicas.job_rate(events, ms, device="cuda")
    kernel_ms = float(np.mean(probe_ms)) if probe_ms else None
    hbm, peak_kind = peaks()
    u_evt = {k: v / events for k, v in units.items()}

    def roofline_of(name, k_ms, n_timed):
        if not k_ms or name not in KERNEL_BYTES:
            return None
        # bytes of one launch: the kernel processes the whole batch (B events) per launch,
        # split evenly over its launches per batch
        bytes_per_launch = KERNEL_BYTES[name](u_evt) * B / launches[name]
        ach = bytes_per_launch / (k_ms / 1e3) / 1e9
        return {"bound": "hbm", "kernel": name, "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                "traffic": (NCU_DRAM_BYTES_PER_EVENT[name] * B / launches[name]
                            if name in NCU_DRAM_BYTES_PER_EVENT else None),
                "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"
                if peak_kind == "measured" else "fallback 6650 GB/s",
                "bytes_per_launch": bytes_per_launch, "launch_ms": k_ms, "launches_timed": n_timed}

    roof = roofline_of(top, kernel_ms, len(probe_ms))
    # the second kernel of the census, timed the same way over a shorter run
    second = sorted(census, key=census.get)[-2] if len(census) > 1 else None
    roof_next = None
    if second:
        chain.set_probe(second)
        chain.prepare(B)
        probe_ms.clear()
        pipeline(chain, torch, max(a.steps // 4, 10), sub, lambda slot: probe_ms.extend(
            m for _, m in chain.probe_read(slot)))
        roof_next = roofline_of(second, float(np.mean(probe_ms)) if probe_ms else None, len(probe_ms))
    chain_ach = chain_bytes(u_evt) * value / world / 1e9
    chain.set_probe(None)
    chain.close()

    out = {"metric": METRIC, "value": value, "unit": "events/s", "n_gpus": world, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "u16/u32 int, f32 hits and cuts, f64 fits", "data": DATA,
           "config": {"workload": "PU50 batched chain: %d events per launch sequence (captured graph), %d batches "
                                  "in flight, inputs in a device-resident pool" % (B, a.slots),
                      "pu": PU, "events_per_step": B, "distinct_events": len(raws),
                      "input_bytes": input_bytes,
                      "l2": "inputs larger than L2: %d distinct events, %.0f MB of raw records, cycled"
                            % (len(raws), input_bytes / 1e6),
                      "parallelism": "replicas (events shard across GPUs, no collective)"},
           "gpu_launches": launches_per_batch * a.steps,
           "launch_tuning": tuning,
           "clocks": clocks,
           "roofline": roof, "roofline_next": roof_next,
           "chain_roofline": {"achieved": chain_ach, "peak": hbm, "unit": "GB/s", "frac": chain_ach / hbm,
                              "bytes_per_event": chain_bytes(u_evt)},
           "units_per_event": u_evt,
           "cut_margin": {"decisions_within_4_ulp_per_event": margins["cut_decisions_on_boundary"] / events,
                          "events_with_capacity_flags": margins["flagged_events"], "events": events},
           "kernel_shares": {k: round(v / total_ms, 4) for k, v in
                             sorted(census.items(), key=lambda x: -x[1])[:12]},
           "result_bytes_per_step": result_bytes[0] / max(1, a.steps)}

    # ------------------------------------------------------------ batched, uneven pileup
    # 64 events per launch with PU uniform in [20, 200] (the batched-chain
    # configuration), device-resident inputs, the same tuning, and the
    # container capacities widened for PU 200 (at the reference's, most of
    # these events would be truncated: no tuples above PU ~80)
    if rank == 0 and world == 1 and a.mixed_batches:
        rng = np.random.default_rng(3)
        mpus = rng.uniform(20.0, 200.0, B * a.mixed_batches)
        with cf.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
            mraws = list(ex.map(lambda k: det.event(SEED0 + 200000 + k, float(mpus[k]), model="calibrated"),
                                range(len(mpus))))
        mnw = [len(r) // 4 for r in mraws]
        mb = [mnw[i * B:(i + 1) * B] for i in range(a.mixed_batches)]
        mchain = pixgpu.Chain(det.es, max_events=B, max_words_per_batch=max(sum(x) for x in mb) + 1024,
                              slots=2, device=dev, pool_words=sum(mnw) + 64 * len(mnw) + 4096,
                              caps=PU200_CAPS)
        load_tuning(mchain)
        mh = []
        for r in mraws:
            h = mchain.pool_put(r)
            while h is None:
                time.sleep(0.001)
                h = mchain.pool_put(r)
            mh.append(h)
        mbatches = [mh[i * B:(i + 1) * B] for i in range(a.mixed_batches)]
        mchain.prepare(B)
        mflags = [0]

        def mdone(slot):
            mflags[0] += mchain.summary(slot)["n_flagged_events"]
        msub = lambda i: mchain.submit_pooled(mbatches[i % len(mbatches)], keep=True)  # noqa: E731
        pipeline(mchain, torch, a.warmup, msub, lambda s: None)
        msteps = max(8, a.steps // 4)
        mms = pipeline(mchain, torch, msteps, msub, mdone)
        slot_gb = mchain.slot_bytes() / 1e9
        mchain.close()
        out["batched_mixed_pu"] = {"pu": "uniform 20-200", "events_per_batch": B, "distinct_events": len(mraws),
                                   "mean_words_per_event": float(np.mean(mnw)), "steps": msteps,
                                   "events_per_s": msteps * B / (mms / 1e3), "ms_per_step": mms / msteps,
                                   "caps": PU200_CAPS, "slot_gb": slot_gb,
                                   "events_with_capacity_flags": mflags[0], "events_timed": msteps * B}

    # ------------------------------------------------------------ end to end through pg_submit
    nbh = len(raws) // B
    host_batches = [raws[(i % nbh) * B:(i % nbh) * B + B] for i in range(nbh)]

    def e2e_leg(scan):
        ec = pixgpu.Chain(det.es, max_events=B, max_words_per_batch=max_words, slots=a.slots, device=dev,
                          fed_scan=scan)
        load_tuning(ec)
        ec.prepare(B)
        h2d = [0]
        d2h = [0]
        fed_list = struct.unpack_from("<%dI" % struct.unpack_from("<I", det.es[4], 0)[0], det.es[4], 4)
        n_scan = sum(1 for f in fed_list if f != 40 and f < 4096)  # FED table entries per event

        def e2e_done(slot):
            sm = ec.summary(slot)
            d2h[0] += sm["result_bytes"]
            if scan == "host":  # words, one FED byte per word pair, offsets
                h2d[0] += 4 * sm["n_digis"] + sm["n_digis"] // 2 + 4 * (sm["n_events"] + 1)

        sub = lambda i: ec.submit(host_batches[i % nbh])  # noqa: E731
        pipeline(ec, torch, a.warmup, sub, lambda s: None)
        t0 = time.perf_counter()
        ems = pipeline(ec, torch, a.steps, sub, e2e_done)
        wall = time.perf_counter() - t0
        ec.close()
        if scan == "device":  # whole FED blocks (records less their directories) and the FED table
            for i in range(a.steps):
                batch = host_batches[i % nbh]
                h2d[0] += sum(len(r) - 4 - 8 * struct.unpack_from("<I", r, 0)[0] for r in batch)
                h2d[0] += 8 * n_scan * len(batch)
        rate, ems = replicas.job_rate(events, ems, device="cuda")
        return {"value": rate, "unit": "events/s",
                "h2d_bytes_per_step": h2d[0] / a.steps, "d2h_bytes_per_step": d2h[0] / a.steps,
                "host_wall_events_per_s": events / wall,
                "path": ("pg_submit: host FED scan + H2D of words" if scan == "host" else
                         "pg_submit: H2D of whole FED blocks + device FED scan") +
                        " + chain + results into mapped host memory"}

    legs = {scan: e2e_leg(scan) for scan in ("host", "device")}
    # the headline is the faster of the two public configurations (pg_config.fed_scan);
    # both give the same products (tests/test_gpu_errors.py)
    best_scan = max(legs, key=lambda k: legs[k]["value"])
    out["e2e"] = dict(legs[best_scan], fed_scan=best_scan)
    out["e2e_by_fed_scan"] = {k: v["value"] for k, v in legs.items()}

    if rank == 0 and world == 1:
        # ------------------------------------------------------------ one event per launch (plain chain)
        pe = {}
        for label, slots, graphs in (("1 stream", 1, False), ("4 streams", 4, False)):
            c1 = pixgpu.Chain(det.es, max_events=1, max_words_per_batch=int(max(nw)) + 1024, slots=slots,
                              device=dev, use_graphs=graphs, pool_words=sum(nw) + 64 * len(nw) + 4096)
            load_tuning(c1)
            hs = [c1.pool_put(r) for r in raws]
            sub1 = lambda i: c1.submit_pooled([hs[i % len(hs)]], keep=True)  # noqa: E731
            pipeline(c1, torch, 8, sub1, lambda s: None)
            pms = pipeline(c1, torch, a.per_event, sub1, lambda s: None)
            pe[label] = a.per_event / (pms / 1e3)
            if slots == 1:
                # latency of one event alone: submit, wait, on the host clock
                lat = []
                for i in range(min(a.per_event, 256)):
                    t0 = time.perf_counter()
                    s1 = c1.submit_pooled([hs[i % len(hs)]], keep=True)
                    c1.wait(s1)
                    lat.append(time.perf_counter() - t0)
                    c1.release(s1)
                pe_lat = {"p50_ms": 1e3 * float(np.percentile(lat, 50)), "p99_ms": 1e3 * float(np.percentile(lat, 99)),
                          "events": len(lat)}
            c1.close()
        best = max(pe.values())
        out["per_event"] = {"events_per_s": pe, "latency_1_stream": pe_lat,
                            "mode": "one event per launch sequence, plain launches (no graph), device-resident inputs"}
        out["batched_vs_per_event"] = value / best

        # ------------------------------------------------------------ serving loop: load sweep
        if a.serve:
            sv, by_slots = {}, {}
            best_ok = None
            # the default number of batches in flight over the whole load
            # range, then fewer in flight (larger batches) over the upper part
            knee = (0.7, 0.725, 0.75, 0.775, 0.8, 0.825, 0.85)
            for slots_n, fracs in ((a.serve_slots, (0.2, 0.35, 0.5, 0.6, 0.65) + knee + (0.9,)), (4, knee), (3, knee)):
                if slots_n in by_slots:
                    continue
                sc = pixgpu.Chain(det.es, max_events=a.serve_batch, max_words_per_batch=int(max(nw)) * a.serve_batch,
                                  slots=slots_n, device=dev, pool_words=64 * 1000 * 1000)
                load_tuning(sc)
                sc.prepare(a.serve_batch)
                best_n = None
                for frac in fracs:
                    rate = frac * value
                    st, lat = sc.serve(raws, a.serve, rate_hz=rate, max_batch=a.serve_batch, seed=11,
                                       upload_threads=4)
                    pt = {"offered_hz": st["offered_hz"], "events_per_s": st["events_per_s"], "p50_ms": st["p50_ms"],
                          "p99_ms": st["p99_ms"], "mean_batch": st["mean_batch"], "batches": st["batches"],
                          "admission_waits": st["admission_waits"]}
                    if slots_n == a.serve_slots:
                        sv["%.0f%% of batched throughput" % (100 * frac)] = pt
                    if st["p99_ms"] < 5.0 and (best_n is None or st["events_per_s"] > best_n["events_per_s"]):
                        best_n = dict(pt, load=frac, slots=slots_n)
                sc.close()
                by_slots[slots_n] = best_n
                if best_n and (best_ok is None or best_n["events_per_s"] > best_ok["events_per_s"]):
                    best_ok = best_n
            out["serving"] = {"pu": PU, "requests": a.serve, "max_batch": a.serve_batch, "slots": a.serve_slots,
                              "points": sv,
                              "best_under_5ms_p99_by_slots": {str(k): v for k, v in by_slots.items()},
                              "best_under_5ms_p99": best_ok,
                              "best_under_5ms_p99_vs_per_event": (best_ok["events_per_s"] / best) if best_ok else None}

        # ------------------------------------------------------------ serving, uneven pileup (10-100 kHz)
        if a.serve_mixed:
            rng = np.random.default_rng(7)
            pus = np.exp(rng.uniform(np.log(30), np.log(250), 128))
            with cf.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
                mraws = list(ex.map(lambda k: det.event(SEED0 + 300000 + k, float(pus[k]), model="calibrated"),
                                    range(len(pus))))
            mb_serve = 16
            mc = pixgpu.Chain(det.es, max_events=mb_serve, max_words_per_batch=mb_serve * 300000, slots=3,
                              device=dev, pool_words=96 * 1000 * 1000, caps=pixgpu.WIDE_CAPS)
            load_tuning(mc)
            mc.prepare(mb_serve)
            mv = {}
            flagged = [0]

            def on_result(req, ev, res):
                if res["flags"] & ~(1 << 16):  # bit 16: compact result truncated, not a chain capacity
                    flagged[0] += 1
            for rate in (10000.0, 30000.0, 100000.0):
                st, _ = mc.serve(mraws, a.serve_mixed, rate_hz=rate, max_batch=mb_serve, seed=13, upload_threads=4,
                                 on_result=on_result)
                mv["%.0f kHz" % (rate / 1e3)] = {"offered_hz": st["offered_hz"], "events_per_s": st["events_per_s"],
                                                 "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
                                                 "mean_batch": st["mean_batch"],
                                                 "admission_waits": st["admission_waits"]}
            slot_gb = mc.slot_bytes() / 1e9
            mc.close()
            out["serving_mixed_pu"] = {"pu": "log-uniform 30-250", "distinct_events": len(mraws),
                                       "requests_per_point": a.serve_mixed, "max_batch": mb_serve, "slots": 3,
                                       "caps": pixgpu.WIDE_CAPS, "slot_gb": slot_gb,
                                       "results_with_capacity_flags": flagged[0], "points": mv,
                                       "note": "offered rates above the sustained rate are admission-limited: "
                                               "arrivals wait for pool space and free slots"}

        # ------------------------------------------------------------ dense event model, batched
        draws = make_events(det, 2 * B, base=SEED0 + 400000, model="dense")
        dnw = [len(r) // 4 for r in draws]
        dchain = pixgpu.Chain(det.es, max_events=B, max_words_per_batch=int(max(dnw)) * B + 1024, slots=a.slots,
                              device=dev, pool_words=sum(dnw) + 64 * len(dnw) + 4096)
        load_tuning(dchain)
        dh = [dchain.pool_put(r) for r in draws]
        dbatches = [dh[:B], dh[B:2 * B]]
        dchain.prepare(B)
        dunits = collections.Counter()
        dsub = lambda i: dchain.submit_pooled(dbatches[i % 2], keep=True)  # noqa: E731
        pipeline(dchain, torch, a.warmup, dsub, lambda s: None)
        dsteps = max(8, a.steps // 4)
        dms = pipeline(dchain, torch, dsteps, dsub, lambda s: dunits.update(units_of(dchain.summary(s))))
        dchain.close()
        out["dense_pu50"] = {"events_per_s": dsteps * B / (dms / 1e3), "steps": dsteps,
                             "units_per_event": {k: v / (dsteps * B) for k, v in dunits.items()},
                             "model": "every track prompt and above 0.5 GeV (ps_default_event_config)"}

        # ------------------------------------------------------------ fits: FP64 and mixed precision
        out["fits"] = fit_leg(det, dev, torch)

        # ------------------------------------------------------------ CPU baseline
        import oracle
        cores = os.cpu_count() or 1
        n_cpu = int(max(cores, min(len(raws), a.cpu_seconds * 9.0 * cores)))
        sample = raws[:n_cpu]
        if oracle.ref_available():
            d = tempfile.mkdtemp()
            det.write(d)
            wall_c, lat_c = oracle.ref_time_events(d, sample, cores)
            kind = "reference"
        else:
            d = None
            wall_c, lat_c = oracle.Oracle(det.es).time_events(sample, cores)
            kind = "port"
        out["cpu_baseline"] = {"value": len(sample) / wall_c, "unit": "events/s", "cores": cores, "kind": kind,
                               "sample": "%d distinct PU50 events, one chain instance per thread" % len(sample),
                               "cpu_model": cpu_model(),
                               "latency_p50_ms": 1e3 * float(np.percentile(lat_c, 50)),
                               "latency_p99_ms": 1e3 * float(np.percentile(lat_c, 99))}
        # the reference's plain chain on 100 PU20 events, one thread (config 1)
        c1raws = make_events(det, 100, pu=20, base=SEED0, model="dense")
        if oracle.ref_available():
            wall_1, lat_1 = oracle.ref_time_events(d, c1raws, 1)
        else:
            wall_1, lat_1 = oracle.Oracle(det.es).time_events(c1raws, 1)
        out["cpu_pu20_one_thread"] = {"events_per_s": 100 / wall_1, "events": 100, "threads": 1, "kind": kind,
                                      "latency_p50_ms": 1e3 * float(np.percentile(lat_1, 50)),
                                      "latency_p99_ms": 1e3 * float(np.percentile(lat_1, 99)),
                                      "model": "power-law tracks above 0.5 GeV (the dense model), ~25k digis"}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def load_tuning(chain):
    """The committed launch-shape table (every tuned batch size), when present."""
    if os.path.exists(TUNE_CACHE):
        chain.tune_load(TUNE_CACHE)


def apply_tuning(chain, B, raws, a):
    """Launch shapes for B-event batches: the committed cache for this device, or
    the autotuner's choice (with --autotune, or when the cache has no entry)."""
    import pixgpu
    src = "cache"
    n = chain.tune_load(TUNE_CACHE) if (os.path.exists(TUNE_CACHE) and not a.autotune) else 0
    gain = None
    if n == 0:
        src = "autotuned in this run"
        gain = chain.autotune(raws[:B], repeats=3)
        if a.tune_out:
            chain.tune_save(a.tune_out)
    table = {k: v for k, v in chain.tune_table(B).items() if v}
    return {"source": src, "events_per_batch": B, "grid_scales": table, "tuner_gain_ms_per_batch": gain,
            "kernels_tunable": len(pixgpu.tune_kernel_names())}


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
