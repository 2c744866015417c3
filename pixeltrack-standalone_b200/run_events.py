#!/usr/bin/env python
"""Runs the B200 pixel chain on seeded synthetic events: the counterpart of
the reference's `cuda --numberOfStreams S --maxEvents N` driver for this
chain.  Events are generated once, uploaded into the device pool, and the
chain is launched `--repeat` times over batches of `--batch` events.

  python pixeltrack-standalone_b200/run_events.py --events 64 --batch 64 --pu 50 --repeat 3
  python pixeltrack-standalone_b200/run_events.py --events 64 --batch 64 --pu 20 --pu-max 200 --caps wide

--probe adds, after the timed loop, the median wall latency of one batch
(submit to results on the host) and the device time of every kernel of a
batch, timed with events captured around each launch (pg_set_probe).
"""
import argparse
import collections
import concurrent.futures as cf
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import pixgpu  # noqa: E402


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--events", type=int, default=64)
    p.add_argument("--batch", type=int, default=64)
    p.add_argument("--pu", type=float, default=50)
    p.add_argument("--pu-max", type=float, default=0,
                   help="uneven pileup: event k takes a seeded PU uniform in [--pu, --pu-max]")
    p.add_argument("--caps", choices=["reference", "wide"], default="reference",
                   help="container capacities: the reference's, or pixgpu.WIDE_CAPS (high pileup)")
    p.add_argument("--repeat", type=int, default=3)
    p.add_argument("--slots", type=int, default=1)
    p.add_argument("--seed", type=int, default=pixgpu.BASE_SEED + 1000)
    p.add_argument("--model", choices=["calibrated", "dense"], default="calibrated",
                   help="event model of the generator (pixgpu.Detector.event)")
    p.add_argument("--no-graphs", action="store_true")
    p.add_argument("--probe", action="store_true", help="per-kernel device times of a batch")
    p.add_argument("--fed-scan", choices=["host", "device"], default="host",
                   help="device: raw records go to the device whole (pg_submit) and the FED scan runs there; "
                        "host: records are unpacked once into the device-resident pool")
    p.add_argument("--tuning", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning",
                                                    "launch_tuning.txt"),
                   help="launch-shape cache to load ('' for the default shapes)")
    a = p.parse_args()
    det = pixgpu.Detector()
    rng = np.random.default_rng(a.seed)
    pus = rng.uniform(a.pu, a.pu_max, a.events) if a.pu_max > a.pu else np.full(a.events, a.pu)
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        raws = list(ex.map(lambda k: det.event(a.seed + k, float(pus[k]), model=a.model), range(a.events)))
    words = [len(r) // 4 for r in raws]
    device_scan = a.fed_scan == "device"
    chain = pixgpu.Chain(det.es, max_events=a.batch, max_words_per_batch=max(words) * a.batch + 1024, slots=a.slots,
                         use_graphs=not a.no_graphs, pool_words=0 if device_scan else max(sum(words) + 64 * len(words), 400000) + 4096,
                         fed_scan=a.fed_scan, caps=pixgpu.WIDE_CAPS if a.caps == "wide" else None)
    if a.tuning and os.path.exists(a.tuning):
        chain.tune_load(a.tuning)
    if device_scan:
        batches = [raws[i:i + a.batch] for i in range(0, len(raws), a.batch)]
        submit = lambda b: chain.submit(b)  # noqa: E731
    else:
        handles = [chain.pool_put(r) for r in raws]
        if any(h is None for h in handles):
            raise RuntimeError("pool admission failed")
        batches = [handles[i:i + a.batch] for i in range(0, len(handles), a.batch)]
        submit = lambda b: chain.submit_pooled(b, keep=True)  # noqa: E731
    done = 0
    t0 = time.perf_counter()
    for _ in range(a.repeat):
        for b in batches:
            s = submit(b)
            chain.wait(s)
            done += len(b)
            chain.release(s)
    dt = time.perf_counter() - t0
    pu = ("%g-%g" % (a.pu, a.pu_max)) if a.pu_max > a.pu else "%g" % a.pu
    print("processed %d events (PU %s, batches of %d) in %.3f s: %.1f events/s" % (done, pu, a.batch, dt, done / dt))
    if a.probe:
        lat = []
        for b in batches * 3:
            t1 = time.perf_counter()
            s = submit(b)
            chain.wait(s)
            lat.append(time.perf_counter() - t1)
            chain.release(s)
        lat.sort()
        census, launches = collections.defaultdict(float), collections.Counter()
        chain.set_probe("*")
        for b in batches:
            s = submit(b)
            chain.wait(s)
            for name, ms in chain.probe_read(s):
                census[name] += ms / len(batches)
                launches[name] += 1
            chain.release(s)
        chain.set_probe(None)
        print("batch wall latency: median %.3f ms; kernel launches per batch %d, device time %.3f ms" %
              (1e3 * lat[len(lat) // 2], sum(launches.values()) // len(batches), sum(census.values())))
        for name, ms in sorted(census.items(), key=lambda x: -x[1]):
            print("  %-22s %8.1f us  x%d" % (name, 1e3 * ms, launches[name] // len(batches)))
    chain.close()


if __name__ == "__main__":
    main()
