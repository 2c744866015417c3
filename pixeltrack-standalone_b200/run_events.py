#!/usr/bin/env python
"""Runs the B200 pixel chain on seeded synthetic events: the counterpart of
the reference's `cuda --numberOfStreams S --maxEvents N` driver for this
chain.  Events are generated once, uploaded into the device pool, and the
chain is launched `--repeat` times over batches of `--batch` events.

  python pixeltrack-standalone_b200/run_events.py --events 64 --batch 64 --pu 50 --repeat 3
"""
import argparse
import concurrent.futures as cf
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import pixgpu  # noqa: E402


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--events", type=int, default=64)
    p.add_argument("--batch", type=int, default=64)
    p.add_argument("--pu", type=float, default=50)
    p.add_argument("--repeat", type=int, default=3)
    p.add_argument("--slots", type=int, default=1)
    p.add_argument("--seed", type=int, default=pixgpu.BASE_SEED + 1000)
    p.add_argument("--no-graphs", action="store_true")
    a = p.parse_args()
    det = pixgpu.Detector()
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        raws = list(ex.map(lambda k: det.event(a.seed + k, a.pu), range(a.events)))
    words = [len(r) // 4 for r in raws]
    chain = pixgpu.Chain(det.es, max_events=a.batch, max_words_per_batch=max(words) * a.batch + 1024, slots=a.slots,
                         use_graphs=not a.no_graphs, pool_words=sum(words) + 64 * len(words) + 4096)
    handles = [chain.pool_put(r) for r in raws]
    if any(h is None for h in handles):
        raise RuntimeError("pool admission failed")
    batches = [handles[i:i + a.batch] for i in range(0, len(handles), a.batch)]
    done = 0
    t0 = time.perf_counter()
    for _ in range(a.repeat):
        for b in batches:
            s = chain.submit_pooled(b, keep=True)
            chain.wait(s)
            done += len(b)
            chain.release(s)
    dt = time.perf_counter() - t0
    print("processed %d events (PU %g, batches of %d) in %.3f s: %.1f events/s" % (done, a.pu, a.batch, dt, done / dt))
    chain.close()


if __name__ == "__main__":
    main()
