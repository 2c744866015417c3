#!/usr/bin/env python
"""Launch-shape autotuner driver: tunes the grid scale of every tunable
kernel (pg_autotune) for each batch size on seeded synthetic events, and
writes the per-device cache that Chain.tune_load, run_events.py and bench.py
read.

  python pixeltrack-standalone_b200/tune_launches.py --sizes 1,2,4,8,16,32,64 --pu 50 --model calibrated

Entries of other devices already in the cache file are kept.
"""
import argparse
import concurrent.futures as cf
import os
import sys
import tempfile

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import pixgpu  # noqa: E402

DEFAULT_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning", "launch_tuning.txt")


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--sizes", default="1,2,4,8,16,32,64", help="batch sizes to tune")
    p.add_argument("--pu", type=float, default=50)
    p.add_argument("--model", default=pixgpu.BENCH_MODEL, help="event model of the tuning events (dense, calibrated)")
    p.add_argument("--repeats", type=int, default=3, help="timed batches per trial (median)")
    p.add_argument("--seed", type=int, default=pixgpu.BASE_SEED + 9000)
    p.add_argument("--out", default=DEFAULT_CACHE)
    a = p.parse_args()
    sizes = sorted({int(x) for x in a.sizes.split(",") if x.strip()})
    det = pixgpu.Detector()
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        raws = list(ex.map(lambda k: det.event(a.seed + k, a.pu, model=a.model), range(max(sizes))))
    words = max(len(r) // 4 for r in raws)
    chain = pixgpu.Chain(det.es, max_events=max(sizes), max_words_per_batch=words * max(sizes) + 1024, slots=1)
    try:
        for n in sizes:
            gain = chain.autotune(raws[:n], repeats=a.repeats)
            moved = {k: v for k, v in chain.tune_table(n).items() if v}
            print("batch %3d: %.3f ms saved per batch; %s" % (n, gain, moved), flush=True)
        tmp = os.path.join(tempfile.mkdtemp(), "tune.txt")
        chain.tune_save(tmp)
        mine = [ln for ln in open(tmp) if ln.strip() and not ln.startswith("#")]
        device = mine[0].split("|")[0] if mine else None
        keep = []
        if os.path.exists(a.out):
            keep = [ln for ln in open(a.out) if ln.strip() and not ln.startswith("#") and ln.split("|")[0] != device]
        os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
        with open(a.out, "w") as f:
            f.write(open(tmp).readline())
            f.writelines(keep + mine)
        print("wrote %s (%d entries for %s)" % (a.out, len(mine), device))
    finally:
        chain.close()


if __name__ == "__main__":
    main()
