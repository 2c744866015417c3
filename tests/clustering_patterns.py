"""The digi patterns of the reference's clustering test
(src/serial/test/gpuClustering_t.h:36-206), restated as data for the
clustering entry points, with the checks that test applies after the
charge cut (:244-279).  Variant kn (0..4) of the reference's generator:
odd variants add a noise module (666) of single-pixel clusters below the
charge threshold; variant 0 makes the isolated pixel of module 42 low; variant
2 makes the holes pattern and the even-id patterns low."""
import numpy as np

INV_ID = 9999
Y_ORDER = [5, 7, 9, 1, 3, 0, 4, 8, 2, 6]


def patterns(kn):
    """(module ids, x, y, charges, number of clusters generated) of variant kn."""
    ids, xs, ys, adcs = [], [], [], []
    ncl = 0

    def px(i, x, y, a):
        ids.append(i)
        xs.append(x)
        ys.append(y)
        adcs.append(a)

    def invalid():
        px(INV_ID, 0, 0, 0)

    if kn % 2 == 1:  # noise module: 1000 single pixels 3 apart
        for x in range(0, 140, 3):
            for y in range(0, 400, 3):
                if ncl >= 1000:
                    break
                px(666, x, y, 1000)
                ncl += 1
            if ncl >= 1000:
                break
    mid, x0 = 42, 10
    ncl += 1
    px(mid, x0, x0, 100 if kn == 0 else 5000)        # isolated
    ncl += 1
    px(mid, x0, 0, 5000)                              # first column
    ncl += 1
    px(mid, x0 + 80, 2, 5000)                         # first columns
    px(mid, x0 + 80, 1, 5000)
    ncl += 1
    px(mid, x0, 415, 5000)                            # last column
    ncl += 1
    px(mid, x0 + 80, 415, 2500)                       # last columns
    px(mid, x0 + 80, 414, 2500)
    ncl += 1
    for x in range(20, 25):                           # diagonal
        px(mid, x, x, 1000)
    ncl += 1
    for x in range(45, 40, -1):                       # reversed diagonal
        px(mid, x, x, 1000)
    ncl += 1
    invalid()                                         # an error word inside the module
    messy = [21, 25, 23, 24, 22]
    for x in messy:                                   # messy
        px(mid, x, 20 + x, 1000)
    ncl += 1
    for x in messy:                                   # holes
        px(mid, x, 100, 100 if kn == 2 else 1000)
        if x % 2 == 0:
            px(mid, x, 101, 1000)
    ncl += 1
    px(0, 10, 10, 5000)                               # module 0
    for mid in range(11, 1801, 2):                    # every odd module id
        if (mid // 20) % 2:
            invalid()
        for x in range(0, 40, 4):
            ncl += 1
            if (mid // 10) % 2:
                for k in range(10):
                    px(mid, x, x + Y_ORDER[k], 100)
                    px(mid, x + 1, x + Y_ORDER[k] + 2, 1000)
            else:
                for k in range(10):
                    px(mid, x, x + Y_ORDER[9 - k], 10 if kn == 2 else 1000)
                    if Y_ORDER[k] == 3:
                        continue                      # hole
                    if mid == 51:
                        invalid()
                        invalid()
                    px(mid, x + 1, x + Y_ORDER[k] + 2, 10 if kn == 2 else 1000)
    return (np.array(ids, np.uint16), np.array(xs, np.uint16), np.array(ys, np.uint16), np.array(adcs, np.uint16),
            ncl)


def reference_checks(ids_in, res):
    """The checks of gpuClustering_t.h:244-279 on a clustering result: no
    pixel of the noise module survives the charge cut, every kept pixel has
    a cluster index below its module's count, and each module's clusters are
    numbered 0..n-1 without holes."""
    mod, clus, nclus = res["moduleInd"], res["clus"], res["clusInModule"]
    assert not np.any(mod == 666), "a noise pixel survived the charge cut"
    keep = mod != INV_ID
    assert np.all(clus[keep] >= 0)
    assert np.all(clus[keep] < nclus[mod[keep]])
    ids = sorted(set((int(m) * 1000 + int(c)) for m, c in zip(mod[keep], clus[keep])))
    by_module = {}
    for v in ids:
        by_module.setdefault(v // 1000, []).append(v % 1000)
    for m, cs in by_module.items():
        assert cs == list(range(len(cs))), (m, cs[:10])
        assert len(cs) == nclus[m], (m, len(cs), nclus[m])
