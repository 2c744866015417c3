"""A data directory for the reference's event processor: the synthetic
detector's conditions (cablingMap.bin, fedIds.bin, gain.bin, cpefast.bin,
beamspot.bin), `raw.bin` with the events, and the expected counts the
Source reads for the CountValidator (digicluster.bin: modules, digis and
clusters per event; tracks.bin; vertices.bin), taken from the oracle."""
import os
import struct


def write_data_dir(directory, det, raws, counts=True):
    import oracle
    det.write(directory)
    with open(os.path.join(directory, "raw.bin"), "wb") as f:
        for r in raws:
            f.write(r)
    if not counts:
        return None
    orc = oracle.Oracle(det.es)
    want = []
    with open(os.path.join(directory, "digicluster.bin"), "wb") as dc, \
            open(os.path.join(directory, "tracks.bin"), "wb") as tr, \
            open(os.path.join(directory, "vertices.bin"), "wb") as vx:
        for r in raws:
            o = orc.process(r, ["nModules", "nDigis", "nClusters", "nTuples", "nVertices"])
            dc.write(struct.pack("<III", o["nModules"], o["nDigis"], o["nClusters"]))
            tr.write(struct.pack("<I", o["nTuples"]))
            vx.write(struct.pack("<I", o["nVertices"]))
            want.append(o)
    return want
