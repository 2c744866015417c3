// Batch workspace layout and the launch sequence of the whole chain.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "pixgpu_internal.cuh"

namespace pixgpu {

namespace {

struct Carver {
  char* base;
  size_t off = 0;
  template <typename T>
  void take(T*& p, size_t count) {
    off = (off + 255) & ~size_t(255);
    p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += count * sizeof(T);
  }
};

void layout(Workspace& ws, Carver& c, uint32_t E, uint32_t W, const Caps& cap) {
  ws.maxEvents = E;
  ws.wordCap = W;
  ws.cap = cap;
  c.take(ws.words, W);
  c.take(ws.fedIds, W / 2 + 2);
  c.take(ws.wordOffsets, E + 1);
  c.take(ws.input, 1);
  c.take(ws.ev, E);
  c.take(ws.xx, W);
  c.take(ws.yy, W);
  c.take(ws.adc, W);
  c.take(ws.moduleInd, W);
  c.take(ws.clus, W);
  c.take(ws.pdigi, W);
  c.take(ws.rawIdArr, W);
  c.take(ws.errors, size_t(E) * kErrCap);
  c.take(ws.errWordIdx, size_t(E) * kErrCap);
  c.take(ws.moduleStart, size_t(E) * kModStride);
  c.take(ws.clusInModule, size_t(E) * kModStride);
  c.take(ws.moduleId, size_t(E) * kModStride);
  c.take(ws.clusModuleStart, size_t(E) * kModStride);
  size_t H = size_t(E) * cap.hits;
  c.take(ws.xl, H);
  c.take(ws.yl, H);
  c.take(ws.xerr, H);
  c.take(ws.yerr, H);
  c.take(ws.xg, H);
  c.take(ws.yg, H);
  c.take(ws.zg, H);
  c.take(ws.rg, H);
  c.take(ws.charge, H);
  c.take(ws.iphi, H);
  c.take(ws.xsize, H);
  c.take(ws.ysize, H);
  c.take(ws.detInd, H);
  c.take(ws.phiOff, size_t(E) * kPhiStride);
  c.take(ws.phiBins, H);
  c.take(ws.phiRec, H);
  c.take(ws.agc, E);
  c.take(ws.jCount, size_t(E) * (cap.jCap + 1));
  c.take(ws.jOffset, size_t(E) * (cap.jCap + 1));
  size_t C = size_t(E) * cap.cells;
  c.take(ws.cellInner, C);
  c.take(ws.cellOuter, C);
  c.take(ws.cellPair, C);
  c.take(ws.cellDoubletId, C);
  c.take(ws.cellUsed, C);
  c.take(ws.ohCount, size_t(E) * (cap.hits + 1));
  c.take(ws.ohOff, size_t(E) * (cap.hits + 1));
  c.take(ws.hitTouch, size_t(E) * cap.hits);
  c.take(ws.fishHits, size_t(E) * cap.hits);
  c.take(ws.ohCells, C);
  c.take(ws.ohRec, C);
  c.take(ws.ohDet, C);
  size_t C1 = size_t(E) * (cap.cells + 1);
  c.take(ws.nbrCount, C1);
  c.take(ws.nbrOff, C1);
  c.take(ws.nbr, size_t(E) * cap.edges);
  c.take(ws.startTupleCount, C1);
  c.take(ws.startTupleOff, C1);
  c.take(ws.startHitCount, C1);
  c.take(ws.startHitOff, C1);
  c.take(ws.tupleOff, size_t(E) * (cap.tuples + 1));
  c.take(ws.tupleHits, size_t(E) * cap.tupleHits());
  c.take(ws.tupleDet, size_t(E) * cap.tupleHits());
  c.take(ws.tupleCells, size_t(E) * cap.tupleCells());
  c.take(ws.quality, size_t(E) * cap.tuples);
  c.take(ws.trkCount, C1);
  c.take(ws.trkOff, C1);
  c.take(ws.trk, size_t(E) * cap.tupleCells());
  c.take(ws.candidates, C);
  c.take(ws.tmOff, size_t(E) * 16);
  c.take(ws.tmBins, size_t(E) * cap.tuples);  // bins beyond cap.multiplicity only under its overflow flag
  size_t T = size_t(E) * cap.tuples;
  c.take(ws.state, T * 5);
  c.take(ws.cov, T * 15);
  c.take(ws.pt, T);
  c.take(ws.eta, T);
  c.take(ws.chi2, T);
  c.take(ws.h2tCount, size_t(E) * (cap.hits + 1));
  c.take(ws.h2tOff, size_t(E) * (cap.hits + 1));
  c.take(ws.h2t, size_t(E) * cap.h2t);
  size_t V = size_t(E) * kMaxVtx;
  c.take(ws.zv, V);
  c.take(ws.wv, V);
  c.take(ws.vchi2, V);
  c.take(ws.ptv2, V);
  c.take(ws.ndof, V);
  c.take(ws.sortInd, V);
  c.take(ws.idv, T);
  c.take(ws.scratchA, size_t(E) * cap.scratch);
  c.take(ws.scratchB, size_t(E) * cap.scratch);
  {
    const uint32_t longest = std::max(std::max(cap.jCap, cap.cells), std::max(cap.hits, kPhiTot));
    ws.scanTiles = (longest + kScanTile - 1) / kScanTile + 1;
  }
  c.take(ws.scanState, size_t(E) * kScanCalls * ws.scanTiles);
  c.take(ws.scanTicket, size_t(E) * kScanCalls);
  c.take(ws.scanEpoch, E);
  c.take(ws.bigSeg, size_t(E) * kBigSegCap);
  c.take(ws.segList, size_t(E) * cap.cells);
}

// the pair opened by probeBegin when its name matched (-1: none).  Records use
// cudaEventRecordExternal so that under stream capture they become event
// record nodes of the graph rather than capture-internal dependencies.
thread_local int tProbeOpen = -1;

}  // namespace

thread_local KernelProbe* tProbe = nullptr;

void probeBegin(const char* name, cudaStream_t s) {
  tProbeOpen = -1;
  KernelProbe* p = tProbe;
  if (!p || p->used >= kProbeMax) return;
  if (!(p->name[0] == '*' && p->name[1] == 0) && std::strcmp(p->name, name) != 0) return;
  tProbeOpen = int(p->used);
  p->launched[p->used] = name;
  cudaEventRecordWithFlags(p->ev[2 * p->used], s, cudaEventRecordExternal);
}

void probeEnd(cudaStream_t s) {
  KernelProbe* p = tProbe;
  if (!p || tProbeOpen < 0) return;
  cudaEventRecordWithFlags(p->ev[2 * tProbeOpen + 1], s, cudaEventRecordExternal);
  p->used = uint32_t(tProbeOpen) + 1;
  tProbeOpen = -1;
}

size_t workspaceBytes(uint32_t maxEvents, uint32_t wordCap, const Caps& cap) {
  Workspace ws;
  Carver c{nullptr};
  layout(ws, c, maxEvents, wordCap, cap);
  return c.off + 256;
}

void workspaceCarve(Workspace& ws, void* base, uint32_t maxEvents, uint32_t wordCap, const Caps& cap) {
  Carver c{static_cast<char*>(base)};
  layout(ws, c, maxEvents, wordCap, cap);
}

cudaError_t runChain(const DeviceES& es, Workspace& ws, uint32_t nEvents, cudaStream_t stream, bool riemann,
                     int vertexAlgo) {
  cudaError_t err;
  if (ws.scan.on) launchFedScan(ws, nEvents, stream);
  if ((err = runLocal(es, ws, nEvents, stream)) != cudaSuccess) return err;
  if ((err = runCA(es, ws, nEvents, stream)) != cudaSuccess) return err;
  if ((err = runFits(es, ws, nEvents, stream, riemann)) != cudaSuccess) return err;
  if ((err = runCleaners(ws, nEvents, stream)) != cudaSuccess) return err;
  if ((err = runVertices(ws, nEvents, stream, vertexAlgo)) != cudaSuccess) return err;
  return cudaSuccess;
}

}  // namespace pixgpu
