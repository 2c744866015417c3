// Broken-line helix fits on B200, one thread per tuple, FP64 as in the
// reference, for 3-hit tuples, 4-hit tuples and 5-hit tuples fitted on
// their first four hits (fit5as4).  Reference: plugin-PixelTriplets/
// BrokenLineFitOnGPU.h:25-182 (kernelBLFastFit/kernelBLFit), BrokenLine.h:46-504,
// choleskyInversion.h:22-161, TrajectoryStateSoA.h:30-47.
//
// Products are accumulated over the inner index in ascending order, starting
// from the first term, and the kernels are compiled without FMA contraction,
// so results agree with the serial build to the last bit except where the
// device and host transcendental functions (atan2, sin, cos, log, asinhf)
// round differently.
#include "device_utils.cuh"
#include "pixgpu_internal.cuh"

namespace pixgpu {

namespace {

#include "fit_linalg.cuh"
#include "k_fit_riemann.cuh"

__device__ __forceinline__ double multScatt(double length, double B, double R, double slope) {
  double pt2 = fmin(20., B * R);
  pt2 *= pt2;
  constexpr double XXI_0 = 0.06 / 16.;
  constexpr double fact = 0.7 * ((13.6 / 1000.) * (13.6 / 1000.));
  return fact / (pt2 * (1. + sqr(slope))) * (fabs(length) * XXI_0) * sqr(1. + 0.038 * log(fabs(length) * XXI_0));
}

__device__ __forceinline__ M<2, 2> rotationMatrix(double slope) {
  M<2, 2> r;
  r(0, 0) = 1. / sqrt(1. + sqr(slope));
  r(0, 1) = slope * r(0, 0);
  r(1, 0) = -r(0, 1);
  r(1, 1) = r(0, 0);
  return r;
}

__device__ __forceinline__ double cross2D(double ax, double ay, double bx, double by) { return ax * by - ay * bx; }

__device__ void translateKarimaki(double* par, M<3, 3>& cov, double x0, double y0) {
  double s0, c0;
  s0 = sin(par[0]);
  c0 = cos(par[0]);
  double DP = x0 * c0 + y0 * s0;
  double DO = x0 * s0 - y0 * c0 + par[1];
  double uu = 1 + par[2] * par[1];
  double C = -par[2] * y0 + uu * c0;
  double BB = par[2] * x0 + uu * s0;
  double A = 2. * DO + par[2] * (sqr(DO) + sqr(DP));
  double U = sqrt(1. + par[2] * A);
  double xi = 1. / (sqr(BB) + sqr(C));
  double v = 1. + par[2] * DO;
  double lambda = (0.5 * A) / (U * sqr(1. + U));
  double mu = 1. / (U * (1. + U)) + par[2] * lambda;
  double zeta = sqr(DO) + sqr(DP);
  M<3, 3> J;
  J(0, 0) = xi * uu * v;
  J(0, 1) = -xi * sqr(par[2]) * DP;
  J(0, 2) = xi * DP;
  J(1, 0) = 2. * mu * uu * DP;
  J(1, 1) = 2. * mu * v;
  J(1, 2) = mu * zeta - lambda * A;
  J(2, 0) = 0;
  J(2, 1) = 0;
  J(2, 2) = 1.;
  par[0] = atan2(BB, C);
  par[1] = A / (1 + U);
  cov = sandwich(J, cov);
}

template <int N>
__device__ M<N, N> matrixCu(const double* w, const double* S, const double* VarBeta) {
  constexpr int n = N;
  M<N, N> C;
#pragma unroll
  for (int k = 0; k < N * N; ++k) C.a[k] = 0;
#pragma unroll
  for (int i = 0; i < n; ++i) {
    C(i, i) = w[i];
    if (i > 1) C(i, i) += 1. / (VarBeta[i - 1] * sqr(S[i] - S[i - 1]));
    if (i > 0 && i < n - 1)
      C(i, i) += (1. / VarBeta[i]) * sqr((S[i + 1] - S[i - 1]) / ((S[i + 1] - S[i]) * (S[i] - S[i - 1])));
    if (i < n - 2) C(i, i) += 1. / (VarBeta[i + 1] * sqr(S[i + 1] - S[i]));
    if (i > 0 && i < n - 1)
      C(i, i + 1) = 1. / (VarBeta[i] * (S[i + 1] - S[i])) * (-(S[i + 1] - S[i - 1]) / ((S[i + 1] - S[i]) * (S[i] - S[i - 1])));
    if (i < n - 2)
      C(i, i + 1) += 1. / (VarBeta[i + 1] * (S[i + 1] - S[i])) *
                     (-(S[i + 2] - S[i]) / ((S[i + 2] - S[i + 1]) * (S[i + 1] - S[i])));
    if (i < n - 2) C(i, i + 2) = 1. / (VarBeta[i + 1] * (S[i + 2] - S[i + 1]) * (S[i + 1] - S[i]));
    C(i, i) *= 0.5;
  }
  M<N, N> R;
#pragma unroll
  for (int j = 0; j < n; ++j)
#pragma unroll
    for (int i = 0; i < n; ++i) R(i, j) = C(i, j) + C(j, i);
  return R;
}


// hits: x,y,z of hit i at H[3*i+k]; ge: 6 floats per hit
template <int N>
__device__ void blFit(const double* H3, const float* ge, double B, FitOut& out) {
  constexpr int n = N;
  auto H = [&](int r, int c) { return H3[3 * c + r]; };
  double ff[4];
  {
    double ax = H(0, n / 2) - H(0, 0), ay = H(1, n / 2) - H(1, 0);
    double bx = H(0, n - 1) - H(0, n / 2), by = H(1, n - 1) - H(1, n / 2);
    double cx = H(0, 0) - H(0, n - 1), cy = H(1, 0) - H(1, n - 1);
    double tmp = 0.5 / cross2D(cx, cy, ax, ay);
    double csq = cx * cx + cy * cy, asq = ax * ax + ay * ay, bsq = bx * bx + by * by;
    ff[0] = H(0, 0) - (ay * csq + cy * asq) * tmp;
    ff[1] = H(1, 0) + (ax * csq + cx * asq) * tmp;
    ff[2] = sqrt(asq * bsq * csq) / (2. * fabs(cross2D(bx, by, ax, ay)));
    double dx = H(0, 0) - ff[0], dy = H(1, 0) - ff[1];
    double ex = H(0, n - 1) - ff[0], ey = H(1, n - 1) - ff[1];
    ff[3] = ff[2] * atan2(cross2D(dx, dy, ex, ey), dx * ex + dy * ey) / (H(2, n - 1) - H(2, 0));
  }
  int q;
  double radii[2][N], s[N], S[N], Z[N], VarBeta[N];
  {
    double dx = H(0, 1) - H(0, 0), dy = H(1, 1) - H(1, 0);
    double ex = H(0, n - 1) - H(0, n - 2), ey = H(1, n - 1) - H(1, n - 2);
    q = cross2D(dx, dy, ex, ey) > 0 ? -1 : 1;
    const double slope = -q / ff[3];
    M<2, 2> R = rotationMatrix(slope);
#pragma unroll
    for (int i = 0; i < n; ++i) {
      radii[0][i] = H(0, i) - ff[0] * 1.0;
      radii[1][i] = H(1, i) - ff[1] * 1.0;
    }
    double nrm = sqrt(ff[0] * ff[0] + ff[1] * ff[1]);
    double e0 = (-ff[2] * ff[0]) / nrm, e1 = (-ff[2] * ff[1]) / nrm;
#pragma unroll
    for (int i = 0; i < n; ++i)
      s[i] = q * ff[2] * atan2(cross2D(radii[0][i], radii[1][i], e0, e1), radii[0][i] * e0 + radii[1][i] * e1);
#pragma unroll
    for (int i = 0; i < n; ++i) {
      double p0 = s[i], p1 = H(2, i);
      S[i] = R(0, 0) * p0 + R(0, 1) * p1;
      Z[i] = R(1, 0) * p0 + R(1, 1) * p1;
    }
    VarBeta[0] = VarBeta[n - 1] = 0;
#pragma unroll
    for (int i = 1; i < n - 1; ++i)
      VarBeta[i] = multScatt(S[i + 1] - S[i], B, ff[2], slope) + multScatt(S[i] - S[i - 1], B, ff[2], slope);
  }
  // ---- line fit
  double lpar[2];
  M<2, 2> lcov;
  double lchi2;
  {
    const double slope = -q / ff[3];
    M<2, 2> R = rotationMatrix(slope);
    M<3, 3> V;
    M<2, 3> J;
#pragma unroll
    for (int k = 0; k < 9; ++k) V.a[k] = 0;
#pragma unroll
    for (int k = 0; k < 6; ++k) J.a[k] = 0;
    double w[N];
#pragma unroll
    for (int i = 0; i < n; ++i) {
      const float* g = ge + 6 * i;
      V(0, 0) = g[0];
      V(0, 1) = V(1, 0) = g[1];
      V(0, 2) = V(2, 0) = g[3];
      V(1, 1) = g[2];
      V(2, 1) = V(1, 2) = g[4];
      V(2, 2) = g[5];
      double tmp = 1. / sqrt(radii[0][i] * radii[0][i] + radii[1][i] * radii[1][i]);
      J(0, 0) = radii[1][i] * tmp;
      J(0, 1) = -radii[0][i] * tmp;
      J(1, 2) = 1.;
      M<2, 2> P = mul(mul(mul(mul(R, J), V), tr(J)), tr(R));
      w[i] = 1. / P(1, 1);
    }
    double r_u[N];
#pragma unroll
    for (int i = 0; i < n; ++i) r_u[i] = w[i] * Z[i];
    M<N, N> I;
    invert(matrixCu<N>(w, S, VarBeta), I);
    double u[N];
#pragma unroll
    for (int i = 0; i < n; ++i) {
      double acc = I(i, 0) * r_u[0];
#pragma unroll
      for (int k = 1; k < n; ++k) acc += I(i, k) * r_u[k];
      u[i] = acc;
    }
    lpar[0] = (u[1] - u[0]) / (S[1] - S[0]);
    lpar[1] = u[0];
    double idiff = 1. / (S[1] - S[0]);
    lcov(0, 0) = (I(0, 0) - 2 * I(0, 1) + I(1, 1)) * sqr(idiff) + multScatt(S[1] - S[0], B, ff[2], slope);
    lcov(0, 1) = (I(0, 1) - I(0, 0)) * idiff;
    lcov(1, 0) = (I(0, 1) - I(0, 0)) * idiff;
    lcov(1, 1) = I(0, 0);
    M<2, 2> jac;
    jac(0, 0) = 1.;
    jac(0, 1) = 0;
    jac(1, 0) = -S[0];
    jac(1, 1) = 1.;
    lpar[1] += -lpar[0] * S[0];
    lcov = sandwich(jac, lcov);
    double t = R(0, 0) - lpar[0] * R(0, 1);
    jac(1, 1) = 1. / t;
    jac(0, 0) = jac(1, 1) * jac(1, 1);
    jac(0, 1) = 0;
    jac(1, 0) = lpar[1] * R(0, 1) * jac(0, 0);
    lpar[1] = lpar[1] * jac(1, 1);
    lpar[0] = (R(0, 1) + lpar[0] * R(0, 0)) * jac(1, 1);
    lcov = sandwich(jac, lcov);
    lchi2 = 0;
#pragma unroll
    for (int i = 0; i < n; ++i) {
      lchi2 += w[i] * sqr(Z[i] - u[i]);
      if (i > 0 && i < n - 1)
        lchi2 += sqr(u[i - 1] / (S[i] - S[i - 1]) - u[i] * (S[i + 1] - S[i - 1]) / ((S[i + 1] - S[i]) * (S[i] - S[i - 1])) +
                     u[i + 1] / (S[i + 1] - S[i])) /
                 VarBeta[i];
    }
  }
  // ---- circle fit
  double cpar[3];
  M<3, 3> ccov;
  float cchi2;
  {
    const double slope = -q / ff[3];
#pragma unroll
    for (int i = 0; i < n; ++i) VarBeta[i] *= 1. + sqr(slope);
#pragma unroll
    for (int i = 0; i < n; ++i) Z[i] = sqrt(radii[0][i] * radii[0][i] + radii[1][i] * radii[1][i]) - ff[2];
    double w[N];
#pragma unroll
    for (int i = 0; i < n; ++i) {
      const float* g = ge + 6 * i;
      M<2, 2> V;
      V(0, 0) = g[0];
      V(0, 1) = V(1, 0) = g[1];
      V(1, 1) = g[2];
      M<2, 2> RR = rotationMatrix(-radii[0][i] / radii[1][i]);
      M<2, 2> P = mul(mul(RR, V), tr(RR));
      w[i] = 1. / P(1, 1);
    }
    double r_u[N + 1];
    r_u[n] = 0;
#pragma unroll
    for (int i = 0; i < n; ++i) r_u[i] = w[i] * Z[i];
    M<N + 1, N + 1> C;
    {
      M<N, N> cu = matrixCu<N>(w, s, VarBeta);
#pragma unroll
      for (int j = 0; j < n; ++j)
#pragma unroll
        for (int i = 0; i < n; ++i) C(i, j) = cu(i, j);
    }
    C(n, n) = 0;
#pragma unroll
    for (int i = 0; i < n; ++i) {
      C(i, n) = 0;
      if (i > 0 && i < n - 1)
        C(i, n) += -(s[i + 1] - s[i - 1]) * (s[i + 1] - s[i - 1]) / (2. * VarBeta[i] * (s[i + 1] - s[i]) * (s[i] - s[i - 1]));
      if (i > 1) C(i, n) += (s[i] - s[i - 2]) / (2. * VarBeta[i - 1] * (s[i] - s[i - 1]));
      if (i < n - 2) C(i, n) += (s[i + 2] - s[i]) / (2. * VarBeta[i + 1] * (s[i + 1] - s[i]));
      C(n, i) = C(i, n);
      if (i > 0 && i < n - 1) C(n, n) += sqr(s[i + 1] - s[i - 1]) / (4. * VarBeta[i]);
    }
    M<N + 1, N + 1> I;
    invert(C, I);
    double u[N + 1];
#pragma unroll
    for (int i = 0; i < n + 1; ++i) {
      double acc = I(i, 0) * r_u[0];
#pragma unroll
      for (int k = 1; k < n + 1; ++k) acc += I(i, k) * r_u[k];
      u[i] = acc;
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      double nr = sqrt(radii[0][c] * radii[0][c] + radii[1][c] * radii[1][c]);
      radii[0][c] /= nr;
      radii[1][c] /= nr;
    }
    double dx = H(0, 0) + (-Z[0] + u[0]) * radii[0][0], dy = H(1, 0) + (-Z[0] + u[0]) * radii[1][0];
    double ex = H(0, 1) + (-Z[1] + u[1]) * radii[0][1], ey = H(1, 1) + (-Z[1] + u[1]) * radii[1][1];
    double emdx = ex - dx, emdy = ey - dy;
    cpar[0] = atan2(emdy, emdx);
    cpar[1] = -q * (ff[2] - sqrt(sqr(ff[2]) - 0.25 * (emdx * emdx + emdy * emdy)));
    cpar[2] = q * (1. / ff[2] + u[n]);
    double tmp1 = emdx * emdx + emdy * emdy;
    M<3, 3> J;
    J(0, 0) = (radii[1][0] * emdx - emdy * radii[0][0]) / tmp1;
    J(0, 1) = (radii[1][1] * emdx - emdy * radii[0][1]) / tmp1;
    J(0, 2) = 0;
    J(1, 0) = (q / 2) * (emdx * radii[0][0] + emdy * radii[1][0]) / sqrt(sqr(2 * ff[2]) - tmp1);
    J(1, 1) = (q / 2) * (emdx * radii[0][1] + emdy * radii[1][1]) / sqrt(sqr(2 * ff[2]) - tmp1);
    J(1, 2) = 0;
    J(2, 0) = 0;
    J(2, 1) = 0;
    J(2, 2) = q;
    ccov(0, 0) = I(0, 0);
    ccov(0, 1) = I(0, 1);
    ccov(0, 2) = I(0, n);
    ccov(1, 0) = I(1, 0);
    ccov(1, 1) = I(1, 1);
    ccov(1, 2) = I(1, n);
    ccov(2, 0) = I(n, 0);
    ccov(2, 1) = I(n, 1);
    ccov(2, 2) = I(n, n);
    ccov = sandwich(J, ccov);
    translateKarimaki(cpar, ccov, 0.5 * emdx, 0.5 * emdy);
    ccov(0, 0) += (1 + sqr(slope)) * multScatt(S[1] - S[0], B, ff[2], slope);
    translateKarimaki(cpar, ccov, dx, dy);
    cchi2 = 0;
#pragma unroll
    for (int i = 0; i < n; ++i) {
      cchi2 += w[i] * sqr(Z[i] - u[i]);
      if (i > 0 && i < n - 1)
        cchi2 += sqr(u[i - 1] / (s[i] - s[i - 1]) - u[i] * (s[i + 1] - s[i - 1]) / ((s[i + 1] - s[i]) * (s[i] - s[i - 1])) +
                     u[i + 1] / (s[i + 1] - s[i]) + (s[i + 1] - s[i - 1]) * u[n] / 2) /
                 VarBeta[i];
    }
  }
  float b = 1.f / float(B);
  out.state[0] = float(cpar[0]);
  out.state[1] = float(cpar[1]);
  out.state[2] = float(cpar[2]) * b;
  out.state[3] = float(lpar[0]);
  out.state[4] = float(lpar[1]);
  out.cov[0] = float(ccov(0, 0));
  out.cov[1] = float(ccov(0, 1));
  out.cov[2] = b * float(ccov(0, 2));
  out.cov[3] = out.cov[4] = 0;
  out.cov[5] = float(ccov(1, 1));
  out.cov[6] = b * float(ccov(1, 2));
  out.cov[7] = out.cov[8] = 0;
  out.cov[9] = b * b * float(ccov(2, 2));
  out.cov[10] = out.cov[11] = 0;
  out.cov[12] = float(lcov(0, 0));
  out.cov[13] = float(lcov(0, 1));
  out.cov[14] = float(lcov(1, 1));
  out.pt = float(B) / float(fabs(cpar[2]));
  out.eta = asinhf(float(lpar[0]));
  out.chi2 = float((double(cchi2) + lchi2) / (2 * N - 5));
}

#include "k_fit_mixed.cuh"

// zero the fit results of every stored tuple (the reference's TrackSoA is value-initialised)
// Tuples that no fit writes get zero fit results: those kept out of the
// multiplicity bins (duplicates), and every tuple of an event whose bins
// overflowed (the fits then cover an order-dependent subset).
__global__ void kFitZero(Workspace ws) {
  const uint32_t e = blockIdx.y;
  const uint32_t nt = ws.ev[e].nTuples;
  const bool all = (ws.ev[e].flags & (kFlagFitBinOverflow | kFlagTmOverflow)) != 0;
  const uint32_t* toff = ws.tupleOff + size_t(e) * (ws.cap.tuples + 1);
  const uint8_t* q = ws.quality + size_t(e) * ws.cap.tuples;
  const size_t tb = size_t(e) * ws.cap.tuples;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
    if (!all && toff[t + 1] - toff[t] >= 3 && q[t] != 1) continue;  // 1: duplicate
    for (int k = 0; k < 5; ++k) ws.state[tb * 5 + size_t(t) * 5 + k] = 0.f;
    for (int k = 0; k < 15; ++k) ws.cov[tb * 15 + size_t(t) * 15 + k] = 0.f;
    ws.pt[tb + t] = 0.f;
    ws.eta[tb + t] = 0.f;
    ws.chi2[tb + t] = 0.f;
  }
}

// the fits a chain can run (pg_config riemann_fit, mixed_fit)
enum FitMode { kFitBrokenLine, kFitRiemann, kFitBrokenLineMixed, kFitRiemannMixed };

// the tuples of multiplicity bin nh of every event of the batch, as one flat
// range over the events (uneven events share the whole grid): pre[e] is the
// exclusive prefix of the per-event bin sizes, built by each block
__device__ __forceinline__ uint32_t fitBinPrefix(const Workspace& ws, uint32_t nh, uint32_t nEvents, uint32_t* pre,
                                                 uint32_t* scanSh) {
  uint32_t carry = 0;
  for (uint32_t e0 = 0; e0 < nEvents; e0 += blockDim.x) {
    const uint32_t e = e0 + threadIdx.x;
    const uint32_t v = e < nEvents ? min(ws.tmOff[size_t(e) * 16 + nh], ws.cap.multiplicity) : 0u;
    uint32_t tot;
    const uint32_t x = blockExclusiveScan(v, scanSh, &tot);
    if (e < nEvents) pre[e] = carry + x;
    carry += tot;
  }
  if (threadIdx.x == 0) pre[nEvents] = carry;
  __syncthreads();
  return pre[nEvents];
}

// one thread per (tuple of the multiplicity bin nh); fits the first N hits
template <int N, int kMode = kFitBrokenLine>
__device__ __forceinline__ void blFitBin(const DeviceES& es, const Workspace& ws, uint32_t nh, uint32_t nEvents,
                                         uint32_t* pre, uint32_t* scanSh) {
  const uint32_t total = fitBinPrefix(ws, nh, nEvents, pre, scanSh);
  const double B = double(float(0.0114256972711507));
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
    // the event of flat item g: the last e with pre[e] <= g (empty events skipped)
    uint32_t lo = 0, hi = nEvents;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (pre[mid] <= g)
        lo = mid;
      else
        hi = mid;
    }
    const uint32_t e = lo, k = g - pre[lo];
    const uint32_t start = ws.tmOff[size_t(e) * 16 + 8 + nh];
    const uint32_t* bins = ws.tmBins + size_t(e) * ws.cap.tuples;
    const uint32_t* toff = ws.tupleOff + size_t(e) * (ws.cap.tuples + 1);
    const uint32_t* th = ws.tupleHits + size_t(e) * ws.cap.tupleHits();
    const size_t hb = size_t(e) * ws.cap.hits;
    const size_t tb = size_t(e) * ws.cap.tuples;
    uint32_t tkid = bins[start + k];
    const uint32_t* hid = th + toff[tkid];
    double H[3 * N];
    float ge[6 * N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
      uint32_t hit = hid[i];
      const PfFrame& f = es.det[ws.detInd[hb + hit]].frame;
      float cxx = ws.xerr[hb + hit], cxy = 0, cyy = ws.yerr[hb + hit];
      float* gl = ge + 6 * i;
      gl[0] = f.R11 * (f.R11 * cxx + f.R21 * cxy) + f.R21 * (f.R11 * cxy + f.R21 * cyy);
      gl[1] = f.R11 * (f.R12 * cxx + f.R22 * cxy) + f.R21 * (f.R12 * cxy + f.R22 * cyy);
      gl[2] = f.R12 * (f.R12 * cxx + f.R22 * cxy) + f.R22 * (f.R12 * cxy + f.R22 * cyy);
      gl[3] = f.R11 * (f.R13 * cxx + f.R23 * cxy) + f.R21 * (f.R13 * cxy + f.R23 * cyy);
      gl[4] = f.R12 * (f.R13 * cxx + f.R23 * cxy) + f.R22 * (f.R13 * cxy + f.R23 * cyy);
      gl[5] = f.R13 * (f.R13 * cxx + f.R23 * cxy) + f.R23 * (f.R13 * cxy + f.R23 * cyy);
      H[3 * i + 0] = ws.xg[hb + hit];
      H[3 * i + 1] = ws.yg[hb + hit];
      H[3 * i + 2] = ws.zg[hb + hit];
    }
    FitOut o;
    if constexpr (kMode == kFitRiemann) {
      rfFit<N, double>(H, ge, B, o);
    } else if constexpr (kMode == kFitRiemannMixed) {
      rfFit<N, float>(H, ge, B, o);
    } else if constexpr (kMode == kFitBrokenLineMixed) {
      // the mixed fit takes single-precision hits relative to the first one
      // and the first hit in double precision (k_fit_mixed.cuh)
      float Hf[3 * N];
#pragma unroll
      for (int i = 0; i < N; ++i) {
        Hf[3 * i + 0] = float(H[3 * i + 0] - H[0]);
        Hf[3 * i + 1] = float(H[3 * i + 1] - H[1]);
        Hf[3 * i + 2] = float(H[3 * i + 2]);
      }
      blFitMixed<N>(Hf, ge, H[0], H[1], float(B), B, o);
    } else {
      blFit<N>(H, ge, B, o);
    }
#pragma unroll
    for (int j = 0; j < 5; ++j) ws.state[tb * 5 + size_t(tkid) * 5 + j] = o.state[j];
#pragma unroll
    for (int j = 0; j < 15; ++j) ws.cov[tb * 15 + size_t(tkid) * 15 + j] = o.cov[j];
    ws.pt[tb + tkid] = o.pt;
    ws.eta[tb + tkid] = o.eta;
    ws.chi2[tb + tkid] = o.chi2;
  }
}

// the three multiplicity bins in one launch: blockIdx.z = 0, 1, 2 fits the
// 3-hit tuples, the 4-hit tuples and the first 4 hits of the 5-hit tuples
__global__ void __launch_bounds__(128, 4) kBLFit(DeviceES es, Workspace ws, uint32_t nEvents) {
  __shared__ uint32_t pre[kFlatMaxEvents + 1], scanSh[33];
  if (blockIdx.z == 0)
    blFitBin<3>(es, ws, 3, nEvents, pre, scanSh);
  else
    blFitBin<4>(es, ws, 3 + blockIdx.z, nEvents, pre, scanSh);
}

// the same bins through the Riemann fit (useRiemannFit,
// CAHitNtupletGeneratorOnGPU.cc:116-120; RiemannFitOnGPU.cc:3-110)
__global__ void __launch_bounds__(128) kRiemannFit(DeviceES es, Workspace ws, uint32_t nEvents) {
  __shared__ uint32_t pre[kFlatMaxEvents + 1], scanSh[33];
  if (blockIdx.z == 0)
    blFitBin<3, kFitRiemann>(es, ws, 3, nEvents, pre, scanSh);
  else
    blFitBin<4, kFitRiemann>(es, ws, 3 + blockIdx.z, nEvents, pre, scanSh);
}

// the mixed-precision variants of both fits inside the chain (pg_config
// mixed_fit): a precision choice beside the reference's FP64 fits, whose
// effect on the chain's quality codes and vertices is measured against them
__global__ void __launch_bounds__(128, 4) kBLFitMixed(DeviceES es, Workspace ws, uint32_t nEvents) {
  __shared__ uint32_t pre[kFlatMaxEvents + 1], scanSh[33];
  if (blockIdx.z == 0)
    blFitBin<3, kFitBrokenLineMixed>(es, ws, 3, nEvents, pre, scanSh);
  else
    blFitBin<4, kFitBrokenLineMixed>(es, ws, 3 + blockIdx.z, nEvents, pre, scanSh);
}
__global__ void __launch_bounds__(128) kRiemannFitMixed(DeviceES es, Workspace ws, uint32_t nEvents) {
  __shared__ uint32_t pre[kFlatMaxEvents + 1], scanSh[33];
  if (blockIdx.z == 0)
    blFitBin<3, kFitRiemannMixed>(es, ws, 3, nEvents, pre, scanSh);
  else
    blFitBin<4, kFitRiemannMixed>(es, ws, 3 + blockIdx.z, nEvents, pre, scanSh);
}

// standalone fit of externally supplied tuples (fit workload and tests)
template <int N>
__global__ void kBLFitDirect(uint32_t n, const double* hits, const float* hge, double B, float* state, float* cov,
                             float* pt, float* eta, float* chi2) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    double H[3 * N];
    float ge[6 * N];
#pragma unroll
    for (int k = 0; k < 3 * N; ++k) H[k] = hits[size_t(t) * 3 * N + k];
#pragma unroll
    for (int k = 0; k < 6 * N; ++k) ge[k] = hge[size_t(t) * 6 * N + k];
    FitOut o;
    blFit<N>(H, ge, B, o);
#pragma unroll
    for (int j = 0; j < 5; ++j) state[size_t(t) * 5 + j] = o.state[j];
#pragma unroll
    for (int j = 0; j < 15; ++j) cov[size_t(t) * 15 + j] = o.cov[j];
    pt[t] = o.pt;
    eta[t] = o.eta;
    chi2[t] = o.chi2;
  }
}


}  // namespace

cudaError_t runFits(const DeviceES& es, Workspace& ws, uint32_t nEvents, cudaStream_t stream, bool riemann) {
  const uint32_t gx = nEvents >= 32 ? 8 : (nEvents >= 8 ? 32 : 148);
  dim3 g(gx, nEvents);
  PG_PROBED("kFitZero", stream, kFitZero<<<dim3(tunedGrid(ws, kTuneFitZero, g.x), nEvents), 256, 0, stream>>>(ws));
  // FP64-bound: enough warps per SM to cover the double-precision latency
  const uint32_t fx = nEvents >= 32 ? 16 : (nEvents >= 8 ? 64 : 296);
  // one flat grid over the batch's tuples (z: the multiplicity bin), as many
  // blocks as a grid row per event would have
  const dim3 fg(tunedGrid(ws, kTuneFit, fx) * nEvents, 1, 3);
  if (riemann && ws.ca.mixedFit)
    PG_PROBED("kRiemannFitMixed", stream, kRiemannFitMixed<<<fg, 128, 0, stream>>>(es, ws, nEvents));
  else if (riemann)
    PG_PROBED("kRiemannFit", stream, kRiemannFit<<<fg, 128, 0, stream>>>(es, ws, nEvents));
  else if (ws.ca.mixedFit)
    PG_PROBED("kBLFitMixed", stream, kBLFitMixed<<<fg, 128, 0, stream>>>(es, ws, nEvents));
  else
    PG_PROBED("kBLFit", stream, kBLFit<<<fg, 128, 0, stream>>>(es, ws, nEvents));
  return cudaGetLastError();
}

cudaError_t fitDirect(int N, uint32_t n, const double* hits, const float* ge, double B, float* state, float* cov,
                      float* pt, float* eta, float* chi2, cudaStream_t stream) {
  uint32_t blocks = (n + 127) / 128;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks == 0) return cudaSuccess;
  if (N == 3)
    PG_PROBED("kBLFitDirect", stream, kBLFitDirect<3><<<blocks, 128, 0, stream>>>(n, hits, ge, B, state, cov, pt, eta, chi2));
  else
    PG_PROBED("kBLFitDirect", stream, kBLFitDirect<4><<<blocks, 128, 0, stream>>>(n, hits, ge, B, state, cov, pt, eta, chi2));
  return cudaGetLastError();
}

cudaError_t fitDirectMixed(int N, uint32_t n, const double* hits, const float* ge, double B, float* state, float* cov,
                           float* pt, float* eta, float* chi2, cudaStream_t stream) {
  uint32_t blocks = (n + 127) / 128;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks == 0) return cudaSuccess;
  if (N == 3)
    PG_PROBED("kBLFitDirectMixed", stream,
              kBLFitDirectMixed<3><<<blocks, 128, 0, stream>>>(n, hits, ge, B, state, cov, pt, eta, chi2));
  else
    PG_PROBED("kBLFitDirectMixed", stream,
              kBLFitDirectMixed<4><<<blocks, 128, 0, stream>>>(n, hits, ge, B, state, cov, pt, eta, chi2));
  return cudaGetLastError();
}

cudaError_t fitDirectRiemann(int N, uint32_t n, const double* hits, const float* ge, double B, float* state,
                             float* cov, float* pt, float* eta, float* chi2, bool mixed, cudaStream_t stream) {
  uint32_t blocks = (n + 127) / 128;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks == 0) return cudaSuccess;
  if (N == 3 && !mixed)
    PG_PROBED("kRiemannFitDirect", stream,
              kRiemannFitDirect<3, double><<<blocks, 128, 0, stream>>>(n, hits, ge, B, state, cov, pt, eta, chi2));
  else if (!mixed)
    PG_PROBED("kRiemannFitDirect", stream,
              kRiemannFitDirect<4, double><<<blocks, 128, 0, stream>>>(n, hits, ge, B, state, cov, pt, eta, chi2));
  else if (N == 3)
    PG_PROBED("kRiemannFitDirectMixed", stream,
              kRiemannFitDirect<3, float><<<blocks, 128, 0, stream>>>(n, hits, ge, B, state, cov, pt, eta, chi2));
  else
    PG_PROBED("kRiemannFitDirectMixed", stream,
              kRiemannFitDirect<4, float><<<blocks, 128, 0, stream>>>(n, hits, ge, B, state, cov, pt, eta, chi2));
  return cudaGetLastError();
}

}  // namespace pixgpu
