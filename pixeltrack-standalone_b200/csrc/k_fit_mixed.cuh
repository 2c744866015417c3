// Mixed-precision broken-line fit (included by k_fit.cu inside its
// namespaces, after the FP64 fit whose matrix type and Cholesky inversions it
// reuses).
//
// The arithmetic of the fit runs in FP32: the multiple-scattering
// variances, the rotations and projections of the hit errors, the band
// matrices, the residual weights and the chi2.  FP64 is kept for the two
// Cholesky inversions with the solves that use them, for the covariance
// propagation (Jacobian sandwiches and the Karimaki translation), for the
// three-point reference circle, and for what is measured from that circle:
// the arc lengths and the radial residuals, which are small differences and
// angles of vectors as long as the radius.  The steps follow
// BrokenLine.h:46-504 exactly as the FP64 path does; only the precision
// differs.

template <int R, int C>
struct MF {
  float a[R * C];
  __device__ __forceinline__ float& operator()(int i, int j) { return a[i + j * R]; }
  __device__ __forceinline__ float operator()(int i, int j) const { return a[i + j * R]; }
};

template <int R, int K, int C>
__device__ __forceinline__ MF<R, C> mulf(const MF<R, K>& x, const MF<K, C>& y) {
  MF<R, C> r;
#pragma unroll
  for (int j = 0; j < C; ++j)
#pragma unroll
    for (int i = 0; i < R; ++i) {
      float s = x(i, 0) * y(0, j);
#pragma unroll
      for (int k = 1; k < K; ++k) s += x(i, k) * y(k, j);
      r(i, j) = s;
    }
  return r;
}

template <int R, int C>
__device__ __forceinline__ MF<C, R> trf(const MF<R, C>& x) {
  MF<C, R> r;
#pragma unroll
  for (int j = 0; j < C; ++j)
#pragma unroll
    for (int i = 0; i < R; ++i) r(j, i) = x(i, j);
  return r;
}

__device__ __forceinline__ float sqrf(float a) { return a * a; }

__device__ __forceinline__ float multScattF(float length, float B, float R, float slope) {
  float pt2 = fminf(20.f, B * R);
  pt2 *= pt2;
  constexpr float XXI_0 = 0.06f / 16.f;
  constexpr float fact = 0.7f * ((13.6f / 1000.f) * (13.6f / 1000.f));
  return fact / (pt2 * (1.f + sqrf(slope))) * (fabsf(length) * XXI_0) * sqrf(1.f + 0.038f * logf(fabsf(length) * XXI_0));
}

__device__ __forceinline__ MF<2, 2> rotationMatrixF(float slope) {
  MF<2, 2> r;
  r(0, 0) = 1.f / sqrtf(1.f + sqrf(slope));
  r(0, 1) = slope * r(0, 0);
  r(1, 0) = -r(0, 1);
  r(1, 1) = r(0, 0);
  return r;
}

__device__ __forceinline__ float cross2DF(float ax, float ay, float bx, float by) { return ax * by - ay * bx; }

template <int N>
__device__ MF<N, N> matrixCuF(const float* w, const float* S, const float* VarBeta) {
  constexpr int n = N;
  MF<N, N> C;
#pragma unroll
  for (int k = 0; k < N * N; ++k) C.a[k] = 0;
#pragma unroll
  for (int i = 0; i < n; ++i) {
    C(i, i) = w[i];
    if (i > 1) C(i, i) += 1.f / (VarBeta[i - 1] * sqrf(S[i] - S[i - 1]));
    if (i > 0 && i < n - 1)
      C(i, i) += (1.f / VarBeta[i]) * sqrf((S[i + 1] - S[i - 1]) / ((S[i + 1] - S[i]) * (S[i] - S[i - 1])));
    if (i < n - 2) C(i, i) += 1.f / (VarBeta[i + 1] * sqrf(S[i + 1] - S[i]));
    if (i > 0 && i < n - 1)
      C(i, i + 1) =
          1.f / (VarBeta[i] * (S[i + 1] - S[i])) * (-(S[i + 1] - S[i - 1]) / ((S[i + 1] - S[i]) * (S[i] - S[i - 1])));
    if (i < n - 2)
      C(i, i + 1) += 1.f / (VarBeta[i + 1] * (S[i + 1] - S[i])) *
                     (-(S[i + 2] - S[i]) / ((S[i + 2] - S[i + 1]) * (S[i + 1] - S[i])));
    if (i < n - 2) C(i, i + 2) = 1.f / (VarBeta[i + 1] * (S[i + 2] - S[i + 1]) * (S[i + 1] - S[i]));
    C(i, i) *= 0.5f;
  }
  MF<N, N> R;
#pragma unroll
  for (int j = 0; j < n; ++j)
#pragma unroll
    for (int i = 0; i < n; ++i) R(i, j) = C(i, j) + C(j, i);
  return R;
}

// FP32 band matrix -> FP64 inverse
template <int N>
__device__ __forceinline__ void invertToDouble(const MF<N, N>& c, M<N, N>& inv) {
  M<N, N> d;
#pragma unroll
  for (int k = 0; k < N * N; ++k) d.a[k] = double(c.a[k]);
  invert(d, inv);
}

// hits: x,y,z of hit i at H[3*i+k] in FP32, with x and y taken relative to
// the first hit (x0, y0), the differences formed in FP64 from the inputs:
// the circle's sagitta is a small difference of transverse positions, and
// FP32 absolute coordinates would lose it.  ge: 6 floats per hit.
template <int N>
__device__ void blFitMixed(const float* H3, const float* ge, double x0, double y0, float Bf, double B, FitOut& out) {
  constexpr int n = N;
  auto H = [&](int r, int c) { return H3[3 * c + r]; };
  // the fast fit (the reference circle every residual is taken against) in
  // FP64: for a straight-looking track its centre is a ratio of small
  // differences, and every later FP32 step inherits its error
  float ff[4];
  double fc0, fc1, fc2;  // the circle in FP64, for the arc lengths below
  {
    auto Hd = [&](int r, int c) { return double(H3[3 * c + r]); };
    double ax = Hd(0, n / 2) - Hd(0, 0), ay = Hd(1, n / 2) - Hd(1, 0);
    double bx = Hd(0, n - 1) - Hd(0, n / 2), by = Hd(1, n - 1) - Hd(1, n / 2);
    double cx = Hd(0, 0) - Hd(0, n - 1), cy = Hd(1, 0) - Hd(1, n - 1);
    double tmp = 0.5 / cross2D(cx, cy, ax, ay);
    double csq = cx * cx + cy * cy, asq = ax * ax + ay * ay, bsq = bx * bx + by * by;
    const double f0 = Hd(0, 0) - (ay * csq + cy * asq) * tmp;
    const double f1 = Hd(1, 0) + (ax * csq + cx * asq) * tmp;
    const double f2 = sqrt(asq * bsq * csq) / (2. * fabs(cross2D(bx, by, ax, ay)));
    double dx = Hd(0, 0) - f0, dy = Hd(1, 0) - f1;
    double ex = Hd(0, n - 1) - f0, ey = Hd(1, n - 1) - f1;
    ff[0] = float(f0);
    ff[1] = float(f1);
    ff[2] = float(f2);
    fc0 = f0;
    fc1 = f1;
    fc2 = f2;
    ff[3] = float(f2 * atan2(cross2D(dx, dy, ex, ey), dx * ex + dy * ey) / (Hd(2, n - 1) - Hd(2, 0)));
  }
  int q;
  float radii[2][N], s[N], S[N], Z[N], VarBeta[N];
  {
    float dx = H(0, 1) - H(0, 0), dy = H(1, 1) - H(1, 0);
    float ex = H(0, n - 1) - H(0, n - 2), ey = H(1, n - 1) - H(1, n - 2);
    q = cross2DF(dx, dy, ex, ey) > 0 ? -1 : 1;
    const float slope = -q / ff[3];
    MF<2, 2> R = rotationMatrixF(slope);
    // the arc lengths in FP64: the radius vectors are as long as the radius
    // (metres for a stiff track) and the angles between them small, so in
    // FP32 their cross products, and the circle centre itself, would carry
    // errors of the size of the arc lengths' last digits times the radius
    double rd[2][N];
#pragma unroll
    for (int i = 0; i < n; ++i) {
      rd[0][i] = double(H(0, i)) - fc0;
      rd[1][i] = double(H(1, i)) - fc1;
      radii[0][i] = float(rd[0][i]);
      radii[1][i] = float(rd[1][i]);
    }
    // the circle centre in the beam-line frame gives the direction of the
    // point of closest approach
    const double cax = fc0 + x0, cay = fc1 + y0;
    const double nrm = sqrt(cax * cax + cay * cay);
    const double e0 = (-fc2 * cax) / nrm, e1 = (-fc2 * cay) / nrm;
#pragma unroll
    for (int i = 0; i < n; ++i)
      s[i] = float(q * fc2 * atan2(cross2D(rd[0][i], rd[1][i], e0, e1), rd[0][i] * e0 + rd[1][i] * e1));
#pragma unroll
    for (int i = 0; i < n; ++i) {
      float p0 = s[i], p1 = H(2, i);
      S[i] = R(0, 0) * p0 + R(0, 1) * p1;
      Z[i] = R(1, 0) * p0 + R(1, 1) * p1;
    }
    VarBeta[0] = VarBeta[n - 1] = 0;
#pragma unroll
    for (int i = 1; i < n - 1; ++i)
      VarBeta[i] = multScattF(S[i + 1] - S[i], Bf, ff[2], slope) + multScattF(S[i] - S[i - 1], Bf, ff[2], slope);
  }
  // ---- line fit
  float lpar[2];
  M<2, 2> lcov;
  float lchi2;
  {
    const float slope = -q / ff[3];
    MF<2, 2> R = rotationMatrixF(slope);
    MF<3, 3> V;
    MF<2, 3> J;
#pragma unroll
    for (int k = 0; k < 9; ++k) V.a[k] = 0;
#pragma unroll
    for (int k = 0; k < 6; ++k) J.a[k] = 0;
    float w[N];
#pragma unroll
    for (int i = 0; i < n; ++i) {
      const float* g = ge + 6 * i;
      V(0, 0) = g[0];
      V(0, 1) = V(1, 0) = g[1];
      V(0, 2) = V(2, 0) = g[3];
      V(1, 1) = g[2];
      V(2, 1) = V(1, 2) = g[4];
      V(2, 2) = g[5];
      float tmp = 1.f / sqrtf(radii[0][i] * radii[0][i] + radii[1][i] * radii[1][i]);
      J(0, 0) = radii[1][i] * tmp;
      J(0, 1) = -radii[0][i] * tmp;
      J(1, 2) = 1.f;
      MF<2, 2> P = mulf(mulf(mulf(mulf(R, J), V), trf(J)), trf(R));
      w[i] = 1.f / P(1, 1);
    }
    M<N, N> I;
    invertToDouble<N>(matrixCuF<N>(w, S, VarBeta), I);
    double u[N];
#pragma unroll
    for (int i = 0; i < n; ++i) {
      double acc = I(i, 0) * double(w[0] * Z[0]);
#pragma unroll
      for (int k = 1; k < n; ++k) acc += I(i, k) * double(w[k] * Z[k]);
      u[i] = acc;
    }
    lpar[0] = float(u[1] - u[0]) / (S[1] - S[0]);
    lpar[1] = float(u[0]);
    const double idiff = 1. / double(S[1] - S[0]);
    lcov(0, 0) = (I(0, 0) - 2 * I(0, 1) + I(1, 1)) * sqr(idiff) + double(multScattF(S[1] - S[0], Bf, ff[2], slope));
    lcov(0, 1) = (I(0, 1) - I(0, 0)) * idiff;
    lcov(1, 0) = (I(0, 1) - I(0, 0)) * idiff;
    lcov(1, 1) = I(0, 0);
    M<2, 2> jac;
    jac(0, 0) = 1.;
    jac(0, 1) = 0;
    jac(1, 0) = -double(S[0]);
    jac(1, 1) = 1.;
    lpar[1] += -lpar[0] * S[0];
    lcov = sandwich(jac, lcov);
    const float t = R(0, 0) - lpar[0] * R(0, 1);
    jac(1, 1) = 1. / double(t);
    jac(0, 0) = jac(1, 1) * jac(1, 1);
    jac(0, 1) = 0;
    jac(1, 0) = double(lpar[1]) * double(R(0, 1)) * jac(0, 0);
    lpar[1] = lpar[1] / t;
    lpar[0] = (R(0, 1) + lpar[0] * R(0, 0)) / t;
    lcov = sandwich(jac, lcov);
    lchi2 = 0;
#pragma unroll
    for (int i = 0; i < n; ++i) {
      const float ui = float(u[i]);
      lchi2 += w[i] * sqrf(Z[i] - ui);
      if (i > 0 && i < n - 1)
        lchi2 += sqrf(float(u[i - 1]) / (S[i] - S[i - 1]) -
                      ui * (S[i + 1] - S[i - 1]) / ((S[i + 1] - S[i]) * (S[i] - S[i - 1])) +
                      float(u[i + 1]) / (S[i + 1] - S[i])) /
                 VarBeta[i];
    }
  }
  // ---- circle fit
  double cpar[3];
  M<3, 3> ccov;
  float cchi2;
  {
    const float slope = -q / ff[3];
#pragma unroll
    for (int i = 0; i < n; ++i) VarBeta[i] *= 1.f + sqrf(slope);
#pragma unroll
    for (int i = 0; i < n; ++i) {
      // radial residual to the reference circle: a difference of two numbers
      // of the size of the radius (metres at high pT), formed in FP64
      const double r0 = double(H(0, i)) - double(ff[0]), r1 = double(H(1, i)) - double(ff[1]);
      Z[i] = float(sqrt(r0 * r0 + r1 * r1) - double(ff[2]));
    }
    float w[N];
#pragma unroll
    for (int i = 0; i < n; ++i) {
      const float* g = ge + 6 * i;
      MF<2, 2> V;
      V(0, 0) = g[0];
      V(0, 1) = V(1, 0) = g[1];
      V(1, 1) = g[2];
      MF<2, 2> RR = rotationMatrixF(-radii[0][i] / radii[1][i]);
      MF<2, 2> P = mulf(mulf(RR, V), trf(RR));
      w[i] = 1.f / P(1, 1);
    }
    MF<N + 1, N + 1> C;
    {
      MF<N, N> cu = matrixCuF<N>(w, s, VarBeta);
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
        C(i, n) +=
            -(s[i + 1] - s[i - 1]) * (s[i + 1] - s[i - 1]) / (2.f * VarBeta[i] * (s[i + 1] - s[i]) * (s[i] - s[i - 1]));
      if (i > 1) C(i, n) += (s[i] - s[i - 2]) / (2.f * VarBeta[i - 1] * (s[i] - s[i - 1]));
      if (i < n - 2) C(i, n) += (s[i + 2] - s[i]) / (2.f * VarBeta[i + 1] * (s[i + 1] - s[i]));
      C(n, i) = C(i, n);
      if (i > 0 && i < n - 1) C(n, n) += sqrf(s[i + 1] - s[i - 1]) / (4.f * VarBeta[i]);
    }
    M<N + 1, N + 1> I;
    invertToDouble<N + 1>(C, I);
    double u[N + 1];
#pragma unroll
    for (int i = 0; i < n + 1; ++i) {
      double acc = 0;
#pragma unroll
      for (int k = 0; k < n; ++k) acc += I(i, k) * double(w[k] * Z[k]);
      u[i] = acc;
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const float nr = sqrtf(radii[0][c] * radii[0][c] + radii[1][c] * radii[1][c]);
      radii[0][c] /= nr;
      radii[1][c] /= nr;
    }
    const float u0 = float(u[0]), u1 = float(u[1]);
    const float dx = H(0, 0) + (-Z[0] + u0) * radii[0][0], dy = H(1, 0) + (-Z[0] + u0) * radii[1][0];
    const float ex = H(0, 1) + (-Z[1] + u1) * radii[0][1], ey = H(1, 1) + (-Z[1] + u1) * radii[1][1];
    const float emdx = ex - dx, emdy = ey - dy;
    cpar[0] = double(atan2f(emdy, emdx));
    // R - sqrt(R^2 - a) in the form without cancellation
    const float quarter = 0.25f * (emdx * emdx + emdy * emdy);
    cpar[1] = double(-q * (quarter / (ff[2] + sqrtf(sqrf(ff[2]) - quarter))));
    cpar[2] = double(q * (1.f / ff[2] + float(u[n])));
    const float tmp1 = emdx * emdx + emdy * emdy;
    M<3, 3> J;
    J(0, 0) = double((radii[1][0] * emdx - emdy * radii[0][0]) / tmp1);
    J(0, 1) = double((radii[1][1] * emdx - emdy * radii[0][1]) / tmp1);
    J(0, 2) = 0;
    J(1, 0) = double((q / 2) * (emdx * radii[0][0] + emdy * radii[1][0]) / sqrtf(sqrf(2 * ff[2]) - tmp1));
    J(1, 1) = double((q / 2) * (emdx * radii[0][1] + emdy * radii[1][1]) / sqrtf(sqrf(2 * ff[2]) - tmp1));
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
    translateKarimaki(cpar, ccov, 0.5 * double(emdx), 0.5 * double(emdy));
    ccov(0, 0) += double((1.f + sqrf(slope)) * multScattF(S[1] - S[0], Bf, ff[2], slope));
    translateKarimaki(cpar, ccov, double(dx) + x0, double(dy) + y0);
    cchi2 = 0;
#pragma unroll
    for (int i = 0; i < n; ++i) {
      const float ui = float(u[i]);
      cchi2 += w[i] * sqrf(Z[i] - ui);
      if (i > 0 && i < n - 1)
        cchi2 += sqrf(float(u[i - 1]) / (s[i] - s[i - 1]) -
                      ui * (s[i + 1] - s[i - 1]) / ((s[i + 1] - s[i]) * (s[i] - s[i - 1])) +
                      float(u[i + 1]) / (s[i + 1] - s[i]) + (s[i + 1] - s[i - 1]) * float(u[n]) / 2) /
                 VarBeta[i];
    }
  }
  const float b = 1.f / Bf;
  out.state[0] = float(cpar[0]);
  out.state[1] = float(cpar[1]);
  out.state[2] = float(cpar[2]) * b;
  out.state[3] = lpar[0];
  out.state[4] = lpar[1];
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
  out.pt = Bf / fabsf(float(cpar[2]));
  out.eta = asinhf(lpar[0]);
  out.chi2 = (cchi2 + lchi2) / float(2 * N - 5);
  (void)B;
}

// standalone mixed-precision fit of externally supplied tuples
template <int N>
__global__ void kBLFitDirectMixed(uint32_t n, const double* hits, const float* hge, double B, float* state,
                                  float* cov, float* pt, float* eta, float* chi2) {
  const float Bf = float(B);
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    float H[3 * N];
    float ge[6 * N];
    const double* h = hits + size_t(t) * 3 * N;
    const double x0 = h[0], y0 = h[1];
#pragma unroll
    for (int i = 0; i < N; ++i) {
      H[3 * i + 0] = float(h[3 * i + 0] - x0);
      H[3 * i + 1] = float(h[3 * i + 1] - y0);
      H[3 * i + 2] = float(h[3 * i + 2]);
    }
#pragma unroll
    for (int k = 0; k < 6 * N; ++k) ge[k] = hge[size_t(t) * 6 * N + k];
    FitOut o;
    blFitMixed<N>(H, ge, x0, y0, Bf, B, o);
#pragma unroll
    for (int j = 0; j < 5; ++j) state[size_t(t) * 5 + j] = o.state[j];
#pragma unroll
    for (int j = 0; j < 15; ++j) cov[size_t(t) * 15 + j] = o.cov[j];
    pt[t] = o.pt;
    eta[t] = o.eta;
    chi2[t] = o.chi2;
  }
}
