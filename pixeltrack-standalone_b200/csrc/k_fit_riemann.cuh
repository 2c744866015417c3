// Riemann helix fit on B200, one thread per tuple, FP64 as in the reference:
// Fast_fit, Circle_fit (with its error propagation), Line_fit and the
// perigee conversion of plugin-PixelTriplets/RiemannFit.h:31-758 and
// FitUtils.h:89-214, packed as kernelLineFit does (RiemannFitOnGPU.h:156-162,
// TrajectoryStateSoA.h:21-38).  The reference runs it as three kernels with
// per-fit scratch in global memory; here one thread carries a tuple from
// the hits to the packed track state, its matrices in registers and local
// memory.
//
// The smallest eigenvector of the 3x3 Riemann matrix comes from a
// closed-form solver: eigenvalues from the depressed characteristic cubic
// (trigonometric roots) of the matrix scaled by its largest coefficient and
// shifted by its mean diagonal; the eigenvector as the longest cross product
// of two rows of (C - w I) when the smallest eigenvalue is at least as
// isolated as the largest, otherwise from the 2x2 restriction of C to the
// plane orthogonal to the largest eigenvector.  The single-precision solve of
// the numerical Jacobian (min_eigen3D_fast, RiemannFit.h:328-334) rounds the
// matrix to single precision, solves it in double precision and rounds the
// eigenvector to single precision.
//
// Included inside the anonymous namespace of k_fit.cu, after M, mul, tr,
// sandwich, invert and FitOut.

#include <type_traits>

constexpr double kRfDeriv = 1.e-4;  // FitUtils.h:12
constexpr double kRfPi = 3.14159265358979323846;

// choleskyInversion.h:28-40 + symmetrisation; d may alias s
__device__ __forceinline__ void invert(const M<2, 2>& s, M<2, 2>& d) {
  const double luc0 = 1.0 / s(0, 0);
  const double luc1 = s(1, 0) * s(1, 0) * luc0;
  const double luc2 = 1.0 / (s(1, 1) - luc1);
  const double li21 = luc1 * luc0 * luc2;
  const double d10 = -s(1, 0) * luc0 * luc2;
  d(0, 0) = li21 + luc0;
  d(1, 0) = d10;
  d(1, 1) = luc2;
  d(0, 1) = d10;
}

template <typename T>
__device__ __forceinline__ void rfCross(const T* a, const T* b, T* r) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}
template <typename T>
__device__ __forceinline__ T rfDot(const T* a, const T* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// a unit vector orthogonal to the unit vector u
template <typename T>
__device__ __forceinline__ void rfOrtho(const T* u, T* e) {
  int ax = 0;
  if (fabs(u[1]) < fabs(u[ax])) ax = 1;
  if (fabs(u[2]) < fabs(u[ax])) ax = 2;
  T a[3] = {T(0), T(0), T(0)};
  a[ax] = T(1);
  rfCross(u, a, e);
  const T inv = T(1) / sqrt(rfDot(e, e));
  for (int k = 0; k < 3; ++k) e[k] *= inv;
}

// unit null vector of a rank-2 symmetric 3x3 (rows Mx[0..2])
template <typename T>
__device__ void rfNull(const T (*Mx)[3], T* v) {
  T x[3][3];
  rfCross(Mx[0], Mx[1], x[0]);
  rfCross(Mx[0], Mx[2], x[1]);
  rfCross(Mx[1], Mx[2], x[2]);
  const T n[3] = {rfDot(x[0], x[0]), rfDot(x[1], x[1]), rfDot(x[2], x[2])};
  int b = 0;
  if (n[1] > n[b]) b = 1;
  if (n[2] > n[b]) b = 2;
  if (n[b] > T(0)) {
    const T inv = T(1) / sqrt(n[b]);
    for (int k = 0; k < 3; ++k) v[k] = x[b][k] * inv;
    return;
  }
  const T r[3] = {rfDot(Mx[0], Mx[0]), rfDot(Mx[1], Mx[1]), rfDot(Mx[2], Mx[2])};
  int br = 0;
  if (r[1] > r[br]) br = 1;
  if (r[2] > r[br]) br = 2;
  if (!(r[br] > T(0))) {
    v[0] = T(1), v[1] = T(0), v[2] = T(0);
    return;
  }
  T u[3];
  const T inv = T(1) / sqrt(r[br]);
  for (int k = 0; k < 3; ++k) u[k] = Mx[br][k] * inv;
  rfOrtho(u, v);
}

// smallest eigenvalue w0 and its unit eigenvector v of the symmetric A
template <typename T>
__device__ void rfMinEigen(const T (*A)[3], T& w0, T* v) {
  T s = T(0);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) s = fabs(A[i][j]) > s ? fabs(A[i][j]) : s;
  v[0] = T(1), v[1] = T(0), v[2] = T(0);
  if (!(s > T(0))) {
    w0 = T(0);
    return;
  }
  const T is = T(1) / s;
  T C[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) C[i][j] = A[i][j] * is;
  const T m = (C[0][0] + C[1][1] + C[2][2]) / T(3);
  for (int i = 0; i < 3; ++i) C[i][i] -= m;
  const T p2 = (C[0][0] * C[0][0] + C[1][1] * C[1][1] + C[2][2] * C[2][2] +
                T(2) * (C[0][1] * C[0][1] + C[0][2] * C[0][2] + C[1][2] * C[1][2])) /
               T(6);
  if (!(p2 > T(0))) {
    w0 = m * s;
    return;
  }
  const T p = sqrt(p2);
  const T det = C[0][0] * (C[1][1] * C[2][2] - C[1][2] * C[2][1]) - C[0][1] * (C[1][0] * C[2][2] - C[1][2] * C[2][0]) +
                C[0][2] * (C[1][0] * C[2][1] - C[1][1] * C[2][0]);
  T r = det / (T(2) * p2 * p);
  r = r < T(-1) ? T(-1) : (r > T(1) ? T(1) : r);
  const T phi = acos(r) / T(3);
  const T third = T(2.0943951023931954923);  // 2 pi / 3
  const T c2 = T(2) * p * cos(phi);
  T c0 = T(2) * p * cos(phi + third);
  const T c1 = T(2) * p * cos(phi + T(2) * third);
  T Mx[3][3];
  if (c1 - c0 >= c2 - c1) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) Mx[i][j] = C[i][j] - (i == j ? c0 : T(0));
    rfNull(Mx, v);
  } else {
    T u2[3], e[3], f[3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) Mx[i][j] = C[i][j] - (i == j ? c2 : T(0));
    rfNull(Mx, u2);
    rfOrtho(u2, e);
    rfCross(u2, e, f);
    T Ce[3], Cf[3];
    for (int i = 0; i < 3; ++i) {
      Ce[i] = C[i][0] * e[0] + C[i][1] * e[1] + C[i][2] * e[2];
      Cf[i] = C[i][0] * f[0] + C[i][1] * f[1] + C[i][2] * f[2];
    }
    const T pee = rfDot(e, Ce), pef = rfDot(e, Cf), pff = rfDot(f, Cf);
    const T t = T(0.5) * atan2(T(2) * pef, pee - pff);
    const T ct = cos(t), st = sin(t);
    for (int k = 0; k < 3; ++k) v[k] = -st * e[k] + ct * f[k];
    const T mid = T(0.5) * (pee + pff), half = hypot(T(0.5) * (pee - pff), pef);
    c0 = mid - half;
  }
  w0 = (m + c0) * s;
}

// computeRadLenUniformMaterial (RiemannFit.h:31-40)
template <int N, typename S>
__device__ __forceinline__ void rfRadLen(const S* len, S* rl) {
  constexpr S XX_0_inv = S(0.06 / 16.);
  rl[0] = len[0] * XX_0_inv;
#pragma unroll
  for (int j = 1; j < N; ++j) rl[j] = fabs(len[j] - len[j - 1]) * XX_0_inv;
}

// Fast_fit (RiemannFit.h:368-418), in precision S
template <int N, typename S>
__device__ __forceinline__ void rfFastFit(const double* Hd, S* ff) {
  constexpr int n = N;
  auto H = [&](int k) { return S(Hd[k]); };
  const S bX = H(3 * (n / 2)) - H(0), bY = H(3 * (n / 2) + 1) - H(1);
  const S cX = H(3 * (n - 1)) - H(0), cY = H(3 * (n - 1) + 1) - H(1);
  const S b2 = bX * bX + bY * bY;
  const S c2 = cX * cX + cY * cY;
  const bool flip = fabs(bX) < fabs(bY);
  const S bx = flip ? bY : bX, by = flip ? bX : bY;
  const S cx = flip ? cY : cX, cy = flip ? cX : cY;
  const S div = S(2) * (cx * by - bx * cy);
  const S Y0 = (cx * b2 - bx * c2) / div;
  const S X0 = (S(0.5) * b2 - Y0 * by) / bx;
  ff[0] = H(0) + (flip ? Y0 : X0);
  ff[1] = H(1) + (flip ? X0 : Y0);
  ff[2] = sqrt(X0 * X0 + Y0 * Y0);
  const S dX = H(0) - ff[0], dY = H(1) - ff[1];
  const S eX = H(3 * (n - 1)) - ff[0], eY = H(3 * (n - 1) + 1) - ff[1];
  const S dr = ff[2] * atan2(dX * eY - dY * eX, dX * eX + dY * eY);
  const S dz = H(3 * (n - 1) + 2) - H(2);
  ff[3] = dr / dz;
}

template <int R, int C>
__device__ __forceinline__ M<R, C> rfZero() {
  M<R, C> m;
#pragma unroll
  for (int k = 0; k < R * C; ++k) m.a[k] = 0.;
  return m;
}

struct RfCircle {  // Rfit::circle_fit: chi2 in single precision
  double par[3];
  M<3, 3> cov;
  int q;
  float chi2;
};

struct RfLine {
  double par[2];
  M<2, 2> cov;
  double chi2;
};

// Circle_fit (RiemannFit.h:448-758), V the 2N x 2N transverse covariance.
// S is the precision of the multiple-scattering model and of the
// single-precision eigen-solves of J2 (double: the reference's arithmetic).
template <int N, typename S>
__device__ void rfCircleFit(const double* H, M<2 * N, 2 * N>& V, const S* ff, const S* rad, double B,
                            RfCircle& circle) {
  constexpr int n = N;
  // ---- weights: cov_carttorad_prefit (:232-254) and Scatter_cov_rad (:123-157)
  // (the projections of the hit covariances stay in double precision: the
  // radial variance of a hit can cancel to ~1e-16)
  M<N, N> covRad = rfZero<N, N>();
#pragma unroll
  for (int i = 0; i < n; ++i) {
    if (rad[i] < S(1.e-4)) {
      covRad(i, i) = V(i, i);
    } else {
      const double f0 = ff[0], f1 = ff[1];
      const double ax = H[3 * i], ay = H[3 * i + 1];
      const double bx = ax - f0, by = ay - f1;
      const double x2 = ax * bx + ay * by;
      const double y2 = ax * by - ay * bx;
      const double tan_c = -y2 / x2;
      const double tan_c2 = tan_c * tan_c;
      covRad(i, i) = 1. / (1. + tan_c2) * (V(i, i) + V(i + n, i + n) * tan_c2 + 2 * V(i, i + n) * tan_c);
    }
  }
  M<N, N> scat;
  {
    const S p_t = fmin(S(20), ff[2] * S(B));
    const S p_2 = p_t * p_t * (S(1) + S(1) / (ff[3] * ff[3]));
    S theta = atan(ff[3]);
    theta = theta < S(0) ? theta + S(kRfPi) : theta;
    // the arc lengths feed log(radiation length): kept in double precision,
    // where near-equal lengths of two hits stay distinct
    double len[N], rld[N];
    S rl[N], sig2[N];
    const double f0 = ff[0], f1 = ff[1], f2 = ff[2], f3 = ff[3];
    const double fac = sqrt(1. + 1. / (f3 * f3));
#pragma unroll
    for (int i = 0; i < n; ++i) {
      const double px = H[3 * i] - f0, py = H[3 * i + 1] - f1;
      const double cross = (-f0) * py - (-f1) * px;
      const double dot = (-f0) * px + (-f1) * py;
      len[i] = fabs(atan2(cross, dot) * f2) * fac;
    }
    rfRadLen<N>(len, rld);
#pragma unroll
    for (int i = 0; i < n; ++i) rl[i] = S(rld[i]);
    const S st = sin(theta);
    const S k = S(0.000225) / (p_2 * (st * st));
#pragma unroll
    for (int i = 0; i < n; ++i) {
      const S g = S(1) + S(0.038) * log(rl[i]);
      sig2[i] = g * g * rl[i] * k;
    }
#pragma unroll
    for (int a = 0; a < n; ++a)
#pragma unroll
      for (int b = a; b < n; ++b) {
        S t = S(0);
#pragma unroll
        for (int i = 0; i < a; ++i) t += (rad[a] - rad[i]) * (rad[b] - rad[i]) * sig2[i];
        scat(a, b) = t;
        scat(b, a) = t;
      }
  }
  // cov_radtocart (:168-190) added onto V, in double precision
  {
    double ri[N];
#pragma unroll
    for (int i = 0; i < n; ++i) ri[i] = 1. / sqrt(H[3 * i] * H[3 * i] + H[3 * i + 1] * H[3 * i + 1]);
#pragma unroll
    for (int i = 0; i < n; ++i)
#pragma unroll
      for (int j = i; j < n; ++j) {
        const double c = scat(i, j);
        const double xi = H[3 * i], yi = H[3 * i + 1], xj = H[3 * j], yj = H[3 * j + 1];
        const double c00 = c * yi * ri[i] * yj * ri[j];
        const double c11 = c * xi * ri[i] * xj * ri[j];
        const double c01 = -c * yi * ri[i] * xj * ri[j];
        const double c10 = -c * xi * ri[i] * yj * ri[j];
        V(i, j) += c00;
        V(i + n, j + n) += c11;
        V(i, j + n) += c01;
        if (j != i) {
          V(j, i) += c00;
          V(j + n, i + n) += c11;
          V(i + n, j) += c10;
          V(j + n, i) += c01;
          V(j, i + n) += c10;
        } else {
          V(i + n, i) += c01;
        }
      }
  }
#pragma unroll
  for (int k = 0; k < n * n; ++k) covRad.a[k] += scat.a[k];
  M<N, N> G;
  invert(covRad, G);
  double renorm = 0.;
#pragma unroll
  for (int k = 0; k < n * n; ++k) renorm += G.a[k];
  const double rinv = 1. / renorm;
#pragma unroll
  for (int k = 0; k < n * n; ++k) G.a[k] *= rinv;
  double w[N];
#pragma unroll
  for (int j = 0; j < n; ++j) {
    double s = G(0, j);
#pragma unroll
    for (int i = 1; i < n; ++i) s += G(i, j);
    w[j] = s;
  }
  // ---- space transformation (:475-493)
  double h0 = 0., h1 = 0.;
#pragma unroll
  for (int i = 0; i < n; ++i) h0 += H[3 * i], h1 += H[3 * i + 1];
  h0 /= n;
  h1 /= n;
  M<3, N> p3;
  double mc[2 * N];
#pragma unroll
  for (int i = 0; i < n; ++i) {
    p3(0, i) = H[3 * i] - h0;
    p3(1, i) = H[3 * i + 1] - h1;
    mc[i] = p3(0, i);
    mc[i + n] = p3(1, i);
  }
  double q = 0.;
#pragma unroll
  for (int k = 0; k < 2 * n; ++k) q += mc[k] * mc[k];
  const double s = sqrt(n * 1. / q);
#pragma unroll
  for (int i = 0; i < n; ++i) {
    p3(0, i) *= s;
    p3(1, i) *= s;
    p3(2, i) = p3(0, i) * p3(0, i) + p3(1, i) * p3(1, i);
  }
  // ---- cost function (:497-519)
  double r0[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double t = p3(k, 0) * w[0];
#pragma unroll
    for (int i = 1; i < n; ++i) t += p3(k, i) * w[i];
    r0[k] = t;
  }
  M<3, N> X;
#pragma unroll
  for (int i = 0; i < n; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) X(k, i) = p3(k, i) - r0[k];
  const M<3, 3> A = mul(mul(X, G), tr(X));
  double chi2, v[3];
  {
    double a[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) a[i][j] = A(i, j);
    rfMinEigen(a, chi2, v);
  }
  if (!(v[2] > 0))
#pragma unroll
    for (int k = 0; k < 3; ++k) v[k] *= -1;
  const double c = (-v[0]) * r0[0] + (-v[1]) * r0[1] + (-v[2]) * r0[2];
  // ---- circle parameters (:523-537)
  const double h = sqrt(1. - sqr(v[2]) - 4. * c * v[2]);
  const double v2x2_inv = 1. / (2. * v[2]);
  const double s_inv = 1. / s;
  const double pu[3] = {-v[0] * v2x2_inv, -v[1] * v2x2_inv, h * v2x2_inv};
  circle.par[0] = pu[0] * s_inv + h0;
  circle.par[1] = pu[1] * s_inv + h1;
  circle.par[2] = pu[2] * s_inv;
  circle.q = ((H[3] - H[0]) * (circle.par[1] - H[1]) - (H[4] - H[1]) * (circle.par[0] - H[0]) > 0) ? -1 : 1;
  circle.chi2 = float(fabs(chi2) * renorm * 1. / sqr(2 * v[2] * pu[2] * s));
  // ---- error propagation (:540-756)
  constexpr int n2 = 2 * N;
  double cmV;  // mc^T V mc
  {
    double rv[2 * N];
#pragma unroll
    for (int j = 0; j < n2; ++j) {
      double t = mc[0] * V(0, j);
#pragma unroll
      for (int i = 1; i < n2; ++i) t += mc[i] * V(i, j);
      rv[j] = t;
    }
    cmV = rv[0] * mc[0];
#pragma unroll
    for (int j = 1; j < n2; ++j) cmV += rv[j] * mc[j];
  }
  double vsq = 0.;
#pragma unroll
  for (int k = 0; k < n2 * n2; ++k) vsq += V.a[k] * V.a[k];
  const double K = sqr(sqr(s)) * 1. / (4. * q * n) * (2. * vsq + 4. * cmV);
  // covariances of the centred, scaled points: C[a][b], a <= b
  M<N, N> Cm[6];  // 00, 01, 02, 11, 12, 22
  M<N, N> V10;
#pragma unroll
  for (int i = 0; i < n; ++i)
#pragma unroll
    for (int j = 0; j < n; ++j) {
      const int lo = i <= j ? i : j, hi = i <= j ? j : i;
      Cm[0](i, j) = sqr(s) * V(lo, hi) + K * (mc[lo] * mc[hi]);
      Cm[1](i, j) = sqr(s) * V(i, j + n) + K * (mc[i] * mc[j + n]);
      Cm[3](i, j) = sqr(s) * V(lo + n, hi + n) + K * (mc[lo + n] * mc[hi + n]);
    }
#pragma unroll
  for (int i = 0; i < n; ++i)
#pragma unroll
    for (int j = 0; j < n; ++j) V10(i, j) = Cm[1](j, i);
#pragma unroll
  for (int i = 0; i < n; ++i)
#pragma unroll
    for (int j = 0; j < n; ++j) {
      const double t0 = p3(0, j), t1 = p3(1, j);
      Cm[2](i, j) = 2. * (Cm[0](i, j) * t0 + Cm[1](i, j) * t1);
      Cm[4](i, j) = 2. * (V10(i, j) * t0 + Cm[3](i, j) * t1);
    }
#pragma unroll
  for (int i = 0; i < n; ++i)
#pragma unroll
    for (int j = i; j < n; ++j) {
      const double t00 = p3(0, i) * p3(0, j), t01 = p3(0, i) * p3(1, j), t11 = p3(1, i) * p3(1, j);
      const double t10 = p3(0, j) * p3(1, i);
      const double a00 = Cm[0](i, j), a01 = Cm[1](i, j), a10 = V10(i, j), a11 = Cm[3](i, j);
      const double x = 2. * (a00 * a00 + a00 * a01 + a11 * a10 + a11 * a11) +
                       4. * (a00 * t00 + a01 * t01 + a10 * t10 + a11 * t11);
      Cm[5](i, j) = x;
      Cm[5](j, i) = x;
    }
  constexpr int nu[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
  // index of the pair (a, b), a <= b, in Cm / D
  auto pairIdx = [](int a, int b) { return a == 0 ? b : (a == 1 ? 2 + b : 5); };
  M<3, 3> C0;
#pragma unroll
  for (int p = 0; p < 6; ++p) {
    const M<N, N>& Cab = Cm[p];
    double rw[N];
#pragma unroll
    for (int j = 0; j < n; ++j) {
      double t = w[0] * Cab(0, j);
#pragma unroll
      for (int i = 1; i < n; ++i) t += w[i] * Cab(i, j);
      rw[j] = t;
    }
    double t = rw[0] * w[0];
#pragma unroll
    for (int j = 1; j < n; ++j) t += rw[j] * w[j];
    C0(nu[p][0], nu[p][1]) = t;
    C0(nu[p][1], nu[p][0]) = t;
  }
  M<N, N> Hm;
#pragma unroll
  for (int i = 0; i < n; ++i)
#pragma unroll
    for (int j = 0; j < n; ++j) Hm(i, j) = (i == j ? 1. : 0.) - w[j];
  const M<N, 3> sv = mul(Hm, tr(p3));
  M<N, N> D[6];  // cov(s_v) blocks, a <= b; the others are their transposes
#pragma unroll
  for (int p = 0; p < 6; ++p) {
    const M<N, N> t = mul(mul(Hm, Cm[p]), tr(Hm));
#pragma unroll
    for (int i = 0; i < n; ++i)
#pragma unroll
      for (int j = 0; j < n; ++j) D[p](i, j) = t(i, j) * (w[i] * w[j]);
  }
  auto Dat = [&](int a, int b, int r, int m) {
    return a <= b ? D[pairIdx(a, b)](r, m) : D[pairIdx(b, a)](m, r);
  };
  auto mv = [&](int a, int b, int col, bool twice, double* out) {
#pragma unroll
    for (int r = 0; r < n; ++r) {
      double t = (twice ? 2. * Dat(a, b, r, 0) : Dat(a, b, r, 0)) * sv(0, col);
#pragma unroll
      for (int m = 1; m < n; ++m) t += (twice ? 2. * Dat(a, b, r, m) : Dat(a, b, r, m)) * sv(m, col);
      out[r] = t;
    }
  };
  auto dotc = [&](int col, const double* x) {
    double t = sv(0, col) * x[0];
#pragma unroll
    for (int r = 1; r < n; ++r) t += sv(r, col) * x[r];
    return t;
  };
  M<6, 6> E;
#pragma unroll 1
  for (int a = 0; a < 6; ++a) {
    const int i = nu[a][0], j = nu[a][1];
#pragma unroll 1
    for (int b = a; b < 6; ++b) {
      const int k = nu[b][0], l = nu[b][1];
      double t0[N], t1[N], u[N], z[N];
      if (l == k) {
        mv(j, l, l, true, t0);
        if (i == j) {
#pragma unroll
          for (int r = 0; r < n; ++r) t1[r] = t0[r];
        } else {
          mv(i, l, l, true, t1);
        }
      } else {
        mv(j, l, k, false, u);
        mv(j, k, l, false, z);
#pragma unroll
        for (int r = 0; r < n; ++r) t0[r] = u[r] + z[r];
        if (i == j) {
#pragma unroll
          for (int r = 0; r < n; ++r) t1[r] = t0[r];
        } else {
          mv(i, l, k, false, u);
          mv(i, k, l, false, z);
#pragma unroll
          for (int r = 0; r < n; ++r) t1[r] = u[r] + z[r];
        }
      }
      double e;
      if (i == j) {
        double tt[N];
#pragma unroll
        for (int r = 0; r < n; ++r) tt[r] = t0[r] + t1[r];
        e = 0. + dotc(i, tt);
      } else {
        e = 0. + (dotc(i, t0) + dotc(j, t1));
      }
      E(a, b) = e;
      E(b, a) = e;
    }
  }
  M<3, 6> J2;  // numerical Jacobian of the smallest eigenvector
#pragma unroll 1
  for (int a = 0; a < 6; ++a) {
    const int i = nu[a][0], j = nu[a][1];
    const double dl = fabs(A(i, j) * kRfDeriv);
    double ad[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int m = 0; m < 3; ++m) ad[r][m] = A(r, m);
    ad[i][j] = A(i, j) + dl;
    if (j != i) ad[j][i] = A(j, i) + dl;
    double vf[3];
    if constexpr (std::is_same<S, float>::value) {
      // the single-precision solve of the reference, natively
      float af[3][3], vs[3], ws;
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int m = 0; m < 3; ++m) af[r][m] = float(ad[r][m]);
      rfMinEigen(af, ws, vs);
#pragma unroll
      for (int k = 0; k < 3; ++k) vf[k] = vs[k];
    } else {
      // the single-precision matrix solved in double precision, rounded
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int m = 0; m < 3; ++m) ad[r][m] = double(float(ad[r][m]));
      double wd;
      rfMinEigen(ad, wd, vf);
#pragma unroll
      for (int k = 0; k < 3; ++k) vf[k] = double(float(vf[k]));
    }
    const int sign = (vf[2] > 0) ? 1 : -1;
#pragma unroll
    for (int k = 0; k < 3; ++k) J2(k, a) = (vf[k] * sign - v[k]) / dl;
  }
  M<4, 4> Cvc;
  {
    const M<3, 3> t0 = mul(mul(J2, E), tr(J2));
    double t1[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      double t = (-t0(r, 0)) * r0[0];
#pragma unroll
      for (int k = 1; k < 3; ++k) t += (-t0(r, k)) * r0[k];
      t1[r] = t;
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
#pragma unroll
      for (int k = 0; k < 3; ++k) Cvc(r, k) = t0(r, k);
      Cvc(r, 3) = t1[r];
      Cvc(3, r) = t1[r];
    }
    auto quad = [](const double* x, const M<3, 3>& m) {
      double rr[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) rr[j] = x[0] * m(0, j) + x[1] * m(1, j) + x[2] * m(2, j);
      return rr[0] * x[0] + rr[1] * x[1] + rr[2] * x[2];
    };
    double cs = 0.;
#pragma unroll
    for (int k = 0; k < 9; ++k) cs += C0.a[k] * t0.a[k];
    Cvc(3, 3) = quad(v, C0) + cs + quad(r0, t0);
  }
  M<3, 4> J3;
  {
    const double t = 1. / h;
    J3(0, 0) = -v2x2_inv, J3(0, 1) = 0, J3(0, 2) = v[0] * sqr(v2x2_inv) * 2., J3(0, 3) = 0;
    J3(1, 0) = 0, J3(1, 1) = -v2x2_inv, J3(1, 2) = v[1] * sqr(v2x2_inv) * 2., J3(1, 3) = 0;
    J3(2, 0) = v[0] * v2x2_inv * t, J3(2, 1) = v[1] * v2x2_inv * t;
    J3(2, 2) = -h * sqr(v2x2_inv) * 2. - (2. * c + v[2]) * v2x2_inv * t, J3(2, 3) = -t;
  }
  double jvj;
  {
    double jq[2 * N], rv[2 * N];
#pragma unroll
    for (int k = 0; k < n2; ++k) jq[k] = mc[k] * s * 1. / n;
#pragma unroll
    for (int j = 0; j < n2; ++j) {
      double t = jq[0] * V(0, j);
#pragma unroll
      for (int i = 1; i < n2; ++i) t += jq[i] * V(i, j);
      rv[j] = t;
    }
    jvj = rv[0] * jq[0];
#pragma unroll
    for (int j = 1; j < n2; ++j) jvj += rv[j] * jq[j];
  }
  const M<3, 3> cu = mul(mul(J3, Cvc), tr(J3));
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) circle.cov(a, b) = cu(a, b) * sqr(s_inv) + (pu[a] * pu[b]) * jvj;
}

// Line_fit (RiemannFit.h:777-929) with Scatter_cov_line (:62-107); S is
// the precision of the rotation, the arc lengths and the scattering model
template <int N, typename S>
__device__ void rfLineFit(const double* H, const float* ge, const RfCircle& circle, const S* ff, double B,
                          RfLine& line) {
  constexpr int n = N;
  S theta = S(-circle.q) * atan(ff[3]);
  theta = theta < S(0) ? theta + S(kRfPi) : theta;
  const double sn = sin(theta), cs = cos(theta);
  M<2, 2> rot;
  rot(0, 0) = sn, rot(0, 1) = cs, rot(1, 0) = -cs, rot(1, 1) = sn;
  const double o0 = circle.par[0], o1 = circle.par[1];
  M<6, 6> Cov = rfZero<6, 6>();
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) Cov(a, b) = circle.cov(a, b);
  double szz[N], sArcD[N];  // cov_sz(1,1) and the arc length per hit
  S sArc[N], zz[N];
#pragma unroll
  for (int i = 0; i < n; ++i) {
    const S so0 = S(o0), so1 = S(o1);
    const S px = S(H[3 * i]) - so0, py = S(H[3 * i + 1]) - so1;
    const S cross = (-so0) * py - (-so1) * px;
    const S dot = (-so0) * px + (-so1) * py;
    S at;
    if constexpr (std::is_same<S, double>::value) {
      at = S(-circle.q) * atan2(cross, dot);
      sArcD[i] = at * circle.par[2];
    } else {
      const double dpx = H[3 * i] - o0, dpy = H[3 * i + 1] - o1;
      const double atd = -circle.q * atan2((-o0) * dpy - (-o1) * dpx, (-o0) * dpx + (-o1) * dpy);
      sArcD[i] = atd * circle.par[2];
      at = S(atd);
    }
    sArc[i] = S(sArcD[i]);
    const S temp0 = S(-circle.q) * S(circle.par[2]) * S(1) / (dot * dot + cross * cross);
    M<2, 6> Jx = rfZero<2, 6>();
    Jx(0, 0) = -temp0 * ((py + so1) * dot - (px - so0) * cross);
    Jx(0, 1) = temp0 * ((px + so0) * dot - (so1 - py) * cross);
    Jx(0, 2) = at;
    Jx(0, 3) = temp0 * (so1 * dot + so0 * cross);
    Jx(0, 4) = temp0 * (-so0 * dot + so1 * cross);
    Jx(1, 5) = 1.;
    const float* g = ge + 6 * i;
    Cov(3, 3) = g[0];
    Cov(4, 4) = g[2];
    Cov(5, 5) = g[5];
    Cov(3, 4) = Cov(4, 3) = g[1];
    Cov(3, 5) = Cov(5, 3) = g[3];
    Cov(4, 5) = Cov(5, 4) = g[4];
    const M<2, 2> t = sandwich(Jx, Cov);
    szz[i] = sandwich(rot, t)(1, 1);
    zz[i] = S(H[3 * i + 2]);
  }
  M<N, N> cms;
  {
    const S p_t = fmin(S(20), ff[2] * S(B));
    const S p_2 = p_t * p_t * (S(1) + S(1) / (ff[3] * ff[3]));
    // 3D path lengths in double precision (they feed log(radiation length))
    double Sv[N], rld[N];
    S rl[N], sig2[N];
#pragma unroll
    for (int i = 0; i < n; ++i) Sv[i] = sqrt(sArcD[i] * sArcD[i] + H[3 * i + 2] * H[3 * i + 2]);
    rfRadLen<N>(Sv, rld);
#pragma unroll
    for (int i = 0; i < n; ++i) rl[i] = S(rld[i]);
#pragma unroll
    for (int i = 0; i < n; ++i) {
      const S g = S(1) + S(0.038) * log(rl[i]);
      sig2[i] = S(.000225) / p_2 * (g * g) * rl[i];
    }
#pragma unroll
    for (int k = 0; k < n; ++k)
#pragma unroll
      for (int l = k; l < n; ++l) {
        double t = k == l ? szz[k] : 0.;
#pragma unroll
        for (int i = 0; i < k; ++i) t += double(S(fabs(Sv[k] - Sv[i]) * fabs(Sv[l] - Sv[i])) * sig2[i]);
        cms(k, l) = t;
        cms(l, k) = t;
      }
  }
  M<2, N> A;
  M<N, 1> zc;
#pragma unroll
  for (int i = 0; i < n; ++i) {
    A(0, i) = 1.;
    if constexpr (std::is_same<S, double>::value) {
      A(1, i) = S(rot(0, 0)) * sArc[i] + S(rot(0, 1)) * zz[i];
      zc(i, 0) = S(rot(1, 0)) * sArc[i] + S(rot(1, 1)) * zz[i];
    } else {
      // the s-z rotation in FP64 from the FP64 arc lengths: rotating with the
      // rounded matrix and back with the exact one would tilt the line
      A(1, i) = rot(0, 0) * sArcD[i] + rot(0, 1) * H[3 * i + 2];
      zc(i, 0) = rot(1, 0) * sArcD[i] + rot(1, 1) * H[3 * i + 2];
    }
  }
  M<N, N> Vyi;
  invert(cms, Vyi);
  M<2, 2> Cp = mul(mul(A, Vyi), tr(A));
  invert(Cp, Cp);
  const M<2, 1> sol = mul(mul(mul(Cp, A), Vyi), zc);
  const double cf = 1. / (sn - sol(1, 0) * cs);
  M<2, 2> J;
  J(0, 0) = 0., J(0, 1) = cf * cf, J(1, 0) = cf, J(1, 1) = sol(0, 0) * cs * cf * cf;
  line.par[0] = cf * (sol(1, 0) * sn + cs);
  line.par[1] = cf * sol(0, 0);
  line.cov = sandwich(J, Cp);
  M<N, 1> res;
#pragma unroll
  for (int i = 0; i < n; ++i) res(i, 0) = zc(i, 0) - (A(0, i) * sol(0, 0) + A(1, i) * sol(1, 0));
  line.chi2 = mul(mul(tr(res), Vyi), res)(0, 0);
}

// fromCircleToPerigee (FitUtils.h:198-214)
__device__ void rfToPerigee(RfCircle& c) {
  const double temp0 = c.par[0] * c.par[0] + c.par[1] * c.par[1];
  const double temp1 = sqrt(temp0);
  const double pak0 = atan2(c.q * c.par[0], -c.q * c.par[1]), pak1 = c.q * (temp1 - c.par[2]), pak2 = c.q / c.par[2];
  const double temp2 = sqr(c.par[0]) * 1. / temp0;
  const double temp3 = 1. / temp1 * c.q;
  M<3, 3> J4 = rfZero<3, 3>();
  J4(0, 0) = -c.par[1] * temp2 * 1. / sqr(c.par[0]);
  J4(0, 1) = temp2 * 1. / c.par[0];
  J4(1, 0) = c.par[0] * temp3;
  J4(1, 1) = c.par[1] * temp3;
  J4(1, 2) = -c.q;
  J4(2, 2) = -c.q / (c.par[2] * c.par[2]);
  c.cov = sandwich(J4, c.cov);
  c.par[0] = pak0, c.par[1] = pak1, c.par[2] = pak2;
}

// one tuple: hits H[3*i+k], ge[6*i+k]; the TrackSoA fields of kernelLineFit.
// S = double: the reference's arithmetic.  S = float: the mixed-precision
// variant (single precision for the multiple-scattering models, the s-z
// projection and the single-precision eigen-solves of the numerical
// Jacobian; double precision kept for the prefit circle, the path lengths
// of the radiation-length model, the Riemann matrix and its smallest
// eigenvector (the circle), the Cholesky inversions with their solves, and
// the covariance propagation).
template <int N, typename S>
__device__ void rfFit(const double* H, const float* ge, double B, FitOut& o) {
  constexpr int n = N;
  // the prefit circle in double precision: in single precision the three
  // points of a stiff track can turn collinear
  double ffd[4];
  rfFastFit<N>(H, ffd);
  S ff[4] = {S(ffd[0]), S(ffd[1]), S(ffd[2]), S(ffd[3])}, rad[N];
#pragma unroll
  for (int i = 0; i < n; ++i) {
    const S x = S(H[3 * i]), y = S(H[3 * i + 1]);
    rad[i] = sqrt(x * x + y * y);
  }
  M<2 * N, 2 * N> V = rfZero<2 * N, 2 * N>();  // loadCovariance2D (FitUtils.h:89-118)
#pragma unroll
  for (int i = 0; i < n; ++i) {
    V(i, i) = ge[6 * i + 0];
    V(i + n, i + n) = ge[6 * i + 2];
    V(i, i + n) = V(i + n, i) = ge[6 * i + 1];
  }
  RfCircle circle;
  rfCircleFit<N, S>(H, V, ff, rad, B, circle);
  RfLine line;
  rfLineFit<N, S>(H, ge, circle, ff, B, line);
  rfToPerigee(circle);
  const float b = 1.f / float(B);
  o.state[0] = float(circle.par[0]);
  o.state[1] = float(circle.par[1]);
  o.state[2] = float(circle.par[2]) * b;
  o.state[3] = float(line.par[0]);
  o.state[4] = float(line.par[1]);
  o.cov[0] = float(circle.cov(0, 0));
  o.cov[1] = float(circle.cov(0, 1));
  o.cov[2] = b * float(circle.cov(0, 2));
  o.cov[4] = o.cov[3] = 0;
  o.cov[5] = float(circle.cov(1, 1));
  o.cov[6] = b * float(circle.cov(1, 2));
  o.cov[8] = o.cov[7] = 0;
  o.cov[9] = b * b * float(circle.cov(2, 2));
  o.cov[11] = o.cov[10] = 0;
  o.cov[12] = float(line.cov(0, 0));
  o.cov[13] = float(line.cov(0, 1));
  o.cov[14] = float(line.cov(1, 1));
  o.pt = float(B / fabs(circle.par[2]));
  o.eta = asinhf(float(line.par[0]));
  o.chi2 = float((circle.chi2 + line.chi2) / (2 * N - 5));
}

// standalone Riemann fit of externally supplied tuples
template <int N, typename S>
__global__ void __launch_bounds__(128) kRiemannFitDirect(uint32_t n, const double* hits, const float* hge, double B,
                                                         float* state, float* cov, float* pt, float* eta,
                                                         float* chi2) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    double H[3 * N];
    float ge[6 * N];
#pragma unroll
    for (int k = 0; k < 3 * N; ++k) H[k] = hits[size_t(t) * 3 * N + k];
#pragma unroll
    for (int k = 0; k < 6 * N; ++k) ge[k] = hge[size_t(t) * 6 * N + k];
    FitOut o;
    rfFit<N, S>(H, ge, B, o);
#pragma unroll
    for (int j = 0; j < 5; ++j) state[size_t(t) * 5 + j] = o.state[j];
#pragma unroll
    for (int j = 0; j < 15; ++j) cov[size_t(t) * 15 + j] = o.cov[j];
    pt[t] = o.pt;
    eta[t] = o.eta;
    chi2[t] = o.chi2;
  }
}
