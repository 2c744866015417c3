// Oracle (checker only): broken-line helix fit of one tuple, restating
// plugin-PixelTriplets/BrokenLine.h (BL_Fast_fit :215-237,
// prepareBrokenLineData :119-162, MatrixC_u :173-203, BL_Circle_fit :256-382,
// BL_Line_fit :401-490, MultScatt :46-59, RotationMatrix :68-75,
// TranslateKarimaki :85-108), the Cholesky inversion of
// plugin-PixelTriplets/choleskyInversion.h:22-161 and the result packing of
// BrokenLineFitOnGPU.h:152-159 / TrajectoryStateSoA.h:30-47.
//
// Matrix products are accumulated over the inner index in ascending order,
// starting from the first term; that is the evaluation order of the
// linear-algebra layer the serial build is compiled with here.
#include <cmath>
#include <cstring>

#include "oracle.h"

namespace oracle {

namespace {

inline double sqr(double a) { return a * a; }

// column-major small dense matrix
template <int R, int C>
struct M {
  double a[R * C];
  double& operator()(int i, int j) { return a[i + j * R]; }
  double operator()(int i, int j) const { return a[i + j * R]; }
  static M zero() {
    M m;
    for (int k = 0; k < R * C; ++k) m.a[k] = 0;
    return m;
  }
};

template <int R, int K, int C>
M<R, C> mul(const M<R, K>& x, const M<K, C>& y) {
  M<R, C> r;
  for (int j = 0; j < C; ++j)
    for (int i = 0; i < R; ++i) {
      double s = x(i, 0) * y(0, j);
      for (int k = 1; k < K; ++k) s += x(i, k) * y(k, j);
      r(i, j) = s;
    }
  return r;
}
template <int R, int C>
M<C, R> tr(const M<R, C>& x) {
  M<C, R> r;
  for (int j = 0; j < C; ++j)
    for (int i = 0; i < R; ++i) r(j, i) = x(i, j);
  return r;
}
// (A * B * A^T) evaluated left to right
template <int R, int C>
M<R, R> sandwich(const M<R, C>& a, const M<C, C>& b) {
  return mul(mul(a, b), tr(a));
}

// ---- choleskyInversion.h:22-161 (positive-definite inverse, n = 3, 4, 5) ------
void invert33(const M<3, 3>& s, M<3, 3>& d) {
  double luc0 = 1.0 / s(0, 0);
  double luc1 = s(1, 0);
  double luc2 = s(1, 1) - luc0 * luc1 * luc1;
  luc2 = 1.0 / luc2;
  double luc3 = s(2, 0);
  double luc4 = (s(2, 1) - luc0 * luc1 * luc3);
  double luc5 = s(2, 2) - (luc0 * luc3 * luc3 + (luc2 * luc4) * luc4);
  luc5 = 1.0 / luc5;
  double li21 = -luc0 * luc1;
  double li32 = -(luc2 * luc4);
  double li31 = (luc1 * (luc2 * luc4) - luc3) * luc0;
  d(0, 0) = luc5 * li31 * li31 + li21 * li21 * luc2 + luc0;
  d(1, 0) = luc5 * li31 * li32 + li21 * luc2;
  d(1, 1) = luc5 * li32 * li32 + luc2;
  d(2, 0) = luc5 * li31;
  d(2, 1) = luc5 * li32;
  d(2, 2) = luc5;
  d(0, 1) = d(1, 0);
  d(0, 2) = d(2, 0);
  d(1, 2) = d(2, 1);
}

void invert44(const M<4, 4>& s, M<4, 4>& d) {
  double luc0 = 1.0 / s(0, 0);
  double luc1 = s(1, 0);
  double luc2 = s(1, 1) - luc0 * luc1 * luc1;
  luc2 = 1.0 / luc2;
  double luc3 = s(2, 0);
  double luc4 = (s(2, 1) - luc0 * luc1 * luc3);
  double luc5 = s(2, 2) - (luc0 * luc3 * luc3 + luc2 * luc4 * luc4);
  luc5 = 1.0 / luc5;
  double luc6 = s(3, 0);
  double luc7 = (s(3, 1) - luc0 * luc1 * luc6);
  double luc8 = (s(3, 2) - luc0 * luc3 * luc6 - luc2 * luc4 * luc7);
  double luc9 = s(3, 3) - (luc0 * luc6 * luc6 + luc2 * luc7 * luc7 + luc8 * (luc8 * luc5));
  luc9 = 1.0 / luc9;
  double li21 = -luc1 * luc0;
  double li32 = -luc2 * luc4;
  double li31 = (luc1 * (luc2 * luc4) - luc3) * luc0;
  double li43 = -(luc8 * luc5);
  double li42 = (luc4 * luc8 * luc5 - luc7) * luc2;
  double li41 = (-luc1 * (luc2 * luc4) * (luc8 * luc5) + luc1 * (luc2 * luc7) + luc3 * (luc8 * luc5) - luc6) * luc0;
  d(0, 0) = luc9 * li41 * li41 + luc5 * li31 * li31 + luc2 * li21 * li21 + luc0;
  d(1, 0) = luc9 * li41 * li42 + luc5 * li31 * li32 + luc2 * li21;
  d(1, 1) = luc9 * li42 * li42 + luc5 * li32 * li32 + luc2;
  d(2, 0) = luc9 * li41 * li43 + luc5 * li31;
  d(2, 1) = luc9 * li42 * li43 + luc5 * li32;
  d(2, 2) = luc9 * li43 * li43 + luc5;
  d(3, 0) = luc9 * li41;
  d(3, 1) = luc9 * li42;
  d(3, 2) = luc9 * li43;
  d(3, 3) = luc9;
  d(0, 1) = d(1, 0);
  d(0, 2) = d(2, 0);
  d(1, 2) = d(2, 1);
  d(0, 3) = d(3, 0);
  d(1, 3) = d(3, 1);
  d(2, 3) = d(3, 2);
}

void invert55(const M<5, 5>& s, M<5, 5>& d) {
  double luc0 = 1.0 / s(0, 0);
  double luc1 = s(1, 0);
  double luc2 = s(1, 1) - luc0 * luc1 * luc1;
  luc2 = 1.0 / luc2;
  double luc3 = s(2, 0);
  double luc4 = (s(2, 1) - luc0 * luc1 * luc3);
  double luc5 = s(2, 2) - (luc0 * luc3 * luc3 + luc2 * luc4 * luc4);
  luc5 = 1.0 / luc5;
  double luc6 = s(3, 0);
  double luc7 = (s(3, 1) - luc0 * luc1 * luc6);
  double luc8 = (s(3, 2) - luc0 * luc3 * luc6 - luc2 * luc4 * luc7);
  double luc9 = s(3, 3) - (luc0 * luc6 * luc6 + luc2 * luc7 * luc7 + luc8 * (luc8 * luc5));
  luc9 = 1.0 / luc9;
  double luc10 = s(4, 0);
  double luc11 = (s(4, 1) - luc0 * luc1 * luc10);
  double luc12 = (s(4, 2) - luc0 * luc3 * luc10 - luc2 * luc4 * luc11);
  double luc13 = (s(4, 3) - luc0 * luc6 * luc10 - luc2 * luc7 * luc11 - luc5 * luc8 * luc12);
  double luc14 = s(4, 4) - (luc0 * luc10 * luc10 + luc2 * luc11 * luc11 + luc5 * luc12 * luc12 + luc9 * luc13 * luc13);
  luc14 = 1.0 / luc14;
  double li21 = -luc1 * luc0;
  double li32 = -luc2 * luc4;
  double li31 = (luc1 * (luc2 * luc4) - luc3) * luc0;
  double li43 = -(luc8 * luc5);
  double li42 = (luc4 * luc8 * luc5 - luc7) * luc2;
  double li41 = (-luc1 * (luc2 * luc4) * (luc8 * luc5) + luc1 * (luc2 * luc7) + luc3 * (luc8 * luc5) - luc6) * luc0;
  double li54 = -luc13 * luc9;
  double li53 = (luc13 * luc8 * luc9 - luc12) * luc5;
  double li52 = (-luc4 * luc8 * luc13 * luc5 * luc9 + luc4 * luc12 * luc5 + luc7 * luc13 * luc9 - luc11) * luc2;
  double li51 = (luc1 * luc4 * luc8 * luc13 * luc2 * luc5 * luc9 - luc13 * luc8 * luc3 * luc9 * luc5 -
                 luc12 * luc4 * luc1 * luc2 * luc5 - luc13 * luc7 * luc1 * luc9 * luc2 + luc11 * luc1 * luc2 +
                 luc12 * luc3 * luc5 + luc13 * luc6 * luc9 - luc10) *
                luc0;
  d(0, 0) = luc14 * li51 * li51 + luc9 * li41 * li41 + luc5 * li31 * li31 + luc2 * li21 * li21 + luc0;
  d(1, 0) = luc14 * li51 * li52 + luc9 * li41 * li42 + luc5 * li31 * li32 + luc2 * li21;
  d(1, 1) = luc14 * li52 * li52 + luc9 * li42 * li42 + luc5 * li32 * li32 + luc2;
  d(2, 0) = luc14 * li51 * li53 + luc9 * li41 * li43 + luc5 * li31;
  d(2, 1) = luc14 * li52 * li53 + luc9 * li42 * li43 + luc5 * li32;
  d(2, 2) = luc14 * li53 * li53 + luc9 * li43 * li43 + luc5;
  d(3, 0) = luc14 * li51 * li54 + luc9 * li41;
  d(3, 1) = luc14 * li52 * li54 + luc9 * li42;
  d(3, 2) = luc14 * li53 * li54 + luc9 * li43;
  d(3, 3) = luc14 * li54 * li54 + luc9;
  d(4, 0) = luc14 * li51;
  d(4, 1) = luc14 * li52;
  d(4, 2) = luc14 * li53;
  d(4, 3) = luc14 * li54;
  d(4, 4) = luc14;
  for (int i = 0; i < 5; ++i)
    for (int j = i + 1; j < 5; ++j) d(i, j) = d(j, i);
}

template <int N>
void invert(const M<N, N>& s, M<N, N>& d);
template <>
void invert<3>(const M<3, 3>& s, M<3, 3>& d) { invert33(s, d); }
template <>
void invert<4>(const M<4, 4>& s, M<4, 4>& d) { invert44(s, d); }
template <>
void invert<5>(const M<5, 5>& s, M<5, 5>& d) { invert55(s, d); }

// BrokenLine.h:46-59
double multScatt(double length, double B, double R, int /*layer*/, double slope) {
  double pt2 = std::min(20., B * R);
  pt2 *= pt2;
  constexpr double XXI_0 = 0.06 / 16.;
  constexpr double geometry_factor = 0.7;
  constexpr double fact = geometry_factor * ((13.6 / 1000.) * (13.6 / 1000.));
  return fact / (pt2 * (1. + sqr(slope))) * (std::abs(length) * XXI_0) * sqr(1. + 0.038 * std::log(std::abs(length) * XXI_0));
}

// BrokenLine.h:68-75
M<2, 2> rotationMatrix(double slope) {
  M<2, 2> r;
  r(0, 0) = 1. / std::sqrt(1. + sqr(slope));
  r(0, 1) = slope * r(0, 0);
  r(1, 0) = -r(0, 1);
  r(1, 1) = r(0, 0);
  return r;
}

inline double cross2D(double ax, double ay, double bx, double by) { return ax * by - ay * bx; }

struct CircleFit {
  double par[3];
  M<3, 3> cov;
  int q;
  float chi2;
};
struct LineFit {
  double par[2];
  M<2, 2> cov;
  double chi2;
};

// BrokenLine.h:85-108
void translateKarimaki(CircleFit& c, double x0, double y0, M<3, 3>& J) {
  double DP = x0 * std::cos(c.par[0]) + y0 * std::sin(c.par[0]);
  double DO = x0 * std::sin(c.par[0]) - y0 * std::cos(c.par[0]) + c.par[1];
  double uu = 1 + c.par[2] * c.par[1];
  double C = -c.par[2] * y0 + uu * std::cos(c.par[0]);
  double BB = c.par[2] * x0 + uu * std::sin(c.par[0]);
  double A = 2. * DO + c.par[2] * (sqr(DO) + sqr(DP));
  double U = std::sqrt(1. + c.par[2] * A);
  double xi = 1. / (sqr(BB) + sqr(C));
  double v = 1. + c.par[2] * DO;
  double lambda = (0.5 * A) / (U * sqr(1. + U));
  double mu = 1. / (U * (1. + U)) + c.par[2] * lambda;
  double zeta = sqr(DO) + sqr(DP);
  J(0, 0) = xi * uu * v;
  J(0, 1) = -xi * sqr(c.par[2]) * DP;
  J(0, 2) = xi * DP;
  J(1, 0) = 2. * mu * uu * DP;
  J(1, 1) = 2. * mu * v;
  J(1, 2) = mu * zeta - lambda * A;
  J(2, 0) = 0;
  J(2, 1) = 0;
  J(2, 2) = 1.;
  c.par[0] = std::atan2(BB, C);
  c.par[1] = A / (1 + U);
  c.cov = sandwich(J, c.cov);
}

// BrokenLine.h:173-203
template <int N>
M<N, N> matrixCu(const double* w, const double* S, const double* VarBeta) {
  constexpr int n = N;
  M<N, N> C = M<N, N>::zero();
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
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) R(i, j) = C(i, j) + C(j, i);
  return R;
}

template <int N>
void fitN(const double* hitsIn, const float* ge, double B, float* state, float* cov15, float* ptOut, float* etaOut,
          float* chi2Out) {
  constexpr int n = N;
  auto H = [&](int r, int c) { return hitsIn[3 * c + r]; };
  // ---- BL_Fast_fit
  double ff[4];
  {
    double ax = H(0, n / 2) - H(0, 0), ay = H(1, n / 2) - H(1, 0);
    double bx = H(0, n - 1) - H(0, n / 2), by = H(1, n - 1) - H(1, n / 2);
    double cx = H(0, 0) - H(0, n - 1), cy = H(1, 0) - H(1, n - 1);
    double tmp = 0.5 / cross2D(cx, cy, ax, ay);
    double csq = cx * cx + cy * cy, asq = ax * ax + ay * ay, bsq = bx * bx + by * by;
    ff[0] = H(0, 0) - (ay * csq + cy * asq) * tmp;
    ff[1] = H(1, 0) + (ax * csq + cx * asq) * tmp;
    ff[2] = std::sqrt(asq * bsq * csq) / (2. * std::abs(cross2D(bx, by, ax, ay)));
    double dx = H(0, 0) - ff[0], dy = H(1, 0) - ff[1];
    double ex = H(0, n - 1) - ff[0], ey = H(1, n - 1) - ff[1];
    ff[3] = ff[2] * std::atan2(cross2D(dx, dy, ex, ey), dx * ex + dy * ey) / (H(2, n - 1) - H(2, 0));
  }
  // ---- prepareBrokenLineData
  int q;
  double radii[2][N], s[N], S[N], Z[N], VarBeta[N];
  {
    double dx = H(0, 1) - H(0, 0), dy = H(1, 1) - H(1, 0);
    double ex = H(0, n - 1) - H(0, n - 2), ey = H(1, n - 1) - H(1, n - 2);
    q = cross2D(dx, dy, ex, ey) > 0 ? -1 : 1;
    const double slope = -q / ff[3];
    M<2, 2> R = rotationMatrix(slope);
    for (int i = 0; i < n; ++i) {
      radii[0][i] = H(0, i) - ff[0] * 1.0;
      radii[1][i] = H(1, i) - ff[1] * 1.0;
    }
    double nrm = std::sqrt(ff[0] * ff[0] + ff[1] * ff[1]);
    double e0 = (-ff[2] * ff[0]) / nrm, e1 = (-ff[2] * ff[1]) / nrm;
    for (int i = 0; i < n; ++i)
      s[i] = q * ff[2] * std::atan2(cross2D(radii[0][i], radii[1][i], e0, e1), radii[0][i] * e0 + radii[1][i] * e1);
    for (int i = 0; i < n; ++i) {
      double p0 = s[i], p1 = H(2, i);
      S[i] = R(0, 0) * p0 + R(0, 1) * p1;
      Z[i] = R(1, 0) * p0 + R(1, 1) * p1;
    }
    VarBeta[0] = VarBeta[n - 1] = 0;
    for (int i = 1; i < n - 1; ++i)
      VarBeta[i] = multScatt(S[i + 1] - S[i], B, ff[2], i + 2, slope) + multScatt(S[i] - S[i - 1], B, ff[2], i + 1, slope);
  }
  // ---- BL_Line_fit (uses VarBeta before the circle fit rescales it)
  LineFit line;
  {
    const double slope = -q / ff[3];
    M<2, 2> R = rotationMatrix(slope);
    M<3, 3> V = M<3, 3>::zero();
    M<2, 3> J = M<2, 3>::zero();
    double w[N];
    for (int i = 0; i < n; ++i) {
      const float* g = ge + 6 * i;
      V(0, 0) = g[0];
      V(0, 1) = V(1, 0) = g[1];
      V(0, 2) = V(2, 0) = g[3];
      V(1, 1) = g[2];
      V(2, 1) = V(1, 2) = g[4];
      V(2, 2) = g[5];
      double tmp = 1. / std::sqrt(radii[0][i] * radii[0][i] + radii[1][i] * radii[1][i]);
      J(0, 0) = radii[1][i] * tmp;
      J(0, 1) = -radii[0][i] * tmp;
      J(1, 2) = 1.;
      M<2, 2> P = mul(mul(mul(mul(R, J), V), tr(J)), tr(R));
      w[i] = 1. / P(1, 1);
    }
    double r_u[N];
    for (int i = 0; i < n; ++i) r_u[i] = w[i] * Z[i];
    M<N, N> I;
    invert<N>(matrixCu<N>(w, S, VarBeta), I);
    double u[N];
    for (int i = 0; i < n; ++i) {
      double acc = I(i, 0) * r_u[0];
      for (int k = 1; k < n; ++k) acc += I(i, k) * r_u[k];
      u[i] = acc;
    }
    line.par[0] = (u[1] - u[0]) / (S[1] - S[0]);
    line.par[1] = u[0];
    double idiff = 1. / (S[1] - S[0]);
    line.cov(0, 0) = (I(0, 0) - 2 * I(0, 1) + I(1, 1)) * sqr(idiff) + multScatt(S[1] - S[0], B, ff[2], 2, slope);
    line.cov(0, 1) = (I(0, 1) - I(0, 0)) * idiff;
    line.cov(1, 0) = (I(0, 1) - I(0, 0)) * idiff;
    line.cov(1, 1) = I(0, 0);
    M<2, 2> jac;
    jac(0, 0) = 1.;
    jac(0, 1) = 0;
    jac(1, 0) = -S[0];
    jac(1, 1) = 1.;
    line.par[1] += -line.par[0] * S[0];
    line.cov = sandwich(jac, line.cov);
    double t = R(0, 0) - line.par[0] * R(0, 1);
    jac(1, 1) = 1. / t;
    jac(0, 0) = jac(1, 1) * jac(1, 1);
    jac(0, 1) = 0;
    jac(1, 0) = line.par[1] * R(0, 1) * jac(0, 0);
    line.par[1] = line.par[1] * jac(1, 1);
    line.par[0] = (R(0, 1) + line.par[0] * R(0, 0)) * jac(1, 1);
    line.cov = sandwich(jac, line.cov);
    line.chi2 = 0;
    for (int i = 0; i < n; ++i) {
      line.chi2 += w[i] * sqr(Z[i] - u[i]);
      if (i > 0 && i < n - 1)
        line.chi2 += sqr(u[i - 1] / (S[i] - S[i - 1]) - u[i] * (S[i + 1] - S[i - 1]) / ((S[i + 1] - S[i]) * (S[i] - S[i - 1])) +
                         u[i + 1] / (S[i + 1] - S[i])) /
                     VarBeta[i];
    }
  }
  // ---- BL_Circle_fit
  CircleFit circle;
  {
    circle.q = q;
    const double slope = -q / ff[3];
    for (int i = 0; i < n; ++i) VarBeta[i] *= 1. + sqr(slope);
    for (int i = 0; i < n; ++i) Z[i] = std::sqrt(radii[0][i] * radii[0][i] + radii[1][i] * radii[1][i]) - ff[2];
    double w[N];
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
    for (int i = 0; i < n; ++i) r_u[i] = w[i] * Z[i];
    M<N + 1, N + 1> C;
    {
      M<N, N> cu = matrixCu<N>(w, s, VarBeta);
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) C(i, j) = cu(i, j);
    }
    C(n, n) = 0;
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
    invert<N + 1>(C, I);
    double u[N + 1];
    for (int i = 0; i < n + 1; ++i) {
      double acc = I(i, 0) * r_u[0];
      for (int k = 1; k < n + 1; ++k) acc += I(i, k) * r_u[k];
      u[i] = acc;
    }
    for (int c = 0; c < 2; ++c) {
      double nr = std::sqrt(radii[0][c] * radii[0][c] + radii[1][c] * radii[1][c]);
      radii[0][c] /= nr;
      radii[1][c] /= nr;
    }
    double dx = H(0, 0) + (-Z[0] + u[0]) * radii[0][0], dy = H(1, 0) + (-Z[0] + u[0]) * radii[1][0];
    double ex = H(0, 1) + (-Z[1] + u[1]) * radii[0][1], ey = H(1, 1) + (-Z[1] + u[1]) * radii[1][1];
    double emdx = ex - dx, emdy = ey - dy;
    circle.par[0] = std::atan2(emdy, emdx);
    circle.par[1] = -circle.q * (ff[2] - std::sqrt(sqr(ff[2]) - 0.25 * (emdx * emdx + emdy * emdy)));
    circle.par[2] = circle.q * (1. / ff[2] + u[n]);
    double tmp1 = emdx * emdx + emdy * emdy;
    M<3, 3> J;
    J(0, 0) = (radii[1][0] * emdx - emdy * radii[0][0]) / tmp1;
    J(0, 1) = (radii[1][1] * emdx - emdy * radii[0][1]) / tmp1;
    J(0, 2) = 0;
    J(1, 0) = (circle.q / 2) * (emdx * radii[0][0] + emdy * radii[1][0]) / std::sqrt(sqr(2 * ff[2]) - tmp1);
    J(1, 1) = (circle.q / 2) * (emdx * radii[0][1] + emdy * radii[1][1]) / std::sqrt(sqr(2 * ff[2]) - tmp1);
    J(1, 2) = 0;
    J(2, 0) = 0;
    J(2, 1) = 0;
    J(2, 2) = circle.q;
    circle.cov(0, 0) = I(0, 0);
    circle.cov(0, 1) = I(0, 1);
    circle.cov(0, 2) = I(0, n);
    circle.cov(1, 0) = I(1, 0);
    circle.cov(1, 1) = I(1, 1);
    circle.cov(1, 2) = I(1, n);
    circle.cov(2, 0) = I(n, 0);
    circle.cov(2, 1) = I(n, 1);
    circle.cov(2, 2) = I(n, n);
    circle.cov = sandwich(J, circle.cov);
    translateKarimaki(circle, 0.5 * emdx, 0.5 * emdy, J);
    circle.cov(0, 0) += (1 + sqr(slope)) * multScatt(S[1] - S[0], B, ff[2], 2, slope);
    translateKarimaki(circle, dx, dy, J);
    circle.chi2 = 0;
    for (int i = 0; i < n; ++i) {
      circle.chi2 += w[i] * sqr(Z[i] - u[i]);
      if (i > 0 && i < n - 1)
        circle.chi2 += sqr(u[i - 1] / (s[i] - s[i - 1]) - u[i] * (s[i + 1] - s[i - 1]) / ((s[i + 1] - s[i]) * (s[i] - s[i - 1])) +
                           u[i + 1] / (s[i + 1] - s[i]) + (s[i + 1] - s[i - 1]) * u[n] / 2) /
                       VarBeta[i];
    }
  }
  // ---- kernelBLFit result packing (BrokenLineFitOnGPU.h:156-159, TrajectoryStateSoA.h:30-47)
  float b = 1.f / float(B);
  state[0] = float(circle.par[0]);
  state[1] = float(circle.par[1]);
  state[2] = float(circle.par[2]);
  state[3] = float(line.par[0]);
  state[4] = float(line.par[1]);
  state[2] *= b;
  cov15[0] = float(circle.cov(0, 0));
  cov15[1] = float(circle.cov(0, 1));
  cov15[2] = b * float(circle.cov(0, 2));
  cov15[4] = cov15[3] = 0;
  cov15[5] = float(circle.cov(1, 1));
  cov15[6] = b * float(circle.cov(1, 2));
  cov15[8] = cov15[7] = 0;
  cov15[9] = b * b * float(circle.cov(2, 2));
  cov15[11] = cov15[10] = 0;
  cov15[12] = float(line.cov(0, 0));
  cov15[13] = float(line.cov(0, 1));
  cov15[14] = float(line.cov(1, 1));
  *ptOut = float(B) / float(std::abs(circle.par[2]));
  *etaOut = asinhf(float(line.par[0]));
  *chi2Out = float((circle.chi2 + line.chi2) / (2 * N - 5));
}

}  // namespace

void brokenLineFit(int N, const double* hits, const float* hits_ge, double B, float* state5, float* cov15, float* pt,
                   float* eta, float* chi2) {
  if (N == 3)
    fitN<3>(hits, hits_ge, B, state5, cov15, pt, eta, chi2);
  else
    fitN<4>(hits, hits_ge, B, state5, cov15, pt, eta, chi2);
}

}  // namespace oracle
