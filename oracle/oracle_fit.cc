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
#include "oracle_mat.h"

namespace oracle {

namespace {


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
