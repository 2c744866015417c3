// Oracle (checker only): Riemann helix fit of one tuple, restating
// plugin-PixelTriplets/RiemannFit.h (computeRadLenUniformMaterial :31-40,
// Scatter_cov_line :62-107, Scatter_cov_rad :123-157, cov_radtocart
// :168-190, cov_carttorad_prefit :232-254, Weight_circle :268-270, Charge
// :281-286, min_eigen3D :303-315, min_eigen3D_fast :328-334, Fast_fit
// :368-418, Circle_fit :448-758, Line_fit :777-929), FitUtils.h
// (loadCovariance2D :89-118, fromCircleToPerigee :198-214, d :12) and the
// result packing of kernelLineFit (RiemannFitOnGPU.h:156-162,
// TrajectoryStateSoA.h:21-38).
//
// The eigen-decompositions come from sym_eigen.h (the reference takes them
// from its un-vendored linear-algebra dependency).  min_eigen3D_fast rounds
// the matrix to single precision as the reference does; its eigenvector is
// then computed in double precision and rounded to single precision, which
// keeps the reference's single-precision quantisation of the numerical
// Jacobian J2 without depending on single-precision trigonometric functions.
//
// Expressions are evaluated left to right as written in the reference, with
// matrix products accumulated over the inner index in ascending order.
#include <cmath>

#include "oracle.h"
#include "oracle_mat.h"
#include "sym_eigen.h"

namespace oracle {

namespace {

constexpr double kDeriv = 1.e-4;  // FitUtils.h:12, relative step of J2
constexpr double kPi = 3.14159265358979323846;

struct RCircle {  // Rfit::circle_fit (FitResult.h:25-35): chi2 is single precision
  double par[3];
  M<3, 3> cov;
  int q;
  float chi2;
};

struct RLine {
  double par[2];
  M<2, 2> cov;
  double chi2;
};

// computeRadLenUniformMaterial (RiemannFit.h:31-40)
template <int N>
void radLen(const double* len, double* rl) {
  constexpr double XX_0_inv = 0.06 / 16.;
  rl[0] = len[0] * XX_0_inv;
  for (int j = 1; j < N; ++j) rl[j] = std::abs(len[j] - len[j - 1]) * XX_0_inv;
}

// min_eigen3D (RiemannFit.h:303-315)
void minEigen3D(const M<3, 3>& A, double& chi2, double* v) {
  double a[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a[i][j] = A(i, j);
  symeig::minEigen3(a, chi2, v);
}

// min_eigen3D_fast (RiemannFit.h:328-334)
void minEigen3DFast(const M<3, 3>& A, double* v) {
  double a[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a[i][j] = double(float(A(i, j)));
  double w;
  symeig::minEigen3(a, w, v);
  for (int k = 0; k < 3; ++k) v[k] = double(float(v[k]));
}

// Fast_fit (RiemannFit.h:368-418); H column-major 3xN
template <int N>
void fastFit(const double* H, double* ff) {
  constexpr int n = N;
  const double bX = H[3 * (n / 2)] - H[0], bY = H[3 * (n / 2) + 1] - H[1];
  const double cX = H[3 * (n - 1)] - H[0], cY = H[3 * (n - 1) + 1] - H[1];
  const double b2 = bX * bX + bY * bY;
  const double c2 = cX * cX + cY * cY;
  const bool flip = std::abs(bX) < std::abs(bY);
  const double bx = flip ? bY : bX, by = flip ? bX : bY;
  const double cx = flip ? cY : cX, cy = flip ? cX : cY;
  const double div = 2. * (cx * by - bx * cy);
  const double Y0 = (cx * b2 - bx * c2) / div;
  const double X0 = (0.5 * b2 - Y0 * by) / bx;
  ff[0] = H[0] + (flip ? Y0 : X0);
  ff[1] = H[1] + (flip ? X0 : Y0);
  ff[2] = std::sqrt(sqr(X0) + sqr(Y0));
  const double dX = H[0] - ff[0], dY = H[1] - ff[1];
  const double eX = H[3 * (n - 1)] - ff[0], eY = H[3 * (n - 1) + 1] - ff[1];
  const double dr = ff[2] * std::atan2(dX * eY - dY * eX, dX * eX + dY * eY);
  const double dz = H[3 * (n - 1) + 2] - H[2];
  ff[3] = dr / dz;
}

// Scatter_cov_rad (RiemannFit.h:123-157)
template <int N>
M<N, N> scatterCovRad(const double* H, const double* ff, const double* rad, double B) {
  double p_t = std::min(20., ff[2] * B);
  double p_2 = p_t * p_t * (1. + 1. / (ff[3] * ff[3]));
  double theta = std::atan(ff[3]);
  theta = theta < 0. ? theta + kPi : theta;
  double len[N], rl[N], sig2[N];
  const double fac = std::sqrt(1. + 1. / (ff[3] * ff[3]));
  for (int i = 0; i < N; ++i) {
    const double px = H[3 * i] - ff[0], py = H[3 * i + 1] - ff[1];
    const double cross = (-ff[0]) * py - (-ff[1]) * px;
    const double dot = (-ff[0]) * px + (-ff[1]) * py;
    len[i] = std::abs(std::atan2(cross, dot) * ff[2]) * fac;
  }
  radLen<N>(len, rl);
  const double k = 0.000225 / (p_2 * sqr(std::sin(theta)));
  for (int i = 0; i < N; ++i) sig2[i] = sqr(1. + 0.038 * std::log(rl[i])) * rl[i] * k;
  M<N, N> r = M<N, N>::zero();
  for (int a = 0; a < N; ++a)
    for (int b = a; b < N; ++b) {
      double s = 0.;
      for (int i = 0; i < a; ++i) s += (rad[a] - rad[i]) * (rad[b] - rad[i]) * sig2[i];
      r(a, b) = s;
      r(b, a) = s;
    }
  return r;
}

// cov_radtocart (RiemannFit.h:168-190), added onto V
template <int N>
void addRadToCart(const double* H, const M<N, N>& cr, const double* rad, M<2 * N, 2 * N>& V) {
  constexpr int n = N;
  M<2 * N, 2 * N> cc;
  double ri[N];
  for (int i = 0; i < n; ++i) ri[i] = 1. / rad[i];
  for (int i = 0; i < n; ++i)
    for (int j = i; j < n; ++j) {
      const double c = cr(i, j);
      const double xi = H[3 * i], yi = H[3 * i + 1], xj = H[3 * j], yj = H[3 * j + 1];
      cc(i, j) = c * yi * ri[i] * yj * ri[j];
      cc(i + n, j + n) = c * xi * ri[i] * xj * ri[j];
      cc(i, j + n) = -c * yi * ri[i] * xj * ri[j];
      cc(i + n, j) = -c * xi * ri[i] * yj * ri[j];
      cc(j, i) = cc(i, j);
      cc(j + n, i + n) = cc(i + n, j + n);
      cc(j + n, i) = cc(i, j + n);
      cc(j, i + n) = cc(i + n, j);
    }
  for (int k = 0; k < 4 * n * n; ++k) V.a[k] += cc.a[k];
}

// Circle_fit (RiemannFit.h:448-758) with error propagation; V is the 2N x 2N
// covariance of the transverse coordinates (loadCovariance2D ordering)
template <int N>
RCircle circleFit(const double* H, M<2 * N, 2 * N> V, const double* ff, const double* rad, double B) {
  constexpr int n = N;
  // ---- weights (:457-471): cov_carttorad_prefit (:232-254) + scattering
  M<N, N> covRad = M<N, N>::zero();
  for (int i = 0; i < n; ++i) {
    if (rad[i] < 1.e-4) {
      covRad(i, i) = V(i, i);
    } else {
      const double ax = H[3 * i], ay = H[3 * i + 1];
      const double bx = ax - ff[0], by = ay - ff[1];
      const double x2 = ax * bx + ay * by;
      const double y2 = ax * by - ay * bx;
      const double tan_c = -y2 / x2;
      const double tan_c2 = sqr(tan_c);
      covRad(i, i) = 1. / (1. + tan_c2) * (V(i, i) + V(i + n, i + n) * tan_c2 + 2 * V(i, i + n) * tan_c);
    }
  }
  const M<N, N> scat = scatterCovRad<N>(H, ff, rad, B);
  addRadToCart<N>(H, scat, rad, V);
  for (int k = 0; k < n * n; ++k) covRad.a[k] += scat.a[k];
  M<N, N> G;
  invert<N>(covRad, G);
  double renorm = 0.;
  for (int k = 0; k < n * n; ++k) renorm += G.a[k];
  const double rinv = 1. / renorm;
  for (int k = 0; k < n * n; ++k) G.a[k] *= rinv;
  double w[N];  // Weight_circle (:268-270): column sums
  for (int j = 0; j < n; ++j) {
    double s = G(0, j);
    for (int i = 1; i < n; ++i) s += G(i, j);
    w[j] = s;
  }
  // ---- space transformation (:475-493)
  double h0 = 0., h1 = 0.;
  for (int i = 0; i < n; ++i) h0 += H[3 * i], h1 += H[3 * i + 1];
  h0 /= n;
  h1 /= n;
  M<3, N> p3;
  double mc[2 * N];
  for (int i = 0; i < n; ++i) {
    p3(0, i) = H[3 * i] - h0;
    p3(1, i) = H[3 * i + 1] - h1;
    mc[i] = p3(0, i);
    mc[i + n] = p3(1, i);
  }
  double q = 0.;
  for (int k = 0; k < 2 * n; ++k) q += mc[k] * mc[k];
  const double s = std::sqrt(n * 1. / q);
  for (int i = 0; i < n; ++i) {
    p3(0, i) *= s;
    p3(1, i) *= s;
    p3(2, i) = p3(0, i) * p3(0, i) + p3(1, i) * p3(1, i);
  }
  // ---- cost function (:497-519)
  double r0[3];
  for (int k = 0; k < 3; ++k) {
    double t = p3(k, 0) * w[0];
    for (int i = 1; i < n; ++i) t += p3(k, i) * w[i];
    r0[k] = t;
  }
  M<3, N> X;
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) X(k, i) = p3(k, i) - r0[k];
  const M<3, 3> A = mul(mul(X, G), tr(X));
  double chi2, v[3];
  minEigen3D(A, chi2, v);
  if (!(v[2] > 0))
    for (int k = 0; k < 3; ++k) v[k] *= -1;
  const double c = (-v[0]) * r0[0] + (-v[1]) * r0[1] + (-v[2]) * r0[2];
  // ---- circle parameters (:523-537)
  const double h = std::sqrt(1. - sqr(v[2]) - 4. * c * v[2]);
  const double v2x2_inv = 1. / (2. * v[2]);
  const double s_inv = 1. / s;
  const double pu[3] = {-v[0] * v2x2_inv, -v[1] * v2x2_inv, h * v2x2_inv};
  RCircle circle;
  circle.par[0] = pu[0] * s_inv + h0;
  circle.par[1] = pu[1] * s_inv + h1;
  circle.par[2] = pu[2] * s_inv;
  // Charge (:281-286)
  circle.q = ((H[3] - H[0]) * (circle.par[1] - H[1]) - (H[4] - H[1]) * (circle.par[0] - H[0]) > 0) ? -1 : 1;
  circle.chi2 = float(std::abs(chi2) * renorm * 1. / sqr(2 * v[2] * pu[2] * s));
  // ---- error propagation (:540-756)
  constexpr int n2 = 2 * N;
  double cmV;  // mc^T V mc
  {
    double rv[2 * N];
    for (int j = 0; j < n2; ++j) {
      double t = mc[0] * V(0, j);
      for (int i = 1; i < n2; ++i) t += mc[i] * V(i, j);
      rv[j] = t;
    }
    cmV = rv[0] * mc[0];
    for (int j = 1; j < n2; ++j) cmV += rv[j] * mc[j];
  }
  double vsq = 0.;
  for (int k = 0; k < n2 * n2; ++k) vsq += V.a[k] * V.a[k];
  const double K = sqr(sqr(s)) * 1. / (4. * q * n) * (2. * vsq + 4. * cmV);
  // Vcs = s^2 V + K mc mc^T (symmetric as evaluated); blocks V00, V01, V11
  M<N, N> V00, V01, V10, V11, C02, C12, C22;
  auto vcs = [&](int i, int j) { return sqr(s) * V(i, j) + K * (mc[i] * mc[j]); };
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      V00(i, j) = vcs(i <= j ? i : j, i <= j ? j : i);
      V01(i, j) = vcs(i, j + n);
      V11(i, j) = vcs((i <= j ? i : j) + n, (i <= j ? j : i) + n);
    }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) V10(i, j) = V01(j, i);
  // t0(i,j) = x_j, t1(i,j) = y_j, t00 = x_i x_j, t01 = x_i y_j, t11 = y_i y_j, t10 = y_i x_j
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      const double t0 = p3(0, j), t1 = p3(1, j);
      C02(i, j) = 2. * (V00(i, j) * t0 + V01(i, j) * t1);
      C12(i, j) = 2. * (V10(i, j) * t0 + V11(i, j) * t1);
    }
  for (int i = 0; i < n; ++i)
    for (int j = i; j < n; ++j) {
      const double t00 = p3(0, i) * p3(0, j), t01 = p3(0, i) * p3(1, j), t11 = p3(1, i) * p3(1, j);
      const double t10 = p3(0, j) * p3(1, i);
      const double v = 2. * (V00(i, j) * V00(i, j) + V00(i, j) * V01(i, j) + V11(i, j) * V10(i, j) + V11(i, j) * V11(i, j)) +
                       4. * (V00(i, j) * t00 + V01(i, j) * t01 + V10(i, j) * t10 + V11(i, j) * t11);
      C22(i, j) = v;
      C22(j, i) = v;
    }
  const M<N, N>* Cp[3][3] = {{&V00, &V01, &C02}, {nullptr, &V11, &C12}, {nullptr, nullptr, &C22}};
  M<3, 3> C0;  // covariance of the centre of gravity
  for (int a = 0; a < 3; ++a)
    for (int b = a; b < 3; ++b) {
      const M<N, N>& Cab = *Cp[a][b];
      double rw[N];
      for (int j = 0; j < n; ++j) {
        double t = w[0] * Cab(0, j);
        for (int i = 1; i < n; ++i) t += w[i] * Cab(i, j);
        rw[j] = t;
      }
      double t = rw[0] * w[0];
      for (int j = 1; j < n; ++j) t += rw[j] * w[j];
      C0(a, b) = t;
      C0(b, a) = t;
    }
  M<N, N> W, Hm;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      W(i, j) = w[i] * w[j];
      Hm(i, j) = (i == j ? 1. : 0.) - w[j];
    }
  const M<N, 3> sv = mul(Hm, tr(p3));
  M<N, N> D[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = a; b < 3; ++b) {
      const M<N, N> t = mul(mul(Hm, *Cp[a][b]), tr(Hm));
      for (int k = 0; k < n * n; ++k) D[a][b].a[k] = t.a[k] * W.a[k];
    }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < a; ++b) D[a][b] = tr(D[b][a]);
  constexpr int nu[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
  // D * col(sv, c), optionally scaled by 2 first
  auto mv = [&](const M<N, N>& Dm, int col, bool twice, double* out) {
    for (int r = 0; r < n; ++r) {
      double t = (twice ? 2. * Dm(r, 0) : Dm(r, 0)) * sv(0, col);
      for (int m = 1; m < n; ++m) t += (twice ? 2. * Dm(r, m) : Dm(r, m)) * sv(m, col);
      out[r] = t;
    }
  };
  auto dotc = [&](int col, const double* x) {
    double t = sv(0, col) * x[0];
    for (int r = 1; r < n; ++r) t += sv(r, col) * x[r];
    return t;
  };
  M<6, 6> E;
  for (int a = 0; a < 6; ++a) {
    const int i = nu[a][0], j = nu[a][1];
    for (int b = a; b < 6; ++b) {
      const int k = nu[b][0], l = nu[b][1];
      double t0[N], t1[N], u[N], z[N];
      if (l == k) {
        mv(D[j][l], l, true, t0);
        if (i == j)
          for (int r = 0; r < n; ++r) t1[r] = t0[r];
        else
          mv(D[i][l], l, true, t1);
      } else {
        mv(D[j][l], k, false, u);
        mv(D[j][k], l, false, z);
        for (int r = 0; r < n; ++r) t0[r] = u[r] + z[r];
        if (i == j) {
          for (int r = 0; r < n; ++r) t1[r] = t0[r];
        } else {
          mv(D[i][l], k, false, u);
          mv(D[i][k], l, false, z);
          for (int r = 0; r < n; ++r) t1[r] = u[r] + z[r];
        }
      }
      double e;
      if (i == j) {
        double tt[N];
        for (int r = 0; r < n; ++r) tt[r] = t0[r] + t1[r];
        e = 0. + dotc(i, tt);
      } else {
        e = 0. + (dotc(i, t0) + dotc(j, t1));
      }
      E(a, b) = e;
      if (b != a) E(b, a) = e;
    }
  }
  M<3, 6> J2;  // numerical Jacobian of the smallest eigenvector
  for (int a = 0; a < 6; ++a) {
    const int i = nu[a][0], j = nu[a][1];
    M<3, 3> Ad = A;
    const double dl = std::abs(A(i, j) * kDeriv);
    Ad(i, j) = A(i, j) + dl;
    if (j != i) Ad(j, i) = A(j, i) + dl;
    double vf[3];
    minEigen3DFast(Ad, vf);
    const int sign = (vf[2] > 0) ? 1 : -1;
    for (int k = 0; k < 3; ++k) J2(k, a) = (vf[k] * sign - v[k]) / dl;
  }
  M<4, 4> Cvc;
  {
    const M<3, 3> t0 = mul(mul(J2, E), tr(J2));
    double t1[3];
    for (int r = 0; r < 3; ++r) {
      double t = (-t0(r, 0)) * r0[0];
      for (int k = 1; k < 3; ++k) t += (-t0(r, k)) * r0[k];
      t1[r] = t;
    }
    for (int r = 0; r < 3; ++r) {
      for (int k = 0; k < 3; ++k) Cvc(r, k) = t0(r, k);
      Cvc(r, 3) = t1[r];
      Cvc(3, r) = t1[r];
    }
    auto quad = [](const double* x, const M<3, 3>& m) {
      double rr[3];
      for (int j = 0; j < 3; ++j) rr[j] = x[0] * m(0, j) + x[1] * m(1, j) + x[2] * m(2, j);
      return rr[0] * x[0] + rr[1] * x[1] + rr[2] * x[2];
    };
    double cs = 0.;
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
  double jq[2 * N];
  for (int k = 0; k < n2; ++k) jq[k] = mc[k] * s * 1. / n;
  double jvj;
  {
    double rv[2 * N];
    for (int j = 0; j < n2; ++j) {
      double t = jq[0] * V(0, j);
      for (int i = 1; i < n2; ++i) t += jq[i] * V(i, j);
      rv[j] = t;
    }
    jvj = rv[0] * jq[0];
    for (int j = 1; j < n2; ++j) jvj += rv[j] * jq[j];
  }
  const M<3, 3> cu = mul(mul(J3, Cvc), tr(J3));
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) circle.cov(a, b) = cu(a, b) * sqr(s_inv) + (pu[a] * pu[b]) * jvj;
  return circle;
}

// Line_fit (RiemannFit.h:777-929) with Scatter_cov_line (:62-107)
template <int N>
RLine lineFit(const double* H, const float* ge, const RCircle& circle, const double* ff, double B) {
  constexpr int n = N;
  double theta = -circle.q * std::atan(ff[3]);
  theta = theta < 0. ? theta + kPi : theta;
  const double sn = std::sin(theta), cs = std::cos(theta);
  M<2, 2> rot;
  rot(0, 0) = sn, rot(0, 1) = cs, rot(1, 0) = -cs, rot(1, 1) = sn;
  const double o0 = circle.par[0], o1 = circle.par[1];
  M<6, 6> Cov = M<6, 6>::zero();
  M<2, 2> covSz[N];
  double sArc[N], zz[N];
  for (int i = 0; i < n; ++i) {
    const double px = H[3 * i] - o0, py = H[3 * i + 1] - o1;
    const double cross = (-o0) * py - (-o1) * px;
    const double dot = (-o0) * px + (-o1) * py;
    const double at = -circle.q * std::atan2(cross, dot);
    sArc[i] = at * circle.par[2];
    const double temp0 = -circle.q * circle.par[2] * 1. / (sqr(dot) + sqr(cross));
    const double d_X0 = -temp0 * ((py + o1) * dot - (px - o0) * cross);
    const double d_Y0 = temp0 * ((px + o0) * dot - (o1 - py) * cross);
    const double d_R = at;
    const double d_x = temp0 * (o1 * dot + o0 * cross);
    const double d_y = temp0 * (-o0 * dot + o1 * cross);
    M<2, 6> Jx = M<2, 6>::zero();
    Jx(0, 0) = d_X0, Jx(0, 1) = d_Y0, Jx(0, 2) = d_R, Jx(0, 3) = d_x, Jx(0, 4) = d_y;
    Jx(1, 5) = 1.;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) Cov(a, b) = circle.cov(a, b);
    const float* g = ge + 6 * i;
    Cov(3, 3) = g[0];
    Cov(4, 4) = g[2];
    Cov(5, 5) = g[5];
    Cov(3, 4) = Cov(4, 3) = g[1];
    Cov(3, 5) = Cov(5, 3) = g[3];
    Cov(4, 5) = Cov(5, 4) = g[4];
    const M<2, 2> t = sandwich(Jx, Cov);
    covSz[i] = sandwich(rot, t);
    zz[i] = H[3 * i + 2];
  }
  // Scatter_cov_line: errors orthogonal to the rotated s axis
  M<N, N> cms;
  {
    double p_t = std::min(20., ff[2] * B);
    double p_2 = p_t * p_t * (1. + 1. / (ff[3] * ff[3]));
    double S[N], rl[N], sig2[N];
    for (int i = 0; i < n; ++i) S[i] = std::sqrt(sArc[i] * sArc[i] + zz[i] * zz[i]);
    radLen<N>(S, rl);
    for (int i = 0; i < n; ++i) sig2[i] = .000225 / p_2 * sqr(1. + 0.038 * std::log(rl[i])) * rl[i];
    for (int k = 0; k < n; ++k)
      for (int l = k; l < n; ++l) {
        double t = k == l ? covSz[k](1, 1) : 0.;
        for (int i = 0; i < k; ++i) t += std::abs(S[k] - S[i]) * std::abs(S[l] - S[i]) * sig2[i];
        cms(k, l) = t;
        cms(l, k) = t;
      }
  }
  double sr[N], zr[N];  // rotated points
  for (int i = 0; i < n; ++i) {
    sr[i] = rot(0, 0) * sArc[i] + rot(0, 1) * zz[i];
    zr[i] = rot(1, 0) * sArc[i] + rot(1, 1) * zz[i];
  }
  M<2, N> A;
  for (int i = 0; i < n; ++i) A(0, i) = 1., A(1, i) = sr[i];
  M<N, N> Vyi;
  invert<N>(cms, Vyi);
  M<2, 2> Cp = mul(mul(A, Vyi), tr(A));
  invert<2>(Cp, Cp);
  M<N, 1> zc;
  for (int i = 0; i < n; ++i) zc(i, 0) = zr[i];
  const M<2, 1> sol = mul(mul(mul(Cp, A), Vyi), zc);
  const double cf = 1. / (sn - sol(1, 0) * cs);
  M<2, 2> J;
  J(0, 0) = 0., J(0, 1) = cf * cf, J(1, 0) = cf, J(1, 1) = sol(0, 0) * cs * cf * cf;
  RLine line;
  line.par[0] = cf * (sol(1, 0) * sn + cs);
  line.par[1] = cf * sol(0, 0);
  line.cov = sandwich(J, Cp);
  M<N, 1> res;
  for (int i = 0; i < n; ++i) res(i, 0) = zr[i] - (A(0, i) * sol(0, 0) + A(1, i) * sol(1, 0));
  line.chi2 = mul(mul(tr(res), Vyi), res)(0, 0);
  return line;
}

// fromCircleToPerigee (FitUtils.h:198-214)
void toPerigee(RCircle& c) {
  const double temp0 = c.par[0] * c.par[0] + c.par[1] * c.par[1];
  const double temp1 = std::sqrt(temp0);
  const double pak[3] = {std::atan2(c.q * c.par[0], -c.q * c.par[1]), c.q * (temp1 - c.par[2]), c.q / c.par[2]};
  const double temp2 = sqr(c.par[0]) * 1. / temp0;
  const double temp3 = 1. / temp1 * c.q;
  M<3, 3> J4 = M<3, 3>::zero();
  J4(0, 0) = -c.par[1] * temp2 * 1. / sqr(c.par[0]);
  J4(0, 1) = temp2 * 1. / c.par[0];
  J4(1, 0) = c.par[0] * temp3;
  J4(1, 1) = c.par[1] * temp3;
  J4(1, 2) = -c.q;
  J4(2, 2) = -c.q / (c.par[2] * c.par[2]);
  c.cov = sandwich(J4, c.cov);
  for (int k = 0; k < 3; ++k) c.par[k] = pak[k];
}

template <int N>
void fitN(const double* H, const float* ge, double B, float* state, float* cov15, float* ptOut, float* etaOut,
          float* chi2Out) {
  constexpr int n = N;
  double ff[4], rad[N];
  fastFit<N>(H, ff);
  for (int i = 0; i < n; ++i) rad[i] = std::sqrt(H[3 * i] * H[3 * i] + H[3 * i + 1] * H[3 * i + 1]);
  // loadCovariance2D (FitUtils.h:89-118)
  M<2 * N, 2 * N> V = M<2 * N, 2 * N>::zero();
  for (int i = 0; i < n; ++i) {
    V(i, i) = ge[6 * i + 0];
    V(i + n, i + n) = ge[6 * i + 2];
    V(i, i + n) = V(i + n, i) = ge[6 * i + 1];
  }
  RCircle circle = circleFit<N>(H, V, ff, rad, B);
  const RLine line = lineFit<N>(H, ge, circle, ff, B);
  toPerigee(circle);
  // kernelLineFit packing (RiemannFitOnGPU.h:156-162, TrajectoryStateSoA.h:21-38)
  const float b = 1.f / float(B);
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
  *ptOut = float(B / std::abs(circle.par[2]));
  *etaOut = asinhf(float(line.par[0]));
  *chi2Out = float((circle.chi2 + line.chi2) / (2 * N - 5));
}

}  // namespace

void riemannFit(int N, const double* hits, const float* hits_ge, double B, float* state5, float* cov15, float* pt,
                float* eta, float* chi2) {
  if (N == 3)
    fitN<3>(hits, hits_ge, B, state5, cov15, pt, eta, chi2);
  else
    fitN<4>(hits, hits_ge, B, state5, cov15, pt, eta, chi2);
}

}  // namespace oracle
