// Oracle (checker only): closed-form eigen-decomposition of small symmetric
// matrices, the part of the Riemann fit that the reference delegates to its
// un-vendored linear-algebra dependency (Eigen, cms-patatrack/eigen @
// adbb8e379ab50707b44e33303f700868a9ce2f9f:
// SelfAdjointEigenSolver::computeDirect, called from
// plugin-PixelTriplets/RiemannFit.h:303-351).  Written here from the
// mathematics of the published method, not from that library:
//
//  3x3: the matrix is scaled by its largest |coefficient| and shifted by the
//  mean of its diagonal, C = A/s - m I.  Its eigenvalues are the roots of the
//  depressed characteristic cubic, m + 2 p cos(phi + 2 pi k / 3) with
//  p = sqrt(tr(C^2) / 6) and phi = acos(det(C / p) / 2) / 3 (k = 1 smallest,
//  k = 2 middle, k = 0 largest).  The eigenvector of the smallest eigenvalue
//  is the longest pairwise cross product of the rows of (C - w0 I) when that
//  eigenvalue is at least as isolated as the largest one; otherwise the
//  largest eigenvalue's vector u is extracted that way and the smallest one
//  is the lower eigenvector of the 2x2 restriction of C to the plane
//  orthogonal to u (angle from atan2), whose eigenvalues then replace the
//  trigonometric roots of that pair.  The isolated root is accurate to
//  rounding; the two roots of a near-double pair are not (the cubic's
//  sensitivity there is ~sqrt(eps)), hence the restriction.  Eigenvalues are
//  returned ascending.
//
//  2x2: eigenvalues from the mean and the half-difference norm, eigenvectors
//  from the atan2 rotation angle.
//
// Parity of the Riemann fit is unpinned at this boundary: the reference's
// tests print their fit results without expected values, and its eigen-solver
// is not in the reference tree.  What matters downstream is the direction of
// the smallest eigenvector (its sign is fixed by the caller) and the smallest
// eigenvalue, both of which any accurate solver reproduces to rounding.
#pragma once

#include <cmath>

namespace symeig {

template <typename T>
inline void cross3(const T* a, const T* b, T* r) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}

template <typename T>
inline T dot3(const T* a, const T* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// a unit vector orthogonal to the unit vector u
template <typename T>
inline void orthoUnit(const T* u, T* e) {
  int ax = 0;  // the axis least aligned with u
  if (std::abs(u[1]) < std::abs(u[ax])) ax = 1;
  if (std::abs(u[2]) < std::abs(u[ax])) ax = 2;
  T a[3] = {T(0), T(0), T(0)};
  a[ax] = T(1);
  cross3(u, a, e);
  const T inv = T(1) / std::sqrt(dot3(e, e));
  for (int k = 0; k < 3; ++k) e[k] *= inv;
}

// unit vector spanning the null space of the (rank-2) symmetric M: the
// longest cross product of two of its rows; for a lower rank, a unit vector
// orthogonal to its longest row
template <typename T>
inline void nullVector(const T M[3][3], T* v) {
  T x[3][3];
  cross3(M[0], M[1], x[0]);
  cross3(M[0], M[2], x[1]);
  cross3(M[1], M[2], x[2]);
  T n[3] = {dot3(x[0], x[0]), dot3(x[1], x[1]), dot3(x[2], x[2])};
  int b = 0;
  if (n[1] > n[b]) b = 1;
  if (n[2] > n[b]) b = 2;
  if (n[b] > T(0)) {
    const T inv = T(1) / std::sqrt(n[b]);
    for (int k = 0; k < 3; ++k) v[k] = x[b][k] * inv;
    return;
  }
  T r[3] = {dot3(M[0], M[0]), dot3(M[1], M[1]), dot3(M[2], M[2])};
  int br = 0;
  if (r[1] > r[br]) br = 1;
  if (r[2] > r[br]) br = 2;
  if (!(r[br] > T(0))) {
    v[0] = T(1), v[1] = T(0), v[2] = T(0);
    return;
  }
  T u[3];
  const T inv = T(1) / std::sqrt(r[br]);
  for (int k = 0; k < 3; ++k) u[k] = M[br][k] * inv;
  orthoUnit(u, v);
}

// A symmetric (both triangles read); w ascending; V(:,k) = V[i][k] the unit
// eigenvector of w[k].  Only column 0 (the smallest) and the eigenvalues are
// needed by the fit; the other two columns complete an orthonormal basis.
template <typename T>
inline void symEigen3(const T A[3][3], T w[3], T V[3][3]) {
  T s = T(0);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) s = std::abs(A[i][j]) > s ? std::abs(A[i][j]) : s;
  T C[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) V[i][j] = i == j ? T(1) : T(0);
  if (!(s > T(0))) {
    w[0] = w[1] = w[2] = T(0);
    return;
  }
  const T is = T(1) / s;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) C[i][j] = A[i][j] * is;
  const T m = (C[0][0] + C[1][1] + C[2][2]) / T(3);
  for (int i = 0; i < 3; ++i) C[i][i] -= m;
  const T p2 = (C[0][0] * C[0][0] + C[1][1] * C[1][1] + C[2][2] * C[2][2] +
                T(2) * (C[0][1] * C[0][1] + C[0][2] * C[0][2] + C[1][2] * C[1][2])) /
               T(6);
  if (!(p2 > T(0))) {
    w[0] = w[1] = w[2] = m * s;
    return;
  }
  const T p = std::sqrt(p2);
  const T det = C[0][0] * (C[1][1] * C[2][2] - C[1][2] * C[2][1]) - C[0][1] * (C[1][0] * C[2][2] - C[1][2] * C[2][0]) +
                C[0][2] * (C[1][0] * C[2][1] - C[1][1] * C[2][0]);
  T r = det / (T(2) * p2 * p);
  r = r < T(-1) ? T(-1) : (r > T(1) ? T(1) : r);
  const T phi = std::acos(r) / T(3);
  const T third = T(2.0943951023931954923);  // 2 pi / 3
  // eigenvalues of C (scaled, shifted)
  const T c2 = T(2) * p * std::cos(phi);
  T c0 = T(2) * p * std::cos(phi + third);
  T c1 = T(2) * p * std::cos(phi + T(2) * third);
  T M[3][3];
  T v0[3], u2[3];
  if (c1 - c0 >= c2 - c1) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) M[i][j] = C[i][j] - (i == j ? c0 : T(0));
    nullVector(M, v0);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) M[i][j] = C[i][j] - (i == j ? c2 : T(0));
    nullVector(M, u2);
    // make u2 exactly orthogonal to v0
    const T d = dot3(u2, v0);
    for (int k = 0; k < 3; ++k) u2[k] -= d * v0[k];
    const T nn = dot3(u2, u2);
    if (nn > T(0)) {
      const T inv = T(1) / std::sqrt(nn);
      for (int k = 0; k < 3; ++k) u2[k] *= inv;
    } else {
      orthoUnit(v0, u2);
    }
  } else {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) M[i][j] = C[i][j] - (i == j ? c2 : T(0));
    nullVector(M, u2);
    // orthonormal basis (e, f) of the plane orthogonal to u2
    T e[3], f[3];
    orthoUnit(u2, e);
    cross3(u2, e, f);
    T Ce[3], Cf[3];
    for (int i = 0; i < 3; ++i) {
      Ce[i] = C[i][0] * e[0] + C[i][1] * e[1] + C[i][2] * e[2];
      Cf[i] = C[i][0] * f[0] + C[i][1] * f[1] + C[i][2] * f[2];
    }
    const T pee = dot3(e, Ce), pef = dot3(e, Cf), pff = dot3(f, Cf);
    // lower eigenvector of [[pee, pef], [pef, pff]]: angle of the upper one + pi/2
    const T t = T(0.5) * std::atan2(T(2) * pef, pee - pff);
    const T ct = std::cos(t), st = std::sin(t);
    for (int k = 0; k < 3; ++k) v0[k] = -st * e[k] + ct * f[k];
    // the pair's eigenvalues from the restriction: near a double root they
    // are better conditioned than the trigonometric roots
    const T mid = T(0.5) * (pee + pff), half = std::hypot(T(0.5) * (pee - pff), pef);
    c0 = mid - half;
    c1 = mid + half;
  }
  T v1[3];
  cross3(u2, v0, v1);
  for (int k = 0; k < 3; ++k) {
    V[k][0] = v0[k];
    V[k][1] = v1[k];
    V[k][2] = u2[k];
  }
  w[0] = (m + c0) * s;
  w[1] = (m + c1) * s;
  w[2] = (m + c2) * s;
}

// 2x2 symmetric: w ascending, V columns the unit eigenvectors
template <typename T>
inline void symEigen2(const T A[2][2], T w[2], T V[2][2]) {
  const T a = A[0][0], b = A[0][1], c = A[1][1];
  const T mean = T(0.5) * (a + c);
  const T half = std::hypot(T(0.5) * (a - c), b);
  w[0] = mean - half;
  w[1] = mean + half;
  const T t = T(0.5) * std::atan2(T(2) * b, a - c);  // angle of the upper vector
  const T ct = std::cos(t), st = std::sin(t);
  V[0][1] = ct, V[1][1] = st;
  V[0][0] = -st, V[1][0] = ct;
}

// smallest eigenvalue and its unit eigenvector of a symmetric 3x3
template <typename T>
inline void minEigen3(const T A[3][3], T& w0, T* v) {
  T w[3], V[3][3];
  symEigen3(A, w, V);
  w0 = w[0];
  for (int k = 0; k < 3; ++k) v[k] = V[k][0];
}

}  // namespace symeig
