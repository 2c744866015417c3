// Small dense column-major FP64 matrices for the helix fits: products
// accumulated over the inner index in ascending order from the first term,
// and the positive-definite inversions of plugin-PixelTriplets/
// choleskyInversion.h:22-161 (n = 3, 4, 5).  FitOut is one fitted track in
// the TrackSoA layout (TrajectoryStateSoA.h:21-38).
//
// Included inside the anonymous namespace of k_fit.cu.  The file uses only
// __device__ and __forceinline__ from CUDA, so that the fits' arithmetic can
// also be compiled for the host by the tests.
#pragma once

__device__ __forceinline__ double sqr(double a) { return a * a; }

template <int R, int C>
struct M {
  double a[R * C];
  __device__ __forceinline__ double& operator()(int i, int j) { return a[i + j * R]; }
  __device__ __forceinline__ double operator()(int i, int j) const { return a[i + j * R]; }
};

template <int R, int K, int C>
__device__ __forceinline__ M<R, C> mul(const M<R, K>& x, const M<K, C>& y) {
  M<R, C> r;
#pragma unroll
  for (int j = 0; j < C; ++j)
#pragma unroll
    for (int i = 0; i < R; ++i) {
      double s = x(i, 0) * y(0, j);
#pragma unroll
      for (int k = 1; k < K; ++k) s += x(i, k) * y(k, j);
      r(i, j) = s;
    }
  return r;
}
template <int R, int C>
__device__ __forceinline__ M<C, R> tr(const M<R, C>& x) {
  M<C, R> r;
#pragma unroll
  for (int j = 0; j < C; ++j)
#pragma unroll
    for (int i = 0; i < R; ++i) r(j, i) = x(i, j);
  return r;
}
template <int R, int C>
__device__ __forceinline__ M<R, R> sandwich(const M<R, C>& a, const M<C, C>& b) {
  return mul(mul(a, b), tr(a));
}

// positive-definite inverse (choleskyInversion.h:22-161), n = 3, 4, 5
__device__ void invert(const M<3, 3>& s, M<3, 3>& d) {
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

__device__ void invert(const M<4, 4>& s, M<4, 4>& d) {
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

__device__ void invert(const M<5, 5>& s, M<5, 5>& d) {
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
#pragma unroll
  for (int i = 0; i < 5; ++i)
#pragma unroll
    for (int j = i + 1; j < 5; ++j) d(i, j) = d(j, i);
}

struct FitOut {
  float state[5], cov[15], pt, eta, chi2;
};
