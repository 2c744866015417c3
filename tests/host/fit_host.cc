// Test infrastructure: the device helix-fit code of the B200 library
// (pixeltrack-standalone_b200/csrc/fit_linalg.cuh, k_fit_riemann.cuh)
// compiled by the host compiler, so that tests without a GPU can compare the
// kernel's arithmetic with the oracle operation by operation.  The device
// and host builds differ only in their transcendental functions.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>

#define __device__
#define __forceinline__ inline
#define __global__
#define __launch_bounds__(x)
using std::acos;
using std::atan;
using std::atan2;
using std::cos;
using std::fabs;
using std::fmin;
using std::hypot;
using std::log;
using std::sin;
using std::sqrt;

namespace {
struct Dim3 {
  unsigned x = 0;
};
Dim3 blockIdx, blockDim, gridDim, threadIdx;  // for the kernel bodies, never run

#include "fit_linalg.cuh"
#include "k_fit_riemann.cuh"

template <int N, typename S>
void fitAll(uint32_t n, const double* hits, const float* ge, double B, float* state, float* cov, float* pt, float* eta,
            float* chi2) {
  for (uint32_t t = 0; t < n; ++t) {
    FitOut o;
    rfFit<N, S>(hits + size_t(t) * 3 * N, ge + size_t(t) * 6 * N, B, o);
    std::memcpy(state + size_t(t) * 5, o.state, sizeof o.state);
    std::memcpy(cov + size_t(t) * 15, o.cov, sizeof o.cov);
    pt[t] = o.pt;
    eta[t] = o.eta;
    chi2[t] = o.chi2;
  }
}
}  // namespace

extern "C" int hf_fit_riemann(int N, int mixed, uint32_t n, const double* hits, const float* ge, double B, float* state,
                              float* cov, float* pt, float* eta, float* chi2) {
  if (N == 3 && !mixed)
    fitAll<3, double>(n, hits, ge, B, state, cov, pt, eta, chi2);
  else if (N == 4 && !mixed)
    fitAll<4, double>(n, hits, ge, B, state, cov, pt, eta, chi2);
  else if (N == 3)
    fitAll<3, float>(n, hits, ge, B, state, cov, pt, eta, chi2);
  else if (N == 4)
    fitAll<4, float>(n, hits, ge, B, state, cov, pt, eta, chi2);
  else
    return -1;
  return 0;
}
