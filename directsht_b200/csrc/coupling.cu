// Mode-coupling matrix of pseudo-Cl on the device: MaskDeconvolution.get_M
// (sht/mask_deconvolution.py:171-192),
//   M[l1][l2] = (2 l2 + 1)/(4 pi) sum_{l3 = |l1-l2|..l1+l2, l1+l2+l3 even} (2 l3 + 1) W[l3] w(l1,l2,l3)^2
// with w the Wigner 3j symbol (l1 l2 l3; 0 0 0) (sht/threej000.py:9-41).
//
// One thread per (l1, l2) walks l3 upwards in steps of 2 with the square of the closed form
//   w^2 = (J-2l1)! (J-2l2)! (J-2l3)! / (J+1)! x [g! / ((g-l1)! (g-l2)! (g-l3)!)]^2,  J = 2g,
// whose ratio between l3 + 2 and l3 is a rational function of (J, g, l1, l2, l3) (five
// products and one division per step); the first value, at l3 = |l1 - l2|, is
//   (2a-2b)! (2b)! / (2a+1)! x C(a, b)^2   (a = max(l1, l2), b = min)
// from lgamma.  The reference instead fills a table of every 3j with l <= 2 Nl - 2 by a
// recursion in (j2, j3); the values agree to rounding (about 1e-13 relative at Nl = 1024).
// FP64 pipe bound: about Nl^3 / 3 steps in all.
#include "dsht_internal.cuh"

namespace dsht {
namespace {

__global__ void mode_coupling_kernel(int Nl, const double* __restrict__ W, int nW, double* __restrict__ M) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (int64_t)Nl * Nl) return;
  const int l1 = (int)(t / Nl), l2 = (int)(t % Nl);
  const int a = max(l1, l2), b = min(l1, l2);
  // l3 = a - b: J = 2a, g = a
  double w2 = exp(lgamma(2.0 * (a - b) + 1.0) + lgamma(2.0 * b + 1.0) - lgamma(2.0 * a + 2.0) +
                  2.0 * (lgamma(a + 1.0) - lgamma(a - b + 1.0) - lgamma(b + 1.0)));
  double s = 0.0;
  for (int l3 = a - b; l3 <= a + b; l3 += 2) {
    if (l3 < nW) s = fma((2.0 * l3 + 1.0) * W[l3], w2, s);
    if (l3 + 2 > a + b) break;
    const double J = (double)(l1 + l2 + l3), g = 0.5 * J;
    const double num = (J + 2 - 2 * l1) * (J + 1 - 2 * l1) * (J + 2 - 2 * l2) * (J + 1 - 2 * l2);
    const double den = (J - 2 * l3) * (J - 2 * l3 - 1) * (J + 3) * (J + 2);
    const double f = (g + 1) * (g - l3) / ((g + 1 - l1) * (g + 1 - l2));
    w2 *= num / den * f * f;
  }
  M[t] = s * (2.0 * l2 + 1.0) / (4.0 * M_PI);
}

}  // namespace
}  // namespace dsht

using namespace dsht;

extern "C" int dsht_mode_coupling(int Nl, const double* W, int nW, double* M, void* stream) {
  if (Nl < 1 || Nl > 46340 || nW < 0 || (nW > 0 && !W) || !M)
    return set_error(DSHT_ERR_INVALID, "invalid arguments (Nl=%d, nW=%d)", Nl, nW);
  const int64_t n = (int64_t)Nl * Nl;
  mode_coupling_kernel<<<(unsigned)((n + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(Nl, W, nW, M);
  count_launches(1);
  return launch_error("mode_coupling_kernel");
}
