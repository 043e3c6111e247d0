// Pseudo-spectrum of alm vectors on the device: DirectSHT.alm2cl (sht/sht.py:95-109),
//   cl[l] = (Re(a_l0)^2 + 2 sum_{m=1..l} |a_lm|^2) / (2l + 1),
// for nmaps alm vectors (complex128, Healpy order m(2Nl-1-m)/2 + l) at alm + k*alm_stride
// doubles.  One warp per (map, l): the lanes stride over m and the squares are summed in
// FP64 with a shuffle tree.  The reads of one warp are strided (consecutive m of one l are
// Nl-m rows apart), so the kernel is latency-bound and tiny: 16 B read per (l, m).
#include "dsht_internal.cuh"

namespace dsht {
namespace {

constexpr int kClWarps = 8;

__global__ void __launch_bounds__(32 * kClWarps)
alm2cl_kernel(int Nl, int nmaps, const double* __restrict__ alm, int64_t alm_stride, double* __restrict__ cl) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t task = (int64_t)blockIdx.x * kClWarps + warp;
  if (task >= (int64_t)Nl * nmaps) return;
  const int k = (int)(task / Nl);
  const int l = (int)(task % Nl);
  const double* a = alm + (size_t)k * alm_stride;
  double s = 0.0;
  for (int m = 1 + lane; m <= l; m += 32) {
    const int64_t i = hp_index(l, m, Nl);
    const double re = a[2 * i], im = a[2 * i + 1];
    s = fma(re, re, fma(im, im, s));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) {
    const double r0 = a[2 * hp_index(l, 0, Nl)];
    cl[(size_t)k * Nl + l] = (r0 * r0 + 2.0 * s) / (2.0 * l + 1.0);
  }
}

}  // namespace
}  // namespace dsht

using namespace dsht;

extern "C" int dsht_alm2cl_device(int Nl, int nmaps, const double* alm, int64_t alm_stride, double* cl,
                                  void* stream) {
  if (Nl < 1 || nmaps < 1 || !alm || !cl || (nmaps > 1 && alm_stride < 2 * (int64_t)Nl * (Nl + 1) / 2))
    return set_error(DSHT_ERR_INVALID, "invalid arguments (Nl=%d, nmaps=%d, alm_stride=%lld)", Nl, nmaps,
                     (long long)alm_stride);
  const int64_t tasks = (int64_t)Nl * nmaps;
  const int64_t blocks = (tasks + kClWarps - 1) / kClWarps;
  if (blocks > 0x7fffffffLL) return set_error(DSHT_ERR_INVALID, "too many spectra (%lld)", (long long)tasks);
  alm2cl_kernel<<<(unsigned)blocks, 32 * kClWarps, 0, reinterpret_cast<cudaStream_t>(stream)>>>(Nl, nmaps, alm,
                                                                                                alm_stride, cl);
  count_launches(1);
  return launch_error("alm2cl_kernel");
}
