// Rotation of the polar points' alm back to the original frame, added to the equatorial alm.
//
// The polar points were rotated by +90 deg about y (Euler ZYZ (0, 90, 0)); their alm a'
// map back with Wigner d^l(pi/2):  a_lm = sum_{m'=-l..l} d^l_{m'm}(pi/2) a'_lm'.  For a
// real field (a'_{l,-m'} = (-1)^m' conj a'_lm') this is
//   Re a_lm = d_{0m} Re a'_l0 + 2 sum_{m'>0, l+m+m' even} d_{m'm} Re a'_lm'
//   Im a_lm =                   2 sum_{m'>0, l+m+m' odd}  d_{m'm} Im a'_lm'
// This stands in for healpy's Rotator(rot=(0,90,0), eulertype='ZYZ', inv=True).rotate_alm
// called at sht/sht.py:138-139.  d_{k,m}(pi/2) is generated per output m by the downward
// three-term recursion in k of Trapani & Navaza (Acta Cryst. A62, 262, 2006),
//   sqrt((l+k)(l-k+1)) d_{k-1,m} = 2m d_{k,m} - sqrt((l-k)(l+k+1)) d_{k+1,m},
// from d_{l,m} = (-1)^(l-m) 2^-l sqrt(C(2l, l+m)); values below the double range are
// carried with a binary exponent.  One CTA per l; each thread runs two interleaved output
// columns m.  FP64 compute bound: about 5 DFMA per (l, m, m').
#include "dsht_internal.cuh"

namespace dsht {
namespace {

constexpr int kRotThreads = 256;

__global__ void __launch_bounds__(kRotThreads)
rotate_back_kernel(int Nl, const double* __restrict__ alm_rot, const double* __restrict__ alm_add,
                   double* __restrict__ alm_out, const unsigned* __restrict__ flags) {
  extern __shared__ double sm[];
  const int l = Nl - 1 - blockIdx.x;  // largest l first
  const bool has_polar = (flags == nullptr) || ((*flags & kFlagHasPolar) != 0);
  if (!has_polar) {
    for (int m = threadIdx.x; m <= l; m += blockDim.x) {
      const int64_t i = hp_index(l, m, Nl);
      alm_out[2 * i] = alm_add[2 * i];
      alm_out[2 * i + 1] = alm_add[2 * i + 1];
    }
    return;
  }
  double* a_re = sm;                 // [l+1]
  double* a_im = a_re + (l + 1);     // [l+1]
  double* c1 = a_im + (l + 1);       // [l+1] sqrt((l-k)(l+k+1))
  double* c2 = c1 + (l + 1);         // [l+1] 1/sqrt((l+k)(l-k+1))
  double* rat = c2 + (l + 1);        // [l+1] r[k]: d_{l,k-1} = r[k] d_{l,k}
  double* st_m = rat + (l + 1);      // [l+1] start mantissa d_{l,m}
  int* st_e = reinterpret_cast<int*>(st_m + (l + 1));  // [l+1] start exponent
  for (int k = threadIdx.x; k <= l; k += blockDim.x) {
    const int64_t i = hp_index(l, k, Nl);
    a_re[k] = alm_rot[2 * i];
    a_im[k] = alm_rot[2 * i + 1];
    c1[k] = sqrt((double)(l - k) * (double)(l + k + 1));
    c2[k] = (k >= 1) ? 1.0 / sqrt((double)(l + k) * (double)(l - k + 1)) : 0.0;
    rat[k] = (k >= 1) ? -sqrt((double)(l + k) / (double)(l - k + 1)) : 1.0;
  }
  __syncthreads();
  // Start column d_{l,m} = 2^-l P(m), P(m) = prod_{k=m+1..l} r[k] (P(l) = 1).  Warp 0
  // splits m into 32 chunks [lo, hi): T = prod_{k=lo+1..hi} r[k] links P(hi) to P(lo); an
  // exclusive suffix product over lanes gives P(hi), and each lane walks its chunk down.
  // Values are carried as (mantissa, binary exponent) so nothing under- or overflows.
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    auto rr = [&](int k) { return (k >= 1 && k <= l) ? rat[k] : 1.0; };
    const int per = (l + 1 + 31) / 32;
    const int lo = min(lane * per, l + 1), hi = min(lo + per, l + 1);
    double tm = 1.0;
    int te = 0;
    for (int k = lo + 1; k <= hi; ++k) {
      int de;
      tm = frexp(tm * rr(k), &de);
      te += de;
    }
    double pm = tm;  // inclusive suffix product over lanes >= lane
    int pe = te;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double om = __shfl_down_sync(0xffffffffu, pm, o);
      const int oe = __shfl_down_sync(0xffffffffu, pe, o);
      if (lane + o < 32) {
        int de;
        pm = frexp(pm * om, &de);
        pe += oe + de;
      }
    }
    double vm = __shfl_down_sync(0xffffffffu, pm, 1);
    int ve = __shfl_down_sync(0xffffffffu, pe, 1);
    if (lane == 31) {
      vm = 1.0;
      ve = 0;
    }
    for (int m = hi - 1; m >= lo; --m) {
      int de;
      vm = frexp(vm * rr(m + 1), &de);
      ve += de;
      st_m[m] = vm;
      st_e[m] = ve - l;
    }
  }
  __syncthreads();
  const double big = 0x1p256, small = 0x1p-256;
  // Two interleaved output columns per thread (independent recurrences).
  const int step = 2 * blockDim.x;
  for (int ma = threadIdx.x; ma <= l; ma += step) {
    const int mb = ma + blockDim.x;
    const bool hb = mb <= l;
    double cur_a = st_m[ma], nxt_a = 0.0, cur_b = hb ? st_m[mb] : 0.0, nxt_b = 0.0;
    int Ea = st_e[ma], Eb = hb ? st_e[mb] : 0;
    double sca = (Ea > -1000) ? ldexp(1.0, Ea) : 0.0;
    double scb = (hb && Eb > -1000) ? ldexp(1.0, Eb) : 0.0;
    double re_a = 0.0, im_a = 0.0, re_b = 0.0, im_b = 0.0;
    const double twoa = 2.0 * ma, twob = 2.0 * mb;
    for (int k = l; k >= 0; --k) {
      const double da = cur_a * sca, db = cur_b * scb;
      const double ar = a_re[k], ai = a_im[k];
      const double wk = (k == 0) ? 1.0 : 2.0;
      if (((l + ma + k) & 1) == 0) re_a = fma(wk * da, ar, re_a);
      else if (k > 0) im_a = fma(2.0 * da, ai, im_a);
      if (((l + mb + k) & 1) == 0) re_b = fma(wk * db, ar, re_b);
      else if (k > 0) im_b = fma(2.0 * db, ai, im_b);
      if (k == 0) break;
      double pa = (twoa * cur_a - c1[k] * nxt_a) * c2[k];
      double pb = (twob * cur_b - c1[k] * nxt_b) * c2[k];
      if (fabs(pa) > big) {
        pa *= small;
        cur_a *= small;
        Ea += 256;
        sca = (Ea > -1000) ? ldexp(1.0, Ea) : 0.0;
      }
      if (fabs(pb) > big) {
        pb *= small;
        cur_b *= small;
        Eb += 256;
        scb = (Eb > -1000) ? ldexp(1.0, Eb) : 0.0;
      }
      nxt_a = cur_a;
      cur_a = pa;
      nxt_b = cur_b;
      cur_b = pb;
    }
    {
      const int64_t i = hp_index(l, ma, Nl);
      alm_out[2 * i] = alm_add[2 * i] + re_a;
      alm_out[2 * i + 1] = alm_add[2 * i + 1] + im_a;
    }
    if (hb) {
      const int64_t i = hp_index(l, mb, Nl);
      alm_out[2 * i] = alm_add[2 * i] + re_b;
      alm_out[2 * i + 1] = alm_add[2 * i + 1] + im_b;
    }
  }
}

}  // namespace

void launch_rotate_back(const Geometry& g, const double* alm_rot, const double* alm_add, double* alm_out,
                        const unsigned* flags, cudaStream_t s) {
  const size_t smem = (size_t)g.Nl * (6 * sizeof(double) + sizeof(int)) + 64;
  cudaFuncSetAttribute(rotate_back_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  rotate_back_kernel<<<g.Nl, kRotThreads, smem, s>>>(g.Nl, alm_rot, alm_add, alm_out, flags);
  count_launches(1);
}

}  // namespace dsht
