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
// carried with a binary exponent.  One CTA per l, one thread per output m.  FP64 compute
// bound: about 5 DFMA per (l, m, m').
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
  double* st_m = c2 + (l + 1);       // [l+1] start mantissa d_{l,m}
  int* st_e = reinterpret_cast<int*>(st_m + (l + 1));  // [l+1] start exponent
  for (int k = threadIdx.x; k <= l; k += blockDim.x) {
    const int64_t i = hp_index(l, k, Nl);
    a_re[k] = alm_rot[2 * i];
    a_im[k] = alm_rot[2 * i + 1];
    c1[k] = sqrt((double)(l - k) * (double)(l + k + 1));
    c2[k] = (k >= 1) ? 1.0 / sqrt((double)(l + k) * (double)(l - k + 1)) : 0.0;
  }
  if (threadIdx.x == 0) {
    // d_{l,m} from m = l down: ratio d_{l,m-1}/d_{l,m} = -sqrt((l+m)/(l-m+1)).
    double v = 1.0;
    int e = -l;
    st_m[l] = v;
    st_e[l] = e;
    for (int m = l; m >= 1; --m) {
      v *= -sqrt((double)(l + m) / (double)(l - m + 1));
      int de;
      v = frexp(v, &de);
      e += de;
      st_m[m - 1] = v;
      st_e[m - 1] = e;
    }
  }
  __syncthreads();
  const double big = 0x1p256, small = 0x1p-256;
  for (int m = threadIdx.x; m <= l; m += blockDim.x) {
    double cur = st_m[m], nxt = 0.0;
    int E = st_e[m];
    double scale = (E > -1000) ? ldexp(1.0, E) : 0.0;
    double re = 0.0, im = 0.0;
    const double twom = 2.0 * m;
    for (int k = l; k >= 0; --k) {
      const double d = cur * scale;
      if (k == 0) {
        re = fma(d, a_re[0], re);
      } else if (((l + m + k) & 1) == 0) {
        re = fma(2.0 * d, a_re[k], re);
      } else {
        im = fma(2.0 * d, a_im[k], im);
      }
      if (k == 0) break;
      double prv = (twom * cur - c1[k] * nxt) * c2[k];
      if (fabs(prv) > big) {
        prv *= small;
        cur *= small;
        E += 256;
        scale = (E > -1000) ? ldexp(1.0, E) : 0.0;
      }
      nxt = cur;
      cur = prv;
    }
    const int64_t i = hp_index(l, m, Nl);
    alm_out[2 * i] = alm_add[2 * i] + re;
    alm_out[2 * i + 1] = alm_add[2 * i + 1] + im;
  }
}

}  // namespace

void launch_rotate_back(const Geometry& g, const double* alm_rot, const double* alm_add, double* alm_out,
                        const unsigned* flags, cudaStream_t s) {
  const size_t smem = (size_t)g.Nl * (5 * sizeof(double) + sizeof(int)) + 64;
  cudaFuncSetAttribute(rotate_back_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  rotate_back_kernel<<<g.Nl, kRotThreads, smem, s>>>(g.Nl, alm_rot, alm_add, alm_out, flags);
  count_launches(1);
}

}  // namespace dsht
