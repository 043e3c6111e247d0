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
  // a'_{l,k} pre-scaled by 2 (the k = 0 term has weight 1 on the real part).
  for (int k = threadIdx.x; k <= l; k += blockDim.x) {
    a_re[k] *= (k >= 1) ? 2.0 : 1.0;
    a_im[k] *= 2.0;
  }
  __syncthreads();
  // Output column m: d_{k,m} for k = l .. 0 by the downward recurrence.  With pi = m & 1,
  // the terms with k = l, l-2, ... go to Re if pi == 0 and to Im if pi == 1 (l+m+k even
  // <-> real), so each column adds alternately into acc0 (rows k = l, l-2, ...) and acc1.
  // acc0/acc1 are kept in the recurrence's scaled units (x 2^-E) and rescaled with it.
  const double big = 0x1p256, small = 0x1p-256;
  const int step = 2 * blockDim.x;
  for (int ma = threadIdx.x; ma <= l; ma += step) {
    const int mb = ma + blockDim.x;
    const bool hb = mb <= l;
    const double* A0a = (ma & 1) ? a_im : a_re;  // k = l, l-2, ...
    const double* A1a = (ma & 1) ? a_re : a_im;  // k = l-1, l-3, ...
    const double* A0b = (mb & 1) ? a_im : a_re;
    const double* A1b = (mb & 1) ? a_re : a_im;
    double ca = st_m[ma], na = 0.0, cb = hb ? st_m[mb] : 0.0, nb = 0.0;
    int Ea = st_e[ma], Eb = hb ? st_e[mb] : 0;
    double s0a = 0.0, s1a = 0.0, s0b = 0.0, s1b = 0.0;
    const double twoa = 2.0 * ma, twob = 2.0 * mb;
    int k = l;
    // Pairs (k, k-1) while k >= 1; the single k = 0 term is handled after the loop.
    for (int it = 0; k >= 2; ++it) {
      // row k (acc0)
      s0a = fma(ca, A0a[k], s0a);
      s0b = fma(cb, A0b[k], s0b);
      double pa = (twoa * ca - c1[k] * na) * c2[k];
      double pb = (twob * cb - c1[k] * nb) * c2[k];
      na = ca;
      ca = pa;
      nb = cb;
      cb = pb;
      // row k-1 (acc1)
      s1a = fma(ca, A1a[k - 1], s1a);
      s1b = fma(cb, A1b[k - 1], s1b);
      pa = (twoa * ca - c1[k - 1] * na) * c2[k - 1];
      pb = (twob * cb - c1[k - 1] * nb) * c2[k - 1];
      na = ca;
      ca = pa;
      nb = cb;
      cb = pb;
      k -= 2;
      if ((it & 1) == 1) {  // growth per step is bounded, so checking every 4 steps is safe
        if (fabs(ca) > big) {
          ca *= small; na *= small; s0a *= small; s1a *= small; Ea += 256;
        }
        if (fabs(cb) > big) {
          cb *= small; nb *= small; s0b *= small; s1b *= small; Eb += 256;
        }
      }
    }
    // Remaining rows: k == 1 (then 0) or k == 0.
    if (k == 1) {
      s0a = fma(ca, A0a[1], s0a);
      s0b = fma(cb, A0b[1], s0b);
      const double pa = (twoa * ca - c1[1] * na) * c2[1];
      const double pb = (twob * cb - c1[1] * nb) * c2[1];
      na = ca; ca = pa; nb = cb; cb = pb;
      // k = 0 follows k = 1 in acc1's sequence (l odd): the weight-1 real term counts
      // when l + m is even, i.e. m odd, and acc1 is then the real part.
      s1a = fma(ca, ((ma & 1) ? a_re[0] : 0.0), s1a);
      s1b = fma(cb, ((mb & 1) ? a_re[0] : 0.0), s1b);
    } else {  // k == 0 in acc0's sequence (l even): counts when m is even (acc0 real)
      s0a = fma(ca, ((ma & 1) ? 0.0 : a_re[0]), s0a);
      s0b = fma(cb, ((mb & 1) ? 0.0 : a_re[0]), s0b);
    }
    const double fa = (Ea > -1074) ? ldexp(1.0, Ea) : 0.0;
    const double fb = (Eb > -1074) ? ldexp(1.0, Eb) : 0.0;
    // acc0 holds Re when m even, Im when m odd (and acc1 the other).
    const double rea = ((ma & 1) ? s1a : s0a) * fa, ima = ((ma & 1) ? s0a : s1a) * fa;
    {
      const int64_t i = hp_index(l, ma, Nl);
      alm_out[2 * i] = alm_add[2 * i] + rea;
      alm_out[2 * i + 1] = alm_add[2 * i + 1] + ima;
    }
    if (hb) {
      const double reb = ((mb & 1) ? s1b : s0b) * fb, imb = ((mb & 1) ? s0b : s1b) * fb;
      const int64_t i = hp_index(l, mb, Nl);
      alm_out[2 * i] = alm_add[2 * i] + reb;
      alm_out[2 * i + 1] = alm_add[2 * i + 1] + imb;
    }
  }
}

// Several maps per CTA (kMaps of them, map index blockIdx.y * kMaps + g): the d_{k,m}
// recurrence of a column is shared by all maps, each map adds its own two sums, so the
// cost per map falls from about 5 to about 2 DFMA per (l, m, m').  One column per thread;
// io[map] += R(rot[map]) in place; a map whose flags show no polar point is skipped (its
// rotated alm are zero).
template <int kMaps>
__global__ void __launch_bounds__(kRotThreads)
rotate_back_maps_kernel(int Nl, int nmaps, const RotMaps maps) {
  extern __shared__ double sm[];
  const int l = Nl - 1 - blockIdx.x;
  const int map0 = blockIdx.y * kMaps;
  const int nm = min(kMaps, nmaps - map0);
  double* a_re = sm;                         // [kMaps][l+1]
  double* a_im = a_re + kMaps * (l + 1);     // [kMaps][l+1]
  double* c1 = a_im + kMaps * (l + 1);
  double* c2 = c1 + (l + 1);
  double* rat = c2 + (l + 1);
  double* st_m = rat + (l + 1);
  int* st_e = reinterpret_cast<int*>(st_m + (l + 1));
  for (int k = threadIdx.x; k <= l; k += blockDim.x) {
    const int64_t i = hp_index(l, k, Nl);
#pragma unroll
    for (int g = 0; g < kMaps; ++g) {
      const bool ok = g < nm && (!maps.flags[map0 + g] || (*maps.flags[map0 + g] & kFlagHasPolar));
      const double* src = maps.rot[ok ? map0 + g : 0];
      a_re[g * (l + 1) + k] = ok ? src[2 * i] * ((k >= 1) ? 2.0 : 1.0) : 0.0;
      a_im[g * (l + 1) + k] = ok ? src[2 * i + 1] * 2.0 : 0.0;
    }
    c1[k] = sqrt((double)(l - k) * (double)(l + k + 1));
    c2[k] = (k >= 1) ? 1.0 / sqrt((double)(l + k) * (double)(l - k + 1)) : 0.0;
    rat[k] = (k >= 1) ? -sqrt((double)(l + k) / (double)(l - k + 1)) : 1.0;
  }
  __syncthreads();
  if (threadIdx.x < 32) {  // start column, as in rotate_back_kernel
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
    double pm = tm;
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
  const int L1 = l + 1;
  for (int m = threadIdx.x; m <= l; m += blockDim.x) {
    // rows k = l, l-2, ... read A0 (Re when m even), rows l-1, l-3, ... read A1.
    const double* A0 = (m & 1) ? a_im : a_re;
    const double* A1 = (m & 1) ? a_re : a_im;
    double c = st_m[m], n = 0.0;
    int E = st_e[m];
    double s0[kMaps], s1[kMaps];
#pragma unroll
    for (int g = 0; g < kMaps; ++g) s0[g] = s1[g] = 0.0;
    const double two_m = 2.0 * m;
    int k = l;
    for (int it = 0; k >= 2; ++it) {
#pragma unroll
      for (int g = 0; g < kMaps; ++g) s0[g] = fma(c, A0[g * L1 + k], s0[g]);
      double p = (two_m * c - c1[k] * n) * c2[k];
      n = c;
      c = p;
#pragma unroll
      for (int g = 0; g < kMaps; ++g) s1[g] = fma(c, A1[g * L1 + k - 1], s1[g]);
      p = (two_m * c - c1[k - 1] * n) * c2[k - 1];
      n = c;
      c = p;
      k -= 2;
      if ((it & 1) == 1 && fabs(c) > big) {
        c *= small;
        n *= small;
#pragma unroll
        for (int g = 0; g < kMaps; ++g) {
          s0[g] *= small;
          s1[g] *= small;
        }
        E += 256;
      }
    }
    if (k == 1) {
#pragma unroll
      for (int g = 0; g < kMaps; ++g) s0[g] = fma(c, A0[g * L1 + 1], s0[g]);
      const double p = (two_m * c - c1[1] * n) * c2[1];
      n = c;
      c = p;
      if (m & 1) {
#pragma unroll
        for (int g = 0; g < kMaps; ++g) s1[g] = fma(c, a_re[g * L1], s1[g]);
      }
    } else if (!(m & 1)) {
#pragma unroll
      for (int g = 0; g < kMaps; ++g) s0[g] = fma(c, a_re[g * L1], s0[g]);
    }
    const double f = (E > -1074) ? ldexp(1.0, E) : 0.0;
    const int64_t i = hp_index(l, m, Nl);
#pragma unroll
    for (int g = 0; g < kMaps; ++g) {
      if (g < nm && (!maps.flags[map0 + g] || (*maps.flags[map0 + g] & kFlagHasPolar))) {
        double* out = maps.io[map0 + g];
        const double re = ((m & 1) ? s1[g] : s0[g]) * f, im = ((m & 1) ? s0[g] : s1[g]) * f;
        out[2 * i] += re;
        out[2 * i + 1] += im;
      }
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

template <int kMaps>
static void rotate_maps_launch(const Geometry& g, const RotMaps& maps, int nmaps, size_t smem, cudaStream_t s) {
  cudaFuncSetAttribute(rotate_back_maps_kernel<kMaps>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 grid(g.Nl, (nmaps + kMaps - 1) / kMaps);
  rotate_back_maps_kernel<kMaps><<<grid, kRotThreads, smem, s>>>(g.Nl, nmaps, maps);
  count_launches(1);
}

void launch_rotate_back_maps(const Geometry& g, const RotMaps& maps, int nmaps, cudaStream_t s) {
  if (nmaps <= 0) return;
  // As many maps per CTA (8, 4, 2, 1) as the shared-memory limit allows for this Nl; eight
  // only while two such CTAs still fit an SM (at Nl=1024 one 8-map CTA per SM took 0.131 ms
  // per map, two 4-map CTAs per SM 0.107: the recurrence is latency-bound, so residency wins
  // over sharing it between more maps).
  auto bytes = [&](int k) { return (size_t)g.Nl * ((5 + 2 * k) * sizeof(double) + sizeof(int)) + 64; };
  const size_t lim = 227 * 1024;
  if (nmaps > 4 && 2 * (bytes(8) + 1024) <= 228 * 1024)
    rotate_maps_launch<8>(g, maps, nmaps, bytes(8), s);
  else if (nmaps > 2 && bytes(4) <= lim)
    rotate_maps_launch<4>(g, maps, nmaps, bytes(4), s);
  else if (nmaps == 2 && bytes(2) <= lim)
    rotate_maps_launch<2>(g, maps, nmaps, bytes(2), s);
  else
    rotate_maps_launch<1>(g, maps, nmaps, bytes(1), s);
}

}  // namespace dsht
