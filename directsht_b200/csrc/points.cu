// Per-point classification, x-bin search, Hermite weights and the counting sort by bin.
//
// Each point goes to one of four sets: equatorial with cos(theta) >= 0 / < 0, or polar
// (|cos theta| >= xmax, sht/sht.py:128-130) rotated by +90 deg about y and split by the
// sign of the rotated cos.  The bin is numpy's digitize(|x|, x_nodes) - 1 (right-open,
// sht/sht.py:212) and t = (|x| - x_j)/dx (sht/sht.py:221); the payload is cos phi, sin phi
// and w * {(2t+1)(1-t)^2, t(1-t)^2, t^2(3-2t), t^2(t-1)} (sht/sht.py:239-240).
//
// Sort: key = set*(Nx-1) + bin.  The count pass bins every point (its key, 4 bytes) and
// histograms the keys in shared memory (one global add per live key and block); a one-block
// exclusive scan cuts every key into pieces of at most piece_max points; the scatter pass
// reserves a contiguous range per key and block with one global add, recomputes each
// point's 32-byte record (cos phi, sin phi, w, t) -- one DRAM sector -- from its inputs and
// writes it to its sorted slot; the bin-sum kernels form w h_k(t) themselves (the NUFFT bin
// sums take the record (phi, 0, w, t) instead).  HBM bytes per point: 16 read + 4 written
// (count), 28 read + 32 written (scatter), against the algorithmic 24 read + 32 written.
#include "dsht_internal.cuh"

namespace dsht {
namespace {

constexpr int kPointThreads = 256;
constexpr int kScatterTile = 8192;  // points per block in the scatter pass: 1221 blocks at N = 1e7,
                                    // several waves of 3 resident blocks per SM

// The binning of one point: key = set * nbins + bin (DSHT_KEY_DROP when it is in no set)
// and its flag bits.  x = cos(theta) for equatorial points; a polar point (|cos theta| >=
// xmax in __call__) is rotated by +90 deg about y, n = (s cos p, s sin p, c) -> (c, s sin p,
// -s cos p), and binned by its rotated x = -sin(theta) cos(phi) -- the cosine of the rotated
// theta that the reference bins (sht/sht.py:190), without the acos/cos round trip.
// st, c = sin, cos of theta; cp = cos phi (read for polar points only).  The scatter pass
// computes x with the same operations, so the two passes agree on it bit for bit.
struct KeyOut {
  uint32_t key;
  unsigned flag;
  double x;  // the signed x that was binned
};

__device__ __forceinline__ KeyOut point_key(const Geometry& g, double inv_dx, int mode, double th, double st, double c,
                                            const double* phi_p) {
  KeyOut o;
  o.key = DSHT_KEY_DROP;
  o.flag = 0;
  o.x = 0.0;
  double x;
  int set;
  const double xv = fabs(c);
  if (mode == DSHT_MODE_CALL && xv >= g.xmax) {
    double sp, cp;
    sincos(*phi_p, &sp, &cp);
    x = -__dmul_rn(st, cp);
    if (!(x < g.xmax && x > -g.xmax)) {  // the rotated point is still polar
      o.flag = kFlagPolarRange;
      return o;
    }
    set = 2;
    o.flag = kFlagHasPolar;
  } else if (mode == DSHT_MODE_CALL && !(xv < g.xmax)) {
    return o;  // NaN theta: in neither set (sht/sht.py:129-130)
  } else {
    if (!(th >= 0.0 && th > g.acos_xmax && th < g.acos_mxmax)) {  // sht/sht.py:171-172
      o.flag = kFlagThetaRange;
      return o;
    }
    x = c;
    set = 0;
  }
  if (!(x >= 0.0)) set += 1;  // x < 0 half (sht/sht.py:193)
  const double ax = fabs(x);
  // digitize: x_j <= ax < x_{j+1} with x_j = j * dx exactly as numpy builds the grid.
  int j = (int)(ax * inv_dx);
  if (j > g.nbins - 1) j = g.nbins - 1;
  if (j < 0) j = 0;
  if (ax < (double)j * g.dx) j -= 1;
  else if (j + 1 <= g.nbins && ax >= (double)(j + 1) * g.dx) j += 1;
  if (j < 0 || j >= g.nbins) {
    o.flag = (set >= 2) ? kFlagPolarRange : kFlagThetaRange;
    return o;
  }
  o.key = (uint32_t)(set * g.nbins + j);
  o.x = x;
  return o;
}

// FP32 screen of point_key: the same decisions (polar or not, rotated range, sign of x, bin)
// from FP32 sines and cosines, accepted only when no decision lies within the screen of its
// boundary; otherwise (and for every point that raises a flag or is NaN) false, and the
// FP64 path decides.  The sines and cosines are the hardware approximations __sincosf,
// whose absolute error is at most 2^-21.41 (3.6e-7) for arguments in [-pi, pi] (CUDA C
// Programming Guide, intrinsic functions).  Bound on the FP32 x: theta in [0, 3.14] rounds
// to float within 1.2e-7 (and stays below pi), so |sin, cos error| <= 4.8e-7; phi (|phi| <=
// 8) rounds within 2.4e-7 and is brought into [-pi, pi] by one exact (Sterbenz) subtraction
// of the float 2 pi (1.75e-7 from 2 pi) and a clamp to the largest float below pi (at most
// 2.6e-7), so its cosine errs by at most 1.03e-6; the product rounds once: |x32 - x| <
// 1.6e-6, and the screen is 3e-6.  The bin coordinate
// u = |x| / dx errs by at most screen / dx plus its own rounding (nbins 2^-24 per
// operation): bin_guard bounds both.  So an accepted key is the FP64 key.
constexpr float kScreenX = 3e-6f;

__device__ __forceinline__ bool screen_key(const Geometry& g, float inv_dx_f, float bin_guard, float xmax_f, int mode,
                                           double th, double ph, uint32_t* key, unsigned* flag) {
  // the bounds below hold for theta in [0, 3.14] and |phi| <= 8
  if (!(th >= 0.0 && th <= 3.14)) return false;
  float sf, cf;
  __sincosf((float)th, &sf, &cf);
  float x;
  int set;
  *flag = 0;
  if (mode == DSHT_MODE_CALL) {
    const float xv = fabsf(cf);
    if (!(fabsf(xv - xmax_f) >= kScreenX)) return false;  // near the polar boundary, or NaN
    if (xv > xmax_f) {
      if (!(fabs(ph) <= 8.0)) return false;
      constexpr float kTwoPiF = 6.28318548f;  // the float nearest 2 pi
      constexpr float kPiBelow = 3.14159250f;  // the largest float below pi
      float pf = (float)ph;
      if (pf > kPiBelow) pf -= kTwoPiF;
      else if (pf < -kPiBelow) pf += kTwoPiF;
      pf = fminf(fmaxf(pf, -kPiBelow), kPiBelow);
      float sp, cp;
      __sincosf(pf, &sp, &cp);
      x = -sf * cp;
      if (!(fabsf(x) <= xmax_f - kScreenX)) return false;  // near or beyond the rotated range
      set = 2;
      *flag = kFlagHasPolar;
    } else {
      if (!(th >= 0.0 && th > g.acos_xmax && th < g.acos_mxmax)) return false;
      x = cf;
      set = 0;
    }
  } else {
    if (!(th >= 0.0 && th > g.acos_xmax && th < g.acos_mxmax)) return false;
    x = cf;
    set = 0;
  }
  if (!(fabsf(x) >= kScreenX)) return false;  // the sign of x near 0
  if (x < 0.0f) set += 1;
  const float u = fabsf(x) * inv_dx_f;
  const int j = (int)u;
  const float fr = u - (float)j;
  if (!(fr >= bin_guard && fr <= 1.0f - bin_guard) || j >= g.nbins) return false;
  *key = (uint32_t)(set * g.nbins + j);
  return true;
}

// Count pass: the key of every point (4 bytes written) and a shared-memory histogram of the
// keys (one global add per live key and block).  Reads theta and phi (phi for every point in
// __call__ mode: polar candidates are a third of a survey footprint, so their phi loads
// touch most sectors anyway, and loading every phi alongside theta keeps the loads
// independent).  Four points per thread per round, all their loads issued first.  Keys come
// from the FP32 screen; the points it leaves undecided (~2 % at Nx = 2048) are queued in
// shared memory and decided by the FP64 path a few rounds later by whole warps, so the FP64
// sines and cosines run for those points only.
constexpr int kCountUnroll = 4;
constexpr int kQueueRounds = 2;  // rounds of kCountUnroll * blockDim points between queue flushes

__global__ void __launch_bounds__(kPointThreads)
count_kernel(Geometry g, int mode, const double* __restrict__ theta, const double* __restrict__ phi,
             int64_t N, uint32_t* __restrict__ keys, uint32_t* __restrict__ count, unsigned* __restrict__ flags,
             float bin_guard) {
  extern __shared__ uint32_t hist[];  // [nkeys], then the queue [kQueueRounds * kCountUnroll * blockDim]
  uint32_t* queue = hist + g.nkeys;
  __shared__ int qn;
  for (int k = threadIdx.x; k < g.nkeys; k += blockDim.x) hist[k] = 0;
  if (threadIdx.x == 0) qn = 0;
  __syncthreads();
  unsigned fl = 0;
  const double inv_dx = 1.0 / g.dx;
  const float inv_dx_f = (float)inv_dx, xmax_f = (float)g.xmax;
  const int64_t span = (int64_t)kCountUnroll * blockDim.x;
  const int64_t stride = (int64_t)gridDim.x * span;
  const bool call = mode == DSHT_MODE_CALL;
  int round = 0;
  // block-uniform trip count: every thread reaches every flush
  for (int64_t base = (int64_t)blockIdx.x * span; base < N; base += stride) {
    double th[kCountUnroll], ph[kCountUnroll];
#pragma unroll
    for (int u = 0; u < kCountUnroll; ++u) {
      const int64_t i = base + (int64_t)u * blockDim.x + threadIdx.x;
      th[u] = 0.0;
      ph[u] = 0.0;
      if (i < N) {
        th[u] = theta[i];
        if (call) ph[u] = phi[i];
      }
    }
#pragma unroll
    for (int u = 0; u < kCountUnroll; ++u) {
      const int64_t i = base + (int64_t)u * blockDim.x + threadIdx.x;
      if (i < N) {
        uint32_t key;
        unsigned f;
        if (screen_key(g, inv_dx_f, bin_guard, xmax_f, mode, th[u], ph[u], &key, &f)) {
          keys[i] = key;
          fl |= f;
          atomicAdd(&hist[key], 1u);
        } else {
          queue[atomicAdd(&qn, 1)] = (uint32_t)i;
        }
      }
    }
    if (++round == kQueueRounds || base + stride >= N) {
      round = 0;
      __syncthreads();
      const int nq = qn;
      for (int q = threadIdx.x; q < nq; q += blockDim.x) {
        const int64_t k = queue[q];
        const double t = theta[k];
        double st, c;
        sincos(t, &st, &c);
        const KeyOut o = point_key(g, inv_dx, mode, t, st, c, phi + k);
        keys[k] = o.key;
        fl |= o.flag;
        if (o.key != DSHT_KEY_DROP) atomicAdd(&hist[o.key], 1u);
      }
      __syncthreads();
      if (threadIdx.x == 0) qn = 0;
      __syncthreads();
    }
  }
  if (fl) atomicOr(flags, fl);
  __syncthreads();
  for (int k = threadIdx.x; k < g.nkeys; k += blockDim.x)
    if (hist[k]) atomicAdd(&count[k], hist[k]);
}

// Single-block exclusive scans: key offsets, pieces per key, and the piece list.
constexpr int kScanThreads = 1024;

__device__ __forceinline__ uint32_t block_scan_excl(uint32_t v, uint32_t* warp_tot, uint32_t* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint32_t t = (lane < (int)(blockDim.x >> 5)) ? warp_tot[lane] : 0u;
    uint32_t s = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    warp_tot[lane] = s - t;
    if (lane == 31) *total = s;
  }
  __syncthreads();
  uint32_t r = x - v + warp_tot[wid];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kScanThreads)
scan_kernel(int nkeys, int nbins, int piece_max, int64_t pmax, const uint32_t* __restrict__ count,
            uint32_t* __restrict__ offset, uint32_t* __restrict__ cursor, int* __restrict__ piece_first,
            int* __restrict__ piece_key, int64_t* __restrict__ piece_start, int* __restrict__ piece_len,
            int* __restrict__ npieces) {
  __shared__ uint32_t warp_tot[32];
  __shared__ uint32_t total;
  __shared__ uint32_t carry_off, carry_pc;
  if (threadIdx.x == 0) { carry_off = 0; carry_pc = 0; }
  __syncthreads();
  for (int base = 0; base < nkeys; base += blockDim.x) {
    const int k = base + threadIdx.x;
    const uint32_t c = (k < nkeys) ? count[k] : 0u;
    const uint32_t pc = (c + piece_max - 1) / piece_max;
    uint32_t o = block_scan_excl(c, warp_tot, &total);
    const uint32_t tot_c = total;
    uint32_t p = block_scan_excl(pc, warp_tot, &total);
    const uint32_t tot_p = total;
    o += carry_off;
    p += carry_pc;
    if (k < nkeys) {
      offset[k] = o;
      cursor[k] = o;
      piece_first[k] = (int)p;
      for (uint32_t q = 0; q < pc; ++q) {
        const int64_t pi = (int64_t)p + q;
        if (pi < pmax) {
          piece_key[pi] = k;
          piece_start[pi] = (int64_t)o + (int64_t)q * piece_max;
          const uint32_t rem = c - q * piece_max;
          piece_len[pi] = (int)(rem < (uint32_t)piece_max ? rem : (uint32_t)piece_max);
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) { carry_off += tot_c; carry_pc += tot_p; }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    offset[nkeys] = carry_off;
    piece_first[nkeys] = (int)carry_pc;
    *npieces = (int)carry_pc;
  }
}

// Largest |w h_k| of a point as float bits (non-negative floats order like their bits).
__device__ __forceinline__ uint32_t gmax_bits(const double* h) {
  return __float_as_uint((float)fmax(fmax(fabs(h[0]), fabs(h[1])), fmax(fabs(h[2]), fabs(h[3]))));
}

// Scatter pass: every point's 32-byte record (cos phi, sin phi, w, t) -- one DRAM sector --
// to its sorted slot.  The record is recomputed from theta, phi, w and the key of the count
// pass: for a rotated polar point the azimuth of (c, s sin p, -s cos p), kept as its cosine
// and sine (c / rho, s sin p / rho), and t = (|x| - x_j) / dx (sht/sht.py:221).
// PHI: the record holds (phi, 0, w, t) instead -- the azimuth itself (of the rotated point
// for polar points, in [0, 2 pi)), which is what the NUFFT bin sums spread by; equatorial
// points then need no sine or cosine of phi at all.
template <typename WT, bool PHI>
__global__ void __launch_bounds__(kPointThreads)
scatter_kernel(Geometry g, const double* __restrict__ theta, const double* __restrict__ phi,
               const WT* __restrict__ w, int64_t N, const uint32_t* __restrict__ keys, uint32_t* __restrict__ cursor,
               double* __restrict__ pay, uint32_t* __restrict__ sidx) {
  extern __shared__ uint32_t loc[];  // [nkeys] local counts, then local bases
  const int64_t lo = (int64_t)blockIdx.x * kScatterTile;
  const int64_t hi = min(lo + (int64_t)kScatterTile, N);
  for (int k = threadIdx.x; k < g.nkeys; k += blockDim.x) loc[k] = 0;
  __syncthreads();
  constexpr int kUnroll = 4;
  const int64_t step = (int64_t)kUnroll * blockDim.x;
  for (int64_t b = lo + threadIdx.x; b < hi; b += step) {
    uint32_t k[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int64_t i = b + (int64_t)u * blockDim.x;
      k[u] = (i < hi) ? keys[i] : DSHT_KEY_DROP;
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
      if (k[u] != DSHT_KEY_DROP) atomicAdd(&loc[k[u]], 1u);
  }
  __syncthreads();
  // one global reservation per (block, key); eight of a thread's in flight at once
  for (int k0 = threadIdx.x; k0 < g.nkeys; k0 += 8 * blockDim.x) {
    uint32_t c[8], r[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = k0 + u * blockDim.x;
      c[u] = k < g.nkeys ? loc[k] : 0u;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (c[u]) r[u] = atomicAdd(&cursor[k0 + u * blockDim.x], c[u]);
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (c[u]) loc[k0 + u * blockDim.x] = r[u];
  }
  __syncthreads();
  const int polar_key0 = 2 * g.nbins;
  const double inv_dx = 1.0 / g.dx;
  for (int64_t b = lo + threadIdx.x; b < hi; b += step) {
    uint32_t k[kUnroll], pos[kUnroll];
    double th[kUnroll], ph[kUnroll], wi[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const int64_t i = b + (int64_t)u * blockDim.x;
      k[u] = DSHT_KEY_DROP;
      if (i < hi) {
        k[u] = keys[i];
        th[u] = theta[i];
        ph[u] = phi[i];
        wi[u] = (double)w[i];
      }
    }
    // the slots first: their shared-memory round trips overlap the record arithmetic
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
      if (k[u] != DSHT_KEY_DROP) pos[u] = atomicAdd(&loc[k[u]], 1u);
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      if (k[u] == DSHT_KEY_DROP) continue;
      double st, c, sp, cp;
      sincos(th[u], &st, &c);
      double cphi, sphi, x = c;
      if constexpr (PHI) {
        constexpr double two_pi = 6.28318530717958647693;
        sphi = 0.0;
        if ((int)k[u] >= polar_key0) {
          sincos(ph[u], &sp, &cp);
          x = -__dmul_rn(st, cp);
          cphi = atan2(st * sp, c);  // azimuth of the rotated point (c, s sin p, -s cos p)
        } else {
          cphi = ph[u];
          if (!(cphi >= 0.0 && cphi < two_pi)) cphi -= two_pi * floor(cphi / two_pi);
        }
        if (cphi < 0.0) cphi += two_pi;
      } else {
        sincos(ph[u], &sp, &cp);
        cphi = cp;
        sphi = sp;
        if ((int)k[u] >= polar_key0) {
          x = -__dmul_rn(st, cp);
          const double ny = st * sp;
          const double rho = sqrt(ny * ny + c * c);
          cphi = 1.0;
          sphi = 0.0;
          if (rho > 0.0) {
            const double ir = 1.0 / rho;
            cphi = c * ir;
            sphi = ny * ir;
          }
        }
      }
      const int kk = (int)k[u];  // bin j = key - set nbins, without an integer division
      const int j = kk - g.nbins * ((kk >= g.nbins) + (kk >= 2 * g.nbins) + (kk >= 3 * g.nbins));
      // t = (|x| - x_j) / dx in the reference's rounding (sht/sht.py:221); the NUFFT route
      // (mixed levels) takes the product with 1/dx, within an ulp of it
      const double t = PHI ? (fabs(x) - (double)j * g.dx) * inv_dx
                           : __ddiv_rn(__dadd_rn(fabs(x), -(double)j * g.dx), g.dx);
      double2* out = reinterpret_cast<double2*>(pay + (size_t)kRec * pos[u]);  // one 32-byte sector
      out[0] = make_double2(cphi, sphi);
      out[1] = make_double2(wi[u], t);
      if (sidx) sidx[pos[u]] = (uint32_t)(b + (int64_t)u * blockDim.x);
    }
  }
}

// Another weight map on the same sorted points (multi-map transforms share the sort): the
// record's w becomes w[sidx[pos]].
template <typename WT>
__global__ void __launch_bounds__(kPointThreads)
gather_kernel(int64_t N, const uint32_t* __restrict__ total, const uint32_t* __restrict__ sidx,
              const WT* __restrict__ w, double* __restrict__ pay) {
  const int64_t n = (int64_t)*total;
  for (int64_t pos = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; pos < n && pos < N;
       pos += (int64_t)gridDim.x * blockDim.x)
    pay[(size_t)kRec * pos + 2] = (double)w[sidx[pos]];
}

// Largest |w h_k| of every piece (float bits; the fixed-point scale of the tensor-core
// sums): one warp per piece reads its sorted records (w, t) in order.
__global__ void __launch_bounds__(kPointThreads)
piecemax_kernel(const double* __restrict__ pay, const int* __restrict__ npieces_p, int64_t pmax,
                const int64_t* __restrict__ piece_start, const int* __restrict__ piece_len,
                uint32_t* __restrict__ piecemax, double* __restrict__ wsum) {
  const int lane = threadIdx.x & 31;
  const int64_t np = min((int64_t)*npieces_p, pmax);
  const int64_t wstride = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t pc = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); pc < np; pc += wstride) {
    const int64_t st = piece_start[pc];
    const int len = piece_len[pc];
    uint32_t mx = 0;
    double ws = 0.0;
    const double2* base = reinterpret_cast<const double2*>(pay + (size_t)kRec * st) + 1;
    int i = lane;
    for (; i + 96 < len; i += 128) {  // four records in flight per lane
      const double2 a = base[2 * i], b = base[2 * (i + 32)], c = base[2 * (i + 64)], d = base[2 * (i + 96)];
      double h[4];
      hermite(a.y, a.x, h);
      mx = max(mx, gmax_bits(h));
      hermite(b.y, b.x, h);
      mx = max(mx, gmax_bits(h));
      hermite(c.y, c.x, h);
      mx = max(mx, gmax_bits(h));
      hermite(d.y, d.x, h);
      mx = max(mx, gmax_bits(h));
      ws += (fabs(a.x) + fabs(b.x)) + (fabs(c.x) + fabs(d.x));
    }
    for (; i < len; i += 32) {
      const double2 a = base[2 * i];
      double h[4];
      hermite(a.y, a.x, h);
      mx = max(mx, gmax_bits(h));
      ws += fabs(a.x);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      ws += __shfl_xor_sync(0xffffffffu, ws, o);
    }
    if (lane == 0) {
      piecemax[pc] = mx;
      wsum[pc] = ws;
    }
  }
}

__global__ void publish_flags_kernel(const StatusOut st, int n, unsigned* all) {
  const int k = threadIdx.x;
  if (k >= n) return;
  const unsigned f = *st.slot[k];
  atomicOr(all, f);
  if (st.status[k]) *st.status[k] = f;
}

}  // namespace

void launch_points(const Geometry& g, const double* theta, const double* phi, const void* w, int w_f32,
                   int64_t N, int mode, const Workspace& ws, cudaStream_t s, bool phi_record) {
  cudaMemsetAsync(ws.count, 0, sizeof(uint32_t) * (g.nkeys + 1), s);
  cudaMemsetAsync(ws.flags, 0, sizeof(unsigned), s);
  const size_t hsmem = sizeof(uint32_t) * g.nkeys;
  const size_t csmem = hsmem + sizeof(uint32_t) * kQueueRounds * kCountUnroll * kPointThreads;
  cudaFuncSetAttribute(count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csmem);
  if (N > 0) {
    int64_t blocks = (N + kPointThreads * 2 * kCountUnroll - 1) / (kPointThreads * 2 * kCountUnroll);
    if (blocks > 148 * 4) blocks = 148 * 4;  // fewer, longer blocks: fewer per-block key flushes
    // fraction-of-bin guard of the FP32 screen: the x bound over dx, plus the rounding of
    // u = |x| / dx (four roundings of a value below nbins)
    const float guard = (float)(kScreenX / g.dx + 4.0 * g.nbins * 5.960464477539063e-08 + 1e-6);
    count_kernel<<<(unsigned)blocks, kPointThreads, csmem, s>>>(g, mode, theta, phi, N, ws.key, ws.count,
                                                                ws.flags, guard);
    count_launches(1);
  }
  scan_kernel<<<1, kScanThreads, 0, s>>>(g.nkeys, g.nbins, ws.piece_max, ws.pmax, ws.count, ws.offset,
                                         ws.cursor, ws.piece_first, ws.piece_key, ws.piece_start,
                                         ws.piece_len, ws.npieces);
  count_launches(1);
  if (N > 0) {
    const int64_t blocks = (N + kScatterTile - 1) / kScatterTile;
    auto go = [&](auto kern, const auto* wp) {
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsmem);
      kern<<<(unsigned)blocks, kPointThreads, hsmem, s>>>(g, theta, phi, wp, N, ws.key, ws.cursor, ws.pay,
                                                          ws.sidx);
    };
    if (phi_record) {
      if (w_f32) go(scatter_kernel<float, true>, reinterpret_cast<const float*>(w));
      else go(scatter_kernel<double, true>, reinterpret_cast<const double*>(w));
    } else {
      if (w_f32) go(scatter_kernel<float, false>, reinterpret_cast<const float*>(w));
      else go(scatter_kernel<double, false>, reinterpret_cast<const double*>(w));
    }
    count_launches(1);
  }
}

void launch_gather(const Geometry& g, const void* w, int w_f32, int64_t N, const Workspace& ws, cudaStream_t s) {
  if (N <= 0) return;
  int64_t blocks = (N + kPointThreads - 1) / kPointThreads;
  if (blocks > 148 * 16) blocks = 148 * 16;
  const uint32_t* total = ws.offset + g.nkeys;
  if (w_f32)
    gather_kernel<float><<<(unsigned)blocks, kPointThreads, 0, s>>>(N, total, ws.sidx,
                                                                    reinterpret_cast<const float*>(w), ws.pay);
  else
    gather_kernel<double><<<(unsigned)blocks, kPointThreads, 0, s>>>(N, total, ws.sidx,
                                                                     reinterpret_cast<const double*>(w), ws.pay);
  count_launches(1);
}

void launch_piece_maxima(const Workspace& ws, cudaStream_t s) {
  int64_t blocks = (ws.pmax + (kPointThreads / 32) - 1) / (kPointThreads / 32);
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  piecemax_kernel<<<(unsigned)blocks, kPointThreads, 0, s>>>(ws.pay, ws.npieces, ws.pmax, ws.piece_start,
                                                              ws.piece_len, ws.piecemax, ws.wsum);
  count_launches(1);
}

void launch_publish_flags(const StatusOut& st, int n, unsigned* all, cudaStream_t s) {
  if (n <= 0) return;
  publish_flags_kernel<<<1, 32, 0, s>>>(st, n, all);
  count_launches(1);
}

}  // namespace dsht
