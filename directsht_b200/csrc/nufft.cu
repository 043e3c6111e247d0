// Per-bin sums by a type-1 non-uniform FFT (the MIXED level's default bin-sum method).
//
// For one piece (points of one (set, bin) key) the sums of sht/shared_interp_funcs.py:88-105,
//   v_k[m] = sum_p g_k(p) e^{i m phi_p},  g_k = w h_k(t) (sht/sht.py:239-240),  0 <= m < Nl,
// are the Fourier coefficients of four real point distributions on the circle.  Each point
// is spread onto a periodic real grid of n = 4 * 2^ceil(log2 Nl) cells (oversampling 2 of
// the 2 Nl frequencies -Nl < m < Nl) with the "exponential of semicircle" kernel
//   psi(x) = exp(beta (sqrt(1 - (2x/W)^2) - 1)),  |x| < W/2 cells,  W = 12, beta = 2.30 W
// (Barnett, Magland & af Klinteberg, SIAM J. Sci. Comput. 41 (2019) C479), then
//   v_k[m] = (sum_j G_k[j] e^{2 pi i m j / n}) / Psi(m),  Psi(m) = int psi(x) e^{-2 pi i m x/n} dx
// up to a relative error of about 5e-12 of sum_p |g_k(p)| (aliasing of the truncated
// kernel).  The two real grids of a pair (k, k+1) form one complex sequence, so four
// grids take two complex FFTs; v_k and v_(k+1) come apart by the conjugate symmetry of a
// real sequence's transform.
//
// Kernel values: psi at the W cells next to a point is a polynomial of degree 11 in the
// point's fractional cell offset, one polynomial per cell (Chebyshev interpolants,
// converted to monomials on the host; max error 1e-13 of psi(0)).  They are passed as a
// kernel parameter, so every Horner step is one DFMA with a uniform operand.
//
// One CTA per piece (persistent over pieces): the power of two above the piece's sum |w|
// sets a fixed-point step; the piece's points are spread as 46-bit fixed-point
// values, each added as two native 32-bit shared-memory reductions (low 16 bits, high
// bits), so the sums are exact and independent of the order of the adds; the planes
// (bank = cell mod 32) are converted to FP64 in place, then an in-place
// decimation-in-frequency FFT (radix-16 passes and one radix-2/4/8 pass, the 16-point DFTs
// in registers, twiddles staged in shared memory), then each thread reads the outputs of
// its m from their digit-reversed positions, divides by Psi(m) and writes the piece's
// partial sums [8][Nl] (FP64, k-major, re | im).  The grid index i is stored at i + i/16
// (one 16-byte pad per 16 entries) so that the last pass's unit-stride butterflies hit
// distinct banks.  FP64 throughout; no tensor cores: per point about 130 DFMA for the
// kernel values and 96 reductions for the spread, per piece 2 x 5 n log2 n for the FFTs --
// against 24 x Nl flop per point for the direct sums.
#include <cmath>
#include <mutex>
#include <vector>

#include "dsht_internal.cuh"

namespace dsht {

constexpr int kEsW = 12;     // kernel width in cells
constexpr int kEsDeg = 11;   // polynomial degree per cell
constexpr double kEsBeta = 2.30 * kEsW;

// Kernel-parameter copy of the per-cell polynomials: c[i][d], cell i = 0..W-1 of a point
// whose cell is c0 is (c0 - W/2 + 1 + i) and its offset x = f + W/2 - 1 - i, f = u - c0.
struct EsPoly {
  double c[kEsW][kEsDeg + 1];
};

namespace {

constexpr int kNuThreads = 512;

__device__ __forceinline__ int padi(int i) { return i + (i >> 4); }

// v (|v| < 2^51) as a double, exactly, through the binade of 1.5 2^52 (no conversion
// instruction).
__device__ __forceinline__ double from_fixed(long long v) {
  return __longlong_as_double(v + 0x4338000000000000ll) - 6755399441055744.0;
}

__device__ __forceinline__ double2 cmul2(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

// cos, sin of 2 pi e / 16 for a compile-time e (after unrolling).
__device__ __forceinline__ double cos16(int e) {
  constexpr double kCos1 = 0.92387953251128675613, kCos2 = 0.70710678118654752440, kCos3 = 0.38268343236508977173;
  switch (e & 15) {
    case 0: return 1.0;
    case 1: return kCos1;
    case 2: return kCos2;
    case 3: return kCos3;
    case 4: return 0.0;
    case 5: return -kCos3;
    case 6: return -kCos2;
    case 7: return -kCos1;
    case 8: return -1.0;
    case 9: return -kCos1;
    case 10: return -kCos2;
    case 11: return -kCos3;
    case 12: return 0.0;
    case 13: return kCos3;
    case 14: return kCos2;
    default: return kCos1;
  }
}
__device__ __forceinline__ double sin16(int e) { return cos16(e - 4); }

// v * e^{2 pi i e / R}; the quarter turns are exact swaps and sign changes.
template <int R>
__device__ __forceinline__ double2 rot(double2 v, int e) {
  const int e16 = (e * (16 / R)) & 15;
  if (e16 == 0) return v;
  if (e16 == 4) return make_double2(-v.y, v.x);
  if (e16 == 8) return make_double2(-v.x, -v.y);
  if (e16 == 12) return make_double2(v.y, -v.x);
  const double c = cos16(e16), s = sin16(e16);
  return make_double2(fma(v.x, c, -v.y * s), fma(v.x, s, v.y * c));
}

// In-register R-point DFT with the + sign, y_S = sum_r x_r e^{2 pi i r S / R}.  R = 8, 16
// split as 4 x (R/4): radix-4 over r = 4-blocks, twiddle, R/4-point DFTs; output S lands
// in register dreg<R>(S).
template <int R>
__device__ __forceinline__ constexpr int dreg(int S) {
  return R <= 4 ? S : (R / 4) * (S % 4) + S / 4;
}

__device__ __forceinline__ void dft4(double2& x0, double2& x1, double2& x2, double2& x3) {
  const double2 a0 = make_double2(x0.x + x2.x, x0.y + x2.y), a1 = make_double2(x0.x - x2.x, x0.y - x2.y);
  const double2 b0 = make_double2(x1.x + x3.x, x1.y + x3.y), b1 = make_double2(x1.x - x3.x, x1.y - x3.y);
  x0 = make_double2(a0.x + b0.x, a0.y + b0.y);
  x2 = make_double2(a0.x - b0.x, a0.y - b0.y);
  x1 = make_double2(a1.x - b1.y, a1.y + b1.x);  // a1 + i b1
  x3 = make_double2(a1.x + b1.y, a1.y - b1.x);  // a1 - i b1
}

template <int R>
__device__ __forceinline__ void dft(double2 (&x)[R]) {
  if constexpr (R == 2) {
    const double2 a = x[0], b = x[1];
    x[0] = make_double2(a.x + b.x, a.y + b.y);
    x[1] = make_double2(a.x - b.x, a.y - b.y);
  } else if constexpr (R == 4) {
    dft4(x[0], x[1], x[2], x[3]);
  } else {
    constexpr int R2 = R / 4;
    // radix 4 over the blocks of R2: element t + R2 r, output s goes to register t + R2 s
#pragma unroll
    for (int t = 0; t < R2; ++t) {
      dft4(x[t], x[t + R2], x[t + 2 * R2], x[t + 3 * R2]);
#pragma unroll
      for (int s = 1; s < 4; ++s) x[t + R2 * s] = rot<R>(x[t + R2 * s], t * s);
    }
    // R2-point DFTs of each s: registers R2 s .. R2 s + R2 - 1, output k' in register R2 s + k'
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      if constexpr (R2 == 2) {
        const double2 a = x[R2 * s], b = x[R2 * s + 1];
        x[R2 * s] = make_double2(a.x + b.x, a.y + b.y);
        x[R2 * s + 1] = make_double2(a.x - b.x, a.y - b.y);
      } else {
        dft4(x[R2 * s], x[R2 * s + 1], x[R2 * s + 2], x[R2 * s + 3]);
      }
    }
  }
}

// One decimation-in-frequency pass of radix R over span L on `nseq` padded sequences of
// length n: butterfly (b, j), base = b L + j, elements base + r L/R; outputs S times
// e^{2 pi i j S / L} back to base + S L/R.  tw[i] = e^{2 pi i i / n}.
template <int R>
__device__ __forceinline__ void fft_pass(double2* zs, int nseq, int seq_stride, int logn, int logL,
                                         const double2* __restrict__ tw) {
  constexpr int logR = R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : 4;
  const int logs = logL - logR;  // log2 of the stride L/R
  const int nb = 1 << (logn - logR);
  for (int q = threadIdx.x; q < nseq * nb; q += blockDim.x) {
    const int seq = q >> (logn - logR), qq = q & (nb - 1);
    const int j = qq & ((1 << logs) - 1);
    const int base = ((qq >> logs) << logL) + j;
    double2* z = zs + seq * seq_stride;
    double2 x[R];
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = z[padi(base + (r << logs))];
    dft<R>(x);
    if (j) {
      const double2 w1 = tw[j << (logn - logL)];
      double2 ws = w1;
#pragma unroll
      for (int S = 1; S < R; ++S) {
        x[dreg<R>(S)] = cmul2(x[dreg<R>(S)], ws);
        if (S + 1 < R) ws = cmul2(ws, w1);
      }
    }
#pragma unroll
    for (int S = 0; S < R; ++S) z[padi(base + (S << logs))] = x[dreg<R>(S)];
  }
}

// Position of output k after the passes (radix 16 first, then 2^(logn % 4)).
__device__ __forceinline__ int fft_pos(int k, int logn) {
  int pos = 0, lg = logn;
  while (lg >= 4) {
    lg -= 4;
    pos += (k & 15) << lg;
    k >>= 4;
  }
  return pos + k;  // the last pass (radix 2^lg) leaves its digit in place
}

template <int NSEQ>
__device__ void fft_all(double2* zs, int seq_stride, int logn, const double2* __restrict__ tw) {
  int logL = logn;
  while (logL >= 4) {
    fft_pass<16>(zs, NSEQ, seq_stride, logn, logL, tw);
    logL -= 4;
    __syncthreads();
  }
  if (logL == 1) fft_pass<2>(zs, NSEQ, seq_stride, logn, logL, tw);
  else if (logL == 2) fft_pass<4>(zs, NSEQ, seq_stride, logn, logL, tw);
  else if (logL == 3) fft_pass<8>(zs, NSEQ, seq_stride, logn, logL, tw);
  __syncthreads();
}

constexpr int kMaxTw = 8192 / 16;  // twiddles of the largest grid (Nl = 2048)
constexpr int kMaxNl = 2048;

// Shared-memory bytes of a launch: the grids, then the twiddles e^{2 pi i j/n} (j < n/16)
// and 1/Psi(m).
size_t nufft_smem_bytes(int logn, int nseq) {
  const size_t n = (size_t)1 << logn;
  return 16 * nseq * (n + n / 16) + 16 * kMaxTw + 8 * kMaxNl;
}

// V = hi 2^16 + lo (|V| < 2^51) as a double, exactly.
__device__ __forceinline__ double from_parts(unsigned hi, unsigned lo) {
  return from_fixed((long long)(int)hi * 65536 + (long long)lo);
}

// KP: Hermite weights per pass, 4 (two sequences; n <= 4096) or 2 (one sequence; n = 8192).
//
// Spread layout: while points are spread, the 136 slots (544 words) of each 128-cell group g
// of a sequence hold four planes of 128 words: the low 16 bits and the high bits of the
// fixed-point sums of the sequence's real part (k) and imaginary part (k + 1), word
// 544 g + 128 plane + cell % 128 -- a multiple of 32 plus the cell, so consecutive cells
// fall in consecutive banks, across groups too.  Every fixed-point value X (|X| < 2^47)
// is added as two native 32-bit reductions, lo = X mod 2^16 and hi = X >> 16: the low sums
// stay below 2^32 for up to 65536 points per cell and the high sums below 2^31, so
// hi 2^16 + lo is the exact sum.  Points are taken in record order (random cells): a warp's
// 32 reductions fall on random banks.  (Taking them in cell order was measured slower:
// several points of a piece share a cell, and same-word reductions serialise.)
template <int KP>
__global__ void __launch_bounds__(kNuThreads, 1)
nufft_sums_kernel(int Nl, int logn, const double* __restrict__ pay, const int* __restrict__ npieces_p,
                  int64_t pmax, const int64_t* __restrict__ piece_start, const int* __restrict__ piece_len,
                  const double* __restrict__ dinv, const double2* __restrict__ tw, const EsPoly es,
                  double* __restrict__ partial, double* __restrict__ wsum) {
  constexpr int NSEQ = KP / 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ unsigned long long red[1];
  __shared__ double wred[32];
  const int n = 1 << logn, ng = n >> 4;
  const int seq_stride = n + (n >> 4);  // double2 slots per sequence
  double2* zs = reinterpret_cast<double2*>(smem_raw);
  unsigned* zw = reinterpret_cast<unsigned*>(smem_raw);
  double2* tws = reinterpret_cast<double2*>(smem_raw + (size_t)16 * NSEQ * seq_stride);
  double* dinvs = reinterpret_cast<double*>(tws + kMaxTw);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int i = threadIdx.x; i < ng; i += blockDim.x) tws[i] = tw[i];
  for (int m = threadIdx.x; m < Nl; m += blockDim.x) dinvs[m] = dinv[m];
  __syncthreads();
  const double u_per_rad = (double)n * 0.15915494309189533577;  // n / (2 pi)
  const int npieces = (int)min((int64_t)*npieces_p, pmax);
  // sum |w| of a piece with a margin for its own rounding, and max |w| (only to detect
  // non-finite weights).  The bound 2^e above it bounds every grid value (|h_k| <= 1,
  // psi <= 1), so the spread runs in fixed point of step 2^(e - 46) with integer reductions:
  // the grid does not depend on the order of the adds.  The sum itself is summed in whatever
  // order the sort left the points; e can only differ between runs when the sum lies within
  // its rounding (~len 2^-53 relative) of a power of two.  This thread's share of a piece,
  // from its point pfrom on, four loads in flight:
  auto bound_part = [&](const double* r0, int l, int pfrom, double& wa, unsigned long long& mb) {
    const int bd = blockDim.x;
    int p = pfrom;
    for (; p + 3 * bd < l; p += 4 * bd) {
      const double a0 = fabs(r0[(size_t)kRec * p + 2]), a1 = fabs(r0[(size_t)kRec * (p + bd) + 2]);
      const double a2 = fabs(r0[(size_t)kRec * (p + 2 * bd) + 2]), a3 = fabs(r0[(size_t)kRec * (p + 3 * bd) + 2]);
      wa += (a0 + a1) + (a2 + a3);
      mb = max(max(mb, (unsigned long long)__double_as_longlong(a0)),
               max((unsigned long long)__double_as_longlong(a1),
                   max((unsigned long long)__double_as_longlong(a2), (unsigned long long)__double_as_longlong(a3))));
    }
    for (; p < l; p += bd) {
      const double a = fabs(r0[(size_t)kRec * p + 2]);
      wa += a;
      mb = max(mb, (unsigned long long)__double_as_longlong(a));
    }
  };
  // The shares of the CTA's first piece here; those of every later piece while the piece
  // before it is summed (the first four loads are issued before that piece's extraction
  // phase and summed after it).
  double wabs_n = 0.0;
  unsigned long long mbits_n = 0ull;
  if ((int)blockIdx.x < npieces)
    bound_part(pay + (size_t)kRec * piece_start[blockIdx.x], piece_len[blockIdx.x], threadIdx.x, wabs_n, mbits_n);
  for (int piece = blockIdx.x; piece < npieces; piece += gridDim.x) {
    const int64_t start = piece_start[piece];
    const int len = piece_len[piece];
    const double* rec0 = pay + (size_t)kRec * start;
    const int nxt = piece + (int)gridDim.x;
    // The next piece's records into L2 while this one is summed (warp 0).
    if (warp == 0 && nxt < npieces)
      prefetch_l2(pay + (size_t)kRec * piece_start[nxt], sizeof(double) * kRec * (size_t)piece_len[nxt], lane, 32);
    unsigned long long mbits = mbits_n;
    double wabs = wabs_n;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mbits = max(mbits, __shfl_xor_sync(0xffffffffu, mbits, o));
      wabs += __shfl_xor_sync(0xffffffffu, wabs, o);
    }
    if (threadIdx.x == 0) red[0] = 0ull;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
      atomicMax(&red[0], mbits);
      wred[threadIdx.x >> 5] = wabs;
    }
    __syncthreads();
    double wsum_p = 0.0;
#pragma unroll
    for (int i = 0; i < kNuThreads / 32; ++i) wsum_p += wred[i];
    const double wbound = wsum_p * (1.0 + (double)len * 0x1p-52);
    if (threadIdx.x == 0) wsum[piece] = wbound;
    int ebound = 0;
    if (wbound > 0.0) frexp(wbound, &ebound);  // wbound < 2^ebound
    // a NaN or infinite weight makes every sum of the piece NaN, as the direct sums would
    const double fx_step = red[0] >= 0x7ff0000000000000ull ? __longlong_as_double(0x7ff8000000000000ll)
                                                             : ldexp(1.0, ebound - 46);
    const double fx_scale = ldexp(1.0, 46 - ebound);
    for (int kp = 0; kp < 4; kp += KP) {
      for (int i = threadIdx.x; i < NSEQ * seq_stride; i += blockDim.x) zs[i] = make_double2(0.0, 0.0);
      __syncthreads();
      {
        // Points in record order, lane l of round r taking point 32 r + l.  (An order that
        // starts the lanes of a warp on 32 different banks removed 90 % of the reductions'
        // bank conflicts but was measured no faster.)  The next round's record is loaded
        // while the current point is spread.
        const int rounds = (len + 31) >> 5;
        int r = warp;
        double2 nx0 = make_double2(0.0, 0.0), nx1 = make_double2(0.0, 0.0);
        if (r < rounds && 32 * r + lane < len) {
          const double2* rec = reinterpret_cast<const double2*>(rec0 + (size_t)kRec * (32 * r + lane));
          nx0 = rec[0];
          nx1 = rec[1];
        }
        for (; r < rounds; r += nwarps) {
          const int pnt = 32 * r + lane;
          const double phi = nx0.x;  // in [0, 2 pi): the sort's azimuth record
          const double2 r1 = nx1;    // (w, t)
          const int pn = pnt + 32 * nwarps;
          if (pn < len) {
            const double2* rec = reinterpret_cast<const double2*>(rec0 + (size_t)kRec * pn);
            nx0 = rec[0];
            nx1 = rec[1];
          }
          if (pnt >= len) continue;
          const double u = phi * u_per_rad;
          const double fl = floor(u);
          const double sv = 2.0 * (u - fl) - 1.0;
          const int cb = (int)fl - kEsW / 2 + 1;
          double h[4];
          hermite(r1.y, r1.x, h);
          // the pass's weights in fixed-point units: sequence q holds k = kp + 2q, kp + 2q + 1
          double ga[NSEQ], gb[NSEQ];
#pragma unroll
          for (int sq = 0; sq < NSEQ; ++sq) {
            const bool lo = kp + 2 * sq == 0;
            ga[sq] = (lo ? h[0] : h[2]) * fx_scale;
            gb[sq] = (lo ? h[1] : h[3]) * fx_scale;
          }
          // kernel values six at a time (six independent Horner chains; a rolled loop keeps the
          // live registers within the 128 of a 512-thread CTA)
#pragma unroll 1
          for (int i0 = 0; i0 < kEsW; i0 += 6) {
            double ker[6];
#pragma unroll
            for (int i = 0; i < 6; ++i) {
              double acc = es.c[i0 + i][kEsDeg];
#pragma unroll
              for (int d = kEsDeg - 1; d >= 0; --d) acc = fma(acc, sv, es.c[i0 + i][d]);
              ker[i] = acc;
            }
#pragma unroll
            for (int i = 0; i < 6; ++i) {
              const int cell = (cb + i0 + i) & (n - 1);
              const int wo = 544 * (cell >> 7) + (cell & 127);
#pragma unroll
              for (int sq = 0; sq < NSEQ; ++sq) {
                unsigned* z = zw + 4 * sq * seq_stride + wo;
                // X = rint(g ker) by one FMA into the 1.5 2^52 binade (one rounding); its low
                // 16 bits and X >> 16 straight from the two words of the result
                const double da = fma(ga[sq], ker[i], 6755399441055744.0);
                const double db = fma(gb[sq], ker[i], 6755399441055744.0);
                const unsigned la = (unsigned)__double2loint(da), lb = (unsigned)__double2loint(db);
                const unsigned ha = (unsigned)(__double2hiint(da) - 0x43380000);
                const unsigned hb = (unsigned)(__double2hiint(db) - 0x43380000);
                atomicAdd(z, la & 0xffffu);
                atomicAdd(z + 128, __funnelshift_r(la, ha, 16));
                atomicAdd(z + 256, lb & 0xffffu);
                atomicAdd(z + 384, __funnelshift_r(lb, hb, 16));
              }
            }
          }
        }
        __syncthreads();
      }
      // planes -> FP64 complex slots, in place, 2048 cells (16 whole groups) at a time:
      // every thread reads four cells' words, then all write their padded slots
      for (int e0 = 0; e0 < NSEQ * n; e0 += 4 * kNuThreads) {
        unsigned v[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int e = e0 + threadIdx.x + kNuThreads * i;
          if (e < NSEQ * n) {
            const int sq = e >> logn, c = e & (n - 1);
            const unsigned* w = zw + 4 * sq * seq_stride + 544 * (c >> 7) + (c & 127);
            v[i][0] = w[0];
            v[i][1] = w[128];
            v[i][2] = w[256];
            v[i][3] = w[384];
          }
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int e = e0 + threadIdx.x + kNuThreads * i;
          if (e < NSEQ * n) {
            const int sq = e >> logn, c = e & (n - 1);
            zs[sq * seq_stride + padi(c)] = make_double2(from_parts(v[i][1], v[i][0]), from_parts(v[i][3], v[i][2]));
          }
        }
        __syncthreads();
      }
      fft_all<NSEQ>(zs, seq_stride, logn, tws);
      // the next piece's first four weights per thread, in flight during the extraction
      const bool last_pass = kp + KP >= 4;
      const double* nrec = nullptr;
      int nlen = 0;
      double nq[4] = {0.0, 0.0, 0.0, 0.0};
      if (last_pass && nxt < npieces) {
        nrec = pay + (size_t)kRec * piece_start[nxt];
        nlen = piece_len[nxt];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int p = threadIdx.x + u * (int)blockDim.x;
          if (p < nlen) nq[u] = fabs(nrec[(size_t)kRec * p + 2]);
        }
      }
      // v_k0 = (Z[m] + conj Z[-m]) / 2, v_k1 = (Z[m] - conj Z[-m]) / 2i, each over Psi(m)
      for (int m = threadIdx.x; m < Nl; m += blockDim.x) {
        const int pm = padi(fft_pos(m, logn)), pn = padi(fft_pos((n - m) & (n - 1), logn));
        const double di = 0.5 * fx_step * dinvs[m];
#pragma unroll
        for (int sq = 0; sq < NSEQ; ++sq) {
          const double2 a = zs[sq * seq_stride + pm], b = zs[sq * seq_stride + pn];
          const int k0 = kp + 2 * sq;
          double* o = partial + ((size_t)piece * 8 + 2 * k0) * Nl + m;
          o[0] = (a.x + b.x) * di;
          o[(size_t)Nl] = (a.y - b.y) * di;
          o[(size_t)2 * Nl] = (a.y + b.y) * di;
          o[(size_t)3 * Nl] = (b.x - a.x) * di;
        }
      }
      __syncthreads();
      if (last_pass) {
        wabs_n = (nq[0] + nq[1]) + (nq[2] + nq[3]);
        mbits_n = max(max((unsigned long long)__double_as_longlong(nq[0]), (unsigned long long)__double_as_longlong(nq[1])),
                      max((unsigned long long)__double_as_longlong(nq[2]), (unsigned long long)__double_as_longlong(nq[3])));
        if (nrec) bound_part(nrec, nlen, threadIdx.x + 4 * (int)blockDim.x, wabs_n, mbits_n);
      }
    }
  }
}

}  // namespace

// ---- host: kernel polynomials and the deconvolution factors ----------------------------

namespace {

double es_kernel(double x) {
  const double z = 2.0 * x / kEsW;
  if (!(std::fabs(z) < 1.0)) return 0.0;
  return std::exp(kEsBeta * (std::sqrt(1.0 - z * z) - 1.0));
}

// Chebyshev interpolation of psi(f + W/2 - 1 - i) at kEsDeg + 1 nodes in s = 2f - 1,
// converted to monomial coefficients in s.
EsPoly make_es_poly() {
  EsPoly P{};
  constexpr int np = kEsDeg + 1;
  const double pi = 3.14159265358979323846;
  for (int i = 0; i < kEsW; ++i) {
    double y[np], s[np];
    for (int j = 0; j < np; ++j) {
      s[j] = std::cos(pi * (j + 0.5) / np);
      y[j] = es_kernel((s[j] + 1.0) / 2.0 + kEsW / 2 - 1 - i);
    }
    double a[np];  // Chebyshev coefficients
    for (int k = 0; k < np; ++k) {
      double acc = 0.0;
      for (int j = 0; j < np; ++j) acc += y[j] * std::cos(pi * k * (j + 0.5) / np);
      a[k] = acc * (k == 0 ? 1.0 : 2.0) / np;
    }
    // sum_k a_k T_k(s) in monomials: T_(k+1) = 2 s T_k - T_(k-1)
    std::vector<double> tkm(np, 0.0), tk(np, 0.0), tkp(np, 0.0);
    tkm[0] = 1.0;  // T_0
    tk[1] = 1.0;   // T_1
    for (int d = 0; d < np; ++d) P.c[i][d] = a[0] * tkm[d] + (np > 1 ? a[1] * tk[d] : 0.0);
    for (int k = 1; k + 1 < np; ++k) {
      for (int d = 0; d < np; ++d) tkp[d] = (d > 0 ? 2.0 * tk[d - 1] : 0.0) - tkm[d];
      for (int d = 0; d < np; ++d) P.c[i][d] += a[k + 1] * tkp[d];
      tkm.swap(tk);
      tk.swap(tkp);
    }
  }
  return P;
}

// Gauss-Legendre nodes and weights on [-1, 1] (Newton iteration on P_q from the
// Chebyshev-like initial guesses).
void gauss_legendre(int q, std::vector<double>& x, std::vector<double>& w) {
  const double pi = 3.14159265358979323846;
  x.assign(q, 0.0);
  w.assign(q, 0.0);
  for (int i = 0; i < (q + 1) / 2; ++i) {
    double z = std::cos(pi * (i + 0.75) / (q + 0.5)), dp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= q; ++k) {
        const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      if (q == 1) p0 = 1.0;
      dp = q * (z * p1 - p0) / (z * z - 1.0);
      const double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    x[i] = -z;
    x[q - 1 - i] = z;
    w[i] = w[q - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}

}  // namespace

int nufft_logn(int Nl) {
  int lg = 0;  // n = 4 * 2^ceil(log2 Nl), at least 128 (one 128-cell spread group)
  while ((1 << lg) < Nl) ++lg;
  lg += 2;
  return lg < 7 ? 7 : lg;
}

const EsPoly& es_poly() {
  static const EsPoly P = make_es_poly();
  return P;
}

// 1 / Psi(m), m < Nl, and the twiddles e^{2 pi i i / n}, i < n, for a plan.
void nufft_host_tables(int Nl, int logn, std::vector<double>& dinv, std::vector<double>& tw) {
  const int n = 1 << logn;
  const double pi = 3.14159265358979323846;
  std::vector<double> gx, gw;
  gauss_legendre(96, gx, gw);
  dinv.assign(Nl, 0.0);
  for (int m = 0; m < Nl; ++m) {
    double acc = 0.0;
    for (size_t i = 0; i < gx.size(); ++i) {
      const double x = gx[i] * (kEsW / 2.0);
      acc += gw[i] * es_kernel(x) * std::cos(2.0 * pi * m * x / n);
    }
    dinv[m] = 1.0 / (acc * (kEsW / 2.0));
  }
  tw.assign(2 * (size_t)n, 0.0);
  for (int i = 0; i < n; ++i) {
    tw[2 * i] = std::cos(2.0 * pi * i / n);
    tw[2 * i + 1] = std::sin(2.0 * pi * i / n);
  }
}

int launch_bin_sums_nufft(const Geometry& g, const Workspace& ws, int logn, const double* dinv, const double* tw,
                          cudaStream_t s) {
  const int kp = logn <= 12 ? 4 : 2;
  const size_t smem = nufft_smem_bytes(logn, kp / 2);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int64_t grid = ws.pmax < sms ? ws.pmax : sms;
  if (grid < 1) grid = 1;
  auto go = [&](auto kern) -> int {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return set_cuda_error(e, "nufft attributes", __FILE__, __LINE__);
    kern<<<(unsigned)grid, kNuThreads, smem, s>>>(g.Nl, logn, ws.pay, ws.npieces, ws.pmax, ws.piece_start,
                                                  ws.piece_len, dinv, reinterpret_cast<const double2*>(tw),
                                                  es_poly(), ws.partial, ws.wsum);
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_cuda_error(e, "nufft launch", __FILE__, __LINE__);
    count_launches(1);
    return DSHT_OK;
  };
  if (logn > 13) return set_error(DSHT_ERR_INVALID, "NUFFT bin sums support Nl <= 2048 (Nl=%d)", g.Nl);
  return kp == 4 ? go(nufft_sums_kernel<4>) : go(nufft_sums_kernel<2>);
}

}  // namespace dsht

extern "C" int dsht_test_nufft_tables(int Nl, int* logn, double* poly, double* dinv) {
  if (Nl < 1 || Nl > 2048 || !logn || !poly || !dinv)
    return dsht::set_error(DSHT_ERR_INVALID, "invalid arguments");
  *logn = dsht::nufft_logn(Nl);
  const dsht::EsPoly& P = dsht::es_poly();
  for (int i = 0; i < dsht::kEsW; ++i)
    for (int d = 0; d <= dsht::kEsDeg; ++d) poly[i * (dsht::kEsDeg + 1) + d] = P.c[i][d];
  std::vector<double> dv, tw;
  dsht::nufft_host_tables(Nl, *logn, dv, tw);
  for (int m = 0; m < Nl; ++m) dinv[m] = dv[m];
  return DSHT_OK;
}
