// FP64 per-bin sums ("v's") for every m: the plain-FP64 scatter.
//
//   v[k][re][m] = sum_{p in piece} g_k(p) cos(m phi_p),  v[k][im][m] = ... sin(m phi_p)
//
// (sht/shared_interp_funcs.py:88-105, sht/interp_funcs_py.py:16-35, with the points
// already sorted by bin).  One CTA per piece (<= piece_max points of one bin); each
// thread owns 8 consecutive m and keeps their 4 x 2 sums in registers, so there are no
// atomics: the piece's partial sums are written once, coalesced.  cos/sin(m phi) come
// from an angle-addition recurrence in registers: per point the thread starts from
// e^{i m0 phi} = T2[t/16] * T1[t%16] (two small power tables per point staged in shared
// memory, built from cos/sin of phi by squaring) and steps by e^{i phi} 7 times.
// Compute bound on the FP64 pipe:
// 12 DFMA per (point, m).
#include "dsht_internal.cuh"

namespace dsht {
namespace {

constexpr int kMPerThread = 8;
constexpr int kMaxThreads = 128;                    // 1024 m per CTA
constexpr int kMBlock = kMPerThread * kMaxThreads;  // m covered by one CTA (blockIdx.y)

struct __align__(16) cplx {
  double re, im;
};

__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}

template <int TP>
__global__ void __launch_bounds__(kMaxThreads, 3)
bin_sums_fp64_kernel(int Nl, int64_t N, const double* __restrict__ pay, const int* __restrict__ npieces_p,
                     int64_t pmax, const int64_t* __restrict__ piece_start, const int* __restrict__ piece_len,
                     double* __restrict__ partial) {
  __shared__ cplx sT1[TP][16];
  __shared__ cplx sT2[TP][8];
  __shared__ cplx sE1[TP];
  __shared__ double sG[TP][4];

  const int npieces = (int)min((int64_t)*npieces_p, pmax);
  const int tid = threadIdx.x;
  const int mblk = blockIdx.y;
  const int m0 = mblk * kMBlock + kMPerThread * tid;
  for (int piece = blockIdx.x; piece < npieces; piece += gridDim.x) {
    const int64_t start = piece_start[piece];
    const int len = piece_len[piece];
    double ar[kMPerThread][4], ai[kMPerThread][4];
#pragma unroll
    for (int r = 0; r < kMPerThread; ++r)
#pragma unroll
      for (int k = 0; k < 4; ++k) ar[r][k] = ai[r][k] = 0.0;

    for (int base = 0; base < len; base += TP) {
      const int np = min(TP, len - base);
      __syncthreads();
      // Two threads per point build its tables.
      {
        const int p = tid >> 1, half = tid & 1;
        if (p < np) {
          const int64_t i = start + base + p;
          const double* rp = pay + kRec * i;
          const cplx e1 = {rp[0], rp[1]};
          cplx e8 = cmul(e1, e1);
          e8 = cmul(e8, e8);
          e8 = cmul(e8, e8);
          if (half == 0) {
            cplx z = {1.0, 0.0};
            sT1[p][0] = z;
#pragma unroll
            for (int a = 1; a < 16; ++a) {
              z = cmul(z, e8);
              sT1[p][a] = z;
            }
          } else {
            cplx e128 = e8;
#pragma unroll
            for (int k = 0; k < 4; ++k) e128 = cmul(e128, e128);
            cplx z = {1.0, 0.0};
            for (int k = 0; k < mblk * 8; ++k) z = cmul(z, e128);  // e^{i 1024 mblk phi}
            sT2[p][0] = z;
#pragma unroll
            for (int b = 1; b < 8; ++b) {
              z = cmul(z, e128);
              sT2[p][b] = z;
            }
            sE1[p] = e1;
            double h[4];
            hermite(rp[3], rp[2], h);
            sG[p][0] = h[0];
            sG[p][1] = h[1];
            sG[p][2] = h[2];
            sG[p][3] = h[3];
          }
        }
      }
      __syncthreads();
      const int a = tid & 15, b = tid >> 4;
      for (int p = 0; p < np; ++p) {
        cplx z = cmul(sT2[p][b], sT1[p][a]);
        const cplx e1 = sE1[p];
        const double q0 = sG[p][0], q1 = sG[p][1], q2 = sG[p][2], q3 = sG[p][3];
#pragma unroll
        for (int r = 0; r < kMPerThread; ++r) {
          ar[r][0] = fma(q0, z.re, ar[r][0]);
          ai[r][0] = fma(q0, z.im, ai[r][0]);
          ar[r][1] = fma(q1, z.re, ar[r][1]);
          ai[r][1] = fma(q1, z.im, ai[r][1]);
          ar[r][2] = fma(q2, z.re, ar[r][2]);
          ai[r][2] = fma(q2, z.im, ai[r][2]);
          ar[r][3] = fma(q3, z.re, ar[r][3]);
          ai[r][3] = fma(q3, z.im, ai[r][3]);
          if (r + 1 < kMPerThread) z = cmul(z, e1);
        }
      }
    }
    // partial[piece][k*2 + ri][m]
    double* out = partial + (size_t)piece * 8 * Nl;
    if (m0 + kMPerThread <= Nl && (Nl % 2 == 0)) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        double2* pr = reinterpret_cast<double2*>(out + (size_t)(2 * k) * Nl + m0);
        double2* pi = reinterpret_cast<double2*>(out + (size_t)(2 * k + 1) * Nl + m0);
#pragma unroll
        for (int r = 0; r < kMPerThread; r += 2) {
          pr[r / 2] = make_double2(ar[r][k], ar[r + 1][k]);
          pi[r / 2] = make_double2(ai[r][k], ai[r + 1][k]);
        }
      }
    } else {
#pragma unroll
      for (int r = 0; r < kMPerThread; ++r) {
        const int m = m0 + r;
        if (m < Nl) {
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            out[(size_t)(2 * k) * Nl + m] = ar[r][k];
            out[(size_t)(2 * k + 1) * Nl + m] = ai[r][k];
          }
        }
      }
    }
  }
}

}  // namespace

void launch_bin_sums_fp64(const Geometry& g, const Workspace& ws, cudaStream_t s) {
  const int mblocks = (g.Nl + kMBlock - 1) / kMBlock;
  int threads = (g.Nl + kMPerThread - 1) / kMPerThread;
  if (threads > kMaxThreads) threads = kMaxThreads;
  threads = ((threads + 31) / 32) * 32;
  int64_t grid = ws.pmax;
  if (grid > 65535 * 8) grid = 65535 * 8;
  if (grid < 1) grid = 1;
  dim3 gd((unsigned)grid, mblocks);
  if (threads >= 128) {
    bin_sums_fp64_kernel<64><<<gd, threads, 0, s>>>(g.Nl, ws.npts, ws.pay, ws.npieces, ws.pmax, ws.piece_start,
                                                    ws.piece_len, ws.partial);
    count_launches(1);
  } else {
    bin_sums_fp64_kernel<16><<<gd, threads, 0, s>>>(g.Nl, ws.npts, ws.pay, ws.npieces, ws.pmax, ws.piece_start,
                                                    ws.piece_len, ws.partial);
    count_launches(1);
  }
}

}  // namespace dsht
