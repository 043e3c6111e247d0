// FP64 contraction of the stored tables with the folded node sums: a per-m GEMV.
//
//   alm_equ[lm] = sum_j Yv[lm,j] A_q[m,j] + Yd[lm,j] B_q[m,j],  q = equ even/odd by (l-m)%2
//   alm_pol[lm] = same with the polar q                     (sht/sht.py:266-279)
//
// A CTA owns 16 consecutive rows l of one m and streams its table rows once; the fold
// values of the m (both parities, both sets) are staged per node tile in shared memory
// and reused by every row.  Each warp owns two rows of equal parity, so every fold value
// read from shared memory feeds two rows.  Tiles without points are skipped.  HBM bound:
// 16 B of table per (l, m, j).
#include "dsht_internal.cuh"

namespace dsht {
namespace {

constexpr int kContractThreads = 256;
constexpr int kRowsPerCta = 16;
constexpr int kTile = 128;  // nodes per shared-memory tile

__global__ void __launch_bounds__(kContractThreads)
contract_fp64_kernel(int Nl, int Nx, const double* __restrict__ Yv, const double* __restrict__ Yd,
                     const double* __restrict__ fold, const uint8_t* __restrict__ live, int ntile,
                     double* __restrict__ alm_equ, double* __restrict__ alm_pol) {
  __shared__ double4 sF[4][kTile];
  const int m = blockIdx.y;
  const int l0 = m + blockIdx.x * kRowsPerCta;
  if (l0 >= Nl) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int par = warp & 1;
  const int ra = par + 4 * (warp >> 1);     // row offsets of this warp: ra, ra + 2
  const int la = l0 + ra, lb = l0 + ra + 2;
  const bool va = la < Nl, vb = lb < Nl;
  const double* yva = Yv + hp_index(va ? la : m, m, Nl) * Nx;
  const double* yda = Yd + hp_index(va ? la : m, m, Nl) * Nx;
  const double* yvb = Yv + hp_index(vb ? lb : m, m, Nl) * Nx;
  const double* ydb = Yd + hp_index(vb ? lb : m, m, Nl) * Nx;
  const double4* F = reinterpret_cast<const double4*>(fold) + (size_t)m * 4 * Nx;

  double ea_r = 0, ea_i = 0, pa_r = 0, pa_i = 0;  // row a: equatorial, polar
  double eb_r = 0, eb_i = 0, pb_r = 0, pb_i = 0;  // row b
  for (int t = 0; t < ntile; ++t) {
    if (!live[t] && !live[ntile + t]) continue;
    const int j0 = t * kTile;
    __syncthreads();
    for (int e = threadIdx.x; e < 4 * kTile; e += blockDim.x) {
      const int q = e / kTile, jj = e % kTile;
      sF[q][jj] = (j0 + jj < Nx) ? F[(size_t)q * Nx + j0 + jj] : make_double4(0, 0, 0, 0);
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kTile / 32; ++u) {
      const int jj = lane + 32 * u;
      const int j = j0 + jj;
      if (j < Nx) {
        const double4 fe = sF[par][jj];
        const double4 fp = sF[2 + par][jj];
        if (va) {
          const double v = yva[j], d = yda[j];
          ea_r = fma(v, fe.x, fma(d, fe.z, ea_r));
          ea_i = fma(v, fe.y, fma(d, fe.w, ea_i));
          pa_r = fma(v, fp.x, fma(d, fp.z, pa_r));
          pa_i = fma(v, fp.y, fma(d, fp.w, pa_i));
        }
        if (vb) {
          const double v = yvb[j], d = ydb[j];
          eb_r = fma(v, fe.x, fma(d, fe.z, eb_r));
          eb_i = fma(v, fe.y, fma(d, fe.w, eb_i));
          pb_r = fma(v, fp.x, fma(d, fp.z, pb_r));
          pb_i = fma(v, fp.y, fma(d, fp.w, pb_i));
        }
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ea_r += __shfl_xor_sync(0xffffffffu, ea_r, o);
    ea_i += __shfl_xor_sync(0xffffffffu, ea_i, o);
    pa_r += __shfl_xor_sync(0xffffffffu, pa_r, o);
    pa_i += __shfl_xor_sync(0xffffffffu, pa_i, o);
    eb_r += __shfl_xor_sync(0xffffffffu, eb_r, o);
    eb_i += __shfl_xor_sync(0xffffffffu, eb_i, o);
    pb_r += __shfl_xor_sync(0xffffffffu, pb_r, o);
    pb_i += __shfl_xor_sync(0xffffffffu, pb_i, o);
  }
  if (lane == 0) {
    if (va) {
      const int64_t i = hp_index(la, m, Nl);
      alm_equ[2 * i] = ea_r;
      alm_equ[2 * i + 1] = ea_i;
      alm_pol[2 * i] = pa_r;
      alm_pol[2 * i + 1] = pa_i;
    }
    if (vb) {
      const int64_t i = hp_index(lb, m, Nl);
      alm_equ[2 * i] = eb_r;
      alm_equ[2 * i + 1] = eb_i;
      alm_pol[2 * i] = pb_r;
      alm_pol[2 * i + 1] = pb_i;
    }
  }
}

}  // namespace

int contract_tile() { return kTile; }

void launch_contract_fp64(const Geometry& g, const double* Yv, const double* Yd, const Workspace& ws,
                          cudaStream_t s) {
  const int ntile = (g.Nx + kTile - 1) / kTile;
  dim3 grid((g.Nl + kRowsPerCta - 1) / kRowsPerCta, g.Nl);
  contract_fp64_kernel<<<grid, kContractThreads, 0, s>>>(g.Nl, g.Nx, Yv, Yd, ws.fold, ws.tile_live, ntile,
                                                         ws.alm_equ, ws.alm_pol);
  count_launches(1);
}

}  // namespace dsht
