// Heavy nodes of the FP32-table contraction, done in FP64 with the table values
// regenerated on the fly.
//
// The FP32-table level (DSHT_PREC_MIXED) rounds the table entries, the folded node sums
// and the in-tile partial sums to float: about 2^-24 relative per node contribution.  Spread
// over many nodes these errors average out (4.6e-8 x max|alm| at 1e7 points over 1600
// nodes), but when a large share of the weight sits at one node its rounding errors do not,
// and the result can reach a few 1e-7 x max|alm|.  So, per transform:
//
//   1. piecemax_kernel (points.cu) also writes each bin piece's sum of |w|;
//   2. heavy_select_kernel (one block) sums them per node j of each half h (equatorial /
//      rotated polar), the node collecting bins j (h_0, h_1 terms) and j - 1 (h_2, h_3),
//      and marks the nodes holding more than 1/kHeavyDiv of the total |w| (fewer than
//      2 kHeavyDiv of them, since every point feeds two nodes), listed in node order;
//   3. the fold writes zeros for the marked nodes into the FP32 fold (fold.cu);
//   4. heavy_otf_kernel writes, for every (l, m), the marked nodes' contribution computed in
//      FP64: fold values re-summed from the per-piece bin sums exactly as fold.cu sums them,
//      and Yv, Yd regenerated by the recurrences of recurrence.cuh -- bitwise the values of
//      the FP64 tables, so no table memory is read;
//   5. the FP32 contraction then adds its (light-node) sums to these instead of storing.
//
// The remaining FP32 error comes from nodes holding at most 1/kHeavyDiv of the weight each:
// its rms is ~2^-24 sqrt(sum_j share_j^2) <= 2^-24 sqrt(2/kHeavyDiv) of the contributions.
// A transform without heavy nodes pays for the |w| sums and one small select launch only.
#include "recurrence.cuh"

namespace dsht {
namespace {

constexpr int kSelectThreads = 1024;

// Sums of |w| per (half, node) and the list of heavy ones, in (half, node) order.
__global__ void __launch_bounds__(kSelectThreads)
heavy_select_kernel(int nbins, int Nx, const int* __restrict__ npieces_p, int64_t pmax,
                    const int* __restrict__ piece_first, const double* __restrict__ wsum,
                    double* __restrict__ nodew, uint8_t* __restrict__ flag, int* __restrict__ list,
                    int* __restrict__ n_out) {
  __shared__ double red[32];
  __shared__ double total_s;
  __shared__ uint32_t warp_tot[32];
  __shared__ uint32_t carry;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t np = min((int64_t)*npieces_p, pmax);
  // total |w| (fixed order: strided per thread, then a tree)
  double t = 0.0;
  for (int64_t pc = tid; pc < np; pc += blockDim.x) t += wsum[pc];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if (lane == 0) red[warp] = t;
  __syncthreads();
  if (warp == 0) {
    double v = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) {
      total_s = v;
      carry = 0;
    }
  }
  __syncthreads();
  const double thr = total_s / (double)kHeavyDiv;
  // |w| per (half h, node j): one warp per entry, lanes over the pieces of its four keys
  const int ne = 2 * Nx;
  for (int e = warp; e < ne; e += blockDim.x >> 5) {
    const int h = e / Nx, j = e - h * Nx;
    double s = 0.0;
    for (int sset = 2 * h; sset < 2 * h + 2; ++sset)
      for (int b = j - 1; b <= j; ++b) {
        if (b < 0 || b >= nbins) continue;
        const int key = sset * nbins + b;
        for (int pc = piece_first[key] + lane; pc < piece_first[key + 1]; pc += 32) s += wsum[pc];
      }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) nodew[e] = s;
  }
  __syncthreads();
  // heavy flags and the ordered list (block-wide exclusive scans over chunks of entries)
  for (int base = 0; base < ne; base += blockDim.x) {
    const int e = base + tid;
    const uint32_t hv = (e < ne && total_s > 0.0 && nodew[e] > thr) ? 1u : 0u;
    uint32_t x = hv;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
      const uint32_t wt = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0u;
      uint32_t sc = wt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, sc, o);
        if (lane >= o) sc += y;
      }
      warp_tot[lane] = sc - wt;
    }
    __syncthreads();
    const uint32_t pos = carry + warp_tot[warp] + x - hv;
    if (e < ne) {
      const bool keep = hv && pos < (uint32_t)kHeavyMax;
      flag[e] = keep ? 1 : 0;
      if (keep) list[pos] = e;
    }
    __syncthreads();
    if (tid == blockDim.x - 1) carry = pos + hv;
    __syncthreads();
  }
  if (tid == 0) *n_out = (int)min(carry, (uint32_t)kHeavyMax);
}

// One warp per m walks l = m .. Nl-1 for 32 heavy nodes at a time (lane = node).
template <typename PT>
__global__ void __launch_bounds__(32)
heavy_otf_kernel(int Nl, int Nx, int nbins, double dx, const int* __restrict__ n_p, const int* __restrict__ list,
                 const int* __restrict__ piece_first, const PT* __restrict__ partial, double* __restrict__ alm_equ,
                 double* __restrict__ alm_pol) {
  const int n = *n_p;
  if (n == 0) return;
  extern __shared__ double smm[];  // [Nl] diagonal factors, then 32 Coef
  Coef* cf = reinterpret_cast<Coef*>(smm + Nl);
  const int m = blockIdx.x, lane = threadIdx.x;
  for (int k = lane + 1; k <= m; k += 32) smm[k] = diag_factor(k);
  __syncwarp();
  for (int c0 = 0; c0 < n; c0 += 32) {
    const int e = c0 + lane;
    const bool active = e < n;
    const int ent = active ? list[e] : 0;
    const int h = ent / Nx, j = ent - h * Nx;
    // FP64 fold values of node j for this m, summed as fold_kernel sums them:
    // set s: A = V0(bin j) + V2(bin j-1), B = dx (V1(bin j) + V3(bin j-1)), V = vr - i vi.
    double A[2][2], B[2][2];  // [set of the half][re, im]
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      double ar = 0.0, ai = 0.0, br = 0.0, bi = 0.0;
      const int sset = 2 * h + q;
      if (active && j < nbins) {
        const int key = sset * nbins + j;
        for (int p = piece_first[key]; p < piece_first[key + 1]; ++p) {
          const PT* v = partial + (size_t)p * 8 * Nl + m;
          ar += v[0];
          ai -= v[(size_t)Nl];
          br += v[(size_t)2 * Nl];
          bi -= v[(size_t)3 * Nl];
        }
      }
      if (active && j >= 1) {
        const int key = sset * nbins + j - 1;
        for (int p = piece_first[key]; p < piece_first[key + 1]; ++p) {
          const PT* v = partial + (size_t)p * 8 * Nl + m;
          ar += v[(size_t)4 * Nl];
          ai -= v[(size_t)5 * Nl];
          br += v[(size_t)6 * Nl];
          bi -= v[(size_t)7 * Nl];
        }
      }
      A[q][0] = ar;
      A[q][1] = ai;
      B[q][0] = dx * br;
      B[q][1] = dx * bi;
    }
    // even rows (l - m even) take A(x >= 0) + A(x < 0), odd rows the difference
    double Fa[2][2], Fb[2][2];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      Fa[0][c] = A[0][c] + A[1][c];
      Fa[1][c] = A[0][c] - A[1][c];
      Fb[0][c] = B[0][c] + B[1][c];
      Fb[1][c] = B[0][c] - B[1][c];
    }
    double x, omx2, sx;
    node_x(j, dx, &x, &omx2, &sx);
    const double ymm = diag_value(m, sx, smm);
    ColumnState st;
    for (int l0 = m; l0 < Nl; l0 += 32) {
      __syncwarp();
      if (l0 + lane < Nl) cf[lane] = make_coef(l0 + lane, m);
      __syncwarp();
      const int lend = min(l0 + 32, Nl);
      for (int l = l0; l < lend; ++l) {
        double y, d;
        const Coef c = cf[l - l0];
        if (l == m) column_first(m, x, omx2, ymm, &st, &y, &d);
        else if (l == m + 1) column_second(m, c, &st, &y, &d);
        else column_step(m, l, c, &st, &y, &d);
        const double yv = __dmul_rn(y, c.nrm), yd = __dmul_rn(d, c.nrm);  // the FP64 table values
        const int par = (l - m) & 1;
        double re = active ? fma(yv, Fa[par][0], yd * Fb[par][0]) : 0.0;
        double im = active ? fma(yv, Fa[par][1], yd * Fb[par][1]) : 0.0;
        double v[4] = {h == 0 ? re : 0.0, h == 0 ? im : 0.0, h == 1 ? re : 0.0, h == 1 ? im : 0.0};
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
        if (lane < 4) {
          const int64_t idx = hp_index(l, m, Nl);
          double* out = (lane < 2 ? alm_equ : alm_pol) + 2 * idx + (lane & 1);
          const double add = v[lane];
          *out = c0 == 0 ? add : *out + add;
        }
      }
    }
  }
}

}  // namespace

void launch_heavy_select(const Geometry& g, const Workspace& ws, int slot, cudaStream_t s) {
  heavy_select_kernel<<<1, kSelectThreads, 0, s>>>(g.nbins, g.Nx, ws.npieces, ws.pmax, ws.piece_first, ws.wsum,
                                                   ws.nodew, ws.heavy_flag + (size_t)slot * 2 * g.Nx,
                                                   ws.heavy_list + (size_t)slot * kHeavyMax, ws.heavy_n + slot);
  count_launches(1);
}

void launch_heavy_otf(const Geometry& g, const Workspace& ws, int slot, double* alm_equ, double* alm_pol,
                      cudaStream_t s) {
  const size_t smem = sizeof(double) * (size_t)g.Nl + sizeof(Coef) * 32;
  const int* n = ws.heavy_n + slot;
  const int* list = ws.heavy_list + (size_t)slot * kHeavyMax;
  if (ws.partial_f32) {
    cudaFuncSetAttribute(heavy_otf_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    heavy_otf_kernel<float><<<g.Nl, 32, smem, s>>>(g.Nl, g.Nx, g.nbins, g.dx, n, list, ws.piece_first,
                                                   reinterpret_cast<const float*>(ws.partial), alm_equ, alm_pol);
  } else {
    cudaFuncSetAttribute(heavy_otf_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    heavy_otf_kernel<double><<<g.Nl, 32, smem, s>>>(g.Nl, g.Nx, g.nbins, g.dx, n, list, ws.piece_first,
                                                    ws.partial, alm_equ, alm_pol);
  }
  count_launches(1);
}

}  // namespace dsht
