// Fold the per-piece bin sums onto the spline nodes and combine the x >= 0 / x < 0 halves.
//
// The contraction of the reference (sht/sht.py:274-277, sht/interp_funcs_py.py:59-60),
//   alm[lm] = sum_b Yv[lm,b] V0[b] + dx Yd[lm,b] V1[b] + Yv[lm,b+1] V2[b] + dx Yd[lm,b+1] V3[b],
// with V = vr - i vi, is linear in the table entries, so each node j collects
//   A[m,j] = V0[m,j] + V2[m,j-1],   B[m,j] = dx (V1[m,j] + V3[m,j-1]).
// The x < 0 half enters with (-1)^(l-m) (sht/sht.py:279); rows with l-m even use
// A+ + A-, odd rows A+ - A-, for the equatorial and the rotated polar sets.
// Output fold[m][q][j] = (A re, A im, B re, B im), q = {equ even, equ odd, pol even, pol odd},
// FP64, for the FP64-table contraction (the tensor-core contraction takes its fold straight
// as digits, digits.cu).  Partial sums are FP64 (plain path) or FP32 (tensor-core bin sums);
// they are added in FP64.
#include "dsht_internal.cuh"

namespace dsht {
namespace {

constexpr int kFoldThreads = 128;

template <typename T>
__global__ void __launch_bounds__(kFoldThreads)
fold_kernel(int Nl, int Nx, int nbins, double dx, const int* __restrict__ piece_first,
            const T* __restrict__ partial, double4* __restrict__ fold) {
  const int j = blockIdx.x;
  const int m = blockIdx.y * blockDim.x + threadIdx.x;
  if (m >= Nl) return;
  double A[4][2], B[4][2];
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    double ar = 0.0, ai = 0.0, br = 0.0, bi = 0.0;
    if (j < nbins) {  // bin j: its left node carries V0, V1
      const int key = s * nbins + j;
      for (int p = piece_first[key]; p < piece_first[key + 1]; ++p) {
        const T* v = partial + (size_t)p * 8 * Nl + m;
        ar += v[0];
        ai -= v[(size_t)Nl];
        br += v[(size_t)2 * Nl];
        bi -= v[(size_t)3 * Nl];
      }
    }
    if (j >= 1) {  // bin j-1: its right node carries V2, V3
      const int key = s * nbins + j - 1;
      for (int p = piece_first[key]; p < piece_first[key + 1]; ++p) {
        const T* v = partial + (size_t)p * 8 * Nl + m;
        ar += v[(size_t)4 * Nl];
        ai -= v[(size_t)5 * Nl];
        br += v[(size_t)6 * Nl];
        bi -= v[(size_t)7 * Nl];
      }
    }
    A[s][0] = ar;
    A[s][1] = ai;
    B[s][0] = dx * br;
    B[s][1] = dx * bi;
  }
  double4* out = fold + ((size_t)m * 4) * Nx + j;
  out[0] = make_double4(A[0][0] + A[1][0], A[0][1] + A[1][1], B[0][0] + B[1][0], B[0][1] + B[1][1]);
  out[(size_t)Nx] = make_double4(A[0][0] - A[1][0], A[0][1] - A[1][1], B[0][0] - B[1][0], B[0][1] - B[1][1]);
  out[(size_t)2 * Nx] = make_double4(A[2][0] + A[3][0], A[2][1] + A[3][1], B[2][0] + B[3][0], B[2][1] + B[3][1]);
  out[(size_t)3 * Nx] = make_double4(A[2][0] - A[3][0], A[2][1] - A[3][1], B[2][0] - B[3][0], B[2][1] - B[3][1]);
}

// tile_live[h][t] = 1 when any point of the equatorial (h = 0) or polar (h = 1) sets
// touches a node of the tile t of kContractTile nodes.
__global__ void tile_live_kernel(int nbins, int ntile, int tile, const uint32_t* __restrict__ count,
                                 uint8_t* __restrict__ live, int accumulate) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntile) return;
  for (int h = 0; h < 2; ++h) {
    uint8_t any = 0;
    const int j0 = t * tile - 1, j1 = t * tile + tile;  // bins feeding nodes [t*tile, t*tile+tile)
    for (int s = 2 * h; s < 2 * h + 2; ++s)
      for (int j = max(j0, 0); j < min(j1, nbins); ++j) any |= (count[s * nbins + j] != 0);
    if (!accumulate) live[h * ntile + t] = any;
    else if (any) live[h * ntile + t] = 1;
  }
}

}  // namespace

int contract_tile();

void launch_fold(const Geometry& g, const Workspace& ws, cudaStream_t s) {
  dim3 grid(g.Nx, (g.Nl + kFoldThreads - 1) / kFoldThreads);
  double4* f64 = reinterpret_cast<double4*>(ws.fold);
  if (ws.partial_f32)
    fold_kernel<float><<<grid, kFoldThreads, 0, s>>>(g.Nl, g.Nx, g.nbins, g.dx, ws.piece_first,
                                                     reinterpret_cast<const float*>(ws.partial), f64);
  else
    fold_kernel<double><<<grid, kFoldThreads, 0, s>>>(g.Nl, g.Nx, g.nbins, g.dx, ws.piece_first, ws.partial, f64);
  count_launches(1);
  const int tile = contract_tile();
  const int ntile = (g.Nx + tile - 1) / tile;
  tile_live_kernel<<<(ntile + 127) / 128, 128, 0, s>>>(g.nbins, ntile, tile, ws.count, ws.tile_live, 0);
  count_launches(1);
  const int ntile2 = (g.Nx + 255) / 256;
  tile_live_kernel<<<(ntile2 + 127) / 128, 128, 0, s>>>(g.nbins, ntile2, 256, ws.count, ws.tile_live2, 0);
  count_launches(1);
}

}  // namespace dsht
