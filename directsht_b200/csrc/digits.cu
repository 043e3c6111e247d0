// Fixed-point digit tables and folds for the tensor-core contraction (contract_tc.cu).
//
// The contraction alm[lm] = sum_j Yv[lm,j] A[m,j] + Yd[lm,j] B[m,j] (sht/sht.py:266-277,
// sht/interp_funcs_py.py:46-60) is a dot product over K = 2 Nx entries per row:
//   T[r, k] = Yv[r, k] (k < Nx),  dx Yd[r, k - Nx] (Nx <= k < 2 Nx),
//   F[k, c] = A_c[k]   (k < Nx),  B_c[k - Nx] / dx.
// Both sides are stored as 31-bit fixed point with one power-of-two scale per table row
// (2^er > 1.01 max_k |T[r, k]|) and per fold column (2^ec > 1.01 x the largest node weight,
// which bounds |A| and |B/dx| for every m): X = rint(T 2^(31 - er)), |X| < 2^31 - 2^24.
// X is written as four balanced base-256 digits, X = d0 2^24 + d1 2^16 + d2 2^8 + d3 with
// every digit a signed byte: the bytes of (X + 0x808080) ^ 0x808080.  Digit d of every
// entry forms plane d (int8, K-major rows of Kp bytes, Kp = 2 Nx rounded up to 64).
//
// Table rows are stored grouped by the parity of l - m: for each m the rows l = m, m+2, ...
// (n_e(m) = (Nl - m + 1)/2 of them) and then l = m+1, m+3, ... -- the even and odd rows
// contract with different folds (the x < 0 half enters with (-1)^(l-m), sht/sht.py:279).
// Fold digits of a pass of G maps: plane-major [m][parity][digit][4 G columns][Kp] with
// column 4 g + 2 h + ri = (map g, half h = equatorial / rotated polar, re | im).
//
// Quantisation error of an entry: <= 2^-32 of its row's (column's) scale; a contraction sum
// errs by at most about 2^-30 (max|T| sum|F| + max|F| sum|T|), far less for spread sets.
#include "recurrence.cuh"

namespace dsht {
namespace {

constexpr int kFoldNodes = 16;  // nodes per fold_digits block (32 m x 16 nodes, 512 threads)
constexpr int kStageRow = kFoldNodes + 4;  // bytes per staging row (a 4-byte pad: lanes store to
                                           // rows 20 bytes apart, i.e. 32 different banks)
constexpr double kScaleMargin = 1.01;  // scale > 1.01 x bound: |X| < 2^31 / 1.01 < 2^31 - 2^24

// Smallest e with kScaleMargin * v <= 2^e (v >= 0; 0 for v = 0).
__device__ __forceinline__ int scale_exp(double v) {
  if (!(v > 0.0) || !isfinite(v)) return 0;
  int e;
  frexp(v * kScaleMargin, &e);  // v * margin = f 2^e with f in [0.5, 1)
  return e;
}

// The four signed digit bytes of rint(v 2^sh) packed little-endian: byte i = digit 3 - i.
__device__ __forceinline__ uint32_t digit_word(double v, int sh) {
  const long long X = __double2ll_rn(ldexp(v, sh));
  return (uint32_t)((int)X + 0x808080) ^ 0x808080u;
}

// The same for v 2^sh given as the product (|v 2^sh| < 2^31): one DADD puts it into the
// binade of 1.5 2^52, whose low word is then the rounded integer.
__device__ __forceinline__ uint32_t digit_word_scaled(double vs) {
  const int X = __double2loint(vs + 6755399441055744.0);
  return (uint32_t)(X + 0x808080) ^ 0x808080u;
}

// Grouped row of Healpy row (l, m).
__device__ __forceinline__ int64_t grouped_row(int l, int m, int Nl) {
  const int64_t base = hp_index(m, m, Nl);
  const int k = l - m;
  const int ne = (Nl - m + 1) / 2;
  return base + ((k & 1) ? ne + (k >> 1) : (k >> 1));
}

// Row exponents of the FP64 tables rows [row0, row0 + nrows) (Healpy order, row r at
// Y + (r - row0) * Nx): one warp per row.
__global__ void table_rowexp_kernel(int Nl, int Nx, double dx, int64_t row0, int64_t nrows, const double* __restrict__ Yv,
                                    const double* __restrict__ Yd, int16_t* __restrict__ rexp) {
  const int lane = threadIdx.x & 31;
  const int64_t wstride = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < nrows; i += wstride) {
    const double* v = Yv + i * Nx;
    const double* d = Yd + i * Nx;
    double mx = 0.0;
    for (int j = lane; j < Nx; j += 32) mx = fmax(mx, fmax(fabs(v[j]), fabs(dx * d[j])));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) {
      // Healpy row r = row0 + i -> (l, m)
      const int64_t r = row0 + i;
      int m = (int)((2.0 * Nl + 1.0 - sqrt((2.0 * Nl + 1.0) * (2.0 * Nl + 1.0) - 8.0 * (double)r)) / 2.0);
      if (m < 0) m = 0;
      while (m > 0 && hp_index(m, m, Nl) > r) --m;
      while (m + 1 < Nl && hp_index(m + 1, m + 1, Nl) <= r) ++m;
      const int l = (int)(r - hp_index(m, m, Nl)) + m;
      rexp[grouped_row(l, m, Nl)] = (int16_t)scale_exp(mx);
    }
  }
}

// Digits of rows [row0, row0 + nrows): one thread per (row, 4 consecutive k).
__global__ void table_digits_kernel(int Nl, int Nx, int Kp, double dx, int64_t row0, int64_t nrows,
                                    const double* __restrict__ Yv, const double* __restrict__ Yd,
                                    const int16_t* __restrict__ rexp, int64_t plane, uint8_t* __restrict__ dig) {
  const int words = Kp / 4;
  const int64_t total = nrows * words;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / words;
    const int k0 = (int)(t - i * words) * 4;
    const int64_t r = row0 + i;
    int m = (int)((2.0 * Nl + 1.0 - sqrt((2.0 * Nl + 1.0) * (2.0 * Nl + 1.0) - 8.0 * (double)r)) / 2.0);
    if (m < 0) m = 0;
    while (m > 0 && hp_index(m, m, Nl) > r) --m;
    while (m + 1 < Nl && hp_index(m + 1, m + 1, Nl) <= r) ++m;
    const int l = (int)(r - hp_index(m, m, Nl)) + m;
    const int64_t g = grouped_row(l, m, Nl);
    const int sh = 31 - rexp[g];
    uint32_t b[4] = {0u, 0u, 0u, 0u};  // plane d: byte e = digit d of entry k0 + e
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int k = k0 + e;
      double v = 0.0;
      if (k < Nx) v = Yv[i * Nx + k];
      else if (k < 2 * Nx) v = dx * Yd[i * Nx + (k - Nx)];
      const uint32_t w = digit_word(v, sh);
#pragma unroll
      for (int d = 0; d < 4; ++d) b[d] |= ((w >> (8 * (3 - d))) & 0xffu) << (8 * e);
    }
#pragma unroll
    for (int d = 0; d < 4; ++d) *reinterpret_cast<uint32_t*>(dig + d * plane + g * Kp + k0) = b[d];
  }
}

// Table values back from the digits (rows in Healpy order r0.. r0 + n, both tables):
// Y = 2^(er - 31) X with X from the four digit bytes.  which = 0: Yv, 1: Yd.
__global__ void table_decode_kernel(int Nl, int Nx, int Kp, double dx, int which, int64_t r0, int64_t n,
                                    const uint8_t* __restrict__ dig, int64_t plane, const int16_t* __restrict__ rexp,
                                    double* __restrict__ out) {
  const int64_t total = n * Nx;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / Nx;
    const int j = (int)(t - i * Nx);
    const int64_t r = r0 + i;
    int m = (int)((2.0 * Nl + 1.0 - sqrt((2.0 * Nl + 1.0) * (2.0 * Nl + 1.0) - 8.0 * (double)r)) / 2.0);
    if (m < 0) m = 0;
    while (m > 0 && hp_index(m, m, Nl) > r) --m;
    while (m + 1 < Nl && hp_index(m + 1, m + 1, Nl) <= r) ++m;
    const int l = (int)(r - hp_index(m, m, Nl)) + m;
    const int64_t g = grouped_row(l, m, Nl);
    const int k = which == 0 ? j : Nx + j;
    long long X = 0;
#pragma unroll
    for (int d = 0; d < 4; ++d) X = X * 256 + (long long)(int8_t)dig[d * plane + g * Kp + k];
    double v = ldexp((double)X, rexp[g] - 31);
    if (which == 1) v /= dx;
    out[t] = v;
  }
}

// Per-map fold scales: the largest |w| sum feeding a node of each half (bins j - 1 and j of
// both sets of the half), which bounds |A| and |B/dx| for every m.
__global__ void __launch_bounds__(256)
fold_scale_kernel(int nbins, int Nx, const int* __restrict__ piece_first, const double* __restrict__ wsum,
                  unsigned long long* __restrict__ cmax) {
  // one warp per node entry e = (half h, node j): the sum of |w| over the pieces of bins
  // j - 1 and j of both sets of the half; the largest per half goes to cmax[h] as the bits
  // of a non-negative double (which order like the values)
  __shared__ unsigned long long red[2];
  const int lane = threadIdx.x & 31;
  if (threadIdx.x < 2) red[threadIdx.x] = 0ull;
  __syncthreads();
  const int e = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (e < 2 * Nx) {
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
    if (lane == 0 && s > 0.0) atomicMax(&red[h], (unsigned long long)__double_as_longlong(s));
  }
  __syncthreads();
  if (threadIdx.x < 2 && red[threadIdx.x]) atomicMax(&cmax[threadIdx.x], red[threadIdx.x]);
}

// Fold of one map straight into digits.  A block covers 32 m x 16 nodes (512 threads, two
// blocks per SM, so one block's loads overlap the other's stores): warp = node, lane = m
// while the per-piece sums are read (consecutive m: coalesced), then the digit bytes go
// through shared memory so that consecutive threads store consecutive nodes.  Staging rows
// (one per (parity, digit, column, K half, m), 16 node bytes each) are 20 bytes apart with
// m fastest, so the 32 lanes of a warp store into 32 different banks.
// Sums as fold_kernel forms them (set s: A = V0(bin j) + V2(bin j-1), B = dx (V1(bin j) +
// V3(bin j-1)), V = vr - i vi; even rows A+ + A-, odd rows A+ - A-), stored as B/dx.
template <typename PT>
__global__ void __launch_bounds__(32 * kFoldNodes, 2)
fold_digits_kernel(int Nl, int Nx, int nbins, int Kp, const int* __restrict__ piece_first,
                   const PT* __restrict__ partial, const unsigned long long* __restrict__ cmax,
                   int16_t* __restrict__ cexp, int map, int ncols, uint8_t* __restrict__ fdig) {
  // stage[row][kStageRow], row = (((par * 4 + d) * 4 + c) * 2 + kh) * 32 + m, byte j of the
  // row = node j0 + j (dynamic: 2048 rows)
  extern __shared__ __align__(16) uint8_t stage[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int m0 = blockIdx.y * 32, j0 = blockIdx.x * kFoldNodes;
  const int m = m0 + lane, j = j0 + warp;
  const int e0 = scale_exp(__longlong_as_double((long long)cmax[0]));
  const int e1 = scale_exp(__longlong_as_double((long long)cmax[1]));
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {  // the column scales of the contraction
    cexp[0] = (int16_t)e0;
    cexp[1] = (int16_t)e1;
  }
  // 2^(31 - e): the fixed-point factor of each half (exact products)
  const double f0 = ldexp(1.0, 31 - e0), f1 = ldexp(1.0, 31 - e1);
  // Per half h (sets 2h, 2h+1): the piece ranges of the four keys feeding node j -- bin j
  // (rows 0-3 of its pieces) and bin j - 1 (rows 4-7) of each set.  The first piece of
  // every key is read before any further ones, so 16 loads are in flight together (most
  // bins are one piece).  acc[set][A re, A im, B re, B im] with V = vr - i vi.
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    int pa[2][2], pb[2][2];
#pragma unroll
    for (int si = 0; si < 2; ++si)
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const bool ok = m < Nl && j < Nx && (b ? j >= 1 : j < nbins);
        const int key = (2 * h + si) * nbins + j - b;
        pa[si][b] = ok ? piece_first[key] : 0;
        pb[si][b] = ok ? piece_first[key + 1] : 0;
      }
    double acc[2][4];
#pragma unroll
    for (int si = 0; si < 2; ++si) {
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[si][q] = 0.0;
#pragma unroll
      for (int b = 0; b < 2; ++b)
        if (pa[si][b] < pb[si][b]) {
          const PT* v = partial + (size_t)pa[si][b] * 8 * Nl + (size_t)(4 * b) * Nl + m;
          acc[si][0] += v[0];
          acc[si][1] -= v[(size_t)Nl];
          acc[si][2] += v[(size_t)2 * Nl];
          acc[si][3] -= v[(size_t)3 * Nl];
        }
    }
#pragma unroll
    for (int si = 0; si < 2; ++si)
#pragma unroll
      for (int b = 0; b < 2; ++b)
        for (int p = pa[si][b] + 1; p < pb[si][b]; ++p) {
          const PT* v = partial + (size_t)p * 8 * Nl + (size_t)(4 * b) * Nl + m;
          acc[si][0] += v[0];
          acc[si][1] -= v[(size_t)Nl];
          acc[si][2] += v[(size_t)2 * Nl];
          acc[si][3] -= v[(size_t)3 * Nl];
        }
    const double fh = h ? f1 : f0;
    // entries (par, ri, kh): kh = 0 the A entry, 1 the B/dx entry; even rows A+ + A-, odd A+ - A-
#pragma unroll
    for (int par = 0; par < 2; ++par)
#pragma unroll
      for (int ri = 0; ri < 2; ++ri)
#pragma unroll
        for (int kh = 0; kh < 2; ++kh) {
          const double a = acc[0][2 * kh + ri], b = acc[1][2 * kh + ri];
          const uint32_t w = digit_word_scaled((par ? a - b : a + b) * fh);
          const int c = 2 * h + ri;
#pragma unroll
          for (int d = 0; d < 4; ++d)
            stage[(((((par * 4 + d) * 4 + c) * 2 + kh) * 32) + lane) * kStageRow + warp] =
                (uint8_t)(w >> (8 * (3 - d)));
        }
  }
  __syncthreads();
  // 2048 rows x kFoldNodes/4 words; word w covers 4 nodes of one (par, d, c, kh, m) row.
  constexpr int kWords = kFoldNodes / 4;
  const int nj = min(kFoldNodes, Nx - j0);
  for (int w = threadIdx.x; w < 32 * 2 * 4 * 4 * 2 * kWords; w += blockDim.x) {
    const int q = w % kWords;      // 4-node group
    const int row = w / kWords;    // (((par * 4 + d) * 4 + c) * 2 + kh) * 32 + ml
    const int ml = row & 31;
    const int kh = (row >> 5) & 1;
    const int c = (row >> 6) & 3;
    const int d = (row >> 8) & 3;
    const int par = (row >> 10) & 1;
    const int mm = m0 + ml;
    if (mm >= Nl || 4 * q >= nj) continue;
    const uint32_t word = *reinterpret_cast<const uint32_t*>(stage + row * kStageRow + 4 * q);
    uint8_t* dst = fdig + ((((size_t)mm * 2 + par) * 4 + d) * ncols + 4 * map + c) * (size_t)Kp + (size_t)kh * Nx + j0 +
                   4 * q;
    if (4 * q + 4 <= nj && ((reinterpret_cast<uintptr_t>(dst) & 3) == 0)) {
      *reinterpret_cast<uint32_t*>(dst) = word;
    } else {
      for (int e = 0; e < 4 && 4 * q + e < nj; ++e) dst[e] = (uint8_t)(word >> (8 * e));
    }
  }
}

}  // namespace

int digit_kp(int Nx) { return (2 * Nx + 63) / 64 * 64; }

void launch_table_rowexp(const Geometry& g, int64_t row0, int64_t nrows, const double* Yv, const double* Yd,
                         int16_t* rexp, cudaStream_t s) {
  int64_t blocks = (nrows + 7) / 8;
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  table_rowexp_kernel<<<(unsigned)blocks, 256, 0, s>>>(g.Nl, g.Nx, g.dx, row0, nrows, Yv, Yd, rexp);
  count_launches(1);
}

void launch_table_digits(const Geometry& g, int64_t row0, int64_t nrows, const double* Yv, const double* Yd,
                         const int16_t* rexp, uint8_t* dig, cudaStream_t s) {
  const int Kp = digit_kp(g.Nx);
  const int64_t total = nrows * (Kp / 4);
  int64_t blocks = (total + 255) / 256;
  if (blocks > 148 * 64) blocks = 148 * 64;
  if (blocks < 1) blocks = 1;
  table_digits_kernel<<<(unsigned)blocks, 256, 0, s>>>(g.Nl, g.Nx, Kp, g.dx, row0, nrows, Yv, Yd, rexp,
                                                       (int64_t)g.Nlm * Kp, dig);
  count_launches(1);
}

void launch_table_decode(const Geometry& g, int which, int64_t r0, int64_t n, const uint8_t* dig,
                         const int16_t* rexp, double* out, cudaStream_t s) {
  const int Kp = digit_kp(g.Nx);
  int64_t blocks = (n * g.Nx + 255) / 256;
  if (blocks > 148 * 64) blocks = 148 * 64;
  if (blocks < 1) blocks = 1;
  table_decode_kernel<<<(unsigned)blocks, 256, 0, s>>>(g.Nl, g.Nx, Kp, g.dx, which, r0, n, dig,
                                                       (int64_t)g.Nlm * Kp, rexp, out);
  count_launches(1);
}

void launch_fold_scale(const Geometry& g, const Workspace& ws, unsigned long long* cmax, cudaStream_t s) {
  cudaMemsetAsync(cmax, 0, 2 * sizeof(unsigned long long), s);
  const int blocks = (2 * g.Nx + 7) / 8;
  fold_scale_kernel<<<blocks, 256, 0, s>>>(g.nbins, g.Nx, ws.piece_first, ws.wsum, cmax);
  count_launches(1);
}

void launch_fold_digits(const Geometry& g, const Workspace& ws, const unsigned long long* cmax, int16_t* cexp,
                        int map, int ncols, uint8_t* fdig, cudaStream_t s) {
  const int Kp = digit_kp(g.Nx);
  dim3 grid((g.Nx + kFoldNodes - 1) / kFoldNodes, (g.Nl + 31) / 32);
  constexpr int kStageBytes = 32 * 2 * 4 * 4 * 2 * kStageRow;
  cudaFuncSetAttribute(fold_digits_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, kStageBytes);
  cudaFuncSetAttribute(fold_digits_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, kStageBytes);
  if (ws.partial_f32)
    fold_digits_kernel<float><<<grid, 32 * kFoldNodes, kStageBytes, s>>>(g.Nl, g.Nx, g.nbins, Kp, ws.piece_first,
                                                              reinterpret_cast<const float*>(ws.partial), cmax,
                                                              cexp, map, ncols, fdig);
  else
    fold_digits_kernel<double><<<grid, 32 * kFoldNodes, kStageBytes, s>>>(g.Nl, g.Nx, g.nbins, Kp, ws.piece_first,
                                                               ws.partial, cmax, cexp, map, ncols, fdig);
  count_launches(1);
}

}  // namespace dsht
