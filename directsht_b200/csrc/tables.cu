// FP64 Ylm / dYlm tables on the spline nodes.
//
// One thread per (m, node j) walks l = m .. Nl-1 with the reference's recurrences
// (sht/legendre_py.py:4-39, :84-101 for Ylm; :41-60, :104-117 for dYlm/dx) and writes
// both tables, already multiplied by sqrt((2l+1)/4pi) (sht/legendre_py.py:67-82).
// Every product and sum is a separately rounded __dmul_rn/__dadd_rn in the reference's
// order, so the tables come out as the numpy/numba path computes them.
// Roofline: HBM write bound, 16 B written per (l, m, j).
#include "recurrence.cuh"

namespace dsht {
namespace {

constexpr int kTableThreads = 256;

// TO = double: the FP64 tables (the template keeps the store type explicit).
// Columns m = m0 + blockIdx.y; row r of the tables lands at (r - row_base) * Nx.
template <typename TO>
__global__ void __launch_bounds__(kTableThreads)
table_kernel(int Nl, int Nx, double step, TO* __restrict__ Yv, TO* __restrict__ Yd, int m0, int64_t row_base) {
  extern __shared__ double smem_raw[];
  const int m = m0 + blockIdx.y;
  Coef* cf = reinterpret_cast<Coef*>(smem_raw);       // [Nl]
  double* smm = smem_raw + (size_t)Nl * 6;            // [m+1] sqrt(1 - 1/(2m'))
  for (int l = threadIdx.x; l < Nl; l += blockDim.x) cf[l] = make_coef(l, m);
  for (int k = threadIdx.x + 1; k <= m; k += blockDim.x) smm[k] = diag_factor(k);
  __syncthreads();

  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= Nx) return;
  double x, omx2, sx;
  node_x(j, step, &x, &omx2, &sx);               // numpy: arange(Nx) * (xmax/(Nx-1))
  const double ymm = diag_value(m, sx, smm);     // Y_mm (sht/legendre_py.py:28-30)

  const int64_t row0 = hp_index(m, m, Nl) - row_base;
  TO* yv = Yv + row0 * Nx + j;
  TO* yd = Yd + row0 * Nx + j;
  ColumnState st;
  double y, d;
  column_first(m, x, omx2, ymm, &st, &y, &d);
  yv[0] = (TO)__dmul_rn(y, cf[m].nrm);
  yd[0] = (TO)__dmul_rn(d, cf[m].nrm);
  if (m + 1 >= Nl) return;
  column_second(m, cf[m + 1], &st, &y, &d);
  yv[(size_t)Nx] = (TO)__dmul_rn(y, cf[m + 1].nrm);
  yd[(size_t)Nx] = (TO)__dmul_rn(d, cf[m + 1].nrm);
  for (int l = m + 2; l < Nl; ++l) {
    const Coef c = cf[l];
    column_step(m, l, c, &st, &y, &d);
    const size_t off = (size_t)(l - m) * Nx;
    yv[off] = (TO)__dmul_rn(y, c.nrm);
    yd[off] = (TO)__dmul_rn(d, c.nrm);
  }
}

// out[m][k][j] = table row (l = m + k, m) at node j for k < Nl - m, else 0 (the JAX path's
// Yv[m, l-m, :] layout with its unphysical entries nulled, sht/legendre_jax.py:14-25).
// Grid: x over node chunks, y = k, z = m; consecutive threads take consecutive nodes.
template <typename TI>
__global__ void table_mlayout_kernel(int Nl, int Nx, const TI* __restrict__ t, double* __restrict__ out) {
  const int m = blockIdx.z, k = blockIdx.y;
  double* o = out + ((size_t)m * Nl + k) * Nx;
  const TI* src = k < Nl - m ? t + (size_t)hp_index(m + k, m, Nl) * Nx : nullptr;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < Nx; j += gridDim.x * blockDim.x)
    o[j] = src ? (double)src[j] : 0.0;
}

}  // namespace

void launch_table_mlayout(const Geometry& g, const double* t64, double* out, cudaStream_t s) {
  dim3 grid((g.Nx + 255) / 256 < 8 ? (g.Nx + 255) / 256 : 8, g.Nl, g.Nl);
  table_mlayout_kernel<double><<<grid, 256, 0, s>>>(g.Nl, g.Nx, t64, out);
  count_launches(1);
}

template <typename TO>
static void tables_launch(const Geometry& g, TO* Yv, TO* Yd, int m0, int m1, cudaStream_t s) {
  const size_t smem = (size_t)g.Nl * sizeof(Coef) + (size_t)(g.Nl + 1) * sizeof(double);
  cudaFuncSetAttribute(table_kernel<TO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 grid((g.Nx + kTableThreads - 1) / kTableThreads, m1 - m0);
  table_kernel<TO><<<grid, kTableThreads, smem, s>>>(g.Nl, g.Nx, g.dx, Yv, Yd, m0, hp_index(m0, m0, g.Nl));
  count_launches(1);
}

void launch_tables(const Geometry& g, double* Yv, double* Yd, cudaStream_t s) {
  tables_launch(g, Yv, Yd, 0, g.Nl, s);
}

void launch_tables_cols(const Geometry& g, int m0, int m1, double* Yv, double* Yd, cudaStream_t s) {
  tables_launch(g, Yv, Yd, m0, m1, s);
}

}  // namespace dsht
