// FP64 Ylm / dYlm tables on the spline nodes.
//
// One thread per (m, node j) walks l = m .. Nl-1 with the reference's recurrences
// (sht/legendre_py.py:4-39, :84-101 for Ylm; :41-60, :104-117 for dYlm/dx) and writes
// both tables, already multiplied by sqrt((2l+1)/4pi) (sht/legendre_py.py:67-82).
// Every product and sum is a separately rounded __dmul_rn/__dadd_rn in the reference's
// order, so the tables come out as the numpy/numba path computes them.
// Roofline: HBM write bound, 16 B written per (l, m, j).
#include "dsht_internal.cuh"

namespace dsht {
namespace {

constexpr int kTableThreads = 256;

// Per-l coefficients of the column m, built once per block in shared memory:
//   a = 2l-1, b = l+m-1, f2 = sqrt((l-m-1)/(l+m-1)), q = sqrt((l-m)/(l+m))/(l-m),
//   dc = (l+m) * sqrt((l-m)/(l+m)), nrm = sqrt((2l+1)/4/pi)
struct Coef {
  double a, b, f2, q, dc, nrm;
};

// TO = double: the FP64 tables; TO = float: the same FP64 values rounded once to float.
template <typename TO>
__global__ void __launch_bounds__(kTableThreads)
table_kernel(int Nl, int Nx, double step, TO* __restrict__ Yv, TO* __restrict__ Yd) {
  extern __shared__ double smem_raw[];
  const int m = blockIdx.y;
  Coef* cf = reinterpret_cast<Coef*>(smem_raw);       // [Nl]
  double* smm = smem_raw + (size_t)Nl * 6;            // [m+1] sqrt(1 - 1/(2m'))
  for (int l = threadIdx.x; l < Nl; l += blockDim.x) {
    Coef c;
    c.a = (double)(2 * l - 1);
    c.b = (double)(l + m - 1);
    c.f2 = (l >= m + 2) ? sqrt((double)(l - m - 1) / (double)(l + m - 1)) : 0.0;
    double f1 = (l > m) ? sqrt((double)(l - m) / (double)(l + m)) : 0.0;
    c.q = (l > m) ? f1 / (double)(l - m) : 0.0;
    c.dc = (double)(l + m) * f1;
    c.nrm = sqrt((double)(2 * l + 1) / 4.0 / M_PI);
    cf[l] = c;
  }
  for (int k = threadIdx.x + 1; k <= m; k += blockDim.x) smm[k] = sqrt(1.0 - 1.0 / (double)(2 * k));
  __syncthreads();

  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= Nx) return;
  const double x = (double)j * step;               // numpy: arange(Nx) * (xmax/(Nx-1))
  const double x2 = __dmul_rn(x, x);
  const double omx2 = __dadd_rn(1.0, -x2);
  const double sx = sqrt(omx2);

  // Y_mm by the diagonal recurrence (sht/legendre_py.py:28-30).
  double ymm = 1.0;
  for (int k = 1; k <= m; ++k) ymm = __dmul_rn(__dmul_rn(-smm[k], sx), ymm);

  const int64_t row0 = hp_index(m, m, Nl);
  TO* yv = Yv + row0 * Nx + j;
  TO* yd = Yd + row0 * Nx + j;

  // l = m
  double y2 = 0.0, y1 = ymm;  // y2 = Y_{l-2}, y1 = Y_{l-1}
  {
    double d;
    if (m == 0) {
      d = 0.0;
    } else {  // ((l+m) f1) Y_{l-1} with f1 = 0, minus (l x) Y_l, over 1-x^2
      d = __ddiv_rn(__dadd_rn(0.0, -__dmul_rn(__dmul_rn((double)m, x), ymm)), omx2);
    }
    const double n = cf[m].nrm;
    yv[0] = (TO)__dmul_rn(ymm, n);
    yd[0] = (TO)__dmul_rn(d, n);
  }
  if (m + 1 >= Nl) return;
  // l = m + 1: Y = sqrt(2m+1) x Y_mm (sht/legendre_py.py:32-34); m = 0 row is x itself.
  double y;
  if (m == 0) {
    y = x;
  } else {
    y = __dmul_rn(__dmul_rn(sqrt(2.0 * m + 1.0), x), ymm);
  }
  {
    const int l = m + 1;
    double d;
    if (m == 0) {
      d = 1.0;
    } else {
      d = __ddiv_rn(__dadd_rn(__dmul_rn(cf[l].dc, y1), -__dmul_rn(__dmul_rn((double)l, x), y)), omx2);
    }
    const double n = cf[l].nrm;
    yv[(size_t)Nx] = (TO)__dmul_rn(y, n);
    yd[(size_t)Nx] = (TO)__dmul_rn(d, n);
  }
  y2 = y1;
  y1 = y;
  for (int l = m + 2; l < Nl; ++l) {
    const Coef c = cf[l];
    // ((2l-1) x) Y_{l-1} - ((l+m-1) Y_{l-2}) f2, times f1/(l-m)  (sht/legendre_py.py:98-100)
    double t = __dadd_rn(__dmul_rn(__dmul_rn(c.a, x), y1), -__dmul_rn(__dmul_rn(c.b, y2), c.f2));
    y = __dmul_rn(t, c.q);
    double d;
    if (m == 0) {  // l/(1-x^2) (Y_{l-1} - x Y_l)  (sht/legendre_py.py:56)
      d = __dmul_rn(__ddiv_rn((double)l, omx2), __dadd_rn(y1, -__dmul_rn(x, y)));
    } else {       // ((l+m) f1 Y_{l-1} - l x Y_l) / (1-x^2)  (sht/legendre_py.py:115-116)
      d = __ddiv_rn(__dadd_rn(__dmul_rn(c.dc, y1), -__dmul_rn(__dmul_rn((double)l, x), y)), omx2);
    }
    const size_t off = (size_t)(l - m) * Nx;
    yv[off] = (TO)__dmul_rn(y, c.nrm);
    yd[off] = (TO)__dmul_rn(d, c.nrm);
    y2 = y1;
    y1 = y;
  }
}

__global__ void to_f32_kernel(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                              float* __restrict__ a32, float* __restrict__ b32) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    a32[i] = (float)a[i];
    b32[i] = (float)b[i];
  }
}

}  // namespace

void launch_tables_to_f32(const Geometry& g, const double* Yv, const double* Yd, float* Yv32, float* Yd32,
                          cudaStream_t s) {
  const int64_t n = g.Nlm * (int64_t)g.Nx;
  to_f32_kernel<<<148 * 16, 256, 0, s>>>(n, Yv, Yd, Yv32, Yd32);
  count_launches(1);
}

template <typename TO>
static void tables_launch(const Geometry& g, TO* Yv, TO* Yd, cudaStream_t s) {
  const size_t smem = (size_t)g.Nl * sizeof(Coef) + (size_t)(g.Nl + 1) * sizeof(double);
  cudaFuncSetAttribute(table_kernel<TO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 grid((g.Nx + kTableThreads - 1) / kTableThreads, g.Nl);
  table_kernel<TO><<<grid, kTableThreads, smem, s>>>(g.Nl, g.Nx, g.dx, Yv, Yd);
  count_launches(1);
}

void launch_tables(const Geometry& g, double* Yv, double* Yd, cudaStream_t s) { tables_launch(g, Yv, Yd, s); }

void launch_tables_f32(const Geometry& g, float* Yv, float* Yd, cudaStream_t s) { tables_launch(g, Yv, Yd, s); }

}  // namespace dsht
