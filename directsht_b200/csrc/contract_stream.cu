// Streaming contraction of the FP64 tables with the folded node sums (the FP64 and
// DSHT_PREC_MIXED_F64_TABLES levels), fed by TMA through a two-stage shared-memory ring.
//
//   alm_equ[lm] = sum_j Yv[lm,j] A_q[m,j] + Yd[lm,j] B_q[m,j],  q = equ even/odd by (l-m)%2
//   alm_pol[lm] = same with the polar q                     (sht/sht.py:266-279)
//
// Persistent CTAs walk work items (m, 16 consecutive rows l).  Warp 0 (one thread) is the
// producer: for every live tile of 256 nodes it issues one 2D tensor-map TMA load per table
// (a 16-row x 256-node box of Yv and of Yd) and one bulk copy per fold row (4 q), all
// completing on the stage's mbarrier.  Warps 1-8 consume: each owns two rows of equal
// parity and the 256 nodes of the tile (8 per lane); the FP64 fold values in shared memory
// feed both rows.  HBM bound: 16 bytes of table per (l, m, node).
#include <cudaTypedefs.h>

#include <algorithm>

#include "dsht_internal.cuh"
#include "tc_ptx.cuh"

namespace dsht {
namespace {

constexpr int kTJ = 256;                  // nodes per tile
constexpr int kConsumers = 8;             // warps 1..8
constexpr int kThreads = 32 * (1 + kConsumers);
constexpr int kStagesC = 2;

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          tc::smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(tc::smem_addr(bar))
      : "memory");
}

// 2D tiled TMA load of a kRows x kTJ box of a table (x = node, y = table row).
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* tm, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(tc::smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(tc::smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
                   tc::smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// Work items in m order: group index g < groups(m) = ceil((Nl - m) / kRows).
template <int kRows>
__device__ __forceinline__ void item_of(int64_t item, int Nl, int* m_out, int* g_out) {
  // cumulative groups before m: G(m) = sum_{m' < m} ceil((Nl - m') / kRows); binary search.
  int lo = 0, hi = Nl;  // find largest m with G(m) <= item
  auto G = [&](int m) -> int64_t {
    // sum_{n = Nl-m+1}^{Nl} ceil(n / R) with n = Nl - m'
    auto S = [](int64_t n) -> int64_t {  // sum_{k=1}^{n} ceil(k / R)
      const int64_t q = n / kRows, r = n % kRows;
      return kRows * q * (q + 1) / 2 + r * (q + 1);
    };
    return S(Nl) - S(Nl - m);
  };
  while (hi - lo > 1) {
    const int mid = (lo + hi) / 2;
    if (G(mid) <= item) lo = mid;
    else hi = mid;
  }
  *m_out = lo;
  *g_out = (int)(item - G(lo));
}

constexpr int kRows = 16;                 // rows per work item
constexpr int kRowsPerWarp = kRows / 8;   // same parity, stride 2
constexpr int kTab = kRows * kTJ * sizeof(double);   // one of Yv, Yd
constexpr int kFold = 4 * kTJ * sizeof(double4);     // 4 q x kTJ
constexpr int kStage = 2 * kTab + kFold;
constexpr int kStreamBytes = kStagesC * kStage + 128 + 128;

__global__ void __launch_bounds__(kThreads, 1)
contract_stream_kernel(int Nl, int Nx, int64_t nitems, const __grid_constant__ CUtensorMap tmv,
                       const __grid_constant__ CUtensorMap tmd, const double4* __restrict__ fold,
                       const uint8_t* __restrict__ live, int ntile, double* __restrict__ alm_equ,
                       double* __restrict__ alm_pol, unsigned* __restrict__ err) {
  constexpr int RW = kRowsPerWarp;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStagesC * kStage);
  uint64_t* empty = full + kStagesC;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(empty + kStagesC);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < kStagesC; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], kConsumers);
    }
    *abort_flag = 0;
    tc::mbar_fence_init();
  }
  __syncthreads();

  if (warp == 0) {
    // ---- producer (one thread) --------------------------------------------------------
    if (lane == 0) {
      uint32_t n = 0;  // stages issued
      for (int64_t item = blockIdx.x; item < nitems && !*abort_flag; item += gridDim.x) {
        int m, g;
        item_of<kRows>(item, Nl, &m, &g);
        const int l0 = m + g * kRows;
        const int64_t row0 = hp_index(l0, m, Nl);
        for (int t = 0; t < ntile; ++t) {
          if (!live[t] && !live[ntile + t]) continue;
          const int s = n % kStagesC;
          const uint32_t use = n / kStagesC;
          if (use > 0 && !tc::mbar_wait(&empty[s], (use - 1) & 1, abort_flag)) {
            *abort_flag = 1;
            atomicOr(err, kFlagTimeout);
            break;
          }
          const int j0 = t * kTJ;
          const int nj = min(kTJ, Nx - j0);
          uint8_t* st = smem + s * kStage;
          const uint32_t fold_bytes = nj * sizeof(double4);
          // The table boxes always transfer kRows x kTJ elements (zero fill out of range).
          mbar_arrive_tx(&full[s], 2u * kTab + 4u * fold_bytes);
          tma_load_2d(st, &tmv, j0, (int)row0, &full[s]);
          tma_load_2d(st + kTab, &tmd, j0, (int)row0, &full[s]);
          for (int q = 0; q < 4; ++q)
            bulk_g2s(st + 2 * kTab + q * kTJ * sizeof(double4), fold + ((size_t)m * 4 + q) * Nx + j0, fold_bytes,
                     &full[s]);
          ++n;
        }
      }
    }
    __syncwarp();
  } else {
    // ---- consumers: warp cw owns the RW rows par + 2 RW (cw >> 1) + 2 i ---------------
    const int cw = warp - 1;
    const int par = cw & 1;
    const int rbase = par + 2 * RW * (cw >> 1);
    uint32_t n = 0;
    for (int64_t item = blockIdx.x; item < nitems; item += gridDim.x) {
      int m, g;
      item_of<kRows>(item, Nl, &m, &g);
      const int l0 = m + g * kRows;
      double acc[RW][4];
#pragma unroll
      for (int i = 0; i < RW; ++i)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[i][c] = 0.0;
      for (int t = 0; t < ntile; ++t) {
        if (!live[t] && !live[ntile + t]) continue;
        const int s = n % kStagesC;
        const uint32_t use = n / kStagesC;
        bool ok = !*abort_flag;
        if (ok && !tc::mbar_wait(&full[s], use & 1, abort_flag)) {
          *abort_flag = 1;
          atomicOr(err, kFlagTimeout);
          ok = false;
        }
        if (ok) {
          const uint8_t* st = smem + s * kStage;
          const double* Tv = reinterpret_cast<const double*>(st);
          const double* Td = reinterpret_cast<const double*>(st + kTab);
          const double4* Fe = reinterpret_cast<const double4*>(st + 2 * kTab) + par * kTJ;
          const int nj = min(kTJ, Nx - t * kTJ);
#pragma unroll 4
          for (int jj = lane; jj < nj; jj += 32) {
            const double4 fe = Fe[jj], fp = Fe[2 * kTJ + jj];
#pragma unroll
            for (int i = 0; i < RW; ++i) {
              const int r = rbase + 2 * i;
              const double v = Tv[r * kTJ + jj], d = Td[r * kTJ + jj];
              acc[i][0] = fma(v, fe.x, fma(d, fe.z, acc[i][0]));
              acc[i][1] = fma(v, fe.y, fma(d, fe.w, acc[i][1]));
              acc[i][2] = fma(v, fp.x, fma(d, fp.z, acc[i][2]));
              acc[i][3] = fma(v, fp.y, fma(d, fp.w, acc[i][3]));
            }
          }
        }
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&empty[s]);
        ++n;
      }
#pragma unroll
      for (int i = 0; i < RW; ++i)
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) acc[i][c] += __shfl_xor_sync(0xffffffffu, acc[i][c], o);
      if (lane == 0) {
#pragma unroll
        for (int i = 0; i < RW; ++i) {
          const int l = l0 + rbase + 2 * i;
          if (l < Nl) {
            const int64_t idx = hp_index(l, m, Nl);
            alm_equ[2 * idx] = acc[i][0];
            alm_equ[2 * idx + 1] = acc[i][1];
            alm_pol[2 * idx] = acc[i][2];
            alm_pol[2 * idx + 1] = acc[i][3];
          }
        }
      }
    }
  }
  // Drain: every issued stage has been consumed (consumers waited on all of them).
  __syncthreads();
}

}  // namespace

bool contract_stream_ok(const Geometry& g) {
  // Bulk copies need 16-byte aligned row segments.
  return ((size_t)g.Nx * sizeof(double)) % 16 == 0;
}

int make_table_tmap(CUtensorMap* tm, const void* base, int Nx, int64_t Nlm) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return set_error(DSHT_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  const cuuint64_t dims[2] = {(cuuint64_t)Nx, (cuuint64_t)Nlm};
  const cuuint64_t strides[1] = {(cuuint64_t)Nx * sizeof(double)};
  const cuuint32_t box[2] = {(cuuint32_t)kTJ, (cuuint32_t)kRows};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = encode(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void*>(base), dims, strides, box, estr,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(DSHT_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return DSHT_OK;
}

void launch_contract_stream(const Geometry& g, const CUtensorMap& tmv, const CUtensorMap& tmd, const double* fold,
                            const uint8_t* live, double* alm_equ, double* alm_pol, unsigned* flags, cudaStream_t s) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ntile = (g.Nx + kTJ - 1) / kTJ;
  int64_t nitems = 0;
  for (int m = 0; m < g.Nl; ++m) nitems += (g.Nl - m + kRows - 1) / kRows;
  const int64_t grid = nitems < sms ? nitems : sms;
  cudaFuncSetAttribute(contract_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kStreamBytes);
  contract_stream_kernel<<<(unsigned)grid, kThreads, kStreamBytes, s>>>(
      g.Nl, g.Nx, nitems, tmv, tmd, reinterpret_cast<const double4*>(fold), live, ntile, alm_equ, alm_pol, flags);
  count_launches(1);
}

}  // namespace dsht
