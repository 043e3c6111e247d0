// Streaming contraction of the stored tables with the folded node sums, fed by TMA bulk
// copies (cp.async.bulk) through a two-stage shared-memory ring.
//
//   alm_equ[lm] = sum_j Yv[lm,j] A_q[m,j] + Yd[lm,j] B_q[m,j],  q = equ even/odd by (l-m)%2
//   alm_pol[lm] = same with the polar q                     (sht/sht.py:266-279)
//
// Persistent CTAs walk work items (m, 16 consecutive rows l).  Warp 0 (one thread) is the
// producer: for every live tile of 256 nodes it issues one 2D tensor-map TMA load per table
// (a 16-row x 256-node box of Yv and of Yd) and one bulk copy per fold row (4 q), all
// completing on the stage's mbarrier.
// Warps 1-8 consume: each owns two rows of equal parity and the 256 nodes of the tile
// (8 per lane), accumulating in FP64; the fold values in shared memory feed both rows.
// HBM bound: sizeof(T) x 2 bytes of table per (l, m, node).  T = double (FP64 plans) or
// float (FP32 copy of the tables used by mixed-precision plans).
#include <cudaTypedefs.h>

#include "dsht_internal.cuh"
#include "tc_ptx.cuh"

namespace dsht {
namespace {

constexpr int kRows = 16;
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

template <typename T>
struct StageLayout {
  static constexpr int kTab = kRows * kTJ * sizeof(T);   // one of Yv, Yd
  static constexpr int kFold = 4 * kTJ * 32;              // 4 q x kTJ x double4
  static constexpr int kStage = 2 * kTab + kFold;
  static constexpr int kBytes = kStagesC * kStage + 128 + 128;
};

template <typename T>
__global__ void __launch_bounds__(kThreads, 1)
contract_stream_kernel(int Nl, int Nx, int64_t nitems, const __grid_constant__ CUtensorMap tmv,
                       const __grid_constant__ CUtensorMap tmd, const double* __restrict__ fold, const uint8_t* __restrict__ live, int ntile,
                       double* __restrict__ alm_equ, double* __restrict__ alm_pol, unsigned* __restrict__ err) {
  using L = StageLayout<T>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStagesC * L::kStage);
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
        item_of(item, Nl, &m, &g);
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
          uint8_t* st = smem + s * L::kStage;
          const uint32_t fold_bytes = nj * 32;
          // The table boxes always transfer kRows x kTJ elements (zero fill out of range).
          mbar_arrive_tx(&full[s], 2u * L::kTab + 4u * fold_bytes);
          tma_load_2d(st, &tmv, j0, (int)row0, &full[s]);
          tma_load_2d(st + L::kTab, &tmd, j0, (int)row0, &full[s]);
          for (int q = 0; q < 4; ++q)
            bulk_g2s(st + 2 * L::kTab + q * kTJ * 32, fold + ((size_t)m * 4 + q) * Nx * 4 + (size_t)j0 * 4,
                     fold_bytes, &full[s]);
          ++n;
        }
      }
    }
    __syncwarp();
  } else {
    // ---- consumers: warp cw owns rows ra = par + 4 (cw >> 1) and ra + 2 ----------------
    const int cw = warp - 1;
    const int par = cw & 1;
    const int ra = par + 4 * (cw >> 1);
    uint32_t n = 0;
    for (int64_t item = blockIdx.x; item < nitems; item += gridDim.x) {
      int m, g;
      item_of(item, Nl, &m, &g);
      const int l0 = m + g * kRows;
      const int la = l0 + ra, lb = l0 + ra + 2;
      const bool va = la < Nl, vb = lb < Nl;
      double ea_r = 0, ea_i = 0, pa_r = 0, pa_i = 0, eb_r = 0, eb_i = 0, pb_r = 0, pb_i = 0;
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
          const uint8_t* st = smem + s * L::kStage;
          const T* Ta = reinterpret_cast<const T*>(st) + ra * kTJ;
          const T* Da = reinterpret_cast<const T*>(st + L::kTab) + ra * kTJ;
          const double4* Fe = reinterpret_cast<const double4*>(st + 2 * L::kTab) + par * kTJ;
          const double4* Fp = Fe + 2 * kTJ;
          const int nj = min(kTJ, Nx - t * kTJ);
#pragma unroll 4
          for (int jj = lane; jj < nj; jj += 32) {
            const double4 fe = Fe[jj], fp = Fp[jj];
            if (va) {
              const double v = (double)Ta[jj], d = (double)Da[jj];
              ea_r = fma(v, fe.x, fma(d, fe.z, ea_r));
              ea_i = fma(v, fe.y, fma(d, fe.w, ea_i));
              pa_r = fma(v, fp.x, fma(d, fp.z, pa_r));
              pa_i = fma(v, fp.y, fma(d, fp.w, pa_i));
            }
            if (vb) {
              const double v = (double)Ta[2 * kTJ + jj], d = (double)Da[2 * kTJ + jj];
              eb_r = fma(v, fe.x, fma(d, fe.z, eb_r));
              eb_i = fma(v, fe.y, fma(d, fe.w, eb_i));
              pb_r = fma(v, fp.x, fma(d, fp.z, pb_r));
              pb_i = fma(v, fp.y, fma(d, fp.w, pb_i));
            }
          }
        }
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&empty[s]);
        ++n;
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
  }
  // Drain: every issued stage has been consumed (consumers waited on all of them).
  __syncthreads();
}

}  // namespace

bool contract_stream_ok(const Geometry& g, size_t elem_bytes) {
  // Bulk copies need 16-byte aligned row segments.
  return ((size_t)g.Nx * elem_bytes) % 16 == 0;
}

int make_table_tmap(CUtensorMap* tm, const void* base, size_t elem_bytes, int Nx, int64_t Nlm) {
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
  const cuuint64_t strides[1] = {(cuuint64_t)Nx * elem_bytes};
  const cuuint32_t box[2] = {(cuuint32_t)kTJ, (cuuint32_t)kRows};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = encode(tm, elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                      const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(DSHT_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return DSHT_OK;
}

template <typename T>
void launch_contract_stream(const Geometry& g, const CUtensorMap& tmv, const CUtensorMap& tmd, const Workspace& ws,
                            cudaStream_t s) {
  using L = StageLayout<T>;
  cudaFuncSetAttribute(contract_stream_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::kBytes);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ntile = (g.Nx + kTJ - 1) / kTJ;
  int64_t nitems = 0;
  for (int m = 0; m < g.Nl; ++m) nitems += (g.Nl - m + kRows - 1) / kRows;
  const int64_t grid = nitems < sms ? nitems : sms;
  contract_stream_kernel<T><<<(unsigned)grid, kThreads, L::kBytes, s>>>(
      g.Nl, g.Nx, nitems, tmv, tmd, ws.fold, ws.tile_live2, ntile, ws.alm_equ, ws.alm_pol, ws.flags);
  count_launches(1);
}

template void launch_contract_stream<double>(const Geometry&, const CUtensorMap&, const CUtensorMap&,
                                             const Workspace&, cudaStream_t);
template void launch_contract_stream<float>(const Geometry&, const CUtensorMap&, const CUtensorMap&,
                                            const Workspace&, cudaStream_t);

}  // namespace dsht
