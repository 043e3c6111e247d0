// Streaming contraction of the stored tables with the folded node sums, fed by TMA bulk
// copies (cp.async.bulk) through a two-stage shared-memory ring.
//
//   alm_equ[lm] = sum_j Yv[lm,j] A_q[m,j] + Yd[lm,j] B_q[m,j],  q = equ even/odd by (l-m)%2
//   alm_pol[lm] = same with the polar q                     (sht/sht.py:266-279)
//
// Persistent CTAs walk work items (m, R consecutive rows l).  Warp 0 (one thread) is the
// producer: for every live tile of 256 nodes it issues one 2D tensor-map TMA load per table
// (an R-row x 256-node box of Yv and of Yd) and one bulk copy per fold row (4 q), all
// completing on the stage's mbarrier.  Warps 1-8 consume: each owns R/8 rows of equal
// parity and the 256 nodes of the tile (8 per lane); the FP64 fold values in shared memory
// feed all its rows.  FP64 tables: double tables and fold, R = 16, FP64 FMAs.  FP32
// tables: float tables and fold, R = 32, FP32 FMAs within a tile, FP64 sums across tiles.
// HBM bound: 2 sizeof(T) bytes of table per (l, m, node).
#include <cudaTypedefs.h>

#include <algorithm>
#include <type_traits>

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

// FP64 tables: double tables and fold, 16 rows per item, FP64 FMAs.  FP32 tables (the
// DSHT_PREC_MIXED level): float tables and fold, 32 rows per item, FP32 FMAs within a
// tile and FP64 sums across tiles -- half the HBM traffic.
template <bool kMixed, int kG = 1, int kRowsSet = 0>
struct StageLayout {
  using T = typename std::conditional<kMixed, float, double>::type;
  using F4 = typename std::conditional<kMixed, float4, double4>::type;
  static constexpr int kRows = kRowsSet ? kRowsSet : kMixed ? 32 : 16;
  static constexpr int kRowsPerWarp = kRows / 8;               // same parity, stride 2
  static constexpr int kTab = kRows * kTJ * sizeof(T);         // one of Yv, Yd
  static constexpr int kFold = 4 * kTJ * sizeof(F4);           // 4 q x kTJ, one map
  static constexpr int kStage = 2 * kTab + kG * kFold;
  static constexpr int kBytes = kStagesC * kStage + 128 + 128;
};

// kG maps per pass (multi-map transforms): map g's fold at fold_v + g * fold_stride (F4
// elements) and its alm at out.equ[g], out.pol[g] (2 Nlm doubles each).  The
// table tile in shared memory serves all kG maps, so a pass reads the tables once.  Passes
// of three or four maps take 16-row items (two rows per warp), which keeps the FP64
// accumulators of all maps in registers.
template <bool kMixed, int kG, int kRowsSet = 0>
__global__ void __launch_bounds__(kThreads, 1)
contract_stream_kernel(int Nl, int Nx, int64_t nitems, const __grid_constant__ CUtensorMap tmv,
                       const __grid_constant__ CUtensorMap tmd, const void* __restrict__ fold_v,
                       int64_t fold_stride, const uint8_t* __restrict__ live, int ntile,
                       const MapOut out, unsigned* __restrict__ err) {
  using L = StageLayout<kMixed, kG, kRowsSet>;
  using T = typename L::T;
  using F4 = typename L::F4;
  constexpr int kRows = L::kRows;
  constexpr int RW = L::kRowsPerWarp;
  const F4* fold = reinterpret_cast<const F4*>(fold_v);
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
          uint8_t* st = smem + s * L::kStage;
          const uint32_t fold_bytes = nj * sizeof(F4);
          // The table boxes always transfer kRows x kTJ elements (zero fill out of range).
          mbar_arrive_tx(&full[s], 2u * L::kTab + 4u * kG * fold_bytes);
          tma_load_2d(st, &tmv, j0, (int)row0, &full[s]);
          tma_load_2d(st + L::kTab, &tmd, j0, (int)row0, &full[s]);
#pragma unroll
          for (int gm = 0; gm < kG; ++gm)
            for (int q = 0; q < 4; ++q)
              bulk_g2s(st + 2 * L::kTab + gm * L::kFold + q * kTJ * sizeof(F4),
                       fold + gm * fold_stride + ((size_t)m * 4 + q) * Nx + j0, fold_bytes, &full[s]);
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
      double acc[kG][RW][4];
#pragma unroll
      for (int gm = 0; gm < kG; ++gm)
#pragma unroll
        for (int i = 0; i < RW; ++i)
#pragma unroll
          for (int c = 0; c < 4; ++c) acc[gm][i][c] = 0.0;
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
          const T* Tv = reinterpret_cast<const T*>(st);
          const T* Td = reinterpret_cast<const T*>(st + L::kTab);
          const int nj = min(kTJ, Nx - t * kTJ);
          T part[kG][RW][4];
#pragma unroll
          for (int gm = 0; gm < kG; ++gm)
#pragma unroll
            for (int i = 0; i < RW; ++i)
#pragma unroll
              for (int c = 0; c < 4; ++c) part[gm][i][c] = (T)0;
#pragma unroll(kG == 1 ? 4 : 2)
          for (int jj = lane; jj < nj; jj += 32) {
            T v[RW], d[RW];
#pragma unroll
            for (int i = 0; i < RW; ++i) {
              const int r = rbase + 2 * i;
              v[i] = Tv[r * kTJ + jj];
              d[i] = Td[r * kTJ + jj];
            }
#pragma unroll
            for (int gm = 0; gm < kG; ++gm) {
              const F4* Fe = reinterpret_cast<const F4*>(st + 2 * L::kTab + gm * L::kFold) + par * kTJ;
              const F4 fe = Fe[jj], fp = Fe[2 * kTJ + jj];
#pragma unroll
              for (int i = 0; i < RW; ++i) {
                part[gm][i][0] = fma(v[i], fe.x, fma(d[i], fe.z, part[gm][i][0]));
                part[gm][i][1] = fma(v[i], fe.y, fma(d[i], fe.w, part[gm][i][1]));
                part[gm][i][2] = fma(v[i], fp.x, fma(d[i], fp.z, part[gm][i][2]));
                part[gm][i][3] = fma(v[i], fp.y, fma(d[i], fp.w, part[gm][i][3]));
              }
            }
          }
#pragma unroll
          for (int gm = 0; gm < kG; ++gm)
#pragma unroll
            for (int i = 0; i < RW; ++i)
#pragma unroll
              for (int c = 0; c < 4; ++c) acc[gm][i][c] += (double)part[gm][i][c];
        }
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&empty[s]);
        ++n;
      }
#pragma unroll
      for (int gm = 0; gm < kG; ++gm)
#pragma unroll
        for (int i = 0; i < RW; ++i)
#pragma unroll
          for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[gm][i][c] += __shfl_xor_sync(0xffffffffu, acc[gm][i][c], o);
      if (lane == 0) {
#pragma unroll
        for (int gm = 0; gm < kG; ++gm) {
          // outputs that already hold heavy-node FP64 sums (heavy.cu) are added to
          const bool add = out.heavy_n[gm] != nullptr && *out.heavy_n[gm] > 0;
#pragma unroll
          for (int i = 0; i < RW; ++i) {
            const int l = l0 + rbase + 2 * i;
            if (l < Nl) {
              const int64_t idx = hp_index(l, m, Nl);
              double* ae = out.equ[gm];
              double* ap = out.pol[gm];
              if (add) {
                ae[2 * idx] += acc[gm][i][0];
                ae[2 * idx + 1] += acc[gm][i][1];
                ap[2 * idx] += acc[gm][i][2];
                ap[2 * idx + 1] += acc[gm][i][3];
              } else {
                ae[2 * idx] = acc[gm][i][0];
                ae[2 * idx + 1] = acc[gm][i][1];
                ap[2 * idx] = acc[gm][i][2];
                ap[2 * idx + 1] = acc[gm][i][3];
              }
            }
          }
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

int make_table_tmap(CUtensorMap* tm, const void* base, size_t elem_bytes, int Nx, int64_t Nlm, int rows) {
  const int kRows = rows > 0 ? rows : elem_bytes == 8 ? StageLayout<false, 1>::kRows : StageLayout<true, 1>::kRows;
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

template <bool kMixed, int kG, int kRowsSet = 0>
static void stream_launch(const Geometry& g, const CUtensorMap& tmv, const CUtensorMap& tmd, const void* fold,
                          int64_t fold_stride, const uint8_t* live, const MapOut& out, unsigned* flags,
                          cudaStream_t s) {
  using L = StageLayout<kMixed, kG, kRowsSet>;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ntile = (g.Nx + kTJ - 1) / kTJ;
  int64_t nitems = 0;
  for (int m = 0; m < g.Nl; ++m) nitems += (g.Nl - m + L::kRows - 1) / L::kRows;
  const int64_t grid = nitems < sms ? nitems : sms;
  auto kern = contract_stream_kernel<kMixed, kG, kRowsSet>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L::kBytes);
  kern<<<(unsigned)grid, kThreads, L::kBytes, s>>>(g.Nl, g.Nx, nitems, tmv, tmd, fold, fold_stride, live, ntile,
                                                   out, flags);
  count_launches(1);
}

void launch_contract_stream(const Geometry& g, bool mixed, const CUtensorMap& tmv, const CUtensorMap& tmd,
                            const Workspace& ws, cudaStream_t s, const int* heavy_n) {
  MapOut out{};
  out.equ[0] = ws.alm_equ;
  out.pol[0] = ws.alm_pol;
  out.heavy_n[0] = heavy_n;
  if (mixed)
    stream_launch<true, 1>(g, tmv, tmd, ws.fold, 0, ws.tile_live2, out, ws.flags, s);
  else
    stream_launch<false, 1>(g, tmv, tmd, ws.fold, 0, ws.tile_live2, out, ws.flags, s);
}

int contract_stream_max_maps(bool mixed) { return mixed ? kMaxPass : 1; }

void launch_contract_pass(const Geometry& g, bool mixed, const CUtensorMap& tmv, const CUtensorMap& tmd,
                          const CUtensorMap& tmv16, const CUtensorMap& tmd16, const void* fold, int64_t fold_stride,
                          int nmaps, const uint8_t* live, const MapOut& out, unsigned* flags, cudaStream_t s) {
  if (mixed && nmaps == 4)
    stream_launch<true, 4, 16>(g, tmv16, tmd16, fold, fold_stride, live, out, flags, s);
  else if (mixed && nmaps == 3)
    stream_launch<true, 3, 16>(g, tmv16, tmd16, fold, fold_stride, live, out, flags, s);
  else if (mixed && nmaps == 2)
    stream_launch<true, 2>(g, tmv, tmd, fold, fold_stride, live, out, flags, s);
  else if (mixed)
    stream_launch<true, 1>(g, tmv, tmd, fold, fold_stride, live, out, flags, s);
  else  // FP64 tables: one map per pass (two stages of two maps' FP64 folds do not fit)
    for (int k = 0; k < nmaps; ++k) {
      MapOut o1{};
      o1.equ[0] = out.equ[k];
      o1.pol[0] = out.pol[k];
      o1.heavy_n[0] = out.heavy_n[k];
      stream_launch<false, 1>(g, tmv, tmd, static_cast<const double4*>(fold) + fold_stride * k, 0, live, o1, flags,
                              s);
    }
}

}  // namespace dsht
