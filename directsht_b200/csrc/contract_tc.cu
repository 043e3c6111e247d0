// Tensor-core contraction of digit tables with digit folds (tcgen05 kind::i8, exact S32).
//
//   alm_equ[lm] = sum_k T[lm, k] F_equ,q[k],  alm_pol[lm] likewise,  q = parity of l - m
//   (sht/sht.py:266-279, sht/interp_funcs_py.py:46-60; T, F and their digits: digits.cu)
//
// For one (m, parity) the rows l = m + par, m + par + 2, ... form a contiguous block of the
// grouped digit table, and every map / half / re|im of the pass is one column of the fold,
// so the contraction is a GEMM D = T F with M = the block's rows (tiles of 128), N = the
// pass's columns (NC: 16, 32 or 64, four per map) and K = 2 Nx.  With four signed digits
// per operand, T = sum_i A_i 2^(24-8i), F = sum_j B_j 2^(24-8j), the classes
// W_c = sum_{i+j=c} A_i B_j (c = 0..4) leave out only products below 2^-40 of the row
// scale times the column scale (class 4 is needed: the dropped products do not shrink with
// the entries, and a fold column can hold one large node beside many small ones).
// The digit planes B_0..B_3 of a stage are consecutive in shared memory, so one MMA of A_i
// against consecutive planes B_j..B_k adds to W_(i+j)..W_(i+k) at once: five MMAs per
// 32-byte K step (A_0 B_0; A_1 B_0..3, which starts W_1..W_4; A_0 B_1..3; A_2 B_0..2;
// A_3 B_0..1).  Integer sums are exact (|W_c| <= 4 K 2^14 <= 2^30 for K <= 16384); the
// epilogue forms V = W_0 2^32 + W_1 2^24 + W_2 2^16 + W_3 2^8 + W_4 in int64 and the
// value 2^(er+ec-46) V.
//
// Warp roles: warp 0 (one thread) claims work items from a global counter and issues TMA
// loads -- one 3D box of 4 digit planes x 128 rows x 64 bytes of the table and one of 4
// planes x NC columns x 64 bytes of the fold per stage -- into a ring of stages; warp 1
// allocates TMEM and issues the MMAs from one thread;
// warps 2-5 read the accumulators (TMEM lanes 32 (w % 4) ..) and write the alm, while the
// next tile accumulates into the other TMEM buffer.  Every wait is bounded and records
// kFlagTimeout instead of hanging.  No cluster multicast anywhere.
//
// Items are claimed in order (m, parity, row tile) by whichever CTA is free, so the row tiles
// of one (m, parity) block run at about the same time on different SMs and the block's fold
// slice (NC x 32 bytes per node) comes from DRAM once and from L2 for the other tiles.  (A
// fixed round-robin assignment let the CTAs drift apart, and the slice was read from DRAM
// about once per tile: +25 % of DRAM traffic at Nl = 2048 with 32 columns.)
//
// Bound: HBM (the table digits, 8 B per (l, m, node), half the FP64 pair) while N is
// small; each table byte is read once per pass however many maps the pass holds.
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>

#include "dsht_internal.cuh"
#include "tc_ptx.cuh"

namespace dsht {
namespace {

constexpr int kChunk = 64;    // K bytes per stage: one 64-byte swizzled row per operand row
constexpr int kTileRows = 128;
constexpr int kEpiWarps = 4;
constexpr int kTcThreads = 32 * (2 + kEpiWarps);
constexpr int kItemRing = 16;  // claimed items in flight: the producer leads the epilogue by <= kStages + 3

template <int NC>
struct TcLayout {
  static constexpr int kA = 4 * kTileRows * kChunk;  // 32 KB: digit planes A_0..A_3
  static constexpr int kB = 4 * NC * kChunk;         // digit planes B_0..B_3
  static constexpr int kStage = kA + kB;
  static constexpr int kStages = (200 * 1024) / kStage > 6 ? 6 : (200 * 1024) / kStage;
  static constexpr int kAcc = 5 * NC;                // TMEM columns of W_0..W_4
  static constexpr int kBufs = 2 * kAcc <= 512 ? 2 : 1;
  static constexpr uint32_t kTmemCols = kBufs * kAcc <= 32 ? 32 : kBufs * kAcc <= 64 ? 64
                                        : kBufs * kAcc <= 128 ? 128 : kBufs * kAcc <= 256 ? 256 : 512;
  static constexpr int kBarOff = kStages * kStage;
  static constexpr int kBytes = kBarOff + 512 + 1024;  // barriers, TMEM address, item ring, alignment slack
};

// Work item i: (m, parity, row tile) packed as m | par << 16 | tile << 17.
__device__ __forceinline__ void item_decode(uint32_t v, int* m, int* par, int* tile) {
  *m = (int)(v & 0xffffu);
  *par = (int)((v >> 16) & 1u);
  *tile = (int)(v >> 17);
}

template <int NC>
__global__ void __launch_bounds__(kTcThreads, 1)
contract_tc_kernel(int Nl, int nchunks, const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   const uint32_t* __restrict__ items, int nitems, const int16_t* __restrict__ rexp,
                   const int16_t* __restrict__ cexp, int ncols, const TcOut out, unsigned* __restrict__ err,
                   unsigned* __restrict__ next_item, int stall) {
  using L = TcLayout<NC>;
  constexpr int S = L::kStages;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L::kBarOff);
  uint64_t* empty = full + S;
  uint64_t* tfull = empty + S;       // [2] MMA -> epilogue
  uint64_t* tempty = tfull + 2;      // [2] epilogue -> MMA
  uint64_t* drain = tempty + 2;      // [1] every MMA issued has completed
  uint64_t* item_full = drain + 1;   // [kItemRing] producer -> MMA issuer and epilogue
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(item_full + kItemRing);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  int* item_ring = reinterpret_cast<int*>(tmem_slot + 2);  // [kItemRing] claimed item, -1 = none left
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&tfull[b], 1);
      tc::mbar_init(&tempty[b], kEpiWarps);
    }
    tc::mbar_init(drain, 1);
    for (int r = 0; r < kItemRing; ++r) tc::mbar_init(&item_full[r], 1);
    *abort_flag = 0;
    tc::mbar_fence_init();
  }
  if (warp == 1) tc::tmem_alloc(tmem_slot, L::kTmemCols);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  auto fail = [&]() {
    *abort_flag = 1;
    atomicOr(err, kFlagTimeout);
  };

  if (warp == 0) {
    // ---- TMA producer (one thread) --------------------------------------------------------
    if (lane == 0) {
      uint32_t n = 0, j = 0;
      bool ok = true;
      while (ok) {
        int it = (int)atomicAdd(next_item, 1u);
        if (it >= nitems) it = -1;
        item_ring[j % kItemRing] = it;
        tc::mbar_arrive(&item_full[j % kItemRing]);  // releases the ring entry
        ++j;
        if (it < 0) break;
        int m, par, tile;
        item_decode(items[it], &m, &par, &tile);
        const int ne = (Nl - m + 1) / 2;
        const int row0 = (int)hp_index(m, m, Nl) + (par ? ne : 0) + tile * kTileRows;
        const int zb = (m * 2 + par) * 4;
        for (int c = 0; c < nchunks; ++c, ++n) {
          const int s = n % S;
          const uint32_t use = n / S;
          if (use > 0 && !tc::mbar_wait(&empty[s], (use - 1) & 1, abort_flag)) {
            fail();
            ok = false;
            break;
          }
          uint8_t* st = smem + s * L::kStage;
          tc::mbar_arrive_expect_tx(&full[s], (uint32_t)L::kStage);
          tc::tma_load_3d(st, &tmA, c * kChunk, row0, 0, &full[s]);
          tc::tma_load_3d(st + L::kA, &tmB, c * kChunk, 0, zb, &full[s]);
        }
      }
      // No TMA may still be writing shared memory when the block leaves: wait for the last
      // stages issued (their phases have completed already unless the run aborted).
      const uint32_t last = n < (uint32_t)S ? n : (uint32_t)S;
      for (uint32_t k = 0; k < last; ++k) {
        const uint32_t i = n - 1 - k;
        const long long t0 = clock64();
        while (!tc::mbar_try_wait_for(&full[i % S], (i / S) & 1, 10000u))
          if (clock64() - t0 > (1ll << 31)) {
            atomicOr(err, kFlagTimeout);
            break;
          }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ---- MMA issuer (one thread) ----------------------------------------------------------
    if (lane == 0) {
      constexpr uint32_t i4 = tc::idesc_i8(kTileRows, 4 * NC, true, true);
      constexpr uint32_t i3 = tc::idesc_i8(kTileRows, 3 * NC, true, true);
      constexpr uint32_t i2 = tc::idesc_i8(kTileRows, 2 * NC, true, true);
      constexpr uint32_t i1 = tc::idesc_i8(kTileRows, NC, true, true);
      constexpr uint32_t kPlaneA = kTileRows * kChunk, kPlaneB = NC * kChunk;
      uint32_t n = 0;
      bool ok = true;
      for (uint32_t iter = 0; ok; ++iter) {
        if (!tc::mbar_wait(&item_full[iter % kItemRing], (iter / kItemRing) & 1, abort_flag)) {
          fail();
          break;
        }
        if (item_ring[iter % kItemRing] < 0) break;
        const uint32_t b = L::kBufs == 2 ? (iter & 1) : 0;
        const uint32_t use_b = L::kBufs == 2 ? (iter >> 1) : iter;
        if (use_b > 0 && !tc::mbar_wait(&tempty[b], (use_b - 1) & 1, abort_flag)) {
          fail();
          ok = false;
          break;
        }
        tc::tc_fence_after();
        const uint32_t d = tmem + b * L::kAcc;
        for (int c = 0; c < nchunks; ++c, ++n) {
          const int s = n % S;
          if (!tc::mbar_wait(&full[s], (n / S) & 1, abort_flag)) {
            fail();
            ok = false;
            break;
          }
          tc::tc_fence_after();
          const uint32_t A = tc::smem_addr(smem + s * L::kStage);
          const uint32_t B = A + L::kA;
#pragma unroll
          for (int kk = 0; kk < kChunk / 32; ++kk) {
            const uint32_t off = kk * 32;  // 32 int8 along K per MMA
            const bool acc = c > 0 || kk > 0;
            const uint64_t a0 = tc::desc_k_sw64(A + off), a1 = tc::desc_k_sw64(A + kPlaneA + off),
                           a2 = tc::desc_k_sw64(A + 2 * kPlaneA + off), a3 = tc::desc_k_sw64(A + 3 * kPlaneA + off);
            const uint64_t b0 = tc::desc_k_sw64(B + off), b1 = tc::desc_k_sw64(B + kPlaneB + off);
            // each first MMA of an item starts only columns no earlier MMA of it wrote
            tc::mma_i8(d, a0, b0, i1, acc);                // W0
            tc::mma_i8(d + NC, a1, b0, i4, acc);           // W1..W4
            tc::mma_i8(d + NC, a0, b1, i3, true);          // W1..W3
            tc::mma_i8(d + 2 * NC, a2, b0, i3, true);      // W2..W4
            tc::mma_i8(d + 3 * NC, a3, b0, i2, true);      // W3..W4
          }
          tc::mma_commit(&empty[s]);
        }
        // stall != 0 (test hook): block 0 never signals its first tile, so the epilogue's
        // bounded wait runs out and the launch reports kFlagTimeout
        if (ok && !(stall && blockIdx.x == 0 && iter == 0)) tc::mma_commit(&tfull[b]);
      }
      // every MMA issued has completed before TMEM is released
      tc::mma_commit(drain);
      const long long t0 = clock64();
      while (!tc::mbar_try_wait_for(drain, 0, 10000u))
        if (clock64() - t0 > (1ll << 31)) {
          atomicOr(err, kFlagTimeout);
          break;
        }
    }
    __syncwarp();
  } else {
    // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 -----------------------------
    const int q = warp & 3;
    for (uint32_t iter = 0;; ++iter) {
      if (*abort_flag || !tc::mbar_wait(&item_full[iter % kItemRing], (iter / kItemRing) & 1, abort_flag)) {
        if (lane == 0) fail();
        break;
      }
      const int it = item_ring[iter % kItemRing];
      if (it < 0) break;
      const uint32_t b = L::kBufs == 2 ? (iter & 1) : 0;
      const uint32_t use_b = L::kBufs == 2 ? (iter >> 1) : iter;
      if (*abort_flag || !tc::mbar_wait(&tfull[b], use_b & 1, abort_flag)) {
        if (lane == 0) fail();
        break;
      }
      tc::tc_fence_after();
      int m, par, tile;
      item_decode(items[it], &m, &par, &tile);
      const int ne = (Nl - m + 1) / 2;
      const int nrows = par ? (Nl - m) / 2 : ne;
      const int rr = tile * kTileRows + 32 * q + lane;  // row within the (m, parity) block
      const bool valid = rr < nrows;
      const int64_t g = hp_index(m, m, Nl) + (par ? ne : 0) + rr;
      const int er = valid ? rexp[g] : 0;
      const int l = m + par + 2 * rr;
      const int64_t idx = hp_index(l, m, Nl);
      const uint32_t tbase = tmem + ((uint32_t)(32 * q) << 16) + b * L::kAcc;
#pragma unroll
      for (int c0 = 0; c0 < NC; c0 += 16) {
        uint32_t w[5][16];
#pragma unroll
        for (int k = 0; k < 5; ++k) tc::tmem_ld16_nowait(tbase + k * NC + c0, w[k]);
        tc::tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int col = c0 + i;
          if (!valid || col >= ncols) continue;
          const long long V = ((long long)(int)w[0][i] << 32) + ((long long)(int)w[1][i] << 24) +
                              ((long long)(int)w[2][i] << 16) + ((long long)(int)w[3][i] << 8) +
                              (long long)(int)w[4][i];
          const int map = col >> 2, h = (col >> 1) & 1, ri = col & 1;
          const double v = ldexp((double)V, er + cexp[2 * map + h] - 46);
          double* o = h ? out.pol[map] : out.equ[map];
          o[2 * idx + ri] = v;
        }
      }
      tc::tc_fence_before();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&tempty[b]);
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  if (warp == 1) tc::tmem_dealloc(tmem, L::kTmemCols);
}

// Test hook (dsht_test_stall_next_contraction): the next launch leaves one wait unsatisfied.
std::atomic<int> g_stall_next{0};

PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &qr) == cudaSuccess &&
        qr == cudaDriverEntryPointSuccess)
      encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  return encode;
}

// 3D uint8 tensor map (x = K bytes of a row, y = row, z = plane), 64-byte swizzle, boxes
// of 64 x box_rows x 4.
int make_digit_tmap(CUtensorMap* tm, const void* base, int64_t kp, int64_t rows, int64_t planes, int box_rows) {
  auto encode = tmap_encoder();
  if (!encode) return set_error(DSHT_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  const cuuint64_t dims[3] = {(cuuint64_t)kp, (cuuint64_t)rows, (cuuint64_t)planes};
  const cuuint64_t strides[2] = {(cuuint64_t)kp, (cuuint64_t)(kp * rows)};
  const cuuint32_t box[3] = {(cuuint32_t)kChunk, (cuuint32_t)box_rows, 4u};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = encode(tm, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides, box, estr,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(DSHT_ERR_CUDA, "cuTensorMapEncodeTiled (digits) failed (%d)", (int)r);
  return DSHT_OK;
}

template <int NC>
int tc_launch(const Geometry& g, const CUtensorMap& tmA, const uint8_t* fdig, int fdig_cols, const uint32_t* items,
              int nitems, const int16_t* rexp, const int16_t* cexp, int ncols, const TcOut& out, unsigned* flags,
              unsigned* next_item, cudaStream_t s) {
  using L = TcLayout<NC>;
  alignas(64) CUtensorMap tmB;
  const int kp = digit_kp(g.Nx);
  // fold digits [Nl][2][4][fdig_cols][Kp] viewed as (Kp, fdig_cols, Nl * 8); boxes of NC
  // columns (columns beyond fdig_cols read as zeros, those beyond ncols are not stored)
  int rc = make_digit_tmap(&tmB, fdig, kp, fdig_cols, (int64_t)g.Nl * 8, NC);
  if (rc) return rc;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = nitems < sms ? nitems : sms;
  auto kern = contract_tc_kernel<NC>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L::kBytes);
  const int stall = g_stall_next.exchange(0);
  cudaMemsetAsync(next_item, 0, sizeof(unsigned), s);
  kern<<<grid, kTcThreads, L::kBytes, s>>>(g.Nl, kp / kChunk, tmA, tmB, items, nitems, rexp, cexp, ncols, out, flags,
                                           next_item, stall);
  count_launches(1);
  return DSHT_OK;
}

}  // namespace

int tc_fold_cols(int nmaps) { return nmaps <= 4 ? 16 : nmaps <= 8 ? 32 : 64; }

int make_table_digit_tmap(CUtensorMap* tm, const uint8_t* dig, int Nx, int64_t Nlm) {
  return make_digit_tmap(tm, dig, digit_kp(Nx), Nlm, 4, kTileRows);
}

std::vector<uint32_t> tc_items(int Nl) {
  std::vector<uint32_t> v;
  for (int m = 0; m < Nl; ++m)
    for (int par = 0; par < 2; ++par) {
      const int n = par ? (Nl - m) / 2 : (Nl - m + 1) / 2;
      for (int t = 0; t * kTileRows < n; ++t) v.push_back((uint32_t)m | ((uint32_t)par << 16) | ((uint32_t)t << 17));
    }
  return v;
}

int launch_contract_tc(const Geometry& g, const CUtensorMap& tmA, const uint32_t* items, int nitems,
                       const int16_t* rexp, const uint8_t* fdig, int fdig_cols, const int16_t* cexp, int nmaps,
                       const TcOut& out, unsigned* flags, unsigned* next_item, cudaStream_t s) {
  if (nmaps < 1 || nmaps > kTcMaxMaps || 4 * nmaps > fdig_cols)
    return set_error(DSHT_ERR_INVALID, "tensor-core pass of %d maps (%d fold columns)", nmaps, fdig_cols);
  const int nc = tc_fold_cols(nmaps);
  const int ncols = 4 * nmaps;
  auto go = [&](auto launch) {
    return launch(g, tmA, fdig, fdig_cols, items, nitems, rexp, cexp, ncols, out, flags, next_item, s);
  };
  if (nc == 16) return go(tc_launch<16>);
  if (nc == 32) return go(tc_launch<32>);
  return go(tc_launch<64>);
}

}  // namespace dsht

extern "C" int dsht_test_stall_next_contraction(void) {
  dsht::g_stall_next.store(1);
  return DSHT_OK;
}
