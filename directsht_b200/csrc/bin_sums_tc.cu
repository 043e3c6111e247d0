// Tensor-core per-bin sums for the mixed-precision path (tcgen05 kind::i8, exact S32
// accumulation of fixed-point slices -- an Ozaki-style split).
//
// For one piece (<= piece_max points of one bin) the sums
//   v[k][m] = sum_p g_k(p) e^{i m phi_p},  k = 0..3 Hermite weights,  m < Nl
// (sht/shared_interp_funcs.py:88-105) are one real GEMM once m is factored as
// m = Cf a + c (a < 16):  e^{i m phi} = e^{i Cf a phi} e^{i c phi}, so
//   D[row, col] = sum_p L[row, p] R[col, p]
// with rows = 2 (16 k + a) + (re|im) of L = g_k e^{i Cf a phi} / scale   (M = 128)
// and  cols = (re|im, c)    of R = e^{i c phi}                           (N = 2 CH),
// and Vr = D[re,Rr] - D[im,Ri], Vi = D[re,Ri] + D[im,Rr] (neighbouring TMEM lanes, one
// warp shuffle).  The points of the piece are
// the K dimension, 64 per pipeline stage.  When Cf > CH the c range is covered by
// Cf/CH column groups (grid.y).
//
// Operands: per point, FP64 anchors (powers of e^{i phi} by squaring and short
// recurrences) stored as FP32; per value, X = rint(x q) with q = 2^22 - 2^10 by one FP32
// FMA against 1.5*2^23, split into its bytes X = X0 2^16 + X1 2^8 + X2 (X0 signed,
// X1, X2 unsigned).  Eight tcgen05.mma.kind::i8 per K step accumulate exactly in S32
// TMEM: W0 = A0B0, W1 = A0B1 + A1B0, W2 = A0B2 + A1B1 + A2B0, W3 = A1B2 + A2B1, and
// D = (2^32 W0 + 2^24 W1 + 2^16 W2 + 2^8 W3) / q^2 in FP64.  Integer accumulation has no
// rounding (FP32 tensor-core accumulation truncates and biases long sums), so the error
// is the quantisation plus the dropped A2B2 term: about 5.6e-8 rms per product, relative
// to the piece's largest |L|, mean below 1e-9.  Pieces of up to 2048 points keep every
// S32 sum below 2^31.
//
// Warp roles: warps 0-7 generate operands into a 3-stage shared-memory ring (64-byte
// swizzled K-major int8 tiles) and run the epilogue (warps 0-3 own TMEM lanes 0-127);
// warp 8 issues the MMAs from one thread.  Stages are handed over with mbarriers (full:
// producers -> MMA, empty: tcgen05.commit -> producers).  Every wait is bounded.
#include "dsht_internal.cuh"
#include "tc_ptx.cuh"

namespace dsht {
namespace {

constexpr int kBK = 64;                 // points per stage: one 64-byte row of int8
constexpr int kProducers = 256;         // warps 0-7
constexpr int kThreads = kProducers + 32;
constexpr int kM = 128;
constexpr int kStages = 3;
constexpr float kQf = 4193280.0f;       // 2^22 - 2^10: |X| < 2^22, so X >> 16 fits int8
constexpr double kQ = 4193280.0;
constexpr float kMagic = 12582912.0f;   // 1.5 * 2^23 (bit pattern 0x4B400000)
// Per-k scale factors: |h_1|, |h_3| <= 4/27 while max(h_0, h_2) >= 1/2, so
// |w h_1|, |w h_3| <= (8/27) max_k |w h_k| over a piece; their rows use 0.3 of the
// piece's scale (1.75 more bits).
__device__ constexpr double kKScale[4] = {1.0, 0.3, 1.0, 0.3};
__device__ constexpr double kInvKScale[4] = {1.0, 1.0 / 0.3, 1.0, 1.0 / 0.3};

struct cplx {
  double re, im;
};
__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
// rint(x q) for |x| <= 1: one FMA puts x q into the binade of 1.5*2^23, where the
// float's bit pattern minus that of 1.5*2^23 is the rounded integer.
__device__ __forceinline__ int quant(float x) { return __float_as_int(fmaf(x, kQf, kMagic)) - 0x4B400000; }

// Byte B of a, b, c, d packed into one word (the slices of X are its bytes 2, 1, 0).
template <int B>
__device__ __forceinline__ uint32_t pack4(int a, int b, int c, int d) {
  const uint32_t lo = __byte_perm((uint32_t)a, (uint32_t)b, B | ((4 + B) << 4));
  const uint32_t hi = __byte_perm((uint32_t)c, (uint32_t)d, B | ((4 + B) << 4));
  return __byte_perm(lo, hi, 0x5410);
}

__device__ __forceinline__ void bar_producers() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

// Shared-memory descriptor: K-major operand in the 64-byte swizzle layout (rows of 64 B,
// 8-row atoms of 512 B packed: stride byte offset 512).
__device__ __forceinline__ uint64_t desc_k_sw64(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;
  d |= (uint64_t)(512u >> 4) << 32;
  d |= (uint64_t)1u << 46;
  d |= (uint64_t)4u << 61;  // 64-byte swizzle
  return d;
}

// Instruction descriptor of kind::i8 (D s32, both K-major, M x N); a/b signed or not.
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N, bool a_signed, bool b_signed) {
  return (2u << 4) | ((a_signed ? 1u : 0u) << 7) | ((b_signed ? 1u : 0u) << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate)
      : "memory");
}

template <int CH>
struct Layout {
  static constexpr int N = 2 * CH;
  static constexpr int kTileA = kM * 64;                      // bytes of one A slice tile
  static constexpr int kTileB = N * 64;
  static constexpr int kStage = 3 * kTileA + 3 * kTileB;      // A0..A2, B0..B2
  static constexpr int kAnchorBytes = kBK * (8 + (CH / 2 + 1) * 8 + 17 * 8 + 4 * 4);
  static constexpr int kUnion = 2 * kAnchorBytes;
  static constexpr int kUnionOff = kStages * kStage;
  static constexpr int kMiscOff = kUnionOff + ((kUnion + 1023) / 1024) * 1024;
  static constexpr int kBytes = kMiscOff + 256 + 1024;        // + alignment slack
  // W0..W3 in columns [jN, (j+1)N); the epilogue reads 32-column windows starting below
  // 3N + CH, so 3N + CH + 32 columns must exist.
  static constexpr int kNeed = (4 * N > 3 * N + CH + 32) ? 4 * N : 3 * N + CH + 32;
  static constexpr uint32_t kTmemCols = (kNeed <= 32) ? 32 : (kNeed <= 64) ? 64 : (kNeed <= 128) ? 128
                                       : (kNeed <= 256) ? 256 : 512;
  static_assert(kNeed <= 512, "accumulators must fit TMEM");
};

template <int CH>
__global__ void __launch_bounds__(kThreads, 1)
bin_sums_tc_kernel(int Nl, int Cf, int64_t Npay, const double* __restrict__ pay, const int* __restrict__ npieces_p,
                   int64_t pmax, const int64_t* __restrict__ piece_start, const int* __restrict__ piece_len,
                   const uint32_t* __restrict__ piecemax,
                   float* __restrict__ partial, unsigned* __restrict__ err_flags) {
  using Lay = Layout<CH>;
  constexpr int N = Lay::N;
  constexpr int S = kStages;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* uni = smem + Lay::kUnionOff;
  // Row strides are padded by one entry so that lanes holding consecutive points hit
  // different banks.
  constexpr int kEcStride = CH / 2 + 1, kEaStride = 17;
  // Two anchor buffers (block b uses buffer b & 1), each laid out as
  //   e1 [64] e^{i phi} | ec [64][CH/2+1] e^{i (cbase + 2u) phi} | ea [64][17] e^{i Cf a phi} | gk [64][4]
  auto e1_of = [&](int buf) { return reinterpret_cast<float2*>(uni + buf * Lay::kAnchorBytes); };
  auto ec_of = [&](int buf) { return e1_of(buf) + kBK; };
  auto ea_of = [&](int buf) { return ec_of(buf) + kBK * kEcStride; };
  auto gk_of = [&](int buf) { return reinterpret_cast<float*>(ea_of(buf) + kBK * kEaStride); };
  uint8_t* misc = smem + Lay::kMiscOff;
  uint64_t* full = reinterpret_cast<uint64_t*>(misc);            // [S]
  uint64_t* empty = full + S;                                    // [S]
  uint64_t* done = full + 2 * S;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(misc + 128);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(misc + 132);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cbase = blockIdx.y * CH;
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      tc::mbar_init(&full[s], kProducers / 32);
      tc::mbar_init(&empty[s], 1);
    }
    tc::mbar_init(done, 1);
    *abort_flag = 0;
    tc::mbar_fence_init();
  }
  if (warp == 0) tc::tmem_alloc(tmem_slot, Lay::kTmemCols);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const int npieces = (int)min((int64_t)*npieces_p, pmax);
  uint32_t blk_count = 0;
  uint32_t piece_iter = 0;

  for (int piece = blockIdx.x; piece < npieces; piece += gridDim.x, ++piece_iter) {
    const int64_t start = piece_start[piece];
    const int len = piece_len[piece];
    const int nblk = (len + kBK - 1) / kBK;

    if (warp < 8) {
      // ---- scale: largest |g_k| of the piece (gathered by the sort) -------------------
      // Round the scale up so that |g_k| / scale <= 1 holds after rounding too.
      double scale = (double)__uint_as_float(piecemax[piece]) * (1.0 + 1.0 / 1048576.0);
      if (!(scale > 0.0) || !isfinite(scale)) scale = 1.0;
      const double inv_scale = 1.0 / scale;

      // ---- phase 1: anchors of block b (FP64 math, FP32 storage) into buffer b & 1 ----
      // Threads 0-127: ec of point t%64, entries [h CH/4, (h+1) CH/4), h = t/64.
      // Threads 128-255: ea of point t%64, entries [8h, 8h+8), and e1, g for h = 1.
      // Lanes of a warp hold consecutive points (warp-uniform branches); every thread runs
      // two interleaved recurrences so that FP64 latency overlaps.  All starting powers are
      // powers of two of e^{i phi} (CH, Cf are), so they come from straight-line squaring.
      // The record of block b+1 is loaded into registers while block b is processed.
      const int p_me = tid & 63, hq = (tid >> 6) & 1;
      const bool is_ec = tid < 128;
      const bool need_wt = !is_ec && hq == 1;
      double r_c = 0.0, r_s = 0.0, r_w = 0.0, r_t = 0.0;  // record of the next block's point
      auto load_rec = [&](int b) {
        if (b * kBK + p_me < len) {
          const double* r = pay + (size_t)kRec * (start + (int64_t)b * kBK + p_me);
          r_c = r[0];
          r_s = r[1];
          if (need_wt) {
            r_w = r[2];
            r_t = r[3];
          }
        }
      };
      load_rec(0);
      auto phase1 = [&](int b) {
        if (*abort_flag) return;
        const int buf = b & 1;
        float2* e1 = e1_of(buf);
        float2* ec = ec_of(buf);
        float2* ea = ea_of(buf);
        float* gk = gk_of(buf);
        const int np = min(kBK, len - b * kBK);
        const int p = p_me;
        const cplx z1 = {r_c, r_s};
        const double wv = r_w, tv = r_t;
        if (b + 1 < nblk) load_rec(b + 1);
        if (p < np) {
          // z^(2^j) for 2^j = CH/4, CH/2, CH
          cplx zq = z1;
#pragma unroll
          for (int q = 1; q < CH / 4; q <<= 1) zq = cmul(zq, zq);
          const cplx zh = cmul(zq, zq);      // z^(CH/2)
          const cplx zf = cmul(zh, zh);      // z^CH
          if (is_ec) {
            constexpr int H = CH / 8;  // entries per chain
            const int u0 = hq * (CH / 4);
            const cplx st = cmul(z1, z1);
            // za = z^(cbase + 2 u0): cbase in {0, CH}, 2 u0 in {0, CH/2}
            cplx za = hq ? zh : cplx{1.0, 0.0};
            if (cbase) za = cmul(za, zf);
            cplx zb = cmul(za, zq);            // z^(cbase + 2 u0 + CH/4) = za st^H
            for (int u = 0; u < H; ++u) {
              ec[p * kEcStride + u0 + u] = make_float2((float)za.re, (float)za.im);
              ec[p * kEcStride + u0 + H + u] = make_float2((float)zb.re, (float)zb.im);
              za = cmul(za, st);
              zb = cmul(zb, st);
            }
          } else {
            const int a0 = 8 * hq;
            const cplx st = (Cf == CH) ? zf : cmul(zf, zf);  // z^Cf, Cf in {CH, 2 CH}
            const cplx s2 = cmul(st, st), s4 = cmul(s2, s2);
            cplx za = hq ? cmul(s4, s4) : cplx{1.0, 0.0};     // st^a0
            cplx zb = cmul(za, s4);
#pragma unroll
            for (int a = 0; a < 4; ++a) {
              ea[p * kEaStride + a0 + a] = make_float2((float)za.re, (float)za.im);
              ea[p * kEaStride + a0 + 4 + a] = make_float2((float)zb.re, (float)zb.im);
              za = cmul(za, st);
              zb = cmul(zb, st);
            }
            if (hq == 1) {
              e1[p] = make_float2((float)z1.re, (float)z1.im);
              double h[4];
              hermite(tv, wv, h);
#pragma unroll
              for (int k = 0; k < 4; ++k) gk[p * 4 + k] = (float)(h[k] * inv_scale * kInvKScale[k]);
            }
          }
        } else {  // padding points contribute zero
          if (is_ec) {
            for (int u = hq * (CH / 4); u < (hq + 1) * (CH / 4); ++u) ec[p * kEcStride + u] = make_float2(0.f, 0.f);
          } else {
            for (int a = 8 * hq; a < 8 * hq + 8; ++a) ea[p * kEaStride + a] = make_float2(0.f, 0.f);
            if (hq == 1) {
              e1[p] = make_float2(0.f, 0.f);
#pragma unroll
              for (int k = 0; k < 4; ++k) gk[p * 4 + k] = 0.f;
            }
          }
        }
      };

      phase1(0);
      bar_producers();
      for (int b = 0; b < nblk; ++b) {
        const uint32_t g = blk_count + b;
        const int stage = g % S;
        const uint32_t use = g / S;
        if (b + 1 < nblk) phase1(b + 1);  // overlaps with the other warps' slicing
        // ---- wait until the MMAs that last read this stage are done -------------------
        if (use > 0 && !*abort_flag) {
          if (!tc::mbar_wait(&empty[stage], (use - 1) & 1, abort_flag)) {
            *abort_flag = 1;
            atomicOr(err_flags, kFlagTimeout);
          }
        }
        // ---- phase 2: int8 slice tiles of block b from buffer b & 1 ---------------------
        uint8_t* st_base = smem + stage * Lay::kStage;
        if (!*abort_flag) {
          const int buf = b & 1;
          const float2* e1 = e1_of(buf);
          const float2* ec = ec_of(buf);
          const float2* ea = ea_of(buf);
          const float* gk = gk_of(buf);
          constexpr int nB = 4 * (CH / 2);  // (16-point chunk h, c pair)
          constexpr int nA = 4 * 32;        // (16-point chunk h, k, a pair)
          for (int u = tid; u < nB + nA; u += kProducers) {
            int h, rows[4];
            uint8_t* base;
            int tile_bytes;
            uint32_t w[4][3][4];  // [value][slice][word of 4 points]
            const bool isB = u < nB;
            int cp = 0, k = 0, ap = 0;
            if (isB) {
              h = u / (CH / 2);
              cp = u % (CH / 2);
              rows[0] = 2 * cp;            // Re e^{i c phi},       c = 2cp
              rows[1] = CH + 2 * cp;       // Im e^{i c phi}
              rows[2] = 2 * cp + 1;        // Re e^{i (c+1) phi}
              rows[3] = CH + 2 * cp + 1;   // Im e^{i (c+1) phi}
              base = st_base + 3 * Lay::kTileA;
              tile_bytes = Lay::kTileB;
            } else {
              // A rows 2 (16 k + a) + (re|im): the two halves of a complex row sit in
              // neighbouring TMEM lanes, so the epilogue combines them with one shuffle.
              const int v = u - nB;
              h = v >> 5;
              k = (v & 31) >> 3;
              ap = v & 7;
              const int j0 = 16 * k + 2 * ap;
              rows[0] = 2 * j0;          // re, a = 2ap
              rows[1] = 2 * j0 + 1;      // im
              rows[2] = 2 * j0 + 2;      // re, a = 2ap + 1
              rows[3] = 2 * j0 + 3;      // im
              base = st_base;
              tile_bytes = Lay::kTileA;
            }
            // The first row each lane writes is chosen so that the eight lanes of a quarter
            // warp cover all eight 16-byte bank groups: B units swap the pair members on
            // lane bit 2; A units swap the a pair on lane bit 1 and re/im on lane bit 2.
            const bool odd = ((lane >> 2) & 1) != 0;
            const bool swap_a = !isB && ((lane >> 1) & 1) != 0;
            if (isB ? odd : swap_a) {
              const int r0 = rows[0], r1 = rows[1];
              rows[0] = rows[2];
              rows[1] = rows[3];
              rows[2] = r0;
              rows[3] = r1;
            }
            if (!isB && odd) {
              int r = rows[0];
              rows[0] = rows[1];
              rows[1] = r;
              r = rows[2];
              rows[2] = rows[3];
              rows[3] = r;
            }
#pragma unroll
            for (int t = 0; t < 4; ++t) {
              int X[4][4];  // [value][point]
#pragma unroll
              for (int jj = 0; jj < 4; ++jj) {
                const int p = 16 * h + 4 * t + jj;
                float v0, v1, v2, v3;
                if (isB) {
                  const float2 z = ec[p * kEcStride + cp];
                  const float2 s = e1[p];
                  v0 = z.x;
                  v1 = z.y;
                  v2 = fmaf(z.x, s.x, -z.y * s.y);
                  v3 = fmaf(z.x, s.y, z.y * s.x);
                } else {
                  const float gg = gk[p * 4 + k];
                  const float2 z0 = ea[p * kEaStride + 2 * ap + (swap_a ? 1 : 0)];
                  const float2 z1 = ea[p * kEaStride + 2 * ap + (swap_a ? 0 : 1)];
                  v0 = gg * (odd ? z0.y : z0.x);
                  v1 = gg * (odd ? z0.x : z0.y);
                  v2 = gg * (odd ? z1.y : z1.x);
                  v3 = gg * (odd ? z1.x : z1.y);
                }
                if (isB && odd) {
                  const float t0 = v0, t1 = v1;
                  v0 = v2;
                  v1 = v3;
                  v2 = t0;
                  v3 = t1;
                }
                X[0][jj] = quant(v0);
                X[1][jj] = quant(v1);
                X[2][jj] = quant(v2);
                X[3][jj] = quant(v3);
              }
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                // 4 x 4 byte transpose: slice s of the four points is byte (2 - s) of X.
                const uint32_t t0 = __byte_perm((uint32_t)X[e][0], (uint32_t)X[e][1], 0x5140);
                const uint32_t t1 = __byte_perm((uint32_t)X[e][0], (uint32_t)X[e][1], 0x7362);
                const uint32_t u0 = __byte_perm((uint32_t)X[e][2], (uint32_t)X[e][3], 0x5140);
                const uint32_t u1 = __byte_perm((uint32_t)X[e][2], (uint32_t)X[e][3], 0x7362);
                w[e][0][t] = __byte_perm(t1, u1, 0x5410);
                w[e][1][t] = __byte_perm(t0, u0, 0x7632);
                w[e][2][t] = __byte_perm(t0, u0, 0x5410);
              }
            }
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              uint8_t* rowp = base + rows[e] * 64 + ((h ^ ((rows[e] >> 1) & 3)) << 4);
#pragma unroll
              for (int sl = 0; sl < 3; ++sl)
                *reinterpret_cast<uint4*>(rowp + sl * tile_bytes) =
                    make_uint4(w[e][sl][0], w[e][sl][1], w[e][sl][2], w[e][sl][3]);
            }
          }
        }
        tc::fence_async_smem();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&full[stage]);
        bar_producers();  // anchors of block b consumed, anchors of block b+1 complete
      }

      // ---- epilogue: warps 0-3 own TMEM lanes 0-127 -----------------------------------
      // Lane r holds row r = 2 (16 k + a) + ri of D.  For every c:
      //   Vr = D[re, Rr] - D[im, Ri],  Vi = D[re, Ri] + D[im, Rr],
      // so each lane sends its D[., Ri] to its neighbour (lane r ^ 1) and keeps D[., Rr]:
      // the re lane writes Vr, the im lane Vi, for m = Cf a + cbase + c.
      if (warp < 4) {
        bool ok = !*abort_flag;
        if (ok && !tc::mbar_wait(done, piece_iter & 1, abort_flag)) {
          *abort_flag = 1;
          atomicOr(err_flags, kFlagTimeout);
          ok = false;
        }
        tc::tc_fence_after();
        const int r = tid;  // TMEM lane == GEMM row
        const int ri = r & 1, j = r >> 1;
        const int k = j >> 4, a = j & 15;
        const double f = scale * kKScale[k] / (kQ * kQ);
        const uint32_t lane_off = (uint32_t)(warp * 32) << 16;
        float* out = partial + ((size_t)piece * 8 + 2 * k + ri) * Nl;
        const int m0 = Cf * a + cbase;
        for (int cb = 0; cb < CH; cb += 8) {
          double drr[8], dri[8];
#pragma unroll
          for (int half = 0; half < 2; ++half) {
            const uint32_t col = (half ? CH : 0) + cb;
            uint32_t w0[8], w1[8], w2[8], w3[8];
            if (ok) {
              tc::tmem_ld8(tmem + lane_off + col, w0);
              tc::tmem_ld8(tmem + lane_off + N + col, w1);
              tc::tmem_ld8(tmem + lane_off + 2 * N + col, w2);
              tc::tmem_ld8(tmem + lane_off + 3 * N + col, w3);
            }
            double* dst = half ? dri : drr;
#pragma unroll
            for (int i = 0; i < 8; ++i)
              dst[i] = ok ? (4294967296.0 * (double)(int)w0[i] + 16777216.0 * (double)(int)w1[i] +
                             65536.0 * (double)(int)w2[i] + 256.0 * (double)(int)w3[i]) * f
                          : 0.0;
          }
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const double x = __shfl_xor_sync(0xffffffffu, dri[i], 1);
            const double v = ri ? x + drr[i] : drr[i] - x;
            if (m0 + cb + i < Nl) out[m0 + cb + i] = (float)v;
          }
        }
        tc::tc_fence_before();
      }
    } else {
      // ---- MMA issuer (one thread of warp 8) --------------------------------------------
      constexpr uint32_t iSS = idesc_i8(kM, N, true, true), iSU = idesc_i8(kM, N, true, false),
                         iUS = idesc_i8(kM, N, false, true), iUU = idesc_i8(kM, N, false, false);
      for (int b = 0; b < nblk && lane == 0; ++b) {
        const uint32_t g = blk_count + b;
        const int stage = g % S;
        const uint32_t use = g / S;
        bool ok = !*abort_flag;
        if (ok && !tc::mbar_wait(&full[stage], use & 1, abort_flag)) {
          *abort_flag = 1;
          atomicOr(err_flags, kFlagTimeout);
          ok = false;
        }
        tc::tc_fence_after();
        if (ok) {
          const uint32_t base = tc::smem_addr(smem + stage * Lay::kStage);
          uint32_t A[3], B[3];
#pragma unroll
          for (int t = 0; t < 3; ++t) {
            A[t] = base + t * Lay::kTileA;
            B[t] = base + 3 * Lay::kTileA + t * Lay::kTileB;
          }
#pragma unroll
          for (int kk = 0; kk < kBK / 32; ++kk) {
            const uint32_t off = kk * 32;  // 32 int8 along K
            const bool acc = (b > 0) || (kk > 0);
            const uint32_t W0 = tmem, W1 = tmem + N, W2 = tmem + 2 * N, W3 = tmem + 3 * N;
            const uint64_t a0 = desc_k_sw64(A[0] + off), a1 = desc_k_sw64(A[1] + off),
                           a2 = desc_k_sw64(A[2] + off);
            const uint64_t b0 = desc_k_sw64(B[0] + off), b1 = desc_k_sw64(B[1] + off),
                           b2 = desc_k_sw64(B[2] + off);
            mma_i8(W0, a0, b0, iSS, acc);
            mma_i8(W1, a0, b1, iSU, acc);
            mma_i8(W1, a1, b0, iUS, true);
            mma_i8(W2, a0, b2, iSU, acc);
            mma_i8(W2, a1, b1, iUU, true);
            mma_i8(W2, a2, b0, iUS, true);
            mma_i8(W3, a1, b2, iUU, acc);
            mma_i8(W3, a2, b1, iUU, true);
          }
        }
        tc::mma_commit(&empty[stage]);
      }
      if (lane == 0) tc::mma_commit(done);
      __syncwarp();
    }
    blk_count += nblk;
    __syncthreads();  // the epilogue has read TMEM; the next piece may overwrite it
    tc::tc_fence_after();
  }
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, Lay::kTmemCols);
  }
}

template <int CH>
void launch_ch(const Geometry& g, const Workspace& ws, int Cf, cudaStream_t s) {
  using Lay = Layout<CH>;
  cudaFuncSetAttribute(bin_sums_tc_kernel<CH>, cudaFuncAttributeMaxDynamicSharedMemorySize, Lay::kBytes);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int groups = Cf / CH;
  int64_t per = (sms + groups - 1) / groups;
  int64_t grid = ws.pmax < per ? ws.pmax : per;
  if (grid < 1) grid = 1;
  dim3 gd((unsigned)grid, groups);
  bin_sums_tc_kernel<CH><<<gd, kThreads, Lay::kBytes, s>>>(g.Nl, Cf, ws.npts, ws.pay, ws.npieces, ws.pmax,
                                                           ws.piece_start, ws.piece_len, ws.piecemax,
                                                           reinterpret_cast<float*>(ws.partial),
                                                           ws.flags);
  count_launches(1);
}

}  // namespace

int tc_inner_factor(int Nl) {
  int need = (Nl + 15) / 16;
  int C = 8;
  while (C < need) C *= 2;
  return C;
}

int launch_bin_sums_tc(const Geometry& g, const Workspace& ws, cudaStream_t s) {
  const int Cf = tc_inner_factor(g.Nl);
  switch (Cf) {
    case 8: launch_ch<8>(g, ws, 8, s); break;
    case 16: launch_ch<16>(g, ws, 16, s); break;
    case 32: launch_ch<32>(g, ws, 32, s); break;
    case 64: launch_ch<64>(g, ws, 64, s); break;
    case 128: launch_ch<64>(g, ws, 128, s); break;  // two column groups
    default: return set_error(DSHT_ERR_INVALID, "mixed precision supports Nl <= 2048 (Nl=%d)", g.Nl);
  }
  return DSHT_OK;
}

}  // namespace dsht
