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
// Operands: per point, FP64 anchors (powers of e^{i phi} by Chebyshev recurrences): the
// B values e^{i c phi} rounded to fixed point in FP64, e^{i Cf a phi} stored as FP32 and
// multiplied by g_k / scale in FP32 by the slicers; per value, X = rint(x q) with
// q = 2^22 - 2^10 (one DFMA against 1.5*2^52, or one FP32 FMA against 1.5*2^23),
// written in balanced base-256 digits X = X0 2^16 + X1 2^8 + X2
// with every digit a signed byte: the bytes of Z = (X + 0x8080) ^ 0x8080 (adding 128 to
// the two low digit positions and flipping their top bits maps [0, 255] onto
// [-128, 127]).  Five tcgen05.mma.kind::i8 per K step accumulate exactly in S32 TMEM:
// W0 = A0B0, W1 = A0B1 + A1B0, W2 = A0B2 + A1B1 + A2B0, W3 = A1B2 + A2B1 (B0 and B1 form
// one 2N-row operand, so A_i [B0|B1] adds to W_i and W_(i+1) in one instruction), and
// D = (2^32 W0 + 2^24 W1 + 2^16 W2 + 2^8 W3) / q^2 in FP64.  Integer accumulation has no
// rounding (FP32 tensor-core accumulation truncates and biases long sums), so the error
// is the quantisation plus the dropped A2B2 term: about 5.6e-8 rms per product, relative
// to the piece's largest |L|, mean below 1e-9.  Pieces of up to 2048 points keep every
// S32 sum below 2^31.
//
// Warp roles: warps 6-9 (one per SM sub-partition) compute the FP64 anchors of a block
// into one of two anchor buffers, one block ahead, two threads per point (warps 6-7 the
// heavier half, on the sub-partitions without a B slicer warp); warps 0-5
// quantise and slice them into a ring of 64-byte-swizzled K-major int8 tiles (warps 0-1
// the B tiles, 2-5 the A tiles); warp 10 issues the MMAs from one thread; warps 0-3 run
// each piece's epilogue (TMEM lanes 0-127) while warps 4-5 and the anchor warps start the
// next piece.  Hand-overs are mbarriers (afull/aempty: anchors <-> slicers, full/empty:
// slicers <-> MMA via tcgen05.commit, done: MMA -> epilogue, tfree: epilogue -> MMA).
// Every wait is bounded.
//
// FP64 is the limiting pipe: while int8 MMAs run, an SM sub-partition issues about one
// FP64 warp instruction in 16 clocks (one in 2 on an SM that has not used its tensor
// cores, about one in 5 after), while FP32 keeps its full rate.  So the FP64 work is
// spread over all four sub-partitions and kept to recurrences of one DFMA per value.
#include "dsht_internal.cuh"
#include "tc_ptx.cuh"

namespace dsht {
namespace {

constexpr int kBK = 64;                 // points per stage: one 64-byte row of int8
constexpr int kSlicerWarps = 6;         // warps 0-5: int8 slice tiles (0-3: epilogue too)
constexpr int kAnchorWarps = 4;         // warps 6-9: FP64 anchors, one block ahead
constexpr int kBThreads = 64;           // slicer threads 0-63: B tiles, 64-191: A tiles
constexpr int kSlicers = 32 * kSlicerWarps;
constexpr int kThreads = 32 * (kSlicerWarps + kAnchorWarps + 1);  // + warp 10: MMA issuer
constexpr int kM = 128;
constexpr float kQf = 4193280.0f;       // 2^22 - 2^10: |X| < 2^22, so X >> 16 fits int8
constexpr double kQ = 4193280.0;
constexpr float kMagic = 12582912.0f;   // 1.5 * 2^23 (bit pattern 0x4B400000)
// Per-k scale factors: |h_1|, |h_3| <= 4/27 while max(h_0, h_2) >= 1/2, so
// |w h_1|, |w h_3| <= (8/27) max_k |w h_k| over a piece; their rows use 0.3 of the
// piece's scale (1.75 more bits).
__device__ constexpr double kKScale[4] = {1.0, 0.3, 1.0, 0.3};
__device__ constexpr double kInvKScale[4] = {1.0, 1.0 / 0.3, 1.0, 1.0 / 0.3};

// Fixed-point scale of a piece: its largest |g_k| (float bits from the sort), rounded up
// so that |g_k| / scale <= 1 holds after rounding too.
__device__ __forceinline__ double tc_scale(uint32_t bits) {
  const double s = (double)__uint_as_float(bits) * (1.0 + 1.0 / 1048576.0);
  return (s > 0.0 && isfinite(s)) ? s : 1.0;
}

struct cplx {
  double re, im;
};
__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
// Z = (rint(x q) + 0x8080) ^ 0x8080 of an FP64 value, whose bytes are the balanced
// digits: one DFMA puts x q + 0x8080 into the binade of 1.5*2^52, whose low word is then
// the rounded integer (no conversion instruction).
__device__ __forceinline__ int zfix(double x) {
  return __double2loint(fma(x, kQ, 6755399441055744.0 + 32896.0)) ^ 0x8080;
}

// rint(x q) + 0x8080 for |x| <= 1: one FMA puts x q into the binade of 1.5*2^23, where
// the float's bit pattern minus that of 1.5*2^23 is the rounded integer.  The flip of the
// two low digits' top bits is applied to the packed slice words.
__device__ __forceinline__ int quant(float x) {
  return __float_as_int(fmaf(x, kQf, kMagic)) - (0x4B400000 - 0x8080);
}

using tc::desc_k_sw64;
using tc::idesc_i8;
using tc::mma_i8;

// One slicing unit: 16 points (chunk h of the 64-point block) x 4 operand rows.  `values`
// writes the four fixed-point values of point pp into X[0..3]; they are byte-transposed
// into the three slice tiles (slice s of four points is byte 2 - s of X) and stored as
// 16-byte chunks of the 64-byte swizzled K-major rows (chunk h XOR (row / 2) & 3).  A
// quarter warp's first stores land in four distinct 16-byte bank groups.  kFlip: X is
// X + 0x8080 and the low slices' top bits are flipped here (else X is Z already).
template <bool kFlip, typename F>
__device__ __forceinline__ void slice_unit(uint8_t* base, int tile_bytes, int h, const int* rows, F values) {
  uint32_t w[4][3][4];  // [value][slice][word of 4 points]
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    int X[4][4];  // [point][value]
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) values(16 * h + 4 * t + jj, X[jj]);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const uint32_t t0 = __byte_perm((uint32_t)X[0][e], (uint32_t)X[1][e], 0x5140);
      const uint32_t t1 = __byte_perm((uint32_t)X[0][e], (uint32_t)X[1][e], 0x7362);
      const uint32_t u0 = __byte_perm((uint32_t)X[2][e], (uint32_t)X[3][e], 0x5140);
      const uint32_t u1 = __byte_perm((uint32_t)X[2][e], (uint32_t)X[3][e], 0x7362);
      w[e][0][t] = __byte_perm(t1, u1, 0x5410);
      w[e][1][t] = __byte_perm(t0, u0, 0x7632) ^ (kFlip ? 0x80808080u : 0u);
      w[e][2][t] = __byte_perm(t0, u0, 0x5410) ^ (kFlip ? 0x80808080u : 0u);
    }
  }
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    uint8_t* rowp = base + rows[e] * 64 + ((h ^ ((rows[e] >> 1) & 3)) << 4);
#pragma unroll
    for (int sl = 0; sl < 3; ++sl)
      *reinterpret_cast<uint4*>(rowp + sl * tile_bytes) = make_uint4(w[e][sl][0], w[e][sl][1], w[e][sl][2], w[e][sl][3]);
  }
}

template <int CH>
struct Layout {
  static constexpr int N = 2 * CH;
  static constexpr int kTileA = kM * 64;                      // bytes of one A slice tile
  static constexpr int kTileB = N * 64;
  static constexpr int kStage = 3 * kTileA + 3 * kTileB;      // A0..A2, B0..B2
  // Anchor buffer: eb [64][CH + 2] int2 (fixed-point e^{i c phi}; rows padded by 16 bytes
  // so that a quarter warp's 16-byte stores of different points hit different banks),
  // ea [64][17] float2, gk [64][4] float.
  static constexpr int kEbStride = CH + 2;                    // int2 per point
  static constexpr int kAnchorBytes = kBK * (kEbStride * 8 + 17 * 8 + 4 * 4);
  static constexpr int kUnion = 2 * kAnchorBytes;
  // As many operand stages (3 or 2) as fit beside the two anchor buffers.
  static constexpr int kStagesFit = (3 * kStage + ((kUnion + 1023) / 1024) * 1024 + 256 + 1024 <= 227 * 1024) ? 3 : 2;
  static constexpr int kUnionOff = kStagesFit * kStage;
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
bin_sums_tc_kernel(int Nl, int Cf, const double* __restrict__ pay, const int* __restrict__ npieces_p, int64_t pmax,
                   const int64_t* __restrict__ piece_start, const int* __restrict__ piece_len,
                   const uint32_t* __restrict__ piecemax, float* __restrict__ partial,
                   unsigned* __restrict__ err_flags) {
  using Lay = Layout<CH>;
  constexpr int N = Lay::N;
  constexpr int S = Lay::kStagesFit;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* uni = smem + Lay::kUnionOff;
  // Row strides are padded by one entry so that lanes holding consecutive points hit
  // different banks.
  constexpr int kEbStride = Lay::kEbStride, kEaStride = 17;
  // Two anchor buffers (global block g uses buffer g & 1), each laid out as
  //   eb [64][CH+2] int2 rint(q e^{i (cbase + c) phi}) | ea [64][17] e^{i Cf a phi} | gk [64][4]
  auto eb_of = [&](int buf) { return reinterpret_cast<int2*>(uni + buf * Lay::kAnchorBytes); };
  auto ea_of = [&](int buf) { return reinterpret_cast<float2*>(eb_of(buf) + kBK * kEbStride); };
  auto gk_of = [&](int buf) { return reinterpret_cast<float*>(ea_of(buf) + kBK * kEaStride); };
  uint8_t* misc = smem + Lay::kMiscOff;
  uint64_t* full = reinterpret_cast<uint64_t*>(misc);            // [S]  slicers -> MMA
  uint64_t* empty = full + S;                                    // [S]  MMA commit -> slicers
  uint64_t* done = full + 2 * S;                                 // [1]  MMA commit -> epilogue
  uint64_t* afull = done + 1;                                    // [2]  anchor warps -> slicers
  uint64_t* aempty = afull + 2;                                  // [2]  slicers -> anchor warps
  uint64_t* tfree = aempty + 2;                                  // [1]  epilogue -> MMA
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(misc + 192);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(misc + 196);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cbase = blockIdx.y * CH;
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      tc::mbar_init(&full[s], kSlicerWarps);
      tc::mbar_init(&empty[s], 1);
    }
    tc::mbar_init(done, 1);
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&afull[b], kAnchorWarps);
      tc::mbar_init(&aempty[b], kSlicerWarps);
    }
    tc::mbar_init(tfree, 4);
    *abort_flag = 0;
    tc::mbar_fence_init();
  }
  if (warp == 0) tc::tmem_alloc(tmem_slot, Lay::kTmemCols);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int npieces = (int)min((int64_t)*npieces_p, pmax);
  auto fail = [&]() {
    *abort_flag = 1;
    atomicOr(err_flags, kFlagTimeout);
  };

  if (warp >= kSlicerWarps && warp < kSlicerWarps + kAnchorWarps) {
    // ==== anchor warps: FP64 powers of e^{i phi} (FP32 storage) one block ahead ========
    // Two threads per point p of the block, one warp per SM sub-partition (FP64 is the
    // scarce pipe while the MMAs run): half 0 the c chains below CH/2 and the Hermite
    // weights, half 1 the c chains from CH/2 and e^{i Cf a phi}.  The powers come from
    // Chebyshev recurrences
    // E_(c+d) = 2 cos(d phi) E_c - E_(c-d) (one DFMA per component and value): four
    // interleaved chains of step 2 give e^{i c phi} for c = cbase + {2u, 2u + 1, CH/2 + 2u,
    // CH/2 + 2u + 1}, one chain of step Cf gives e^{i Cf a phi}; their seeds are products
    // of powers of two of e^{i phi}.  FP64 throughout (the recurrences lose about
    // steps^2 ulp, far below the 2^-22 fixed-point step).  Then the Hermite weights
    // g_k / scale.  The records of the point in the next two blocks are loaded meanwhile.
    // half 1 (the heavier) on warps 6-7, i.e. sub-partitions 2-3, where no B slicer warp runs
    const int p = (tid - kSlicers) & 63, half = ((tid - kSlicers) >> 6) ^ 1;
    uint32_t g = 0;
    for (int piece = blockIdx.x; piece < npieces && !*abort_flag; piece += gridDim.x) {
      const int64_t start = piece_start[piece];
      const int len = piece_len[piece];
      const int nblk = (len + kBK - 1) / kBK;
      const double inv_scale = 1.0 / tc_scale(piecemax[piece]);
      // Records of the point in the next two blocks (loads run two blocks ahead).
      double c0 = 0.0, s0 = 0.0, w0 = 0.0, t0 = 0.0, c1 = 0.0, s1 = 0.0, w1 = 0.0, t1 = 0.0;
      auto load = [&](int b, double& c, double& sn, double& w, double& t) {
        if (b * kBK + p < len) {
          const double2* rec = reinterpret_cast<const double2*>(pay + (size_t)kRec * (start + (int64_t)b * kBK + p));
          const double2 r0 = rec[0], r1 = rec[1];
          c = r0.x;
          sn = r0.y;
          w = r1.x;
          t = r1.y;
        }
      };
      load(0, c0, s0, w0, t0);
      if (nblk > 1) load(1, c1, s1, w1, t1);
      for (int b = 0; b < nblk; ++b, ++g) {
        const cplx z1 = {c0, s0};
        const double wv = w0, tv = t0;
        c0 = c1;
        s0 = s1;
        w0 = w1;
        t0 = t1;
        if (b + 2 < nblk) load(b + 2, c1, s1, w1, t1);
        const int buf = g & 1;
        if (g >= 2 && !tc::mbar_wait(&aempty[buf], ((g >> 1) - 1) & 1, abort_flag)) {
          fail();
          break;
        }
        int4* eb = reinterpret_cast<int4*>(eb_of(buf) + p * kEbStride);  // pairs of c
        float2* ea = ea_of(buf);
        float* gk = gk_of(buf);
        constexpr int H = CH / 4;  // c pairs per half of the c range
        if (b * kBK + p < len) {
          cplx zq = z1;
#pragma unroll
          for (int q = 1; q < CH / 4; q <<= 1) zq = cmul(zq, zq);  // z^(CH/4)
          const cplx zh = cmul(zq, zq);                              // z^(CH/2)
          const cplx zf = (cbase || half) ? cmul(zh, zh) : cplx{0.0, 0.0};  // z^CH
          const cplx z2 = cmul(z1, z1);
          const cplx zb = cbase ? zf : cplx{1.0, 0.0};               // z^cbase
          const double m2 = 2.0 * z2.re;                             // 2 cos 2 phi
          // chains: P = z^(c0 + 2u) and Q = P z with the previous value of each (u - 1);
          // c0 = cbase (half 0) or cbase + CH/2 (half 1)
          const cplx P0 = half ? cmul(zb, zh) : zb;
          cplx P = P0, Q = cmul(P0, z1);
          cplx Pp = cmul(P0, cplx{z2.re, -z2.im});                   // z^(c0 - 2)
          cplx Qp = cmul(P0, cplx{z1.re, -z1.im});                   // z^(c0 - 1)
          int4* ebh = eb + half * H;
#pragma unroll
          for (int u = 0; u < H; ++u) {
            // pair v = (c, c + 1) with c = 2v; pairs with bit 2 of v set are stored as
            // (c + 1, c) (see the slicers' row order)
            const int4 pq = make_int4(zfix(P.re), zfix(P.im), zfix(Q.re), zfix(Q.im));
            const bool swp = ((half * H + u) >> 2) & 1;
            ebh[u] = swp ? make_int4(pq.z, pq.w, pq.x, pq.y) : pq;
            if (u + 1 < H) {
              const cplx Pn = {fma(m2, P.re, -Pp.re), fma(m2, P.im, -Pp.im)};
              const cplx Qn = {fma(m2, Q.re, -Qp.re), fma(m2, Q.im, -Qp.im)};
              Pp = P;
              Qp = Q;
              P = Pn;
              Q = Qn;
            }
          }
          if (half) {
            const cplx sc = (Cf == CH) ? zf : cmul(zf, zf);         // z^Cf, Cf in {CH, 2 CH}
            const double mf = 2.0 * sc.re;                           // 2 cos Cf phi
            cplx Aa = {1.0, 0.0}, Ap = {sc.re, -sc.im};              // z^0, z^-Cf
#pragma unroll
            for (int u = 0; u < 16; ++u) {
              // a with bit 2 set: stored as (im, re) (see the slicers' row order)
              ea[p * kEaStride + u] = ((u >> 2) & 1) ? make_float2((float)Aa.im, (float)Aa.re)
                                                     : make_float2((float)Aa.re, (float)Aa.im);
              const cplx An = {fma(mf, Aa.re, -Ap.re), fma(mf, Aa.im, -Ap.im)};
              Ap = Aa;
              Aa = An;
            }
          } else {
            double h[4];
            hermite(tv, wv, h);
#pragma unroll
            for (int k = 0; k < 4; ++k) gk[p * 4 + k] = (float)(h[k] * inv_scale * kInvKScale[k]);
          }
        } else {  // padding points contribute zero
          for (int u = 0; u < H; ++u) eb[half * H + u] = make_int4(0, 0, 0, 0);
          if (half) {
            for (int u = 0; u < 16; ++u) ea[p * kEaStride + u] = make_float2(0.f, 0.f);
          } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) gk[p * 4 + k] = 0.f;
          }
        }
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&afull[buf]);
      }
    }
  } else if (warp < kSlicerWarps) {
    // ==== slicer warps: int8 slice tiles; warps 0-3 also run the epilogue ==============
    uint32_t g = 0, piece_iter = 0;
    for (int piece = blockIdx.x; piece < npieces; piece += gridDim.x, ++piece_iter) {
      const int len = piece_len[piece];
      const int nblk = (len + kBK - 1) / kBK;
      for (int b = 0; b < nblk; ++b, ++g) {
        const int stage = g % S;
        const uint32_t use = g / S;
        const int buf = g & 1;
        bool ok = !*abort_flag;
        if (ok && !tc::mbar_wait(&afull[buf], (g >> 1) & 1, abort_flag)) {
          fail();
          ok = false;
        }
        if (ok && use > 0 && !tc::mbar_wait(&empty[stage], (use - 1) & 1, abort_flag)) {
          fail();
          ok = false;
        }
        uint8_t* st_base = smem + stage * Lay::kStage;
        if (ok) {
          const int4* eb = reinterpret_cast<const int4*>(eb_of(buf));
          const float2* ea = ea_of(buf);
          const float* gk = gk_of(buf);
          constexpr int nB = 4 * (CH / 4);  // (16-point chunk h, c pairs cp and cp + CH/4)
          constexpr int nA = 4 * 32;        // (16-point chunk h, k, a pair)
          // The B and A units are separate straight-line paths; a B thread takes two units.
          if (tid < nB) {
            const int h = tid / (CH / 4);
#pragma unroll
            for (int e2 = 0; e2 < 2; ++e2) {
              const int cp = tid % (CH / 4) + e2 * (CH / 4);
              // Re/Im of c = 2 cp and c + 1 (rows c and CH + c).  Lanes with bit 2 of cp
              // set hold the pair as (c + 1, c), so a quarter warp's stores cover both rows
              // of a 128-byte line and all four swizzle chunks: no bank conflicts.
              const bool sw = (cp >> 2) & 1;
              const int rows[4] = {2 * cp + sw, CH + 2 * cp + sw, 2 * cp + 1 - sw, CH + 2 * cp + 1 - sw};
              slice_unit<false>(st_base + 3 * Lay::kTileA, Lay::kTileB, h, rows, [&](int pp, int* X) {
                const int4 q = eb[pp * (kEbStride / 2) + cp];  // already fixed point
                X[0] = q.x;
                X[1] = q.y;
                X[2] = q.z;
                X[3] = q.w;
              });
            }
          } else if (tid >= kBThreads && tid < kBThreads + nA) {
            // A rows 2 (16 k + a) + (re|im): the two halves of a complex row sit in
            // neighbouring TMEM lanes, so the epilogue combines them with one shuffle.
            // A unit takes the a pair (ap, ap + 8).
            const int v = tid - kBThreads;
            const int h = v >> 5, k = (v & 31) >> 3, ap = v & 7;
            const int j0 = 16 * k + ap;
            // lanes with bit 2 of ap set read (im, re) pairs and store rows (im, re): no
            // bank conflicts (as for the B units)
            const int sw = (ap >> 2) & 1;
            const int rows[4] = {2 * j0 + sw, 2 * j0 + 1 - sw, 2 * j0 + 16 + sw, 2 * j0 + 17 - sw};
            slice_unit<true>(st_base, Lay::kTileA, h, rows, [&](int pp, int* X) {
              const float gg = gk[pp * 4 + k];
              const float2 z0 = ea[pp * kEaStride + ap];
              const float2 z1 = ea[pp * kEaStride + ap + 8];
              X[0] = quant(gg * z0.x);
              X[1] = quant(gg * z0.y);
              X[2] = quant(gg * z1.x);
              X[3] = quant(gg * z1.y);
            });
          }
        }
        tc::fence_async_smem();
        __syncwarp();
        if (lane == 0) {
          tc::mbar_arrive(&full[stage]);
          tc::mbar_arrive(&aempty[buf]);
        }
      }

      // ---- epilogue: warps 0-3 own TMEM lanes 0-127 -----------------------------------
      // Lane r holds row r = 2 (16 k + a) + ri of D.  For every c:
      //   Vr = D[re, Rr] - D[im, Ri],  Vi = D[re, Ri] + D[im, Rr],
      // so each lane sends its D[., Ri] to its neighbour (lane r ^ 1) and keeps D[., Rr]:
      // the re lane writes Vr, the im lane Vi, for m = Cf a + cbase + c.  Warps 4-7 go on
      // with the next piece meanwhile.
      if (warp < 4) {
        bool ok = !*abort_flag;
        if (ok && !tc::mbar_wait(done, piece_iter & 1, abort_flag)) {
          fail();
          ok = false;
        }
        tc::tc_fence_after();
        const int r = tid;  // TMEM lane == GEMM row
        const int ri = r & 1, j = r >> 1;
        const int k = j >> 4, a = j & 15;
        const double f = tc_scale(piecemax[piece]) * kKScale[k] / (kQ * kQ);
        const uint32_t lane_off = (uint32_t)(warp * 32) << 16;
        float* out = partial + ((size_t)piece * 8 + 2 * k + ri) * Nl;
        const int m0 = Cf * a + cbase;
        // D q^2 / 2^8 = 2^24 W0 + 2^16 W1 + 2^8 W2 + W3 is an exact integer below 2^50, so
        // the re/im combination is done in int64 too and each output needs one conversion
        // (through the bit pattern of 1.5 2^52: no conversion-pipe instruction).
        const double fs = f * 256.0;
        const bool vec_out = (Nl & 3) == 0;
        for (int cb = 0; cb < CH; cb += 8) {
          long long T[2][8];
#pragma unroll
          for (int half = 0; half < 2; ++half) {
            uint32_t w[4][8];
            if (ok) {
#pragma unroll
              for (int q = 0; q < 4; ++q) tc::tmem_ld8_nowait(tmem + lane_off + q * N + (half ? CH : 0) + cb, w[q]);
              tc::tmem_wait_ld();
            }
#pragma unroll
            for (int i = 0; i < 8; ++i)
              T[half][i] = ok ? ((long long)(int)w[0][i] << 24) + ((long long)(int)w[1][i] << 16) +
                                    ((long long)(int)w[2][i] << 8) + (long long)(int)w[3][i]
                              : 0ll;
          }
          float o8[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const long long x = __shfl_xor_sync(0xffffffffu, T[1][i], 1);
            const long long v = ri ? x + T[0][i] : T[0][i] - x;
            const double dv = __longlong_as_double(v + 0x4338000000000000ll) - 6755399441055744.0;
            o8[i] = (float)(dv * fs);
          }
          if (vec_out && m0 + cb + 8 <= Nl) {  // 16-byte aligned: Nl % 4 == 0, m0 + cb % 8 == 0
            float4* o4 = reinterpret_cast<float4*>(out + m0 + cb);
            o4[0] = make_float4(o8[0], o8[1], o8[2], o8[3]);
            o4[1] = make_float4(o8[4], o8[5], o8[6], o8[7]);
          } else {
#pragma unroll
            for (int i = 0; i < 8; ++i)
              if (m0 + cb + i < Nl) out[m0 + cb + i] = o8[i];
          }
        }
        tc::tc_fence_before();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(tfree);
      }
    }
  } else if (warp == kSlicerWarps + kAnchorWarps) {
    // ==== MMA issuer (one thread) ======================================================
    constexpr uint32_t i1 = idesc_i8(kM, N, true, true), i2 = idesc_i8(kM, 2 * N, true, true);
    static_assert(2 * N <= 256, "B0|B1 must be one MMA operand");
    if (lane == 0) {
      uint32_t g = 0, piece_iter = 0;
      for (int piece = blockIdx.x; piece < npieces; piece += gridDim.x, ++piece_iter) {
        const int len = piece_len[piece];
        const int nblk = (len + kBK - 1) / kBK;
        bool ok = !*abort_flag;
        // the previous piece's epilogue has read TMEM
        if (ok && piece_iter > 0 && !tc::mbar_wait(tfree, (piece_iter - 1) & 1, abort_flag)) {
          fail();
          ok = false;
        }
        tc::tc_fence_after();
        for (int b = 0; b < nblk; ++b, ++g) {
          const int stage = g % S;
          const uint32_t use = g / S;
          if (ok && !tc::mbar_wait(&full[stage], use & 1, abort_flag)) {
            fail();
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
              const uint64_t a0 = desc_k_sw64(A[0] + off), a1 = desc_k_sw64(A[1] + off),
                             a2 = desc_k_sw64(A[2] + off);
              const uint64_t b01 = desc_k_sw64(B[0] + off), b2 = desc_k_sw64(B[2] + off);
              // B0 and B1 are consecutive tiles, one 2N-row operand: A_i [B0|B1] lands on
              // W_i, W_(i+1) (columns iN .. (i+2)N).  W2, W3 are started by the B2
              // products, W0 and W1 by A0 [B0|B1].
              mma_i8(tmem + 2 * N, a0, b2, i1, acc);
              mma_i8(tmem + 3 * N, a1, b2, i1, acc);
              mma_i8(tmem, a0, b01, i2, acc);
              mma_i8(tmem + N, a1, b01, i2, true);
              mma_i8(tmem + 2 * N, a2, b01, i2, true);
            }
          }
          tc::mma_commit(&empty[stage]);
        }
        tc::mma_commit(done);
      }
    }
    __syncwarp();
  }
  __syncthreads();
  if (warp == 0) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, Lay::kTmemCols);
  }
}

template <int CH>
int launch_ch(const Geometry& g, const Workspace& ws, int Cf, cudaStream_t s) {
  using Lay = Layout<CH>;
  cudaError_t e =
      cudaFuncSetAttribute(bin_sums_tc_kernel<CH>, cudaFuncAttributeMaxDynamicSharedMemorySize, Lay::kBytes);
  if (e != cudaSuccess) return set_cuda_error(e, "bin_sums_tc attributes", __FILE__, __LINE__);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int groups = Cf / CH;
  int64_t per = (sms + groups - 1) / groups;
  int64_t grid = ws.pmax < per ? ws.pmax : per;
  if (grid < 1) grid = 1;
  dim3 gd((unsigned)grid, groups);
  bin_sums_tc_kernel<CH><<<gd, kThreads, Lay::kBytes, s>>>(g.Nl, Cf, ws.pay, ws.npieces, ws.pmax,
                                                           ws.piece_start, ws.piece_len, ws.piecemax,
                                                           reinterpret_cast<float*>(ws.partial),
                                                           ws.flags);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_cuda_error(e, "bin_sums_tc launch", __FILE__, __LINE__);
  count_launches(1);
  return DSHT_OK;
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
  launch_piece_maxima(ws, s);
  switch (Cf) {
    case 8: return launch_ch<8>(g, ws, 8, s);
    case 16: return launch_ch<16>(g, ws, 16, s);
    case 32: return launch_ch<32>(g, ws, 32, s);
    case 64: return launch_ch<64>(g, ws, 64, s);
    case 128: return launch_ch<64>(g, ws, 128, s);  // two column groups
    default: return set_error(DSHT_ERR_INVALID, "mixed precision supports Nl <= 2048 (Nl=%d)", g.Nl);
  }
}

}  // namespace dsht
