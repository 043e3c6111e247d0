// Internal declarations shared by the DirectSHT B200 kernels.
//
// Data layout in HBM (Nlm = Nl(Nl+1)/2, rows in Healpy order m(2Nl-1-m)/2 + l):
//   tables   Yv, Yd      double [Nlm][Nx]          (sht/sht.py:50-56 layout, numpy path)
//   points   key         uint32 [N]                set*(Nx-1) + bin, or DSHT_KEY_DROP
//            sorted      double [N][4]             (cos phi, sin phi, w, t) by key
//   pieces   <= 1 bin each, <= piece_max points    (key, start, len)
//   partial  double [piece][8][Nl]                 (k, re/im) bin sums for every m
//   fold     double [Nl][4 q][Nx][4]               q = {equ even, equ odd, pol even, pol odd}
//                                                  entries (A re, A im, B re, B im)
//   alm      double2 [Nlm]                         complex128, Healpy order
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include <vector>

#include "../../include/dsht.h"

#define DSHT_KEY_DROP 0xffffffffu

namespace dsht {

// Number of point sets: {equatorial, rotated polar} x {cos >= 0, cos < 0}.
constexpr int kSets = 4;
// Error-flag bits written by the point kernel.
constexpr unsigned kFlagThetaRange = 1u;   // basic_sht assertion (sht/sht.py:171-172)
constexpr unsigned kFlagPolarRange = 2u;   // rotated polar point still outside (-xmax, xmax)
constexpr unsigned kFlagHasPolar = 4u;     // at least one point went through the rotation
constexpr unsigned kFlagTimeout = 8u;      // a bounded wait in a tensor-core kernel gave up

struct Geometry {
  int Nl, Nx;
  double xmax;
  double dx;          // xmax / (Nx-1), the numpy grid step  (sht/sht.py:48)
  double acos_xmax;   // numpy arccos(xmax), arccos(-xmax) (sht/sht.py:171)
  double acos_mxmax;
  int64_t Nlm;
  int nbins;          // Nx - 1 right-open bins
  int nkeys;          // kSets * nbins
};

// Output pointers of one tensor-core contraction pass (contract_tc.cu): map k's equatorial
// alm to equ[k], its rotated-polar alm to pol[k] (2 Nlm doubles each).
constexpr int kTcMaxMaps = 8;
struct TcOut {
  double* equ[kTcMaxMaps];
  double* pol[kTcMaxMaps];
};


// Maps of one batched rotation: io[k] += R(rot[k]) when *flags[k] has polar points.
constexpr int kMaxRot = 8;
struct RotMaps {
  const double* rot[kMaxRot];
  double* io[kMaxRot];
  const unsigned* flags[kMaxRot];
};

// Flag words of finished transforms: *all |= *slot[k]; status[k] (if set) = *slot[k].
struct StatusOut {
  const unsigned* slot[kMaxRot];
  unsigned* status[kMaxRot];
};

// Workspace carve-up for one execute call.
struct Workspace {
  uint32_t* key;        // [N]
  double* pay;          // [N][4] sorted records (cos phi, sin phi, w, t)
  uint32_t* sidx;       // [N] input index of each sorted slot (multi-map transforms)
  uint32_t* piecemax;   // [pmax] largest |w h_k| of the piece's points (float bits)
  double* wsum;         // [pmax] sum of |w| of the piece's points (fold digit scales)
  uint32_t* count;      // [nkeys + 1]
  uint32_t* offset;     // [nkeys + 1]
  uint32_t* cursor;     // [nkeys]
  int* piece_first;     // [nkeys + 1]  first piece of each key (exclusive scan)
  int* piece_key;       // [pmax]
  int64_t* piece_start; // [pmax]
  int* piece_len;       // [pmax]
  int* npieces;         // [1]
  unsigned* flags;      // [1]
  double* partial;      // [pmax][8][Nl]
  double* fold;         // [Nl][4][Nx][4] FP64 fold; the tensor-core route's fold digits
                        // [Nl][2][4][4 tc_maps][Kp] (int8) share this region
  int16_t* cexp;        // [tc_maps][2] fold column scale exponents (tensor-core route)
  unsigned long long* cmax;  // [tc_maps][2] largest node |w| sum per half (bits of a double)
  unsigned* tc_next;    // [1] work counter of the tensor-core contraction
  int tc_maps;          // maps one tensor-core contraction pass can hold
  uint8_t* tile_live;   // [2][ceil(Nx/128)] tiles of the fallback contraction
  uint8_t* tile_live2;  // [2][ceil(Nx/256)] tiles of the streaming contraction
  double* alm_equ;      // [Nlm][2]
  double* alm_pol;      // [Nlm][2] (x nmaps for multi-map transforms)
  int64_t npts;         // N, the stride of pay
  int partial_f32;      // partial sums stored as float (tensor-core path) instead of double
  int64_t pmax;
  int piece_max;
  unsigned* slot_flags; // [kMaxRot] flags of the transforms awaiting rotation (multi-transform calls)
  unsigned* all_flags;  // [1] OR of every finished transform's flags
  size_t bytes;
};

// multi: add the records of multi-transform calls (gather indices, rotation and flag slots);
// tc_maps: maps one tensor-core contraction pass holds (fold digit columns).
size_t workspace_layout(const Geometry& g, int64_t N, int piece_max, uint8_t* base, Workspace* ws,
                        bool multi = false, int tc_maps = 1);
int default_piece_max(const Geometry& g, int64_t N);
int plan_piece_max(const dsht_plan_s* p, int64_t N);
// How a transform of N points runs on a plan: tensor-core bin sums (tc), tensor-core
// contraction of the digit tables (digits), else the FP64 tables streamed by TMA (streamed)
// or, for Nx whose rows are not 16-byte multiples, the FP64 fallback kernel.
struct Route {
  bool tc, digits, streamed;
};
Route plan_route(const dsht_plan_s* p, int64_t N);

// Kernels launched by api.cu (each file owns its launch helpers).
void launch_tables(const Geometry& g, double* Yv, double* Yd, cudaStream_t s);
void launch_points(const Geometry& g, const double* theta, const double* phi, const void* w, int w_f32,
                   int64_t N, int mode, const Workspace& ws, cudaStream_t s,
                   bool phi_record = false);
void launch_gather(const Geometry& g, const void* w, int w_f32, int64_t N, const Workspace& ws, cudaStream_t s);
// Largest |w h_k| of every piece of the sorted records (needed by the tensor-core sums).
void launch_piece_maxima(const Workspace& ws, cudaStream_t s);
void launch_publish_flags(const StatusOut& st, int n, unsigned* all, cudaStream_t s);
void launch_bin_sums_fp64(const Geometry& g, const Workspace& ws, cudaStream_t s);
int launch_bin_sums_tc(const Geometry& g, const Workspace& ws, cudaStream_t s);
// NUFFT bin sums (nufft.cu): FP64 partial sums [piece][8][Nl] and the pieces' |w| sums.
int nufft_logn(int Nl);
void nufft_host_tables(int Nl, int logn, std::vector<double>& dinv, std::vector<double>& tw);
int launch_bin_sums_nufft(const Geometry& g, const Workspace& ws, int logn, const double* dinv, const double* tw,
                          cudaStream_t s);
constexpr int kNufftPiece = 8192;  // default points per piece of the NUFFT sums
constexpr int kNufftMinPerKey = 512;  // AUTO bin sums: NUFFT from this many points per key on average
constexpr int kFp64MaxPerKey = 28;    // AUTO bin sums: FP64 direct sums below this many per key
int tc_inner_factor(int Nl);
// FP64 fold of the current map into ws.fold, and the live-tile flags of the contractions.
void launch_fold(const Geometry& g, const Workspace& ws, cudaStream_t s);
// Digit tables and folds (digits.cu) and the tensor-core contraction (contract_tc.cu).
int digit_kp(int Nx);                   // bytes per digit row: 2 Nx rounded up to 64
constexpr int kTcMaxNx = 8192;          // S32 class sums stay below 2^31 for 2 Nx <= 16384
void launch_tables_cols(const Geometry& g, int m0, int m1, double* Yv, double* Yd, cudaStream_t s);
void launch_table_rowexp(const Geometry& g, int64_t row0, int64_t nrows, const double* Yv, const double* Yd,
                         int16_t* rexp, cudaStream_t s);
void launch_table_digits(const Geometry& g, int64_t row0, int64_t nrows, const double* Yv, const double* Yd,
                         const int16_t* rexp, uint8_t* dig, cudaStream_t s);
void launch_table_decode(const Geometry& g, int which, int64_t r0, int64_t n, const uint8_t* dig,
                         const int16_t* rexp, double* out, cudaStream_t s);
void launch_fold_scale(const Geometry& g, const Workspace& ws, unsigned long long* cmax, cudaStream_t s);
void launch_fold_digits(const Geometry& g, const Workspace& ws, const unsigned long long* cmax, int16_t* cexp,
                        int map, int ncols,
                        uint8_t* fdig, cudaStream_t s);
int make_table_digit_tmap(CUtensorMap* tm, const uint8_t* dig, int Nx, int64_t Nlm);
std::vector<uint32_t> tc_items(int Nl);
int launch_contract_tc(const Geometry& g, const CUtensorMap& tmA, const uint32_t* items, int nitems,
                       const int16_t* rexp, const uint8_t* fdig, int fdig_cols, const int16_t* cexp, int nmaps,
                       const TcOut& out, unsigned* flags, unsigned* next_item, cudaStream_t s);

void launch_contract_fp64(const Geometry& g, const double* Yv, const double* Yd,
                          const Workspace& ws, cudaStream_t s);
bool contract_stream_ok(const Geometry& g);
// FP64 tables through TMA (contract_stream.cu): alm of the fold to alm_equ / alm_pol.
void launch_contract_stream(const Geometry& g, const CUtensorMap& tmv, const CUtensorMap& tmd, const double* fold,
                            const uint8_t* live, double* alm_equ, double* alm_pol, unsigned* flags, cudaStream_t s);
// 2D tensor map of an FP64 table (node x row), boxes of 256 nodes x 16 rows.
int make_table_tmap(CUtensorMap* tm, const void* base, int Nx, int64_t Nlm);
// An FP64 table in the JAX path's layout out[m][l - m][j] (Nl x Nl x Nx doubles, zeros
// where l >= Nl) on the device.
void launch_table_mlayout(const Geometry& g, const double* t64, double* out, cudaStream_t s);
void launch_rotate_back(const Geometry& g, const double* alm_rot, const double* alm_add,
                        double* alm_out, const unsigned* flags, cudaStream_t s);
// alm io[k] += R(rot[k]) for k < nmaps <= kMaxRot (a map without polar points is left as it is).
void launch_rotate_back_maps(const Geometry& g, const RotMaps& maps, int nmaps, cudaStream_t s);

// Hint: bring [p, p + bytes) into L2 (cp.async.bulk.prefetch.L2, 16-byte aligned chunks of at
// most 32 KB; the unaligned ends are left out).  lane, nlanes: the calling threads share the
// chunks.  A prefetch only warms the cache: it reads nothing into registers and cannot fault
// on the addresses of a live buffer.
__device__ __forceinline__ void prefetch_l2(const void* p, size_t bytes, int lane, int nlanes) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const uintptr_t a0 = (a + 15) & ~uintptr_t(15);
  if (bytes <= a0 - a) return;
  const size_t n = (bytes - (a0 - a)) & ~size_t(15);
  for (size_t off = (size_t)lane * 32768; off < n; off += (size_t)nlanes * 32768) {
    const size_t sz = n - off < 32768 ? n - off : 32768;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a0 + off), "r"((unsigned)sz) : "memory");
  }
}

// Hermite weights w * {(2t+1)(1-t)^2, t(1-t)^2, t^2(3-2t), t^2(t-1)} of one point, in the
// rounding order of sht/sht.py:239-240.
__device__ __forceinline__ void hermite(double t, double wi, double* out4) {
  const double omt = __dadd_rn(1.0, -t);
  const double omt2 = __dmul_rn(omt, omt);
  const double t2 = __dmul_rn(t, t);
  out4[0] = __dmul_rn(wi, __dmul_rn(__dadd_rn(__dmul_rn(2.0, t), 1.0), omt2));
  out4[1] = __dmul_rn(wi, __dmul_rn(t, omt2));
  out4[2] = __dmul_rn(wi, __dmul_rn(t2, __dadd_rn(3.0, -__dmul_rn(2.0, t))));
  out4[3] = __dmul_rn(wi, __dmul_rn(t2, __dadd_rn(t, -1.0)));
}

// The sorted record of a point: (cos phi, sin phi, w, t), 32 bytes.
constexpr int kRec = 4;

// Healpy index of (l, m).
__host__ __device__ inline int64_t hp_index(int l, int m, int Nl) {
  return ((int64_t)m * (2 * Nl - 1 - m)) / 2 + l;
}

}  // namespace dsht

// A plan: geometry, its FP64 tables, and buffers it owns (see api.cu).
#include <mutex>
struct dsht_plan_s {
  dsht::Geometry g;
  int device = 0;
  double* Yv = nullptr;  // FP64 tables (null in a compact plan)
  double* Yd = nullptr;
  alignas(64) CUtensorMap tmYv, tmYd;
  bool tm64 = false;
  // Digit tables of the tensor-core contraction (digits.cu): 4 planes [Nlm][Kp] int8 in
  // rows grouped by parity, row exponents, the work items and the TMA map of the planes.
  uint8_t* dig = nullptr;
  int16_t* rexp = nullptr;
  uint32_t* tc_items = nullptr;
  int tc_nitems = 0;
  alignas(64) CUtensorMap tmDig;
  bool tmdig = false;
  // Plan-owned buffers, grown on demand (used when the caller passes no workspace and by
  // the host-pointer entry points).
  void* ws = nullptr;
  size_t ws_bytes = 0;
  double* in = nullptr;  // [3][N] device copies of host inputs
  int64_t in_n = 0;
  double* alm = nullptr;  // [2 Nlm]
  unsigned* h_flags = nullptr;  // pinned
  int precision = DSHT_PREC_FP64;
  // Type-1 NUFFT bin sums (nufft.cu): grid of 2^nu_logn cells, 1/Psi(m) [Nl] and the
  // twiddles e^{2 pi i i/n} [n] (complex), built at plan creation for Nl <= 2048.
  int nu_logn = 0;
  double* nu_dinv = nullptr;
  double* nu_tw = nullptr;
  int tune_bin_sums = DSHT_BIN_SUMS_AUTO;
  int tune_piece_max = 0;      // points per bin piece (0: chosen from N and the method)
  int tune_maps_per_pass = 0;  // maps per multi-map contraction pass (0: the most that fit)
  // Stage timers: one event per stage boundary of a call, in stream order; the interval
  // from mark k to mark k+1 belongs to stage ev_stage[k] (-1: no stage).  Summed per stage
  // into prof_ms when the call has synchronised.
  static constexpr int kProfMarks = 4096;
  bool prof = false;
  cudaEvent_t* ev = nullptr;  // [kProfMarks], created by dsht_profile_enable
  int8_t ev_stage[kProfMarks] = {};
  int ev_n = 0;
  double prof_ms[DSHT_STAGE_COUNT] = {};
  int64_t prof_calls = 0;
  std::mutex mu;
};

namespace dsht {
Geometry make_geometry(int Nl, int Nx, double xmax);
// Enqueue the whole transform on `s` (flags are left in ws.flags; no synchronisation).
int run_pipeline(dsht_plan_s* p, const double* theta, const double* phi, const double* w, int64_t N, int mode,
                 double* alm, const Workspace& ws, cudaStream_t s);
// The stages after the sort: bin sums, fold, contraction, rotation.
int run_after_sort(dsht_plan_s* p, int64_t N, int mode, double* alm, const Workspace& ws, cudaStream_t s,
                   bool marks);
// One transform of a multi-transform call.  same_points: the points are those of the
// previous item (its sort is reused and only the weights are gathered again).
struct Item {
  const double* theta;
  const double* phi;
  const void* w;
  int w_f32;
  int64_t N;
  double* alm;
  bool same_points;
  unsigned* status;  // device word that receives the item's flags, or null
};
// Bin sums of a tensor-core-route transform: the NUFFT (default) or the tensor-core direct
// sums; sets w2.partial_f32 to the layout written.
int launch_bin_sums_mixed(const dsht_plan_s* p, Workspace& w2, int64_t N, cudaStream_t s);
int plan_bin_method(const dsht_plan_s* p, int64_t N);
bool plan_uses_nufft(const dsht_plan_s* p, int64_t N);
// Runs the items in order; every finished item's flags are OR-ed into ws.all_flags.
int run_items(dsht_plan_s* p, const Item* items, int n, int mode, const Workspace& ws, cudaStream_t s);
// After the stream has been synchronised: fold the stage events into the plan's totals.
void collect_profile(dsht_plan_s* p);
// Stage boundary on stream s when profiling: what follows belongs to `stage` (-1: none).
void prof_mark(dsht_plan_s* p, int stage, cudaStream_t s);
// Map device flag bits to a DSHT status code (and set the error message).
int flags_to_status(unsigned f, int mode);
}  // namespace dsht

#define DSHT_CUDA_OK(expr)                                   \
  do {                                                       \
    cudaError_t _e = (expr);                                 \
    if (_e != cudaSuccess) return dsht::set_cuda_error(_e, #expr, __FILE__, __LINE__); \
  } while (0)

namespace dsht {
int set_error(int code, const char* fmt, ...);
// Adds n to the process-wide count of kernels this library launched.
void count_launches(int n);
int set_cuda_error(cudaError_t e, const char* what, const char* file, int line);
// First kernel-launch error since the last call (recorded by count_launches), as a status.
int launch_error(const char* where);
}  // namespace dsht
