// C ABI of libdsht_b200.so: plans, workspace, the execute pipeline, table queries and the
// drop-ins for the reference's ctypes library.  See include/dsht.h.
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "dsht_internal.cuh"

namespace dsht {

static thread_local std::string g_last_error;
static std::atomic<int64_t> g_launches{0};

static thread_local cudaError_t g_launch_error = cudaSuccess;

// Every launch helper calls this right after its launches: it counts them and keeps the
// first launch error of the thread (launch_error() reports and clears it).
void count_launches(int n) {
  g_launches.fetch_add(n, std::memory_order_relaxed);
  const cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess && g_launch_error == cudaSuccess) g_launch_error = e;
}

int launch_error(const char* where) {
  const cudaError_t e = g_launch_error;
  g_launch_error = cudaSuccess;
  cudaGetLastError();
  return e == cudaSuccess ? 0 : set_cuda_error(e, where, __FILE__, __LINE__);
}

int set_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int set_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
  return set_error(e == cudaErrorMemoryAllocation ? DSHT_ERR_NOMEM : DSHT_ERR_CUDA, "%s failed: %s (%s:%d)",
                   what, cudaGetErrorString(e), file, line);
}

static size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Points per bin piece: at most 2048 (the S32 sums of the tensor path stay exact), at
// least 256, and about N/2048 in between.  Smaller pieces keep the fixed-point scale of
// the tensor path (the piece's largest |w h_k|) closer to its typical weight.
int default_piece_max(const Geometry& g, int64_t N) {
  int64_t p = (N + 2047) / 2048;
  if (p < 256) p = 256;
  if (p > 2048) p = 2048;
  return (int)p;
}

size_t workspace_layout(const Geometry& g, int64_t N, int piece_max, uint8_t* base, Workspace* ws, bool multi,
                        int tc_maps) {
  size_t off = 0;
  auto take = [&](size_t bytes) -> uint8_t* {
    uint8_t* p = base ? base + off : nullptr;
    off = align_up(off + bytes, 256);
    return p;
  };
  const int64_t n = N > 0 ? N : 1;
  // Pieces of a transform of up to n points.  A workspace laid out for the NUFFT sums' large
  // pieces also serves the smaller transforms of a batch, which may take the direct sums:
  // their pieces of default_piece_max(N) or at most 2048 points number at most
  // max(2048, N / 2048) beyond one per key, with N below the NUFFT threshold.
  int64_t extra = (n + piece_max - 1) / piece_max;
  if (piece_max > 2048) {
    const int64_t direct_n = std::min<int64_t>(n, (int64_t)kNufftMinPerKey * g.nkeys);
    extra = std::max<int64_t>(extra, std::max<int64_t>(2048, (direct_n + 2047) / 2048));
  }
  const int64_t pmax = std::min<int64_t>(g.nkeys, n) + extra;
  const int tile = 128;
  const int ntile = (g.Nx + tile - 1) / tile;
  Workspace w{};
  w.key = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * n));
  w.pay = reinterpret_cast<double*>(take(sizeof(double) * kRec * n));
  const bool maps = multi;
  if (maps) {
    w.sidx = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * n));
  }
  w.count = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * (g.nkeys + 1)));
  w.offset = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * (g.nkeys + 1)));
  w.cursor = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * (g.nkeys + 1)));
  w.piece_first = reinterpret_cast<int*>(take(sizeof(int) * (g.nkeys + 1)));
  w.piece_key = reinterpret_cast<int*>(take(sizeof(int) * pmax));
  w.piece_start = reinterpret_cast<int64_t*>(take(sizeof(int64_t) * pmax));
  w.piece_len = reinterpret_cast<int*>(take(sizeof(int) * pmax));
  w.piecemax = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * pmax));
  w.wsum = reinterpret_cast<double*>(take(sizeof(double) * pmax));
  w.npieces = reinterpret_cast<int*>(take(sizeof(int)));
  w.flags = reinterpret_cast<unsigned*>(take(sizeof(unsigned)));
  if (maps) {
    w.slot_flags = reinterpret_cast<unsigned*>(take(sizeof(unsigned) * kMaxRot));
    w.all_flags = reinterpret_cast<unsigned*>(take(sizeof(unsigned)));
  }
  w.partial = reinterpret_cast<double*>(take(sizeof(double) * 8 * (size_t)g.Nl * pmax));
  // The FP64 fold of one map, or the tensor-core route's fold digits ([Nl][2][4][4 tc_maps]
  // [Kp] int8), whichever is larger: a call's route uses one of them.
  w.tc_maps = std::max(1, std::min(tc_maps, kTcMaxMaps));
  const size_t fold_bytes = sizeof(double) * 16 * (size_t)g.Nl * g.Nx;
  const size_t fdig_bytes = (size_t)g.Nl * 8 * 4 * w.tc_maps * (size_t)digit_kp(g.Nx);
  w.fold = reinterpret_cast<double*>(take(std::max(fold_bytes, fdig_bytes)));
  w.cexp = reinterpret_cast<int16_t*>(take(sizeof(int16_t) * 2 * w.tc_maps));
  w.cmax = reinterpret_cast<unsigned long long*>(take(sizeof(unsigned long long) * 2 * w.tc_maps));
  w.tc_next = reinterpret_cast<unsigned*>(take(sizeof(unsigned)));
  w.tile_live = reinterpret_cast<uint8_t*>(take(2 * (size_t)ntile));
  w.tile_live2 = reinterpret_cast<uint8_t*>(take(2 * (size_t)((g.Nx + 255) / 256)));
  w.alm_equ = reinterpret_cast<double*>(take(sizeof(double) * 2 * (size_t)g.Nlm));
  w.alm_pol = reinterpret_cast<double*>(take(sizeof(double) * 2 * (size_t)g.Nlm * (maps ? kMaxRot : 1)));
  w.npts = n;
  w.pmax = pmax;
  w.piece_max = piece_max;
  w.bytes = off;
  if (ws) *ws = w;
  return off;
}

// The mixed levels' bin-sum method for one transform of N points (chosen per transform, so
// the transforms of one batch call may differ).  AUTO compares the average points per bin
// key with two measured crossovers: a NUFFT piece pays a fixed FFT (about 15 us of one SM at
// Nl = 1024) and little per point, so it wins from kNufftMinPerKey points per key; the
// tensor-core sums pay a GEMM tile and its epilogue per piece and 0.2-0.3 ns per point
// (device-wide), the FP64 direct sums little per piece and 1-2 ns per point, so below
// kFp64MaxPerKey points per key (pieces of a few points) the FP64 sums are the fastest.
int plan_bin_method(const dsht_plan_s* p, int64_t N) {
  const int t = p->tune_bin_sums;
  if (t == DSHT_BIN_SUMS_FP64 || t == DSHT_BIN_SUMS_TC) return t;
  if (p->nu_dinv && (t == DSHT_BIN_SUMS_NUFFT || N >= (int64_t)kNufftMinPerKey * p->g.nkeys))
    return DSHT_BIN_SUMS_NUFFT;
  if (t == DSHT_BIN_SUMS_AUTO && N < (int64_t)kFp64MaxPerKey * p->g.nkeys) return DSHT_BIN_SUMS_FP64;
  return DSHT_BIN_SUMS_TC;
}

bool plan_uses_nufft(const dsht_plan_s* p, int64_t N) {
  return plan_route(p, N).tc && plan_bin_method(p, N) == DSHT_BIN_SUMS_NUFFT;
}

// Pieces of the direct sums stay at or below 2048 points (the tensor path's S32 sums stay
// exact); the NUFFT sums pay one FFT per piece, so theirs are larger.
int plan_piece_max(const dsht_plan_s* p, int64_t N) {
  const bool nufft = plan_uses_nufft(p, N);
  int pm = p->tune_piece_max > 0 ? p->tune_piece_max : nufft ? kNufftPiece : default_piece_max(p->g, N);
  if (!nufft && pm > 2048) pm = 2048;
  return pm;
}

// Bin sums of one transform of N points on the mixed route (sorted records in w2.pay).
int launch_bin_sums_mixed(const dsht_plan_s* p, Workspace& w2, int64_t N, cudaStream_t s) {
  switch (plan_bin_method(p, N)) {
    case DSHT_BIN_SUMS_NUFFT:
      w2.partial_f32 = 0;
      return launch_bin_sums_nufft(p->g, w2, p->nu_logn, p->nu_dinv, p->nu_tw, s);
    case DSHT_BIN_SUMS_FP64:
      w2.partial_f32 = 0;
      launch_piece_maxima(w2, s);  // the |w| sums (fold digit scales)
      launch_bin_sums_fp64(p->g, w2, s);
      return DSHT_OK;
    default:
      w2.partial_f32 = 1;
      return launch_bin_sums_tc(p->g, w2, s);  // piece maxima and |w| sums first
  }
}

Route plan_route(const dsht_plan_s* p, int64_t N) {
  Route r{};
  r.tc = p->precision != DSHT_PREC_FP64 && N >= DSHT_MIXED_MIN_POINTS;
  // The digit tables serve tensor-core transforms at the MIXED level and every transform
  // of a plan that holds no FP64 tables; everything else contracts the FP64 tables.
  r.digits = p->tmdig && ((r.tc && p->precision == DSHT_PREC_MIXED) || !p->Yv);
  r.streamed = r.digits || p->tm64;
  return r;
}

// Builds the digit tables of rows [row0, row0 + nrows) from FP64 tables (Healpy order)
// held at Yv, Yd for exactly those rows.
static void digits_from_rows(dsht_plan_s* p, int64_t row0, int64_t nrows, const double* Yv, const double* Yd,
                             cudaStream_t s) {
  launch_table_rowexp(p->g, row0, nrows, Yv, Yd, p->rexp, s);
  launch_table_digits(p->g, row0, nrows, Yv, Yd, p->rexp, p->dig, s);
}

// Allocates the digit tables, the tensor-core work items and the tensor map; fills the
// tables from the plan's FP64 tables, or (plans without them) from FP64 columns built a
// few m at a time into temporary buffers.
static int build_digits(dsht_plan_s* p) {
  const Geometry& g = p->g;
  if (g.Nx > kTcMaxNx || g.Nl > 2048) return set_error(DSHT_ERR_INVALID, "digit tables need Nx <= %d", kTcMaxNx);
  const size_t kp = (size_t)digit_kp(g.Nx);
  cudaError_t e = cudaMalloc(&p->dig, 4 * (size_t)g.Nlm * kp);
  if (e == cudaSuccess) e = cudaMalloc(&p->rexp, sizeof(int16_t) * (size_t)g.Nlm);
  const std::vector<uint32_t> items = tc_items(g.Nl);
  if (e == cudaSuccess) e = cudaMalloc(&p->tc_items, sizeof(uint32_t) * items.size());
  if (e == cudaSuccess)
    e = cudaMemcpy(p->tc_items, items.data(), sizeof(uint32_t) * items.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(p->dig);
    cudaFree(p->rexp);
    cudaFree(p->tc_items);
    p->dig = nullptr;
    p->rexp = nullptr;
    p->tc_items = nullptr;
    cudaGetLastError();
    return set_cuda_error(e, "digit table allocation", __FILE__, __LINE__);
  }
  p->tc_nitems = (int)items.size();
  if (p->Yv) {
    digits_from_rows(p, 0, g.Nlm, p->Yv, p->Yd, 0);
  } else {
    // columns m0 .. m1 - 1 with at most ~2^26 table entries per pass through the buffers
    const int64_t cap = std::max<int64_t>((int64_t)1 << 26, (int64_t)g.Nl * g.Nx);
    double *tv = nullptr, *td = nullptr;
    e = cudaMalloc(&tv, sizeof(double) * cap);
    if (e == cudaSuccess) e = cudaMalloc(&td, sizeof(double) * cap);
    if (e != cudaSuccess) {
      cudaFree(tv);
      cudaFree(td);
      cudaGetLastError();
      return set_cuda_error(e, "digit table build buffers", __FILE__, __LINE__);
    }
    for (int m0 = 0; m0 < g.Nl;) {
      int m1 = m0 + 1;
      while (m1 < g.Nl && (hp_index(m1 + 1, m1 + 1, g.Nl) - hp_index(m0, m0, g.Nl)) * g.Nx <= cap) ++m1;
      const int64_t r0 = hp_index(m0, m0, g.Nl), r1 = hp_index(m1, m1, g.Nl);
      launch_tables_cols(g, m0, m1, tv, td, 0);
      digits_from_rows(p, r0, r1 - r0, tv, td, 0);
      m0 = m1;
    }
    e = cudaDeviceSynchronize();
    cudaFree(tv);
    cudaFree(td);
    if (e != cudaSuccess) return set_cuda_error(e, "digit table build", __FILE__, __LINE__);
  }
  DSHT_CUDA_OK(cudaDeviceSynchronize());
  DSHT_CUDA_OK(cudaGetLastError());
  if (int rc = make_table_digit_tmap(&p->tmDig, p->dig, g.Nx, g.Nlm)) return rc;
  p->tmdig = true;
  return DSHT_OK;
}

Geometry make_geometry(int Nl, int Nx, double xmax) {
  Geometry g{};
  g.Nl = Nl;
  g.Nx = Nx;
  g.xmax = xmax;
  g.dx = xmax / (double)(Nx - 1);
  g.acos_xmax = std::acos(xmax);
  g.acos_mxmax = std::acos(-xmax);
  g.Nlm = (int64_t)Nl * (Nl + 1) / 2;
  g.nbins = Nx - 1;
  g.nkeys = kSets * g.nbins;
  return g;
}

// The stages after the sort: bin sums, fold, contraction, rotation (stage events 1..5 when
// `marks` is set).  Reads the sorted payload ws.pay; leaves the device flags in ws.flags.
int run_after_sort(dsht_plan_s* p, int64_t N, int mode, double* alm, const Workspace& ws, cudaStream_t s,
                   bool marks) {
  const Geometry& g = p->g;
  auto mark = [&](int stage) {
    if (marks) prof_mark(p, stage, s);
  };
  Workspace w2 = ws;
  // Small transforms run the FP64 stages even on a mixed-precision plan.
  const Route rt = plan_route(p, N);
  if (rt.tc) {
    if (int rc = launch_bin_sums_mixed(p, w2, N, s)) return rc;
  } else {
    if (rt.digits) launch_piece_maxima(ws, s);  // the |w| sums (fold digit scales)
    launch_bin_sums_fp64(g, ws, s);
    w2.partial_f32 = 0;
  }
  if (rt.digits) {
    mark(DSHT_STAGE_FOLD);
    uint8_t* fdig = reinterpret_cast<uint8_t*>(ws.fold);
    launch_fold_scale(g, w2, ws.cmax, s);
    launch_fold_digits(g, w2, ws.cmax, ws.cexp, 0, 4, fdig, s);
    mark(DSHT_STAGE_CONTRACT);
    TcOut out{};
    out.equ[0] = ws.alm_equ;
    out.pol[0] = ws.alm_pol;
    if (int rc = launch_contract_tc(g, p->tmDig, p->tc_items, p->tc_nitems, p->rexp, fdig, 4, ws.cexp, 1, out,
                                    ws.flags, ws.tc_next, s))
      return rc;
  } else {
    mark(DSHT_STAGE_FOLD);
    launch_fold(g, w2, s);
    mark(DSHT_STAGE_CONTRACT);
    if (p->tm64)
      launch_contract_stream(g, p->tmYv, p->tmYd, ws.fold, ws.tile_live2, ws.alm_equ, ws.alm_pol, ws.flags, s);
    else
      launch_contract_fp64(g, p->Yv, p->Yd, ws, s);
  }
  mark(DSHT_STAGE_ROTATE);
  if (mode == DSHT_MODE_CALL) {
    launch_rotate_back(g, ws.alm_pol, ws.alm_equ, alm, ws.flags, s);
  } else {
    DSHT_CUDA_OK(cudaMemcpyAsync(alm, ws.alm_equ, sizeof(double) * 2 * g.Nlm, cudaMemcpyDeviceToDevice, s));
  }
  mark(-1);
  if (int rc = launch_error("kernel launch")) return rc;
  DSHT_CUDA_OK(cudaGetLastError());
  return DSHT_OK;
}

// Runs the whole pipeline on `s`; leaves the device flags in ws.flags.
int run_pipeline(dsht_plan_s* p, const double* theta, const double* phi, const double* w, int64_t N,
                        int mode, double* alm, const Workspace& ws, cudaStream_t s) {
  p->ev_n = 0;
  prof_mark(p, DSHT_STAGE_POINTS, s);
  launch_points(p->g, theta, phi, w, 0, N, mode, ws, s, plan_uses_nufft(p, N));
  prof_mark(p, DSHT_STAGE_BIN_SUMS, s);
  return run_after_sort(p, N, mode, alm, ws, s, true);
}

// Items of one class on the tensor-core route: passes of up to ws.tc_maps items (at most
// kMaxRot, the rotation batch); each item's fold goes straight to digits in its column slot,
// and one contraction launch per pass reads every table tile once for all of them.
static int run_class_digits(dsht_plan_s* p, const Item* items, const std::vector<int>& list, int mode,
                            const Workspace& ws, cudaStream_t s, int* sorted_item) {
  const Geometry& g = p->g;
  const int64_t nlm2 = 2 * g.Nlm;
  const Route rt = plan_route(p, items[list[0]].N);
  const int G = std::min(ws.tc_maps, kMaxRot);
  const int fcols = 4 * ws.tc_maps;
  uint8_t* fdig = reinterpret_cast<uint8_t*>(ws.fold);
  std::vector<int> pass;
  for (size_t li = 0; li < list.size(); ++li) {
    const int i = list[li];
    const Item& item = items[i];
    const int slot = (int)pass.size();
    Workspace w2 = ws;
    w2.flags = ws.slot_flags + slot;
    if (item.same_points && *sorted_item >= 0) {
      prof_mark(p, DSHT_STAGE_BIN_SUMS, s);  // the weight gather counts with the bin sums
      launch_gather(g, item.w, item.w_f32, item.N, ws, s);
    } else {
      prof_mark(p, DSHT_STAGE_POINTS, s);
      Workspace wp = ws;
      wp.piece_max = plan_piece_max(p, item.N);
      if (!(li + 1 < list.size() && items[list[li + 1]].same_points)) wp.sidx = nullptr;
      launch_points(g, item.theta, item.phi, item.w, item.w_f32, item.N, mode, wp, s, plan_uses_nufft(p, item.N));
      *sorted_item = i;
    }
    prof_mark(p, DSHT_STAGE_BIN_SUMS, s);
    DSHT_CUDA_OK(cudaMemcpyAsync(w2.flags, ws.flags, sizeof(unsigned), cudaMemcpyDeviceToDevice, s));
    if (rt.tc) {
      if (int rc = launch_bin_sums_mixed(p, w2, item.N, s)) return rc;
    } else {
      launch_piece_maxima(w2, s);
      launch_bin_sums_fp64(g, w2, s);
      w2.partial_f32 = 0;
    }
    prof_mark(p, DSHT_STAGE_FOLD, s);
    launch_fold_scale(g, w2, ws.cmax + 2 * slot, s);
    launch_fold_digits(g, w2, ws.cmax + 2 * slot, ws.cexp + 2 * slot, slot, fcols, fdig, s);
    pass.push_back(i);
    if ((int)pass.size() < G && li + 1 < list.size()) continue;
    TcOut out{};
    RotMaps rm{};
    StatusOut so{};
    for (size_t k = 0; k < pass.size(); ++k) {
      out.equ[k] = items[pass[k]].alm;
      out.pol[k] = ws.alm_pol + nlm2 * k;
      rm.rot[k] = out.pol[k];
      rm.io[k] = items[pass[k]].alm;
      rm.flags[k] = ws.slot_flags + k;
      so.slot[k] = ws.slot_flags + k;
      so.status[k] = items[pass[k]].status;
    }
    prof_mark(p, DSHT_STAGE_CONTRACT, s);
    if (int rc = launch_contract_tc(g, p->tmDig, p->tc_items, p->tc_nitems, p->rexp, fdig, fcols, ws.cexp,
                                    (int)pass.size(), out, ws.slot_flags, ws.tc_next, s))
      return rc;
    prof_mark(p, DSHT_STAGE_ROTATE, s);
    if (mode == DSHT_MODE_CALL) launch_rotate_back_maps(g, rm, (int)pass.size(), s);
    launch_publish_flags(so, (int)pass.size(), ws.all_flags, s);
    pass.clear();
  }
  return DSHT_OK;
}

// Several transforms in one call: multi-map transforms (one point set, the later maps marked
// same_points) and batches of independent transforms on one plan.  Each point set is
// classified and sorted once; a same_points item only gathers its weights into the sorted
// payload.  Bin sums and the fold run per item.  On the digit tables the contraction runs
// in passes of up to ws.tc_maps items that share one read of the tables
// (run_class_digits); on the FP64 tables once per item.  Equatorial alm go straight to
// item.alm, polar alm to a rotation slot, and one batched rotation per kMaxRot slots adds
// them back.  Items with N < DSHT_MIXED_MIN_POINTS on a mixed plan run the FP64 bin sums,
// in their own class.
int run_items(dsht_plan_s* p, const Item* items, int n, int mode, const Workspace& ws, cudaStream_t s) {
  const Geometry& g = p->g;
  const int64_t nlm2 = 2 * g.Nlm;
  p->ev_n = 0;
  DSHT_CUDA_OK(cudaMemsetAsync(ws.all_flags, 0, sizeof(unsigned), s));
  // Items in two classes by the precision their size selects; same_points chains stay whole
  // (they share N, hence the class).
  std::vector<int> order[2];
  for (int i = 0; i < n; ++i) order[plan_route(p, items[i].N).tc ? 1 : 0].push_back(i);
  int sorted_item = -1;  // item whose sort the workspace holds
  for (int cls = 0; cls < 2; ++cls) {
    const std::vector<int>& list = order[cls];
    if (list.empty()) continue;
    const Route rt = plan_route(p, items[list[0]].N);
    if (rt.digits) {
      int rc = run_class_digits(p, items, list, mode, ws, s, &sorted_item);
      if (rc) return rc;
      continue;
    }
    // FP64 tables: one contraction per item, rotations batched up to kMaxRot items.
    const bool mixed = rt.tc;
    std::vector<int> pend;                // items awaiting rotation; item pend[k] in slot k
    auto flush_rotation = [&]() -> int {  // rotate and publish every pending item
      if (pend.empty()) return DSHT_OK;
      RotMaps rm{};
      StatusOut so{};
      for (size_t k = 0; k < pend.size(); ++k) {
        rm.rot[k] = ws.alm_pol + nlm2 * k;
        rm.io[k] = items[pend[k]].alm;
        rm.flags[k] = ws.slot_flags + k;
        so.slot[k] = ws.slot_flags + k;
        so.status[k] = items[pend[k]].status;
      }
      prof_mark(p, DSHT_STAGE_ROTATE, s);
      if (mode == DSHT_MODE_CALL) launch_rotate_back_maps(g, rm, (int)pend.size(), s);
      launch_publish_flags(so, (int)pend.size(), ws.all_flags, s);
      pend.clear();
      return DSHT_OK;
    };
    for (size_t li = 0; li < list.size(); ++li) {
      const int i = list[li];
      const Item& item = items[i];
      const int slot = (int)pend.size();
      Workspace w2 = ws;
      w2.flags = ws.slot_flags + slot;
      if (item.same_points && sorted_item >= 0) {
        prof_mark(p, DSHT_STAGE_BIN_SUMS, s);  // the weight gather counts with the bin sums
        launch_gather(g, item.w, item.w_f32, item.N, ws, s);
      } else {
        prof_mark(p, DSHT_STAGE_POINTS, s);
        // The sort keeps the input index of every slot when later items share it.
        Workspace wp = ws;
        wp.piece_max = plan_piece_max(p, item.N);
        if (!(li + 1 < list.size() && items[list[li + 1]].same_points)) wp.sidx = nullptr;
        launch_points(g, item.theta, item.phi, item.w, item.w_f32, item.N, mode, wp, s, plan_uses_nufft(p, item.N));
        sorted_item = i;
      }
      prof_mark(p, DSHT_STAGE_BIN_SUMS, s);
      DSHT_CUDA_OK(cudaMemcpyAsync(w2.flags, ws.flags, sizeof(unsigned), cudaMemcpyDeviceToDevice, s));
      if (mixed) {
        if (int rc = launch_bin_sums_mixed(p, w2, item.N, s)) return rc;
      } else {
        launch_bin_sums_fp64(g, w2, s);
        w2.partial_f32 = 0;
      }
      prof_mark(p, DSHT_STAGE_FOLD, s);
      w2.alm_pol = ws.alm_pol + nlm2 * slot;
      w2.alm_equ = item.alm;
      launch_fold(g, w2, s);
      prof_mark(p, DSHT_STAGE_CONTRACT, s);
      if (rt.streamed)
        launch_contract_stream(g, p->tmYv, p->tmYd, ws.fold, ws.tile_live2, w2.alm_equ, w2.alm_pol, w2.flags, s);
      else
        launch_contract_fp64(g, p->Yv, p->Yd, w2, s);
      pend.push_back(i);
      if (pend.size() >= (size_t)kMaxRot) {
        int rc = flush_rotation();
        if (rc) return rc;
      }
    }
    int rc = flush_rotation();
    if (rc) return rc;
  }
  prof_mark(p, -1, s);
  if (int rc = launch_error("kernel launch")) return rc;
  DSHT_CUDA_OK(cudaGetLastError());
  return DSHT_OK;
}

void prof_mark(dsht_plan_s* p, int stage, cudaStream_t s) {
  if (!p->prof || !p->ev) return;
  if (p->ev_n >= dsht_plan_s::kProfMarks) return;  // later stages of a huge call go uncounted
  cudaEventRecord(p->ev[p->ev_n], s);
  p->ev_stage[p->ev_n] = (int8_t)stage;
  p->ev_n += 1;
}

// After the stream has been synchronised: add every interval between consecutive stage
// marks to its stage's total.
void collect_profile(dsht_plan_s* p) {
  if (!p->prof || !p->ev) return;
  for (int k = 0; k + 1 < p->ev_n; ++k) {
    const int st = p->ev_stage[k];
    float ms = 0.f;
    if (st >= 0 && st < DSHT_STAGE_COUNT && cudaEventElapsedTime(&ms, p->ev[k], p->ev[k + 1]) == cudaSuccess)
      p->prof_ms[st] += ms;
  }
  cudaGetLastError();
  p->ev_n = 0;
  p->prof_calls += 1;
}

int flags_to_status(unsigned f, int mode) {
  if (f & kFlagTimeout)
    return set_error(DSHT_ERR_CUDA, "a tensor-core pipeline wait timed out; results are invalid");
  if (f & kFlagPolarRange)
    return set_error(DSHT_ERR_POLAR_RANGE,
                     "theta must be in [ACos[xmax],ACos[-xmax]). (a polar point is still polar after the "
                     "rotation by 90 degrees; xmax is smaller than sin(pi/4))");
  if (f & kFlagThetaRange) return set_error(DSHT_ERR_THETA_RANGE, "theta must be in [ACos[xmax],ACos[-xmax]).");
  return DSHT_OK;
}

static int ensure_plan_workspace(dsht_plan_s* p, size_t bytes) {
  if (p->ws_bytes >= bytes) return DSHT_OK;
  if (p->ws) cudaFree(p->ws);
  p->ws = nullptr;
  p->ws_bytes = 0;
  DSHT_CUDA_OK(cudaMalloc(&p->ws, bytes));
  p->ws_bytes = bytes;
  return DSHT_OK;
}

}  // namespace dsht

using namespace dsht;


extern "C" {
static size_t call_layout(dsht_plan_s* p, int64_t N, int ntrans, bool multi, uint8_t* base, Workspace* ws);

const char* dsht_last_error(void) { return g_last_error.c_str(); }

const char* dsht_version(void) { return "directsht_b200 0.1 (sm_100a)"; }

int64_t dsht_index(int Nl, int ell, int m) { return hp_index(ell, m, Nl); }

int dsht_plan_create(int Nl, int Nx, double xmax, int flags, dsht_plan_t* plan) {
  if (!plan) return set_error(DSHT_ERR_INVALID, "plan pointer is NULL");
  *plan = nullptr;
  // Nx <= 12288: the sort histograms 4 (Nx - 1) keys in shared memory
  if (Nl < 1 || Nx < 2 || !(xmax > 0.0 && xmax < 1.0) || Nl > 16384 || Nx > 12288)
    return set_error(DSHT_ERR_INVALID, "invalid sizes Nl=%d Nx=%d xmax=%g", Nl, Nx, xmax);
  if (flags & ~DSHT_PLAN_F32_TABLES) return set_error(DSHT_ERR_INVALID, "unknown plan flags %d", flags);
  const bool f32_only = (flags & DSHT_PLAN_F32_TABLES) != 0;
  if (f32_only && (Nx > kTcMaxNx || Nl > 2048))
    return set_error(DSHT_ERR_INVALID, "compact-table plans need Nx <= %d and Nl <= 2048 (Nl=%d Nx=%d)", kTcMaxNx,
                     Nl, Nx);
  dsht_plan_s* p = new dsht_plan_s();
  p->g = make_geometry(Nl, Nx, xmax);
  cudaGetDevice(&p->device);
  auto fail = [&](cudaError_t e, const char* what) {
    cudaFree(p->Yv);
    cudaFree(p->Yd);
    cudaFree(p->nu_dinv);
    cudaFree(p->nu_tw);
    cudaFreeHost(p->h_flags);
    delete p;
    cudaGetLastError();
    return set_cuda_error(e, what, __FILE__, __LINE__);
  };
  cudaError_t e = cudaMallocHost(&p->h_flags, sizeof(unsigned));
  if (e != cudaSuccess) return fail(e, "plan allocation");
  if (Nl <= 2048) {  // the NUFFT bin sums of the mixed levels: 1/Psi(m) and the twiddles
    std::vector<double> dinv, tw;
    p->nu_logn = nufft_logn(Nl);
    nufft_host_tables(Nl, p->nu_logn, dinv, tw);
    e = cudaMalloc(&p->nu_dinv, sizeof(double) * dinv.size());
    if (e == cudaSuccess) e = cudaMalloc(&p->nu_tw, sizeof(double) * tw.size());
    if (e == cudaSuccess) e = cudaMemcpy(p->nu_dinv, dinv.data(), sizeof(double) * dinv.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->nu_tw, tw.data(), sizeof(double) * tw.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(e, "plan allocation");
  }
  if (f32_only) {
    // compact plan: the digit tables alone, built from FP64 columns a few m at a time
    if (int rc = build_digits(p)) {
      dsht_plan_destroy(p);
      return rc;
    }
    p->precision = DSHT_PREC_MIXED;
    *plan = p;
    return DSHT_OK;
  } else {
    const size_t tb = sizeof(double) * (size_t)p->g.Nlm * Nx;
    if (e == cudaSuccess) e = cudaMalloc(&p->Yv, tb);
    if (e == cudaSuccess) e = cudaMalloc(&p->Yd, tb);
    if (e != cudaSuccess) return fail(e, "plan allocation");
    launch_tables(p->g, p->Yv, p->Yd, 0);
  }
  e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return fail(e, "table build");
  if (contract_stream_ok(p->g) && make_table_tmap(&p->tmYv, p->Yv, Nx, p->g.Nlm) == DSHT_OK &&
      make_table_tmap(&p->tmYd, p->Yd, Nx, p->g.Nlm) == DSHT_OK) {
    p->tm64 = true;
  }
  *plan = p;
  return DSHT_OK;
}

int dsht_plan_destroy(dsht_plan_t p) {
  if (!p) return DSHT_OK;
  if (p->ev) {
    for (int k = 0; k < dsht_plan_s::kProfMarks; ++k)
      if (p->ev[k]) cudaEventDestroy(p->ev[k]);
    delete[] p->ev;
  }
  cudaFree(p->Yv);
  cudaFree(p->Yd);
  cudaFree(p->dig);
  cudaFree(p->rexp);
  cudaFree(p->tc_items);
  cudaFree(p->nu_dinv);
  cudaFree(p->nu_tw);
  cudaFree(p->ws);
  cudaFree(p->in);
  cudaFree(p->alm);
  cudaFreeHost(p->h_flags);
  delete p;
  return DSHT_OK;
}

int dsht_set_precision(dsht_plan_t p, int precision) {
  if (!p) return set_error(DSHT_ERR_INVALID, "plan is NULL");
  if (precision != DSHT_PREC_FP64 && precision != DSHT_PREC_MIXED && precision != DSHT_PREC_MIXED_F64_TABLES)
    return set_error(DSHT_ERR_INVALID, "unknown precision %d", precision);
  if (precision != DSHT_PREC_FP64 && p->g.Nl > 2048)
    return set_error(DSHT_ERR_INVALID, "mixed precision supports Nl <= 2048 (Nl=%d)", p->g.Nl);
  if (!p->Yv && precision != DSHT_PREC_MIXED)
    return set_error(DSHT_ERR_INVALID, "this plan holds compact tables only (DSHT_PLAN_F32_TABLES): precision MIXED");
  std::lock_guard<std::mutex> lock(p->mu);
  // MIXED streams the digit tables through the tensor-core contraction (built on first use);
  // where they cannot be built (Nx > kTcMaxNx, or no room beside the FP64 tables) its
  // transforms contract the FP64 tables instead, as DSHT_PREC_MIXED_F64_TABLES does.
  if (precision == DSHT_PREC_MIXED && !p->tmdig && p->g.Nx <= kTcMaxNx && build_digits(p) != DSHT_OK)
    cudaGetLastError();
  p->precision = precision;
  return DSHT_OK;
}

int dsht_plan_tune(dsht_plan_t p, int param, int value) {
  if (!p) return set_error(DSHT_ERR_INVALID, "plan is NULL");
  std::lock_guard<std::mutex> lock(p->mu);
  switch (param) {
    case DSHT_TUNE_PIECE_MAX:
      if (value != 0 && (value < 256 || value > 65536 || value % 32))
        return set_error(DSHT_ERR_INVALID, "piece size %d: 0 or a multiple of 32 in [256, 65536]", value);
      p->tune_piece_max = value;
      return DSHT_OK;
    case DSHT_TUNE_BIN_SUMS:
      if (value < DSHT_BIN_SUMS_AUTO || value > DSHT_BIN_SUMS_FP64)
        return set_error(DSHT_ERR_INVALID, "bin-sum method %d: AUTO (0), NUFFT (1), TC (2) or FP64 (3)", value);
      p->tune_bin_sums = value;
      return DSHT_OK;
    case DSHT_TUNE_MAPS_PER_PASS:
      if (value < 0 || value > kTcMaxMaps)
        return set_error(DSHT_ERR_INVALID, "maps per pass %d: 0 (most) or 1..%d", value, kTcMaxMaps);
      p->tune_maps_per_pass = value;
      return DSHT_OK;
  }
  return set_error(DSHT_ERR_INVALID, "unknown tuning parameter %d", param);
}

int dsht_plan_get_tune(dsht_plan_t p, int param, int* value) {
  if (!p || !value) return set_error(DSHT_ERR_INVALID, "invalid arguments");
  if (param == DSHT_TUNE_PIECE_MAX) *value = p->tune_piece_max;
  else if (param == DSHT_TUNE_MAPS_PER_PASS) *value = p->tune_maps_per_pass;
  else if (param == DSHT_TUNE_BIN_SUMS) *value = p->tune_bin_sums;
  else return set_error(DSHT_ERR_INVALID, "unknown tuning parameter %d", param);
  return DSHT_OK;
}

int dsht_get_precision(dsht_plan_t p, int* precision) {
  if (!p || !precision) return set_error(DSHT_ERR_INVALID, "invalid arguments");
  *precision = p->precision;
  return DSHT_OK;
}

int dsht_profile_enable(dsht_plan_t p, int enable) {
  if (!p) return set_error(DSHT_ERR_INVALID, "plan is NULL");
  std::lock_guard<std::mutex> lock(p->mu);
  if (enable && !p->ev) {
    p->ev = new cudaEvent_t[dsht_plan_s::kProfMarks]();
    for (int k = 0; k < dsht_plan_s::kProfMarks; ++k) DSHT_CUDA_OK(cudaEventCreate(&p->ev[k]));
  }
  p->ev_n = 0;
  p->prof = enable != 0;
  return DSHT_OK;
}

int dsht_profile_read(dsht_plan_t p, double* ms, int64_t* calls, int reset) {
  if (!p) return set_error(DSHT_ERR_INVALID, "plan is NULL");
  std::lock_guard<std::mutex> lock(p->mu);
  // stage marks of the last asynchronous call (dsht_enqueue_*), once its stream has finished
  if (p->ev_n > 0) collect_profile(p);
  if (ms)
    for (int i = 0; i < DSHT_STAGE_COUNT; ++i) ms[i] = p->prof_ms[i];
  if (calls) *calls = p->prof_calls;
  if (reset) {
    for (double& v : p->prof_ms) v = 0.0;
    p->prof_calls = 0;
  }
  return DSHT_OK;
}

int64_t dsht_launch_count(void) { return g_launches.load(); }

int64_t dsht_mixed_min_points(void) { return DSHT_MIXED_MIN_POINTS; }

int dsht_plan_info(dsht_plan_t p, int* Nl, int* Nx, double* xmax, int64_t* Nlm) {
  if (!p) return set_error(DSHT_ERR_INVALID, "plan is NULL");
  if (Nl) *Nl = p->g.Nl;
  if (Nx) *Nx = p->g.Nx;
  if (xmax) *xmax = p->g.xmax;
  if (Nlm) *Nlm = p->g.Nlm;
  return DSHT_OK;
}

int dsht_workspace_size(dsht_plan_t p, int64_t N, size_t* bytes) {
  if (!p || !bytes || N < 0) return set_error(DSHT_ERR_INVALID, "invalid arguments");
  *bytes = call_layout(p, N, 1, false, nullptr, nullptr);
  return DSHT_OK;
}

// Workspace of a call: single transforms use the lean layout; multi-transform calls add
// the gather records, fold digit columns of a contraction pass, rotation and flag slots.
static size_t call_layout(dsht_plan_s* p, int64_t N, int ntrans, bool multi, uint8_t* base, Workspace* ws) {
  // maps per tensor-core contraction pass (digit tables): up to kTcMaxMaps unless tuned
  const int tc = multi ? std::min(std::max(ntrans, 1), p->tune_maps_per_pass > 0 ? p->tune_maps_per_pass
                                                                                  : kTcMaxMaps) : 1;
  return workspace_layout(p->g, N, plan_piece_max(p, N), base, ws, multi, tc);
}

// Resolves the workspace (caller's or the plan's, grown on demand) for a call.
static int call_workspace(dsht_plan_s* p, size_t need, void* workspace, size_t workspace_bytes,
                          std::unique_lock<std::mutex>& lock, uint8_t** base) {
  *base = reinterpret_cast<uint8_t*>(workspace);
  if (*base) {
    if (workspace_bytes < need)
      return set_error(DSHT_ERR_NOMEM, "workspace of %zu bytes is smaller than the %zu needed", workspace_bytes, need);
    return DSHT_OK;
  }
  lock.lock();
  int rc = ensure_plan_workspace(p, need);
  if (rc) return rc;
  *base = reinterpret_cast<uint8_t*>(p->ws);
  return DSHT_OK;
}

// Enqueues nmaps maps of one point set; sync = false leaves the flags in *status (device).
static int maps_device(dsht_plan_t p, const double* theta, const double* phi, const void* w, int w_dtype,
                       int64_t N, int nmaps, int64_t w_stride, int mode, double* alm, void* workspace,
                       size_t workspace_bytes, void* stream, bool sync, unsigned* status) {
  if (!p || !alm || N < 0 || (N > 0 && (!theta || !phi || !w)))
    return set_error(DSHT_ERR_INVALID, "invalid arguments");
  if (mode != DSHT_MODE_CALL && mode != DSHT_MODE_BASIC) return set_error(DSHT_ERR_INVALID, "bad mode %d", mode);
  if (w_dtype != DSHT_W_F64 && w_dtype != DSHT_W_F32) return set_error(DSHT_ERR_INVALID, "bad w_dtype %d", w_dtype);
  if (nmaps < 1 || (nmaps > 1 && w_stride < N))
    return set_error(DSHT_ERR_INVALID, "invalid maps (nmaps=%d, w_stride=%lld)", nmaps, (long long)w_stride);
  if (N > (int64_t)0xfffffff0LL) return set_error(DSHT_ERR_INVALID, "too many points (%lld)", (long long)N);
  if (N == 0 && mode == DSHT_MODE_BASIC)
    return set_error(DSHT_ERR_EMPTY, "The theta array seems to be empty!");
  if (!sync && !workspace) return set_error(DSHT_ERR_INVALID, "an enqueued call needs a caller workspace");
  const bool multi = nmaps > 1 || w_dtype == DSHT_W_F32;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  std::unique_lock<std::mutex> lock(p->mu, std::defer_lock);
  const size_t need = call_layout(p, N, nmaps, multi, nullptr, nullptr);
  uint8_t* base = nullptr;
  int rc = call_workspace(p, need, workspace, workspace_bytes, lock, &base);
  if (rc) return rc;
  if (N == 0) {  // __call__ on no points returns zeros (sht/sht.py:127,150)
    DSHT_CUDA_OK(cudaMemsetAsync(alm, 0, sizeof(double) * 2 * p->g.Nlm * nmaps, s));
    if (status) DSHT_CUDA_OK(cudaMemsetAsync(status, 0, sizeof(unsigned), s));
    return DSHT_OK;
  }
  Workspace ws;
  call_layout(p, N, nmaps, multi, base, &ws);
  const unsigned* flags = ws.flags;
  if (multi) {
    std::vector<Item> items(nmaps);
    const size_t esz = w_dtype == DSHT_W_F32 ? sizeof(float) : sizeof(double);
    for (int k = 0; k < nmaps; ++k)
      items[k] = Item{theta, phi, static_cast<const uint8_t*>(w) + esz * (size_t)w_stride * k,
                      w_dtype == DSHT_W_F32, N, alm + 2 * p->g.Nlm * k, k > 0, nullptr};
    rc = run_items(p, items.data(), nmaps, mode, ws, s);
    flags = ws.all_flags;
  } else {
    rc = run_pipeline(p, theta, phi, static_cast<const double*>(w), N, mode, alm, ws, s);
  }
  if (rc) return rc;
  if (!sync) {
    if (status) DSHT_CUDA_OK(cudaMemcpyAsync(status, flags, sizeof(unsigned), cudaMemcpyDeviceToDevice, s));
    return DSHT_OK;
  }
  unsigned hf = 0;
  DSHT_CUDA_OK(cudaMemcpyAsync(&hf, flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  DSHT_CUDA_OK(cudaStreamSynchronize(s));
  collect_profile(p);
  return flags_to_status(hf, mode);
}

static int execute_device(dsht_plan_t p, const double* theta, const double* phi, const void* w, int w_dtype,
                          int64_t N, int nmaps, int64_t w_stride, int mode, double* alm, void* workspace,
                          size_t workspace_bytes, void* stream) {
  return maps_device(p, theta, phi, w, w_dtype, N, nmaps, w_stride, mode, alm, workspace, workspace_bytes, stream,
                     true, nullptr);
}

// Enqueues a batch of independent transforms on one plan.
static int batch_device(dsht_plan_t p, int ntrans, const double* const* theta, const double* const* phi,
                        const double* const* w, const int64_t* N, int mode, double* const* alm, unsigned* status,
                        void* workspace, size_t workspace_bytes, void* stream, bool sync) {
  if (!p || ntrans < 0 || (ntrans > 0 && (!theta || !phi || !w || !N || !alm)))
    return set_error(DSHT_ERR_INVALID, "invalid arguments");
  if (mode != DSHT_MODE_CALL && mode != DSHT_MODE_BASIC) return set_error(DSHT_ERR_INVALID, "bad mode %d", mode);
  if (!sync && !workspace) return set_error(DSHT_ERR_INVALID, "an enqueued call needs a caller workspace");
  int64_t nmax = 0;
  for (int i = 0; i < ntrans; ++i) {
    if (N[i] < 0 || N[i] > (int64_t)0xfffffff0LL || !alm[i] || (N[i] > 0 && (!theta[i] || !phi[i] || !w[i])))
      return set_error(DSHT_ERR_INVALID, "invalid transform %d of the batch", i);
    if (N[i] == 0 && mode == DSHT_MODE_BASIC)
      return set_error(DSHT_ERR_EMPTY, "The theta array seems to be empty! (transform %d of the batch)", i);
    nmax = std::max(nmax, N[i]);
  }
  if (ntrans == 0) return DSHT_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  std::unique_lock<std::mutex> lock(p->mu, std::defer_lock);
  const size_t need = call_layout(p, nmax, ntrans, true, nullptr, nullptr);
  uint8_t* base = nullptr;
  int rc = call_workspace(p, need, workspace, workspace_bytes, lock, &base);
  if (rc) return rc;
  // The piece layout follows the largest N: every transform uses the same workspace carve.
  Workspace ws;
  call_layout(p, nmax, ntrans, true, base, &ws);
  std::vector<Item> items;
  for (int i = 0; i < ntrans; ++i) {
    if (N[i] == 0) {
      DSHT_CUDA_OK(cudaMemsetAsync(alm[i], 0, sizeof(double) * 2 * p->g.Nlm, s));
      if (status) DSHT_CUDA_OK(cudaMemsetAsync(status + i, 0, sizeof(unsigned), s));
      continue;
    }
    items.push_back(Item{theta[i], phi[i], w[i], 0, N[i], alm[i], false, status ? status + i : nullptr});
  }
  if (!items.empty()) {
    rc = run_items(p, items.data(), (int)items.size(), mode, ws, s);
    if (rc) return rc;
  } else {
    DSHT_CUDA_OK(cudaMemsetAsync(ws.all_flags, 0, sizeof(unsigned), s));
  }
  if (!sync) return DSHT_OK;
  unsigned hf = 0;
  DSHT_CUDA_OK(cudaMemcpyAsync(&hf, ws.all_flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  DSHT_CUDA_OK(cudaStreamSynchronize(s));
  collect_profile(p);
  return flags_to_status(hf, mode);
}

int dsht_test_point_keys(dsht_plan_t p, const double* theta, const double* phi, int64_t N, int mode, uint32_t* keys,
                         unsigned* flags, void* stream) {
  if (!p || N < 1 || N > (int64_t)0xfffffff0LL || !theta || !phi || !keys || !flags)
    return set_error(DSHT_ERR_INVALID, "invalid arguments");
  if (mode != DSHT_MODE_CALL && mode != DSHT_MODE_BASIC) return set_error(DSHT_ERR_INVALID, "bad mode %d", mode);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  std::unique_lock<std::mutex> lock(p->mu, std::defer_lock);
  const size_t need = call_layout(p, N, 1, false, nullptr, nullptr);
  uint8_t* base = nullptr;
  int rc = call_workspace(p, need, nullptr, 0, lock, &base);
  if (rc) return rc;
  Workspace ws;
  call_layout(p, N, 1, false, base, &ws);
  // the sort also moves weights; the keys do not depend on them, so theta stands in
  launch_points(p->g, theta, phi, theta, 0, N, mode, ws, s);
  DSHT_CUDA_OK(cudaMemcpyAsync(keys, ws.key, sizeof(uint32_t) * N, cudaMemcpyDeviceToDevice, s));
  DSHT_CUDA_OK(cudaMemcpyAsync(flags, ws.flags, sizeof(unsigned), cudaMemcpyDeviceToDevice, s));
  DSHT_CUDA_OK(cudaStreamSynchronize(s));
  DSHT_CUDA_OK(cudaGetLastError());
  return DSHT_OK;
}

int dsht_execute(dsht_plan_t p, const double* theta, const double* phi, const double* w, int64_t N, int mode,
                 double* alm, void* workspace, size_t workspace_bytes, void* stream) {
  return execute_device(p, theta, phi, w, DSHT_W_F64, N, 1, N, mode, alm, workspace, workspace_bytes, stream);
}

int dsht_workspace_size_maps(dsht_plan_t p, int64_t N, int nmaps, size_t* bytes) {
  if (!p || !bytes || N < 0 || nmaps < 1) return set_error(DSHT_ERR_INVALID, "invalid arguments");
  // float32 single maps take the multi-transform layout too; size for it.
  *bytes = call_layout(p, N, nmaps, true, nullptr, nullptr);
  return DSHT_OK;
}

int dsht_execute_maps(dsht_plan_t p, const double* theta, const double* phi, const void* w, int w_dtype, int64_t N,
                      int nmaps, int64_t w_stride, int mode, double* alm, void* workspace, size_t workspace_bytes,
                      void* stream) {
  return execute_device(p, theta, phi, w, w_dtype, N, nmaps, w_stride, mode, alm, workspace, workspace_bytes,
                        stream);
}

int dsht_enqueue_maps(dsht_plan_t p, const double* theta, const double* phi, const void* w, int w_dtype, int64_t N,
                      int nmaps, int64_t w_stride, int mode, double* alm, unsigned* status, void* workspace,
                      size_t workspace_bytes, void* stream) {
  return maps_device(p, theta, phi, w, w_dtype, N, nmaps, w_stride, mode, alm, workspace, workspace_bytes, stream,
                     false, status);
}

int dsht_workspace_size_batch(dsht_plan_t p, int64_t max_N, int ntrans, size_t* bytes) {
  if (!p || !bytes || max_N < 0 || ntrans < 1) return set_error(DSHT_ERR_INVALID, "invalid arguments");
  *bytes = call_layout(p, max_N, ntrans, true, nullptr, nullptr);
  return DSHT_OK;
}

int dsht_execute_batch(dsht_plan_t p, int ntrans, const double* const* theta, const double* const* phi,
                       const double* const* w, const int64_t* N, int mode, double* const* alm, void* workspace,
                       size_t workspace_bytes, void* stream) {
  return batch_device(p, ntrans, theta, phi, w, N, mode, alm, nullptr, workspace, workspace_bytes, stream, true);
}

int dsht_enqueue_batch(dsht_plan_t p, int ntrans, const double* const* theta, const double* const* phi,
                       const double* const* w, const int64_t* N, int mode, double* const* alm, unsigned* status,
                       void* workspace, size_t workspace_bytes, void* stream) {
  return batch_device(p, ntrans, theta, phi, w, N, mode, alm, status, workspace, workspace_bytes, stream, false);
}

int dsht_status(unsigned flags, int mode) {
  if (mode != DSHT_MODE_CALL && mode != DSHT_MODE_BASIC) return set_error(DSHT_ERR_INVALID, "bad mode %d", mode);
  return flags_to_status(flags, mode);
}

int dsht_execute_host(dsht_plan_t p, const double* theta, const double* phi, const double* w, int64_t N, int mode,
                      double* alm_host) {
  if (!p || !alm_host || N < 0 || (N > 0 && (!theta || !phi || !w)))
    return set_error(DSHT_ERR_INVALID, "invalid arguments");
  if (N == 0 && mode == DSHT_MODE_BASIC) return set_error(DSHT_ERR_EMPTY, "The theta array seems to be empty!");
  std::lock_guard<std::mutex> lock(p->mu);
  const int piece_max = plan_piece_max(p, N);
  const size_t need = workspace_layout(p->g, N, piece_max, nullptr, nullptr);
  int rc = ensure_plan_workspace(p, need);
  if (rc) return rc;
  if (p->in_n < N) {
    cudaFree(p->in);
    p->in = nullptr;
    p->in_n = 0;
    DSHT_CUDA_OK(cudaMalloc(&p->in, sizeof(double) * 3 * (size_t)N));
    p->in_n = N;
  }
  if (!p->alm) DSHT_CUDA_OK(cudaMalloc(&p->alm, sizeof(double) * 2 * p->g.Nlm));
  cudaStream_t s = 0;
  if (N > 0) {
    DSHT_CUDA_OK(cudaMemcpyAsync(p->in, theta, sizeof(double) * N, cudaMemcpyHostToDevice, s));
    DSHT_CUDA_OK(cudaMemcpyAsync(p->in + N, phi, sizeof(double) * N, cudaMemcpyHostToDevice, s));
    DSHT_CUDA_OK(cudaMemcpyAsync(p->in + 2 * N, w, sizeof(double) * N, cudaMemcpyHostToDevice, s));
  }
  unsigned hf = 0;
  if (N == 0) {
    DSHT_CUDA_OK(cudaMemsetAsync(p->alm, 0, sizeof(double) * 2 * p->g.Nlm, s));
  } else {
    Workspace ws;
    workspace_layout(p->g, N, piece_max, reinterpret_cast<uint8_t*>(p->ws), &ws);
    rc = run_pipeline(p, p->in, p->in + N, p->in + 2 * N, N, mode, p->alm, ws, s);
    if (rc) return rc;
    DSHT_CUDA_OK(cudaMemcpyAsync(p->h_flags, ws.flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  }
  DSHT_CUDA_OK(cudaMemcpyAsync(alm_host, p->alm, sizeof(double) * 2 * p->g.Nlm, cudaMemcpyDeviceToHost, s));
  DSHT_CUDA_OK(cudaStreamSynchronize(s));
  if (N > 0) {
    hf = *p->h_flags;
    collect_profile(p);
  }
  return flags_to_status(hf, mode);
}

int dsht_rotate_back(dsht_plan_t p, const double* alm_rot, const double* alm_add, double* alm_out,
                     void* stream) {
  if (!p || !alm_rot || !alm_out) return set_error(DSHT_ERR_INVALID, "invalid arguments");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (!alm_add) {
    DSHT_CUDA_OK(cudaMemsetAsync(alm_out, 0, sizeof(double) * 2 * p->g.Nlm, s));
    alm_add = alm_out;
  }
  launch_rotate_back(p->g, alm_rot, alm_add, alm_out, nullptr, s);
  DSHT_CUDA_OK(cudaGetLastError());
  return DSHT_OK;
}

// Rows [r0, r0 + n) (Healpy order) of a compact plan's table, decoded from the digits, to
// host memory (through a device buffer of at most 2^24 values at a time).
static int decode_rows_to_host(dsht_plan_s* p, int which, int64_t r0, int64_t n, double* out) {
  const int Nx = p->g.Nx;
  const int64_t per = std::max<int64_t>(1, ((int64_t)1 << 24) / Nx);
  double* buf = nullptr;
  DSHT_CUDA_OK(cudaMalloc(&buf, sizeof(double) * (size_t)std::min(per, n) * Nx));
  int rc = DSHT_OK;
  for (int64_t i = 0; i < n && rc == DSHT_OK; i += per) {
    const int64_t c = std::min(per, n - i);
    launch_table_decode(p->g, which, r0 + i, c, p->dig, p->rexp, buf, 0);
    const cudaError_t e = cudaMemcpy(out + i * Nx, buf, sizeof(double) * (size_t)c * Nx, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = set_cuda_error(e, "table decode", __FILE__, __LINE__);
  }
  cudaFree(buf);
  return rc;
}

int dsht_get_row(dsht_plan_t p, int which, int ell, int m, double* out) {
  if (!p || !out || which < 0 || which > 1 || m < 0 || ell < m || ell >= p->g.Nl)
    return set_error(DSHT_ERR_INVALID, "invalid row (which=%d, l=%d, m=%d)", which, ell, m);
  const int64_t row = hp_index(ell, m, p->g.Nl);
  if (p->Yv) {
    const double* t = which == 0 ? p->Yv : p->Yd;
    DSHT_CUDA_OK(cudaMemcpy(out, t + row * p->g.Nx, sizeof(double) * p->g.Nx, cudaMemcpyDeviceToHost));
    return DSHT_OK;
  }
  return decode_rows_to_host(p, which, row, 1, out);
}

int dsht_get_table(dsht_plan_t p, int which, double* out) {
  if (!p || !out || which < 0 || which > 1) return set_error(DSHT_ERR_INVALID, "invalid arguments");
  const size_t n = (size_t)p->g.Nlm * p->g.Nx;
  if (p->Yv) {
    const double* t = which == 0 ? p->Yv : p->Yd;
    DSHT_CUDA_OK(cudaMemcpy(out, t, sizeof(double) * n, cudaMemcpyDeviceToHost));
    return DSHT_OK;
  }
  return decode_rows_to_host(p, which, 0, p->g.Nlm, out);
}

int dsht_get_table_mlayout(dsht_plan_t p, int which, double* out, int out_on_device, void* stream) {
  if (!p || !out || which < 0 || which > 1) return set_error(DSHT_ERR_INVALID, "invalid arguments");
  const int Nl = p->g.Nl, Nx = p->g.Nx;
  const size_t plane = (size_t)Nl * Nx;  // one m: Nl rows of Nx
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (out_on_device) {
    if (p->Yv) {
      launch_table_mlayout(p->g, which == 0 ? p->Yv : p->Yd, out, s);
    } else {  // compact plan: decode each column's rows into its slice of out
      DSHT_CUDA_OK(cudaMemsetAsync(out, 0, sizeof(double) * plane * Nl, s));
      for (int m = 0; m < Nl; ++m)
        launch_table_decode(p->g, which, hp_index(m, m, Nl), Nl - m, p->dig, p->rexp, out + (size_t)m * plane, s);
    }
    return launch_error("table_mlayout_kernel");
  }
  for (int m = 0; m < Nl; ++m) {
    // Rows l = m..Nl-1 of column m are contiguous in Healpy order; they fill k = l - m.
    const int64_t row0 = hp_index(m, m, Nl);
    const size_t n = (size_t)(Nl - m) * Nx;
    double* dst = out + (size_t)m * plane;
    if (p->Yv) {
      const double* t = (which == 0 ? p->Yv : p->Yd) + (size_t)row0 * Nx;
      DSHT_CUDA_OK(cudaMemcpy(dst, t, sizeof(double) * n, cudaMemcpyDeviceToHost));
    } else if (int rc = decode_rows_to_host(p, which, row0, Nl - m, dst)) {
      return rc;
    }
    std::memset(dst + n, 0, sizeof(double) * (plane - n));  // k >= Nl - m: l >= Nl (unphysical)
  }
  return DSHT_OK;
}

int dsht_alm2cl(int Nl, const double* alm, double* cl) {
  if (Nl < 1 || !alm || !cl) return set_error(DSHT_ERR_INVALID, "invalid arguments");
  for (int l = 0; l < Nl; ++l) {
    const int64_t i0 = hp_index(l, 0, Nl);
    double c = alm[2 * i0] * alm[2 * i0];
    for (int m = 1; m <= l; ++m) {
      const int64_t i = hp_index(l, m, Nl);
      c += 2 * (alm[2 * i] * alm[2 * i] + alm[2 * i + 1] * alm[2 * i + 1]);
    }
    cl[l] = c / (2 * l + 1.0);
  }
  return DSHT_OK;
}

// ---- drop-ins for csht/sht_helper.so ------------------------------------------------------
static std::mutex g_cache_mu;
static std::map<std::tuple<int, int, double, int>, dsht_plan_t> g_cache;

static int cached_plan(int Nl, int Nx, double xmax, dsht_plan_t* out) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_cache_mu);
  auto key = std::make_tuple(Nl, Nx, xmax, dev);
  auto it = g_cache.find(key);
  if (it != g_cache.end()) {
    *out = it->second;
    return DSHT_OK;
  }
  dsht_plan_t p = nullptr;
  int rc = dsht_plan_create(Nl, Nx, xmax, 0, &p);
  if (rc) return rc;
  g_cache[key] = p;
  *out = p;
  return DSHT_OK;
}

int dsht_make_table(int Nl, int Nx, double xmax, double* Yv, double* Yd) {
  dsht_plan_t p = nullptr;
  int rc = cached_plan(Nl, Nx, xmax, &p);
  if (rc) return rc;
  if (Yv && (rc = dsht_get_table(p, 0, Yv))) return rc;
  if (Yd && (rc = dsht_get_table(p, 1, Yd))) return rc;
  return DSHT_OK;
}

int dsht_do_transform(int Nl, int Nx, double xmax, double* Yv, double* Yd, int Np, double* cost, double* phi,
                      double* wt, double* carr, double* sarr) {
  (void)Yv;
  (void)Yd;
  if (Np < 0 || !carr || !sarr || (Np > 0 && (!cost || !phi || !wt)))
    return set_error(DSHT_ERR_INVALID, "invalid arguments");
  dsht_plan_t p = nullptr;
  int rc = cached_plan(Nl, Nx, xmax, &p);
  if (rc) return rc;
  // |cos theta| as theta in [0, pi/2]: no parity, as do_transform leaves it to the caller.
  std::vector<double> th((size_t)Np);
  for (int i = 0; i < Np; ++i) th[i] = std::acos(std::fabs(cost[i]));
  std::vector<double> alm((size_t)2 * p->g.Nlm);
  if (Np == 0) {
    std::memset(carr, 0, sizeof(double) * p->g.Nlm);
    std::memset(sarr, 0, sizeof(double) * p->g.Nlm);
    return DSHT_OK;
  }
  rc = dsht_execute_host(p, th.data(), phi, wt, Np, DSHT_MODE_BASIC, alm.data());
  if (rc) return rc;
  for (int64_t i = 0; i < p->g.Nlm; ++i) {
    carr[i] = alm[2 * i];
    sarr[i] = -alm[2 * i + 1];
  }
  return DSHT_OK;
}

}  // extern "C"
