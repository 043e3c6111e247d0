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

void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

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

int default_piece_max(const Geometry& g, int64_t N) {
  int64_t p = (N + 2047) / 2048;
  if (p < 512) p = 512;
  if (p > 2048) p = 2048;
  return (int)p;
}

size_t workspace_layout(const Geometry& g, int64_t N, int piece_max, uint8_t* base, Workspace* ws, bool maps) {
  size_t off = 0;
  auto take = [&](size_t bytes) -> uint8_t* {
    uint8_t* p = base ? base + off : nullptr;
    off = align_up(off + bytes, 256);
    return p;
  };
  const int64_t n = N > 0 ? N : 1;
  const int64_t pmax = std::min<int64_t>(g.nkeys, n) + (n + piece_max - 1) / piece_max;
  const int tile = 128;
  const int ntile = (g.Nx + tile - 1) / tile;
  Workspace w{};
  w.key = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * n));
  w.rec = reinterpret_cast<double*>(take(sizeof(double) * 3 * n));
  w.pay = reinterpret_cast<double*>(take(sizeof(double) * 6 * n));
  if (maps) {
    w.sidx = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * n));
    w.st = reinterpret_cast<double*>(take(sizeof(double) * n));
  }
  w.count = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * (g.nkeys + 1)));
  w.offset = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * (g.nkeys + 1)));
  w.cursor = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * (g.nkeys + 1)));
  w.piece_first = reinterpret_cast<int*>(take(sizeof(int) * (g.nkeys + 1)));
  w.piece_key = reinterpret_cast<int*>(take(sizeof(int) * pmax));
  w.piece_start = reinterpret_cast<int64_t*>(take(sizeof(int64_t) * pmax));
  w.piece_len = reinterpret_cast<int*>(take(sizeof(int) * pmax));
  w.npieces = reinterpret_cast<int*>(take(sizeof(int)));
  w.flags = reinterpret_cast<unsigned*>(take(sizeof(unsigned)));
  w.partial = reinterpret_cast<double*>(take(sizeof(double) * 8 * (size_t)g.Nl * pmax));
  w.fold = reinterpret_cast<double*>(take(sizeof(double) * 16 * (size_t)g.Nl * g.Nx));
  w.tile_live = reinterpret_cast<uint8_t*>(take(2 * (size_t)ntile));
  w.tile_live2 = reinterpret_cast<uint8_t*>(take(2 * (size_t)((g.Nx + 255) / 256)));
  w.alm_equ = reinterpret_cast<double*>(take(sizeof(double) * 2 * (size_t)g.Nlm));
  w.alm_pol = reinterpret_cast<double*>(take(sizeof(double) * 2 * (size_t)g.Nlm));
  w.npts = n;
  w.pmax = pmax;
  w.piece_max = piece_max;
  w.bytes = off;
  if (ws) *ws = w;
  return off;
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
  auto mark = [&](int i) {
    if (marks && p->prof) cudaEventRecord(p->ev[i], s);
  };
  Workspace w2 = ws;
  // Small transforms run the FP64 stages even on a mixed-precision plan.
  const bool mixed = p->precision != DSHT_PREC_FP64 && N >= DSHT_MIXED_MIN_POINTS;
  const bool f32_tables = mixed && p->precision == DSHT_PREC_MIXED && p->tm32;
  if (mixed) {
    int rc = launch_bin_sums_tc(g, ws, s);
    if (rc) return rc;
    w2.partial_f32 = 1;
  } else {
    launch_bin_sums_fp64(g, ws, s);
    w2.partial_f32 = 0;
  }
  w2.fold_f32 = f32_tables ? 1 : 0;
  mark(2);
  launch_fold(g, w2, s);
  mark(3);
  if (f32_tables)
    launch_contract_stream(g, true, p->tmYv32, p->tmYd32, ws, s);
  else if (p->tm64)
    launch_contract_stream(g, false, p->tmYv, p->tmYd, ws, s);
  else
    launch_contract_fp64(g, p->Yv, p->Yd, ws, s);
  mark(4);
  if (mode == DSHT_MODE_CALL) {
    launch_rotate_back(g, ws.alm_pol, ws.alm_equ, alm, ws.flags, s);
  } else {
    DSHT_CUDA_OK(cudaMemcpyAsync(alm, ws.alm_equ, sizeof(double) * 2 * g.Nlm, cudaMemcpyDeviceToDevice, s));
  }
  mark(5);
  DSHT_CUDA_OK(cudaGetLastError());
  return DSHT_OK;
}

// Runs the whole pipeline on `s`; leaves the device flags in ws.flags.
int run_pipeline(dsht_plan_s* p, const double* theta, const double* phi, const double* w, int64_t N,
                        int mode, double* alm, const Workspace& ws, cudaStream_t s) {
  p->prof_maps = false;
  if (p->prof) cudaEventRecord(p->ev[0], s);
  launch_points(p->g, theta, phi, w, 0, N, mode, ws, s);
  if (p->prof) cudaEventRecord(p->ev[1], s);
  return run_after_sort(p, N, mode, alm, ws, s, true);
}

// Several weight maps on one point set: one classification and sort (which also records the
// input index and t of every sorted slot), then for every further map a gather rebuilds the
// weighted payload and the later stages run again.  Stage events cover the last map.
int run_maps(dsht_plan_s* p, const double* theta, const double* phi, const void* w, int w_f32, int64_t N,
             int nmaps, int64_t w_stride, int mode, double* alm, const Workspace& ws, cudaStream_t s) {
  const size_t esz = w_f32 ? sizeof(float) : sizeof(double);
  const size_t nlm2 = 2 * (size_t)p->g.Nlm;
  p->prof_maps = true;
  if (p->prof) cudaEventRecord(p->ev[0], s);
  launch_points(p->g, theta, phi, w, w_f32, N, mode, ws, s);
  if (p->prof) cudaEventRecord(p->ev[1], s);
  for (int k = 0; k < nmaps; ++k) {
    const bool last = k == nmaps - 1;
    if (last && p->prof) cudaEventRecord(p->ev[DSHT_STAGE_COUNT + 1], s);
    if (k > 0) launch_gather(p->g, static_cast<const uint8_t*>(w) + esz * (size_t)w_stride * k, w_f32, N, ws, s);
    int rc = run_after_sort(p, N, mode, alm + nlm2 * k, ws, s, last);
    if (rc) return rc;
  }
  return DSHT_OK;
}

// After the stream has been synchronised: fold the stage events into the totals.
void collect_profile(dsht_plan_s* p) {
  if (!p->prof) return;
  for (int i = 0; i < DSHT_STAGE_COUNT; ++i) {
    float ms = 0.f;
    cudaEvent_t a = (p->prof_maps && i == DSHT_STAGE_BIN_SUMS) ? p->ev[DSHT_STAGE_COUNT + 1] : p->ev[i];
    if (cudaEventElapsedTime(&ms, a, p->ev[i + 1]) == cudaSuccess) p->prof_ms[i] += ms;
  }
  p->prof_calls += 1;
  p->prof_maps = false;
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

const char* dsht_last_error(void) { return g_last_error.c_str(); }

const char* dsht_version(void) { return "directsht_b200 0.1 (sm_100a)"; }

int64_t dsht_index(int Nl, int ell, int m) { return hp_index(ell, m, Nl); }

int dsht_plan_create(int Nl, int Nx, double xmax, int flags, dsht_plan_t* plan) {
  (void)flags;
  if (!plan) return set_error(DSHT_ERR_INVALID, "plan pointer is NULL");
  *plan = nullptr;
  if (Nl < 1 || Nx < 2 || !(xmax > 0.0 && xmax < 1.0) || Nl > 16384 || Nx > 65536)
    return set_error(DSHT_ERR_INVALID, "invalid sizes Nl=%d Nx=%d xmax=%g", Nl, Nx, xmax);
  dsht_plan_s* p = new dsht_plan_s();
  p->g = make_geometry(Nl, Nx, xmax);
  cudaGetDevice(&p->device);
  const size_t tb = sizeof(double) * (size_t)p->g.Nlm * Nx;
  cudaError_t e = cudaMalloc(&p->Yv, tb);
  if (e == cudaSuccess) e = cudaMalloc(&p->Yd, tb);
  if (e == cudaSuccess) e = cudaMallocHost(&p->h_flags, sizeof(unsigned));
  if (e != cudaSuccess) {
    cudaFree(p->Yv);
    cudaFree(p->Yd);
    delete p;
    return set_cuda_error(e, "plan allocation", __FILE__, __LINE__);
  }
  launch_tables(p->g, p->Yv, p->Yd, 0);
  e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    cudaFree(p->Yv);
    cudaFree(p->Yd);
    cudaFreeHost(p->h_flags);
    delete p;
    return set_cuda_error(e, "table build", __FILE__, __LINE__);
  }
  if (contract_stream_ok(p->g, sizeof(double)) &&
      make_table_tmap(&p->tmYv, p->Yv, sizeof(double), Nx, p->g.Nlm) == DSHT_OK &&
      make_table_tmap(&p->tmYd, p->Yd, sizeof(double), Nx, p->g.Nlm) == DSHT_OK)
    p->tm64 = true;
  *plan = p;
  return DSHT_OK;
}

int dsht_plan_destroy(dsht_plan_t p) {
  if (!p) return DSHT_OK;
  for (auto& e : p->ev)
    if (e) cudaEventDestroy(e);
  cudaFree(p->Yv);
  cudaFree(p->Yd);
  cudaFree(p->Yv32);
  cudaFree(p->Yd32);
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
  std::lock_guard<std::mutex> lock(p->mu);
  if (precision == DSHT_PREC_MIXED && !p->Yv32) {
    const size_t tb = sizeof(float) * (size_t)p->g.Nlm * p->g.Nx;
    cudaError_t e = cudaMalloc(&p->Yv32, tb);
    if (e == cudaSuccess) e = cudaMalloc(&p->Yd32, tb);
    if (e != cudaSuccess) {  // no room for the FP32 copies: stream the FP64 tables instead
      cudaFree(p->Yv32);
      cudaFree(p->Yd32);
      p->Yv32 = nullptr;
      p->Yd32 = nullptr;
      cudaGetLastError();
      p->precision = precision;
      return DSHT_OK;
    }
    launch_tables_to_f32(p->g, p->Yv, p->Yd, p->Yv32, p->Yd32, 0);
    DSHT_CUDA_OK(cudaDeviceSynchronize());
    if (contract_stream_ok(p->g, sizeof(float)) &&
        make_table_tmap(&p->tmYv32, p->Yv32, sizeof(float), p->g.Nx, p->g.Nlm) == DSHT_OK &&
        make_table_tmap(&p->tmYd32, p->Yd32, sizeof(float), p->g.Nx, p->g.Nlm) == DSHT_OK)
      p->tm32 = true;
  }
  p->precision = precision;
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
  if (enable && !p->ev[0])
    for (auto& e : p->ev) DSHT_CUDA_OK(cudaEventCreate(&e));
  p->prof = enable != 0;
  return DSHT_OK;
}

int dsht_profile_read(dsht_plan_t p, double* ms, int64_t* calls, int reset) {
  if (!p) return set_error(DSHT_ERR_INVALID, "plan is NULL");
  std::lock_guard<std::mutex> lock(p->mu);
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
  *bytes = workspace_layout(p->g, N, default_piece_max(p->g, N), nullptr, nullptr);
  return DSHT_OK;
}

static int execute_device(dsht_plan_t p, const double* theta, const double* phi, const void* w, int w_dtype,
                          int64_t N, int nmaps, int64_t w_stride, int mode, double* alm, void* workspace,
                          size_t workspace_bytes, void* stream) {
  if (!p || !alm || N < 0 || (N > 0 && (!theta || !phi || !w)))
    return set_error(DSHT_ERR_INVALID, "invalid arguments");
  if (mode != DSHT_MODE_CALL && mode != DSHT_MODE_BASIC) return set_error(DSHT_ERR_INVALID, "bad mode %d", mode);
  if (w_dtype != DSHT_W_F64 && w_dtype != DSHT_W_F32) return set_error(DSHT_ERR_INVALID, "bad w_dtype %d", w_dtype);
  if (nmaps < 1 || (nmaps > 1 && w_stride < N))
    return set_error(DSHT_ERR_INVALID, "invalid maps (nmaps=%d, w_stride=%lld)", nmaps, (long long)w_stride);
  if (N > (int64_t)0xfffffff0LL) return set_error(DSHT_ERR_INVALID, "too many points (%lld)", (long long)N);
  if (N == 0 && mode == DSHT_MODE_BASIC)
    return set_error(DSHT_ERR_EMPTY, "The theta array seems to be empty!");
  const bool maps = nmaps > 1;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  std::unique_lock<std::mutex> lock(p->mu, std::defer_lock);
  const int piece_max = default_piece_max(p->g, N);
  const size_t need = workspace_layout(p->g, N, piece_max, nullptr, nullptr, maps);
  uint8_t* base = reinterpret_cast<uint8_t*>(workspace);
  if (base) {
    if (workspace_bytes < need)
      return set_error(DSHT_ERR_NOMEM, "workspace of %zu bytes is smaller than the %zu needed", workspace_bytes, need);
  } else {
    lock.lock();
    int rc = ensure_plan_workspace(p, need);
    if (rc) return rc;
    base = reinterpret_cast<uint8_t*>(p->ws);
  }
  if (N == 0) {  // __call__ on no points returns zeros (sht/sht.py:127,150)
    DSHT_CUDA_OK(cudaMemsetAsync(alm, 0, sizeof(double) * 2 * p->g.Nlm * nmaps, s));
    return DSHT_OK;
  }
  Workspace ws;
  workspace_layout(p->g, N, piece_max, base, &ws, maps);
  int rc = maps || w_dtype == DSHT_W_F32
               ? run_maps(p, theta, phi, w, w_dtype == DSHT_W_F32, N, nmaps, w_stride, mode, alm, ws, s)
               : run_pipeline(p, theta, phi, static_cast<const double*>(w), N, mode, alm, ws, s);
  if (rc) return rc;
  unsigned hf = 0;
  DSHT_CUDA_OK(cudaMemcpyAsync(&hf, ws.flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  DSHT_CUDA_OK(cudaStreamSynchronize(s));
  collect_profile(p);
  return flags_to_status(hf, mode);
}

int dsht_execute(dsht_plan_t p, const double* theta, const double* phi, const double* w, int64_t N, int mode,
                 double* alm, void* workspace, size_t workspace_bytes, void* stream) {
  return execute_device(p, theta, phi, w, DSHT_W_F64, N, 1, N, mode, alm, workspace, workspace_bytes, stream);
}

int dsht_workspace_size_maps(dsht_plan_t p, int64_t N, int nmaps, size_t* bytes) {
  if (!p || !bytes || N < 0 || nmaps < 1) return set_error(DSHT_ERR_INVALID, "invalid arguments");
  *bytes = workspace_layout(p->g, N, default_piece_max(p->g, N), nullptr, nullptr, nmaps > 1);
  return DSHT_OK;
}

int dsht_execute_maps(dsht_plan_t p, const double* theta, const double* phi, const void* w, int w_dtype, int64_t N,
                      int nmaps, int64_t w_stride, int mode, double* alm, void* workspace, size_t workspace_bytes,
                      void* stream) {
  return execute_device(p, theta, phi, w, w_dtype, N, nmaps, w_stride, mode, alm, workspace, workspace_bytes,
                        stream);
}

int dsht_execute_host(dsht_plan_t p, const double* theta, const double* phi, const double* w, int64_t N, int mode,
                      double* alm_host) {
  if (!p || !alm_host || N < 0 || (N > 0 && (!theta || !phi || !w)))
    return set_error(DSHT_ERR_INVALID, "invalid arguments");
  if (N == 0 && mode == DSHT_MODE_BASIC) return set_error(DSHT_ERR_EMPTY, "The theta array seems to be empty!");
  std::lock_guard<std::mutex> lock(p->mu);
  const int piece_max = default_piece_max(p->g, N);
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

int dsht_get_row(dsht_plan_t p, int which, int ell, int m, double* out) {
  if (!p || !out || which < 0 || which > 1 || m < 0 || ell < m || ell >= p->g.Nl)
    return set_error(DSHT_ERR_INVALID, "invalid row (which=%d, l=%d, m=%d)", which, ell, m);
  const double* t = which == 0 ? p->Yv : p->Yd;
  DSHT_CUDA_OK(cudaMemcpy(out, t + hp_index(ell, m, p->g.Nl) * p->g.Nx, sizeof(double) * p->g.Nx,
                          cudaMemcpyDeviceToHost));
  return DSHT_OK;
}

int dsht_get_table(dsht_plan_t p, int which, double* out) {
  if (!p || !out || which < 0 || which > 1) return set_error(DSHT_ERR_INVALID, "invalid arguments");
  const double* t = which == 0 ? p->Yv : p->Yd;
  DSHT_CUDA_OK(cudaMemcpy(out, t, sizeof(double) * p->g.Nlm * p->g.Nx, cudaMemcpyDeviceToHost));
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
