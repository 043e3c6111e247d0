// dsht_execute_noalloc: the forward transform with its scratch in a fixed device array.
//
// Some callers cannot allocate device memory at the moment they want a transform: a host
// framework that has reserved nearly all of the GPU's memory for its own pool (and would
// make a cudaMalloc from a library fail or fragment that pool), a plugin host that forbids
// its plugins to allocate device memory on their own, or a latency-critical loop where the
// implicit device-wide synchronisation of cudaMalloc/cudaFree would stall other streams.
// This entry point lets them run the same pipeline as dsht_execute without allocating:
// every intermediate buffer (keys, sorted payload, piece list, per-piece bin sums, folded
// node sums, the two partial alm vectors, flags) is carved out of g_noalloc_scratch, a
// file-scope __device__ array of kNoAllocScratchBytes (64 MiB) that every GPU which loads
// this library holds until the process exits.  Problems whose workspace does not fit are
// rejected with DSHT_ERR_NOMEM before anything is launched.
//
// The array's name in host code is only a host-side stand-in for the device symbol, not a
// device address, so it is never handed to a kernel: the device address is looked up once
// per device with cudaGetSymbolAddress, with that device current, on the first call made
// on that device, and cached.  Every call waits for its stream at the end to read the error
// flags, so no call can be captured into a CUDA graph.  All calls share the one array and it keeps the last call's contents; the
// pipeline clears what must start at zero (the bin counts and the error flags) and
// overwrites everything else it reads, so stale contents never leak into a result.  Calls
// whose kernels overlap on the GPU (on different streams or host threads) race on the
// array and must be serialised by the caller.
#include <mutex>

#include "dsht_internal.cuh"

namespace dsht {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once per device).
int noalloc_scratch(void** out) {
  int dev = 0;
  DSHT_CUDA_OK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return set_error(DSHT_ERR_INVALID, "device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    DSHT_CUDA_OK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return DSHT_OK;
}

}  // namespace
}  // namespace dsht

using namespace dsht;

extern "C" {

size_t dsht_noalloc_scratch_bytes(void) { return kNoAllocScratchBytes; }

int dsht_execute_noalloc(dsht_plan_t p, const double* theta, const double* phi, const double* w, int64_t N,
                         int mode, double* alm, void* stream) {
  if (!p || !alm || N < 0 || (N > 0 && (!theta || !phi || !w)))
    return set_error(DSHT_ERR_INVALID, "invalid arguments");
  if (mode != DSHT_MODE_CALL && mode != DSHT_MODE_BASIC) return set_error(DSHT_ERR_INVALID, "bad mode %d", mode);
  if (N > (int64_t)0xfffffff0LL) return set_error(DSHT_ERR_INVALID, "too many points (%lld)", (long long)N);
  if (N == 0 && mode == DSHT_MODE_BASIC) return set_error(DSHT_ERR_EMPTY, "The theta array seems to be empty!");
  const int piece_max = plan_piece_max(p, N);
  const size_t need = workspace_layout(p->g, N, piece_max, nullptr, nullptr);
  if (need > kNoAllocScratchBytes)
    return set_error(DSHT_ERR_NOMEM,
                     "dsht_execute_noalloc: Nl=%d, Nx=%d, N=%lld needs %zu bytes of scratch, more than the fixed "
                     "%zu; use dsht_execute with a workspace instead",
                     p->g.Nl, p->g.Nx, (long long)N, need, kNoAllocScratchBytes);
  void* base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (N == 0) {
    DSHT_CUDA_OK(cudaMemsetAsync(alm, 0, sizeof(double) * 2 * p->g.Nlm, s));
    return DSHT_OK;
  }
  Workspace ws;
  workspace_layout(p->g, N, piece_max, reinterpret_cast<uint8_t*>(base), &ws);
  rc = run_pipeline(p, theta, phi, w, N, mode, alm, ws, s);
  if (rc) return rc;
  unsigned hf = 0;
  DSHT_CUDA_OK(cudaMemcpyAsync(&hf, ws.flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  DSHT_CUDA_OK(cudaStreamSynchronize(s));
  collect_profile(p);
  return flags_to_status(hf, mode);
}

}  // extern "C"
