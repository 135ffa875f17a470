// fss_static.cu -- fss_align_static: the fused alignment with library-owned scratch.
//
// Some callers cannot allocate device memory at the point where they align: code running
// inside another framework's memory pool that has reserved the whole device, host runtimes
// (FFI / JNI / cgo embeddings) that hand over only input and output buffers, and latency-
// critical request loops where cudaMalloc's implicit synchronisation would stall other
// streams.  fss_align needs scratch beyond its inputs and outputs -- the per-(pair, start)
// best rows that the pick step reduces, and the work counter / status words of the
// persistent grid -- and takes it from the caller.  This entry point takes it instead from
// one file-scope __device__ array of fixed size, so a call allocates nothing.
//
// The array exists once per device that loads the library and lives until process exit.
// Every call shares it: calls whose work overlaps on the GPU (different streams, or
// different host threads without ordering) race on it and must be serialised by the caller.
#include <cuda.h>  // driver types only; the two driver calls are looked up at run time

#include <mutex>
#include <string>

#include "fss_internal.cuh"

namespace fss {
namespace {

constexpr size_t kStaticRows = FSS_STATIC_MAX_ROWS;
constexpr size_t kHeaderBytes = 256;  // work counter + status words, padded
constexpr size_t kStaticBytes = kHeaderBytes + kStaticRows * (1 + 4 + 3) * sizeof(float);

// Host code must never use this symbol as a pointer: the name denotes a host-side stand-in.
// Its device address is looked up per device with cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_align_scratch[kStaticBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
// Per device: the address of g_align_scratch in the context it was resolved in.  A
// cudaDeviceReset destroys that context (and the module with the array); the next call
// then finds another context id and resolves the address again.
struct Slot {
  unsigned long long ctx_id;
  void* addr;
};
Slot g_slot[kMaxDevices] = {};

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;

// Unique id of the context current on this thread (0: none current, or no driver support).
unsigned long long current_context_id() {
  if (!g_ctx_current || !g_ctx_id) {
    cudaDriverEntryPointQueryResult q1, q2;
    void *f1 = nullptr, *f2 = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &q1) !=
            cudaSuccess || q1 != cudaDriverEntryPointSuccess ||
        cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2) !=
            cudaSuccess || q2 != cudaDriverEntryPointSuccess)
      return 0;
    g_ctx_current = reinterpret_cast<CtxGetCurrentFn>(f1);
    g_ctx_id = reinterpret_cast<CtxGetIdFn>(f2);
  }
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (g_ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  if (g_ctx_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

int scratch_address(void** out) {
  int dev = 0;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess)
    return set_error(FSS_ERR_CUDA, std::string("fss_align_static: cudaGetDevice: ") +
                                       cudaGetErrorString(ce));
  if (dev < 0 || dev >= kMaxDevices)
    return set_error(FSS_ERR_UNSUPPORTED, "fss_align_static: device ordinal above 63");
  std::lock_guard<std::mutex> lock(g_mu);
  Slot& slot = g_slot[dev];
  const unsigned long long ctx = current_context_id();
  if (!slot.addr || ctx == 0 || ctx != slot.ctx_id) {
    // first call on this device (or in a new context of it), with the device current:
    // resolve the array's device address
    void* p = nullptr;
    ce = cudaGetSymbolAddress(&p, g_align_scratch);
    if (ce != cudaSuccess || !p)
      return set_error(FSS_ERR_CUDA, std::string("fss_align_static: cudaGetSymbolAddress: ") +
                                         cudaGetErrorString(ce));
    slot.addr = p;
    slot.ctx_id = current_context_id();  // the lookup above made the context current
  }
  *out = slot.addr;
  return FSS_OK;
}

}  // namespace

int align_static_launch(const fss_align_desc* d, cudaStream_t st) {
  if (!d) return set_error(FSS_ERR_INVALID, "fss_align_static: null descriptor");
  if (!d->out_score || !d->out_q || !d->out_t)
    return set_error(FSS_ERR_INVALID, "fss_align_static: out_score, out_q and out_t are required");
  if (d->n_pairs < 0 || d->n_starts <= 0)
    return set_error(FSS_ERR_INVALID, "fss_align_static: needs n_pairs >= 0 and n_starts > 0");
  const long long rows = (long long)d->n_pairs * (long long)d->n_starts;
  if (rows > (long long)kStaticRows)
    return set_error(FSS_ERR_UNSUPPORTED,
                     "fss_align_static: n_pairs * n_starts = " + std::to_string(rows) +
                         " exceeds the static scratch of FSS_STATIC_MAX_ROWS = " +
                         std::to_string(kStaticRows) + " rows; split the batch or use fss_align");
  void* base = nullptr;
  int rc = scratch_address(&base);
  if (rc != FSS_OK) return rc;
  fss_align_desc local = *d;
  unsigned char* b = static_cast<unsigned char*>(base);
  local.scratch = reinterpret_cast<int32_t*>(b);  // zeroed on `st` by the launch itself
  local.row_score = reinterpret_cast<float*>(b + kHeaderBytes);
  local.row_q = local.row_score + kStaticRows;
  local.row_t = local.row_q + 4 * kStaticRows;
  // rows keep the previous call's contents: set this call's scores to NaN first, so a pair
  // the kernel skips (larger than the declared max_* extents) comes back as NaN, not stale
  if (rows > 0) {
    cudaError_t ce = cudaMemsetAsync(local.row_score, 0xFF, (size_t)rows * sizeof(float), st);
    if (ce != cudaSuccess)
      return set_error(FSS_ERR_CUDA, std::string("fss_align_static: row reset: ") +
                                         cudaGetErrorString(ce));
  }
  rc = align_launch(&local, st);
  if (rc != FSS_OK) return rc;
  // the caller's optional status word (device int32) receives this call's flags, ordered
  // after the launch on `st` (bit 0: a pair larger than the declared max_* extents)
  if (d->scratch) {
    cudaError_t ce = cudaMemcpyAsync(d->scratch, local.scratch + 1, sizeof(int32_t),
                                     cudaMemcpyDeviceToDevice, st);
    if (ce != cudaSuccess)
      return set_error(FSS_ERR_CUDA, std::string("fss_align_static: status copy: ") +
                                         cudaGetErrorString(ce));
  }
  return FSS_OK;
}

}  // namespace fss
