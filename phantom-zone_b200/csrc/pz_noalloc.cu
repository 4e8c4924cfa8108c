// pz_noalloc.cu -- batched gates for callers that cannot allocate device memory.
//
// pz_gate_batch_device needs a scratch buffer between its two kernels (the
// key-switched LWE of every gate, written by the key-switch kernel and read by
// the blind-rotation kernel) and obtains it with cudaMallocAsync.  Some hosts
// cannot do that on their gate path: a process whose device memory is fully
// reserved up front by another allocator (a framework's caching pool or a
// fixed per-session budget), or a latency-critical serving thread that must
// not issue allocating CUDA calls.  pz_gate_batch_device_noalloc runs the same
// two kernels with the scratch in a fixed array compiled into this library,
// so it calls no cudaMalloc, cudaFree or other allocating routine.
//
// The array lives in device memory of every GPU that loads the library until
// the process exits.  Its size caps the batch: PZ_NOALLOC_KS_WORDS 32-bit
// words, i.e. floor(PZ_NOALLOC_KS_WORDS / stride) gates per call where stride
// is n + 1 rounded up to 32 (4096 gates for NonInteractiveLTE8Party).  All
// calls share the array and it keeps the last call's contents; nothing needs
// clearing because each call writes every word it later reads.  Calls whose
// work overlaps on the GPU (different streams, or different contexts on the
// same device) race on the array; the caller must serialize them.
#include <mutex>

#include "pz_internal.h"

static __device__ __align__(256) pz::u32 g_noalloc_ks[PZ_NOALLOC_KS_WORDS];

namespace {
constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
pz::u32 *g_addr[MAX_DEVICES] = {};
}  // namespace

namespace pz {
// Drop the cached device address of the array on `device`; the next
// no-alloc call there looks it up again.  Called whenever a context is
// created: a cudaDeviceReset destroys every device object of this library
// (contexts and keys included), and a context created afterwards must not
// reuse an address resolved in the old CUDA context.
void noalloc_forget_device(int device) {
  if (device < 0 || device >= MAX_DEVICES) return;
  std::lock_guard<std::mutex> lock(g_mu);
  g_addr[device] = nullptr;
}
}  // namespace pz

extern "C" pz_status pz_gate_batch_device_noalloc(pz_ctx *c, const pz_key *k, const uint8_t *d_gates,
                                                  const uint64_t *d_c0, const uint64_t *d_c1, uint64_t *d_out,
                                                  size_t count, void *stream) {
  if (!c) return PZ_ERR_INVALID_ARGUMENT;
  if (count == 0) return PZ_OK;
  if (!d_gates || !d_c0 || !d_c1 || !d_out) return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "NULL device buffer");
  if (!k || k->ctx != c) return pz::fail(c, PZ_ERR_KEY_MISMATCH, "key does not belong to this context");
  const size_t stride = pz::ks_stride(c->P);
  const size_t max_count = (size_t)PZ_NOALLOC_KS_WORDS / stride;
  if (count > max_count)
    return pz::fail(c, PZ_ERR_INVALID_ARGUMENT,
                    "pz_gate_batch_device_noalloc: " + std::to_string(count) +
                        " gates exceed the fixed scratch of this parameter set (at most " +
                        std::to_string(max_count) + " gates per call); split the batch");
  if (c->device < 0 || c->device >= MAX_DEVICES) return pz::fail(c, PZ_ERR_NOT_SUPPORTED, "device id out of range");
  PZ_CK(c, cudaSetDevice(c->device));
  pz::u32 *scratch = nullptr;
  {
    // First call on a device (since the last context creation there):
    // resolve the array's device address with that device current (the
    // host-side symbol is not a device address).
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[c->device]) {
      void *p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_ks);
      if (e != cudaSuccess) return pz::cuda_fail(c, "cudaGetSymbolAddress(g_noalloc_ks)", e);
      g_addr[c->device] = (pz::u32 *)p;
    }
    scratch = g_addr[c->device];
  }
  return pz::run_gates(c, k, d_gates, d_c0, d_c1, d_out, count, nullptr, nullptr, (cudaStream_t)stream, scratch,
                       false);
}
