// pz_internal.h -- host-side state shared by the runtime translation units.
#pragma once
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/phantom_zone_b200.h"
#include "pz_kernels.cuh"

struct pz_ctx {
  int param_id = 0, device = 0;
  pz_params P{};
  pz::u32 logn = 0;
  pz::u64 root = 0;
  cudaStream_t stream = nullptr;
  // device tables
  pz::u64 *d_tw = nullptr;        // fw | fws | iw | iws  (4N words)
  unsigned short *d_dlog = nullptr;
  pz::u64 *d_tv = nullptr;        // 6 x br_q/2
  // constants
  pz::RingConsts rc{};
  // device key form: conv_c scales the transformed rows of the keys that the
  // Montgomery products use (aggregation, the NI key switch), br_conv_c those
  // of the blind rotation's RGSW and auto keys (folded products for N = 2048)
  pz::u64 conv_c = 0, conv_cs = 0, br_conv_c = 0, br_conv_cs = 0;
  pz::u64 ni_conv_c = 0, ni_conv_cs = 0;  // the NI key-switch keys (ni_mac: folded when MAC_FOLD_N2048)
  pz::BrParams br{};
  pz::KsParams ks{};
  pz::u32 *d_err = nullptr;  // device error word: DEVERR_* bits set by kernels whose bounded waits ran out
  int grid_limit = 0;
  int pbs_variant = 0;  // blind-rotation launch shape (see pz::PBS_VARIANTS)
  int split_below = -1;  // batches of at most this many gates use the two-CTA kernel (-1: half the SMs)
  int ks_ct = 64;        // key-switch tile: 8, 16, 32 ciphertexts per CTA, 64 = tensor cores (default)
  // autotuned launch shapes per batch-size bucket floor(log2(gates)); a
  // bucket the autotuner has not seen uses the defaults above
  struct Tuned {
    int variant = -1, ks_ct = 0;
  };
  Tuned tuned[48];
  // host-API scratch (guarded by mu)
  std::mutex mu;
  size_t cap = 0;
  pz::u64 *d_c0 = nullptr, *d_c1 = nullptr, *d_out = nullptr;
  unsigned char *d_gates = nullptr;
  pz::u32 *d_ks = nullptr;
  std::string err;
};

struct pz_key {
  pz_ctx *ctx = nullptr;
  pz::u64 *d_rgsw = nullptr, *d_autos = nullptr;
  pz::u32 *d_ksk = nullptr;
  unsigned char *d_ksk8 = nullptr;  // the KSK as byte planes (tensor-core key switch), or null
  size_t bytes = 0;
};

struct pz_ni_ksk {
  pz_ctx *ctx = nullptr;
  pz::u64 *d_ksk = nullptr;  // [2 d][N] evaluation domain, scaled by ni_conv_c (N^{-1})
  pz::u32 d = 0;
  size_t bytes = 0;
};

namespace pz {
// Build k->d_ksk8 from k->d_ksk (when the parameter set's digits fit s8 and
// the rows come in whole 32-row blocks; otherwise, or when the device is out
// of memory, the key keeps the IMAD key-switch kernels only).
void build_ksk8(pz_ctx *c, pz_key *k, cudaStream_t s);
void free_key_arrays(pz_key *k);
// KsParams of context c bound to key k (both KSK forms)
void ks_bind_key(const pz_ctx *c, const pz_key *k, KsParams &ks);
// floor(log2(n)), clamped to the 48 buckets of pz_ctx::tuned
inline int size_bucket(size_t n) {
  const int b = n ? 63 - __builtin_clzll((unsigned long long)n) : 0;
  return b < 47 ? b : 47;
}
int effective_variant(pz_ctx *c, size_t count);
int effective_ks_ct(const pz_ctx *c, size_t count);
// Launch sequence of one batch of gate bootstraps (ks kernel -> pbs kernel).
// Optional wire gather/scatter: in0/in1/out_idx (see KsParams, BrParams).
pz_status run_gates(pz_ctx *c, const pz_key *k, const unsigned char *d_gates, const u64 *d_c0, const u64 *d_c1,
                    u64 *d_out, size_t count, u32 *d_ks_out, u64 *d_rlwe, cudaStream_t s, u32 *d_ks_scratch,
                    bool raw, const u32 *in0 = nullptr, const u32 *in1 = nullptr, const u32 *out_idx = nullptr);
pz_status fail(pz_ctx *ctx, pz_status s, const std::string &msg);
// forget the no-alloc scratch address cached for a device (pz_noalloc.cu)
void noalloc_forget_device(int device);
pz_status cuda_fail(pz_ctx *ctx, const char *what, cudaError_t e);
u32 ks_stride(const pz_params &P);
// DefaultDecomposer parameters for (q, logb, d) (decomposer.rs:158-178)
Decomp decomposer(u64 q, u32 logb, u32 d);

// RandomFillUniformInModulus (random.rs:93-110) over the ChaCha8 stream of
// `seed`, on the device: `total` samples uniform in [0, q), sample k stored at
// dst[(k / row_len) * row_stride + row_off + k % row_len].  Synchronous.
pz_status seeded_fill_u64(pz_ctx *c, const uint8_t seed[32], u64 q, u64 total, u64 row_len, u64 row_stride,
                          u64 row_off, u64 *dst, cudaStream_t st);
pz_status seeded_fill_u32(pz_ctx *c, const uint8_t seed[32], u64 q, u64 total, u64 row_len, u64 row_stride,
                          u64 row_off, u32 *dst, cudaStream_t st);
// `streams` streams at once (seeds[i] -> dst + i * stream_stride, `total`
// samples each, contiguous).  Synchronous.
pz_status seeded_fill_batch_u64(pz_ctx *c, const uint8_t (*seeds)[32], size_t streams, u64 q, u64 total, u64 *dst,
                                u64 stream_stride, cudaStream_t st);

// puncture_p_rng over ChaCha8(seed): the `times`-th 32-byte fill (host)
void crs_puncture(const uint8_t seed[32], size_t times, uint8_t out[32]);
// out[i] = sum_t d_src[t][i] mod q over k device rows of len words (canonical inputs)
cudaError_t launch_sum_mod(const u64 *const *d_src, u32 k, size_t len, u64 q, u64 *out, cudaStream_t st);

// Compiled (levelized) form of a circuit, read by the multi-session executor.
// Wire slots: inputs first (input order), then gate outputs; bit 31 = not().
struct CircuitView {
  size_t n_inputs = 0, n_gates = 0, n_outputs = 0, levels = 0;
  const size_t *level_off = nullptr;  // level l (1..levels) = gates [off[l-1], off[l])
  const unsigned char *type = nullptr;
  const u32 *in0 = nullptr, *in1 = nullptr, *out = nullptr, *outref = nullptr;
};
bool circuit_view(pz_circuit *c, CircuitView *v);
// out[i] = wires[refs[i]] (q - x when bit 31 of refs[i] is set), L words each
cudaError_t launch_gather(const u64 *wires, const u32 *refs, u64 *out, size_t count, size_t L, u64 q,
                          cudaStream_t s);
}  // namespace pz

#define PZ_CK(ctx, call)                                          \
  do {                                                            \
    cudaError_t _e = (call);                                      \
    if (_e != cudaSuccess) return pz::cuda_fail((ctx), #call, _e); \
  } while (0)
