// pz_kernels.cuh -- parameter blocks shared by the kernels and the host runtime.
#pragma once
#include "pz_device.cuh"

namespace pz {

constexpr int MAX_KS_D = 16;   // key-switch decomposition count bound
// Revision of the blind-rotation kernels: bumped with every change to their
// code, so that a profile taken on one revision is not reported for another.
constexpr const char *BR_KERNEL_REVISION = "br-v15";
constexpr int MAX_AUTO_SLOTS = 16;

// Everything the blind rotation needs for one parameter set + server key.
struct BrParams {
  RingConsts rc;
  Decomp da, db, dauto;
  u32 d_a, d_b, d_auto;
  u32 rgsw_rows, auto_rows;
  u32 n, br_q, w, g, emb;
  u32 ks_mask;                     // q_ks - 1: key-switched words are read modulo q_ks
  double q_ks_f, br_q_f;           // mod_switch_odd operands (pbs.rs:416-420)
  u32 auto_k[MAX_AUTO_SLOTS];      // automorphism element mod 2N per key slot
  const unsigned short *dlog;      // [br_q]
  const u64 *tv;                   // [6][br_q/2] test vectors
  const u64 *rgsw;                 // [n][rgsw_rows][N] device layout, scaled by the key form
  const u64 *autos;                // [w+1][auto_rows][N]
  const u32 *out_idx;              // optional scatter: output of gate ct -> LWE out_idx[ct]
  u32 *err;                        // the context's device error word (DEVERR_* bits)
};

// Gate prelude + mod-down + LWE key switch.
struct KsParams {
  u64 Q, qby4;
  u32 mask;                 // q_ks - 1
  double q_ks_f, Q_f;       // pbs.rs:128-132 operands
  Decomp dks;
  u32 d, n, N;
  u32 ksk_stride;           // u32 words per KSK row (>= n+1)
  u32 out_stride;           // u32 words per output LWE (>= n+1)
  u32 raw;                  // inputs are combined LWEs: skip the gate prelude
  const u32 *ksk;           // [d N][ksk_stride]
  // The same KSK as byte planes for the tensor-core key switch (null: not
  // built): plane p holds bits 8p..8p+7 of every entry, in blocks of 32 rows
  // ([planes][d N / 32][ksk8_cols][32], rows permuted inside a block so that
  // one 8-byte load gives a thread its mma fragment; ksk8_cols = n + 1
  // rounded up to KSM_COLS, zero-padded).
  const unsigned char *ksk8;
  u32 planes, ksk8_cols;
  // Optional gather (circuit wires): input i of gate ct is LWE
  // c{i}[in{i}[ct] & WIRE_MASK], negated (q - x) when bit 31 is set.
  const u32 *in0, *in1;
};

// One CTA of the ragged key switch: `count` (<= 16) consecutive items of
// one session descriptor, starting at item `first`.
struct KsTile {
  u32 desc, first, count;
};
constexpr int KS_TILE_CT = 16;

constexpr u32 WIRE_NEG = 0x80000000u;
constexpr u32 WIRE_MASK = 0x7fffffffu;

// Gate codes 0..5 (and, nand, or, nor, xor, xnor).  GATE_RAW marks an input
// that is already the combined LWE (no prelude); the low bits then select
// the test vector.
constexpr unsigned char GATE_RAW = 0x80;

cudaError_t launch_key_convert(int logn, const u64 *in, u64 *out, size_t npolys, const RingConsts &rc,
                               u64 c, u64 cs, cudaStream_t s);
// err: the context's device error word (DEVERR_* bits)
cudaError_t launch_ntt_fwd(int logn, u64 *polys, size_t count, const RingConsts &rc, u32 *err, cudaStream_t s);
cudaError_t launch_ntt_inv(int logn, u64 *polys, size_t count, const RingConsts &rc, u32 *err, cudaStream_t s);
// variant: register cap of the one-digit forms as the blind rotation's
// launch shapes 0 / 1 / 2 (2 / 3 / 4 CTAs per SM; other values: 3)
cudaError_t launch_ext_product(int logn, bool d1, const BrParams &P, u64 *rlwe, const u32 *idx,
                               size_t count, int trivial, cudaStream_t s, int variant = 1);
cudaError_t launch_auto(int logn, bool d1, const BrParams &P, u64 *rlwe, const u32 *slot, size_t count,
                        int trivial, cudaStream_t s, int variant = 1);
// reduce_output: leave every output word reduced mod q_ks (otherwise the
// words may carry multiples of q_ks, and consumers mask with q_ks - 1)
// ct: ciphertexts per CTA (8, 16 or 32)
// Tensor-core key switch: KSM_ROWS ciphertexts x KSM_COLS output columns
// per CTA; launch_ks takes ct = KS_CT_MMA for it.
constexpr int KSM_ROWS = 64, KSM_COLS = 224, KS_CT_MMA = 64;
inline u32 ksk8_cols(u32 n) { return (n + 1 + KSM_COLS - 1) / KSM_COLS * KSM_COLS; }
inline u32 ksk8_planes(u32 mask) {  // bytes of q_ks - 1
  u32 bits = 0;
  while (bits < 32 && (mask >> bits)) bits++;
  return (bits + 7) / 8;
}
// KSK rows (u32, stride ksk_stride, d N rows, n + 1 used columns) -> byte planes
cudaError_t launch_ksk_planes(const u32 *ksk, u32 rows, u32 stride, u32 n, u32 planes, unsigned char *out,
                              cudaStream_t s);
cudaError_t launch_ks(const KsParams &P, const unsigned char *gates, const u64 *c0, const u64 *c1,
                      size_t count, u32 *out, cudaStream_t s, bool reduce_output, int ct = KS_TILE_CT);
cudaError_t launch_pbs(int logn, bool d1, const BrParams &P, const u32 *ks, u32 ks_stride,
                       const unsigned char *gates, u64 *out, size_t count, u64 *rlwe_dbg,
                       int grid_limit, cudaStream_t s, int variant);
// launch-shape variants of the production blind rotation (registers per
// thread capped for 2, 3 or 4 CTAs of 256 threads per SM)
constexpr int PBS_VARIANTS = 3;
// launch shape for small batches (N = 2048, one-digit sets): one ciphertext
// per cluster of two CTAs, a on one SM and b on the other (lower latency)
constexpr int PBS_SPLIT = 3;
// launch shape with every operation's key rows streamed into a shared-memory
// stage by bulk copies (N = 2048, one-digit sets; two CTAs per SM)
constexpr int PBS_BULK = 4;
constexpr int PBS_MAX_VARIANT = PBS_BULK;
// Ragged batches (several sessions / parameter sets in one launch): per-item
// descriptors in device memory; max_* bound the sizes over the descriptors.
cudaError_t launch_ks_ragged(const KsParams *d_descs, const KsTile *d_tiles, size_t ntiles, size_t count,
                             u32 max_n, u32 max_N, u32 max_d, const unsigned char *gates, const u64 *wires,
                             const u32 *in0, const u32 *in1, u32 *out, u32 out_stride, cudaStream_t s);
// The ragged key switch on the tensor cores: tiles of up to KSM_ROWS items,
// every session's key with its byte planes (KsParams::ksk8), d <= 16.
cudaError_t launch_ks_mma_ragged(const KsParams *d_descs, const KsTile *d_tiles, size_t ntiles, size_t count,
                                 u32 max_n, u32 max_N, u32 max_d, const unsigned char *gates, const u64 *wires,
                                 const u32 *in0, const u32 *in1, u32 *out, u32 out_stride, cudaStream_t s);
cudaError_t launch_pbs_ragged(int logn, bool d1, const BrParams *d_descs, const u32 *item_desc, u32 max_br_q,
                              u32 max_n, const u32 *ks, u32 ks_stride, const unsigned char *gates, u64 *out,
                              const u32 *out_idx, size_t count, int grid_limit, cudaStream_t s, int variant);
cudaError_t launch_not(const u64 *in, u64 *out, size_t words, u64 q, cudaStream_t s);
cudaError_t launch_imad_probe(int blocks, int threads, u32 iters, u32 *sink, cudaStream_t s);
cudaError_t launch_pipe_probe(int kind, int blocks, int threads, u32 iters, u32 *sink, cudaStream_t s);
// per launch: blocks * threads * iters * 16 * 8 multiply-adds
size_t pbs_smem_bytes(int logn, u32 br_q, u32 n);
// blind-rotation items resident at once for a launch shape (whole-wave size)
cudaError_t pbs_slots(int logn, bool d1, u32 br_q, u32 n, int variant, size_t *slots);

}  // namespace pz
