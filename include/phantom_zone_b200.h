/*
 * phantom_zone_b200.h -- C ABI of the B200 gate-bootstrap engine.
 *
 * This is the drop-in boundary for phantom-zone's server-side gate
 * evaluation: a Rust `BooleanGates` implementation (or any other FFI host)
 * calls these entry points instead of running `pbs()` on the CPU.  Plain
 * pointers and sizes only; every call returns a pz_status (no panics or
 * exceptions cross the boundary); pz_last_error() describes the last failure
 * of a context.
 *
 * Data formats (all little-endian u64 words, as in the reference):
 *   LWE ciphertext mod Q       [N + 1]      b, a_1 .. a_N      (pbs.rs:423-449)
 *   RLWE ciphertext            [2][N]       a(X), b(X)         (runtime.rs:137-153)
 *   server key, coefficient domain (pz_server_key_view below)
 *
 * Reference interfaces replaced (paths inside gausslabs/phantom-zone):
 *   pz_param_get          bool/parameters.rs:526-726 (parameter constants)
 *   pz_ctx_create         BoolEvaluator::new, bool/evaluator.rs:651-784;
 *                         set_parameter_set, bool/mp_api.rs:35-47,
 *                         bool/ni_mp_api.rs:39-57
 *   pz_key_upload         set_server_key, bool/mp_api.rs:136-145 and
 *                         bool/ni_mp_api.rs:119-132 (ServerKeyEvaluationDomain
 *                         ::from + Shoup*ServerKeyEvaluationDomain::from,
 *                         bool/keys.rs:687-781, 869-1004, 1088-1220)
 *   pz_gate_batch*        BooleanGates::{and,nand,or,nor,xor,xnor}_inplace,
 *                         bool/mod.rs:22-71 -> evaluator.rs:2163-2245 -> pbs()
 *                         pbs.rs:104-233 (batched: many gates per call)
 *   pz_not_batch_device   BooleanGates::not_inplace, evaluator.rs:2247-2250
 *   pz_pbs_batch_device   pbs(), pbs.rs:104-233, on already-combined LWEs
 *   pz_ntt_*_device       Ntt::forward / Ntt::backward, ntt.rs:396-442
 *   pz_rlwe_by_rgsw_device rlwe_by_rgsw_shoup, rgsw/runtime.rs:754-855
 *   pz_rlwe_auto_device   rlwe_auto_shoup, rgsw/runtime.rs:530-643
 *   pz_lwe_key_switch_device lwe_key_switch, lwe.rs:14-44
 */
#ifndef PHANTOM_ZONE_B200_H
#define PHANTOM_ZONE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pz_status {
  PZ_OK = 0,
  PZ_ERR_INVALID_ARGUMENT = 1,
  PZ_ERR_CUDA = 2,
  PZ_ERR_OUT_OF_MEMORY = 3,
  PZ_ERR_NOT_SUPPORTED = 4,
  PZ_ERR_KEY_MISMATCH = 5
} pz_status;

/* Parameter sets, in the order of bool/parameters.rs:526-726. */
enum {
  PZ_I_2P_LB_SR = 0,   /* InteractiveLTE2Party */
  PZ_I_4P = 1,         /* InteractiveLTE4Party */
  PZ_I_8P = 2,         /* InteractiveLTE8Party */
  PZ_NI_2P = 3,        /* NonInteractiveLTE2Party */
  PZ_NI_4P_HB_FR = 4,  /* NonInteractiveLTE4Party */
  PZ_NI_4P_LB_SR = 5,
  PZ_NI_8P = 6,        /* NonInteractiveLTE8Party */
  PZ_SP_TEST = 7,      /* SP_TEST_BOOL_PARAMS (reference test set, N = 512) */
  PZ_NUM_PARAMS = 8
};

/* Gate codes of the batched gate entry points. */
enum { PZ_GATE_AND = 0, PZ_GATE_NAND = 1, PZ_GATE_OR = 2, PZ_GATE_NOR = 3,
       PZ_GATE_XOR = 4, PZ_GATE_XNOR = 5 };

typedef struct pz_params {
  uint64_t rlwe_q;   /* Q */
  uint64_t lwe_q;    /* q_ks (power of two) */
  uint32_t br_q;     /* blind-rotation modulus */
  uint32_t rlwe_n;   /* N */
  uint32_t lwe_n;    /* n */
  uint32_t lwe_logb, lwe_d;
  uint32_t rlrg_logb, rlrg_d_a, rlrg_d_b;
  uint32_t auto_logb, auto_d;
  uint32_t g, w;
  uint32_t lwe_secret_gaussian;
  uint32_t variant;          /* 0 single party, 1 interactive, 2 non-interactive */
  uint32_t embedding_factor; /* 2N / br_q */
  uint32_t rgsw_rows;        /* 2 d_a + 2 d_b */
  uint32_t auto_rows;        /* 2 d_auto */
  uint32_t n_auto_keys;      /* w + 1 */
  uint32_t ni_ks_logb, ni_ks_d; /* ui_to_s key switch decomposition of the NI sets
                                   (parameters.rs:616-697: 1, 50); 0 otherwise */
  uint32_t rgrg_logb, rgrg_d_a, rgrg_d_b; /* RGSW x RGSW decomposition of key aggregation
                                             (rgrg_decomposer_params); 0 when the set has none */
} pz_params;

typedef struct pz_ctx pz_ctx;
typedef struct pz_key pz_key;

/* Expanded server key in the coefficient domain, host memory:
 *   rgsw    [n][2 d_a + 2 d_b][N]  RGSW(X^{emb s_i}) rows A(-sm), B(-sm), A(m), B(m)
 *   autos   [w + 1][2 d_auto][N]   auto keys, rows A then B; slot 0 = -g, slot k = g^k
 *   lwe_ksk [d_ks N][n + 1]        LWE key-switching key, row = [b, a_1 .. a_n] mod q_ks
 * (the contents of ServerKeyEvaluationDomain before its forward NTT). */
typedef struct pz_server_key_view {
  const uint64_t *rgsw;
  const uint64_t *autos;
  const uint64_t *lwe_ksk;
} pz_server_key_view;

const char *pz_status_string(pz_status s);
pz_status pz_param_get(int param_id, pz_params *out);

/* Context: parameter set + device tables + a private stream.  ntt_root = 0
 * selects the library's own 2N-th root of unity; a nonzero value must be a
 * primitive 2N-th root mod Q (outputs do not depend on the choice; the
 * option lets tests compare evaluation-domain words). */
pz_status pz_ctx_create(int param_id, int device, pz_ctx **out);
pz_status pz_ctx_create_ex(int param_id, int device, uint64_t ntt_root, pz_ctx **out);
void pz_ctx_destroy(pz_ctx *ctx);
const char *pz_last_error(const pz_ctx *ctx);
/* Error bits kernels of this context set on the device instead of trapping
 * (bit 0: a bounded wait for a bulk copy into shared memory ran out; the
 * kernel returned and its outputs are not valid).  Synchronizes the device,
 * returns the bits in *bits and clears them.  No reference counterpart (the
 * reference panics on the CPU). */
pz_status pz_ctx_device_error(pz_ctx *ctx, uint32_t *bits);
pz_status pz_ctx_params(const pz_ctx *ctx, pz_params *out);
uint64_t pz_ctx_ntt_root(const pz_ctx *ctx);

/* Server key: expanded, NTT'd and laid out on the context's device. */
pz_status pz_key_upload(pz_ctx *ctx, const pz_server_key_view *key, pz_key **out);
void pz_key_release(pz_key *key);
size_t pz_key_device_bytes(const pz_key *key);

/* out[i] = gate[i](c0[i], c1[i]); c0, c1, out: [count][N + 1].
 * Host memory, synchronous (copies in and out inside the call). */
pz_status pz_gate_batch(pz_ctx *ctx, const pz_key *key, const uint8_t *gates, const uint64_t *c0,
                        const uint64_t *c1, uint64_t *out, size_t count);
/* Same on device memory, asynchronous on `stream` (NULL: the CUDA default stream). */
pz_status pz_gate_batch_device(pz_ctx *ctx, const pz_key *key, const uint8_t *d_gates,
                               const uint64_t *d_c0, const uint64_t *d_c1, uint64_t *d_out,
                               size_t count, void *stream);
/* Same as pz_gate_batch_device for callers that cannot allocate device
 * memory on their gate path (device memory fully reserved by another
 * allocator, or a serving thread that must not make allocating CUDA calls).
 * No counterpart in the reference.  The key-switch scratch between the two
 * kernels is a fixed array compiled into the library (PZ_NOALLOC_KS_WORDS
 * u32 words, kept on every GPU that loads the library until exit), so this
 * call allocates nothing; count is limited to PZ_NOALLOC_KS_WORDS / stride
 * (stride = n + 1 rounded up to 32; 4096 gates at NI_8P) and larger batches
 * are rejected with PZ_ERR_INVALID_ARGUMENT.  The first call on a device
 * looks up the array's device address and should come before any stream
 * capture; creating a context on the device makes the next call look it up
 * again.  A cudaDeviceReset in the process destroys every device object of
 * this library: release contexts and keys before it and create new ones
 * after it.  Every call shares the array: calls whose work overlaps on the
 * GPU race and must be serialized by the caller. */
#define PZ_NOALLOC_KS_WORDS (4096u * 672u)
pz_status pz_gate_batch_device_noalloc(pz_ctx *ctx, const pz_key *key, const uint8_t *d_gates,
                                       const uint64_t *d_c0, const uint64_t *d_c1, uint64_t *d_out,
                                       size_t count, void *stream);
/* Diagnostic variant: also writes the key-switched LWE (d_ks_out
 * [count][n + 1] u32, mod q_ks) and the blind-rotated RLWE (d_rlwe_out
 * [count][2][N]) of each gate; either may be NULL. */
pz_status pz_gate_batch_debug_device(pz_ctx *ctx, const pz_key *key, const uint8_t *d_gates,
                                     const uint64_t *d_c0, const uint64_t *d_c1, uint64_t *d_out,
                                     size_t count, uint32_t *d_ks_out, uint64_t *d_rlwe_out,
                                     void *stream);
/* pbs on combined LWE inputs d_lwe [count][N + 1] with the test vector of
 * gate test_vec[i] (pbs.rs:104-233, no gate prelude). */
pz_status pz_pbs_batch_device(pz_ctx *ctx, const pz_key *key, const uint8_t *d_test_vec,
                              const uint64_t *d_lwe, uint64_t *d_out, size_t count, void *stream);
/* Blind rotation + sample extraction from key-switched LWEs (pbs.rs:146-232:
 * odd mod-switch, dlog buckets, test-vector rotation, blind_rotation,
 * sample_extract): d_ks [count][n + 1] u32 mod q_ks, gate test vector per
 * item, d_out [count][N + 1]. */
pz_status pz_blind_rotate_batch_device(pz_ctx *ctx, const pz_key *key, const uint32_t *d_ks,
                                       const uint8_t *d_test_vec, uint64_t *d_out, size_t count,
                                       void *stream);
/* Measured throughput of 32-bit multiply-add (IMAD) instructions on a device:
 * the integer-pipe denominator of the bootstrap's roofline. */
pz_status pz_probe_imad_rate(int device, double *imad_per_second);
/* Measured rates (instructions per second, whole device) of the pipes the
 * butterflies use, rates[k] for k < min(n, PZ_PIPE_PROBES): 0 mad.lo.u32
 * (IMAD), 1 mad.wide.u32, 2 mad.hi.u32, 3 fma.rn.f64, 4 cvt.rn.f64.u64,
 * 5 cvt.rni.u64.f64, 6 mad.lo.u32 and fma.rn.f64 interleaved (each). */
#define PZ_PIPE_PROBES 7
pz_status pz_probe_pipe_rates(int device, double *rates, size_t n);
/* out = -in (mod Q, unreduced: -0 = Q) on `words` u64 words. */
pz_status pz_not_batch_device(pz_ctx *ctx, const uint64_t *d_in, uint64_t *d_out, size_t words,
                              void *stream);

/* Kernel-level entry points (device memory, asynchronous).  The external
 * product and the automorphism of the one-digit parameter sets run with the
 * register cap of the context's blind-rotation variant (0 / 1 / 2: 2 / 3 / 4
 * CTAs per SM; others: 3). */
pz_status pz_ntt_forward_device(pz_ctx *ctx, uint64_t *d_polys, size_t count, void *stream);
pz_status pz_ntt_backward_device(pz_ctx *ctx, uint64_t *d_polys, size_t count, void *stream);
pz_status pz_rlwe_by_rgsw_device(pz_ctx *ctx, const pz_key *key, uint64_t *d_rlwe,
                                 const uint32_t *d_lwe_index, size_t count, int trivial, void *stream);
pz_status pz_rlwe_auto_device(pz_ctx *ctx, const pz_key *key, uint64_t *d_rlwe,
                              const uint32_t *d_slot, size_t count, int trivial, void *stream);
/* d_lwe_in [count][N + 1] mod q_ks -> d_out [count][n + 1] u32 mod q_ks */
pz_status pz_lwe_key_switch_device(pz_ctx *ctx, const pz_key *key, const uint64_t *d_lwe_in,
                                   uint32_t *d_out, size_t count, void *stream);

/* Blind-rotation launch shape: 0 = one CTA per ciphertext; > 0 caps the grid
 * (the kernel then strides over the batch). */
pz_status pz_ctx_set_pbs_grid_limit(pz_ctx *ctx, int grid_limit);
/* Blind-rotation kernel variant for N = 2048: registers capped for 2, 3 or 4
 * resident CTAs per SM (variant 0, 1, 2; default 0), or 3: each ciphertext on a
 * cluster of two CTAs (a and b on different SMs: lower latency per gate). */
pz_status pz_ctx_set_pbs_variant(pz_ctx *ctx, int variant);
/* Launches of at most max_gates gates use variant 3 whatever the variant set
 * (-1, the default: half the GPU's SMs; 0: only if variant 3 is set). */
pz_status pz_ctx_set_split_threshold(pz_ctx *ctx, int max_gates);
int pz_ctx_pbs_variant(const pz_ctx *ctx);
/* Ciphertexts a blind-rotation launch of shape `variant` (-1: the context's
 * current one) holds resident on the device at once: a batch that is a
 * multiple of it runs in whole waves.  No reference counterpart (the
 * reference runs one bootstrap per call, pbs.rs:104-233). */
pz_status pz_ctx_pbs_slots(pz_ctx *ctx, int variant, size_t *slots);
/* Revision tag of the blind-rotation kernels in this library (changes with
 * their code; a profile applies to the revision it was taken on).  No
 * reference counterpart. */
const char *pz_kernel_revision(void);
/* Autotuner: times every blind-rotation variant on synthetic key-switched
 * LWEs with this key -- `batch` of them, or, from one wave up, the largest
 * whole number of that variant's waves not above `batch` -- and keeps the
 * fastest per ciphertext (*ms: its time for `batch`); then times the
 * key-switch kernel with 8, 16 and 32 ciphertexts per CTA and its
 * tensor-core form (64) on `batch` inputs and keeps the fastest.  Both become the context's defaults and the choice
 * for batches in batch's size bucket (floor(log2(gates))); launches in a
 * bucket never tuned use the defaults.  Setting a variant or a tile by hand
 * clears the per-bucket choices.  No reference counterpart. */
pz_status pz_ctx_autotune(pz_ctx *ctx, const pz_key *key, size_t batch, int *variant, double *ms);
/* Key-switch ciphertexts per CTA: 8, 16 or 32 (integer multiply-adds), or
 * 64 (the default): the tensor-core form (mma.sync s8 digits x u8 KSK byte
 * planes, 64 ciphertexts x 224 output columns per CTA, the input
 * coefficients split over more CTAs for small batches), which a key whose
 * digits do not fit s8 runs as 16. */
pz_status pz_ctx_set_ks_tile(pz_ctx *ctx, int ciphertexts);
/* The blind-rotation variant and key-switch tile a batch of `gates` gates
 * would launch with now. */
pz_status pz_ctx_launch_shape(pz_ctx *ctx, size_t gates, int *variant, int *ks_tile);

/* ---- circuits ------------------------------------------------------------------
 * A circuit records gates instead of executing them (the reference executes
 * each BooleanGates call at once); execution runs the circuit level by level,
 * every gate of a level in one batched launch.  Wires are uint32_t handles;
 * PZ_WIRE_NONE marks an invalid/absent wire.  not() is free (it flips a
 * handle bit).  FheUint8 values are 8 wires, least significant bit first
 * (shortint/enc_dec.rs:11-29). */
#define PZ_WIRE_NONE 0xffffffffu
typedef struct pz_circuit pz_circuit;
pz_status pz_circuit_create(pz_circuit **out);
void pz_circuit_destroy(pz_circuit *c);
const char *pz_circuit_last_error(const pz_circuit *c);
uint32_t pz_circuit_input(pz_circuit *c);
/* BooleanGates::{and,...,xnor}(a, b), bool/mod.rs:22-71 */
uint32_t pz_circuit_gate(pz_circuit *c, int gate, uint32_t a, uint32_t b);
/* BooleanGates::not, evaluator.rs:2318-2322 */
uint32_t pz_circuit_not(pz_circuit *c, uint32_t a);
pz_status pz_circuit_output(pz_circuit *c, uint32_t wire);
pz_status pz_circuit_info(pz_circuit *c, size_t *inputs, size_t *gates, size_t *outputs, size_t *levels,
                          size_t *max_level_width);
pz_status pz_circuit_level_sizes(pz_circuit *c, size_t *sizes, size_t capacity);
/* FheUint8 operators (shortint/mod.rs:63-292 over shortint/ops.rs) */
pz_status pz_u8_add(pz_circuit *c, const uint32_t a[8], const uint32_t b[8], uint32_t out[8],
                    uint32_t *overflow);           /* AddAssign / overflowing_add */
pz_status pz_u8_sub(pz_circuit *c, const uint32_t a[8], const uint32_t b[8], uint32_t out[8],
                    uint32_t *overflow);           /* Sub / overflowing_sub */
pz_status pz_u8_mul(pz_circuit *c, const uint32_t a[8], const uint32_t b[8], uint32_t out[8]);
/* div_rem; when div_zero_flag is non-NULL it is updated like set_div_by_zero_flag
 * (PZ_WIRE_NONE on entry: no flag yet) */
pz_status pz_u8_div_rem(pz_circuit *c, const uint32_t a[8], const uint32_t b[8], uint32_t quotient[8],
                        uint32_t remainder[8], uint32_t *div_zero_flag);
/* op: 0 eq, 1 neq, 2 lt, 3 gt, 4 le, 5 ge */
pz_status pz_u8_cmp(pz_circuit *c, int op, const uint32_t a[8], const uint32_t b[8], uint32_t *out);
/* mux: selector ? a : b */
pz_status pz_u8_mux(pz_circuit *c, const uint32_t a[8], const uint32_t b[8], uint32_t selector,
                    uint32_t out[8]);
/* Execute: inputs [n_inputs][N + 1] in input order, outputs [n_outputs][N + 1]
 * in output order.  _device: device buffers, asynchronous on `stream`;
 * pz_circuit_run: host buffers, synchronous. */
pz_status pz_circuit_run_device(pz_ctx *ctx, const pz_key *key, pz_circuit *c, const uint64_t *d_inputs,
                                uint64_t *d_outputs, void *stream);
pz_status pz_circuit_run(pz_ctx *ctx, const pz_key *key, pz_circuit *c, const uint64_t *inputs,
                         uint64_t *outputs);
/* Capture the whole circuit on these device buffers as one CUDA graph, then
 * replay it with a single launch. */
pz_status pz_circuit_capture_graph(pz_ctx *ctx, const pz_key *key, pz_circuit *c, const uint64_t *d_inputs,
                                   uint64_t *d_outputs, void *stream);
pz_status pz_circuit_replay_graph(pz_circuit *c, void *stream);

/* ---- wire formats (no reference counterpart: the reference serialises nothing) ----
 * Device-form server key as bytes, for checkpoint / restore and for moving a
 * session between processes: a 64-byte header (parameter set, NTT root, key
 * form, sizes) and the device arrays as they are.  Import copies them back
 * without any conversion; a blob from another parameter set, NTT root or key
 * form (a build with another multiply-accumulate reduction) is refused.  With
 * buf = NULL, export only writes the required *size. */
pz_status pz_key_export(const pz_key *key, void *buf, size_t capacity, size_t *size);
pz_status pz_key_import(pz_ctx *ctx, const void *buf, size_t size, pz_key **out);
/* Circuits as bytes (wire handles keep their meaning); a malformed blob is
 * rejected with PZ_ERR_INVALID_ARGUMENT. */
pz_status pz_circuit_serialize(const pz_circuit *c, void *buf, size_t capacity, size_t *size);
pz_status pz_circuit_deserialize(const void *buf, size_t size, pz_circuit **out);

/* ---- seeded server keys (device-side expansion) ------------------------------------
 * What a server receives after key aggregation (SeededInteractiveMultiPartyServerKey,
 * SeededNonInteractiveMultiPartyServerKey; bool/keys.rs:536-781, 851-1004): the RGSW
 * ciphertexts in full, but only the B rows of the auto keys and column 0 of the LWE
 * key-switching key -- their A parts come from CRS-derived ChaCha8 seeds.  The upload
 * regenerates the A parts on the device exactly as ServerKeyEvaluationDomain::from
 * does (keys.rs:687-781; NI: keys.rs:869-1004), then converts like pz_key_upload.
 *   rgsw       [n][2 d_a + 2 d_b][N]  as in pz_server_key_view
 *   auto_b     [w + 1][d_auto][N]     B rows, slots in auto_element_dlogs order
 *                                     (parameters.rs:364-370: 0 = -g, k = g^k)
 *   lwe_ksk_b  [d_ks N]               column 0 of the LWE KSK rows
 *   auto_seed, lwe_ksk_seed           cr_seed.auto_keys_cts_seed(), cr_seed.lwe_ksk_cts_seed()
 * The arrays may be in host or device memory. */
typedef struct pz_seeded_server_key_view {
  const uint64_t *rgsw;
  const uint64_t *auto_b;
  const uint64_t *lwe_ksk_b;
  uint8_t auto_seed[32];
  uint8_t lwe_ksk_seed[32];
} pz_seeded_server_key_view;
pz_status pz_key_upload_seeded(pz_ctx *ctx, const pz_seeded_server_key_view *key, pz_key **out);

/* Seed-expansion primitives, exposed so their words can be checked against
 * published known answers.  The reference expands seeds with rand_chacha
 * 0.3.1's ChaCha8Rng and samples with rand 0.8.5's
 * Uniform::new_inclusive(0, q - 1) (random.rs:93-110); the seeded key upload
 * and the NI unseed use these same functions on the device.
 * pz_chacha_block: the ChaCha block function (rounds 8, 12 or 20) on a full
 * 16-word input state; out = rounds(state) + state.
 * pz_uniform_mod_word: one 64-bit word through the uniform sampler: accepted
 * when lo64(word q) <= 2^64 - 1 - (2^64 - q) mod q, sample = hi64(word q). */
pz_status pz_chacha_block(const uint32_t state[16], int rounds, uint32_t out[16]);
pz_status pz_uniform_mod_word(uint64_t q, uint64_t word, uint64_t *sample, int *accepted);

/* ---- non-interactive input path (NI parameter sets, N = 2048) ---------------------
 * A user of a non-interactive session sends its bools as seeded RLWEs under its own
 * RLWE secret u_j (NonInteractiveBatchedFheBools, bool/ni_mp_api.rs:182-196); the
 * server regenerates the a-parts, key-switches u_j -> s with that user's ui_to_s key
 * and extracts one LWE per bool (KeySwitchWithId + extract, ni_mp_api.rs:217-236,
 * 400-440). */
typedef struct pz_ni_ksk pz_ni_ksk;
/* ui_to_s key of one user: [2 ni_ks_d][N] u64 coefficient domain, rows A then B
 * (ShoupNonInteractiveServerKeyEvaluationDomain::ui_to_s_ksk, bool/keys.rs:1083-1085,
 * before its forward NTT) */
pz_status pz_ni_ksk_upload(pz_ctx *ctx, const uint64_t *ksk, pz_ni_ksk **out);
/* the same key from its B rows [ni_ks_d][N] and its seed
 * (cr_seed.ui_to_s_ks_seed_for_user_i(user), keys.rs:965-1000): A rows regenerated
 * on the device; ksk_b in host or device memory */
pz_status pz_ni_ksk_upload_seeded(pz_ctx *ctx, const uint64_t *ksk_b, const uint8_t seed[32], pz_ni_ksk **out);
void pz_ni_ksk_release(pz_ni_ksk *ksk);
/* NonInteractiveBatchedFheBools::from (ni_mp_api.rs:248-280): d_b [count][N] (the
 * seeded RLWEs' b-parts) -> d_rlwe [count][2][N], a-parts from ChaCha8(seed) in batch
 * order.  Returns when done (it checks the rejection-sampling margin). */
pz_status pz_ni_unseed_device(pz_ctx *ctx, const uint8_t seed[32], const uint64_t *d_b, uint64_t *d_rlwe,
                              size_t count, void *stream);
/* rlwe_key_switch (rgsw/runtime.rs:1001-1063): d_in, d_out [count][2][N] */
pz_status pz_ni_key_switch_device(pz_ctx *ctx, const pz_ni_ksk *ksk, const uint64_t *d_in, uint64_t *d_out,
                                  size_t count, void *stream);
/* BatchedFheBools::extract (ni_mp_api.rs:217-236) = sample_extract (pbs.rs:423-449):
 * d_lwe[c] = bool d_index[c] of the batch d_rlwe [rlwe_count][2][N] (RLWE index / N,
 * coefficient index % N); an index past the batch leaves d_lwe[c] unchanged */
pz_status pz_sample_extract_device(pz_ctx *ctx, const uint64_t *d_rlwe, size_t rlwe_count,
                                   const uint32_t *d_index, uint64_t *d_lwe, size_t count, void *stream);
/* The three steps on host buffers (synchronous): b [rlwe_count][N] -> lwe_out
 * [nbools][N + 1] for bools 0 .. nbools - 1 */
pz_status pz_ni_ingest(pz_ctx *ctx, const pz_ni_ksk *ksk, const uint8_t seed[32], const uint64_t *b,
                       size_t rlwe_count, uint64_t *lwe_out, size_t nbools);

/* ---- server-key aggregation (interactive protocol) ----------------------------------
 * rgsw_by_rgsw_inplace (rgsw/runtime.rs:883-985), batched: d_rgsw0[c] <- d_rgsw0[c] x
 * d_rgsw1[c].  d_rgsw0 [count][4][N]: RGSW in the rlwe x rgsw shape (d_a = d_b = 1),
 * coefficient domain, in place; d_rgsw1 [count][2 rgrg_d_a + 2 rgrg_d_b][N]: RGSW in the
 * rgsw x rgsw shape, coefficient domain (converted on the device).  Returns when done. */
pz_status pz_rgsw_by_rgsw_device(pz_ctx *ctx, uint64_t *d_rgsw0, const uint64_t *d_rgsw1, size_t count,
                                 void *stream);
/* The RGSW step of aggregate_interactive_multi_party_server_key_shares
 * (bool/evaluator.rs:1110-1200): d_rgsw0[c] <- d_rgsw0[c] x d_others[0][c] x ... x
 * d_others[steps - 1][c], the other users in order; d_others [steps][count][rows][N]. */
pz_status pz_aggregate_rgsw_device(pz_ctx *ctx, uint64_t *d_rgsw0, const uint64_t *d_others, size_t steps,
                                   size_t count, void *stream);
/* The whole aggregate_interactive_multi_party_server_key_shares (bool/evaluator.rs:1050-
 * 1200) on one user's share per entry (CommonReferenceSeededInteractiveMultiPartyServer-
 * KeyShare, bool/keys.rs:334-360), u64, coefficient domain, DEVICE memory:
 *   self_leader_rgsws      [segment][2 rlrg_d_a + 2 rlrg_d_b][N]  RGSWs of the LWE indices
 *                          the user leads (multi_party_user_id_lwe_segment)
 *   not_self_leader_rgsws  [lwe_n - segment][2 rgrg_d_a + 2 rgrg_d_b][N]  the other
 *                          indices, in index order
 *   auto_keys              [w + 1][d_auto][N] B rows, auto_element_dlogs order
 *   lwe_ksk                [d_ks N]
 * shares[j] is user j's.  Outputs (DEVICE memory, the SeededInteractiveMultiPartyServerKey
 * form): d_rgsw [lwe_n][4][N], d_auto_b [w + 1][d_auto][N], d_lwe_b [d_ks N].  Returns
 * when done. */
typedef struct pz_server_key_share_view {
  const uint64_t *self_leader_rgsws;
  const uint64_t *not_self_leader_rgsws;
  const uint64_t *auto_keys;
  const uint64_t *lwe_ksk;
} pz_server_key_share_view;
pz_status pz_aggregate_device(pz_ctx *ctx, const pz_server_key_share_view *shares, size_t users,
                              uint64_t *d_rgsw, uint64_t *d_auto_b, uint64_t *d_lwe_b, void *stream);
/* InteractiveMultiPartyCrs (bool/evaluator.rs:78-100) seeds: what = 0 public-key share,
 * 1 auto keys, 2 LWE KSK.  Host only. */
#define PZ_ICRS_PUBLIC_KEY 0
#define PZ_ICRS_AUTO_KEYS 1
#define PZ_ICRS_LWE_KSK 2
pz_status pz_interactive_crs_seed(const uint8_t crs_seed[32], int what, uint8_t out[32]);
/* Aggregation followed by the seeded expansion (keys.rs:687-781): the server key. */
pz_status pz_aggregate_server_key(pz_ctx *ctx, const uint8_t crs_seed[32], const pz_server_key_share_view *shares,
                                  size_t users, pz_key **key_out);

/* ---- server-key aggregation (non-interactive protocol) ------------------------------
 * aggregate_non_interactive_multi_party_server_key_shares (bool/evaluator.rs:1222-1622).
 * One user's share (CommonReferenceSeededNonInteractiveMultiPartyServerKeyShare,
 * bool/keys.rs:1240-1290), every array u64, coefficient domain, DEVICE memory:
 *   ui_to_s_ksk        [ni_ks_d][N]       (a_k s_j + e + beta u_j), a_k from the user's seed
 *   ksk_zero_encs      [users - 1][ni_ks_d][N]  zero encryptions for user l at l (l < own id)
 *                                         or l - 1 (ui_to_s_ksk_zero_encs_for_user_i)
 *   self_leader_cts    [segment][max(rlrg_d_a, rlrg_d_b)][N]  NI RGSW rows of the indices
 *                                         the user leads (multi_party_user_id_lwe_segment)
 *   not_leader_cts     [lwe_n - segment][max(rgrg_d_a, rgrg_d_b)][N]  the other indices,
 *                                         in index order
 *   rgsw_zero_encs     [lwe_n][rgrg_d_a][N]
 *   auto_keys          [w + 1][d_auto][N] B rows, auto_element_dlogs order
 *   lwe_ksk            [d_ks N]           (mod lwe q)
 * Entries are canonical (< the modulus), as the reference's additions assume. */
typedef struct pz_ni_server_key_share_view {
  const uint64_t *ui_to_s_ksk;
  const uint64_t *ksk_zero_encs;
  const uint64_t *self_leader_cts;
  const uint64_t *not_leader_cts;
  const uint64_t *rgsw_zero_encs;
  const uint64_t *auto_keys;
  const uint64_t *lwe_ksk;
} pz_ni_server_key_share_view;
/* NonInteractiveMultiPartyCrs (bool/evaluator.rs:115-172) seeds from the common
 * reference seed: what = 0 auto keys, 1 LWE KSK, 2 ui_to_s KSK of user `index`,
 * 3 NI RGSW of LWE index `index`.  Host only. */
#define PZ_CRS_AUTO_KEYS 0
#define PZ_CRS_LWE_KSK 1
#define PZ_CRS_UI_TO_S_KSK 2
#define PZ_CRS_NI_RGSW 3
pz_status pz_ni_crs_seed(const uint8_t crs_seed[32], int what, size_t index, uint8_t out[32]);
/* The aggregation, outputs in DEVICE memory in the form the reference returns
 * (SeededNonInteractiveMultiPartyServerKey, coefficient domain):
 *   d_ksk_b   [users][ni_ks_d][N]  per-user Ksk(u_j -> s) B rows
 *   d_rgsw    [lwe_n][4][N]        RGSW(X^{z[l]}) in the rlwe x rgsw shape
 *   d_auto_b  [w + 1][d_auto][N]   summed auto key B rows
 *   d_lwe_b   [d_ks N]             summed LWE KSK column 0
 * shares[j] is user j's.  Returns when done. */
pz_status pz_ni_aggregate_device(pz_ctx *ctx, const uint8_t crs_seed[32], const pz_ni_server_key_share_view *shares,
                                 size_t users, uint64_t *d_ksk_b, uint64_t *d_rgsw, uint64_t *d_auto_b,
                                 uint64_t *d_lwe_b, void *stream);
/* Aggregation followed by the expansion to the evaluation form (keys.rs:869-1004):
 * the server key and every user's ui_to_s key (ksks_out[users]). */
pz_status pz_ni_aggregate_server_key(pz_ctx *ctx, const uint8_t crs_seed[32],
                                     const pz_ni_server_key_share_view *shares, size_t users, pz_key **key_out,
                                     pz_ni_ksk **ksks_out);

/* ---- multi-session executor (serving) ---------------------------------------------
 * No reference counterpart: the reference evaluates one gate at a time, in
 * the calling thread, against its thread's one global server key
 * (bool/mp_api.rs:20-26).  A server runs on one device.  A session is a
 * (context, device key) pair of any parameter set sharing the server's ring
 * (all production sets: N = 2048, the same Q); a job is a circuit submitted
 * to a session.  pz_server_step admits pending jobs in arrival order while
 * their wires fit the device arena and their session's key is resident or
 * can be made resident (admission by ciphertext + key bytes; see managed
 * sessions below), then advances every admitted job by one circuit level:
 * the gates of all sessions run as one ragged key-switch launch and one
 * ragged blind-rotation launch per max_items gates, each gate with its own
 * session's parameters and key.  A job admitted while others are mid-circuit
 * starts at its level 1 in the same launches (continuous batching).  Not
 * thread-safe: one host thread drives a server.  Job buffers must stay valid
 * and the circuit unchanged until the job is done. */
typedef struct pz_server pz_server;
typedef struct {
  size_t pending, active, done, failed;
  size_t arena_slots, arena_slots_used, arena_bytes;
  size_t sessions, key_bytes;
  uint64_t steps, gates, launches;
  size_t resident_key_bytes, key_budget; /* key_budget 0: no limit */
  uint64_t key_imports, key_evictions;
} pz_server_stats;
#define PZ_SERVER_DRY_RUN (-1) /* device id of a host-only server: bookkeeping, no GPU work */
/* arena_bytes: device bytes for job wires ((n_inputs + n_gates) x (N + 1) x 8 per job);
 * max_items: gates per ragged launch (larger steps are split) */
pz_status pz_server_create(int device, size_t arena_bytes, size_t max_items, pz_server **out);
void pz_server_destroy(pz_server *s);
const char *pz_server_last_error(const pz_server *s);
pz_status pz_server_add_session(pz_server *s, pz_ctx *ctx, const pz_key *key, uint32_t *session);
/* dry-run servers only: a session of parameter set param_id without a key */
pz_status pz_server_add_virtual_session(pz_server *s, int param_id, uint32_t *session);
/* Managed session: the server holds the session's device key only while it
 * is needed, importing it from the caller's device-form blob (pz_key_export;
 * the blob must stay valid and unchanged while the server exists).  A job of
 * a managed session is admitted when its key is resident or fits the key
 * budget after evicting the least recently used resident managed keys of
 * sessions with no job in flight (import: a plain host-to-device copy of the
 * blob); otherwise it waits, in arrival order.  A job whose key alone exceeds
 * the budget fails (state 3).  No reference counterpart (the reference holds
 * one server key per process, bool/mp_api.rs:128-146). */
pz_status pz_server_add_managed_session(pz_server *s, pz_ctx *ctx, const void *key_blob, size_t blob_bytes,
                                        uint32_t *session);
/* dry-run servers only: a managed session of param_id (residency bookkeeping only) */
pz_status pz_server_add_virtual_managed_session(pz_server *s, int param_id, uint32_t *session);
/* Device bytes resident managed keys may hold (0: no limit, the default). */
pz_status pz_server_set_key_budget(pz_server *s, size_t bytes);
/* *resident = 1 when the session's key is on the device now. */
pz_status pz_server_session_resident(pz_server *s, uint32_t session, int *resident);
/* inputs [n_inputs][N + 1], outputs [n_outputs][N + 1]; device_io = 1: device pointers */
pz_status pz_server_submit(pz_server *s, uint32_t session, pz_circuit *c, const uint64_t *inputs,
                           uint64_t *outputs, int device_io, uint64_t *job);
/* One scheduling step (admit, one level of every admitted job, retire);
 * returns when its device work is complete.  *gates: bootstraps run. */
pz_status pz_server_step(pz_server *s, size_t *gates);
/* state: 0 pending, 1 running, 2 done, 3 failed (needs more than the whole
 * arena); latency = done - submit, queue = admit - submit (ms, -1 if n/a) */
pz_status pz_server_job_status(pz_server *s, uint64_t job, int *state, double *latency_ms, double *queue_ms);
pz_status pz_server_forget(pz_server *s, uint64_t job);
pz_status pz_server_stats_get(pz_server *s, pz_server_stats *out);
/* Ragged blind-rotation launch shape (variant as pz_ctx_set_pbs_variant: 0,
 * 1, 2 or 4 -- steps of at most half the SMs' gates take the two-CTA shape 3
 * by themselves; grid limit 0 = one CTA per gate) */
pz_status pz_server_set_launch(pz_server *s, int pbs_variant, int grid_limit);
/* Autotuner: times the variants 0, 1, 2, 4 x {one CTA per gate, persistent
 * 2 x SMs} on `batch` synthetic gates spread over the sessions with a
 * resident key and keeps the fastest.  Needs an idle server (no admitted
 * job). */
pz_status pz_server_autotune(pz_server *s, size_t batch, int *variant, int *grid_limit, double *ms);
/* Which jobs advance a level at each step.  ALL_READY (default): every
 * admitted job.  CRITICAL_PATH: the jobs with the most levels left always
 * advance; the others fill the step only up to the launch-time tier those
 * already pay for (one CTA per SM, two, ..., then whole waves), deepest
 * first -- a batch of jobs submitted together ends after the same number of
 * steps with fewer partly-filled launches; a short job may wait behind a
 * deep one, so serving keeps ALL_READY.  Results are the same under both. */
#define PZ_SCHEDULE_ALL_READY 0
#define PZ_SCHEDULE_CRITICAL_PATH 1
pz_status pz_server_set_schedule(pz_server *s, int policy);

#ifdef __cplusplus
}
#endif
#endif
