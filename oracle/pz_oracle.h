/*
 * pz_oracle.h -- CPU oracle for the server-side gate bootstrap of phantom-zone.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: only tests/, the
 * smoke() entry point and bench.py's cpu_baseline / reference legs may load
 * it.  The product (phantom-zone_b200/) never links, loads or calls it.
 *
 * It restates, in C++17 with u64 / unsigned __int128 / IEEE double exactly as
 * the Rust code does, the reference's path:
 *   src/pbs.rs:104-482            pbs, blind_rotation, mod_switch_odd,
 *                                 sample_extract, monomial_mul
 *   src/rgsw/runtime.rs:363-855   decompose_r, rlwe_auto(_shoup),
 *                                 rlwe_by_rgsw(_shoup)
 *   src/ntt.rs:24-442             Harvey butterflies, CT forward, GS inverse
 *   src/decomposer.rs:13-309      signed gadget decomposition
 *   src/lwe.rs:14-44              lwe_key_switch
 *   src/backend/modulus_u64.rs    Barrett mul, add/sub/neg, shoup_matrix_fma
 *   src/backend/power_of_2.rs     mask arithmetic mod 2^k
 *   src/bool/evaluator.rs:651-784,2118-2245   dlog map, test vectors, gates
 *   src/bool/parameters.rs:526-726            parameter sets
 * plus a client-side harness (key generation, encryption, decryption) that
 * the reference runs on clients and which is out of the GPU path's scope.
 *
 * Parity status: the Rust reference cannot be built in this environment (no
 * cargo/rustc, no crate sources), and it ships no golden vectors: every
 * reference test draws from an entropy-seeded RNG.  Equality with the Rust
 * binary's output words is therefore UNPINNED.  The oracle is pinned instead
 * by the reference's own property tests, restated in tests/test_oracle.py:
 * NTT vs schoolbook negacyclic product (ntt.rs:510-540), Shoup FMA vs naive
 * u128 (modulus_u64.rs:284-336), decomposition recomposition
 * (decomposer.rs:325-370), Shoup vs non-Shoup external product and
 * automorphism bit-equality (rgsw/mod.rs:526-831), gate truth tables and
 * FheUint8 plaintext semantics under decryption (mp_api.rs:491-695).
 */
#ifndef PZ_ORACLE_H
#define PZ_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  uint64_t rlwe_q;      /* Q */
  uint64_t lwe_q;       /* q_ks, a power of two */
  uint32_t br_q;        /* blind-rotation modulus */
  uint32_t rlwe_n;      /* N */
  uint32_t lwe_n;       /* n */
  uint32_t lwe_logb, lwe_d;          /* key-switch decomposer */
  uint32_t rlrg_logb, rlrg_d_a, rlrg_d_b; /* RLWE x RGSW decomposer */
  uint32_t auto_logb, auto_d;        /* automorphism decomposer */
  uint32_t g, w;                     /* generator, window */
  uint32_t lwe_secret_gaussian;      /* 1: LWE secret from the error distribution */
  uint32_t variant;                  /* 0 single, 1 interactive, 2 non-interactive */
  uint32_t embedding_factor;         /* 2N / br_q */
  uint32_t rgsw_rows;                /* 2 d_a + 2 d_b */
  uint32_t auto_rows;                /* 2 d_auto */
  uint32_t n_auto_keys;              /* w + 1 */
  uint32_t ni_ks_logb, ni_ks_d;      /* ui_to_s key switch decomposition (NI sets; 0 otherwise) */
  uint32_t rgrg_logb, rgrg_d_a, rgrg_d_b; /* RGSW x RGSW decomposition (0: none) */
} orc_param_info;

/* Parameter set ids, in the order of src/bool/parameters.rs:526-726. */
enum {
  ORC_I_2P_LB_SR = 0, ORC_I_4P = 1, ORC_I_8P = 2, ORC_NI_2P = 3,
  ORC_NI_4P_HB_FR = 4, ORC_NI_4P_LB_SR = 5, ORC_NI_8P = 6, ORC_SP_TEST = 7,
  ORC_NUM_PARAMS = 8
};

/* Gate ids: and, nand, or, nor, xor, xnor (evaluator.rs:2163-2245). */
enum { ORC_AND = 0, ORC_NAND = 1, ORC_OR = 2, ORC_NOR = 3, ORC_XOR = 4, ORC_XNOR = 5 };

int orc_param_info_get(int param_id, orc_param_info *out);

/* --- evaluator (BoolEvaluator::new, evaluator.rs:651-784) ------------------ */
void *orc_eval_new(int param_id);
void orc_eval_free(void *ev);
/* psi (the 2N-th root the NTT uses) and its bit-reversed power tables. */
uint64_t orc_eval_psi(void *ev);
void orc_eval_tables(void *ev, uint64_t *psi_br, uint64_t *psi_inv_br, uint64_t *n_inv);
/* test vector (length br_q/2) of a gate, and the dlog map (length br_q) */
void orc_eval_test_vec(void *ev, int gate, uint64_t *out);
void orc_eval_dlog_map(void *ev, uint32_t *out);
/* auto map of key slot k (0 -> -g, k>=1 -> g^k mod br_q): index + sign */
void orc_eval_auto_map(void *ev, int k, uint32_t *index, uint8_t *sign);

/* --- arithmetic pins --------------------------------------------------------- */
void orc_ntt_forward(void *ev, uint64_t *poly, int lazy);
void orc_ntt_backward(void *ev, uint64_t *poly, int lazy);
/* which: 0 lwe (KS), 1 rlrg a, 2 rlrg b, 3 auto; writes d digits */
int orc_decompose(void *ev, int which, uint64_t value, uint64_t *digits);
void orc_shoup_matrix_fma(uint64_t q, uint64_t *out, const uint64_t *a,
                          const uint64_t *a_shoup, const uint64_t *b,
                          size_t rows, size_t n);
uint64_t orc_shoup_repr(uint64_t v, uint64_t q);
uint64_t orc_barrett_mul(void *ev, uint64_t a, uint64_t b);
void orc_negacyclic_mul(uint64_t q, const uint64_t *a, const uint64_t *b,
                        uint64_t *out, size_t n);

/* FheUint8 operations evaluated gate by gate in the reference's order
 * (shortint/mod.rs:63-292 over shortint/ops.rs).  op: 0 add, 1 sub, 2 mul,
 * 3 div_rem, 4 eq, 5 neq, 6 lt, 7 gt, 8 le, 9 ge, 10 mux, 11 overflowing_add,
 * 12 overflowing_sub.  a, b, out, out2: [8][N+1]; comparisons write [1][N+1]. */
int orc_u8_op(void *ev, void *key, int op, const uint64_t *a, const uint64_t *b, const uint64_t *sel,
              uint64_t *out, uint64_t *out2, uint64_t *flag, int *flag_set);
/* The gates operation `op` issues, tallied by gate code (and, nand, or, nor,
 * xor, xnor) without bootstrapping anything (a dry run on zero ciphertexts). */
int orc_u8_gate_mix(void *ev, int op, uint64_t counts[6]);

/* generic pins: the reference's unit tests at their own sizes */
uint64_t orc_generate_prime(uint32_t num_bits, uint64_t modulo, uint64_t upper_bound);
void *orc_ntt_custom_new(uint64_t q, size_t n);
void orc_ntt_custom_free(void *h);
void orc_ntt_custom_forward(void *h, uint64_t *a, int lazy);
void orc_ntt_custom_backward(void *h, uint64_t *a, int lazy);
uint64_t orc_mul_mod_barrett(uint64_t q, uint64_t a, uint64_t b);
uint32_t orc_decompose_custom(uint64_t q, uint32_t logb, uint32_t d, uint64_t value, uint64_t *out);
uint64_t orc_round_value(uint64_t v, uint32_t ignore_bits);
uint64_t orc_recompose(uint64_t q, uint32_t logb, uint32_t d, const uint64_t *limbs);

/* --- server key ----------------------------------------------------------------
 * Coefficient-domain, fully expanded server key (what set_server_key holds
 * before the forward NTT, keys.rs:687-781):
 *   rgsw  [n][2 d_a + 2 d_b][N]  rows A(-sm), B(-sm), A(m), B(m)
 *   autos [w+1][2 d_auto][N]      rows A, B; slot 0 = -g, slot k = g^k
 *   ksk   [d_ks N][n+1]           row = [b, a_1..a_n] mod q_ks
 */
void *orc_key_new(void *ev, const uint64_t *rgsw, const uint64_t *autos,
                  const uint64_t *ksk);
void orc_key_free(void *key);

/* --- the hot path ------------------------------------------------------------- */
void orc_rlwe_by_rgsw(void *ev, void *key, uint64_t *rlwe, uint32_t lwe_index,
                      int trivial, int shoup);
void orc_rlwe_auto(void *ev, void *key, uint64_t *rlwe, uint32_t k, int trivial,
                   int shoup);
void orc_lwe_key_switch(void *ev, void *key, const uint64_t *lwe_in, uint64_t *out);
/* pbs on lwe (N+1 words, in place) with the gate's test vector.  If ks_out
 * (n+1 words) / rlwe_out (2N words) are non-NULL they receive the key-switch
 * output and the blind-rotated accumulator. Returns the number of
 * non-trivial automorphisms executed. */
int orc_pbs(void *ev, void *key, int gate, uint64_t *lwe, uint64_t *ks_out,
            uint64_t *rlwe_out);
/* gate: c0 <- gate(c0, c1) (evaluator.rs:2163-2245) */
void orc_gate(void *ev, void *key, int gate, uint64_t *c0, const uint64_t *c1);
void orc_not(void *ev, uint64_t *c0);
/* independent gates on `threads` host threads, one evaluator scratch per
 * thread (the reference's thread-local evaluator model, mp_api.rs:20-22) */
void orc_gate_batch(void *ev, void *key, const uint8_t *gates, const uint64_t *c0,
                    const uint64_t *c1, uint64_t *out, size_t count, int threads);
void orc_sample_extract(void *ev, const uint64_t *rlwe, uint64_t *lwe, uint32_t index);
/* non-interactive input path (NI parameter sets): unseed a batch of seeded
 * RLWEs (ni_mp_api.rs:248-280), b [count][N] -> rlwe [count][2][N]; key switch
 * u_j -> s (runtime.rs:1001-1063) with Ksk [2 x 50][N] in the coefficient
 * domain (rows A then B), in/out [2][N] */
void orc_ni_unseed(void *ev, const uint8_t seed[32], const uint64_t *b, size_t count, uint64_t *rlwe);
void orc_ni_key_switch(void *ev, const uint64_t *ksk, const uint64_t *in, uint64_t *out);

/* --- client-side harness (reference runs this on clients; out of scope) -------- */
/* ChaCha8 stream (rand_chacha 0.3 layout), for seeding */
/* ChaCha block function with `rounds` rounds on a full 16-word input state
 * (out = rounds(state) + state), and one word through rand 0.8's uniform
 * sampler for [0, q) (returns 1 when accepted; *sample = hi64(word q)). */
void orc_chacha_block(const uint32_t state[16], int rounds, uint32_t out[16]);
int orc_uniform_mod_word(uint64_t q, uint64_t word, uint64_t *sample);
void *orc_rng_new(const uint8_t seed[32]);
void orc_rng_free(void *rng);
uint64_t orc_rng_next_u64(void *rng);
void orc_rng_uniform_mod(void *rng, uint64_t q, uint64_t *out, size_t n);

/* Client keys of `parties` parties from seeds seed_p = 32 x byte(p + 1 + 16*seed_base).
 * Writes the ideal (summed) secrets: s [N] as i32, z [n] as i32, and each
 * party's secrets (s_parts [parties][N], z_parts [parties][n]) if non-NULL. */
void orc_client_keys(void *ev, int parties, int seed_base, int32_t *s, int32_t *z,
                     int32_t *s_parts, int32_t *z_parts);
/* Server key (coefficient domain, layout of orc_key_new) under the ideal
 * secrets, errors drawn from ChaCha8(err_seed).  Encrypting under the summed
 * secret gives the key structure of the interactive/NI protocols' output
 * (which only the client side produces) with less noise. */
void orc_gen_server_key(void *ev, const int32_t *s, const int32_t *z,
                        const uint8_t err_seed[32], uint64_t *rgsw, uint64_t *autos,
                        uint64_t *ksk);
/* NI batched bool encryption under the user's RLWE secret u (ni_mp_api.rs:302-345):
 * b_out [ceil(nbits / N)][N]; and an ideal Ksk(u -> s) [2 x 50][N] (coefficient domain) */
void orc_ni_encrypt_bools(void *ev, const int32_t *u, const uint8_t seed[32], const uint8_t err_seed[32],
                          const uint8_t *bits, size_t nbits, uint64_t *b_out);
void orc_ni_ksk_gen(void *ev, const int32_t *u, const int32_t *s, const uint8_t err_seed[32], uint64_t *ksk);
/* Seeded server key expansion (keys.rs:687-781, 869-1004) before the forward NTT:
 * auto_b [w+1][d_auto][N], lwe_b [d_ks N] -> autos [w+1][2 d_auto][N], ksk [d_ks N][n+1];
 * and one user's ui_to_s key from its B rows [50][N] -> [100][N] */
void orc_expand_seeded_key(void *ev, const uint64_t *auto_b, const uint8_t auto_seed[32], const uint64_t *lwe_b,
                           const uint8_t lwe_seed[32], uint64_t *autos, uint64_t *ksk);
void orc_expand_ni_ksk(void *ev, const uint64_t *b, const uint8_t seed[32], uint64_t *ksk);
/* Key aggregation: rgsw_by_rgsw_inplace (runtime.rs:883-985); rgsw0 [2 d_a + 2 d_b][N]
 * (rlwe x rgsw shape) in place, rgsw1 [2 rgrg_d_a + 2 rgrg_d_b][N]; both coefficient domain.
 * orc_rgsw_encrypt: RGSW(m) under s, which = 0 rlwe x rgsw shape, 1 rgsw x rgsw shape. */
void orc_rgsw_by_rgsw(void *ev, uint64_t *rgsw0, const uint64_t *rgsw1);
void orc_rgsw_encrypt(void *ev, const int32_t *s, const uint64_t *m, int which, const uint8_t seed[32],
                      uint64_t *out);
/* NonInteractiveMultiPartyCrs seeds (evaluator.rs:115-172): what 0 auto keys, 1 LWE KSK,
 * 2 ui_to_s KSK of user `index`, 3 NI RGSW of LWE index `index` */
void orc_ni_crs_seed(const uint8_t crs[32], int what, size_t index, uint8_t out[32]);
/* InteractiveMultiPartyCrs seeds (evaluator.rs:78-100): what 0 public-key share, 1 auto keys, 2 LWE KSK */
void orc_interactive_crs_seed(const uint8_t crs[32], int what, uint8_t out[32]);
/* aggregate_non_interactive_multi_party_server_key_shares (evaluator.rs:1222-1622); per-user
 * pointer arrays in user id order; RGSWs for LWE indices [i0, i1) */
void orc_ni_aggregate(void *ev, const uint8_t crs[32], int users, const uint64_t *const *ui_to_s_ksk,
                      const uint64_t *const *ksk_zero_encs, const uint64_t *const *self_leader,
                      const uint64_t *const *not_leader, const uint64_t *const *zero_encs,
                      const uint64_t *const *auto_keys, const uint64_t *const *lwe_ksk, size_t i0, size_t i1,
                      uint64_t *ksk_out, uint64_t *rgsw_out, uint64_t *auto_out, uint64_t *lwe_out);
/* harness: auto-key / LWE-KSK B parts under (s, z) with CRS-stream A parts */
void orc_gen_seeded_auto_lwe(void *ev, const int32_t *s, const int32_t *z, const uint8_t auto_seed[32],
                             const uint8_t lwe_seed[32], const uint8_t err_seed[32], uint64_t *auto_b,
                             uint64_t *lwe_b);
/* harness: RGSW / KSK parts of one user's NI server key share (evaluator.rs:1624-1975) */
void orc_ni_gen_share(void *ev, const uint8_t crs[32], int user, int users, const int32_t *s, const int32_t *u,
                      const int32_t *z, const uint8_t err_seed[32], uint64_t *ksk, uint64_t *ksk_zero,
                      uint64_t *self_leader, uint64_t *not_leader, uint64_t *zero);
/* LWE_Q encryption of bool under s (lwe.rs:104-137, m = +-Q/8) */
void orc_encrypt_bool(void *ev, void *rng, const int32_t *s, int bit, uint64_t *lwe);
/* noisy m = b - <a, s> (lwe.rs:139-162) and the bool decode (evaluator.rs:243-256)
 * returns 0/1, or -1 when the decode is not 0 or 1 */
int orc_decrypt_bool(void *ev, const int32_t *s, const uint64_t *lwe);
/* multi-party decryption share of one party (multi_party.rs:57-87) */
uint64_t orc_mp_decryption_share(void *ev, void *rng, const int32_t *s_part,
                                 const uint64_t *lwe);
int orc_mp_aggregate_decrypt(void *ev, const uint64_t *lwe, const uint64_t *shares,
                             int parties);

#ifdef __cplusplus
}
#endif
#endif
