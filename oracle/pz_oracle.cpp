// pz_oracle.cpp -- CPU oracle for phantom-zone's server-side gate bootstrap.
//
// TEST INFRASTRUCTURE ONLY (see pz_oracle.h): a restatement of the reference
// Rust path used as the checker of the CUDA product and as the CPU baseline.
// Every function cites the reference file:line it follows.  Arithmetic is
// u64 wrapping / unsigned __int128 / IEEE double exactly where the Rust is.

#include "pz_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <thread>
#include <vector>

namespace {

typedef uint64_t u64;
typedef uint32_t u32;
typedef unsigned __int128 u128;

// ---------------------------------------------------------------------------
// Parameter sets: src/bool/parameters.rs:526-726 (I_2P_LB_SR ... SP_TEST).
// ---------------------------------------------------------------------------
struct Param {
  u64 rlwe_q, lwe_q;
  u32 br_q, rlwe_n, lwe_n;
  u32 lwe_logb, lwe_d;
  u32 rlrg_logb, d_a, d_b;
  u32 auto_logb, auto_d;
  u32 g, w;
  u32 lwe_gauss;  // SecretKeyDistribution::ErrorDistribution for the LWE secret
  u32 variant;    // 0 single, 1 interactive, 2 non-interactive
  u32 rgrg_logb, rgrg_d_a, rgrg_d_b;  // rgrg_decomposer_params (0: none)
};

const u64 Q54 = 18014398509404161ULL;
const Param PARAMS[ORC_NUM_PARAMS] = {
    // I_2P_LB_SR  parameters.rs:526-548
    {Q54, 1ULL << 15, 1u << 11, 1u << 11, 580, 1, 12, 17, 1, 1, 24, 1, 5, 10, 0, 1, 7, 6, 5},
    // I_4P        parameters.rs:550-572
    {Q54, 1ULL << 16, 1u << 11, 1u << 11, 620, 1, 13, 17, 1, 1, 24, 1, 5, 10, 0, 1, 6, 7, 6},
    // I_8P        parameters.rs:574-596
    {Q54, 1ULL << 17, 1u << 12, 1u << 11, 660, 1, 14, 17, 1, 1, 24, 1, 5, 10, 0, 1, 5, 9, 8},
    // NI_2P       parameters.rs:598-623 (LWE secret from the error distribution)
    {Q54, 1ULL << 16, 1u << 12, 1u << 11, 520, 1, 13, 17, 1, 1, 24, 1, 5, 10, 1, 2, 4, 10, 9},
    // NI_4P_HB_FR parameters.rs:625-650
    {Q54, 1ULL << 16, 1u << 11, 1u << 11, 620, 1, 13, 17, 1, 1, 24, 1, 5, 10, 0, 2, 3, 13, 12},
    // NI_4P_LB_SR parameters.rs:652-677
    {Q54, 1ULL << 16, 1u << 12, 1u << 11, 620, 1, 13, 17, 1, 1, 24, 1, 5, 10, 0, 2, 4, 10, 9},
    // NI_8P       parameters.rs:679-704
    {Q54, 1ULL << 17, 1u << 12, 1u << 11, 660, 1, 14, 17, 1, 1, 24, 1, 5, 10, 0, 2, 2, 20, 18},
    // SP_TEST_BOOL_PARAMS parameters.rs:706-726 (the only set with d > 1)
    {268369921ULL, 1ULL << 16, 1u << 9, 1u << 9, 100, 4, 4, 7, 4, 4, 7, 4, 5, 5, 1, 0, 0, 0, 0},
};

inline int clz64(u64 v) { return v ? __builtin_clzll(v) : 64; }

// utils.rs:230-237 log2: exact for powers of two, else bit length.
inline u32 log2_ref(u64 v) {
  if ((v & (v - 1)) == 0) return 63 - clz64(v);
  return 64 - clz64(v);
}

inline u64 reverse_bits64(u64 v) {
  u64 r = 0;
  for (int i = 0; i < 64; i++) { r = (r << 1) | (v & 1); v >>= 1; }
  return r;
}

// utils.rs:145-165 mod_exponent; :167-169 mod_inverse (Fermat).
u64 mod_exponent(u64 a, u64 b, u64 q) {
  u64 acc = a, out = 1;
  while (b != 0) {
    if (b & 1) out = (u64)(((u128)acc * out) % q);
    acc = (u64)(((u128)acc * acc) % q);
    b >>= 1;
  }
  return out;
}
u64 mod_inverse(u64 a, u64 q) { return mod_exponent(a, q - 2, q); }

// ---------------------------------------------------------------------------
// backend/modulus_u64.rs: ModularOpsU64.
// ---------------------------------------------------------------------------
struct ModU64 {
  u64 q, q_twice;
  u32 logq, alpha;
  u128 mu;
  explicit ModU64(u64 q_ = 2) { init(q_); }
  void init(u64 q_) {  // modulus_u64.rs:23-42
    q = q_;
    q_twice = q << 1;
    logq = 64 - clz64(q + 1);
    mu = ((u128)1 << (logq * 2 + 3)) / (u128)q;
    alpha = logq + 3;
  }
  u64 add(u64 a, u64 b) const {  // :46-55 add_mod_fast
    u64 o = a + b;
    if (o >= q) o -= q;
    return o;
  }
  u64 sub(u64 a, u64 b) const {  // :68-77 sub_mod_fast
    return a >= b ? a - b : (q + a) - b;
  }
  u64 neg(u64 a) const { return q - a; }  // :147-149 (not reduced: neg(0) = q)
  u64 mul(u64 a, u64 b) const {           // :106-129 mul_mod_fast (Barrett)
    u128 ab = (u128)a * b;
    u128 tmp = ab >> (logq - 2);
    u128 k = (tmp * mu) >> (alpha + 2);
    u128 kq = k * (u128)q;
    u64 out = (u64)(ab - kq);
    if (out >= q) out -= q;
    return out;
  }
};

// utils.rs:35-47 ShoupMul.
inline u64 shoup_repr(u64 v, u64 q) { return (u64)(((u128)v << 64) / q); }
inline u64 shoup_mul(u64 a, u64 b, u64 b_shoup, u64 q) {
  return b * a - q * (u64)(((u128)b_shoup * a) >> 64);
}

// modulus_u64.rs:231-264 shoup_matrix_fma: out += sum_r a[r] * b[r], lazily in [0, 2q).
void shoup_matrix_fma(u64 q, u64 *out, const u64 *const *a, const u64 *const *a_shoup,
                      const u64 *const *b, size_t rows, size_t n) {
  const u64 q_twice = q << 1;
  for (size_t r = 0; r < rows; r++) {
    for (size_t i = 0; i < n; i++) {
      u64 quotient = (u64)(((u128)a_shoup[r][i] * b[r][i]) >> 64);
      u64 v = a[r][i] * b[r][i] + out[i];
      v = v - q * quotient;
      if (v >= q_twice) v -= q_twice;
      out[i] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// ChaCha8 stream in the rand_chacha 0.3 layout (constants, 8 key words,
// 64-bit block counter, 64-bit stream id 0), consumed as a u32 word stream
// by rand_core 0.6's BlockRng (next_u64 = two words, low first).  Restated
// from the published ChaCha algorithm; agreement with the Rust crate's words
// is unpinned here (no Rust toolchain).
// ---------------------------------------------------------------------------
// The ChaCha block function with `rounds` rounds (RFC 8439 section 2.3 for
// 20) on a full 16-word input state: out = rounds(s) + s.
static inline u32 rotl32(u32 v, int c) { return (v << c) | (v >> (32 - c)); }
void chacha_core(const u32 s[16], int rounds, u32 out[16]) {
  u32 x[16];
  memcpy(x, s, sizeof x);
#define QR(a, b, c, d)                           \
  x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 16);  \
  x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 12);  \
  x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 8);   \
  x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 7);
  for (int r = 0; r < rounds / 2; r++) {
    QR(0, 4, 8, 12) QR(1, 5, 9, 13) QR(2, 6, 10, 14) QR(3, 7, 11, 15)
    QR(0, 5, 10, 15) QR(1, 6, 11, 12) QR(2, 7, 8, 13) QR(3, 4, 9, 14)
  }
#undef QR
  for (int i = 0; i < 16; i++) out[i] = x[i] + s[i];
}

// rand 0.8 UniformInt<u64>::new_inclusive(0, q-1) + sample (random.rs:93-110):
// one word v, accepted when lo64(v q) <= zone = MAX - (2^64 - q) mod q; the
// sample is hi64(v q).
inline bool uniform_word(u64 v, u64 q, u64 &sample) {
  const u64 zone = UINT64_MAX - ((0ull - q) % q);
  const u128 m = (u128)v * q;
  sample = (u64)(m >> 64);
  return (u64)m <= zone;
}

struct ChaCha8 {
  u32 key[8];
  u64 counter = 0;
  u32 buf[16];
  int idx = 16;
  explicit ChaCha8(const uint8_t seed[32]) {
    for (int i = 0; i < 8; i++)
      key[i] = (u32)seed[4 * i] | ((u32)seed[4 * i + 1] << 8) | ((u32)seed[4 * i + 2] << 16) |
               ((u32)seed[4 * i + 3] << 24);
  }
  void block() {
    u32 s[16];
    s[0] = 0x61707865u; s[1] = 0x3320646eu; s[2] = 0x79622d32u; s[3] = 0x6b206574u;
    for (int i = 0; i < 8; i++) s[4 + i] = key[i];
    s[12] = (u32)counter; s[13] = (u32)(counter >> 32); s[14] = 0; s[15] = 0;
    chacha_core(s, 8, buf);
    counter++;
    idx = 0;
  }
  u32 next_u32() {
    if (idx >= 16) block();
    return buf[idx++];
  }
  u64 next_u64() {
    u64 lo = next_u32();
    u64 hi = next_u32();
    return lo | (hi << 32);
  }
  // rand 0.8 UniformInt<u64>::new_inclusive(0, q-1) + sample (widening
  // multiply with rejection zone), random.rs:93-110.
  u64 uniform_mod(u64 q) {
    for (;;) {
      u64 sample;
      if (uniform_word(next_u64(), q, sample)) return sample;
    }
  }
  // Uniform::new(0, m) for usize (exclusive upper bound).
  u64 uniform_below(u64 m) { return uniform_mod(m); }
  // N(0, 3.19) by Box-Muller (client-side error sampling; the reference uses
  // rand_distr's ziggurat -- error words are not part of any parity claim).
  double gaussian() {
    double u1 = ((next_u64() >> 11) + 1) * (1.0 / 9007199254740993.0);
    double u2 = (next_u64() >> 11) * (1.0 / 9007199254740992.0);
    return 3.19 * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

// parameters.rs:482-493 map_element_from_f64 (round half away from zero).
inline u64 map_from_f64(u64 q, double v) {
  v = std::round(v);
  u64 ve = (u64)std::fabs(v);
  if (v < 0.0) return (q - 1) - ve + 1;
  return ve;
}
inline u64 map_from_i64(u64 q, int64_t v) {
  u64 ve = (u64)(v < 0 ? -v : v);
  return v < 0 ? q - ve : ve;
}

// utils.rs:75-110 fill_random_ternary_secret_with_hamming_weight.
void ternary_secret(ChaCha8 &rng, int32_t *out, size_t size, size_t hw) {
  std::vector<uint8_t> bytes((hw + 7) / 8);
  for (auto &b : bytes) b = (uint8_t)rng.next_u32();  // fill_bytes consumes u32 words
  std::vector<size_t> idx(size);
  for (size_t i = 0; i < size; i++) idx[i] = i;
  for (size_t i = 0; i < size; i++) out[i] = 0;
  size_t bit = 0, byte = 0;
  for (size_t i = 0; i < hw; i++) {
    size_t s = (size_t)rng.uniform_below(idx.size());
    int curr = (bytes[byte] >> bit) & 1;
    out[idx[s]] = curr ? 1 : -1;
    idx[s] = idx.back();
    idx.pop_back();
    if (bit == 7) { bit = 0; byte++; } else { bit++; }
  }
}

// ---------------------------------------------------------------------------
// ntt.rs: Harvey butterflies and the negacyclic NTT.
// ---------------------------------------------------------------------------
// ntt.rs:31-49
inline void fwd_bf_4q(u64 &x, u64 &y, u64 w, u64 ws, u64 q, u64 q2) {
  if (x >= q2) x -= q2;
  u64 t = shoup_mul(y, w, ws, q);
  u64 ox = x + t, oy = x + q2 - t;
  x = ox; y = oy;
}
// ntt.rs:51-75
inline void fwd_bf_2q(u64 &x, u64 &y, u64 w, u64 ws, u64 q, u64 q2) {
  if (x >= q2) x -= q2;
  u64 t = shoup_mul(y, w, ws, q);
  u64 ox = x + t, oy = x - t;
  x = std::min(ox, ox - q2);
  y = std::min(oy, oy + q2);
}
// ntt.rs:84-104
inline void inv_bf_2q(u64 &x, u64 &y, u64 w, u64 ws, u64 q, u64 q2) {
  u64 xd = x + y;
  if (xd >= q2) xd -= q2;
  u64 t = x + q2 - y;
  y = shoup_mul(t, w, ws, q);
  x = xd;
}

struct Ntt {  // NttBackendU64, ntt.rs:310-442
  u64 q = 0, q2 = 0, n_inv = 0, n_inv_s = 0, psi = 0;
  size_t n = 0;
  std::vector<u64> psi_bo, psi_inv_bo, psi_bo_s, psi_inv_bo_s;

  void init(u64 q_, size_t n_) {  // ntt.rs:323-385
    q = q_; q2 = 2 * q; n = n_;
    uint8_t zero[32] = {0};
    ChaCha8 rng(zero);
    psi = find_primitive_root(q, 2 * n, rng);
    u64 psi_inv = mod_inverse(psi, q);
    ModU64 m(q);
    std::vector<u64> pw(n), pwi(n);
    u64 rp = 1, rpi = 1;
    for (size_t i = 0; i < n; i++) {
      pw[i] = rp; pwi[i] = rpi;
      rp = m.mul(rp, psi); rpi = m.mul(rpi, psi_inv);
    }
    psi_bo.assign(n, 0); psi_inv_bo.assign(n, 0);
    int shift = clz64(n) + 1;
    for (size_t i = 0; i < n; i++) {
      size_t bo = (size_t)(reverse_bits64(i) >> shift);
      psi_bo[bo] = pw[i]; psi_inv_bo[bo] = pwi[i];
    }
    psi_bo_s.resize(n); psi_inv_bo_s.resize(n);
    for (size_t i = 0; i < n; i++) {
      psi_bo_s[i] = shoup_repr(psi_bo[i], q);
      psi_inv_bo_s[i] = shoup_repr(psi_inv_bo[i], q);
    }
    n_inv = mod_inverse((u64)n, q);
    n_inv_s = shoup_repr(n_inv, q);
  }
  // ntt.rs:283-307 find_primitive_root
  static u64 find_primitive_root(u64 q, u64 n, ChaCha8 &rng) {
    u64 t = (q - 1) / n;
    for (int i = 0; i < 100; i++) {
      u64 omega = rng.next_u64() % q;
      omega = mod_exponent(omega, t, q);
      if (mod_exponent(omega, n >> 1, q) == 1) continue;
      return omega;
    }
    throw std::runtime_error("no primitive root");
  }
  // ntt.rs:110-180 (lazy: output in [0,2q); full: [0,q))
  void forward(u64 *a, bool lazy) const {
    size_t t = n, m = 1;
    while (m < n) {
      t >>= 1;
      const u64 *w = &psi_bo[m], *ws = &psi_bo_s[m];
      if (t == 1) {
        for (size_t i = 0; i < n / 2; i++) {
          u64 x = a[2 * i], y = a[2 * i + 1];
          fwd_bf_2q(x, y, w[i], ws[i], q, q2);
          if (!lazy) { x = std::min(x, x - q); y = std::min(y, y - q); }
          a[2 * i] = x; a[2 * i + 1] = y;
        }
      } else {
        for (size_t i = 0; i < m; i++) {
          u64 *blk = a + 2 * i * t;
          for (size_t j = 0; j < t; j++) fwd_bf_4q(blk[j], blk[j + t], w[i], ws[i], q, q2);
        }
      }
      m <<= 1;
    }
  }
  // ntt.rs:187-278 (n^{-1} folded into the last stage; lazy output in [0,2q))
  void backward(u64 *a, bool lazy) const {
    size_t m = n >> 1, t = 1;
    while (m > 0) {
      if (m == 1) {
        for (size_t j = 0; j < t; j++) {
          u64 x = a[j], y = a[j + t];
          inv_bf_2q(x, y, psi_inv_bo[1], psi_inv_bo_s[1], q, q2);
          x = shoup_mul(x, n_inv, n_inv_s, q);
          y = shoup_mul(y, n_inv, n_inv_s, q);
          if (!lazy) { x = std::min(x, x - q); y = std::min(y, y - q); }
          a[j] = x; a[j + t] = y;
        }
      } else {
        const u64 *w = &psi_inv_bo[m], *ws = &psi_inv_bo_s[m];
        for (size_t i = 0; i < m; i++) {
          u64 *blk = a + 2 * i * t;
          for (size_t j = 0; j < t; j++) inv_bf_2q(blk[j], blk[j + t], w[i], ws[i], q, q2);
        }
      }
      t *= 2;
      m >>= 1;
    }
  }
};

// ---------------------------------------------------------------------------
// decomposer.rs: DefaultDecomposer (signed gadget decomposition).
// ---------------------------------------------------------------------------
struct Decomposer {
  u64 q = 0, b = 0, b_mask = 0, bby2 = 0;
  u32 logq = 0, logb = 0, d = 0, ignore_bits = 0;
  void init(u64 q_, u32 logb_, u32 d_) {  // decomposer.rs:158-178
    q = q_; logb = logb_; d = d_;
    logq = log2_ref(q);
    if (logq < logb * d) throw std::runtime_error("decomposer: logq < logb*d");
    ignore_bits = logq - logb * d;
    b = 1ULL << logb; b_mask = b - 1; bby2 = 1ULL << (logb - 1);
  }
  // decomposer.rs:13-21
  u64 gadget(u32 i) const { return 1ULL << (logb * i + ignore_bits); }
  // decomposer.rs:302-309
  static u64 round_value(u64 value, u32 ib) {
    if (ib == 0) return value;
    u64 ignored_msb = (value & ((1ULL << ib) - 1)) >> (ib - 1);
    return (value >> ib) + ignored_msb;
  }
  // decomposer.rs:217-234 decompose_iter + :261-300 next() (branch-free form)
  void decompose(u64 value, u64 *out) const {
    if (value >= (q >> 1)) value = ~(q - value) + 1;  // wrapping, as in release builds
    value = round_value(value, ignore_bits);
    for (u32 j = 0; j < d; j++) {
      u64 k = value & b_mask;
      value = (value - k) >> logb;
      bool cb = k > bby2 || (k == bby2 && (value & 1) == 1);
      u64 carry = cb ? 1 : 0;
      u64 neg_carry = 0 - carry;
      value = value + carry;
      out[j] = (neg_carry & q) + k - (carry << logb);
    }
  }
};

// rgsw/keygen.rs:16-41 generate_auto_map
void generate_auto_map(size_t ring_size, int64_t k, std::vector<u32> &index,
                       std::vector<uint8_t> &sign) {
  if ((k & 1) == 0) throw std::runtime_error("auto must be odd");
  u64 kk = k < 0 ? (u64)(2 * ring_size) - ((u64)(-k) % (2 * ring_size)) : (u64)k;
  index.resize(ring_size); sign.resize(ring_size);
  for (size_t i = 0; i < ring_size; i++) {
    u64 to = (i * kk) % (2 * ring_size);
    bool s = true;
    if (to >= ring_size) { to -= ring_size; s = false; }
    index[i] = (u32)to; sign[i] = s;
  }
}

struct Eval;

// Eval-domain server key with Shoup companions (keys.rs:687-781, 1193-1220).
struct Key {
  size_t n_lwe, rgsw_rows, auto_rows, N;
  std::vector<u64> rgsw, rgsw_s;      // [n][rows][N] eval domain
  std::vector<u64> autos, autos_s;    // [w+1][auto_rows][N]
  std::vector<u64> ksk;               // [d_ks N][n+1] mod q_ks
  const u64 *rgsw_row(size_t i, size_t r) const { return &rgsw[(i * rgsw_rows + r) * N]; }
  const u64 *rgsw_row_s(size_t i, size_t r) const { return &rgsw_s[(i * rgsw_rows + r) * N]; }
  const u64 *auto_row(size_t k, size_t r) const { return &autos[(k * auto_rows + r) * N]; }
  const u64 *auto_row_s(size_t k, size_t r) const { return &autos_s[(k * auto_rows + r) * N]; }
};

// BoolEvaluator state (evaluator.rs:651-784) + per-thread scratch.
struct Eval {
  Param p;
  size_t N, n;
  u64 Q;
  ModU64 rmod;
  u64 ks_mask;  // ModulusPowerOf2 mask (power_of_2.rs:95-104)
  Ntt ntt;
  Decomposer dec_lwe, dec_a, dec_b, dec_auto;
  Decomposer dec_ni;      // non_interactive_ui_to_s_key_switch_decomposer (NI sets only)
  Decomposer dec_rgrg_a, dec_rgrg_b;  // rgsw_rgsw_decomposer (parameters.rs:276-298)
  std::vector<u32> dlog;  // g_k_dlog_map
  u32 emb;
  std::vector<std::vector<u64>> test_vec;  // per gate
  std::vector<std::vector<u32>> auto_idx;  // [w+1][N]
  std::vector<std::vector<uint8_t>> auto_sign;
  u64 qby4, true_el, false_el;

  explicit Eval(int pid) : p(PARAMS[pid]) {
    N = p.rlwe_n; n = p.lwe_n; Q = p.rlwe_q;
    rmod.init(Q);
    ks_mask = p.lwe_q - 1;
    ntt.init(Q, N);
    dec_lwe.init(p.lwe_q, p.lwe_logb, p.lwe_d);
    dec_a.init(Q, p.rlrg_logb, p.d_a);
    dec_b.init(Q, p.rlrg_logb, p.d_b);
    dec_auto.init(Q, p.auto_logb, p.auto_d);
    // parameters.rs:616-697: ui_to_s key switch (logb 1, d 50) of the NI sets
    if (p.variant == 2) dec_ni.init(Q, 1, 50);
    if (p.rgrg_logb) {
      dec_rgrg_a.init(Q, p.rgrg_logb, p.rgrg_d_a);
      dec_rgrg_b.init(Q, p.rgrg_logb, p.rgrg_d_b);
    }
    // evaluator.rs:664-673 dlog map over Z*_{br_q} = +-g^k
    u32 q = p.br_q;
    dlog.assign(q, 0);
    for (u32 i = 0; i < q / 4; i++) {
      u64 v = mod_exponent(p.g, i, q);
      dlog[v] = i;
      dlog[q - v] = i + q / 4;
    }
    emb = (2 * p.rlwe_n) / q;  // evaluator.rs:675
    // evaluator.rs:231-242, 224-230: Q/8, -Q/8, Q/4
    true_el = Q >> 3;
    false_el = (Q - 1) - true_el + 1;
    qby4 = Q >> 2;
    // evaluator.rs:688-726 test vectors, pre-permuted by X -> X^{-g}
    std::vector<u32> ami; std::vector<uint8_t> ams;
    u32 qby2 = q >> 1, qby8 = q >> 3;
    generate_auto_map(qby2, -(int64_t)p.g, ami, ams);
    auto init_tv = [&](u32 part, u64 before, u64 after) {
      std::vector<u64> tv(qby2), out(qby2);
      for (u32 i = 0; i < qby2; i++) tv[i] = i < part ? before : after;
      for (u32 i = 0; i < qby2; i++) out[ami[i]] = ams[i] ? tv[i] : rmod.neg(tv[i]);
      return out;
    };
    test_vec.resize(6);
    test_vec[ORC_AND] = init_tv(3 * qby8, false_el, true_el);
    test_vec[ORC_NAND] = init_tv(3 * qby8, true_el, false_el);
    test_vec[ORC_OR] = init_tv(qby8, false_el, true_el);
    test_vec[ORC_NOR] = init_tv(qby8, true_el, false_el);
    test_vec[ORC_XOR] = init_tv(qby8, false_el, true_el);
    test_vec[ORC_XNOR] = init_tv(qby8, true_el, false_el);
    // evaluator.rs:728-743 auto maps [-g, g^1, ..., g^w] over the N-ring
    auto_idx.resize(p.w + 1); auto_sign.resize(p.w + 1);
    for (u32 i = 0; i <= p.w; i++) {
      int64_t el = i == 0 ? -(int64_t)p.g : (int64_t)(mod_exponent(p.g, i, 1ULL << 62) % q);
      generate_auto_map(N, el, auto_idx[i], auto_sign[i]);
    }
  }
  // pbs.rs:416-420 (f64 exactly as the Rust)
  static size_t mod_switch_odd(double v, double from_q, double to_q) {
    size_t odd = (size_t)std::floor((v * to_q) / from_q);
    return odd + ((odd & 1) ^ 1);
  }
};

// Scratch of one evaluator (ScratchMemory, evaluator.rs:174-207).
struct Scratch {
  std::vector<u64> dec;  // max(d_a, d_b, d_auto) x N
  std::vector<u64> tmp;  // 2 x N
  std::vector<u64> lwe;  // n + 1
  explicit Scratch(const Eval &e) {
    size_t d = std::max<size_t>(std::max(e.p.d_a, e.p.d_b), e.p.auto_d);
    dec.assign(d * e.N, 0); tmp.assign(2 * e.N, 0); lwe.assign(e.n + 1, 0);
  }
};

// runtime.rs:382-399 decompose_r
void decompose_r(const Decomposer &dcp, const u64 *r, u64 *out, size_t N) {
  u64 dig[64];
  for (size_t i = 0; i < N; i++) {
    dcp.decompose(r[i], dig);
    for (u32 j = 0; j < dcp.d; j++) out[j * N + i] = dig[j];
  }
}

// runtime.rs:754-855 rlwe_by_rgsw_shoup (shoup=true) and :651-747 rlwe_by_rgsw.
void rlwe_by_rgsw(const Eval &e, const Key &k, Scratch &sc, u64 *rlwe, size_t si, bool trivial,
                  bool shoup) {
  const size_t N = e.N, da = e.p.d_a, db = e.p.d_b;
  u64 *ta = &sc.tmp[0], *tb = &sc.tmp[N];
  std::fill(sc.tmp.begin(), sc.tmp.end(), 0);
  const u64 *ap[64], *aps[64], *bp[64];
  auto mac = [&](u64 *out, size_t row0, size_t rows) {
    if (shoup) {
      for (size_t j = 0; j < rows; j++) {
        ap[j] = k.rgsw_row(si, row0 + j); aps[j] = k.rgsw_row_s(si, row0 + j); bp[j] = &sc.dec[j * N];
      }
      shoup_matrix_fma(e.Q, out, ap, aps, bp, rows, N);
    } else {  // poly_fma_routine, runtime.rs:363-372 (elwise_fma_mut: add(o, mul(a,b)))
      for (size_t j = 0; j < rows; j++) {
        const u64 *a = k.rgsw_row(si, row0 + j), *b = &sc.dec[j * N];
        for (size_t i = 0; i < N; i++) out[i] = e.rmod.add(out[i], e.rmod.mul(b[i], a[i]));
      }
    }
  };
  if (!trivial) {
    decompose_r(e.dec_a, rlwe, sc.dec.data(), N);
    for (size_t j = 0; j < da; j++) e.ntt.forward(&sc.dec[j * N], shoup);
    mac(ta, 0, da);   // A(-sm)
    mac(tb, da, da);  // B(-sm)
  }
  decompose_r(e.dec_b, rlwe + N, sc.dec.data(), N);
  for (size_t j = 0; j < db; j++) e.ntt.forward(&sc.dec[j * N], shoup);
  mac(ta, 2 * da, db);       // A(m)
  mac(tb, 2 * da + db, db);  // B(m)
  e.ntt.backward(ta, false);
  e.ntt.backward(tb, false);
  memcpy(rlwe, ta, N * 8);
  memcpy(rlwe + N, tb, N * 8);
}

// runtime.rs:530-643 rlwe_auto_shoup (shoup=true) and :412-522 rlwe_auto.
void rlwe_auto(const Eval &e, const Key &k, Scratch &sc, u64 *rlwe, size_t ak, bool trivial,
               bool shoup) {
  const size_t N = e.N, d = e.p.auto_d;
  const std::vector<u32> &idx = e.auto_idx[ak];
  const std::vector<uint8_t> &sgn = e.auto_sign[ak];
  u64 *a = rlwe, *b = rlwe + N;
  if (!trivial) {
    u64 *ta = &sc.tmp[0], *tb = &sc.tmp[N];
    std::fill(sc.tmp.begin(), sc.tmp.end(), 0);
    u64 dig[64];
    for (size_t i = 0; i < N; i++) {
      u64 el = sgn[i] ? a[i] : e.rmod.neg(a[i]);
      e.dec_auto.decompose(el, dig);
      for (size_t j = 0; j < d; j++) sc.dec[j * N + idx[i]] = dig[j];
    }
    for (size_t j = 0; j < d; j++) e.ntt.forward(&sc.dec[j * N], shoup);
    const u64 *ap[64], *aps[64], *bp[64];
    if (shoup) {
      for (size_t j = 0; j < d; j++) {
        ap[j] = k.auto_row(ak, j); aps[j] = k.auto_row_s(ak, j); bp[j] = &sc.dec[j * N];
      }
      shoup_matrix_fma(e.Q, ta, ap, aps, bp, d, N);
      for (size_t j = 0; j < d; j++) { ap[j] = k.auto_row(ak, d + j); aps[j] = k.auto_row_s(ak, d + j); }
      shoup_matrix_fma(e.Q, tb, ap, aps, bp, d, N);
    } else {
      for (size_t j = 0; j < d; j++) {
        const u64 *ka = k.auto_row(ak, j), *kb = k.auto_row(ak, d + j), *x = &sc.dec[j * N];
        for (size_t i = 0; i < N; i++) {
          ta[i] = e.rmod.add(ta[i], e.rmod.mul(x[i], ka[i]));
          tb[i] = e.rmod.add(tb[i], e.rmod.mul(x[i], kb[i]));
        }
      }
    }
    e.ntt.backward(ta, false);
    e.ntt.backward(tb, false);
    for (size_t i = 0; i < N; i++) {
      if (!sgn[i]) tb[idx[i]] = e.rmod.sub(tb[idx[i]], b[i]);
      else tb[idx[i]] = e.rmod.add(tb[idx[i]], b[i]);
    }
    memcpy(a, ta, N * 8);
    memcpy(b, tb, N * 8);
  } else {
    u64 *row = &sc.dec[0];  // scratch_for_rlwe_auto_trivial_case
    for (size_t i = 0; i < N; i++) row[idx[i]] = sgn[i] ? b[i] : e.rmod.neg(b[i]);
    memcpy(b, row, N * 8);
  }
}

// lwe.rs:14-44 with ModulusPowerOf2 ops (power_of_2.rs:13-92).
void lwe_key_switch(const Eval &e, const Key &k, const u64 *in, u64 *out) {
  const size_t N = e.N, n = e.n, d = e.p.lwe_d;
  const u64 mask = e.ks_mask;
  for (size_t c = 0; c <= n; c++) out[c] = 0;
  u64 dig[64];
  for (size_t i = 0; i < N; i++) {
    e.dec_lwe.decompose(in[1 + i], dig);
    for (size_t j = 0; j < d; j++) {
      const u64 *row = &k.ksk[(i * d + j) * (n + 1)];
      const u64 c = dig[j];
      for (size_t col = 0; col <= n; col++) out[col] = (out[col] + row[col] * c) & mask;
    }
  }
  out[0] = (out[0] + in[0]) & mask;
}

// pbs.rs:423-449 sample_extract
void sample_extract(const Eval &e, const u64 *rlwe, u64 *lwe, size_t index) {
  const size_t N = e.N;
  u64 *to = lwe + 1;
  const u64 *from = rlwe;
  for (size_t i = 0; i < index + 1; i++) to[i] = from[index - i];
  for (size_t i = index + 1; i < N; i++) to[i] = e.rmod.neg(from[N + index - i]);
  lwe[0] = rlwe[N + index];
}

// pbs.rs:454-482 monomial_mul
void monomial_mul(const Eval &e, const u64 *p_in, u64 *p_out, size_t mon_exp, bool mon_sign,
                  size_t ring_size) {
  for (size_t i = 0; i < ring_size; i++) {
    size_t to = i + mon_exp;
    bool s = mon_sign;
    if (to >= ring_size) { to -= ring_size; s = !s; }
    p_out[to] = s ? p_in[i] : e.rmod.neg(p_in[i]);
  }
}

// pbs.rs:240-414 blind_rotation; returns the number of non-trivial autos.
int blind_rotation(const Eval &e, const Key &k, Scratch &sc, u64 *rlwe,
                   const std::vector<std::vector<u32>> &gk_to_si) {
  bool is_trivial = true;
  int autos = 0;
  const size_t q = e.p.br_q, q_by_4 = q >> 2, w = e.p.w;
  auto do_rgsw = [&](size_t bucket) {
    for (u32 s : gk_to_si[bucket]) {
      rlwe_by_rgsw(e, k, sc, rlwe, s, is_trivial, true);
      is_trivial = false;
    }
  };
  auto do_auto = [&](size_t v) {
    if (!is_trivial) autos++;
    rlwe_auto(e, k, sc, rlwe, v, is_trivial, true);
  };
  // -(g^k), pbs.rs:276-321
  size_t v = 0;
  for (size_t i = q_by_4 - 1; i >= 1; i--) {
    do_rgsw(q_by_4 + i);
    v += 1;
    if (!gk_to_si[q_by_4 + i - 1].empty() || v == w || i == 1) { do_auto(v); v = 0; }
  }
  // -(g^0), pbs.rs:323-355
  do_rgsw(q_by_4);
  do_auto(0);
  // +(g^k), pbs.rs:357-396
  v = 0;
  for (size_t i = q_by_4 - 1; i >= 1; i--) {
    do_rgsw(i);
    v += 1;
    if (!gk_to_si[i - 1].empty() || v == w || i == 1) { do_auto(v); v = 0; }
  }
  // +(g^0), pbs.rs:398-412
  do_rgsw(0);
  return autos;
}

// pbs.rs:104-233 pbs
int pbs(const Eval &e, const Key &k, Scratch &sc, const u64 *test_vec, u64 *lwe_in,
        u64 *ks_out, u64 *rlwe_out) {
  const size_t N = e.N, br_q = e.p.br_q;
  const double rlwe_qf = (double)e.Q, lwe_qf = (double)e.p.lwe_q, br_qf = (double)br_q;
  // moddown Q -> q_ks, pbs.rs:128-132
  for (size_t i = 0; i <= N; i++) {
    double v = std::round(((double)lwe_in[i] * lwe_qf) / rlwe_qf);
    lwe_in[i] = (u64)v;
  }
  // key switch, pbs.rs:136-143
  u64 *ks = sc.lwe.data();
  lwe_key_switch(e, k, lwe_in, ks);
  if (ks_out) memcpy(ks_out, ks, (e.n + 1) * 8);
  // odd moddown + dlog buckets, pbs.rs:147-161
  std::vector<std::vector<u32>> g_k_si(br_q >> 1);
  for (size_t i = 0; i < e.n; i++) {
    size_t odd = Eval::mod_switch_odd((double)ks[1 + i], lwe_qf, br_qf);
    g_k_si[e.dlog[odd]].push_back((u32)i);
  }
  // b and trivial test RLWE, pbs.rs:163-211
  size_t g = e.p.g;
  size_t g_times_b = (g * Eval::mod_switch_odd((double)ks[0], lwe_qf, br_qf)) % br_q;
  size_t br_qby2 = br_q >> 1;
  bool sign = true;
  size_t exp = g_times_b;
  if (exp > br_qby2) { exp -= br_qby2; sign = false; }
  std::vector<u64> rlwe(2 * N, 0);
  if (e.emb == 1) {
    monomial_mul(e, test_vec, &rlwe[N], exp, sign, br_qby2);
  } else {
    monomial_mul(e, test_vec, lwe_in, exp, sign, br_qby2);  // lwe_in[..br_q/2] as scratch
    for (size_t i = 0; i < br_qby2; i++) rlwe[N + e.emb * i] = lwe_in[i];
  }
  int autos = blind_rotation(e, k, sc, rlwe.data(), g_k_si);
  if (rlwe_out) memcpy(rlwe_out, rlwe.data(), 2 * N * 8);
  sample_extract(e, rlwe.data(), lwe_in, 0);  // pbs.rs:232
  return autos;
}

// evaluator.rs:2118-2123 and :2126-2133 (xor/xnor add no Q/4)
void gate_prelude(const Eval &e, int gate, u64 *c0, const u64 *c1) {
  const size_t L = e.N + 1;
  if (gate == ORC_XOR || gate == ORC_XNOR) {
    for (size_t i = 0; i < L; i++) c0[i] = e.rmod.sub(c0[i], c1[i]);
    for (size_t i = 0; i < L; i++) c0[i] = e.rmod.add(c0[i], c0[i]);
  } else {
    for (size_t i = 0; i < L; i++) c0[i] = e.rmod.add(c0[i], c1[i]);
    c0[0] = e.rmod.add(c0[0], e.qby4);
  }
}

void gate(const Eval &e, const Key &k, Scratch &sc, int g, u64 *c0, const u64 *c1) {
  gate_prelude(e, g, c0, c1);
  pbs(e, k, sc, e.test_vec[g].data(), c0, nullptr, nullptr);
}

// ---------------------------------------------------------------------------
// shortint/ops.rs restated sequentially: every gate bootstraps immediately,
// in the reference's order, through gate() above.  A ciphertext is a
// std::vector<u64> of N+1 words.
// ---------------------------------------------------------------------------
typedef std::vector<u64> Ct;
struct SEval {
  const Eval &e;
  const Key *k;  // null: a dry run that only tallies the gates (no bootstrap)
  Scratch sc;
  uint64_t *tally = nullptr;  // gates issued, by gate code
  SEval(const Eval &e_, const Key *k_) : e(e_), k(k_), sc(e_) {}
  Ct g(int t, const Ct &a, const Ct &b) {  // gate(a, b): BooleanGates::* (evaluator.rs:2252-2316)
    if (tally) tally[t]++;
    Ct out = a;
    if (k) gate(e, *k, sc, t, out.data(), b.data());
    return out;
  }
  Ct not_(const Ct &a) {  // evaluator.rs:2318-2322
    Ct out = a;
    for (auto &v : out) v = e.rmod.neg(v);
    return out;
  }
};
// ops.rs:5-14
Ct s_half_adder(SEval &s, Ct &a, const Ct &b) {
  Ct carry = s.g(ORC_AND, a, b);
  a = s.g(ORC_XOR, a, b);
  return carry;
}
// ops.rs:16-44
Ct s_full_adder_plain_carry_in(SEval &s, Ct &a, const Ct &b, bool carry_in) {
  Ct a_and_b = s.g(ORC_AND, a, b);
  a = s.g(ORC_XOR, a, b);
  if (carry_in) a_and_b = s.g(ORC_OR, a_and_b, a);
  if (carry_in) a = s.not_(a);
  return a_and_b;
}
// ops.rs:46-59
Ct s_full_adder(SEval &s, Ct &a, const Ct &b, const Ct &carry_in) {
  Ct a_and_b = s.g(ORC_AND, a, b);
  a = s.g(ORC_XOR, a, b);
  Ct a_xor_b_and_c = s.g(ORC_AND, a, carry_in);
  a_and_b = s.g(ORC_OR, a_and_b, a_xor_b_and_c);
  a = s.g(ORC_XOR, a, carry_in);
  return a_and_b;
}
// ops.rs:61-91
void s_adder(SEval &s, std::vector<Ct> &a, const std::vector<Ct> &b, bool carry_in, Ct &cl, Ct &cll) {
  const size_t n = a.size();
  Ct carry = !carry_in ? s_half_adder(s, a[0], b[0]) : s_full_adder_plain_carry_in(s, a[0], b[0], true);
  for (size_t i = 1; i + 2 < n; i++) carry = s_full_adder(s, a[i], b[i], carry);
  cll = s_full_adder(s, a[n - 2], b[n - 2], carry);
  cl = s_full_adder(s, a[n - 1], b[n - 1], cll);
}
// ops.rs:143-187
std::vector<Ct> s_mul(SEval &s, const std::vector<Ct> &a, const std::vector<Ct> &b) {
  std::vector<Ct> carries, out;
  for (int i = 0; i < 8; i++) {
    if (i == 0) {
      out.push_back(s.g(ORC_AND, a[0], b[0]));
    } else if (i == 1) {
      Ct tmp0 = s.g(ORC_AND, a[1], b[0]);
      Ct tmp1 = s.g(ORC_AND, a[0], b[1]);
      carries.push_back(s_half_adder(s, tmp0, tmp1));
      out.push_back(tmp0);
    } else {
      Ct sum = s.g(ORC_AND, a[i], b[0]);
      Ct tmp = s.g(ORC_AND, a[i - 1], b[1]);
      carries[0] = s_full_adder(s, sum, tmp, carries[0]);
      for (int j = 2; j < i; j++) {
        tmp = s.g(ORC_AND, a[i - j], b[j]);
        carries[j - 1] = s_full_adder(s, sum, tmp, carries[j - 1]);
      }
      tmp = s.g(ORC_AND, a[0], b[i]);
      carries.push_back(s_half_adder(s, sum, tmp));
      out.push_back(sum);
    }
  }
  return out;
}
// ops.rs:189-259
void s_division(SEval &s, const std::vector<Ct> &a, const std::vector<Ct> &b, std::vector<Ct> &quot,
                std::vector<Ct> &rem) {
  const size_t n = a.size();
  std::vector<Ct> neg_b;
  for (auto &x : b) neg_b.push_back(s.not_(x));
  std::vector<Ct> remainder, quotient;
  for (size_t i = 0; i < n; i++) {
    remainder.push_back(a[n - 1 - i]);
    std::vector<Ct> subtract = remainder;
    Ct carry = s_full_adder_plain_carry_in(s, subtract[i], neg_b[0], true);
    for (size_t j = 1; j <= i; j++) carry = s_full_adder(s, subtract[i - j], neg_b[j], carry);
    for (size_t j = i + 1; j < n; j++) carry = s.g(ORC_AND, carry, neg_b[j]);
    Ct not_carry = s.not_(carry);
    for (size_t kk = 0; kk < remainder.size(); kk++) {
      subtract[kk] = s.g(ORC_AND, subtract[kk], carry);
      remainder[kk] = s.g(ORC_AND, remainder[kk], not_carry);
      remainder[kk] = s.g(ORC_OR, remainder[kk], subtract[kk]);
    }
    quotient.push_back(carry);
  }
  std::reverse(remainder.begin(), remainder.end());
  std::reverse(quotient.begin(), quotient.end());
  quot = quotient;
  rem = remainder;
}
// ops.rs:261-272
Ct s_is_zero(SEval &s, const std::vector<Ct> &a) {
  std::vector<Ct> na;
  for (auto &x : a) na.push_back(s.not_(x));
  Ct out = na[0];
  for (size_t i = 1; i < na.size(); i++) out = s.g(ORC_AND, out, na[i]);
  return out;
}
// ops.rs:274-287
Ct s_equality(SEval &s, const std::vector<Ct> &a, const std::vector<Ct> &b) {
  Ct out = s.g(ORC_XNOR, a[0], b[0]);
  for (size_t i = 1; i < a.size(); i++) {
    Ct e = s.g(ORC_XNOR, a[i], b[i]);
    out = s.g(ORC_AND, out, e);
  }
  return out;
}
// ops.rs:292-321, :341-356
Ct s_comparator(SEval &s, const std::vector<Ct> &a, const std::vector<Ct> &b) {
  const size_t n = a.size();
  Ct comp = s.not_(b[n - 1]);
  comp = s.g(ORC_AND, comp, a[n - 1]);
  Ct casc = s.g(ORC_XNOR, a[n - 1], b[n - 1]);
  Ct tmp = s.not_(b[n - 2]);
  tmp = s.g(ORC_AND, tmp, a[n - 2]);
  tmp = s.g(ORC_AND, tmp, casc);
  comp = s.g(ORC_OR, comp, tmp);
  for (size_t i = 2; i < n; i++) {
    Ct tmp_casc = s.g(ORC_XNOR, a[n - i], b[n - i]);
    casc = s.g(ORC_AND, casc, tmp_casc);
    Ct t = s.not_(b[n - 1 - i]);
    t = s.g(ORC_AND, t, a[n - 1 - i]);
    t = s.g(ORC_AND, t, casc);
    comp = s.g(ORC_OR, comp, t);
  }
  return comp;
}
// ops.rs:123-141
std::vector<Ct> s_mux(SEval &s, const Ct &sel, const std::vector<Ct> &t, const std::vector<Ct> &f) {
  Ct ns = s.not_(sel);
  std::vector<Ct> out;
  for (size_t i = 0; i < t.size(); i++) {
    Ct sa = s.g(ORC_AND, sel, t[i]);
    Ct sb = s.g(ORC_AND, ns, f[i]);
    out.push_back(s.g(ORC_OR, sa, sb));
  }
  return out;
}

}  // namespace

// ===========================================================================
// extern "C" surface
// ===========================================================================
extern "C" {

int orc_param_info_get(int pid, orc_param_info *o) {
  if (pid < 0 || pid >= ORC_NUM_PARAMS || !o) return -1;
  const Param &p = PARAMS[pid];
  o->rlwe_q = p.rlwe_q; o->lwe_q = p.lwe_q; o->br_q = p.br_q; o->rlwe_n = p.rlwe_n;
  o->lwe_n = p.lwe_n; o->lwe_logb = p.lwe_logb; o->lwe_d = p.lwe_d;
  o->rlrg_logb = p.rlrg_logb; o->rlrg_d_a = p.d_a; o->rlrg_d_b = p.d_b;
  o->auto_logb = p.auto_logb; o->auto_d = p.auto_d; o->g = p.g; o->w = p.w;
  o->lwe_secret_gaussian = p.lwe_gauss; o->variant = p.variant;
  o->embedding_factor = 2 * p.rlwe_n / p.br_q;
  o->rgsw_rows = 2 * p.d_a + 2 * p.d_b; o->auto_rows = 2 * p.auto_d;
  o->n_auto_keys = p.w + 1;
  // parameters.rs:616-697 non_interactive_ui_to_s_key_switch_decomposer (1, 50)
  o->ni_ks_logb = p.variant == 2 ? 1 : 0;
  o->ni_ks_d = p.variant == 2 ? 50 : 0;
  o->rgrg_logb = p.rgrg_logb; o->rgrg_d_a = p.rgrg_d_a; o->rgrg_d_b = p.rgrg_d_b;
  return 0;
}

void *orc_eval_new(int pid) {
  if (pid < 0 || pid >= ORC_NUM_PARAMS) return nullptr;
  return new Eval(pid);
}
void orc_eval_free(void *ev) { delete (Eval *)ev; }
uint64_t orc_eval_psi(void *ev) { return ((Eval *)ev)->ntt.psi; }
void orc_eval_tables(void *ev, uint64_t *psi_br, uint64_t *psi_inv_br, uint64_t *n_inv) {
  Eval &e = *(Eval *)ev;
  memcpy(psi_br, e.ntt.psi_bo.data(), e.N * 8);
  memcpy(psi_inv_br, e.ntt.psi_inv_bo.data(), e.N * 8);
  *n_inv = e.ntt.n_inv;
}
void orc_eval_test_vec(void *ev, int g, uint64_t *out) {
  Eval &e = *(Eval *)ev;
  memcpy(out, e.test_vec[g].data(), e.test_vec[g].size() * 8);
}
void orc_eval_dlog_map(void *ev, uint32_t *out) {
  Eval &e = *(Eval *)ev;
  memcpy(out, e.dlog.data(), e.dlog.size() * 4);
}
void orc_eval_auto_map(void *ev, int k, uint32_t *index, uint8_t *sign) {
  Eval &e = *(Eval *)ev;
  memcpy(index, e.auto_idx[k].data(), e.N * 4);
  memcpy(sign, e.auto_sign[k].data(), e.N);
}

void orc_ntt_forward(void *ev, uint64_t *poly, int lazy) { ((Eval *)ev)->ntt.forward(poly, lazy != 0); }
void orc_ntt_backward(void *ev, uint64_t *poly, int lazy) { ((Eval *)ev)->ntt.backward(poly, lazy != 0); }

int orc_decompose(void *ev, int which, uint64_t value, uint64_t *digits) {
  Eval &e = *(Eval *)ev;
  const Decomposer *d = which == 0 ? &e.dec_lwe : which == 1 ? &e.dec_a : which == 2 ? &e.dec_b : &e.dec_auto;
  d->decompose(value, digits);
  return (int)d->d;
}

void orc_shoup_matrix_fma(uint64_t q, uint64_t *out, const uint64_t *a, const uint64_t *a_shoup,
                          const uint64_t *b, size_t rows, size_t n) {
  std::vector<const u64 *> ap(rows), aps(rows), bp(rows);
  for (size_t r = 0; r < rows; r++) { ap[r] = a + r * n; aps[r] = a_shoup + r * n; bp[r] = b + r * n; }
  shoup_matrix_fma(q, out, ap.data(), aps.data(), bp.data(), rows, n);
}
uint64_t orc_shoup_repr(uint64_t v, uint64_t q) { return shoup_repr(v, q); }
uint64_t orc_barrett_mul(void *ev, uint64_t a, uint64_t b) { return ((Eval *)ev)->rmod.mul(a, b); }

// utils.rs:171-192 negacyclic_mul (schoolbook, u128 products)
void orc_negacyclic_mul(uint64_t q, const uint64_t *a, const uint64_t *b, uint64_t *r, size_t n) {
  for (size_t i = 0; i < n; i++) {
    u64 acc = 0;
    for (size_t j = 0; j <= i; j++) acc = (u64)((acc + (u128)a[j] * b[i - j] % q) % q);
    for (size_t j = i + 1; j < n; j++)
      acc = (u64)((acc + q - (u64)((u128)a[j] * b[n - j + i] % q)) % q);
    r[i] = acc;
  }
}

void *orc_key_new(void *ev, const uint64_t *rgsw, const uint64_t *autos, const uint64_t *ksk) {
  Eval &e = *(Eval *)ev;
  Key *k = new Key();
  const size_t N = e.N;
  k->N = N; k->n_lwe = e.n;
  k->rgsw_rows = 2 * e.p.d_a + 2 * e.p.d_b;
  k->auto_rows = 2 * e.p.auto_d;
  // keys.rs:738-757: copy + forward NTT each RGSW row; :702-736 auto keys
  k->rgsw.assign(rgsw, rgsw + e.n * k->rgsw_rows * N);
  k->autos.assign(autos, autos + (e.p.w + 1) * k->auto_rows * N);
  for (size_t r = 0; r < e.n * k->rgsw_rows; r++) e.ntt.forward(&k->rgsw[r * N], false);
  for (size_t r = 0; r < (e.p.w + 1) * k->auto_rows; r++) e.ntt.forward(&k->autos[r * N], false);
  // keys.rs:1200-1220 Shoup companions (utils.rs:54-73)
  k->rgsw_s.resize(k->rgsw.size()); k->autos_s.resize(k->autos.size());
  for (size_t i = 0; i < k->rgsw.size(); i++) k->rgsw_s[i] = shoup_repr(k->rgsw[i], e.Q);
  for (size_t i = 0; i < k->autos.size(); i++) k->autos_s[i] = shoup_repr(k->autos[i], e.Q);
  k->ksk.assign(ksk, ksk + (size_t)e.p.lwe_d * N * (e.n + 1));
  return k;
}
void orc_key_free(void *key) { delete (Key *)key; }

void orc_rlwe_by_rgsw(void *ev, void *key, uint64_t *rlwe, uint32_t idx, int trivial, int sh) {
  Eval &e = *(Eval *)ev;
  Scratch sc(e);
  rlwe_by_rgsw(e, *(Key *)key, sc, rlwe, idx, trivial != 0, sh != 0);
}
void orc_rlwe_auto(void *ev, void *key, uint64_t *rlwe, uint32_t k, int trivial, int sh) {
  Eval &e = *(Eval *)ev;
  Scratch sc(e);
  rlwe_auto(e, *(Key *)key, sc, rlwe, k, trivial != 0, sh != 0);
}
void orc_lwe_key_switch(void *ev, void *key, const uint64_t *in, uint64_t *out) {
  lwe_key_switch(*(Eval *)ev, *(Key *)key, in, out);
}
int orc_pbs(void *ev, void *key, int g, uint64_t *lwe, uint64_t *ks_out, uint64_t *rlwe_out) {
  Eval &e = *(Eval *)ev;
  Scratch sc(e);
  return pbs(e, *(Key *)key, sc, e.test_vec[g].data(), lwe, ks_out, rlwe_out);
}
void orc_gate(void *ev, void *key, int g, uint64_t *c0, const uint64_t *c1) {
  Eval &e = *(Eval *)ev;
  Scratch sc(e);
  gate(e, *(Key *)key, sc, g, c0, c1);
}
void orc_not(void *ev, uint64_t *c0) {  // evaluator.rs:2247-2250
  Eval &e = *(Eval *)ev;
  for (size_t i = 0; i <= e.N; i++) c0[i] = e.rmod.neg(c0[i]);
}
void orc_gate_batch(void *ev, void *key, const uint8_t *gates, const uint64_t *c0,
                    const uint64_t *c1, uint64_t *out, size_t count, int threads) {
  Eval &e = *(Eval *)ev;
  const Key &k = *(Key *)key;
  const size_t L = e.N + 1;
  if (threads < 1) threads = 1;
  auto work = [&](size_t t) {
    Scratch sc(e);
    for (size_t i = t; i < count; i += (size_t)threads) {
      memcpy(out + i * L, c0 + i * L, L * 8);
      gate(e, k, sc, gates[i], out + i * L, c1 + i * L);
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < threads; t++) th.emplace_back(work, (size_t)t);
  work(0);
  for (auto &x : th) x.join();
}
void orc_sample_extract(void *ev, const uint64_t *rlwe, uint64_t *lwe, uint32_t index) {
  sample_extract(*(Eval *)ev, rlwe, lwe, index);
}

// ---- FheUint8 operations (shortint/mod.rs:63-292), sequential ------------
// a, b: [8][N+1] (LSB first).  op: 0 add, 1 sub, 2 mul, 3 div_rem, 4 eq,
// 5 neq, 6 lt, 7 gt, 8 le, 9 ge, 10 mux (selector = sel), 11 overflowing_add,
// 12 overflowing_sub.  out: [8][N+1] or, for comparisons, [1][N+1]; out2:
// remainder (div_rem) or overflow flag.  flag (div_rem): in/out division by
// zero flag; *flag_set says whether it holds a ciphertext.
static int u8_op(SEval &s, int op, const uint64_t *a, const uint64_t *b, const uint64_t *sel, uint64_t *out,
                 uint64_t *out2, uint64_t *flag, int *flag_set) {
  const Eval &e = s.e;
  const size_t L = e.N + 1;
  std::vector<Ct> A(8), Bv(8);
  for (int i = 0; i < 8; i++) {
    A[i].assign(a + i * L, a + (i + 1) * L);
    Bv[i].assign(b + i * L, b + (i + 1) * L);
  }
  auto put = [&](uint64_t *dst, const std::vector<Ct> &v) {
    for (size_t i = 0; i < v.size(); i++) memcpy(dst + i * L, v[i].data(), L * 8);
  };
  Ct cl, cll;
  switch (op) {
    case 0: case 11: {  // AddAssign (mod.rs:63-70) / overflowing_add (:157-165)
      s_adder(s, A, Bv, false, cl, cll);
      put(out, A);
      if (op == 11 && out2) memcpy(out2, cl.data(), L * 8);
      return 0;
    }
    case 1: case 12: {  // Sub (mod.rs:81-90) / overflowing_sub (:171-179)
      std::vector<Ct> nb;
      for (auto &x : Bv) nb.push_back(s.not_(x));
      s_adder(s, nb, A, true, cl, cll);
      put(out, nb);
      if (op == 12 && out2) { Ct o = s.not_(cl); memcpy(out2, o.data(), L * 8); }
      return 0;
    }
    case 2: put(out, s_mul(s, A, Bv)); return 0;
    case 3: {  // div_rem (mod.rs:187-202) with set_div_by_zero_flag (:42-56)
      if (flag && flag_set) {
        Ct z = s_is_zero(s, Bv);
        if (!*flag_set) { memcpy(flag, z.data(), L * 8); *flag_set = 1; }
        else {
          Ct f(flag, flag + L);
          f = s.g(ORC_OR, f, z);
          memcpy(flag, f.data(), L * 8);
        }
      }
      std::vector<Ct> q, r;
      s_division(s, A, Bv, q, r);
      put(out, q);
      if (out2) put(out2, r);
      return 0;
    }
    case 4: put(out, {s_equality(s, A, Bv)}); return 0;
    case 5: put(out, {s.not_(s_equality(s, A, Bv))}); return 0;
    case 6: put(out, {s_comparator(s, Bv, A)}); return 0;
    case 7: put(out, {s_comparator(s, A, Bv)}); return 0;
    case 8: put(out, {s.not_(s_comparator(s, A, Bv))}); return 0;
    case 9: put(out, {s.not_(s_comparator(s, Bv, A))}); return 0;
    case 10: {
      Ct sl(sel, sel + L);
      put(out, s_mux(s, sl, A, Bv));
      return 0;
    }
  }
  return -1;
}

int orc_u8_op(void *ev, void *key, int op, const uint64_t *a, const uint64_t *b, const uint64_t *sel,
              uint64_t *out, uint64_t *out2, uint64_t *flag, int *flag_set) {
  SEval s(*(Eval *)ev, (const Key *)key);
  return u8_op(s, op, a, b, sel, out, out2, flag, flag_set);
}

// Gates one FheUint8 operation issues, by gate code (and, nand, or, nor, xor,
// xnor): the operation run dry on zero ciphertexts, nothing bootstrapped.
int orc_u8_gate_mix(void *ev, int op, uint64_t counts[6]) {
  const Eval &e = *(Eval *)ev;
  const size_t L = e.N + 1;
  std::vector<uint64_t> a(8 * L, 0), b(8 * L, 0), sel(L, 0), out(8 * L), out2(8 * L), flag(L, 0);
  for (int t = 0; t < 6; t++) counts[t] = 0;
  SEval s(e, nullptr);
  s.tally = counts;
  int fs = 0;
  return u8_op(s, op, a.data(), b.data(), sel.data(), out.data(), out2.data(), flag.data(), &fs);
}

// ---- generic pins (reference unit tests at their own sizes) -----------------
// Deterministic Miller-Rabin for 64-bit integers (bases valid below 2^64);
// stands in for num-bigint-dig's probably_prime used by utils.rs:114-116.
static bool is_prime_u64(u64 n) {
  if (n < 2) return false;
  for (u64 p : {2ull, 3ull, 5ull, 7ull, 11ull, 13ull, 17ull, 19ull, 23ull, 29ull, 31ull, 37ull}) {
    if (n % p == 0) return n == p;
  }
  u64 d = n - 1;
  int s = 0;
  while ((d & 1) == 0) { d >>= 1; s++; }
  for (u64 a : {2ull, 3ull, 5ull, 7ull, 11ull, 13ull, 17ull, 19ull, 23ull, 29ull, 31ull, 37ull}) {
    u64 x = mod_exponent(a, d, n);
    if (x == 1 || x == n - 1) continue;
    bool comp = true;
    for (int r = 1; r < s; r++) {
      x = (u64)(((u128)x * x) % n);
      if (x == n - 1) { comp = false; break; }
    }
    if (comp) return false;
  }
  return true;
}

// utils.rs:122-142 generate_prime (0 when none is found)
uint64_t orc_generate_prime(uint32_t num_bits, uint64_t modulo, uint64_t upper_bound) {
  const int lz = 64 - (int)num_bits;
  u64 t = upper_bound - 1;
  while (t % modulo != 1 && clz64(t) == lz) t -= 1;
  while (!is_prime_u64(t) && clz64(t) == lz && t >= modulo) t -= modulo;
  return (is_prime_u64(t) && clz64(t) == lz) ? t : 0;
}

void *orc_ntt_custom_new(uint64_t q, size_t n) {
  Ntt *t = new Ntt();
  t->init(q, n);
  return t;
}
void orc_ntt_custom_free(void *h) { delete (Ntt *)h; }
void orc_ntt_custom_forward(void *h, uint64_t *a, int lazy) { ((Ntt *)h)->forward(a, lazy != 0); }
void orc_ntt_custom_backward(void *h, uint64_t *a, int lazy) { ((Ntt *)h)->backward(a, lazy != 0); }
uint64_t orc_mul_mod_barrett(uint64_t q, uint64_t a, uint64_t b) { return ModU64(q).mul(a, b); }

// DefaultDecomposer with arbitrary (q, logb, d); returns ignore_bits.
uint32_t orc_decompose_custom(uint64_t q, uint32_t logb, uint32_t d, uint64_t value, uint64_t *out) {
  Decomposer dc;
  dc.init(q, logb, d);
  dc.decompose(value, out);
  return dc.ignore_bits;
}
uint64_t orc_round_value(uint64_t v, uint32_t ignore_bits) { return Decomposer::round_value(v, ignore_bits); }
// decomposer.rs:129-140 recompose with ModularOpsU64
uint64_t orc_recompose(uint64_t q, uint32_t logb, uint32_t d, const uint64_t *limbs) {
  Decomposer dc;
  dc.init(q, logb, d);
  ModU64 m(q);
  u64 v = 0;
  for (u32 j = 0; j < d; j++) v = m.add(v, m.mul(limbs[j], dc.gadget(j)));
  return v;
}

// ---- client harness --------------------------------------------------------
void orc_chacha_block(const uint32_t state[16], int rounds, uint32_t out[16]) { chacha_core(state, rounds, out); }
int orc_uniform_mod_word(uint64_t q, uint64_t word, uint64_t *sample) { return uniform_word(word, q, *sample); }
void *orc_rng_new(const uint8_t seed[32]) { return new ChaCha8(seed); }
void orc_rng_free(void *r) { delete (ChaCha8 *)r; }
uint64_t orc_rng_next_u64(void *r) { return ((ChaCha8 *)r)->next_u64(); }
void orc_rng_uniform_mod(void *r, uint64_t q, uint64_t *out, size_t n) {
  for (size_t i = 0; i < n; i++) out[i] = ((ChaCha8 *)r)->uniform_mod(q);
}

// ClientKey::sk_rlwe / sk_lwe (keys.rs:73-115): seed -> puncture 1 (RLWE), 2 (LWE).
void orc_client_keys(void *ev, int parties, int seed_base, int32_t *s, int32_t *z,
                     int32_t *s_parts, int32_t *z_parts) {
  Eval &e = *(Eval *)ev;
  const size_t N = e.N, n = e.n;
  std::vector<int32_t> sp(N), zp(n);
  for (size_t i = 0; i < N; i++) s[i] = 0;
  for (size_t i = 0; i < n; i++) z[i] = 0;
  for (int p = 0; p < parties; p++) {
    uint8_t seed[32];
    memset(seed, (uint8_t)(p + 1 + 16 * seed_base), 32);
    ChaCha8 main(seed);
    uint8_t s1[32], s2[32];
    for (int i = 0; i < 32; i++) s1[i] = (uint8_t)main.next_u32();  // puncture 1
    for (int i = 0; i < 32; i++) s2[i] = (uint8_t)main.next_u32();  // puncture 2
    ChaCha8 rr(s1), lr(s2);
    ternary_secret(rr, sp.data(), N, N >> 1);
    if (e.p.lwe_gauss) {
      for (size_t i = 0; i < n; i++) zp[i] = (int32_t)std::trunc(lr.gaussian());
    } else {
      ternary_secret(lr, zp.data(), n, n >> 1);
    }
    for (size_t i = 0; i < N; i++) s[i] += sp[i];
    for (size_t i = 0; i < n; i++) z[i] += zp[i];
    if (s_parts) memcpy(s_parts + p * N, sp.data(), N * 4);
    if (z_parts) memcpy(z_parts + p * n, zp.data(), n * 4);
  }
}

// Server key under the ideal secrets (s, z), restating the encryptions of
// keygen.rs:68-160 (RGSW), :306-430 (auto keys), lwe.rs:46-101 (LWE KSK).
void orc_gen_server_key(void *ev, const int32_t *s, const int32_t *z, const uint8_t err_seed[32],
                        uint64_t *rgsw, uint64_t *autos, uint64_t *ksk) {
  Eval &e = *(Eval *)ev;
  const size_t N = e.N, n = e.n;
  const u64 Q = e.Q;
  ChaCha8 rng(err_seed);
  std::vector<u64> s_eval(N), tmp(N), m(N);
  for (size_t i = 0; i < N; i++) s_eval[i] = map_from_i64(Q, s[i]);
  e.ntt.forward(s_eval.data(), false);
  auto a_times_s = [&](const u64 *a, u64 *out) {  // out = a * s (coefficient domain)
    memcpy(out, a, N * 8);
    e.ntt.forward(out, false);
    for (size_t i = 0; i < N; i++) out[i] = e.rmod.mul(out[i], s_eval[i]);
    e.ntt.backward(out, false);
  };
  auto gauss_fill = [&](u64 *out) {
    for (size_t i = 0; i < N; i++) out[i] = map_from_f64(Q, rng.gaussian());
  };
  const size_t da = e.p.d_a, db = e.p.d_b, rows = 2 * da + 2 * db;
  for (size_t li = 0; li < n; li++) {
    // X^{emb * z_i} (utils.rs:195-217)
    std::fill(m.begin(), m.end(), 0);
    int64_t si = (int64_t)z[li] * (int64_t)e.emb;
    if (si < 0) m[N - (size_t)(-si)] = Q - 1; else m[(size_t)si] = 1;
    u64 *ct = rgsw + li * rows * N;
    for (size_t j = 0; j < da; j++) {  // RLWE'(-sm): a += beta m, b = a s + e
      u64 *a = ct + j * N, *b = ct + (da + j) * N;
      for (size_t i = 0; i < N; i++) a[i] = rng.uniform_mod(Q);
      a_times_s(a, tmp.data());
      gauss_fill(b);
      for (size_t i = 0; i < N; i++) b[i] = e.rmod.add(b[i], tmp[i]);
      u64 beta = e.dec_a.gadget((u32)j) % Q;
      for (size_t i = 0; i < N; i++) a[i] = e.rmod.add(a[i], e.rmod.mul(m[i], beta));
    }
    for (size_t j = 0; j < db; j++) {  // RLWE'(m): b = a s + e + beta m
      u64 *a = ct + (2 * da + j) * N, *b = ct + (2 * da + db + j) * N;
      for (size_t i = 0; i < N; i++) a[i] = rng.uniform_mod(Q);
      a_times_s(a, tmp.data());
      gauss_fill(b);
      u64 beta = e.dec_b.gadget((u32)j) % Q;
      for (size_t i = 0; i < N; i++) b[i] = e.rmod.add(e.rmod.add(b[i], e.rmod.mul(m[i], beta)), tmp[i]);
    }
  }
  // auto keys: ksk from -s(X^k) to s (keygen.rs:376-430, :306-363)
  const size_t dauto = e.p.auto_d;
  std::vector<u64> neg_s_auto(N), sm(N);
  for (size_t i = 0; i < N; i++) sm[i] = map_from_i64(Q, s[i]);
  for (size_t kk = 0; kk <= e.p.w; kk++) {
    const auto &idx = e.auto_idx[kk];
    const auto &sg = e.auto_sign[kk];
    for (size_t i = 0; i < N; i++) neg_s_auto[idx[i]] = sg[i] ? e.rmod.neg(sm[i]) : sm[i];
    u64 *key = autos + kk * 2 * dauto * N;
    for (size_t j = 0; j < dauto; j++) {
      u64 *a = key + j * N, *b = key + (dauto + j) * N;
      for (size_t i = 0; i < N; i++) a[i] = rng.uniform_mod(Q);
      a_times_s(a, tmp.data());
      gauss_fill(b);
      u64 beta = e.dec_auto.gadget((u32)j) % Q;
      for (size_t i = 0; i < N; i++) {
        b[i] = e.rmod.add(b[i], tmp[i]);
        b[i] = e.rmod.add(b[i], e.rmod.mul(neg_s_auto[i] % Q, beta));
      }
    }
  }
  // LWE ksk from s (dim N) to z (dim n) mod q_ks (lwe.rs:46-101)
  const u64 qk = e.p.lwe_q, mask = qk - 1;
  const size_t d = e.p.lwe_d;
  std::vector<u64> zm(n);
  for (size_t i = 0; i < n; i++) zm[i] = map_from_i64(qk, z[i]) & mask;
  for (size_t i = 0; i < N; i++) {
    u64 neg_si = (0 - map_from_i64(qk, s[i])) & mask;
    for (size_t j = 0; j < d; j++) {
      u64 *row = ksk + (i * d + j) * (n + 1);
      u64 az = 0;
      for (size_t c = 0; c < n; c++) {
        row[1 + c] = rng.uniform_mod(qk);
        az = (az + row[1 + c] * zm[c]) & mask;
      }
      u64 beta = e.dec_lwe.gadget((u32)j) & mask;
      u64 b = (az + beta * neg_si) & mask;
      b = (b + map_from_f64(qk, rng.gaussian())) & mask;
      row[0] = b;
    }
  }
}

void orc_encrypt_bool(void *ev, void *r, const int32_t *s, int bit, uint64_t *lwe) {
  Eval &e = *(Eval *)ev;
  ChaCha8 &rng = *(ChaCha8 *)r;
  const u64 Q = e.Q;
  u64 m = bit ? e.true_el : e.false_el;
  u64 sa = 0;
  for (size_t i = 0; i < e.N; i++) {
    lwe[1 + i] = rng.uniform_mod(Q);
    sa = e.rmod.add(e.rmod.mul(lwe[1 + i], map_from_i64(Q, s[i]) % Q), sa);
  }
  u64 err = map_from_f64(Q, rng.gaussian());
  lwe[0] = e.rmod.add(e.rmod.add(sa, err), m);
}

static int decode_bool(const Eval &e, u64 m) {  // evaluator.rs:243-256
  u64 qby8 = e.true_el;
  size_t v = (size_t)std::round(((double)(m + qby8) * 4.0) / (double)e.Q) % 4;
  if (v == 0) return 0;
  if (v == 1) return 1;
  return -1;
}

// ---- non-interactive input path ----------------------------------------------
// NonInteractiveBatchedFheBools::from (ni_mp_api.rs:248-280): the a-parts of
// the batch's RLWEs, in order, from one ChaCha8(seed) stream
// (RandomFillUniformInModulus, random.rs:93-110); b copied.
void orc_ni_unseed(void *ev, const uint8_t seed[32], const uint64_t *b, size_t count, uint64_t *rlwe) {
  Eval &e = *(Eval *)ev;
  const size_t N = e.N;
  ChaCha8 prng(seed);
  for (size_t c = 0; c < count; c++) {
    for (size_t i = 0; i < N; i++) rlwe[c * 2 * N + i] = prng.uniform_mod(e.Q);
    memcpy(rlwe + c * 2 * N + N, b + c * N, N * 8);
  }
}

// rlwe_key_switch (runtime.rs:1001-1063) with the key-switching key
// Ksk(u -> s) given in the coefficient domain ([2d][N]: rows A then B); the
// key is sent to the evaluation domain with Shoup companions as
// NonInteractiveServerKeyEvaluationDomain / its Shoup form do.
void orc_ni_key_switch(void *ev, const uint64_t *ksk_coef, const uint64_t *in, uint64_t *out) {
  Eval &e = *(Eval *)ev;
  if (e.p.variant != 2) throw std::runtime_error("not a non-interactive parameter set");
  const size_t N = e.N, d = e.dec_ni.d;
  std::vector<u64> ksk(ksk_coef, ksk_coef + 2 * d * N), ksk_s(2 * d * N);
  for (size_t r = 0; r < 2 * d; r++) e.ntt.forward(&ksk[r * N], false);
  for (size_t i = 0; i < ksk.size(); i++) ksk_s[i] = shoup_repr(ksk[i], e.Q);
  std::vector<u64> tmp_row(in, in + N), dec(d * N), oa(N, 0), ob(N, 0);
  for (size_t i = 0; i < N; i++) tmp_row[i] = e.Q - tmp_row[i];  // elwise_neg_mut
  decompose_r(e.dec_ni, tmp_row.data(), dec.data(), N);
  for (size_t j = 0; j < d; j++) e.ntt.forward(&dec[j * N], true);  // forward_lazy
  const u64 *ap[64] = {}, *aps[64] = {}, *bp[64] = {};
  for (size_t j = 0; j < d; j++) { ap[j] = &ksk[j * N]; aps[j] = &ksk_s[j * N]; bp[j] = &dec[j * N]; }
  shoup_matrix_fma(e.Q, oa.data(), ap, aps, bp, d, N);
  for (size_t j = 0; j < d; j++) { ap[j] = &ksk[(d + j) * N]; aps[j] = &ksk_s[(d + j) * N]; }
  shoup_matrix_fma(e.Q, ob.data(), ap, aps, bp, d, N);
  e.ntt.backward(oa.data(), false);
  e.ntt.backward(ob.data(), false);
  for (size_t i = 0; i < N; i++) ob[i] = e.rmod.add(ob[i], in[N + i]);  // elwise_add_mut
  memcpy(out, oa.data(), N * 8);
  memcpy(out + N, ob.data(), N * 8);
}

// Client side (harness): the NI batched bool encryption of ni_mp_api.rs:302-345
// with seeded_secret_key_encrypt_rlwe (rgsw/keygen.rs:439-481): per RLWE, a
// from ChaCha8(seed), b = e + m + a u, m_i = true_el / false_el for the bools
// of that RLWE and 0 beyond the last; errors from ChaCha8(err_seed).
void orc_ni_encrypt_bools(void *ev, const int32_t *u, const uint8_t seed[32], const uint8_t err_seed[32],
                          const uint8_t *bits, size_t nbits, uint64_t *b_out) {
  Eval &e = *(Eval *)ev;
  const size_t N = e.N, count = (nbits + N - 1) / N;
  ChaCha8 prng(seed), rng(err_seed);
  std::vector<u64> u_eval(N), a(N);
  for (size_t i = 0; i < N; i++) u_eval[i] = map_from_i64(e.Q, u[i]);
  e.ntt.forward(u_eval.data(), false);
  for (size_t c = 0; c < count; c++) {
    for (size_t i = 0; i < N; i++) a[i] = prng.uniform_mod(e.Q);
    e.ntt.forward(a.data(), false);
    for (size_t i = 0; i < N; i++) a[i] = e.rmod.mul(a[i], u_eval[i]);
    e.ntt.backward(a.data(), false);
    u64 *b = b_out + c * N;
    for (size_t i = 0; i < N; i++) {
      const size_t k = c * N + i;
      const u64 m = k < nbits ? (bits[k] ? e.true_el : e.false_el) : 0;
      b[i] = e.rmod.add(e.rmod.add(map_from_f64(e.Q, rng.gaussian()), m), a[i]);
    }
  }
}

// An ideal key-switching key Ksk(u -> s) (harness; the protocol assembles it
// from user shares): row j of part A uniform, part B = a_j s + e_j + g_j u,
// g_j the decomposer's gadget (decomposer.rs:13-21), coefficient domain.
void orc_ni_ksk_gen(void *ev, const int32_t *u, const int32_t *s, const uint8_t err_seed[32], uint64_t *ksk) {
  Eval &e = *(Eval *)ev;
  const size_t N = e.N, d = e.dec_ni.d;
  ChaCha8 rng(err_seed);
  std::vector<u64> s_eval(N), tmp(N);
  for (size_t i = 0; i < N; i++) s_eval[i] = map_from_i64(e.Q, s[i]);
  e.ntt.forward(s_eval.data(), false);
  for (size_t j = 0; j < d; j++) {
    u64 *a = ksk + j * N, *b = ksk + (d + j) * N;
    for (size_t i = 0; i < N; i++) a[i] = rng.uniform_mod(e.Q);
    memcpy(tmp.data(), a, N * 8);
    e.ntt.forward(tmp.data(), false);
    for (size_t i = 0; i < N; i++) tmp[i] = e.rmod.mul(tmp[i], s_eval[i]);
    e.ntt.backward(tmp.data(), false);
    const u64 g = e.dec_ni.gadget((u32)j) % e.Q;
    for (size_t i = 0; i < N; i++) {
      const u64 gu = e.rmod.mul(map_from_i64(e.Q, u[i]) % e.Q, g);
      b[i] = e.rmod.add(e.rmod.add(tmp[i], map_from_f64(e.Q, rng.gaussian())), gu);
    }
  }
}

// ServerKeyEvaluationDomain::from(&Seeded...ServerKey), keys.rs:687-781 and
// (NI) 869-1004, before the forward NTT: auto keys slot by slot in
// auto_element_dlogs order (parameters.rs:364-370), each d_auto A rows from
// the auto stream then its B rows; LWE KSK row by row, words 1..n from the
// ksk stream mod q_ks, word 0 = b.  Outputs in the layout of orc_key_new.
void orc_expand_seeded_key(void *ev, const uint64_t *auto_b, const uint8_t auto_seed[32], const uint64_t *lwe_b,
                           const uint8_t lwe_seed[32], uint64_t *autos, uint64_t *ksk) {
  Eval &e = *(Eval *)ev;
  const size_t N = e.N, n = e.n, da = e.p.auto_d;
  ChaCha8 auto_prng(auto_seed);
  for (size_t k = 0; k <= e.p.w; k++) {
    u64 *key = autos + k * 2 * da * N;
    for (size_t i = 0; i < da * N; i++) key[i] = auto_prng.uniform_mod(e.Q);
    memcpy(key + da * N, auto_b + k * da * N, da * N * 8);
  }
  ChaCha8 ksk_prng(lwe_seed);
  const size_t rows = (size_t)e.p.lwe_d * N;
  for (size_t r = 0; r < rows; r++) {
    u64 *row = ksk + r * (n + 1);
    for (size_t c = 1; c <= n; c++) row[c] = ksk_prng.uniform_mod(e.p.lwe_q);
    row[0] = lwe_b[r];
  }
}

// rgsw_by_rgsw_inplace (runtime.rs:883-985): rgsw0 (rlwe x rgsw shape,
// coefficient domain) <- rgsw0 x rgsw1, rgsw1 given in the coefficient domain
// in the rgsw x rgsw shape (sent to the evaluation domain first, as the
// aggregation does, evaluator.rs:1160-1163).  Every RLWE of rgsw0 -- the
// -sm rows then the m rows -- times RGSW(m1): decompose A with the rgrg A
// decomposer, forward NTT, poly_fma_routine (runtime.rs:363-372) against the
// -sm rows of rgsw1; decompose B with the rgrg B decomposer against the m
// rows; the outputs go back to the coefficient domain.
void orc_rgsw_by_rgsw(void *ev, uint64_t *rgsw0, const uint64_t *rgsw1) {
  Eval &e = *(Eval *)ev;
  if (!e.p.rgrg_logb) throw std::runtime_error("parameter set without RGSW x RGSW");
  const size_t N = e.N, da = e.p.d_a, db = e.p.d_b, ra = e.p.rgrg_d_a, rb = e.p.rgrg_d_b;
  const size_t rows0 = 2 * da + 2 * db, rows1 = 2 * ra + 2 * rb;
  std::vector<u64> k1(rgsw1, rgsw1 + rows1 * N);
  for (size_t r = 0; r < rows1; r++) e.ntt.forward(&k1[r * N], false);
  std::vector<u64> out(rows0 * N, 0), dec(std::max(ra, rb) * N);
  auto fma = [&](u64 *o, size_t krow0, size_t rows) {
    for (size_t j = 0; j < rows; j++) {
      const u64 *k = &k1[(krow0 + j) * N], *x = &dec[j * N];
      for (size_t i = 0; i < N; i++) o[i] = e.rmod.add(o[i], e.rmod.mul(x[i], k[i]));
    }
  };
  auto one = [&](const u64 *a, const u64 *b, u64 *oa, u64 *ob) {
    decompose_r(e.dec_rgrg_a, a, dec.data(), N);
    for (size_t j = 0; j < ra; j++) e.ntt.forward(&dec[j * N], false);
    fma(oa, 0, ra);
    fma(ob, ra, ra);
    decompose_r(e.dec_rgrg_b, b, dec.data(), N);
    for (size_t j = 0; j < rb; j++) e.ntt.forward(&dec[j * N], false);
    fma(oa, 2 * ra, rb);
    fma(ob, 2 * ra + rb, rb);
  };
  for (size_t j = 0; j < da; j++)
    one(rgsw0 + j * N, rgsw0 + (da + j) * N, &out[j * N], &out[(da + j) * N]);
  for (size_t j = 0; j < db; j++)
    one(rgsw0 + (2 * da + j) * N, rgsw0 + (2 * da + db + j) * N, &out[(2 * da + j) * N],
        &out[(2 * da + db + j) * N]);
  for (size_t r = 0; r < rows0; r++) e.ntt.backward(&out[r * N], false);
  memcpy(rgsw0, out.data(), rows0 * N * 8);
}

// puncture_p_rng (utils.rs:219-228) with RandomFill<[u8; 32]> (random.rs:
// 162-175): `times` successive 32-byte fills of ChaCha8(seed), the last one
// kept; a byte is Uniform::new_inclusive(0, 255), i.e. the low byte of one
// u32 word of the stream.
void crs_puncture(const uint8_t seed[32], size_t times, uint8_t out[32]) {
  ChaCha8 r(seed);
  for (size_t t = 0; t < times; t++)
    for (int i = 0; i < 32; i++) out[i] = (uint8_t)r.next_u32();
}

// NonInteractiveMultiPartyCrs (evaluator.rs:115-172): what = 0 auto keys,
// 1 LWE KSK, 2 ui_to_s KSK of user `index`, 3 NI RGSW of LWE index `index`.
void orc_ni_crs_seed(const uint8_t crs[32], int what, size_t index, uint8_t out[32]) {
  uint8_t key[32], t[32];
  crs_puncture(crs, 1, key);  // key_seed
  switch (what) {
    case 0: crs_puncture(key, 2, out); break;
    case 1: crs_puncture(key, 3, out); break;
    case 2: crs_puncture(crs, 2, t); crs_puncture(t, index + 1, out); break;  // ui_to_s_ks_seed
    default: crs_puncture(key, 1, t); crs_puncture(t, index + 1, out); break;  // ni_rgsw_cts_main_seed
  }
}

// InteractiveMultiPartyCrs (evaluator.rs:78-100): what = 0 public-key share,
// 1 auto keys, 2 LWE KSK.
void orc_interactive_crs_seed(const uint8_t crs[32], int what, uint8_t out[32]) {
  uint8_t key[32];
  if (what == 0) {
    crs_puncture(crs, 1, out);
    return;
  }
  crs_puncture(crs, 2, key);  // key_seed
  crs_puncture(key, what == 1 ? 1 : 2, out);
}

// multi_party_user_id_lwe_segment (evaluator.rs:613-626); an empty segment
// when the start passes lwe_n.
void lwe_segment(size_t user, size_t users, size_t n, size_t *b, size_t *e) {
  const size_t per = (n + users - 1) / users;
  *b = per * user;
  *e = std::min(per * (user + 1), n);
  if (*e < *b) *e = *b;
}

struct NiDigits {  // one value to key-switch: its 50 one-bit digits, forward NTT
  std::vector<u64> d;
};

// The key switch of produce_rgsw_ciphertext_from_ni_rgsw (evaluator.rs:
// 542-553 / 581-591) given the value's transformed digits: a = sum_j A_j c_j,
// b = sum_j B_j c_j (elwise_fma_mut), back to the coefficient domain.
void ni_ks_rows(const Eval &e, const u64 *ksk_eval, const u64 *dig, u64 *oa, u64 *ob) {
  const size_t N = e.N, d = e.dec_ni.d;
  std::fill(oa, oa + N, 0);
  std::fill(ob, ob + N, 0);
  for (size_t j = 0; j < d; j++) {
    const u64 *c = dig + j * N, *pa = ksk_eval + j * N, *pb = ksk_eval + (d + j) * N;
    for (size_t i = 0; i < N; i++) {
      ob[i] = e.rmod.add(ob[i], e.rmod.mul(pb[i], c[i]));
      oa[i] = e.rmod.add(oa[i], e.rmod.mul(pa[i], c[i]));
    }
  }
  e.ntt.backward(oa, false);
  e.ntt.backward(ob, false);
}

// The RGSW step of aggregate_non_interactive_multi_party_server_key_shares
// (evaluator.rs:1310-1560) for LWE indices [i0, i1): a_l rows from the
// index's stream (d_max - d_b punctured rows, then d_b rows, negated), zero
// encryptions summed over the users, every value decomposed (50 one-bit
// digits) and transformed once; the leader's RGSW in the rlwe x rgsw shape
// from the last rlrg rows (produce_rgsw_ciphertext_from_ni_rgsw,
// :480-608), then times every other user's RGSW in the rgsw x rgsw shape in
// increasing user id.  ksk_eval [users][2 50][N]: Ksk(u_j -> s) in the
// evaluation domain, A rows (from the user's stream) then aggregated B rows.
// out [i1 - i0][2 d_a + 2 d_b][N], coefficient domain.
void ni_aggregate_rgsw(Eval &e, const uint8_t crs[32], size_t users, const u64 *ksk_eval,
                       const uint64_t *const *self_leader, const uint64_t *const *not_leader,
                       const uint64_t *const *zero_encs, size_t i0, size_t i1, u64 *out) {
  const size_t N = e.N, n = e.n, d = e.dec_ni.d;
  const size_t ra = e.p.rgrg_d_a, rb = e.p.rgrg_d_b, max_d = std::max(ra, rb);
  const size_t la = e.p.d_a, lb = e.p.d_b, max_l = std::max(la, lb), rows0 = 2 * la + 2 * lb;
  const size_t rows1 = 2 * ra + 2 * rb, R = ra + rb;
  std::vector<u64> dig(R * d * N), val(N), other(rows1 * N);
  for (size_t li = i0; li < i1; li++) {
    uint8_t seed[32];
    orc_ni_crs_seed(crs, 3, li, seed);
    ChaCha8 a_prng(seed);
    for (size_t r = 0; r < max_d - rb; r++)  // puncture
      for (size_t i = 0; i < N; i++) a_prng.uniform_mod(e.Q);
    for (size_t v = 0; v < R; v++) {
      if (v < ra) {  // sum_k zero_enc_k row v
        std::fill(val.begin(), val.end(), 0);
        for (size_t k = 0; k < users; k++) {
          const u64 *z = zero_encs[k] + (li * ra + v) * N;
          for (size_t i = 0; i < N; i++) val[i] = e.rmod.add(val[i], z[i]);
        }
      } else {  // -a row (elwise_neg_mut: q - x)
        for (size_t i = 0; i < N; i++) val[i] = e.Q - a_prng.uniform_mod(e.Q);
      }
      u64 *dv = &dig[v * d * N];
      decompose_r(e.dec_ni, val.data(), dv, N);
      for (size_t j = 0; j < d; j++) e.ntt.forward(dv + j * N, false);
    }
    size_t leader = 0;
    for (size_t k = 0; k < users; k++) {
      size_t b, en;
      lwe_segment(k, users, n, &b, &en);
      if (li >= b && li < en) leader = k;
    }
    // leader: values ra - la .. ra (zero encs) and R - lb .. R (-a), its ct rows
    u64 *o = out + (li - i0) * rows0 * N;
    {
      size_t b, en;
      lwe_segment(leader, users, n, &b, &en);
      const u64 *ct = self_leader[leader] + (li - b) * max_l * N;
      const u64 *ke = ksk_eval + leader * 2 * d * N;
      for (size_t r = 0; r < la; r++) {
        u64 *oa = o + r * N, *ob = o + (la + r) * N;
        ni_ks_rows(e, ke, &dig[(ra - la + r) * d * N], oa, ob);
        const u64 *c = ct + (max_l - la + r) * N;
        for (size_t i = 0; i < N; i++) oa[i] = e.rmod.add(oa[i], c[i]);
      }
      for (size_t r = 0; r < lb; r++) {
        u64 *oa = o + (2 * la + r) * N, *ob = o + (2 * la + lb + r) * N;
        ni_ks_rows(e, ke, &dig[(R - lb + r) * d * N], oa, ob);
        const u64 *c = ct + (max_l - lb + r) * N;
        for (size_t i = 0; i < N; i++) ob[i] = e.rmod.add(ob[i], c[i]);
      }
    }
    for (size_t k = 0; k < users; k++) {
      if (k == leader) continue;
      size_t b, en;
      lwe_segment(k, users, n, &b, &en);
      const size_t pos = li < b ? li : li - (en - b);
      const u64 *ct = not_leader[k] + pos * max_d * N;
      const u64 *ke = ksk_eval + k * 2 * d * N;
      for (size_t r = 0; r < ra; r++) {
        u64 *oa = &other[r * N], *ob = &other[(ra + r) * N];
        ni_ks_rows(e, ke, &dig[r * d * N], oa, ob);
        const u64 *c = ct + (max_d - ra + r) * N;
        for (size_t i = 0; i < N; i++) oa[i] = e.rmod.add(oa[i], c[i]);
      }
      for (size_t r = 0; r < rb; r++) {
        u64 *oa = &other[(2 * ra + r) * N], *ob = &other[(2 * ra + rb + r) * N];
        ni_ks_rows(e, ke, &dig[(ra + r) * d * N], oa, ob);
        const u64 *c = ct + (max_d - rb + r) * N;
        for (size_t i = 0; i < N; i++) ob[i] = e.rmod.add(ob[i], c[i]);
      }
      orc_rgsw_by_rgsw(&e, o, other.data());
    }
  }
}

// aggregate_non_interactive_multi_party_server_key_shares (evaluator.rs:
// 1222-1622) on shares given field by field (arrays of per-user pointers,
// user id order): Ksk(u_j -> s) B rows = own ui_to_s_ksk + the other users'
// zero encryptions for j (evaluator.rs:1269-1294), coefficient domain; auto
// keys and LWE KSK summed (:1563-1605); RGSWs of LWE indices [i0, i1).
// ksk_out [users][50][N], rgsw_out [i1 - i0][rows][N], auto_out
// [w + 1][d_auto][N], lwe_out [lwe_d N].
void orc_ni_aggregate(void *ev, const uint8_t crs[32], int users_, const uint64_t *const *ui_to_s_ksk,
                      const uint64_t *const *ksk_zero_encs, const uint64_t *const *self_leader,
                      const uint64_t *const *not_leader, const uint64_t *const *zero_encs,
                      const uint64_t *const *auto_keys, const uint64_t *const *lwe_ksk, size_t i0, size_t i1,
                      uint64_t *ksk_out, uint64_t *rgsw_out, uint64_t *auto_out, uint64_t *lwe_out) {
  Eval &e = *(Eval *)ev;
  if (e.p.variant != 2 || !e.p.rgrg_logb) throw std::runtime_error("not a non-interactive parameter set");
  const size_t users = (size_t)users_, N = e.N, d = e.dec_ni.d;
  for (size_t j = 0; j < users; j++) {
    u64 *o = ksk_out + j * d * N;
    memcpy(o, ui_to_s_ksk[j], d * N * 8);
    for (size_t k = 0; k < users; k++) {
      if (k == j) continue;
      const u64 *z = ksk_zero_encs[k] + (j < k ? j : j - 1) * d * N;
      for (size_t i = 0; i < d * N; i++) o[i] = e.rmod.add(o[i], z[i]);
    }
  }
  const size_t na = (e.p.w + 1) * e.p.auto_d * N;
  std::fill(auto_out, auto_out + na, 0);
  for (size_t k = 0; k < users; k++)
    for (size_t i = 0; i < na; i++) auto_out[i] = e.rmod.add(auto_out[i], auto_keys[k][i]);
  const size_t nl = (size_t)e.p.lwe_d * N;
  const u64 ql = e.p.lwe_q;
  std::fill(lwe_out, lwe_out + nl, 0);
  for (size_t k = 0; k < users; k++)
    for (size_t i = 0; i < nl; i++) {
      const u64 v = lwe_out[i] + lwe_ksk[k][i];
      lwe_out[i] = v >= ql ? v - ql : v;
    }
  if (i1 <= i0) return;
  std::vector<u64> keval(users * 2 * d * N);
  for (size_t j = 0; j < users; j++) {
    uint8_t seed[32];
    orc_ni_crs_seed(crs, 2, j, seed);
    ChaCha8 prng(seed);
    u64 *k = &keval[j * 2 * d * N];
    for (size_t i = 0; i < d * N; i++) k[i] = prng.uniform_mod(e.Q);
    memcpy(k + d * N, ksk_out + j * d * N, d * N * 8);
    for (size_t r = 0; r < 2 * d; r++) e.ntt.forward(k + r * N, false);
  }
  ni_aggregate_rgsw(e, crs, users, keval.data(), self_leader, not_leader, zero_encs, i0, i1, rgsw_out);
}

// Client side (harness): the auto-key and LWE-KSK B parts under (s, z) with
// their A parts from the CRS streams, as the multi-party share routines
// build them (evaluator.rs:1981-2043 -> seeded_auto_key_gen, rgsw/keygen.rs:
// 306-363; seeded_lwe_ksk_keygen, lwe.rs:46-101): the same encryptions as
// orc_gen_server_key, A rows drawn in the order orc_expand_seeded_key
// regenerates them.  auto_b [w + 1][d_auto][N]; lwe_b [d_ks N].
void orc_gen_seeded_auto_lwe(void *ev, const int32_t *s, const int32_t *z, const uint8_t auto_seed[32],
                             const uint8_t lwe_seed[32], const uint8_t err_seed[32], uint64_t *auto_b,
                             uint64_t *lwe_b) {
  Eval &e = *(Eval *)ev;
  const size_t N = e.N, n = e.n, dauto = e.p.auto_d;
  const u64 Q = e.Q;
  ChaCha8 rng(err_seed), ap(auto_seed), lp(lwe_seed);
  std::vector<u64> s_eval(N), tmp(N), a(N), neg_s_auto(N), sm(N);
  for (size_t i = 0; i < N; i++) s_eval[i] = map_from_i64(Q, s[i]);
  e.ntt.forward(s_eval.data(), false);
  for (size_t i = 0; i < N; i++) sm[i] = map_from_i64(Q, s[i]);
  for (size_t kk = 0; kk <= e.p.w; kk++) {
    const auto &idx = e.auto_idx[kk];
    const auto &sg = e.auto_sign[kk];
    for (size_t i = 0; i < N; i++) neg_s_auto[idx[i]] = sg[i] ? e.rmod.neg(sm[i]) : sm[i];
    for (size_t j = 0; j < dauto; j++) {
      for (size_t i = 0; i < N; i++) a[i] = ap.uniform_mod(Q);
      memcpy(tmp.data(), a.data(), N * 8);
      e.ntt.forward(tmp.data(), false);
      for (size_t i = 0; i < N; i++) tmp[i] = e.rmod.mul(tmp[i], s_eval[i]);
      e.ntt.backward(tmp.data(), false);
      u64 *b = auto_b + (kk * dauto + j) * N;
      const u64 beta = e.dec_auto.gadget((u32)j) % Q;
      for (size_t i = 0; i < N; i++) {
        b[i] = e.rmod.add(map_from_f64(Q, rng.gaussian()), tmp[i]);
        b[i] = e.rmod.add(b[i], e.rmod.mul(neg_s_auto[i] % Q, beta));
      }
    }
  }
  const u64 qk = e.p.lwe_q, mask = qk - 1;
  const size_t d = e.p.lwe_d;
  std::vector<u64> zm(n);
  for (size_t i = 0; i < n; i++) zm[i] = map_from_i64(qk, z[i]) & mask;
  for (size_t i = 0; i < N; i++) {
    const u64 neg_si = (0 - map_from_i64(qk, s[i])) & mask;
    for (size_t j = 0; j < d; j++) {
      u64 az = 0;
      for (size_t c = 0; c < n; c++) az = (az + lp.uniform_mod(qk) * zm[c]) & mask;
      const u64 beta = e.dec_lwe.gadget((u32)j) & mask;
      u64 b = (az + beta * neg_si) & mask;
      lwe_b[i * d + j] = (b + map_from_f64(qk, rng.gaussian())) & mask;
    }
  }
}

// Client side (harness): the NI server key share of gen_non_interactive_
// multi_party_key_share (evaluator.rs:1624-1975) for the RGSW and KSK parts,
// with non_interactive_ksk_gen / _zero_encryptions_for_other_party_i
// (multi_party.rs:186-286): s, u RLWE secrets, z the LWE secret of the user;
// errors from ChaCha8(err_seed).  Outputs: ksk [50][N]; ksk_zero [users-1][50][N];
// self_leader [segment][max(rlrg)][N]; not_leader [n - segment][max(rgrg)][N];
// zero [n][rgrg_d_a][N].
void orc_ni_gen_share(void *ev, const uint8_t crs[32], int user, int users, const int32_t *s, const int32_t *u,
                      const int32_t *z, const uint8_t err_seed[32], uint64_t *ksk, uint64_t *ksk_zero,
                      uint64_t *self_leader, uint64_t *not_leader, uint64_t *zero) {
  Eval &e = *(Eval *)ev;
  const size_t N = e.N, n = e.n, d = e.dec_ni.d, Q = e.Q;
  const size_t ra = e.p.rgrg_d_a, rb = e.p.rgrg_d_b, max_d = std::max(ra, rb);
  const size_t max_l = std::max(e.p.d_a, e.p.d_b);
  const Decomposer &dmax = ra >= rb ? e.dec_rgrg_a : e.dec_rgrg_b;
  const Decomposer &lmax = e.p.d_a >= e.p.d_b ? e.dec_a : e.dec_b;
  ChaCha8 rng(err_seed);
  std::vector<u64> s_eval(N), u_eval(N), tmp(N), m(N);
  for (size_t i = 0; i < N; i++) s_eval[i] = map_from_i64(Q, s[i]);
  for (size_t i = 0; i < N; i++) u_eval[i] = map_from_i64(Q, u[i]);
  e.ntt.forward(s_eval.data(), false);
  e.ntt.forward(u_eval.data(), false);
  auto mul_add_err = [&](u64 *row, const std::vector<u64> &sec) {  // row <- row * sec + e
    e.ntt.forward(row, false);
    for (size_t i = 0; i < N; i++) row[i] = e.rmod.mul(row[i], sec[i]);
    e.ntt.backward(row, false);
    for (size_t i = 0; i < N; i++) row[i] = e.rmod.add(row[i], map_from_f64(Q, rng.gaussian()));
  };
  uint8_t seed[32];
  orc_ni_crs_seed(crs, 2, (size_t)user, seed);
  {  // ui_to_s ksk: a s + e + beta u
    ChaCha8 p(seed);
    for (size_t j = 0; j < d; j++) {
      u64 *row = ksk + j * N;
      for (size_t i = 0; i < N; i++) row[i] = p.uniform_mod(Q);
      mul_add_err(row, s_eval);
      const u64 beta = e.dec_ni.gadget((u32)j) % Q;
      for (size_t i = 0; i < N; i++) row[i] = e.rmod.add(row[i], e.rmod.mul(map_from_i64(Q, u[i]), beta));
    }
  }
  size_t t = 0;
  for (int o = 0; o < users; o++) {  // zero encryptions with the other users' a
    if (o == user) continue;
    orc_ni_crs_seed(crs, 2, (size_t)o, seed);
    ChaCha8 p(seed);
    for (size_t j = 0; j < d; j++) {
      u64 *row = ksk_zero + (t * d + j) * N;
      for (size_t i = 0; i < N; i++) row[i] = p.uniform_mod(Q);
      mul_add_err(row, s_eval);
    }
    t++;
  }
  size_t sb, se;
  lwe_segment((size_t)user, (size_t)users, n, &sb, &se);
  for (size_t li = 0; li < n; li++) {
    orc_ni_crs_seed(crs, 3, li, seed);
    {  // zero encryptions a s + e, after d_max - d_a punctured rows
      ChaCha8 p(seed);
      for (size_t r = 0; r < (max_d - ra) * N; r++) p.uniform_mod(Q);
      for (size_t r = 0; r < ra; r++) {
        u64 *row = zero + (li * ra + r) * N;
        for (size_t i = 0; i < N; i++) row[i] = p.uniform_mod(Q);
        mul_add_err(row, s_eval);
      }
    }
    // X^{emb z_l} (utils.rs:195-217)
    std::fill(m.begin(), m.end(), 0);
    const int64_t si = (int64_t)z[li] * (int64_t)e.emb;
    if (si < 0) m[N - (size_t)(-si)] = Q - 1; else m[(size_t)si] = 1;
    const bool lead = li >= sb && li < se;
    const size_t rows = lead ? max_l : max_d;
    const Decomposer &g = lead ? lmax : dmax;
    u64 *ct = lead ? self_leader + (li - sb) * max_l * N : not_leader + (li < sb ? li : li - (se - sb)) * max_d * N;
    ChaCha8 p(seed);
    for (size_t r = 0; r < (max_d - rows) * N; r++) p.uniform_mod(Q);
    for (size_t r = 0; r < rows; r++) {  // u a + e + beta m
      u64 *row = ct + r * N;
      for (size_t i = 0; i < N; i++) row[i] = p.uniform_mod(Q);
      mul_add_err(row, u_eval);
      const u64 beta = g.gadget((u32)r) % Q;
      for (size_t i = 0; i < N; i++) row[i] = e.rmod.add(row[i], e.rmod.mul(m[i], beta));
    }
  }
}

// Client side (harness): RGSW(m) under s in the rlwe x rgsw shape (which = 0)
// or the rgsw x rgsw shape (which = 1), as the key generation builds them
// (rgsw/keygen.rs:68-160): -sm rows a += beta_j m, b = a s + e; m rows
// b = a s + e + beta_j m.  Coefficient domain.
void orc_rgsw_encrypt(void *ev, const int32_t *s, const uint64_t *m, int which, const uint8_t seed[32],
                      uint64_t *out) {
  Eval &e = *(Eval *)ev;
  const size_t N = e.N;
  const Decomposer &dpa = which ? e.dec_rgrg_a : e.dec_a, &dpb = which ? e.dec_rgrg_b : e.dec_b;
  const size_t da = dpa.d, db = dpb.d;
  ChaCha8 rng(seed);
  std::vector<u64> s_eval(N), tmp(N);
  for (size_t i = 0; i < N; i++) s_eval[i] = map_from_i64(e.Q, s[i]);
  e.ntt.forward(s_eval.data(), false);
  auto rlwe_zero = [&](u64 *a, u64 *b) {  // a uniform, b = a s + e
    for (size_t i = 0; i < N; i++) a[i] = rng.uniform_mod(e.Q);
    memcpy(tmp.data(), a, N * 8);
    e.ntt.forward(tmp.data(), false);
    for (size_t i = 0; i < N; i++) tmp[i] = e.rmod.mul(tmp[i], s_eval[i]);
    e.ntt.backward(tmp.data(), false);
    for (size_t i = 0; i < N; i++) b[i] = e.rmod.add(tmp[i], map_from_f64(e.Q, rng.gaussian()));
  };
  for (size_t j = 0; j < da; j++) {
    u64 *a = out + j * N, *b = out + (da + j) * N;
    rlwe_zero(a, b);
    const u64 beta = dpa.gadget((u32)j) % e.Q;
    for (size_t i = 0; i < N; i++) a[i] = e.rmod.add(a[i], e.rmod.mul(m[i] % e.Q, beta));
  }
  for (size_t j = 0; j < db; j++) {
    u64 *a = out + (2 * da + j) * N, *b = out + (2 * da + db + j) * N;
    rlwe_zero(a, b);
    const u64 beta = dpb.gadget((u32)j) % e.Q;
    for (size_t i = 0; i < N; i++) b[i] = e.rmod.add(b[i], e.rmod.mul(m[i] % e.Q, beta));
  }
}

// ui_to_s key of one user from its B rows and seed (keys.rs:965-1000).
void orc_expand_ni_ksk(void *ev, const uint64_t *b, const uint8_t seed[32], uint64_t *ksk) {
  Eval &e = *(Eval *)ev;
  const size_t N = e.N, d = e.dec_ni.d;
  ChaCha8 prng(seed);
  for (size_t i = 0; i < d * N; i++) ksk[i] = prng.uniform_mod(e.Q);
  memcpy(ksk + d * N, b, d * N * 8);
}

int orc_decrypt_bool(void *ev, const int32_t *s, const uint64_t *lwe) {
  Eval &e = *(Eval *)ev;
  const u64 Q = e.Q;
  u64 sa = 0;
  for (size_t i = 0; i < e.N; i++) sa = e.rmod.add(e.rmod.mul(lwe[1 + i] % Q, map_from_i64(Q, s[i]) % Q), sa);
  return decode_bool(e, e.rmod.sub(lwe[0] % Q, sa));
}

uint64_t orc_mp_decryption_share(void *ev, void *r, const int32_t *s_part, const uint64_t *lwe) {
  Eval &e = *(Eval *)ev;
  ChaCha8 &rng = *(ChaCha8 *)r;
  const u64 Q = e.Q;
  u64 share = 0;
  for (size_t i = 0; i < e.N; i++) {
    u64 neg_si = e.rmod.neg(map_from_i64(Q, s_part[i]) % Q) % Q;
    share = e.rmod.add(share, e.rmod.mul(neg_si, lwe[1 + i] % Q));
  }
  return e.rmod.add(share, map_from_f64(Q, rng.gaussian()));
}

int orc_mp_aggregate_decrypt(void *ev, const uint64_t *lwe, const uint64_t *shares, int parties) {
  Eval &e = *(Eval *)ev;
  u64 sum = 0;
  for (int p = 0; p < parties; p++) sum = e.rmod.add(sum, shares[p]);
  return decode_bool(e, e.rmod.add(lwe[0] % e.Q, sum));
}

}  // extern "C"
