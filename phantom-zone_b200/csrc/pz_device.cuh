// pz_device.cuh -- device building blocks of the gate bootstrap (sm_100a).
//
// Modular arithmetic mod the RLWE prime Q (< 2^62):
//   * NTT butterflies use Shoup multiplication by precomputed twiddles
//     (the butterflies of ntt.rs:24-104): forward values grow without
//     reduction (below 45Q after the 11 stages of N = 2048); inverse values
//     stay in [0, 2Q) (Harvey) for generic q, while for N = 2048 the sums
//     grow to < 16Q inside a radix-8 round and are reduced once per round.
//     For N = 2048 the products and reductions use the special form
//     Q = 2^54 - 77823 of that ring's prime.
//   * The pointwise key product of the blind rotation for N = 2048 reduces
//     its 128-bit sums by folding them with 2^54 = 77823 (mod Q) (three
//     32 x 32-bit multiply-adds); the keys are stored as K * N^{-1} mod Q, so
//     the inverse NTT needs no final N^{-1} scaling.  Other ring sizes, and
//     the general-decomposition products of key aggregation and the
//     non-interactive key switch, use Montgomery REDC with R = 2^64 and keys
//     stored as K * N^{-1} * R mod Q.  Two products are summed in 128 bits
//     before one reduction (the d_a = d_b = 1 external product).
//   All results are exact residues; every value that leaves the device code
//   (coefficient domain) is reduced to [0, Q), which is what makes the output
//   independent of the NTT's internal ordering and lazy ranges.
//
// Block NTT: a CTA of T = N/8 threads holds one polynomial in registers, 8
// coefficients per thread.  Stages are grouped in rounds of three (a radix-8
// step per thread); between rounds the coefficients are re-distributed
// through shared memory.  Only the first forward exchange (last inverse
// exchange) crosses warps; all other exchanges stay inside a warp.  Every
// barrier sits on control flow that is uniform across the block.  Shared
// memory is addressed through the swizzle  pos ^ ((pos >> 4) & 15)  which
// makes every read/write pattern used here bank-conflict free for u64 words.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pz {

typedef uint64_t u64;
typedef uint32_t u32;

struct RingConsts {
  u64 q;         // Q
  u64 qinv_neg;  // -Q^{-1} mod 2^64
  u64 n_inv, n_inv_s;  // N^{-1} mod Q and its Shoup companion
  u64 one_s;            // Shoup companion of 1: reduce_any(v) = v mod Q for any v
  u64 iw1n, iw1n_s;     // psi^{-bitrev(1)} N^{-1} (the last inverse stage's twiddle with N^{-1}) + Shoup
  const u64 *fw;  // forward twiddles: pairs (psi^{bitrev(i)}, Shoup companion)
  const u64 *iw;  // inverse twiddles: pairs (psi^{-bitrev(i)}, Shoup companion)
};

// Signed gadget decomposer, decomposer.rs:158-300.
struct Decomp {
  u64 q;
  u64 bmask, bby2;
  u32 logb, d, ignore_bits;
};

__device__ __forceinline__ u64 umulhi(u64 a, u64 b) { return __umul64hi(a, b); }

// utils.rs:43-46: b*a - q*floor(b_shoup*a / 2^64), result in [0, 2q)
__device__ __forceinline__ u64 shoup_mul(u64 x, u64 w, u64 ws, u64 q) {
  return w * x - umulhi(ws, x) * q;
}

// Montgomery REDC of the 128-bit value (hi, lo) < q * 2^64 -> [0, 2q)
__device__ __forceinline__ u64 redc(u64 hi, u64 lo, u64 q, u64 qinv_neg) {
  u64 m = lo * qinv_neg;
  return hi + umulhi(m, q) + (lo != 0 ? 1ull : 0ull);
}

// hi:lo = x a + y c for x, y < 2^62 (lazy forward outputs: < 150 Q < 2^61.3)
// and a, c < Q (keys): in 32-bit limbs the middle column x0 a1 + x1 a0 +
// y0 c1 + y1 c0 stays below 2^63 + 2^55 and the high column below 2^53, so
// both accumulate with mad.wide and no carries; only the low column and the
// final merge carry.
// 1.7 % more blind-rotation throughput on B200 than two 64 x 64 products in
// C (kept under PZ_MAC_C for comparisons).
__device__ __forceinline__ void sum2_128(u64 x, u64 a, u64 y, u64 c, u64 &hi, u64 &lo) {
#ifndef PZ_MAC_C
  asm("{\n\t"
      ".reg .u32 x0, x1, a0, a1, y0, y1, c0, c1, l0, l1, b0, b1, m0, m1, h0, h1;\n\t"
      ".reg .u64 mid, low, lowb, high;\n\t"
      "mov.b64 {x0, x1}, %2;\n\t"
      "mov.b64 {a0, a1}, %3;\n\t"
      "mov.b64 {y0, y1}, %4;\n\t"
      "mov.b64 {c0, c1}, %5;\n\t"
      "mul.wide.u32 mid, y1, c0;\n\t"
      "mad.wide.u32 mid, y0, c1, mid;\n\t"
      "mad.wide.u32 mid, x1, a0, mid;\n\t"
      "mad.wide.u32 mid, x0, a1, mid;\n\t"
      "mul.wide.u32 high, y1, c1;\n\t"
      "mad.wide.u32 high, x1, a1, high;\n\t"
      "mul.wide.u32 low, x0, a0;\n\t"
      "mul.wide.u32 lowb, y0, c0;\n\t"
      "mov.b64 {l0, l1}, low;\n\t"
      "mov.b64 {b0, b1}, lowb;\n\t"
      "mov.b64 {m0, m1}, mid;\n\t"
      "mov.b64 {h0, h1}, high;\n\t"
      "add.cc.u32 l0, l0, b0;\n\t"
      "addc.cc.u32 l1, l1, b1;\n\t"
      "addc.cc.u32 h0, h0, m1;\n\t"
      "addc.u32 h1, h1, 0;\n\t"
      "add.cc.u32 l1, l1, m0;\n\t"
      "addc.cc.u32 h0, h0, 0;\n\t"
      "addc.u32 h1, h1, 0;\n\t"
      "mov.b64 %0, {h0, h1};\n\t"
      "mov.b64 %1, {l0, l1};\n\t"
      "}"
      : "=l"(hi), "=l"(lo)
      : "l"(x), "l"(a), "l"(y), "l"(c));
#else
  lo = x * a;
  hi = __umul64hi(x, a);
  const u64 l = y * c, h = __umul64hi(y, c);
  lo += l;
  hi += h + (lo < l ? 1ull : 0ull);
#endif
}

__device__ __forceinline__ void mul128(u64 a, u64 b, u64 &hi, u64 &lo) {
  lo = a * b;
  hi = umulhi(a, b);
}
// hi:lo = x a for x < 2^62 and a < 2^54, in 32-bit limb columns: the middle
// column x0 a1 + x1 a0 stays below 2^62 + 2^54, so it accumulates with mad.wide and
// only the merge carries (four multiply-adds against about seven for the
// 64 x 64-bit low and high products).
__device__ __forceinline__ void mul128_narrow(u64 x, u64 a, u64 &hi, u64 &lo) {
  asm("{\n\t"
      ".reg .u32 x0, x1, a0, a1, l0, l1, m0, m1, h0, h1;\n\t"
      ".reg .u64 mid, low, high;\n\t"
      "mov.b64 {x0, x1}, %2;\n\t"
      "mov.b64 {a0, a1}, %3;\n\t"
      "mul.wide.u32 mid, x0, a1;\n\t"
      "mad.wide.u32 mid, x1, a0, mid;\n\t"
      "mul.wide.u32 high, x1, a1;\n\t"
      "mul.wide.u32 low, x0, a0;\n\t"
      "mov.b64 {l0, l1}, low;\n\t"
      "mov.b64 {m0, m1}, mid;\n\t"
      "mov.b64 {h0, h1}, high;\n\t"
      "add.cc.u32 l1, l1, m0;\n\t"
      "addc.cc.u32 h0, h0, m1;\n\t"
      "addc.u32 h1, h1, 0;\n\t"
      "mov.b64 %0, {h0, h1};\n\t"
      "mov.b64 %1, {l0, l1};\n\t"
      "}"
      : "=l"(hi), "=l"(lo)
      : "l"(x), "l"(a));
}
__device__ __forceinline__ void mac128(u64 a, u64 b, u64 &hi, u64 &lo) {
  u64 l = a * b, h = umulhi(a, b);
  lo += l;
  hi += h + (lo < l ? 1ull : 0ull);
}

// add_mod_fast / sub_mod_fast of modulus_u64.rs:46-77 (inputs as there)
__device__ __forceinline__ u64 add_mod(u64 a, u64 b, u64 q) {
  u64 o = a + b;
  return o >= q ? o - q : o;
}
__device__ __forceinline__ u64 sub_mod(u64 a, u64 b, u64 q) { return a >= b ? a - b : (q + a) - b; }

// decompose_iter, decomposer.rs:217-234: sign handling + rounding; returns
// the running state consumed digit by digit by decomp_next.
__device__ __forceinline__ u64 decomp_init(u64 v, const Decomp &dp) {
  if (v >= (dp.q >> 1)) v = v - dp.q;  // == !(q - v) + 1 with wrapping
  if (dp.ignore_bits) v = (v >> dp.ignore_bits) + ((v >> (dp.ignore_bits - 1)) & 1ull);
  return v;
}
// DecomposerIter::next, decomposer.rs:264-300 (branch-free carry)
__device__ __forceinline__ u64 decomp_next(u64 &v, const Decomp &dp) {
  u64 k = v & dp.bmask;
  v = (v - k) >> dp.logb;
  u64 c = (k > dp.bby2 || (k == dp.bby2 && (v & 1ull))) ? 1ull : 0ull;
  v += c;
  return ((0ull - c) & dp.q) + k - (c << dp.logb);
}

// decomp_next with the digit as a signed integer k - c 2^logb (the same
// residue mod q; |digit| <= 2^(logb-1))
__device__ __forceinline__ int decomp_next_signed(u64 &v, const Decomp &dp) {
  const u64 k = v & dp.bmask;
  v = (v - k) >> dp.logb;
  const u64 c = (k > dp.bby2 || (k == dp.bby2 && (v & 1ull))) ? 1ull : 0ull;
  v += c;
  return (int)k - (int)(c << dp.logb);
}

// One-digit decomposition (d = 1) with compile-time base 2^LOGB and IGN
// ignored bits: decomp_init + one decomp_next, with everything after the
// rounding shift in 32-bit arithmetic (the rounded value's digit and its next
// bit sit in the low 32 bits).  The N = 2048 parameter sets all use
// (LOGB, IGN) = (17, 37) for RLWE x RGSW and (24, 30) for automorphisms
// (parameters.rs:526-704; the context checks it).
template <int LOGB, int IGN>
__device__ __forceinline__ u64 decompose1(u64 v, u64 q) {
  static_assert(LOGB < 31 && IGN > 0, "digit and next bit in 32 bits");
  if (v >= (q >> 1)) v = v - q;  // decomposer.rs:217-234 (wrapping)
  const u32 r = (u32)(v >> IGN) + (u32)((v >> (IGN - 1)) & 1ull);
  const u32 k = r & ((1u << LOGB) - 1u), half = 1u << (LOGB - 1);
  const bool c = k > half || (k == half && ((r >> LOGB) & 1u));  // decomposer.rs:264-300
  return c ? q + k - (1ull << LOGB) : (u64)k;
}
constexpr int RLRG_LOGB = 17, RLRG_IGN = 37, AUTO_LOGB = 24, AUTO_IGN = 30;

template <int LOGN>
struct NttShape {
  static_assert(LOGN == 9 || LOGN == 11, "ring dimension 512 or 2048");
  static constexpr int N = 1 << LOGN;
  static constexpr int T = N / 8;          // threads per polynomial
  static constexpr int FULL = LOGN / 3;    // full radix-8 rounds
  static constexpr bool PARTIAL = (LOGN % 3) == 2;  // trailing 2-stage round
};

__device__ __forceinline__ int swz(int pos) { return pos ^ ((pos >> 4) & 15); }

// Position held by thread j in register r in full round k (t_k = N >> (3k+3)).
template <int LOGN>
__device__ __forceinline__ int pos_full(int k, int j, int r) {
  const int t = NttShape<LOGN>::N >> (3 * k + 3);
  return (j / t) * 8 * t + (j % t) + t * r;
}
// Position in the trailing 2-stage round: thread j of warp w holds the
// 4-coefficient groups g1 = 64w + lane and g2 = g1 + 32.
__device__ __forceinline__ int pos_partial(int j, int r) {
  int g = (j >> 5) * 64 + (j & 31) + ((r >> 2) << 5);
  return 4 * g + (r & 3);
}
// Position of register r of thread j in the final forward layout (the
// evaluation-domain layout the MAC and the device keys use).
template <int LOGN>
__device__ __forceinline__ int pos_eval(int j, int r) {
  if (NttShape<LOGN>::PARTIAL) return pos_partial(j, r);
  return pos_full<LOGN>(NttShape<LOGN>::FULL - 1, j, r);
}
// Position in the coefficient layout (round 0): j + T r.
template <int LOGN>
__device__ __forceinline__ int pos_coef(int j, int r) { return j + NttShape<LOGN>::T * r; }

// Device key layout: register pair (r, r+1) of thread j is one 16-byte word.
template <int LOGN>
__device__ __forceinline__ int dev_index(int j, int r) {
  return (r >> 1) * (2 * NttShape<LOGN>::T) + 2 * j + (r & 1);
}

// The RLWE prime of every N = 2048 parameter set (parameters.rs:526-704):
// Q = 2^54 - 77823, so q t mod 2^64 = (t << 54) - 77823 t.
constexpr u64 Q_N2048 = 18014398509404161ull;
__device__ __forceinline__ u64 mulq_n2048(u64 t) { return (t << 54) - t * 77823ull; }

// hi64(a b) without the low partial product and without the carry out of
// the two cross terms' low halves: returns hi64(a b) - c, c in {0, 1, 2}.
__device__ __forceinline__ u64 umulhi_lo2(u64 a, u64 b) {
  const u32 a0 = (u32)a, a1 = (u32)(a >> 32), b0 = (u32)b, b1 = (u32)(b >> 32);
  u64 t = (u64)a1 * b1;
  t += __umulhi(a1, b0);
  t += __umulhi(a0, b1);
  return t;
}

// w v - Q floor~(ws v / 2^64) mod 2^64 for Q = Q_N2048, the quotient from
// umulhi_lo2 (at most 2 short): the Shoup product of the N = 2048 butterflies,
// in [0, 4Q) for any 64-bit v.  It is written in 32-bit PTX so that the
// 64-bit additions ride on the multiply-adds (a 64-bit addend of mad.wide):
// fewer live temporaries, and 6 % more blind-rotation throughput on B200
// than the same arithmetic in C (kept under PZ_BFLY_C for comparisons).
__device__ __forceinline__ u64 shoup_spq(u64 v, u64 w, u64 ws) {
#ifdef PZ_BFLY_C
  return w * v - mulq_n2048(umulhi_lo2(ws, v));
#else
  u64 r;
  asm("{\n\t"
      ".reg .u32 v0, v1, w0, w1, s0, s1, h1, h2, q0, q1, t0, t1, z;\n\t"
      ".reg .u64 qt, wy, t, hs;\n\t"
      "mov.b64 {v0, v1}, %1;\n\t"
      "mov.b64 {w0, w1}, %2;\n\t"
      "mov.b64 {s0, s1}, %3;\n\t"
      "mul.hi.u32 h1, s1, v0;\n\t"
      "mul.hi.u32 h2, s0, v1;\n\t"
      "add.cc.u32 h1, h1, h2;\n\t"
      "addc.u32 h2, 0, 0;\n\t"
      "mov.b64 hs, {h1, h2};\n\t"
      "mad.wide.u32 qt, s1, v1, hs;\n\t"      // quotient, at most 2 short
      "mul.wide.u32 wy, w0, v0;\n\t"
      "mov.b64 {t0, t1}, wy;\n\t"
      "mad.lo.u32 t1, w0, v1, t1;\n\t"
      "mad.lo.u32 t1, w1, v0, t1;\n\t"
      "mov.b64 wy, {t0, t1};\n\t"             // w v mod 2^64
      "mov.b64 {q0, q1}, qt;\n\t"
      "mad.wide.u32 t, q0, 77823, wy;\n\t"    // + 77823 qt (low word of qt)
      "mov.b64 {t0, t1}, t;\n\t"
      "mad.lo.u32 t1, q1, 77823, t1;\n\t"     // + 77823 qt (high word)
      "shl.b32 z, q0, 22;\n\t"
      "sub.u32 t1, t1, z;\n\t"                // - qt 2^54
      "mov.b64 %0, {t0, t1};\n\t"
      "}"
      : "=l"(r)
      : "l"(v), "l"(w), "l"(ws));
  return r;
#endif
}

__device__ __forceinline__ u64 reduce_n2048(u64 v) {
  // 2^54 = 77823 (mod Q): v = h 2^54 + l -> l + 77823 h, < 2^54 + 2^27 < 2Q;
  // h < 2^10, so 77823 h < 2^27 is a 32-bit product
  return (v & ((1ull << 54) - 1)) + (u64)((u32)(v >> 54) * 77823u);
}

// Butterfly products with the quotient estimated on the FP64 pipe (the
// default for N = 2048; PZ_BFLY_SHOUP selects the all-integer Shoup product
// for comparisons).  The twiddle tables hold (w, w/Q as a double) instead of
// (w, Shoup(w)).  On B200 the FP64 pipe runs at the integer multiply pipe's
// rate and concurrently with it, and the 64-bit conversions at about a
// quarter of it on their own unit, so the Shoup quotient -- two IMAD.HI and
// an IMAD.WIDE, 2.5-2.65 times an IMAD each -- moves off the busy pipe:
// v -> vr = reduce_n2048(v) < 2^54 + 2^27, qi = rint(f64(vr) * (w/Q)) within
// 6.51 of vr w / Q (three roundings of 2^-53 each on a value below 2^54),
// and raw = w vr - qi Q (mod 2^64) lies in (-6.51 Q, 6.51 Q) (returned with
// 7 Q added, see fp_raw).  The integer work left is the low words of w vr and
// qi Q (two IMAD.WIDE, three IMAD).
#ifdef PZ_BFLY_SHOUP
constexpr bool BFLY_FP64 = false;
#else
constexpr bool BFLY_FP64 = true;
#endif
// (Magic-number conversions measured slower on B200: both conversions as
// 2^52-offset doubles and an FMA in, the mantissa of qd + 2^55 out, -19 %;
// the out conversion alone that way, -10 %: the extra ALU and FP64
// instructions cost more issue slots than the conversion unit's quarter
// rate does.)
constexpr u64 FP_OFF = 7;  // raw + 7 Q in (0.49 Q, 13.51 Q)
// fp_raw returns raw + FP_OFF Q: the offset rides on the quotient as
// qi = rint(f64(vr) (w/Q) - FP_OFF) (one FMA, signed: qi may be negative),
// so w vr - qi Q mod 2^64 is already in (0.49 Q, 13.51 Q).
__device__ __forceinline__ u64 fp_raw(u64 v, u64 w, u64 wq_bits) {
  const u64 vr = reduce_n2048(v);
  u64 qi, r;
  double vd;
  asm("cvt.rn.f64.u64 %0, %1;" : "=d"(vd) : "l"(vr));
  const double qd = __fma_rn(vd, __longlong_as_double((long long)wq_bits), -(double)FP_OFF);
  asm("cvt.rni.s64.f64 %0, %1;" : "=l"(qi) : "d"(qd));
  asm("{\n\t"
      ".reg .u32 v0, v1, w0, w1, q0, q1, t0, t1, z;\n\t"
      ".reg .u64 wy, t;\n\t"
      "mov.b64 {v0, v1}, %1;\n\t"
      "mov.b64 {w0, w1}, %2;\n\t"
      "mov.b64 {q0, q1}, %3;\n\t"
      "mul.wide.u32 wy, w0, v0;\n\t"
      "mov.b64 {t0, t1}, wy;\n\t"
      "mad.lo.u32 t1, w0, v1, t1;\n\t"
      "mad.lo.u32 t1, w1, v0, t1;\n\t"
      "mov.b64 wy, {t0, t1};\n\t"            // w vr mod 2^64
      "mad.wide.u32 t, q0, 77823, wy;\n\t"   // + 77823 qi (low word of qi)
      "mov.b64 {t0, t1}, t;\n\t"
      "mad.lo.u32 t1, q1, 77823, t1;\n\t"    // + 77823 qi (high word)
      "shl.b32 z, q0, 22;\n\t"
      "sub.u32 t1, t1, z;\n\t"               // - qi 2^54
      "mov.b64 %0, {t0, t1};\n\t"
      "}"
      : "=l"(r)
      : "l"(vr), "l"(w), "l"(qi));
  return r;
}

// Forward CT butterfly (the x' = x + wy, y' = x - wy of ntt.rs:31-49) without
// Harvey's conditional subtraction: wy is a Shoup product, so both outputs
// grow by a bounded multiple of q per stage and the Shoup product accepts any
// 64-bit input, so no stage needs a reduction.  Generic q: wy in [0, 2q),
// growth 2q per stage (< 23q after the 11 stages of N = 2048 from inputs
// < q).  Q_N2048 (SPQ): the quotient from umulhi_lo2 is at most 2 short, so
// wy in [0, 4q), growth 4q per stage (< 45q < 2^60 after 11 stages), and
// q * quotient comes from the special form of Q; with the FP64 quotient
// (fp_raw, the default) the growth is < 13.51 Q per stage (< 150 Q).
// x + t and x + c - t as explicit 32-bit carry chains (PZ_BFLY_ADD_PTX, a
// same-box comparison): the high words' carries as addc / subc.
__device__ __forceinline__ void add_sub_ptx(u64 x, u64 t, u64 c, u64 &sum, u64 &dif) {
  asm("{\n\t"
      ".reg .u32 x0, x1, t0, t1, c0, c1, s0, s1, d0, d1;\n\t"
      "mov.b64 {x0, x1}, %2;\n\t"
      "mov.b64 {t0, t1}, %3;\n\t"
      "mov.b64 {c0, c1}, %4;\n\t"
      "add.cc.u32 s0, x0, t0;\n\t"
      "addc.u32 s1, x1, t1;\n\t"
      "add.cc.u32 d0, x0, c0;\n\t"
      "addc.u32 d1, x1, c1;\n\t"
      "sub.cc.u32 d0, d0, t0;\n\t"
      "subc.u32 d1, d1, t1;\n\t"
      "mov.b64 %0, {s0, s1};\n\t"
      "mov.b64 %1, {d0, d1};\n\t"
      "}"
      : "=l"(sum), "=l"(dif)
      : "l"(x), "l"(t), "l"(c));
}

template <bool SPQ>
__device__ __forceinline__ void fbf(u64 &x, u64 &y, u64 w, u64 ws, u64 q) {
  if (SPQ && BFLY_FP64) {  // outputs grow by < 13.51 Q per stage (< 150 Q after 11)
    const u64 r7 = fp_raw(y, w, ws);  // w y + 7 Q (mod Q), in (0.49 Q, 13.51 Q)
    y = x + 2 * FP_OFF * Q_N2048 - r7;
    x = x + r7;
  } else if (SPQ) {
    const u64 t = shoup_spq(y, w, ws);
#ifdef PZ_BFLY_ADD_PTX
    add_sub_ptx(x, t, Q_N2048 << 2, x, y);
#else
    y = x + (Q_N2048 << 2) - t;
    x = x + t;
#endif
  } else {
    const u64 t = shoup_mul(y, w, ws, q);
    y = x + (q << 1) - t;
    x = x + t;
  }
}
// Inverse GS butterfly (x' = x + y, y' = w (x - y), ntt.rs:84-104).  Generic
// q: Harvey's form (x, y < 2q -> x', y' < 2q).  Q_N2048 (SPQ): no reduction of
// the sum -- the rounds let sums grow to < 16 Q and reduce once per round
// with reduce_n2048 -- and y' is a Shoup product whose quotient comes from
// umulhi_lo2 (at most 2 short beyond Shoup's own 1), so y' in [0, 4Q); K Q
// must bound the incoming y (the caller's stage bound: inputs < 2Q, then
// outputs < 4Q after one stage and < 8Q after two, hence K = 2, 4, 8; the
// trailing round that opens the N = 2048 inverse takes inputs < 2.04 Q --
// the blind rotation's folded multiply-accumulates -- hence K = 3, 5 there).

// The blind rotation's multiply-accumulate reduction for N = 2048 (the
// default; PZ_MAC_MONT selects Montgomery REDC there too, for comparisons):
// X = hi 2^64 + lo with hi < 2^52 is X = (lo mod 2^54) + 2^54 u,
// u = hi 2^10 + (lo >> 54) < 2^62, and 2^54 = 77823 (mod Q), so
// X = (lo mod 2^54) + 77823 u0 + 77823 u1 2^32 with u = u1 2^32 + u0; the
// last term, p 2^32 with p = 77823 u1 < 2^47, is (p mod 2^22) 2^32 +
// 77823 (p >> 22).  The result is congruent to X and below
// 2^55 + 2^49 + 2^42 < 2.04 Q: three multiply-adds (two with the 64-bit
// addend riding on them) instead of REDC's 64-bit low and high products.
#ifdef PZ_MAC_MONT
constexpr bool MAC_FOLD_N2048 = false;
#else
constexpr bool MAC_FOLD_N2048 = true;
#endif
__device__ __forceinline__ u64 fold_n2048(u64 hi, u64 lo) {
  u64 r;
  asm("{\n\t"
      ".reg .u32 l0, l1, h0, h1, u0, u1, p0, p1, ph, b1;\n\t"
      ".reg .u64 p, base;\n\t"
      "mov.b64 {l0, l1}, %1;\n\t"
      "mov.b64 {h0, h1}, %2;\n\t"
      "shf.l.wrap.b32 u0, l1, h0, 10;\n\t"    // u mod 2^32
      "shf.l.wrap.b32 u1, h0, h1, 10;\n\t"    // u >> 32 (< 2^30)
      "mul.wide.u32 p, u1, 77823;\n\t"
      "mov.b64 {p0, p1}, p;\n\t"
      "shf.r.wrap.b32 ph, p0, p1, 22;\n\t"    // p >> 22 (< 2^25)
      "and.b32 p0, p0, 0x3FFFFF;\n\t"         // p mod 2^22
      "and.b32 b1, l1, 0x3FFFFF;\n\t"         // (lo mod 2^54) >> 32
      "add.u32 b1, b1, p0;\n\t"
      "mov.b64 base, {l0, b1};\n\t"           // (lo mod 2^54) + (p mod 2^22) 2^32
      "mad.wide.u32 base, u0, 77823, base;\n\t"
      "mad.wide.u32 %0, ph, 77823, base;\n\t"
      "}"
      : "=l"(r)
      : "l"(lo), "l"(hi));
  return r;
}
// Reduction of a multiply-accumulate's 128-bit sum (hi < 2^52): for N = 2048
// the fold above (< 2.04 Q, keys K N^{-1}), else Montgomery REDC (< 2 Q, keys
// K N^{-1} 2^64).  Both are exact residues of the same product.
template <int LOGN>
__device__ __forceinline__ u64 mac_reduce(u64 hi, u64 lo, u64 q, u64 qinv_neg) {
  if constexpr (LOGN == 11 && MAC_FOLD_N2048) return fold_n2048(hi, lo);
  else return redc(hi, lo, q, qinv_neg);
}
// The automorphism's b: product + permuted b (each < 2.04 Q for N = 2048,
// < 2q otherwise), back below 2q.
template <int LOGN>
__device__ __forceinline__ void mac_mul(u64 x, u64 a, u64 &hi, u64 &lo) {
  if constexpr (LOGN == 11) mul128_narrow(x, a, hi, lo);  // x < 150 Q < 2^62, a < Q < 2^54
  else mul128(x, a, hi, lo);
}
template <int LOGN>
__device__ __forceinline__ u64 mac_add_b(u64 v, u64 q2) {
  if constexpr (LOGN == 11 && MAC_FOLD_N2048) return reduce_n2048(v);
  else return v >= q2 ? v - q2 : v;
}

// Stage bounds K of the N = 2048 inverse rounds (stages a, b, c of a round;
// the round that opens an inverse after the multiply-accumulates takes
// inputs < 2.04 Q in stage a, K = 3, and IK_MB in stage b).  The Shoup
// products leave < 4 Q: sums < 4, 8, 16 Q.  The FP64-quotient products
// leave < 13.51 Q: stage b sees < 13.51 Q, stage c < 27.02 Q.
constexpr int IK_B = BFLY_FP64 ? 14 : 4, IK_C = BFLY_FP64 ? 28 : 8, IK_MB = BFLY_FP64 ? 14 : 5;

template <bool SPQ, int K>
__device__ __forceinline__ void ibf(u64 &x, u64 &y, u64 w, u64 ws, u64 q) {
  if (SPQ) {
#ifdef PZ_BFLY_ADD_PTX
    u64 u, t;
    add_sub_ptx(x, y, (u64)K * Q_N2048, u, t);
#else
    const u64 t = x + (u64)K * Q_N2048 - y;
    const u64 u = x + y;
#endif
    y = BFLY_FP64 ? fp_raw(t, w, ws) : shoup_spq(t, w, ws);
    x = u;
  } else {
    const u64 q2 = q << 1;
    u64 u = x + y;
    if (u >= q2) u -= q2;
    const u64 t = x + q2 - y;
    y = shoup_mul(t, w, ws, q);
    x = u;
  }
}

__device__ __forceinline__ u64 ldg(const u64 *p) { return __ldg(p); }

// ---------------------------------------------------------------------------
// Single-polynomial block NTT: three radix-8 rounds (plus the trailing
// 2-stage round for N = 2048).  The transform is called once per polynomial,
// so the whole blind rotation holds a single forward and a single inverse
// copy.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void sync_exchange(bool cross) {
  if (cross) __syncthreads();
  else __syncwarp();
}

// threadIdx.x read afresh: addresses derived from it are recomputed inside
// each transform instead of being hoisted out of the blind-rotation loop and
// kept live in registers for the whole kernel.
__device__ __forceinline__ int tid_opaque() {
  int t;
  asm volatile("mov.u32 %0, %%tid.x;" : "=r"(t));
  return t;
}

// Twiddle pair (w, Shoup(w)) at index i of an interleaved table (one 16-byte
// load).  A volatile asm load, unlike __ldg (an invariant load the compiler
// may hoist out of the transform and keep live), stays inside its round.
__device__ __forceinline__ void tw(const u64 *t, int i, u64 &w, u64 &ws) {
  asm volatile("ld.global.nc.v2.u64 {%0, %1}, [%2];" : "=l"(w), "=l"(ws) : "l"(t + 2 * i));
}

// The transforms below act on one polynomial (x) or, with TWO, on two (x and
// y) at once: both use the same twiddle loads, the same barriers and the same
// exchange steps (y through the second N words of sm), and their butterflies
// are independent instruction streams.  A single-polynomial call passes its
// array as both x and y.
// N = 2048 transforms run modulo Q_N2048 (the context checks it).
template <int LOGN, bool TWO>
__device__ __forceinline__ void fbf2(u64 (&x)[8], u64 (&y)[8], int a, int b, u64 w, u64 ws, u64 q) {
  fbf<LOGN == 11>(x[a], x[b], w, ws, q);
  if (TWO) fbf<LOGN == 11>(y[a], y[b], w, ws, q);
}
template <int LOGN, bool TWO, int K>
__device__ __forceinline__ void ibf2(u64 (&x)[8], u64 (&y)[8], int a, int b, u64 w, u64 ws, u64 q) {
  ibf<LOGN == 11, K>(x[a], x[b], w, ws, q);
  if (TWO) ibf<LOGN == 11, K>(y[a], y[b], w, ws, q);
}
// With the FP64-quotient butterflies the round that opens an inverse
// transform (2 stages, inputs < 2.04 Q, K = 3 and 14) skips its reduction
// (PZ_INV_REDUCE_EVERY_ROUND: reduces, a comparison): its products leave
// < 13.51 Q whatever their input, so its sums stay < 27.02 Q, and every
// radix-8 round takes inputs that large (K = 28, 55, 109; sums < 216.2 Q)
// before its own reduction.
#ifdef PZ_INV_REDUCE_EVERY_ROUND
constexpr bool INV_SKIP = false;
#else
constexpr bool INV_SKIP = BFLY_FP64;
#endif
constexpr int IK_A8 = INV_SKIP ? 28 : 2, IK_B8 = INV_SKIP ? 55 : IK_B, IK_C8 = INV_SKIP ? 109 : IK_C;

// End of an inverse round for N = 2048: every value back below 2Q.
template <int LOGN, bool TWO>
__device__ __forceinline__ void inv_round_reduce(u64 (&x)[8], u64 (&y)[8]) {
  if constexpr (LOGN == 11) {
#pragma unroll
    for (int r = 0; r < 8; r++) {
      x[r] = reduce_n2048(x[r]);
      if (TWO) y[r] = reduce_n2048(y[r]);
    }
  }
}

// Forward radix-8 round k: stages with m = 8^k, 2m and 4m groups; blk is the
// group index of this thread in the first of them.  PF: the round's seven
// twiddle pairs are all loaded before its first butterfly (one load latency
// per round instead of one per stage; 14 more live registers).
template <int LOGN, bool TWO, bool PF = false>
__device__ __forceinline__ void fwd_round8(u64 (&x)[8], u64 (&y)[8], int k, int j, const RingConsts &rc) {
  const int m = 1 << (3 * k);
  const int blk = j >> (LOGN - 3 * k - 3);
  const u64 q = rc.q;
  u64 w[7], ws[7];  // slots: 0 (stage m), 1-2 (stage 2m), 3-6 (stage 4m)
  if (PF) {
    tw(rc.fw, m + blk, w[0], ws[0]);
#pragma unroll
    for (int h = 0; h < 2; h++) tw(rc.fw, 2 * m + 2 * blk + h, w[1 + h], ws[1 + h]);
#pragma unroll
    for (int h = 0; h < 4; h++) tw(rc.fw, 4 * m + 4 * blk + h, w[3 + h], ws[3 + h]);
  }
  if (!PF) tw(rc.fw, m + blk, w[0], ws[0]);
#pragma unroll
  for (int r = 0; r < 4; r++) fbf2<LOGN, TWO>(x, y, r, r + 4, w[0], ws[0], q);
#pragma unroll
  for (int h = 0; h < 2; h++) {
    if (!PF) tw(rc.fw, 2 * m + 2 * blk + h, w[1 + h], ws[1 + h]);
    fbf2<LOGN, TWO>(x, y, 4 * h + 0, 4 * h + 2, w[1 + h], ws[1 + h], q);
    fbf2<LOGN, TWO>(x, y, 4 * h + 1, 4 * h + 3, w[1 + h], ws[1 + h], q);
  }
#pragma unroll
  for (int h = 0; h < 4; h++) {
    if (!PF) tw(rc.fw, 4 * m + 4 * blk + h, w[3 + h], ws[3 + h]);
    fbf2<LOGN, TWO>(x, y, 2 * h, 2 * h + 1, w[3 + h], ws[3 + h], q);
  }
}

// The round's three stages with compile-time bounds (IK_A8..C8 above; the
// Shoup butterflies: inputs < 2Q, sums < 4Q, 8Q, 16Q), then the once-per-round
// reduction.
template <int LOGN, bool TWO, bool PF>
__device__ __forceinline__ void inv_round8_stages(u64 (&x)[8], u64 (&y)[8], int m, int blk, u64 (&w)[7],
                                                  u64 (&ws)[7], const RingConsts &rc) {
  const u64 q = rc.q;
#pragma unroll
  for (int h = 0; h < 4; h++) {
    if (!PF) tw(rc.iw, 4 * m + 4 * blk + h, w[h], ws[h]);
    ibf2<LOGN, TWO, IK_A8>(x, y, 2 * h, 2 * h + 1, w[h], ws[h], q);
  }
#pragma unroll
  for (int h = 0; h < 2; h++) {
    if (!PF) tw(rc.iw, 2 * m + 2 * blk + h, w[4 + h], ws[4 + h]);
    ibf2<LOGN, TWO, IK_B8>(x, y, 4 * h + 0, 4 * h + 2, w[4 + h], ws[4 + h], q);
    ibf2<LOGN, TWO, IK_B8>(x, y, 4 * h + 1, 4 * h + 3, w[4 + h], ws[4 + h], q);
  }
  if (!PF) tw(rc.iw, m + blk, w[6], ws[6]);
#pragma unroll
  for (int r = 0; r < 4; r++) ibf2<LOGN, TWO, IK_C8>(x, y, r, r + 4, w[6], ws[6], q);
  inv_round_reduce<LOGN, TWO>(x, y);
}

template <int LOGN, bool TWO, bool PF = false>
__device__ __forceinline__ void inv_round8(u64 (&x)[8], u64 (&y)[8], int k, int j, const RingConsts &rc) {
  const int m = 1 << (3 * k);
  const int blk = j >> (LOGN - 3 * k - 3);
  u64 w[7], ws[7];  // slots: 0-3 (stage 4m), 4-5 (stage 2m), 6 (stage m)
  if (PF) {
#pragma unroll
    for (int h = 0; h < 4; h++) tw(rc.iw, 4 * m + 4 * blk + h, w[h], ws[h]);
#pragma unroll
    for (int h = 0; h < 2; h++) tw(rc.iw, 2 * m + 2 * blk + h, w[4 + h], ws[4 + h]);
    tw(rc.iw, m + blk, w[6], ws[6]);
  }
  inv_round8_stages<LOGN, TWO, PF>(x, y, m, blk, w, ws, rc);
}

// Trailing 2-stage round (stages with N/4 and N/2 groups); PF as for the
// radix-8 rounds (six twiddle pairs).
template <int LOGN, bool TWO, bool PF = false>
__device__ __forceinline__ void fwd_round4(u64 (&x)[8], u64 (&y)[8], int j, const RingConsts &rc) {
  constexpr int N = 1 << LOGN;
  const u64 q = rc.q;
  u64 w[6], ws[6];  // per h: slot 3h (stage N/4), 3h + 1 + e (stage N/2)
  if (PF) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int g = (j >> 5) * 64 + (j & 31) + (h << 5);
      tw(rc.fw, N / 4 + g, w[3 * h], ws[3 * h]);
#pragma unroll
      for (int e = 0; e < 2; e++) tw(rc.fw, N / 2 + 2 * g + e, w[3 * h + 1 + e], ws[3 * h + 1 + e]);
    }
  }
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int g = (j >> 5) * 64 + (j & 31) + (h << 5);
    if (!PF) tw(rc.fw, N / 4 + g, w[3 * h], ws[3 * h]);
    fbf2<LOGN, TWO>(x, y, 4 * h + 0, 4 * h + 2, w[3 * h], ws[3 * h], q);
    fbf2<LOGN, TWO>(x, y, 4 * h + 1, 4 * h + 3, w[3 * h], ws[3 * h], q);
#pragma unroll
    for (int e = 0; e < 2; e++) {
      if (!PF) tw(rc.fw, N / 2 + 2 * g + e, w[3 * h + 1 + e], ws[3 * h + 1 + e]);
      fbf2<LOGN, TWO>(x, y, 4 * h + 2 * e, 4 * h + 2 * e + 1, w[3 * h + 1 + e], ws[3 * h + 1 + e], q);
    }
  }
}

template <int LOGN, bool TWO, bool PF = false>
__device__ __forceinline__ void inv_round4(u64 (&x)[8], u64 (&y)[8], int j, const RingConsts &rc) {
  constexpr int N = 1 << LOGN;
  const u64 q = rc.q;
  u64 w[6], ws[6];  // per h: slots 3h + e (stage N/2), 3h + 2 (stage N/4)
  if (PF) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int g = (j >> 5) * 64 + (j & 31) + (h << 5);
#pragma unroll
      for (int e = 0; e < 2; e++) tw(rc.iw, N / 2 + 2 * g + e, w[3 * h + e], ws[3 * h + e]);
      tw(rc.iw, N / 4 + g, w[3 * h + 2], ws[3 * h + 2]);
    }
  }
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int g = (j >> 5) * 64 + (j & 31) + (h << 5);
#pragma unroll
    for (int e = 0; e < 2; e++) {
      if (!PF) tw(rc.iw, N / 2 + 2 * g + e, w[3 * h + e], ws[3 * h + e]);
      ibf2<LOGN, TWO, 3>(x, y, 4 * h + 2 * e, 4 * h + 2 * e + 1, w[3 * h + e], ws[3 * h + e], q);
    }
    if (!PF) tw(rc.iw, N / 4 + g, w[3 * h + 2], ws[3 * h + 2]);
    ibf2<LOGN, TWO, IK_MB>(x, y, 4 * h + 0, 4 * h + 2, w[3 * h + 2], ws[3 * h + 2], q);
    ibf2<LOGN, TWO, IK_MB>(x, y, 4 * h + 1, 4 * h + 3, w[3 * h + 2], ws[3 * h + 2], q);
  }
  if (!INV_SKIP) inv_round_reduce<LOGN, TWO>(x, y);  // (N = 2048) sums < 8.2Q -> < 2Q
}

// Layout of full round k: thread j holds base + t r, t = N >> (3k + 3).
template <int LOGN>
__device__ __forceinline__ int base_full(int k, int j) {
  const int lt = LOGN - 3 * k - 3;
  return ((j >> lt) << (lt + 3)) + (j & ((1 << lt) - 1));
}

// Swizzled exchange-buffer address of register r in layout L (0..2: full
// rounds, 3: trailing round).  For N = 2048 the per-thread base absorbs the
// swizzle: in every layout the coefficient position is a disjoint union of
// bit fields from the warp, the lane and r, so swz(pos) reduces to one XOR
// (and at most an immediate offset) per register.  Other sizes use swz()
// directly.
template <int LOGN, int L>
__device__ __forceinline__ int xbase(int j) {
  if constexpr (LOGN == 11) {
    const int w = j >> 5, l = j & 31;
    if constexpr (L == 0) return j ^ ((j >> 4) & 15);                       // pos = j + 256 r
    else if constexpr (L == 1) return (w << 8) + (l ^ (l >> 4));            // 256 w + l + 32 r
    else if constexpr (L == 2) return ((w << 8) + ((l >> 2) << 5) + (l & 3)) ^ ((l >> 2) << 1);  // + 4 r
    else return ((w << 8) + (l << 2)) ^ (l >> 2);                           // 256 w + 4 l + 128 h + e
  } else {
    return L < 3 ? base_full<LOGN>(L, j) : 0;
  }
}
template <int LOGN, int L>
__device__ __forceinline__ int xaddr(int b, int j, int r) {
  if constexpr (LOGN == 11) {
    if constexpr (L == 0) return b + (r << 8);
    else if constexpr (L == 1) return (b ^ (r << 1)) + (r << 5);
    else if constexpr (L == 2) return b ^ ((r << 2) ^ (r >> 2));
    else return b ^ ((r & 3) ^ ((r >> 2) << 3) ^ ((r >> 2) << 7));
  } else {
    return L < 3 ? swz(b + (r << (LOGN - 3 * L - 3))) : swz(pos_partial(j, r));
  }
}

// Move the polynomial(s) from layout LF to layout LT through sm (N words per
// polynomial).
template <int LOGN, int LF, int LT, bool TWO>
__device__ __forceinline__ void xchg(u64 (&x)[8], u64 (&y)[8], u64 *sm, int j) {
  constexpr int N = 1 << LOGN;
  constexpr bool cross = (LF == 0 || LT == 0);
  const int bf = xbase<LOGN, LF>(j), bt = xbase<LOGN, LT>(j);
  sync_exchange(cross);
#pragma unroll
  for (int r = 0; r < 8; r++) {
    const int a = xaddr<LOGN, LF>(bf, j, r);
    sm[a] = x[r];
    if (TWO) sm[N + a] = y[r];
  }
  sync_exchange(cross);
#pragma unroll
  for (int r = 0; r < 8; r++) {
    const int a = xaddr<LOGN, LT>(bt, j, r);
    x[r] = sm[a];
    if (TWO) y[r] = sm[N + a];
  }
}

// Forward negacyclic NTT (CT, ntt.rs:110-143 without reductions): coefficient
// layout in, values < q; evaluation layout out, values < 150 q (see fbf).
// sm: N words (2N with TWO).  The rounds run in a loop (one copy of the round
// body); the exchanges between them are layout-specialised and picked by a
// block-uniform switch.
template <int LOGN, bool TWO, bool PF = false>
__device__ __forceinline__ void ntt_fwd(u64 (&x)[8], u64 (&y)[8], u64 *sm, const RingConsts &rc) {
  typedef NttShape<LOGN> S;
  static_assert(S::FULL == 3, "three radix-8 rounds");
  const int j = tid_opaque();
#pragma unroll 1
  for (int k = 0; k < 3; k++) {
    if (k == 1) xchg<LOGN, 0, 1, TWO>(x, y, sm, j);
    else if (k == 2) xchg<LOGN, 1, 2, TWO>(x, y, sm, j);
    fwd_round8<LOGN, TWO, PF>(x, y, k, j, rc);
  }
  if constexpr (S::PARTIAL) {
    xchg<LOGN, 2, 3, TWO>(x, y, sm, j);
    fwd_round4<LOGN, TWO, PF>(x, y, j, rc);
  }
}

// Inverse negacyclic NTT (GS, ntt.rs:187-230 without the N^{-1} factor):
// evaluation layout in, values < 2q; coefficient layout out, values < 2q.
// sm: N words (2N with TWO).
// LEAD_SYNC = false: the caller has just passed a block barrier after its
// last use of sm.
template <int LOGN, bool TWO, bool LEAD_SYNC = true>
__device__ __forceinline__ void ntt_inv(u64 (&x)[8], u64 (&y)[8], u64 *sm, const RingConsts &rc) {
  typedef NttShape<LOGN> S;
  const int j = tid_opaque();
  // The first exchange below is warp-local, but the previous user of sm may
  // have read it across warps (a transform's last exchange): full barrier.
  if (LEAD_SYNC) __syncthreads();
  if constexpr (S::PARTIAL) {
    inv_round4<LOGN, TWO>(x, y, j, rc);
    xchg<LOGN, 3, 2, TWO>(x, y, sm, j);
  }
#pragma unroll 1
  for (int k = 2; k >= 0; k--) {
    inv_round8<LOGN, TWO>(x, y, k, j, rc);
    if (k == 2) xchg<LOGN, 2, 1, TWO>(x, y, sm, j);
    else if (k == 1) xchg<LOGN, 1, 0, TWO>(x, y, sm, j);
  }
}

// Single-polynomial forms.
template <int LOGN>
__device__ __forceinline__ void ntt_fwd(u64 (&x)[8], u64 *sm, const RingConsts &rc) {
  ntt_fwd<LOGN, false>(x, x, sm, rc);
}
template <int LOGN>
__device__ __forceinline__ void ntt_inv(u64 (&x)[8], u64 *sm, const RingConsts &rc) {
  ntt_inv<LOGN, false>(x, x, sm, rc);
}

// Automorphism X -> X^k (k odd) in the evaluation domain.  The forward
// transform leaves a(psi^(2 brv(p) + 1)) at position p, so a(X^k) holds at p
// the value found at p' with 2 brv(p') + 1 = (2 brv(p) + 1) k mod 2N: a
// permutation of positions (the ring automorphism, signs included).
template <int LOGN>
__device__ __forceinline__ int auto_eval_src(int p, u32 k) {
  const u32 e = 2u * (__brev((u32)p) >> (32 - LOGN)) + 1u;
  const u32 e2 = (e * k) & ((2u << LOGN) - 1u);
  return (int)(__brev((e2 - 1u) >> 1) >> (32 - LOGN));
}

__device__ __forceinline__ u64 reduce4(u64 v, u64 q) {  // [0,4q) -> [0,q)
  const u64 q2 = q << 1;
  if (v >= q2) v -= q2;
  if (v >= q) v -= q;
  return v;
}
__device__ __forceinline__ u64 reduce2(u64 v, u64 q) { return v >= q ? v - q : v; }
// any 64-bit v -> [0, q)
__device__ __forceinline__ u64 reduce_any(u64 v, const RingConsts &rc) {
  return reduce2(shoup_mul(v, 1, rc.one_s, rc.q), rc.q);
}

// 16-byte read-only load that does not allocate in L1 (keys stream through L2).
__device__ __forceinline__ void ld_key2(const u64 *p, u64 &a, u64 &b) {
  asm volatile("ld.global.nc.L1::no_allocate.v2.u64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "l"(p));
}

// Load one device-layout key row into the evaluation layout registers.
template <int LOGN>
__device__ __forceinline__ void load_key_row(const u64 *row, u64 (&k)[8]) {
  const int j = threadIdx.x;
#pragma unroll
  for (int rr = 0; rr < 4; rr++) ld_key2(row + dev_index<LOGN>(j, 2 * rr), k[2 * rr], k[2 * rr + 1]);
}

// ---------------------------------------------------------------------------
// Bulk copies into shared memory (cp.async.bulk, completion counted on an
// mbarrier in bytes).  Sources are this GPU's global memory; no multicast.
// ---------------------------------------------------------------------------
__device__ __forceinline__ u32 smem_addr(const void *p) { return (u32)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(u64 *bar, u32 count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
// make initialised mbarriers visible to the bulk-copy unit (then a block barrier)
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// order this thread's earlier shared-memory accesses before later bulk copies
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// One thread: `bytes` (multiple of 16, both addresses 16-byte aligned) from
// global src to shared dst; completes one phase of *bar (initialised with one
// arrival).
__device__ __forceinline__ void bulk_load(void *dst, const void *src, u32 bytes, u64 *bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
// Wait for the phase of *bar with the given parity to complete, for at most
// about `limit` SM clock cycles; false when the limit ran out.
constexpr long long MBAR_WAIT_LIMIT = 1ll << 31;  // ~1.1 s at 1965 MHz
__device__ __forceinline__ bool mbar_wait(u64 *bar, u32 parity, long long limit = MBAR_WAIT_LIMIT) {
  const u32 a = smem_addr(bar);
  const long long t0 = clock64();
  for (;;) {
    u32 done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > limit) return false;
  }
}
// One thread: ask L2 to fetch `bytes` (a multiple of 16, 16-byte aligned)
// from global memory ahead of their use; no completion to wait for.  Used for
// key rows an operation will read after its transforms (PZ_NO_L2_PF: off,
// for comparisons).
__device__ __forceinline__ void prefetch_l2(const void *p, u32 bytes) {
#ifndef PZ_NO_L2_PF
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
#endif
}

// Error bits a kernel sets in the context's device error word.
constexpr u32 DEVERR_MBAR_TIMEOUT = 1u;

}  // namespace pz
