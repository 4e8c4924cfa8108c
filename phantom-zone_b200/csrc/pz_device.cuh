// pz_device.cuh -- device building blocks of the gate bootstrap (sm_100a).
//
// Modular arithmetic mod the RLWE prime Q (< 2^62):
//   * NTT butterflies use Shoup multiplication by precomputed twiddles
//     (Harvey's lazy butterflies, the algorithm of ntt.rs:24-104): forward
//     values live in [0, 4Q), inverse values in [0, 2Q).
//   * The pointwise key product uses Montgomery REDC with R = 2^64.  Device
//     keys are stored as K * N^{-1} * R mod Q, so REDC(x * K') = x * K * N^{-1}
//     and the inverse NTT needs no final N^{-1} scaling.  Two products are
//     summed in 128 bits before one REDC (the d_a = d_b = 1 external product).
//   All results are exact residues; every value that leaves the device code
//   (coefficient domain) is reduced to [0, Q), which is what makes the output
//   independent of the NTT's internal ordering and lazy ranges.
//
// Block NTT: a CTA of T = N/8 threads holds one polynomial in registers, 8
// coefficients per thread.  Stages are grouped in rounds of three (a radix-8
// step per thread); between rounds the coefficients are re-distributed
// through shared memory.  Only the first forward exchange (last inverse
// exchange) crosses warps; all other exchanges stay inside a warp.  Shared
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
  const u64 *fw, *fws;  // forward twiddles psi^{bitrev(i)}, Shoup companions
  const u64 *iw, *iws;  // inverse twiddles psi^{-bitrev(i)}, Shoup companions
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

__device__ __forceinline__ void mul128(u64 a, u64 b, u64 &hi, u64 &lo) {
  lo = a * b;
  hi = umulhi(a, b);
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

// Harvey forward butterfly, ntt.rs:31-49 (x, y < 4q -> x', y' < 4q)
__device__ __forceinline__ void fbf(u64 &x, u64 &y, u64 w, u64 ws, u64 q) {
  const u64 q2 = q << 1;
  if (x >= q2) x -= q2;
  u64 t = shoup_mul(y, w, ws, q);
  y = x + q2 - t;
  x = x + t;
}
// Harvey inverse butterfly, ntt.rs:84-104 (x, y < 2q -> x', y' < 2q)
__device__ __forceinline__ void ibf(u64 &x, u64 &y, u64 w, u64 ws, u64 q) {
  const u64 q2 = q << 1;
  u64 u = x + y;
  if (u >= q2) u -= q2;
  u64 t = x + q2 - y;
  y = shoup_mul(t, w, ws, q);
  x = u;
}

__device__ __forceinline__ u64 ldg(const u64 *p) { return __ldg(p); }

// One forward radix-8 round: stages with m, 2m, 4m groups; blk = group of this thread.
template <int NP>
__device__ __forceinline__ void fwd_round8(u64 (&x)[NP][8], int m, int blk, const RingConsts &rc) {
  const u64 q = rc.q;
  {
    u64 w = ldg(rc.fw + m + blk), ws = ldg(rc.fws + m + blk);
#pragma unroll
    for (int p = 0; p < NP; p++)
#pragma unroll
      for (int r = 0; r < 4; r++) fbf(x[p][r], x[p][r + 4], w, ws, q);
  }
#pragma unroll
  for (int h = 0; h < 2; h++) {
    int idx = 2 * m + 2 * blk + h;
    u64 w = ldg(rc.fw + idx), ws = ldg(rc.fws + idx);
#pragma unroll
    for (int p = 0; p < NP; p++) {
      fbf(x[p][4 * h + 0], x[p][4 * h + 2], w, ws, q);
      fbf(x[p][4 * h + 1], x[p][4 * h + 3], w, ws, q);
    }
  }
#pragma unroll
  for (int h = 0; h < 4; h++) {
    int idx = 4 * m + 4 * blk + h;
    u64 w = ldg(rc.fw + idx), ws = ldg(rc.fws + idx);
#pragma unroll
    for (int p = 0; p < NP; p++) fbf(x[p][2 * h], x[p][2 * h + 1], w, ws, q);
  }
}

template <int NP>
__device__ __forceinline__ void inv_round8(u64 (&x)[NP][8], int m, int blk, const RingConsts &rc) {
  const u64 q = rc.q;
#pragma unroll
  for (int h = 0; h < 4; h++) {
    int idx = 4 * m + 4 * blk + h;
    u64 w = ldg(rc.iw + idx), ws = ldg(rc.iws + idx);
#pragma unroll
    for (int p = 0; p < NP; p++) ibf(x[p][2 * h], x[p][2 * h + 1], w, ws, q);
  }
#pragma unroll
  for (int h = 0; h < 2; h++) {
    int idx = 2 * m + 2 * blk + h;
    u64 w = ldg(rc.iw + idx), ws = ldg(rc.iws + idx);
#pragma unroll
    for (int p = 0; p < NP; p++) {
      ibf(x[p][4 * h + 0], x[p][4 * h + 2], w, ws, q);
      ibf(x[p][4 * h + 1], x[p][4 * h + 3], w, ws, q);
    }
  }
  {
    u64 w = ldg(rc.iw + m + blk), ws = ldg(rc.iws + m + blk);
#pragma unroll
    for (int p = 0; p < NP; p++)
#pragma unroll
      for (int r = 0; r < 4; r++) ibf(x[p][r], x[p][r + 4], w, ws, q);
  }
}

// Trailing 2-stage round (stages with N/4 and N/2 groups).
template <int LOGN, int NP>
__device__ __forceinline__ void fwd_round4(u64 (&x)[NP][8], int j, const RingConsts &rc) {
  constexpr int N = 1 << LOGN;
  const u64 q = rc.q;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    int g = (j >> 5) * 64 + (j & 31) + (h << 5);
    u64 w = ldg(rc.fw + N / 4 + g), ws = ldg(rc.fws + N / 4 + g);
#pragma unroll
    for (int p = 0; p < NP; p++) {
      fbf(x[p][4 * h + 0], x[p][4 * h + 2], w, ws, q);
      fbf(x[p][4 * h + 1], x[p][4 * h + 3], w, ws, q);
    }
#pragma unroll
    for (int e = 0; e < 2; e++) {
      int idx = N / 2 + 2 * g + e;
      u64 w2 = ldg(rc.fw + idx), ws2 = ldg(rc.fws + idx);
#pragma unroll
      for (int p = 0; p < NP; p++) fbf(x[p][4 * h + 2 * e], x[p][4 * h + 2 * e + 1], w2, ws2, q);
    }
  }
}

template <int LOGN, int NP>
__device__ __forceinline__ void inv_round4(u64 (&x)[NP][8], int j, const RingConsts &rc) {
  constexpr int N = 1 << LOGN;
  const u64 q = rc.q;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    int g = (j >> 5) * 64 + (j & 31) + (h << 5);
#pragma unroll
    for (int e = 0; e < 2; e++) {
      int idx = N / 2 + 2 * g + e;
      u64 w2 = ldg(rc.iw + idx), ws2 = ldg(rc.iws + idx);
#pragma unroll
      for (int p = 0; p < NP; p++) ibf(x[p][4 * h + 2 * e], x[p][4 * h + 2 * e + 1], w2, ws2, q);
    }
    u64 w = ldg(rc.iw + N / 4 + g), ws = ldg(rc.iws + N / 4 + g);
#pragma unroll
    for (int p = 0; p < NP; p++) {
      ibf(x[p][4 * h + 0], x[p][4 * h + 2], w, ws, q);
      ibf(x[p][4 * h + 1], x[p][4 * h + 3], w, ws, q);
    }
  }
}

// Re-distribute NP polynomials from layout `from` to layout `to` through
// shared memory sm (NP * N words).  cross: the exchange crosses warps.
template <int LOGN, int NP, typename FromF, typename ToF>
__device__ __forceinline__ void exchange(u64 (&x)[NP][8], u64 *sm, int j, FromF from, ToF to,
                                         bool cross) {
  constexpr int N = 1 << LOGN;
  if (cross) __syncthreads();
  else __syncwarp();
#pragma unroll
  for (int p = 0; p < NP; p++)
#pragma unroll
    for (int r = 0; r < 8; r++) sm[p * N + swz(from(j, r))] = x[p][r];
  if (cross) __syncthreads();
  else __syncwarp();
#pragma unroll
  for (int p = 0; p < NP; p++)
#pragma unroll
    for (int r = 0; r < 8; r++) x[p][r] = sm[p * N + swz(to(j, r))];
}

// Forward negacyclic NTT (CT, ntt.rs:110-143 without the final reduction):
// input in the coefficient layout, values < 4q; output in the evaluation
// layout, values < 4q.
template <int LOGN, int NP>
__device__ __forceinline__ void ntt_forward(u64 (&x)[NP][8], u64 *sm, const RingConsts &rc) {
  typedef NttShape<LOGN> S;
  const int j = threadIdx.x;
#pragma unroll
  for (int k = 0; k < S::FULL; k++) {
    if (k > 0) {
      exchange<LOGN, NP>(
          x, sm, j, [k](int jj, int r) { return pos_full<LOGN>(k - 1, jj, r); },
          [k](int jj, int r) { return pos_full<LOGN>(k, jj, r); }, k == 1);
    }
    const int t = S::N >> (3 * k + 3);
    fwd_round8<NP>(x, 1 << (3 * k), j / t, rc);
  }
  if (S::PARTIAL) {
    exchange<LOGN, NP>(
        x, sm, j, [](int jj, int r) { return pos_full<LOGN>(S::FULL - 1, jj, r); },
        [](int jj, int r) { return pos_partial(jj, r); }, S::FULL == 1);
    fwd_round4<LOGN, NP>(x, j, rc);
  }
}

// Inverse negacyclic NTT (GS, ntt.rs:187-230 without the N^{-1} factor):
// input in the evaluation layout, values < 2q; output in the coefficient
// layout, values < 2q.
template <int LOGN, int NP>
__device__ __forceinline__ void ntt_inverse(u64 (&x)[NP][8], u64 *sm, const RingConsts &rc) {
  typedef NttShape<LOGN> S;
  const int j = threadIdx.x;
  if (S::PARTIAL) {
    inv_round4<LOGN, NP>(x, j, rc);
    exchange<LOGN, NP>(
        x, sm, j, [](int jj, int r) { return pos_partial(jj, r); },
        [](int jj, int r) { return pos_full<LOGN>(S::FULL - 1, jj, r); }, S::FULL == 1);
  }
#pragma unroll
  for (int k = S::FULL - 1; k >= 0; k--) {
    const int t = S::N >> (3 * k + 3);
    inv_round8<NP>(x, 1 << (3 * k), j / t, rc);
    if (k > 0) {
      exchange<LOGN, NP>(
          x, sm, j, [k](int jj, int r) { return pos_full<LOGN>(k, jj, r); },
          [k](int jj, int r) { return pos_full<LOGN>(k - 1, jj, r); }, k == 1);
    }
  }
}

__device__ __forceinline__ u64 reduce4(u64 v, u64 q) {  // [0,4q) -> [0,q)
  const u64 q2 = q << 1;
  if (v >= q2) v -= q2;
  if (v >= q) v -= q;
  return v;
}
__device__ __forceinline__ u64 reduce2(u64 v, u64 q) { return v >= q ? v - q : v; }

// 16-byte read-only load that does not allocate in L1 (keys stream through L2).
__device__ __forceinline__ void ld_key2(const u64 *p, u64 &a, u64 &b) {
  asm("ld.global.nc.L1::no_allocate.v2.u64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "l"(p));
}

// Load one device-layout key row into the evaluation layout registers.
template <int LOGN>
__device__ __forceinline__ void load_key_row(const u64 *row, u64 (&k)[8]) {
  const int j = threadIdx.x;
#pragma unroll
  for (int rr = 0; rr < 4; rr++) ld_key2(row + dev_index<LOGN>(j, 2 * rr), k[2 * rr], k[2 * rr + 1]);
}

}  // namespace pz
