// pz_kernels.cu -- CUDA kernels of the gate bootstrap for sm_100a.
//
//   key_convert   coefficient-domain key rows -> device evaluation layout
//                 (forward NTT, * N^{-1} * 2^64 mod Q), keys.rs:702-757
//   ntt_fwd/inv   batched negacyclic NTT in the reference's index order
//                 (ntt.rs:409-441), the kernel microbench
//   ext_product   batched RLWE x RGSW (runtime.rs:754-855)
//   rlwe_auto     batched RLWE automorphism (runtime.rs:530-643)
//   ks            gate prelude (evaluator.rs:2118-2133) + mod-down Q -> q_ks
//                 (pbs.rs:128-132) + LWE key switch (lwe.rs:14-44), batched
//   pbs           one CTA per ciphertext: odd mod-switch, dlog buckets, the
//                 blind-rotation schedule, test vector rotation, the whole
//                 blind rotation with the RLWE accumulator in registers,
//                 sample extraction (pbs.rs:146-449)
#include <algorithm>
#include <map>
#include <mutex>
#include <utility>

#include <cooperative_groups.h>

#include "pz_kernels.cuh"

namespace pz {

// Shared memory of the bootstrap operations: 2N words.  Region 0 (N words)
// holds the permuted a(X^k) of an automorphism, region 1 (N words) its b
// before the evaluation-domain permutation; both together are the exchange
// buffer of the two-polynomial transforms (region 0 alone of the
// single-polynomial ones).
constexpr int OP_REGIONS = 2;
// The two-CTA blind rotation: region 0 exchanges / scatter, region 1 schedule
// scratch / permutation of b, regions 2-3 the two digit slots read by the peer.
constexpr int SPLIT_REGIONS = 4;

// Operation codes of the blind-rotation schedule: an external product with
// RGSW key `i` is `i`; an automorphism with key slot v (0 = -g) is
// OP_AUTO | v, plus OP_TRIVIAL while the accumulator is still trivial.
// OP_KEEPB marks an operation whose successor is a non-trivial automorphism:
// it leaves b in the evaluation domain (scaled by N^{-1}, values < 2q), where
// the automorphism permutes it and adds it before its own inverse transform,
// so b skips one inverse and one forward-domain round trip.
constexpr u32 OP_AUTO = 0x8000u, OP_TRIVIAL = 0x4000u, OP_KEEPB = 0x2000u, OP_SLOT = 0x00ffu,
              OP_INDEX = 0x1fffu;

// ---------------------------------------------------------------------------
// Key conversion and NTT microbench
// ---------------------------------------------------------------------------
template <int LOGN>
__global__ void __launch_bounds__(NttShape<LOGN>::T)
    key_convert_kernel(const u64 *in, u64 *out, size_t npolys, RingConsts rc, u64 c, u64 cs) {
  constexpr int N = 1 << LOGN;
  __shared__ u64 sm[N];
  const int j = threadIdx.x;
  for (size_t pidx = blockIdx.x; pidx < npolys; pidx += gridDim.x) {
    const u64 *src = in + pidx * N;
    u64 x[8];
#pragma unroll
    for (int r = 0; r < 8; r++) x[r] = src[pos_coef<LOGN>(j, r)];
    ntt_fwd<LOGN>(x, sm, rc);
    u64 *dst = out + pidx * N;
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const u64 v = reduce2(shoup_mul(x[r], c, cs, rc.q), rc.q);  // Shoup accepts any 64-bit input
      dst[dev_index<LOGN>(j, r)] = v;
    }
    __syncthreads();
  }
}

template <int LOGN>
__global__ void __launch_bounds__(NttShape<LOGN>::T)
    ntt_fwd_kernel(u64 *polys, size_t count, RingConsts rc) {
  constexpr int N = 1 << LOGN;
  __shared__ u64 sm[N];
  const int j = threadIdx.x;
  for (size_t pidx = blockIdx.x; pidx < count; pidx += gridDim.x) {
    u64 *p = polys + pidx * N;
    u64 x[8];
#pragma unroll
    for (int r = 0; r < 8; r++) x[r] = p[pos_coef<LOGN>(j, r)];
    ntt_fwd<LOGN>(x, sm, rc);
#pragma unroll
    for (int r = 0; r < 8; r++) p[pos_eval<LOGN>(j, r)] = reduce_any(x[r], rc);
    __syncthreads();
  }
}

template <int LOGN>
__global__ void __launch_bounds__(NttShape<LOGN>::T)
    ntt_inv_kernel(u64 *polys, size_t count, RingConsts rc) {
  constexpr int N = 1 << LOGN;
  __shared__ u64 sm[N];
  const int j = threadIdx.x;
  for (size_t pidx = blockIdx.x; pidx < count; pidx += gridDim.x) {
    u64 *p = polys + pidx * N;
    u64 x[8];
#pragma unroll
    for (int r = 0; r < 8; r++) x[r] = p[pos_eval<LOGN>(j, r)];
    ntt_inv<LOGN>(x, sm, rc);
#pragma unroll
    for (int r = 0; r < 8; r++)
      p[pos_coef<LOGN>(j, r)] = reduce2(shoup_mul(x[r], rc.n_inv, rc.n_inv_s, rc.q), rc.q);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Batched NTT for N = 2048 (the kernel microbench and the pz_ntt_* entry
// points): persistent CTAs, two polynomials per iteration transformed
// together (shared twiddles and barriers, independent butterfly streams).
// The next pair's 32 KB come into the other half of a double-buffered
// shared-memory stage by one bulk copy (cp.async.bulk + mbarrier) while the
// current pair is transformed, so the loads never stall the transform.
// Outputs go from registers to global memory: the forward in the evaluation
// order (each thread holds two runs of four consecutive words: 32-byte
// stores), the inverse in the coefficient order (warp-contiguous stores).
// The inverse folds N^{-1} into its last stage (x' = N^{-1}(x + y),
// y' = w N^{-1}(x - y)): 1024 products instead of the 2048 of a separate
// scaling.  Every mbarrier wait is bounded; a wait that runs out sets
// DEVERR_MBAR_TIMEOUT in *err and the CTA returns after a bounded wait for
// its other copy in flight.
// ---------------------------------------------------------------------------
constexpr int NTTB_N = 2048;
// every round's twiddles loaded before its first butterfly (PZ_NTTB_NO_PF: per stage)
#ifdef PZ_NTTB_NO_PF
constexpr bool NTTB_PF = false;
#else
constexpr bool NTTB_PF = true;
#endif
constexpr size_t NTTB_SMEM = (size_t)6 * NTTB_N * 8 + 16;  // exchange 2N | 2 stages of 2N | 2 mbarriers

// Last inverse round (k = 0) with N^{-1} folded into its final stage; values
// leave in [0, 4Q).
template <bool TWO>
__device__ __forceinline__ void inv_round8_last_scaled(u64 (&x)[8], u64 (&y)[8], const RingConsts &rc) {
  constexpr int LOGN = 11;
  const u64 q = rc.q;
  u64 w[6], ws[6];  // all of the round's twiddles first (one load latency)
#pragma unroll
  for (int h = 0; h < 4; h++) tw(rc.iw, 4 + h, w[h], ws[h]);
#pragma unroll
  for (int h = 0; h < 2; h++) tw(rc.iw, 2 + h, w[4 + h], ws[4 + h]);
  // the last radix-8 round's bounds
  constexpr int KA = IK_A8, KB = IK_B8, KC = IK_C8;
#pragma unroll
  for (int h = 0; h < 4; h++) ibf2<LOGN, TWO, KA>(x, y, 2 * h, 2 * h + 1, w[h], ws[h], q);
#pragma unroll
  for (int h = 0; h < 2; h++) {
    ibf2<LOGN, TWO, KB>(x, y, 4 * h + 0, 4 * h + 2, w[4 + h], ws[4 + h], q);
    ibf2<LOGN, TWO, KB>(x, y, 4 * h + 1, 4 * h + 3, w[4 + h], ws[4 + h], q);
  }
  auto last = [&](u64 &a, u64 &b) {  // a, b < KC Q here
    const u64 u = a + b, t = a + (u64)KC * Q_N2048 - b;
    a = shoup_spq(u, rc.n_inv, rc.n_inv_s);
    b = shoup_spq(t, rc.iw1n, rc.iw1n_s);
  };
#pragma unroll
  for (int r = 0; r < 4; r++) {
    last(x[r], x[r + 4]);
    if (TWO) last(y[r], y[r + 4]);
  }
}

// Inverse transform of the batch kernel: rounds unrolled (the last one scaled).
template <bool TWO>
__device__ __forceinline__ void ntt_inv_scaled(u64 (&x)[8], u64 (&y)[8], u64 *sm, const RingConsts &rc) {
  constexpr int LOGN = 11;
  const int j = tid_opaque();
  __syncthreads();
  inv_round4<LOGN, TWO, NTTB_PF>(x, y, j, rc);
  xchg<LOGN, 3, 2, TWO>(x, y, sm, j);
  inv_round8<LOGN, TWO, NTTB_PF>(x, y, 2, j, rc);
  xchg<LOGN, 2, 1, TWO>(x, y, sm, j);
  inv_round8<LOGN, TWO, NTTB_PF>(x, y, 1, j, rc);
  xchg<LOGN, 1, 0, TWO>(x, y, sm, j);
  inv_round8_last_scaled<TWO>(x, y, rc);
}

__device__ __forceinline__ void st_global_v4(u64 *p, u64 a, u64 b, u64 c, u64 d) {
  asm volatile("st.global.v4.u64 [%0], {%1, %2, %3, %4};" ::"l"(p), "l"(a), "l"(b), "l"(c), "l"(d) : "memory");
}
__device__ __forceinline__ void lds2(const u64 *p, u64 &a, u64 &b) {
  asm volatile("ld.shared.v2.u64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "r"(smem_addr(p)));
}

template <bool INV>
__global__ void __launch_bounds__(256, 2) ntt_batch_kernel(u64 *polys, size_t count, RingConsts rc, u32 *err) {
  constexpr int N = NTTB_N, LOGN = 11;
  extern __shared__ __align__(128) u64 smem[];
  u64 *xs = smem, *stage = smem + 2 * N, *bar = smem + 6 * N;
  const int j = threadIdx.x;
  const size_t pairs = (count + 1) / 2;
  auto issue = [&](size_t p, int b) {  // one thread: pair p -> stage b
    const size_t first = 2 * p;
    const u32 bytes = (u32)((count - first >= 2 ? 2 : 1) * N * 8);
    fence_proxy_async_smem();
    bulk_load(stage + (size_t)b * 2 * N, polys + first * N, bytes, bar + b);
  };
  if (j == 0) {
    mbar_init(bar, 1);
    mbar_init(bar + 1, 1);
    mbar_init_fence();
  }
  __syncthreads();
  size_t p = blockIdx.x;
  if (j == 0 && p < pairs) issue(p, 0);
  for (u32 it = 0; p < pairs; it++, p += gridDim.x) {
    const int b = it & 1;
    const bool more = p + gridDim.x < pairs;
    // stage b^1 was read in the previous iteration, before that transform's barriers
    if (j == 0 && more) issue(p + gridDim.x, b ^ 1);
    if (!__syncthreads_and(mbar_wait(bar + b, (it >> 1) & 1))) {
      if (j == 0) {
        atomicOr(err, DEVERR_MBAR_TIMEOUT);
        if (more) mbar_wait(bar + (b ^ 1), ((it + 1) >> 1) & 1);  // bounded: the copy issued above
      }
      return;
    }
    const u64 *sx = stage + (size_t)b * 2 * N, *sy = sx + N;
    const bool two = 2 * p + 1 < count;
    u64 *ox = polys + 2 * p * N, *oy = ox + N;
    u64 x[8], y[8];
    if (!INV) {
#pragma unroll
      for (int r = 0; r < 8; r++) {
        x[r] = sx[pos_coef<LOGN>(j, r)];
        y[r] = sy[pos_coef<LOGN>(j, r)];
      }
      ntt_fwd<LOGN, true, NTTB_PF>(x, y, xs, rc);
#pragma unroll
      for (int h = 0; h < 2; h++) {  // registers 4h..4h+3: four consecutive evaluation positions
        const int o = pos_eval<LOGN>(j, 4 * h);
        st_global_v4(ox + o, reduce2(reduce_n2048(x[4 * h]), Q_N2048), reduce2(reduce_n2048(x[4 * h + 1]), Q_N2048),
                     reduce2(reduce_n2048(x[4 * h + 2]), Q_N2048), reduce2(reduce_n2048(x[4 * h + 3]), Q_N2048));
        if (two)
          st_global_v4(oy + o, reduce2(reduce_n2048(y[4 * h]), Q_N2048),
                       reduce2(reduce_n2048(y[4 * h + 1]), Q_N2048), reduce2(reduce_n2048(y[4 * h + 2]), Q_N2048),
                       reduce2(reduce_n2048(y[4 * h + 3]), Q_N2048));
      }
    } else {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int o = pos_eval<LOGN>(j, 4 * h);
        lds2(sx + o, x[4 * h], x[4 * h + 1]);
        lds2(sx + o + 2, x[4 * h + 2], x[4 * h + 3]);
        lds2(sy + o, y[4 * h], y[4 * h + 1]);
        lds2(sy + o + 2, y[4 * h + 2], y[4 * h + 3]);
      }
      ntt_inv_scaled<true>(x, y, xs, rc);
#pragma unroll
      for (int r = 0; r < 8; r++) {
        ox[pos_coef<LOGN>(j, r)] = reduce4(x[r], Q_N2048);
        if (two) oy[pos_coef<LOGN>(j, r)] = reduce4(y[r], Q_N2048);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// One blind-rotation operation on the accumulator acc = (a, b):
//   op = RGSW index i:  acc <- acc x RGSW_i        (rlwe_by_rgsw_shoup, runtime.rs:754-855)
//   op = OP_AUTO | v:   acc <- auto_{k_v}(acc)      (rlwe_auto_shoup, runtime.rs:530-643)
// a is always in the coefficient layout, canonical [0, Q).  b is too, except
// on entry to a non-trivial automorphism (evaluation domain, see OP_KEEPB)
// and on exit from an operation marked OP_KEEPB.  The external product
// transforms its two digit polynomials together and inverts both outputs
// together; the automorphism transforms its single digit polynomial alone.
// The first (trivial) external product of a blind rotation runs the general
// code with a = 0: the a-digits are 0, their products vanish and, since every
// result is reduced to the canonical residue, the words equal those of the
// reference's trivial branch.  Every output is the canonical residue of the
// same polynomial the reference computes (all steps are exact mod Q), so the
// domain in which b(X^k) is added does not change a word.  Device RGSW rows:
// A(-sm) x d_a, B(-sm) x d_a, A(m) x d_b, B(m) x d_b (runtime.rs:174-180);
// auto key rows A x d, B x d.
// ---------------------------------------------------------------------------

// x <- x (pointwise, mac_reduce) from two device-layout key rows, y likewise.
template <int LOGN>
__device__ __forceinline__ void mac_pair(u64 (&x)[8], u64 (&y)[8], const u64 *ka, const u64 *kb,
                                         const u64 *kc, const u64 *kd, const RingConsts &rc) {
  // x' = x ka + y kc, y' = x kb + y kd
  const int j = threadIdx.x;
  const u64 q = rc.q, qi = rc.qinv_neg;
#pragma unroll
  for (int rr = 0; rr < 4; rr++) {
    const int di = dev_index<LOGN>(j, 2 * rr);
    u64 a[2], b[2], c[2], d[2];
    ld_key2(ka + di, a[0], a[1]);
    ld_key2(kb + di, b[0], b[1]);
    ld_key2(kc + di, c[0], c[1]);
    ld_key2(kd + di, d[0], d[1]);
#pragma unroll
    for (int e = 0; e < 2; e++) {
      const int r = 2 * rr + e;
      const u64 xv = x[r], yv = y[r];
      u64 hi, lo, hi2, lo2;
      sum2_128(xv, a[e], yv, c[e], hi, lo);
      sum2_128(xv, b[e], yv, d[e], hi2, lo2);
      x[r] = mac_reduce<LOGN>(hi, lo, q, qi);
      y[r] = mac_reduce<LOGN>(hi2, lo2, q, qi);
    }
  }
}

// Automorphism product: x' = x ka, y' = x kb + y, with y the permuted b in
// the evaluation domain (< 2q; for N = 2048 < 2.04 Q, a folded product); x'
// as mac_reduce leaves it, y' < 2q.
template <int LOGN>
__device__ __forceinline__ void mac_auto(u64 (&x)[8], u64 (&y)[8], const u64 *ka, const u64 *kb,
                                         const RingConsts &rc) {
  const int j = threadIdx.x;
  const u64 q = rc.q, qi = rc.qinv_neg, q2 = rc.q << 1;
#pragma unroll
  for (int rr = 0; rr < 4; rr++) {
    const int di = dev_index<LOGN>(j, 2 * rr);
    u64 a[2], b[2];
    ld_key2(ka + di, a[0], a[1]);
    ld_key2(kb + di, b[0], b[1]);
#pragma unroll
    for (int e = 0; e < 2; e++) {
      const int r = 2 * rr + e;
      u64 hi, lo, hi2, lo2;
      mac_mul<LOGN>(x[r], a[e], hi, lo);
      mac_mul<LOGN>(x[r], b[e], hi2, lo2);
      x[r] = mac_reduce<LOGN>(hi, lo, q, qi);
      y[r] = mac_add_b<LOGN>(mac_reduce<LOGN>(hi2, lo2, q, qi) + y[r], q2);
    }
  }
}

// Lazy accumulation for the general decomposition path: o += x k (mod q), kept in [0, 2q).
template <int LOGN>
__device__ __forceinline__ void mac_accum(u64 (&oa)[8], u64 (&ob)[8], const u64 (&x)[8], const u64 (&y)[8],
                                          const u64 *ka, const u64 *kb, const u64 *kc, const u64 *kd, bool hx,
                                          bool hy, const RingConsts &rc) {
  const u64 q = rc.q, qi = rc.qinv_neg;
  u64 a[8], b[8], c[8], d[8];
  if (hx) { load_key_row<LOGN>(ka, a); load_key_row<LOGN>(kb, b); }
  if (hy) { load_key_row<LOGN>(kc, c); load_key_row<LOGN>(kd, d); }
#pragma unroll
  for (int r = 0; r < 8; r++) {
    u64 hi = 0, lo = 0, hi2 = 0, lo2 = 0;
    if constexpr (LOGN == 11 && MAC_FOLD_N2048) {  // keys K N^{-1}; sums folded, kept below 2Q
      if (hx && hy) {
        sum2_128(x[r], a[r], y[r], c[r], hi, lo);
        sum2_128(x[r], b[r], y[r], d[r], hi2, lo2);
      } else if (hx) {
        mul128_narrow(x[r], a[r], hi, lo);
        mul128_narrow(x[r], b[r], hi2, lo2);
      } else if (hy) {
        mul128_narrow(y[r], c[r], hi, lo);
        mul128_narrow(y[r], d[r], hi2, lo2);
      }
      oa[r] = reduce_n2048(oa[r] + fold_n2048(hi, lo));
      ob[r] = reduce_n2048(ob[r] + fold_n2048(hi2, lo2));
    } else {
      if (hx) { mac128(x[r], a[r], hi, lo); mac128(x[r], b[r], hi2, lo2); }
      if (hy) { mac128(y[r], c[r], hi, lo); mac128(y[r], d[r], hi2, lo2); }
      const u64 va = oa[r] + redc(hi, lo, q, qi), vb = ob[r] + redc(hi2, lo2, q, qi);
      oa[r] = va >= 2 * q ? va - 2 * q : va;
      ob[r] = vb >= 2 * q ? vb - 2 * q : vb;
    }
  }
}

template <int LOGN, bool D1>
__device__ __forceinline__ void bootstrap_op(u64 (&acc)[2][8], u32 op, const BrParams &P, u64 *sm) {
  constexpr int N = 1 << LOGN;
  const u64 q = P.rc.q;
  const int j = threadIdx.x;
  u64(&x)[8] = acc[0];
  u64(&y)[8] = acc[1];
  const bool is_auto = (op & OP_AUTO) != 0;
  const bool keep_b = (op & OP_KEEPB) != 0;
  u64 *s_a = sm, *s_b = sm + N;
  if (is_auto) {
    // a(X) -> a(X^k) with sign (generate_auto_map, keygen.rs:16-41)
    const u32 k = P.auto_k[op & OP_SLOT];
    __syncthreads();
    if (op & OP_TRIVIAL) {  // runtime.rs:625-642: only b is permuted (neg(0) = q kept)
#pragma unroll
      for (int r = 0; r < 8; r++) {
        u32 t = ((u32)pos_coef<LOGN>(j, r) * k) & (2 * N - 1);
        const bool neg = t >= (u32)N;
        if (neg) t -= N;
        s_b[swz(t)] = neg ? q - y[r] : y[r];
      }
      __syncthreads();
#pragma unroll
      for (int r = 0; r < 8; r++) y[r] = s_b[swz(pos_coef<LOGN>(j, r))];
      return;
    }
#pragma unroll
    for (int r = 0; r < 8; r++) {
      u32 t = ((u32)pos_coef<LOGN>(j, r) * k) & (2 * N - 1);
      const bool neg = t >= (u32)N;
      if (neg) t -= N;
      s_a[swz(t)] = neg ? q - x[r] : x[r];
      s_b[swz(pos_eval<LOGN>(j, r))] = y[r];
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 8; r++) y[r] = s_b[swz(auto_eval_src<LOGN>(pos_eval<LOGN>(j, r), k))];
  }
  const u64 *K = is_auto ? P.autos + (size_t)(op & OP_SLOT) * P.auto_rows * N
                         : P.rgsw + (size_t)(op & OP_INDEX) * P.rgsw_rows * N;
  if (D1) {
    if (is_auto) {
#pragma unroll
      for (int r = 0; r < 8; r++) {
        if constexpr (LOGN == 11) {
          x[r] = decompose1<AUTO_LOGB, AUTO_IGN>(s_a[swz(pos_coef<LOGN>(j, r))], q);
        } else {
          u64 st = decomp_init(s_a[swz(pos_coef<LOGN>(j, r))], P.dauto);
          x[r] = decomp_next(st, P.dauto);
        }
      }
      ntt_fwd<LOGN, false>(x, x, sm, P.rc);
      mac_auto<LOGN>(x, y, K, K + N, P.rc);
    } else {
#pragma unroll
      for (int r = 0; r < 8; r++) {
        if constexpr (LOGN == 11) {
          x[r] = decompose1<RLRG_LOGB, RLRG_IGN>(x[r], q);
          y[r] = decompose1<RLRG_LOGB, RLRG_IGN>(y[r], q);
        } else {
          u64 sa = decomp_init(x[r], P.da);
          x[r] = decomp_next(sa, P.da);
          u64 sb = decomp_init(y[r], P.db);
          y[r] = decomp_next(sb, P.db);
        }
      }
      ntt_fwd<LOGN, true>(x, y, sm, P.rc);
      mac_pair<LOGN>(x, y, K, K + N, K + 2 * N, K + 3 * N, P.rc);
    }
  } else {
    // general decomposition counts (SP_TEST: d = 4): digit by digit, lazily
    // accumulated in [0, 2q), one inverse transform at the end
    const u32 da = is_auto ? P.d_auto : P.d_a, db = is_auto ? 0 : P.d_b;
    const Decomp &dpa = is_auto ? P.dauto : P.da;
    u64 sa[8], sb[8], oa[8], ob[8];
#pragma unroll
    for (int r = 0; r < 8; r++) {
      sa[r] = decomp_init(is_auto ? s_a[swz(pos_coef<LOGN>(j, r))] : x[r], dpa);
      sb[r] = is_auto ? 0 : decomp_init(y[r], P.db);
      oa[r] = 0;
      ob[r] = is_auto ? y[r] : 0;  // the automorphism's permuted b (< 2q)
    }
    const u32 dmax = da > db ? da : db;
    for (u32 jd = 0; jd < dmax; jd++) {
      const bool hx = jd < da, hy = jd < db;
#pragma unroll
      for (int r = 0; r < 8; r++) {
        x[r] = hx ? decomp_next(sa[r], dpa) : 0;
        y[r] = hy ? decomp_next(sb[r], P.db) : 0;
      }
      if (hy) ntt_fwd<LOGN, true>(x, y, sm, P.rc);
      else ntt_fwd<LOGN, false>(x, x, sm, P.rc);
      if (is_auto) {
        mac_accum<LOGN>(oa, ob, x, y, K + (size_t)jd * N, K + (size_t)(da + jd) * N, nullptr, nullptr, hx,
                        false, P.rc);
      } else {
        mac_accum<LOGN>(oa, ob, x, y, K + (size_t)jd * N, K + (size_t)(da + jd) * N,
                        K + (size_t)(2 * da + jd) * N, K + (size_t)(2 * da + db + jd) * N, hx, hy, P.rc);
      }
    }
#pragma unroll
    for (int r = 0; r < 8; r++) {
      x[r] = oa[r];
      y[r] = ob[r];
    }
  }
  if (keep_b) {
    ntt_inv<LOGN, false>(x, x, sm, P.rc);
#pragma unroll
    for (int r = 0; r < 8; r++) x[r] = reduce2(x[r], q);
  } else {
    ntt_inv<LOGN, true>(x, y, sm, P.rc);
#pragma unroll
    for (int r = 0; r < 8; r++) {
      x[r] = reduce2(x[r], q);
      y[r] = reduce2(y[r], q);
    }
  }
}

// One-digit (D1) forms come register-capped for MINB = 2, 3 or 4 CTAs per SM,
// picked like the blind rotation's launch shapes (the context's variant).
template <int LOGN, bool D1, int MINB>
__global__ void __launch_bounds__(NttShape<LOGN>::T, MINB)
    ext_product_kernel(BrParams P, u64 *rlwe, const u32 *idx, size_t count, int trivial) {
  constexpr int N = 1 << LOGN;
  extern __shared__ u64 smem[];
  const int j = threadIdx.x;
  for (size_t c = blockIdx.x; c < count; c += gridDim.x) {
    if (idx[c] >= P.n) continue;  // out-of-range key index: the ciphertext is left unchanged
    if (threadIdx.x == 0)  // the key rows, into L2 while the digits are transformed
      prefetch_l2(P.rgsw + (size_t)idx[c] * P.rgsw_rows * N, P.rgsw_rows * (u32)N * 8);
    u64 *p = rlwe + c * 2 * N;
    u64 acc[2][8];
#pragma unroll
    for (int r = 0; r < 8; r++) {
      acc[0][r] = trivial ? 0 : p[pos_coef<LOGN>(j, r)];  // trivial: a = 0 (runtime.rs:790)
      acc[1][r] = p[N + pos_coef<LOGN>(j, r)];
    }
    bootstrap_op<LOGN, D1>(acc, idx[c], P, smem);
#pragma unroll
    for (int r = 0; r < 8; r++) {
      p[pos_coef<LOGN>(j, r)] = acc[0][r];
      p[N + pos_coef<LOGN>(j, r)] = acc[1][r];
    }
    __syncthreads();
  }
}

template <int LOGN, bool D1, int MINB>
__global__ void __launch_bounds__(NttShape<LOGN>::T, MINB)
    auto_kernel(BrParams P, u64 *rlwe, const u32 *slot, size_t count, int trivial) {
  constexpr int N = 1 << LOGN;
  extern __shared__ u64 smem[];
  const int j = threadIdx.x;
  for (size_t c = blockIdx.x; c < count; c += gridDim.x) {
    if (slot[c] > P.w) continue;  // out-of-range key slot: the ciphertext is left unchanged
    if (threadIdx.x == 0) prefetch_l2(P.autos + (size_t)slot[c] * P.auto_rows * N, P.auto_rows * (u32)N * 8);
    u64 *p = rlwe + c * 2 * N;
    u64 acc[2][8];
#pragma unroll
    for (int r = 0; r < 8; r++) {
      acc[0][r] = p[pos_coef<LOGN>(j, r)];
      acc[1][r] = p[N + pos_coef<LOGN>(j, r)];
    }
    if (!trivial) {  // a non-trivial automorphism takes b as N^{-1} NTT(b) (< 2q)
      ntt_fwd<LOGN>(acc[1], smem, P.rc);
#pragma unroll
      for (int r = 0; r < 8; r++) acc[1][r] = shoup_mul(acc[1][r], P.rc.n_inv, P.rc.n_inv_s, P.rc.q);
    }
    bootstrap_op<LOGN, D1>(acc, OP_AUTO | (trivial ? OP_TRIVIAL : 0u) | (slot[c] & OP_SLOT), P, smem);
#pragma unroll
    for (int r = 0; r < 8; r++) {
      p[pos_coef<LOGN>(j, r)] = acc[0][r];
      p[N + pos_coef<LOGN>(j, r)] = acc[1][r];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Gate prelude + mod-down + LWE key switch
// ---------------------------------------------------------------------------
// evaluator.rs:2118-2133 then pbs.rs:128-132 for one coefficient.
__device__ __forceinline__ u64 prelude_moddown(u64 x0, u64 x1, unsigned char gate, bool is_b,
                                               const KsParams &P) {
  u64 v;
  if (P.raw || (gate & GATE_RAW)) {
    v = x0;
  } else if (gate >= 4) {  // xor, xnor: 2 (c0 - c1)
    v = sub_mod(x0, x1, P.Q);
    v = add_mod(v, v, P.Q);
  } else {  // and, nand, or, nor: c0 + c1 (+ Q/4 on b)
    v = add_mod(x0, x1, P.Q);
    if (is_b) v = add_mod(v, P.qby4, P.Q);
  }
  double f = __ddiv_rn(__dmul_rn(__ull2double_rn(v), P.q_ks_f), P.Q_f);
  return (u64)round(f);
}

constexpr int KS_IC = 32;    // LWE coefficients per digit chunk
constexpr int KS_COLS = 128; // output columns per CTA
// digits of one CTA's chunk: CT ciphertexts x KS_IC coefficients x MAX_KS_D (u32)
constexpr size_t ks_dig_bytes(int ct) { return (size_t)ct * KS_IC * MAX_KS_D * 4; }

// Input word `i` of gate ct's operand (gathered through a wire index when
// given; a set WIRE_NEG bit applies not(): q - x, evaluator.rs:2247-2250).
__device__ __forceinline__ u64 operand(const u64 *base, const u32 *idx, int ct, size_t i, size_t L, u64 q) {
  if (!base) return 0;
  if (!idx) return base[(size_t)ct * L + i];
  const u32 w = idx[ct];
  const u64 x = base[(size_t)(w & WIRE_MASK) * L + i];
  return (w & WIRE_NEG) ? q - x : x;
}

// Key switch of ciphertexts [ct0, min(ct0 + CT, count)) for the output
// columns of this CTA (blockIdx.y) over its share of the input coefficients
// (blockIdx.z of gridDim.z).  With one share the sums are stored reduced mod
// q_ks; with several, each CTA adds its partial sums into the zeroed output
// with 32-bit atomics (exact: the result is taken mod q_ks, a power of two
// <= 2^32) and the consumer reduces (value & (q_ks - 1)).
template <int CT>
__device__ __forceinline__ void ks_tile(const KsParams &P, const unsigned char *gates, const u64 *c0, const u64 *c1,
                                        int ct0, int count, u32 *out, u32 (*dig)[KS_IC][MAX_KS_D]) {
  const int tid = threadIdx.x;
  const int col = blockIdx.y * KS_COLS + tid;
  const size_t L = (size_t)P.N + 1;
  const u32 d = P.d;
  const u32 chunks = P.N / KS_IC, per = (chunks + gridDim.z - 1) / gridDim.z;
  const u32 i_begin = blockIdx.z * per * KS_IC;
  const u32 i_end = min(P.N, i_begin + per * KS_IC);
  if (i_begin >= P.N) return;  // uniform per CTA
  u32 acc[CT];
#pragma unroll
  for (int c = 0; c < CT; c++) acc[c] = 0;
  for (u32 i0 = i_begin; i0 < i_end; i0 += KS_IC) {
    __syncthreads();
    for (int e = tid; e < CT * KS_IC; e += KS_COLS) {
      const int c = e / KS_IC, ii = e % KS_IC;
      const int ct = ct0 + c;
      if (ct < count) {
        const size_t off = 1 + i0 + ii;
        const u64 x = prelude_moddown(operand(c0, P.in0, ct, off, L, P.Q), operand(c1, P.in1, ct, off, L, P.Q),
                                      gates ? gates[ct] : 0, false, P);
        u64 st = decomp_init(x, P.dks);
        for (u32 jd = 0; jd < d; jd++) dig[c][ii][jd] = (u32)decomp_next(st, P.dks);
      } else {
        for (u32 jd = 0; jd < d; jd++) dig[c][ii][jd] = 0;
      }
    }
    __syncthreads();
    if (col <= (int)P.n) {
      const u32 *kp = P.ksk + (size_t)i0 * d * P.ksk_stride + col;
      for (int ii = 0; ii < KS_IC; ii++) {
        for (u32 jd = 0; jd < d; jd++) {
          const u32 kv = __ldg(kp);
          kp += P.ksk_stride;
#pragma unroll
          for (int c = 0; c < CT; c++) acc[c] += dig[c][ii][jd] * kv;
        }
      }
    }
  }
  if (col <= (int)P.n) {
#pragma unroll
    for (int c = 0; c < CT; c++) {
      const int ct = ct0 + c;
      if (ct < count) {
        u32 v = acc[c];
        if (col == 0 && blockIdx.z == 0) {
          v += (u32)prelude_moddown(operand(c0, P.in0, ct, 0, L, P.Q), operand(c1, P.in1, ct, 0, L, P.Q),
                                    gates ? gates[ct] : 0, true, P);
        }
        u32 *o = out + (size_t)ct * P.out_stride + col;
        if (gridDim.z == 1) *o = v & P.mask;
        else atomicAdd(o, v);
      }
    }
  }
}

// CT ciphertexts per CTA (8, 16 or 32: picked per batch by the autotuner);
// the digit buffer is dynamic shared memory of ks_dig_bytes(CT).
template <int CT>
__global__ void __launch_bounds__(KS_COLS)
    ks_kernel(KsParams P, const unsigned char *gates, const u64 *c0, const u64 *c1, int count, u32 *out) {
  extern __shared__ __align__(16) u32 ks_dig[];
  ks_tile<CT>(P, gates, c0, c1, blockIdx.x * CT, count, out, (u32 (*)[KS_IC][MAX_KS_D])ks_dig);
}

// Ragged batch: tile blockIdx.x holds up to KS_CT ciphertexts of one session
// (descriptor) -- the KSK rows it streams are that session's.  Ciphertext
// operands are gathered from `wires` through in0/in1 (bit 31 = not()).
__global__ void __launch_bounds__(KS_COLS)
    ks_ragged_kernel(const KsParams *descs, const KsTile *tiles, const unsigned char *gates, const u64 *wires,
                     const u32 *in0, const u32 *in1, u32 *out, u32 out_stride) {
  __shared__ u32 dig[KS_TILE_CT][KS_IC][MAX_KS_D];
  __shared__ KsParams sp;
  const KsTile t = tiles[blockIdx.x];
  if (threadIdx.x == 0) {
    sp = descs[t.desc];
    sp.in0 = in0;
    sp.in1 = in1;
    sp.out_stride = out_stride;
    sp.raw = 0;
  }
  __syncthreads();
  if (blockIdx.y * KS_COLS > sp.n) return;  // no columns of this session here (uniform per CTA)
  ks_tile<KS_TILE_CT>(sp, gates, wires, wires, (int)t.first, (int)(t.first + t.count), out, dig);
}

// ---------------------------------------------------------------------------
// LWE key switch on the tensor cores.  With base-2^logb digits (logb <= 4
// in every parameter set: digits in [-8, 8]) the key switch of a batch is a
// matrix product: [ciphertexts x d N digits] (s8) times [d N x (n + 1)] KSK
// entries mod q_ks.  The KSK is split into byte planes (u8), each plane one
// mma.sync m16n8k32 s8 x u8 product with exact s32 sums (|sum| < d N 8 255 <
// 2^27), folded into the u32 result as sum_p 2^(8p) plane_p -- exact mod
// 2^32, and q_ks divides 2^32.  A CTA owns KSM_ROWS = 64 ciphertexts x
// KSM_COLS = 224 output columns: 8 warps = 4 row fragments (16) x 2 column
// halves (112 = 14 column fragments of 8).  Per chunk of 32 input
// coefficients the CTA writes the 32 d digits of its 64 ciphertexts into
// shared memory (row stride 32 d + 16 bytes: conflict-free fragment loads);
// the KSK planes of each 32-row block stream into a double-buffered stage
// by 16-byte cp.async, one block ahead.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void mma_s8u8(u32 (&d)[4], u32 a0, u32 a1, u32 a2, u32 a3, u32 b0, u32 b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k32.row.col.s32.s8.u8.s32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%10, %10, %10, %10};"
      : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1), "r"(0u));
}

__host__ __device__ constexpr size_t ksm_astride(u32 d) { return (size_t)32 * d + 16; }
constexpr size_t ksm_smem_bytes(u32 d, u32 planes) {
  return (size_t)KSM_ROWS * ksm_astride(d) + 2 * (size_t)planes * KSM_COLS * 32;
}

// One CTA's tile: ciphertexts [ct0, min(ct0 + KSM_ROWS, count)), output
// column block cb, this CTA's share (blockIdx.z of gridDim.z) of the input
// coefficients.  NP bounds the planes (P.planes <= NP, checked per plane).
template <int NP>
__device__ __forceinline__ void ks_mma_tile(const KsParams &P, const unsigned char *gates, const u64 *c0,
                                            const u64 *c1, int ct0, int count, u32 *out, int cb,
                                            unsigned char *ksm) {
  const u32 d = P.d, astride = (u32)ksm_astride(d), planes = P.planes;
  unsigned char *A = ksm;
  unsigned char *Bs = ksm + (size_t)KSM_ROWS * astride;  // [2][NP][KSM_COLS][32]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int mf = warp & 3, nh = warp >> 2;
  const size_t L = (size_t)P.N + 1;
  const u32 kblocks = d * P.N / 32;
  const size_t plane_bytes = (size_t)kblocks * P.ksk8_cols * 32;
  const unsigned char *Bg = P.ksk8 + (size_t)cb * KSM_COLS * 32;
  constexpr int STAGE = NP * KSM_COLS * 32;
  const int chunks16 = (int)planes * KSM_COLS * 2;  // 16-byte pieces per stage
  auto issue = [&](u32 kb) {
    unsigned char *dst = Bs + (size_t)(kb & 1) * STAGE;
    for (int e = tid; e < chunks16; e += 256) {
      const int p = e / (KSM_COLS * 2), r = e % (KSM_COLS * 2);
      cp_async16(dst + (size_t)p * KSM_COLS * 32 + r * 16,
                 Bg + p * plane_bytes + (size_t)kb * P.ksk8_cols * 32 + r * 16);
    }
    cp_async_commit();
  };
  u32 acc[14][4];
#pragma unroll
  for (int f = 0; f < 14; f++)
#pragma unroll
    for (int i = 0; i < 4; i++) acc[f][i] = 0;
  // this CTA's share of the 32-coefficient chunks (grid.z shares for small batches)
  const u32 chunks = P.N / 32, per = (chunks + gridDim.z - 1) / gridDim.z;
  const u32 c_begin = blockIdx.z * per, c_end = min(chunks, c_begin + per);
  if (c_begin >= c_end) return;  // uniform per CTA
  u32 kb = c_begin * d;
  const u32 kb_end = c_end * d;
  issue(kb);
  for (u32 i0 = c_begin * 32; i0 < c_end * 32; i0 += 32) {
    __syncthreads();  // every warp is done with the previous chunk's digits
    for (int e = tid; e < KSM_ROWS * 32; e += 256) {
      const int row = e >> 5, cc = e & 31, ct = ct0 + row;
      unsigned char *dst = A + (size_t)row * astride + (size_t)cc * d;
      if (ct < count) {
        const size_t off = 1 + i0 + cc;
        const u64 x = prelude_moddown(operand(c0, P.in0, ct, off, L, P.Q), operand(c1, P.in1, ct, off, L, P.Q),
                                      gates ? gates[ct] : 0, false, P);
        u64 st = decomp_init(x, P.dks);
        for (u32 j = 0; j < d; j++) dst[j] = (unsigned char)(signed char)decomp_next_signed(st, P.dks);
      } else {
        for (u32 j = 0; j < d; j++) dst[j] = 0;
      }
    }
    for (u32 ks = 0; ks < d; ks++, kb++) {
      cp_async_wait_all();
      __syncthreads();  // stage kb landed for every thread; stage kb + 1 is free; digits written
      if (kb + 1 < kb_end) issue(kb + 1);
      const unsigned char *ar = A + (size_t)(16 * mf + g) * astride + ks * 32 + 4 * t;
      const u32 a0 = *(const u32 *)ar, a1 = *(const u32 *)(ar + 8 * astride);
      const u32 a2 = *(const u32 *)(ar + 16), a3 = *(const u32 *)(ar + 8 * astride + 16);
      const unsigned char *bs = Bs + (size_t)(kb & 1) * STAGE + (size_t)(nh * 112 + g) * 32 + 8 * t;
#pragma unroll
      for (int f = 0; f < 14; f++) {
        u32 r[NP][4];
#pragma unroll
        for (int p = 0; p < NP; p++) {
          if (p < (int)planes) {
            const uint2 b = *(const uint2 *)(bs + (size_t)p * KSM_COLS * 32 + f * 8 * 32);
            mma_s8u8(r[p], a0, a1, a2, a3, b.x, b.y);
          } else {
            r[p][0] = r[p][1] = r[p][2] = r[p][3] = 0;
          }
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
          u32 v = r[0][i];
          if (NP > 1) v += r[1][i] << 8;
          if (NP > 2) v += r[2][i] << 16;
          acc[f][i] += v;
        }
      }
    }
  }
  // fragment element i of column fragment f: row 16 mf + g (+8 for i >= 2),
  // column nh 112 + 8 f + 2 t + (i & 1)
#pragma unroll
  for (int f = 0; f < 14; f++) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int ct = ct0 + 16 * mf + g + (i >= 2 ? 8 : 0);
      const u32 col = (u32)cb * KSM_COLS + nh * 112 + 8 * f + 2 * t + (i & 1);
      if (ct < count && col <= P.n) {
        u32 v = acc[f][i];
        if (col == 0 && blockIdx.z == 0)
          v += (u32)prelude_moddown(operand(c0, P.in0, ct, 0, L, P.Q), operand(c1, P.in1, ct, 0, L, P.Q),
                                    gates ? gates[ct] : 0, true, P);
        u32 *o = out + (size_t)ct * P.out_stride + col;
        if (gridDim.z == 1) *o = v & P.mask;
        else atomicAdd(o, v);  // exact mod 2^32; the consumer reduces mod q_ks
      }
    }
  }
}

template <int NP>
__global__ void __launch_bounds__(256, 2)
    ks_mma_kernel(KsParams P, const unsigned char *gates, const u64 *c0, const u64 *c1, int count, u32 *out) {
  extern __shared__ __align__(16) unsigned char ksm[];
  ks_mma_tile<NP>(P, gates, c0, c1, blockIdx.x * KSM_ROWS, count, out, blockIdx.y, ksm);
}

// Ragged batch on the tensor cores: tile blockIdx.x holds up to KSM_ROWS
// consecutive items of one session (descriptor), whose KSK planes it streams;
// operands are gathered from `wires` through in0/in1 (bit 31 = not()).
__global__ void __launch_bounds__(256, 2)
    ks_mma_ragged_kernel(const KsParams *descs, const KsTile *tiles, const unsigned char *gates, const u64 *wires,
                         const u32 *in0, const u32 *in1, u32 *out, u32 out_stride) {
  extern __shared__ __align__(16) unsigned char ksm[];
  __shared__ KsParams sp;
  const KsTile t = tiles[blockIdx.x];
  if (threadIdx.x == 0) {
    sp = descs[t.desc];
    sp.in0 = in0;
    sp.in1 = in1;
    sp.out_stride = out_stride;
    sp.raw = 0;
  }
  __syncthreads();
  if (blockIdx.y * KSM_COLS > sp.n) return;  // no columns of this session here (uniform per CTA)
  ks_mma_tile<3>(sp, gates, wires, wires, (int)t.first, (int)(t.first + t.count), out, blockIdx.y, ksm);
}

// KSK u32 rows -> byte planes in the fragment order of ks_mma_kernel: row r
// of block r / 32 goes to byte 8 j + 4 h + (k & 3) of its column's 32-byte
// record, k = r mod 32, h = k / 16, j = (k mod 16) / 4 (thread j of a quad
// loads bytes 8 j .. 8 j + 7: rows 4j..4j+3 and 16+4j..16+4j+3).
__global__ void ksk_planes_kernel(const u32 *ksk, u32 rows, u32 stride, u32 n, u32 planes, u32 cols,
                                  unsigned char *out) {
  const size_t total = (size_t)rows * cols, plane_bytes = total;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const u32 r = (u32)(e / cols), c = (u32)(e % cols);
    const u32 v = c <= n ? ksk[(size_t)r * stride + c] : 0u;
    const u32 k = r & 31, pos = 8 * ((k & 15) >> 2) + 4 * (k >> 4) + (k & 3);
    const size_t o = ((size_t)(r >> 5) * cols + c) * 32 + pos;
    for (u32 p = 0; p < planes; p++) out[p * plane_bytes + o] = (unsigned char)(v >> (8 * p));
  }
}

// ---------------------------------------------------------------------------
// The bootstrap: one CTA per ciphertext (grid-stride over the batch)
// ---------------------------------------------------------------------------
// pbs.rs:416-420
__device__ __forceinline__ u32 mod_switch_odd(u32 v, double from_q, double to_q) {
  u64 odd = (u64)floor(__ddiv_rn(__dmul_rn((double)v, to_q), from_q));
  return (u32)(odd + ((odd & 1ull) ^ 1ull));
}

// Shared memory of pbs_kernel: OP_REGIONS x N words, then u16 arrays:
// bucket starts (R + 1), bucket members (n), the schedule (n + R + 1), and
// the schedule length.
size_t pbs_smem_bytes(int logn, u32 br_q, u32 n) {
  const size_t N = (size_t)1 << logn, R = br_q / 2;
  size_t extra = ((R + 1) + n + (n + R + 1)) * 2 + 4;
  extra = (extra + 15) & ~(size_t)15;
  return OP_REGIONS * N * 8 + extra;
}

// Dynamic shared memory of the two-CTA kernel: 4 x N words + the schedule.
static size_t split_smem_bytes(u32 br_q, u32 n) {
  const size_t N = 2048, R = br_q / 2;
  size_t extra = ((R + 1) + n + (n + R + 1)) * 2 + 4;
  extra = (extra + 15) & ~(size_t)15;
  return SPLIT_REGIONS * 8 * N + extra;
}

// Shared-memory arrays of the blind-rotation schedule, after `regions` x N words.
struct SchedSmem {
  unsigned short *start, *list, *ops;
  u32 *nops;
};
template <int LOGN>
__device__ __forceinline__ SchedSmem sched_smem(u64 *smem, int regions, u32 R, u32 n) {
  constexpr int N = 1 << LOGN;
  SchedSmem m;
  m.start = (unsigned short *)(smem + regions * N);  // R + 1
  m.list = m.start + (R + 1);                         // n
  m.ops = m.list + n;                                 // n + R + 1
  m.nops = (u32 *)(((size_t)(m.ops + n + R + 1) + 3) & ~(size_t)3);
  return m;
}

// Odd mod-switch, dlog buckets (pbs.rs:147-161, stable in LWE index) and the
// blind-rotation schedule (pbs.rs:240-414) of one key-switched LWE, built in
// shared memory by the whole CTA (regions 0 and 1 of smem are scratch).
template <int LOGN>
__device__ __forceinline__ void build_schedule(const BrParams &P, const u32 *kso, u64 *smem, const SchedSmem &S) {
  constexpr int N = 1 << LOGN, T = NttShape<LOGN>::T;
  const u32 R = P.br_q >> 1, q4 = P.br_q >> 2, n = P.n;
  const int j = threadIdx.x, lane = j & 31, warp = j >> 5;
  u64 *sm = smem;
  unsigned short *s_start = S.start, *s_list = S.list, *s_ops = S.ops;
  u32 *s_nops = S.nops;
  {
    // ---- odd mod-switch + dlog buckets (pbs.rs:147-161), stable in LWE index
    u32 *cnt = (u32 *)sm;                                 // R counters (region 0)
    unsigned short *keys = (unsigned short *)(cnt + R);   // n keys (region 0)
    u32 *fill = (u32 *)(sm + N);                          // R fill counters (region 1)
    u32 *scan = fill + R;                                 // T partial sums (region 1)
    __syncthreads();
    for (u32 b = j; b < R; b += T) { cnt[b] = 0; fill[b] = 0; }
    __syncthreads();
    for (u32 i = j; i < n; i += T) {
      const u32 odd = mod_switch_odd(kso[1 + i] & P.ks_mask, P.q_ks_f, P.br_q_f);
      const u32 k = P.dlog[odd];
      keys[i] = (unsigned short)k;
      atomicAdd(&cnt[k], 1u);
    }
    __syncthreads();
    {  // exclusive scan of cnt[0..R) into s_start, s_start[R] = n
      const u32 per = (R + T - 1) / T;
      const u32 b0 = j * per;
      u32 local = 0;
      for (u32 b = b0; b < b0 + per && b < R; b++) local += cnt[b];
      u32 incl = local;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        u32 y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane == 31) scan[warp] = incl;
      __syncthreads();
      u32 woff = 0;
      for (int w2 = 0; w2 < warp; w2++) woff += scan[w2];
      u32 run = woff + incl - local;
      for (u32 b = b0; b < b0 + per && b < R; b++) {
        s_start[b] = (unsigned short)run;
        run += cnt[b];
      }
      if (j == 0) s_start[R] = (unsigned short)n;
    }
    __syncthreads();
    if (warp == 0) {  // stable placement: within a bucket, increasing LWE index
      for (u32 i0 = 0; i0 < n; i0 += 32) {
        const u32 i = i0 + lane;
        const bool valid = i < n;
        const u32 k = valid ? keys[i] : 0xFFFFu;
        const u32 peers = __match_any_sync(0xffffffffu, k);
        const u32 rank = __popc(peers & ((1u << lane) - 1u));
        if (valid) s_list[s_start[k] + fill[k] + rank] = (unsigned short)i;
        __syncwarp();
        if (valid && rank == 0) fill[k] += __popc(peers);
        __syncwarp();
      }
    }
    __syncthreads();
    // ---- the blind-rotation schedule (pbs.rs:240-414): buckets of -g^k for
    // k = q/4-1..1, -g^0, +g^k, +g^0, each followed by an automorphism when
    // the next bucket is non-empty, the window w is reached or k == 1; the
    // automorphisms before the first external product act on a trivial RLWE.
    if (j == 0) {
      u32 no = 0;
      bool trivial = true;
      auto bucket = [&](u32 b) {
        const u32 e = s_start[b + 1];
        for (u32 t = s_start[b]; t < e; t++) s_ops[no++] = s_list[t];
        if (e != s_start[b]) trivial = false;
      };
      auto autom = [&](u32 v) {
        if (!trivial) s_ops[no - 1] |= (unsigned short)OP_KEEPB;  // b stays in the evaluation domain
        s_ops[no++] = (unsigned short)(OP_AUTO | (trivial ? OP_TRIVIAL : 0u) | v);
      };
      u32 v = 0;
      for (u32 i = q4 - 1; i >= 1; i--) {  // -(g^k)
        bucket(q4 + i);
        v++;
        if (s_start[q4 + i] != s_start[q4 + i - 1] || v == P.w || i == 1) {
          autom(v);
          v = 0;
        }
      }
      bucket(q4);  // -(g^0)
      autom(0);
      v = 0;
      for (u32 i = q4 - 1; i >= 1; i--) {  // +(g^k)
        bucket(i);
        v++;
        if (s_start[i] != s_start[i - 1] || v == P.w || i == 1) {
          autom(v);
          v = 0;
        }
      }
      bucket(0);  // +(g^0)
      *s_nops = no;
    }
  }
}

// Trivial test RLWE's b: X^{g * odd(b)} * tv, embedded (pbs.rs:163-211), in
// the coefficient layout of this thread.
template <int LOGN>
__device__ __forceinline__ void test_rlwe_b(const BrParams &P, const u32 *kso, u32 gcode, u64 (&b)[8]) {
  const u32 R = P.br_q >> 1;
  const u64 q = P.rc.q;
  const int j = threadIdx.x;
  const u32 odd_b = mod_switch_odd(kso[0] & P.ks_mask, P.q_ks_f, P.br_q_f);
  const u32 gb = (u32)(((u64)P.g * odd_b) % P.br_q);
  u32 mexp = gb;
  bool msign = true;
  if (mexp > R) { mexp -= R; msign = false; }
  u32 gi = gcode & 7u;
  if (gi > 5) gi = 5;  // codes are validated on the host; never index past the 6 test vectors
  const u64 *tv = P.tv + (size_t)gi * R;
#pragma unroll
  for (int r = 0; r < 8; r++) {
    const u32 p = (u32)pos_coef<LOGN>(j, r);
    u64 v = 0;
    if (p % P.emb == 0) {
      const u32 o = p / P.emb;
      u32 s;
      bool sg;
      if (o >= mexp) { s = o - mexp; sg = msign; } else { s = o + R - mexp; sg = !msign; }
      const u64 t = tv[s];
      v = sg ? t : q - t;
    }
    b[r] = v;
  }
}

// L2 prefetch of a blind-rotation operation's key rows (none for a trivial
// automorphism).
template <int LOGN>
__device__ __forceinline__ void prefetch_next_key(const BrParams &P, u32 op) {
  constexpr size_t N = (size_t)1 << LOGN;
  if (op & OP_AUTO) {
    if (!(op & OP_TRIVIAL))
      prefetch_l2(P.autos + (size_t)(op & OP_SLOT) * P.auto_rows * N, P.auto_rows * (u32)N * 8);
  } else {
    prefetch_l2(P.rgsw + (size_t)(op & OP_INDEX) * P.rgsw_rows * N, P.rgsw_rows * (u32)N * 8);
  }
}

// MINB: CTAs per SM the register allocation must allow (launch-shape
// variants chosen at run time, see pz_ctx_set_pbs_variant).
// One gate bootstrap of ciphertext ct (key-switched LWE kso, gate code
// gcode) with the parameters and key of P; the whole CTA takes part.
template <int LOGN, bool D1>
__device__ __forceinline__ void pbs_item(const BrParams &P, int ct, const u32 *kso, u32 gcode, u64 *out,
                                         u64 *rlwe_dbg, u64 *smem) {
  constexpr int N = 1 << LOGN;
  u64 *sm = smem;
  const SchedSmem S = sched_smem<LOGN>(smem, OP_REGIONS, P.br_q >> 1, P.n);
  unsigned short *s_ops = S.ops;
  u32 *s_nops = S.nops;
  const int j = threadIdx.x;
  const u64 q = P.rc.q;
  {
    build_schedule<LOGN>(P, kso, smem, S);
    u64 acc[2][8];
#pragma unroll
    for (int r = 0; r < 8; r++) acc[0][r] = 0;
    test_rlwe_b<LOGN>(P, kso, gcode, acc[1]);
    __syncthreads();

    // ---- blind rotation: one operation per schedule entry; the next
    // operation's key rows are asked into L2 as this one starts
    const u32 nops = *s_nops;
#pragma unroll 1
    for (u32 t = 0; t < nops; t++) {
      if (j == 0 && t + 1 < nops) prefetch_next_key<LOGN>(P, s_ops[t + 1]);
      bootstrap_op<LOGN, D1>(acc, s_ops[t], P, sm);
    }

    // ---- sample extract at index 0 (pbs.rs:423-449)
    u64 *o = out + (size_t)(P.out_idx ? P.out_idx[ct] : (u32)ct) * (N + 1);
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const u32 p = (u32)pos_coef<LOGN>(j, r);
      if (p == 0) {
        o[0] = acc[1][r];
        o[1] = acc[0][r];
      } else {
        o[1 + N - p] = q - acc[0][r];
      }
    }
    if (rlwe_dbg) {
      u64 *d = rlwe_dbg + (size_t)ct * 2 * N;
#pragma unroll
      for (int r = 0; r < 8; r++) {
        d[pos_coef<LOGN>(j, r)] = acc[0][r];
        d[N + pos_coef<LOGN>(j, r)] = acc[1][r];
      }
    }
  }
}

template <int LOGN, bool D1, int MINB>
__global__ void __launch_bounds__(NttShape<LOGN>::T, MINB)
    pbs_kernel(BrParams P, const u32 *ks, u32 ks_stride, const unsigned char *gates, u64 *out, int count,
               u64 *rlwe_dbg) {
  extern __shared__ u64 smem[];
  for (int ct = blockIdx.x; ct < count; ct += gridDim.x)
    pbs_item<LOGN, D1>(P, ct, ks + (size_t)ct * ks_stride, gates[ct], out, rlwe_dbg, smem);
}

// Ragged batch: ciphertext ct uses the parameter set and server key of
// descriptor item_desc[ct] (sessions of different parameter sets in one
// launch); outputs scatter to out_idx[ct].
template <int LOGN, bool D1, int MINB>
__global__ void __launch_bounds__(NttShape<LOGN>::T, MINB)
    pbs_ragged_kernel(const BrParams *descs, const u32 *item_desc, const u32 *ks, u32 ks_stride,
                      const unsigned char *gates, u64 *out, const u32 *out_idx, int count) {
  extern __shared__ u64 smem[];
  __shared__ BrParams sp;
  for (int ct = blockIdx.x; ct < count; ct += gridDim.x) {
    __syncthreads();  // the previous item is done with sp
    if (threadIdx.x == 0) {
      sp = descs[item_desc[ct]];
      sp.out_idx = out_idx;
    }
    __syncthreads();
    pbs_item<LOGN, D1>(sp, ct, ks + (size_t)ct * ks_stride, gates[ct], out, nullptr, smem);
  }
}

// ---------------------------------------------------------------------------
// Blind rotation with the keys streamed into shared memory (launch shape
// PBS_BULK, N = 2048, one-digit decompositions).  Each CTA keeps a 64 KB key
// stage.  Right after an operation's multiply-accumulate has read the stage,
// one thread issues the bulk copy (cp.async.bulk + mbarrier, from this GPU's
// memory, no multicast) of the next operation's key rows -- the 4 RGSW rows
// (64 KB) or the 2 automorphism-key rows (32 KB), contiguous in the device
// layout -- which lands while the CTA runs this operation's inverse
// transform and the next one's decomposition and forward transform.  The
// multiply-accumulate then reads its key from shared memory, not from L2.
// Two CTAs per SM (the stage); the register cap is 128.  Every wait is
// bounded: one that runs out sets DEVERR_MBAR_TIMEOUT and the CTA returns.
// ---------------------------------------------------------------------------
constexpr int BULK_REGIONS = 6;  // 2N words exchange / permutations, 4N words key stage

static size_t bulk_sched_bytes(u32 br_q, u32 n) {
  const size_t R = br_q / 2;
  size_t extra = ((R + 1) + n + (n + R + 1)) * 2 + 4;
  return (extra + 15) & ~(size_t)15;
}
static size_t bulk_smem_bytes(u32 br_q, u32 n) {
  return (size_t)BULK_REGIONS * 8 * 2048 + bulk_sched_bytes(br_q, n) + 16;  // + the mbarrier
}
__device__ __forceinline__ u64 *bulk_bar(u64 *smem, u32 br_q, u32 n) {
  const u32 R = br_q / 2;
  u32 extra = ((R + 1) + n + (n + R + 1)) * 2 + 4;
  extra = (extra + 15) & ~15u;
  return (u64 *)((char *)smem + (size_t)BULK_REGIONS * 8 * 2048 + extra);
}

// Key rows of a keyed operation (not a trivial automorphism): source and bytes.
__device__ __forceinline__ void op_key_rows(const BrParams &P, u32 op, const u64 *&src, u32 &bytes) {
  constexpr size_t N = 2048;
  if (op & OP_AUTO) {
    src = P.autos + (size_t)(op & OP_SLOT) * P.auto_rows * N;
    bytes = P.auto_rows * (u32)N * 8;
  } else {
    src = P.rgsw + (size_t)(op & OP_INDEX) * P.rgsw_rows * N;
    bytes = P.rgsw_rows * (u32)N * 8;
  }
}
__device__ __forceinline__ bool op_keyed(u32 op) { return !((op & OP_AUTO) && (op & OP_TRIVIAL)); }

// mac_pair / mac_auto with the key rows in shared memory (device layout,
// row r at ks + r N).
__device__ __forceinline__ void mac_pair_staged(u64 (&x)[8], u64 (&y)[8], const u64 *ks, const RingConsts &rc) {
  constexpr int LOGN = 11, N = 2048;
  const int j = threadIdx.x;
  const u64 q = rc.q, qi = rc.qinv_neg;
#pragma unroll
  for (int rr = 0; rr < 4; rr++) {
    const int di = dev_index<LOGN>(j, 2 * rr);
    u64 a[2], b[2], c[2], d[2];
    lds2(ks + di, a[0], a[1]);
    lds2(ks + N + di, b[0], b[1]);
    lds2(ks + 2 * N + di, c[0], c[1]);
    lds2(ks + 3 * N + di, d[0], d[1]);
#pragma unroll
    for (int e = 0; e < 2; e++) {
      const int r = 2 * rr + e;
      const u64 xv = x[r], yv = y[r];
      u64 hi, lo, hi2, lo2;
      sum2_128(xv, a[e], yv, c[e], hi, lo);
      sum2_128(xv, b[e], yv, d[e], hi2, lo2);
      x[r] = mac_reduce<LOGN>(hi, lo, q, qi);
      y[r] = mac_reduce<LOGN>(hi2, lo2, q, qi);
    }
  }
}
__device__ __forceinline__ void mac_auto_staged(u64 (&x)[8], u64 (&y)[8], const u64 *ks, const RingConsts &rc) {
  constexpr int LOGN = 11, N = 2048;
  const int j = threadIdx.x;
  const u64 q = rc.q, qi = rc.qinv_neg, q2 = rc.q << 1;
#pragma unroll
  for (int rr = 0; rr < 4; rr++) {
    const int di = dev_index<LOGN>(j, 2 * rr);
    u64 a[2], b[2];
    lds2(ks + di, a[0], a[1]);
    lds2(ks + N + di, b[0], b[1]);
#pragma unroll
    for (int e = 0; e < 2; e++) {
      const int r = 2 * rr + e;
      u64 hi, lo, hi2, lo2;
      mac_mul<LOGN>(x[r], a[e], hi, lo);
      mac_mul<LOGN>(x[r], b[e], hi2, lo2);
      x[r] = mac_reduce<LOGN>(hi, lo, q, qi);
      y[r] = mac_add_b<LOGN>(mac_reduce<LOGN>(hi2, lo2, q, qi) + y[r], q2);
    }
  }
}

// One keyed operation of the staged blind rotation: bootstrap_op's one-digit
// path with the key from the stage (its copy completes phase `parity` of
// *bar); after the multiply-accumulate the copy of the next operation's key
// (next_src, next_bytes; none when next_src is null) is issued into the same
// stage.  False (uniformly over the CTA) when the wait ran out.
__device__ __forceinline__ bool bootstrap_op_staged(u64 (&acc)[2][8], u32 op, const BrParams &P, u64 *sm,
                                                    u64 *stage, u64 *bar, u32 parity, const u64 *next_src,
                                                    u32 next_bytes) {
  constexpr int LOGN = 11, N = 2048;
  const u64 q = P.rc.q;
  const int j = threadIdx.x;
  u64(&x)[8] = acc[0];
  u64(&y)[8] = acc[1];
  const bool is_auto = (op & OP_AUTO) != 0;
  const bool keep_b = (op & OP_KEEPB) != 0;
  u64 *s_a = sm, *s_b = sm + N;
  if (is_auto) {  // non-trivial: a(X^k) with sign, b permuted in the evaluation domain
    const u32 k = P.auto_k[op & OP_SLOT];
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 8; r++) {
      u32 t = ((u32)pos_coef<LOGN>(j, r) * k) & (2 * N - 1);
      const bool neg = t >= (u32)N;
      if (neg) t -= N;
      s_a[swz(t)] = neg ? q - x[r] : x[r];
      s_b[swz(pos_eval<LOGN>(j, r))] = y[r];
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 8; r++) y[r] = s_b[swz(auto_eval_src<LOGN>(pos_eval<LOGN>(j, r), k))];
#pragma unroll
    for (int r = 0; r < 8; r++) x[r] = decompose1<AUTO_LOGB, AUTO_IGN>(s_a[swz(pos_coef<LOGN>(j, r))], q);
    ntt_fwd<LOGN, false>(x, x, sm, P.rc);
  } else {
#pragma unroll
    for (int r = 0; r < 8; r++) {
      x[r] = decompose1<RLRG_LOGB, RLRG_IGN>(x[r], q);
      y[r] = decompose1<RLRG_LOGB, RLRG_IGN>(y[r], q);
    }
    ntt_fwd<LOGN, true>(x, y, sm, P.rc);
  }
  if (!__syncthreads_and(mbar_wait(bar, parity))) {
    if (j == 0) {
      atomicOr(P.err, DEVERR_MBAR_TIMEOUT);
      mbar_wait(bar, parity);  // bounded: the copy this CTA still has in flight
    }
    return false;
  }
  if (is_auto) mac_auto_staged(x, y, stage, P.rc);
  else mac_pair_staged(x, y, stage, P.rc);
  __syncthreads();  // every thread has read the stage (also the exchange barrier of the inverse)
  if (j == 0 && next_src) {
    fence_proxy_async_smem();
    bulk_load(stage, next_src, next_bytes, bar);
  }
  if (keep_b) {
    ntt_inv<LOGN, false, false>(x, x, sm, P.rc);
#pragma unroll
    for (int r = 0; r < 8; r++) x[r] = reduce2(x[r], q);
  } else {
    ntt_inv<LOGN, true, false>(x, y, sm, P.rc);
#pragma unroll
    for (int r = 0; r < 8; r++) {
      x[r] = reduce2(x[r], q);
      y[r] = reduce2(y[r], q);
    }
  }
  return true;
}

// One gate bootstrap with staged keys; `phase` counts this CTA's completed
// waits (the mbarrier's phase parity).  False when a wait ran out.
__device__ __forceinline__ bool pbs_item_staged(const BrParams &P, int ct, const u32 *kso, u32 gcode, u64 *out,
                                                u64 *smem, u64 *bar, u32 &phase) {
  constexpr int LOGN = 11, N = 2048;
  u64 *sm = smem, *stage = smem + 2 * N;
  const SchedSmem S = sched_smem<LOGN>(smem, BULK_REGIONS, P.br_q >> 1, P.n);
  const int j = threadIdx.x;
  const u64 q = P.rc.q;
  build_schedule<LOGN>(P, kso, smem, S);
  u64 acc[2][8];
#pragma unroll
  for (int r = 0; r < 8; r++) acc[0][r] = 0;
  test_rlwe_b<LOGN>(P, kso, gcode, acc[1]);
  __syncthreads();
  const u32 nops = *S.nops;
  u32 t = 0;
  // trivial automorphisms (only before the first external product) need no key
#pragma unroll 1
  for (; t < nops && !op_keyed(S.ops[t]); t++) bootstrap_op<LOGN, true>(acc, S.ops[t], P, sm);
  if (j == 0 && t < nops) {
    const u64 *src;
    u32 bytes;
    op_key_rows(P, S.ops[t], src, bytes);
    fence_proxy_async_smem();
    bulk_load(stage, src, bytes, bar);
  }
#pragma unroll 1
  for (; t < nops; t++) {
    const u64 *nsrc = nullptr;
    u32 nbytes = 0;
    if (t + 1 < nops) op_key_rows(P, S.ops[t + 1], nsrc, nbytes);
    if (!bootstrap_op_staged(acc, S.ops[t], P, sm, stage, bar, phase & 1u, nsrc, nbytes)) return false;
    phase++;
  }
  // ---- sample extract at index 0 (pbs.rs:423-449)
  u64 *o = out + (size_t)(P.out_idx ? P.out_idx[ct] : (u32)ct) * (N + 1);
#pragma unroll
  for (int r = 0; r < 8; r++) {
    const u32 p = (u32)pos_coef<LOGN>(j, r);
    if (p == 0) {
      o[0] = acc[1][r];
      o[1] = acc[0][r];
    } else {
      o[1 + N - p] = q - acc[0][r];
    }
  }
  return true;
}

// The staged-key blind rotation over a ragged batch: item ct uses descriptor
// item_desc[ct] (parameter set and key of its session) and scatters to
// out_idx[ct]; the schedule arrays are laid out for the launch's maximum
// (br_q, n), the mbarrier after them.
__global__ void __launch_bounds__(256, 2)
    pbs_bulk_ragged_kernel(const BrParams *descs, const u32 *item_desc, const u32 *ks, u32 ks_stride,
                           const unsigned char *gates, u64 *out, const u32 *out_idx, int count, u32 max_br_q,
                           u32 max_n) {
  extern __shared__ __align__(128) u64 smem[];
  __shared__ BrParams sp;
  u64 *bar = bulk_bar(smem, max_br_q, max_n);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_init_fence();
  }
  u32 phase = 0;
  for (int ct = blockIdx.x; ct < count; ct += gridDim.x) {
    __syncthreads();  // the previous item is done with sp (and the mbarrier is initialised)
    if (threadIdx.x == 0) {
      sp = descs[item_desc[ct]];
      sp.out_idx = out_idx;
    }
    __syncthreads();
    if (!pbs_item_staged(sp, ct, ks + (size_t)ct * ks_stride, gates[ct], out, smem, bar, phase)) return;
  }
}

__global__ void __launch_bounds__(256, 2)
    pbs_bulk_kernel(BrParams P, const u32 *ks, u32 ks_stride, const unsigned char *gates, u64 *out, int count) {
  extern __shared__ __align__(128) u64 smem[];
  u64 *bar = bulk_bar(smem, P.br_q, P.n);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  u32 phase = 0;
  for (int ct = blockIdx.x; ct < count; ct += gridDim.x)
    if (!pbs_item_staged(P, ct, ks + (size_t)ct * ks_stride, gates[ct], out, smem, bar, phase)) return;
}

// ---------------------------------------------------------------------------
// Low-latency blind rotation: one ciphertext on a cluster of two CTAs (two
// SMs).  CTA rank 0 holds a, rank 1 holds b (same layouts and domains as the
// one-CTA kernel: b is left in the evaluation domain ahead of non-trivial
// automorphisms).  Per operation each CTA transforms only its own polynomial;
// the transformed digits cross to the other CTA through distributed shared
// memory (a two-slot buffer, alternating by operation), with exactly one
// cluster barrier per operation on both CTAs (both build the same schedule
// from the same input), and one more per ciphertext.  External product:
// each CTA forms one output row pair from both digit polynomials.
// Automorphism: rank 0 permutes, decomposes and transforms a(X^k); rank 1
// permutes b in the evaluation domain meanwhile; after the barrier rank 0
// multiplies by the key's A row, rank 1 by its B row and adds b(X^k).  The
// words are those of the one-CTA kernel (every step is the same exact
// arithmetic mod Q).  N = 2048, one-digit decompositions only.
// ---------------------------------------------------------------------------
namespace cg = cooperative_groups;

// out = mac_reduce(x ka + y kb), x, y in the evaluation layout, key rows in the device layout
template <int LOGN>
__device__ __forceinline__ void mac_two_rows(u64 (&x)[8], const u64 (&y)[8], const u64 *ka, const u64 *kb,
                                             const RingConsts &rc) {
  const int j = threadIdx.x;
  const u64 q = rc.q, qi = rc.qinv_neg;
#pragma unroll
  for (int rr = 0; rr < 4; rr++) {
    const int di = dev_index<LOGN>(j, 2 * rr);
    u64 a[2], b[2];
    ld_key2(ka + di, a[0], a[1]);
    ld_key2(kb + di, b[0], b[1]);
#pragma unroll
    for (int e = 0; e < 2; e++) {
      const int r = 2 * rr + e;
      u64 hi, lo;
      sum2_128(x[r], a[e], y[r], b[e], hi, lo);
      x[r] = mac_reduce<LOGN>(hi, lo, q, qi);
    }
  }
}

template <int LOGN>
__device__ __forceinline__ void split_op(u64 (&x)[8], u32 op, u32 t, const BrParams &P, u64 *sm, u64 *slots,
                                         const u64 *peer_slots, unsigned rank, cg::cluster_group &cl) {
  constexpr int N = 1 << LOGN, T = NttShape<LOGN>::T;
  const u64 q = P.rc.q, q2 = P.rc.q << 1;
  const int j = threadIdx.x;
  u64 *own = slots + (t & 1) * N;
  const u64 *peer = peer_slots + (t & 1) * N;
  const bool keep_b = (op & OP_KEEPB) != 0;
  if (op & OP_AUTO) {
    const u32 k = P.auto_k[op & OP_SLOT];
    if (op & OP_TRIVIAL) {  // runtime.rs:625-642: only b, permuted in the coefficient domain
      if (rank == 1) {
        __syncthreads();
#pragma unroll
        for (int r = 0; r < 8; r++) {
          u32 tt = ((u32)pos_coef<LOGN>(j, r) * k) & (2 * N - 1);
          const bool neg = tt >= (u32)N;
          if (neg) tt -= N;
          sm[swz(tt)] = neg ? q - x[r] : x[r];
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < 8; r++) x[r] = sm[swz(pos_coef<LOGN>(j, r))];
      }
      cl.sync();
      return;
    }
    const u64 *K = P.autos + (size_t)(op & OP_SLOT) * P.auto_rows * N;
    if (rank == 0) {  // a(X^k) with sign, one digit, forward transform
      __syncthreads();
#pragma unroll
      for (int r = 0; r < 8; r++) {
        u32 tt = ((u32)pos_coef<LOGN>(j, r) * k) & (2 * N - 1);
        const bool neg = tt >= (u32)N;
        if (neg) tt -= N;
        sm[swz(tt)] = neg ? q - x[r] : x[r];
      }
      __syncthreads();
#pragma unroll
      for (int r = 0; r < 8; r++) x[r] = decompose1<AUTO_LOGB, AUTO_IGN>(sm[swz(pos_coef<LOGN>(j, r))], q);
      ntt_fwd<LOGN, false>(x, x, sm, P.rc);
#pragma unroll
      for (int r = 0; r < 8; r++) own[r * T + j] = x[r];
    } else {  // b in the evaluation domain, permuted there
      u64 *sb = sm + N;
      __syncthreads();
#pragma unroll
      for (int r = 0; r < 8; r++) sb[swz(pos_eval<LOGN>(j, r))] = x[r];
      __syncthreads();
#pragma unroll
      for (int r = 0; r < 8; r++) x[r] = sb[swz(auto_eval_src<LOGN>(pos_eval<LOGN>(j, r), k))];
    }
    cl.sync();
    if (rank == 0) {
      u64 z[8];
#pragma unroll
      for (int r = 0; r < 8; r++) z[r] = 0;
      mac_two_rows<LOGN>(x, z, K, K, P.rc);  // a' = d A (second product is 0)
      ntt_inv<LOGN, false>(x, x, sm, P.rc);
#pragma unroll
      for (int r = 0; r < 8; r++) x[r] = reduce2(x[r], q);
    } else {
      u64 d[8], z[8];
#pragma unroll
      for (int r = 0; r < 8; r++) {
        d[r] = peer[r * T + j];
        z[r] = 0;
      }
      mac_two_rows<LOGN>(d, z, K + N, K + N, P.rc);  // d B
#pragma unroll
      for (int r = 0; r < 8; r++) x[r] = mac_add_b<LOGN>(d[r] + x[r], q2);
      if (!keep_b) {
        ntt_inv<LOGN, false>(x, x, sm, P.rc);
#pragma unroll
        for (int r = 0; r < 8; r++) x[r] = reduce2(x[r], q);
      }
    }
    return;
  }
  // external product: rows A(-sm), B(-sm), A(m), B(m) (d_a = d_b = 1)
  const u64 *K = P.rgsw + (size_t)(op & OP_INDEX) * P.rgsw_rows * N;
#pragma unroll
  for (int r = 0; r < 8; r++) x[r] = decompose1<RLRG_LOGB, RLRG_IGN>(x[r], q);
  ntt_fwd<LOGN, false>(x, x, sm, P.rc);
#pragma unroll
  for (int r = 0; r < 8; r++) own[r * T + j] = x[r];
  cl.sync();
  u64 y[8];
#pragma unroll
  for (int r = 0; r < 8; r++) y[r] = peer[r * T + j];
  // rank 0: a' = da A(-sm) + db A(m); rank 1: b' = da B(-sm) + db B(m)
  if (rank == 0) mac_two_rows<LOGN>(x, y, K, K + 2 * N, P.rc);
  else {
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const u64 tmp = x[r];
      x[r] = y[r];
      y[r] = tmp;
    }
    mac_two_rows<LOGN>(x, y, K + N, K + 3 * N, P.rc);
  }
  if (rank == 0 || !keep_b) {
    ntt_inv<LOGN, false>(x, x, sm, P.rc);
#pragma unroll
    for (int r = 0; r < 8; r++) x[r] = reduce2(x[r], q);
  }
}

template <int LOGN>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(NttShape<LOGN>::T, 2)
    pbs_split_kernel(BrParams P, const u32 *ks, u32 ks_stride, const unsigned char *gates, u64 *out, int count) {
  constexpr int N = 1 << LOGN;
  extern __shared__ u64 smem[];
  cg::cluster_group cl = cg::this_cluster();
  const unsigned rank = cl.block_rank();
  u64 *slots = smem + 2 * N;
  const u64 *peer_slots = cl.map_shared_rank(slots, rank ^ 1u);
  const SchedSmem S = sched_smem<LOGN>(smem, SPLIT_REGIONS, P.br_q >> 1, P.n);
  const int j = threadIdx.x;
  const u64 q = P.rc.q;
  const int ncl = gridDim.x / 2;
  for (int ct = blockIdx.x / 2; ct < count; ct += ncl) {  // both CTAs of a cluster take the same items
    const u32 *kso = ks + (size_t)ct * ks_stride;
    build_schedule<LOGN>(P, kso, smem, S);
    u64 x[8];
    if (rank == 0) {
#pragma unroll
      for (int r = 0; r < 8; r++) x[r] = 0;
    } else {
      test_rlwe_b<LOGN>(P, kso, gates[ct], x);
    }
    __syncthreads();
    const u32 nops = *S.nops;
#pragma unroll 1
    for (u32 t = 0; t < nops; t++) {
      if (j == 0 && t + 1 < nops) prefetch_next_key<LOGN>(P, S.ops[t + 1]);
      split_op<LOGN>(x, S.ops[t], t, P, smem, slots, peer_slots, rank, cl);
    }
    // sample extract at index 0 (pbs.rs:423-449): rank 0 the a-part, rank 1 b[0]
    u64 *o = out + (size_t)(P.out_idx ? P.out_idx[ct] : (u32)ct) * (N + 1);
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const u32 p = (u32)pos_coef<LOGN>(j, r);
      if (rank == 0) {
        if (p == 0) o[1] = x[r];
        else o[1 + N - p] = q - x[r];
      } else if (p == 0) {
        o[0] = x[r];
      }
    }
    cl.sync();  // the digit slots are reused by the next ciphertext
  }
}

// The two-CTA kernel over a ragged batch: item ct uses the parameter set and
// key of descriptor item_desc[ct] (both CTAs of its cluster load the same
// descriptor) and scatters its output to out_idx[ct]; the schedule arrays are
// laid out for the item's own (br_q, n) inside the launch's maximum.
template <int LOGN>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(NttShape<LOGN>::T, 2)
    pbs_split_ragged_kernel(const BrParams *descs, const u32 *item_desc, const u32 *ks, u32 ks_stride,
                            const unsigned char *gates, u64 *out, const u32 *out_idx, int count) {
  constexpr int N = 1 << LOGN;
  extern __shared__ u64 smem[];
  __shared__ BrParams sp;
  cg::cluster_group cl = cg::this_cluster();
  const unsigned rank = cl.block_rank();
  u64 *slots = smem + 2 * N;
  const u64 *peer_slots = cl.map_shared_rank(slots, rank ^ 1u);
  const int j = threadIdx.x;
  const int ncl = gridDim.x / 2;
  for (int ct = blockIdx.x / 2; ct < count; ct += ncl) {  // both CTAs of a cluster take the same items
    if (threadIdx.x == 0) sp = descs[item_desc[ct]];
    __syncthreads();
    const SchedSmem S = sched_smem<LOGN>(smem, SPLIT_REGIONS, sp.br_q >> 1, sp.n);
    const u64 q = sp.rc.q;
    const u32 *kso = ks + (size_t)ct * ks_stride;
    build_schedule<LOGN>(sp, kso, smem, S);
    u64 x[8];
    if (rank == 0) {
#pragma unroll
      for (int r = 0; r < 8; r++) x[r] = 0;
    } else {
      test_rlwe_b<LOGN>(sp, kso, gates[ct], x);
    }
    __syncthreads();
    const u32 nops = *S.nops;
#pragma unroll 1
    for (u32 t = 0; t < nops; t++) {
      if (j == 0 && t + 1 < nops) prefetch_next_key<LOGN>(sp, S.ops[t + 1]);
      split_op<LOGN>(x, S.ops[t], t, sp, smem, slots, peer_slots, rank, cl);
    }
    u64 *o = out + (size_t)out_idx[ct] * (N + 1);
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const u32 p = (u32)pos_coef<LOGN>(j, r);
      if (rank == 0) {
        if (p == 0) o[1] = x[r];
        else o[1 + N - p] = q - x[r];
      } else if (p == 0) {
        o[0] = x[r];
      }
    }
    cl.sync();  // the digit slots and sp are reused by the next ciphertext
  }
}

// Throughput probe for the roofline denominator: 8 independent chains of
// 32-bit multiply-adds per thread (mad.lo.u32, the IMAD the 64-bit modular
// multiplications are built from).  `sink` keeps the chains live.
__global__ void imad_probe_kernel(u32 iters, u32 seed, u32 *sink) {
  u32 x[8];
#pragma unroll
  for (int i = 0; i < 8; i++) x[i] = seed + threadIdx.x * 8 + i;
  const u32 m = seed | 1u, c = seed ^ 0x9e3779b9u;
  for (u32 it = 0; it < iters; it++) {
#pragma unroll
    for (int u = 0; u < 16; u++) {
#pragma unroll
      for (int i = 0; i < 8; i++) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(x[i]) : "r"(m), "r"(c));
    }
  }
  u32 acc = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) acc ^= x[i];
  if (acc == 0x12345678u) sink[blockIdx.x] = acc;
}

cudaError_t launch_imad_probe(int blocks, int threads, u32 iters, u32 *sink, cudaStream_t s) {
  imad_probe_kernel<<<blocks, threads, 0, s>>>(iters, 0x2545F491u, sink);
  return cudaGetLastError();
}

// Pipe-rate probe behind the butterflies' design: 8 independent chains per
// thread of one instruction kind, 16 x 8 per iteration.  KIND 0 mad.lo.u32
// (IMAD), 1 mad.wide.u32 (IMAD.WIDE), 2 mad.hi.u32 (IMAD.HI), 3 fma.rn.f64,
// 4 cvt.rn.f64.u64, 5 cvt.rni.u64.f64, 6 mad.lo.u32 and fma.rn.f64
// interleaved (the rate of each).
template <int KIND>
__global__ void pipe_probe_kernel(u32 iters, u32 seed, u32 *sink) {
  u64 x[8];
  double f[8];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    x[i] = ((u64)(seed + threadIdx.x * 8 + i) << 20) | i;
    f[i] = (double)(seed + threadIdx.x + i);
  }
  const u32 m = seed | 1u, c = seed ^ 0x9e3779b9u;
  const double fm = 1.0000001, fc = 1e-9;
  for (u32 it = 0; it < iters; it++) {
#pragma unroll
    for (int u = 0; u < 16; u++) {
#pragma unroll
      for (int i = 0; i < 8; i++) {
        if (KIND == 0 || KIND == 6) {
          u32 v = (u32)x[i];
          asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(v) : "r"(m), "r"(c));
          x[i] = v;
        }
        if (KIND == 1) asm volatile("mad.wide.u32 %0, %1, %2, %0;" : "+l"(x[i]) : "r"((u32)x[i]), "r"(m));
        if (KIND == 2) {
          u32 v = (u32)x[i];
          asm volatile("mad.hi.u32 %0, %0, %1, %2;" : "+r"(v) : "r"(m), "r"(c));
          x[i] = v;
        }
        if (KIND == 3 || KIND == 6) asm volatile("fma.rn.f64 %0, %0, %1, %2;" : "+d"(f[i]) : "d"(fm), "d"(fc));
        if (KIND == 4) {
          double d;
          asm volatile("cvt.rn.f64.u64 %0, %1;" : "=d"(d) : "l"(x[i]));
          x[i] = (u64)__double_as_longlong(d) >> 3;
        }
        if (KIND == 5) {
          u64 q;
          asm volatile("cvt.rni.u64.f64 %0, %1;" : "=l"(q) : "d"(f[i]));
          f[i] = __longlong_as_double((long long)(q | 0x4100000000000000ull));
        }
      }
    }
  }
  u64 acc = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) acc ^= x[i] ^ (u64)__double_as_longlong(f[i]);
  if (acc == 0x12345678ull) sink[blockIdx.x] = (u32)acc;
}

cudaError_t launch_pipe_probe(int kind, int blocks, int threads, u32 iters, u32 *sink, cudaStream_t s) {
  switch (kind) {
    case 0: pipe_probe_kernel<0><<<blocks, threads, 0, s>>>(iters, 0x2545F491u, sink); break;
    case 1: pipe_probe_kernel<1><<<blocks, threads, 0, s>>>(iters, 0x2545F491u, sink); break;
    case 2: pipe_probe_kernel<2><<<blocks, threads, 0, s>>>(iters, 0x2545F491u, sink); break;
    case 3: pipe_probe_kernel<3><<<blocks, threads, 0, s>>>(iters, 0x2545F491u, sink); break;
    case 4: pipe_probe_kernel<4><<<blocks, threads, 0, s>>>(iters, 0x2545F491u, sink); break;
    case 5: pipe_probe_kernel<5><<<blocks, threads, 0, s>>>(iters, 0x2545F491u, sink); break;
    case 6: pipe_probe_kernel<6><<<blocks, threads, 0, s>>>(iters, 0x2545F491u, sink); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

__global__ void not_kernel(const u64 *in, u64 *out, size_t words, u64 q) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < words; i += (size_t)gridDim.x * blockDim.x)
    out[i] = q - in[i];  // neg = q - a, evaluator.rs:2247-2250
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
static int grid_for(size_t count) { return (int)(count < 65535 * 16 ? count : 65535 * 16); }

cudaError_t launch_key_convert(int logn, const u64 *in, u64 *out, size_t npolys, const RingConsts &rc,
                               u64 c, u64 cs, cudaStream_t s) {
  if (npolys == 0) return cudaSuccess;
  if (logn == 11) key_convert_kernel<11><<<grid_for(npolys), 256, 0, s>>>(in, out, npolys, rc, c, cs);
  else if (logn == 9) key_convert_kernel<9><<<grid_for(npolys), 64, 0, s>>>(in, out, npolys, rc, c, cs);
  else return cudaErrorInvalidValue;
  return cudaGetLastError();
}

template <typename K>
static cudaError_t set_smem(K kernel, size_t bytes);

// Persistent grid of the batched NTT: two CTAs per SM, no more CTAs than pairs.
static int ntt_batch_grid(size_t count) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t pairs = (count + 1) / 2;
  return (int)std::min<size_t>(pairs, (size_t)2 * sms);
}

cudaError_t launch_ntt_fwd(int logn, u64 *polys, size_t count, const RingConsts &rc, u32 *err, cudaStream_t s) {
  if (count == 0) return cudaSuccess;
  if (logn == 11) {
    cudaError_t e = set_smem(ntt_batch_kernel<false>, NTTB_SMEM);
    if (e != cudaSuccess) return e;
    ntt_batch_kernel<false><<<ntt_batch_grid(count), 256, NTTB_SMEM, s>>>(polys, count, rc, err);
  } else if (logn == 9) {
    ntt_fwd_kernel<9><<<grid_for(count), 64, 0, s>>>(polys, count, rc);
  } else {
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_ntt_inv(int logn, u64 *polys, size_t count, const RingConsts &rc, u32 *err, cudaStream_t s) {
  if (count == 0) return cudaSuccess;
  if (logn == 11) {
    cudaError_t e = set_smem(ntt_batch_kernel<true>, NTTB_SMEM);
    if (e != cudaSuccess) return e;
    ntt_batch_kernel<true><<<ntt_batch_grid(count), 256, NTTB_SMEM, s>>>(polys, count, rc, err);
  } else if (logn == 9) {
    ntt_inv_kernel<9><<<grid_for(count), 64, 0, s>>>(polys, count, rc);
  } else {
    return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// Opt the kernel into its dynamic shared memory once (largest size asked so
// far), outside of any launch sequence that may be captured into a graph.
template <typename K>
static cudaError_t set_smem(K kernel, size_t bytes) {
  // the attribute is per kernel and per device: remember the largest size set
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, size_t> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  size_t &have = done[{(const void *)kernel, dev}];
  if (bytes <= have) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) have = bytes;
  return e;
}
cudaError_t launch_ext_product(int logn, bool d1, const BrParams &P, u64 *rlwe, const u32 *idx,
                               size_t count, int trivial, cudaStream_t s, int variant) {
  if (count == 0) return cudaSuccess;
  const size_t N = (size_t)1 << logn, smem = OP_REGIONS * N * 8;
  cudaError_t e;
#define PZ_LAUNCH(LN, DD, MB, TH)                                                                  \
  if ((e = set_smem(ext_product_kernel<LN, DD, MB>, smem)) != cudaSuccess) return e;              \
  ext_product_kernel<LN, DD, MB><<<grid_for(count), TH, smem, s>>>(P, rlwe, idx, count, trivial);
  if (logn == 11 && d1) {
    if (variant == 0) { PZ_LAUNCH(11, true, 2, 256) }
    else if (variant == 2) { PZ_LAUNCH(11, true, 4, 256) }
    else { PZ_LAUNCH(11, true, 3, 256) }
  }
  else if (logn == 11) { PZ_LAUNCH(11, false, 1, 256) }
  else if (logn == 9 && d1) { PZ_LAUNCH(9, true, 1, 64) }
  else if (logn == 9) { PZ_LAUNCH(9, false, 1, 64) }
  else return cudaErrorInvalidValue;
#undef PZ_LAUNCH
  return cudaGetLastError();
}

cudaError_t launch_auto(int logn, bool d1, const BrParams &P, u64 *rlwe, const u32 *slot, size_t count,
                        int trivial, cudaStream_t s, int variant) {
  if (count == 0) return cudaSuccess;
  const size_t N = (size_t)1 << logn, smem = OP_REGIONS * N * 8;
  cudaError_t e;
#define PZ_LAUNCH(LN, DD, MB, TH)                                                           \
  if ((e = set_smem(auto_kernel<LN, DD, MB>, smem)) != cudaSuccess) return e;              \
  auto_kernel<LN, DD, MB><<<grid_for(count), TH, smem, s>>>(P, rlwe, slot, count, trivial);
  if (logn == 11 && d1) {
    if (variant == 0) { PZ_LAUNCH(11, true, 2, 256) }
    else if (variant == 2) { PZ_LAUNCH(11, true, 4, 256) }
    else { PZ_LAUNCH(11, true, 3, 256) }
  }
  else if (logn == 11) { PZ_LAUNCH(11, false, 1, 256) }
  else if (logn == 9 && d1) { PZ_LAUNCH(9, true, 1, 64) }
  else if (logn == 9) { PZ_LAUNCH(9, false, 1, 64) }
  else return cudaErrorInvalidValue;
#undef PZ_LAUNCH
  return cudaGetLastError();
}

// Shares of the input coefficients per key-switch tile: enough CTAs for
// about four per SM (small batches), at least KS_IC coefficients per share.
static unsigned ks_split(size_t tiles_xy, u32 N) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t target = (size_t)4 * sms, chunks = N / KS_IC;
  unsigned z = 1;
  while (tiles_xy * z < target && 2 * z <= chunks) z *= 2;
  return z;
}

__global__ void ks_mask_kernel(u32 *out, size_t count, u32 stride, u32 cols, u32 mask) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count * cols; i += (size_t)gridDim.x * blockDim.x)
    out[(i / cols) * stride + i % cols] &= mask;
}

cudaError_t launch_ks(const KsParams &P, const unsigned char *gates, const u64 *c0, const u64 *c1,
                      size_t count, u32 *out, cudaStream_t s, bool reduce_output, int ct) {
  if (count == 0) return cudaSuccess;
  if (P.d > (u32)MAX_KS_D) return cudaErrorInvalidValue;
  // the tensor-core form needs the key's byte planes; a key without them
  // (digits wider than s8, or no memory for the planes) runs the 16-tile
  if (ct == KS_CT_MMA && (!P.ksk8 || P.planes < 1 || P.planes > 3 || P.d > 16 || (P.d * P.N) % 32 || P.N % 32))
    ct = 16;
  if (ct == KS_CT_MMA) {
    dim3 grid((unsigned)((count + KSM_ROWS - 1) / KSM_ROWS), P.ksk8_cols / KSM_COLS);
    grid.z = ks_split((size_t)grid.x * grid.y, P.N);
    const size_t smem = ksm_smem_bytes(P.d, P.planes);
    cudaError_t e;
    if (grid.z > 1 && (e = cudaMemsetAsync(out, 0, count * P.out_stride * sizeof(u32), s)) != cudaSuccess) return e;
#define PZ_KSM(NP)                                                              if ((e = set_smem(ks_mma_kernel<NP>, smem)) != cudaSuccess) return e;         ks_mma_kernel<NP><<<grid, 256, smem, s>>>(P, gates, c0, c1, (int)count, out);
    if (P.planes == 1) { PZ_KSM(1) }
    else if (P.planes == 2) { PZ_KSM(2) }
    else { PZ_KSM(3) }
#undef PZ_KSM
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (grid.z > 1 && reduce_output) {
      const size_t words = count * (P.n + 1);
      ks_mask_kernel<<<(unsigned)std::min<size_t>((words + 255) / 256, 4096), 256, 0, s>>>(out, count, P.out_stride,
                                                                                          P.n + 1, P.mask);
      return cudaGetLastError();
    }
    return cudaSuccess;
  }
  if (ct != 8 && ct != 16 && ct != 32) return cudaErrorInvalidValue;
  dim3 grid((unsigned)((count + ct - 1) / ct), (unsigned)((P.n + 1 + KS_COLS - 1) / KS_COLS));
  grid.z = ks_split((size_t)grid.x * grid.y, P.N);
  cudaError_t e;
  if (grid.z > 1 && (e = cudaMemsetAsync(out, 0, count * P.out_stride * sizeof(u32), s)) != cudaSuccess) return e;
  const size_t smem = ks_dig_bytes(ct);
#define PZ_KS(CT)                                                              \
  if ((e = set_smem(ks_kernel<CT>, smem)) != cudaSuccess) return e;           \
  ks_kernel<CT><<<grid, KS_COLS, smem, s>>>(P, gates, c0, c1, (int)count, out);
  if (ct == 8) { PZ_KS(8) }
  else if (ct == 16) { PZ_KS(16) }
  else { PZ_KS(32) }
#undef PZ_KS
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (grid.z > 1 && reduce_output) {
    const size_t words = count * (P.n + 1);
    ks_mask_kernel<<<(unsigned)std::min<size_t>((words + 255) / 256, 4096), 256, 0, s>>>(out, count, P.out_stride,
                                                                                        P.n + 1, P.mask);
    return cudaGetLastError();
  }
  return cudaSuccess;
}

cudaError_t launch_ksk_planes(const u32 *ksk, u32 rows, u32 stride, u32 n, u32 planes, unsigned char *out,
                              cudaStream_t s) {
  if (rows % 32 || planes < 1 || planes > 3) return cudaErrorInvalidValue;
  const u32 cols = ksk8_cols(n);
  const size_t total = (size_t)rows * cols;
  ksk_planes_kernel<<<(unsigned)std::min<size_t>((total + 255) / 256, 8192), 256, 0, s>>>(ksk, rows, stride, n,
                                                                                          planes, cols, out);
  return cudaGetLastError();
}

cudaError_t launch_pbs(int logn, bool d1, const BrParams &P, const u32 *ks, u32 ks_stride,
                       const unsigned char *gates, u64 *out, size_t count, u64 *rlwe_dbg, int grid_limit,
                       cudaStream_t s, int variant) {
  if (count == 0) return cudaSuccess;
  const size_t smem = pbs_smem_bytes(logn, P.br_q, P.n);
  int grid = (int)count;
  if (grid_limit > 0 && grid > grid_limit) grid = grid_limit;
  cudaError_t e;
#define PZ_LAUNCH(LN, DD, MB, TH)                                                                    \
  if ((e = set_smem(pbs_kernel<LN, DD, MB>, smem)) != cudaSuccess) return e;                        \
  pbs_kernel<LN, DD, MB><<<grid, TH, smem, s>>>(P, ks, ks_stride, gates, out, (int)count, rlwe_dbg);
  if (logn == 11 && d1 && variant == PBS_SPLIT && rlwe_dbg == nullptr) {
    const size_t ssmem = split_smem_bytes(P.br_q, P.n);
    if ((e = set_smem(pbs_split_kernel<11>, ssmem)) != cudaSuccess) return e;
    pbs_split_kernel<11><<<2 * grid, 256, ssmem, s>>>(P, ks, ks_stride, gates, out, (int)count);
    return cudaGetLastError();
  }
  if (logn == 11 && d1 && variant == PBS_BULK && rlwe_dbg == nullptr) {
    const size_t bsmem = bulk_smem_bytes(P.br_q, P.n);
    if ((e = set_smem(pbs_bulk_kernel, bsmem)) != cudaSuccess) return e;
    pbs_bulk_kernel<<<grid, 256, bsmem, s>>>(P, ks, ks_stride, gates, out, (int)count);
    return cudaGetLastError();
  }
  if (variant > 2) variant = 0;  // shapes without a debug-output form
  if (logn == 11 && d1) {
    if (variant == 0) { PZ_LAUNCH(11, true, 2, 256) }
    else if (variant == 1) { PZ_LAUNCH(11, true, 3, 256) }
    else { PZ_LAUNCH(11, true, 4, 256) }
  }
  else if (logn == 11) { PZ_LAUNCH(11, false, 1, 256) }
  else if (logn == 9 && d1) { PZ_LAUNCH(9, true, 1, 64) }
  else if (logn == 9) { PZ_LAUNCH(9, false, 1, 64) }
  else return cudaErrorInvalidValue;
#undef PZ_LAUNCH
  return cudaGetLastError();
}

// Items a blind-rotation launch holds resident at once on the current device
// with launch shape `variant` (CTAs per SM from the occupancy calculator x
// SMs; one item per two-CTA cluster for the split shape).  A batch that is a
// multiple of this runs in whole waves.
cudaError_t pbs_slots(int logn, bool d1, u32 br_q, u32 n, int variant, size_t *slots) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const size_t smem = pbs_smem_bytes(logn, br_q, n);
  size_t div = 1;
#define PZ_OCC(K, TH, SM)                                                                 \
  if ((e = set_smem(K, SM)) != cudaSuccess) return e;                                      \
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, K, TH, SM);
  if (logn == 11 && d1 && variant == PBS_SPLIT) {
    PZ_OCC(pbs_split_kernel<11>, 256, split_smem_bytes(br_q, n))
    div = 2;
  } else if (logn == 11 && d1 && variant == PBS_BULK) {
    PZ_OCC(pbs_bulk_kernel, 256, bulk_smem_bytes(br_q, n))
  } else if (logn == 11 && d1) {
    if (variant == 0) { PZ_OCC((pbs_kernel<11, true, 2>), 256, smem) }
    else if (variant == 1) { PZ_OCC((pbs_kernel<11, true, 3>), 256, smem) }
    else { PZ_OCC((pbs_kernel<11, true, 4>), 256, smem) }
  } else if (logn == 11) { PZ_OCC((pbs_kernel<11, false, 1>), 256, smem) }
  else if (logn == 9 && d1) { PZ_OCC((pbs_kernel<9, true, 1>), 64, smem) }
  else if (logn == 9) { PZ_OCC((pbs_kernel<9, false, 1>), 64, smem) }
  else return cudaErrorInvalidValue;
#undef PZ_OCC
  if (e != cudaSuccess) return e;
  *slots = std::max<size_t>((size_t)per_sm * sms / div, 1);
  return cudaSuccess;
}

cudaError_t launch_ks_ragged(const KsParams *d_descs, const KsTile *d_tiles, size_t ntiles, size_t count,
                             u32 max_n, u32 max_N, u32 max_d, const unsigned char *gates, const u64 *wires,
                             const u32 *in0, const u32 *in1, u32 *out, u32 out_stride, cudaStream_t s) {
  if (ntiles == 0) return cudaSuccess;
  if (max_d > (u32)MAX_KS_D) return cudaErrorInvalidValue;
  dim3 grid((unsigned)ntiles, (unsigned)((max_n + 1 + KS_COLS - 1) / KS_COLS));
  grid.z = ks_split((size_t)grid.x * grid.y, max_N);
  cudaError_t e;
  if (grid.z > 1 && (e = cudaMemsetAsync(out, 0, count * out_stride * sizeof(u32), s)) != cudaSuccess) return e;
  ks_ragged_kernel<<<grid, KS_COLS, 0, s>>>(d_descs, d_tiles, gates, wires, in0, in1, out, out_stride);
  return cudaGetLastError();
}

cudaError_t launch_ks_mma_ragged(const KsParams *d_descs, const KsTile *d_tiles, size_t ntiles, size_t count,
                                 u32 max_n, u32 max_N, u32 max_d, const unsigned char *gates, const u64 *wires,
                                 const u32 *in0, const u32 *in1, u32 *out, u32 out_stride, cudaStream_t s) {
  if (ntiles == 0) return cudaSuccess;
  if (max_d > 16) return cudaErrorInvalidValue;
  dim3 grid((unsigned)ntiles, ksk8_cols(max_n) / KSM_COLS);
  grid.z = ks_split((size_t)grid.x * grid.y, max_N);
  const size_t smem = ksm_smem_bytes(max_d, 3);
  cudaError_t e;
  if (grid.z > 1 && (e = cudaMemsetAsync(out, 0, count * out_stride * sizeof(u32), s)) != cudaSuccess) return e;
  if ((e = set_smem(ks_mma_ragged_kernel, smem)) != cudaSuccess) return e;
  ks_mma_ragged_kernel<<<grid, 256, smem, s>>>(d_descs, d_tiles, gates, wires, in0, in1, out, out_stride);
  return cudaGetLastError();
}

cudaError_t launch_pbs_ragged(int logn, bool d1, const BrParams *d_descs, const u32 *item_desc, u32 max_br_q,
                              u32 max_n, const u32 *ks, u32 ks_stride, const unsigned char *gates, u64 *out,
                              const u32 *out_idx, size_t count, int grid_limit, cudaStream_t s, int variant) {
  if (count == 0) return cudaSuccess;
  const size_t smem = pbs_smem_bytes(logn, max_br_q, max_n);
  int grid = (int)count;
  if (grid_limit > 0 && grid > grid_limit) grid = grid_limit;
  cudaError_t e;
  if (logn == 11 && d1 && variant == PBS_SPLIT) {
    const size_t ssmem = split_smem_bytes(max_br_q, max_n);
    if ((e = set_smem(pbs_split_ragged_kernel<11>, ssmem)) != cudaSuccess) return e;
    pbs_split_ragged_kernel<11><<<2 * grid, 256, ssmem, s>>>(d_descs, item_desc, ks, ks_stride, gates, out, out_idx,
                                                             (int)count);
    return cudaGetLastError();
  }
  if (logn == 11 && d1 && variant == PBS_BULK) {
    const size_t bsmem = bulk_smem_bytes(max_br_q, max_n);
    if ((e = set_smem(pbs_bulk_ragged_kernel, bsmem)) != cudaSuccess) return e;
    pbs_bulk_ragged_kernel<<<grid, 256, bsmem, s>>>(d_descs, item_desc, ks, ks_stride, gates, out, out_idx,
                                                    (int)count, max_br_q, max_n);
    return cudaGetLastError();
  }
  if (variant > 2) variant = 0;
#define PZ_LAUNCH(LN, DD, MB, TH)                                                                    \
  if ((e = set_smem(pbs_ragged_kernel<LN, DD, MB>, smem)) != cudaSuccess) return e;                 \
  pbs_ragged_kernel<LN, DD, MB><<<grid, TH, smem, s>>>(d_descs, item_desc, ks, ks_stride, gates, out, out_idx, \
                                                       (int)count);
  if (logn == 11 && d1) {
    if (variant == 0) { PZ_LAUNCH(11, true, 2, 256) }
    else if (variant == 1) { PZ_LAUNCH(11, true, 3, 256) }
    else { PZ_LAUNCH(11, true, 4, 256) }
  }
  else if (logn == 11) { PZ_LAUNCH(11, false, 1, 256) }
  else if (logn == 9 && d1) { PZ_LAUNCH(9, true, 1, 64) }
  else if (logn == 9) { PZ_LAUNCH(9, false, 1, 64) }
  else return cudaErrorInvalidValue;
#undef PZ_LAUNCH
  return cudaGetLastError();
}

cudaError_t launch_not(const u64 *in, u64 *out, size_t words, u64 q, cudaStream_t s) {
  if (words == 0) return cudaSuccess;
  size_t blocks = (words + 255) / 256;
  if (blocks > 4096) blocks = 4096;
  not_kernel<<<(unsigned)blocks, 256, 0, s>>>(in, out, words, q);
  return cudaGetLastError();
}

}  // namespace pz
