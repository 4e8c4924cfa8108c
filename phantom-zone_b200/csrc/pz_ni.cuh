// pz_ni.cuh -- pieces shared by the non-interactive translation units: the
// ChaCha8 block function (device, and host for seed derivation), and the
// key-switch multiply-accumulate of one digit pair against a ui_to_s key.
#pragma once
#include "pz_device.cuh"

namespace pz {
namespace ni {

constexpr int NI_T = 256;  // threads per RLWE (8 coefficients each, N = 2048)
constexpr int NI_LOGN = 11;

struct ChaChaKey {
  u32 k[8];
};

inline ChaChaKey chacha_key(const uint8_t seed[32]) {
  ChaChaKey key;
  for (int i = 0; i < 8; i++)
    key.k[i] = (u32)seed[4 * i] | ((u32)seed[4 * i + 1] << 8) | ((u32)seed[4 * i + 2] << 16) |
               ((u32)seed[4 * i + 3] << 24);
  return key;
}

#ifdef __CUDA_ARCH__
#define PZ_HD_UNROLL _Pragma("unroll")
#else
#define PZ_HD_UNROLL
#endif

__host__ __device__ __forceinline__ u32 rotl32(u32 v, int c) { return (v << c) | (v >> (32 - c)); }

// The ChaCha block function (the published algorithm, as RFC 8439 section
// 2.3 states it for 20 rounds) on a full 16-word input state: ROUNDS / 2
// double rounds, then the input added word by word.
template <int ROUNDS>
__host__ __device__ __forceinline__ void chacha_core(const u32 (&s)[16], u32 (&out)[16]) {
  static_assert(ROUNDS % 2 == 0, "double rounds");
  u32 x[16];
PZ_HD_UNROLL
  for (int i = 0; i < 16; i++) x[i] = s[i];
#define PZ_QR(a, b, c, d)                              \
  x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 16);        \
  x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 12);        \
  x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 8);         \
  x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 7);
PZ_HD_UNROLL
  for (int r = 0; r < ROUNDS / 2; r++) {
    PZ_QR(0, 4, 8, 12) PZ_QR(1, 5, 9, 13) PZ_QR(2, 6, 10, 14) PZ_QR(3, 7, 11, 15)
    PZ_QR(0, 5, 10, 15) PZ_QR(1, 6, 11, 12) PZ_QR(2, 7, 8, 13) PZ_QR(3, 4, 9, 14)
  }
#undef PZ_QR
PZ_HD_UNROLL
  for (int i = 0; i < 16; i++) out[i] = x[i] + s[i];
}

// ChaCha8 block `counter` in the rand_chacha 0.3 layout (constants, 8 key
// words, 64-bit block counter in words 12-13, stream id 0 in words 14-15);
// 16 output words, consumed low word first by rand_core's BlockRng.
__host__ __device__ __forceinline__ void chacha8_block(const ChaChaKey &key, u64 counter, u32 (&out)[16]) {
  u32 s[16];
  s[0] = 0x61707865u; s[1] = 0x3320646eu; s[2] = 0x79622d32u; s[3] = 0x6b206574u;
PZ_HD_UNROLL
  for (int i = 0; i < 8; i++) s[4 + i] = key.k[i];
  s[12] = (u32)counter; s[13] = (u32)(counter >> 32); s[14] = 0; s[15] = 0;
  chacha_core<8>(s, out);
}

// rand 0.8's UniformInt<u64> built by new_inclusive(0, q - 1) and sampled
// (the fill of random.rs:93-110): zone = MAX - (2^64 - q) mod q; a 64-bit
// word v is accepted when lo64(v q) <= zone, and the sample is hi64(v q).
__host__ __device__ __forceinline__ u64 uniform_zone(u64 q) { return ~0ull - ((0ull - q) % q); }
__host__ __device__ __forceinline__ bool uniform_from_word(u64 v, u64 q, u64 zone, u64 &sample) {
#ifdef __CUDA_ARCH__
  sample = __umul64hi(v, q);
#else
  sample = (u64)(((unsigned __int128)v * q) >> 64);
#endif
  return v * q <= zone;
}

// oa += x ka + y kc, ob += x kb + y kd (mod Q), kept below 2Q; the key rows
// are in the device layout (register pair -> one 16-byte word) and, with the
// blind rotation's folded reduction (MAC_FOLD_N2048), scaled by N^{-1} only:
// each 128-bit sum is folded with 2^54 = 77823 and the running sum brought
// back below 2Q by reduce_n2048.  Otherwise Montgomery REDC, keys with 2^64.
__device__ __forceinline__ void ni_mac(u64 (&oa)[8], u64 (&ob)[8], const u64 (&x)[8], const u64 (&y)[8],
                                       const u64 *ka, const u64 *kb, const u64 *kc, const u64 *kd, bool two,
                                       const RingConsts &rc) {
  const int j = threadIdx.x;
  const u64 q = rc.q, qi = rc.qinv_neg, q2 = rc.q << 1;
#pragma unroll
  for (int rr = 0; rr < 4; rr++) {
    const int di = dev_index<NI_LOGN>(j, 2 * rr);
    u64 a[2], b[2], c[2] = {0, 0}, d[2] = {0, 0};
    ld_key2(ka + di, a[0], a[1]);
    ld_key2(kb + di, b[0], b[1]);
    if (two) {
      ld_key2(kc + di, c[0], c[1]);
      ld_key2(kd + di, d[0], d[1]);
    }
#pragma unroll
    for (int e = 0; e < 2; e++) {
      const int r = 2 * rr + e;
      u64 hi, lo, hi2, lo2;
      if constexpr (MAC_FOLD_N2048) {  // x, y < 150 Q (lazy forward outputs), keys < Q
        if (two) {
          sum2_128(x[r], a[e], y[r], c[e], hi, lo);
          sum2_128(x[r], b[e], y[r], d[e], hi2, lo2);
        } else {
          mul128_narrow(x[r], a[e], hi, lo);
          mul128_narrow(x[r], b[e], hi2, lo2);
        }
        oa[r] = reduce_n2048(oa[r] + fold_n2048(hi, lo));
        ob[r] = reduce_n2048(ob[r] + fold_n2048(hi2, lo2));
      } else {
        mul128(x[r], a[e], hi, lo);
        mul128(x[r], b[e], hi2, lo2);
        if (two) {
          mac128(y[r], c[e], hi, lo);
          mac128(y[r], d[e], hi2, lo2);
        }
        const u64 va = oa[r] + redc(hi, lo, q, qi), vb = ob[r] + redc(hi2, lo2, q, qi);
        oa[r] = va >= q2 ? va - q2 : va;
        ob[r] = vb >= q2 ? vb - q2 : vb;
      }
    }
  }
}

}  // namespace ni
}  // namespace pz
