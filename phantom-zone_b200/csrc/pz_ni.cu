// pz_ni.cu -- the non-interactive input path on the device: the server side
// of a NonInteractiveBatchedFheBools (ni_mp_api.rs:182-196).
//
//   unseed       a-parts of a batch of seeded RLWEs regenerated from the
//                client's ChaCha8 seed (ni_mp_api.rs:248-280) by the seeded
//                uniform fill below.
//   seeded fill  RandomFillUniformInModulus over one ChaCha8 stream
//                (random.rs:93-110): the keystream is produced
//                block-parallel, each 64-bit word passes the uniform-in-[0, q)
//                acceptance test of rand's UniformInt (widening multiply,
//                rejection zone), and an exclusive scan over the accepted
//                words places sample k at its row-major destination --
//                exactly the order of the sequential stream, rejections
//                included.  Also used to expand seeded server keys.
//   key switch   rlwe_key_switch (runtime.rs:1001-1063) from the user's RLWE
//                secret u_j to the ideal secret s: the 50 one-bit signed
//                digits of -A are transformed two at a time and accumulated
//                against the user's ui_to_s key rows (N^{-1} folded in;
//                sums folded with 2^54 = 77823, see ni_mac), then one
//                inverse transform of both outputs and B' += B.
//   extract      BatchedFheBools::extract (ni_mp_api.rs:217-236): bool i is
//                sample_extract (pbs.rs:423-449) at coefficient i % N of
//                RLWE i / N.
#include <algorithm>
#include <cstring>
#include <vector>

#include "pz_internal.h"
#include "pz_ni.cuh"

using pz::u32;
using pz::u64;

namespace {

using pz::ni::ChaChaKey;
using pz::ni::chacha8_block;
using pz::ni::uniform_from_word;
using pz::ni::ni_mac;
using pz::ni::NI_LOGN;
using pz::ni::NI_T;
constexpr u64 UNSEED_MARGIN = 1024;  // keystream words generated beyond the samples needed

// Block b of stream blockIdx.y: the 8 u64 words 8b..8b+7 of the stream (two
// u32 words each, low first), their samples (high half of v * q) and
// acceptance (low half <= zone).
constexpr int FILL_STREAMS = 64;  // streams per launch (their keys travel as a kernel parameter)
struct ChaChaKeys {
  ChaChaKey k[FILL_STREAMS];
};

__global__ void unseed_candidates_kernel(const __grid_constant__ ChaChaKeys keys, u64 nblocks, u64 q, u64 zone,
                                         u64 *samples, unsigned char *accept, u32 *cnt) {
  const ChaChaKey key = keys.k[blockIdx.y];
  const u64 base = blockIdx.y * nblocks;
  for (u64 b = blockIdx.x * (u64)blockDim.x + threadIdx.x; b < nblocks; b += (u64)gridDim.x * blockDim.x) {
    u32 w[16];
    chacha8_block(key, b, w);
    unsigned m = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const u64 v = (u64)w[2 * i] | ((u64)w[2 * i + 1] << 32);
      u64 sample;
      if (uniform_from_word(v, q, zone, sample)) m |= 1u << i;
      samples[8 * (base + b) + i] = sample;
    }
    accept[base + b] = (unsigned char)m;
    cnt[base + b] = __popc(m);
  }
}

// Exclusive scan of stream blockIdx.x's cnt[0, n) into its off (one CTA per
// stream); off[n] and totals[stream] = the stream's accepted total.
__global__ void __launch_bounds__(1024) unseed_scan_kernel(const u32 *cnt, u64 n, u64 *off, u64 *totals) {
  __shared__ u64 part[1024];
  cnt += blockIdx.x * n;
  off += blockIdx.x * (n + 1);
  const u64 per = (n + blockDim.x - 1) / blockDim.x;
  const u64 b0 = min(n, threadIdx.x * per), b1 = min(n, b0 + per);
  u64 local = 0;
  for (u64 b = b0; b < b1; b++) local += cnt[b];
  part[threadIdx.x] = local;
  __syncthreads();
  for (unsigned o = 1; o < blockDim.x; o <<= 1) {  // inclusive Hillis-Steele scan
    const u64 v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  u64 run = part[threadIdx.x] - local;
  for (u64 b = b0; b < b1; b++) {
    off[b] = run;
    run += cnt[b];
  }
  if (threadIdx.x == blockDim.x - 1) {
    off[n] = part[threadIdx.x];
    totals[blockIdx.x] = part[threadIdx.x];
  }
}

// Accepted sample k (k < total) of stream blockIdx.y ->
// dst[y * stream_stride + (k / row_len) * row_stride + row_off + k % row_len].
template <typename T>
__global__ void seeded_place_kernel(const u64 *samples, const unsigned char *accept, const u64 *off, u64 nblocks,
                                    u64 total, u64 row_len, u64 row_stride, u64 row_off, T *dst, u64 stream_stride) {
  const u64 y = blockIdx.y;
  samples += y * 8 * nblocks;
  accept += y * nblocks;
  off += y * (nblocks + 1);
  dst += y * stream_stride;
  for (u64 b = blockIdx.x * (u64)blockDim.x + threadIdx.x; b < nblocks; b += (u64)gridDim.x * blockDim.x) {
    const unsigned m = accept[b];
    u64 pos = off[b];
#pragma unroll
    for (int i = 0; i < 8; i++) {
      if ((m >> i) & 1u) {
        if (pos < total) dst[(pos / row_len) * row_stride + row_off + pos % row_len] = (T)samples[8 * b + i];
        pos++;
      }
    }
  }
}

// One RLWE per CTA: rlwe_key_switch of in[c] with the user's key rows.
__global__ void __launch_bounds__(NI_T, 2)
    ni_key_switch_kernel(pz::RingConsts rc, pz::Decomp dp, u32 d, const u64 *ksk, const u64 *in, u64 *out,
                         size_t count) {
  constexpr int N = 1 << NI_LOGN;
  extern __shared__ u64 sm[];  // 2N words: exchange buffer of the two-polynomial transforms
  const int j = threadIdx.x;
  const u64 q = rc.q;
  for (size_t c = blockIdx.x; c < count; c += gridDim.x) {
    const u64 *p = in + c * 2 * N;
    u64 st[8], oa[8], ob[8];
#pragma unroll
    for (int r = 0; r < 8; r++) {
      st[r] = pz::decomp_init(q - p[pz::pos_coef<NI_LOGN>(j, r)], dp);  // elwise_neg_mut, then decompose
      oa[r] = 0;
      ob[r] = 0;
    }
#pragma unroll 1
    for (u32 jd = 0; jd < d; jd += 2) {
      const bool two = jd + 1 < d;  // uniform
      u64 x[8], y[8];
#pragma unroll
      for (int r = 0; r < 8; r++) {
        x[r] = pz::decomp_next(st[r], dp);
        y[r] = two ? pz::decomp_next(st[r], dp) : 0;
      }
      if (two) pz::ntt_fwd<NI_LOGN, true>(x, y, sm, rc);
      else pz::ntt_fwd<NI_LOGN, false>(x, x, sm, rc);
      ni_mac(oa, ob, x, y, ksk + (size_t)jd * N, ksk + (size_t)(d + jd) * N, ksk + (size_t)(jd + 1) * N,
             ksk + (size_t)(d + jd + 1) * N, two, rc);
    }
    pz::ntt_inv<NI_LOGN, true>(oa, ob, sm, rc);
    u64 *o = out + c * 2 * N;
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const int pc = pz::pos_coef<NI_LOGN>(j, r);
      o[pc] = pz::reduce2(oa[r], q);
      o[N + pc] = pz::add_mod(pz::reduce2(ob[r], q), p[N + pc], q);  // elwise_add_mut(B', B)
    }
    __syncthreads();
  }
}

// Small batches: the digits of one RLWE split over gridDim.y CTAs.  CTA
// (c, s) runs the decomposition through digit pair `pend` of its share (the
// signed digits carry from low to high, so every share walks the digits
// before its own) and transforms and accumulates only pairs [pbeg, pend);
// its partial (A, B) sums, evaluation domain in [0, 2q), go to
// part[c][s][2][N] in the thread-major order ni_ks_finish_kernel reads.
__global__ void __launch_bounds__(NI_T, 2)
    ni_ks_partial_kernel(pz::RingConsts rc, pz::Decomp dp, u32 d, const u64 *ksk, const u64 *in, u64 *part,
                         size_t count) {
  constexpr int N = 1 << NI_LOGN;
  extern __shared__ u64 sm[];
  const int j = threadIdx.x;
  const u64 q = rc.q;
  const u32 pairs = (d + 1) / 2, share = (pairs + gridDim.y - 1) / gridDim.y;
  const u32 pbeg = blockIdx.y * share, pend = min(pairs, pbeg + share);
  for (size_t c = blockIdx.x; c < count; c += gridDim.x) {
    const u64 *p = in + c * 2 * N;
    u64 st[8], oa[8], ob[8];
#pragma unroll
    for (int r = 0; r < 8; r++) {
      st[r] = pz::decomp_init(q - p[pz::pos_coef<NI_LOGN>(j, r)], dp);  // elwise_neg_mut, then decompose
      oa[r] = 0;
      ob[r] = 0;
    }
#pragma unroll 1
    for (u32 pi = 0; pi < pbeg; pi++) {  // digits of the earlier shares: carries only
#pragma unroll
      for (int r = 0; r < 8; r++) {
        pz::decomp_next(st[r], dp);
        if (2 * pi + 1 < d) pz::decomp_next(st[r], dp);
      }
    }
#pragma unroll 1
    for (u32 pi = pbeg; pi < pend; pi++) {
      const u32 jd = 2 * pi;
      const bool two = jd + 1 < d;  // uniform
      u64 x[8], y[8];
#pragma unroll
      for (int r = 0; r < 8; r++) {
        x[r] = pz::decomp_next(st[r], dp);
        y[r] = two ? pz::decomp_next(st[r], dp) : 0;
      }
      if (two) pz::ntt_fwd<NI_LOGN, true>(x, y, sm, rc);
      else pz::ntt_fwd<NI_LOGN, false>(x, x, sm, rc);
      ni_mac(oa, ob, x, y, ksk + (size_t)jd * N, ksk + (size_t)(d + jd) * N, ksk + (size_t)(jd + 1) * N,
             ksk + (size_t)(d + jd + 1) * N, two, rc);
    }
    u64 *o = part + (c * gridDim.y + blockIdx.y) * 2 * N;
#pragma unroll
    for (int r = 0; r < 8; r++) {
      o[r * NI_T + j] = oa[r];
      o[N + r * NI_T + j] = ob[r];
    }
    __syncthreads();
  }
}

// Sum of the `shares` partials (each < 2q, so the sum is reduced with the
// special form of Q once), one inverse transform of both outputs, B' += B.
__global__ void __launch_bounds__(NI_T, 2)
    ni_ks_finish_kernel(pz::RingConsts rc, const u64 *part, u32 shares, const u64 *in, u64 *out, size_t count) {
  constexpr int N = 1 << NI_LOGN;
  extern __shared__ u64 sm[];
  const int j = threadIdx.x;
  const u64 q = rc.q;
  for (size_t c = blockIdx.x; c < count; c += gridDim.x) {
    u64 oa[8], ob[8];
#pragma unroll
    for (int r = 0; r < 8; r++) oa[r] = ob[r] = 0;
    for (u32 sh = 0; sh < shares; sh++) {
      const u64 *src = part + (c * shares + sh) * 2 * N;
#pragma unroll
      for (int r = 0; r < 8; r++) {
        oa[r] += src[r * NI_T + j];
        ob[r] += src[N + r * NI_T + j];
      }
    }
#pragma unroll
    for (int r = 0; r < 8; r++) {
      oa[r] = pz::reduce_n2048(oa[r]);
      ob[r] = pz::reduce_n2048(ob[r]);
    }
    pz::ntt_inv<NI_LOGN, true>(oa, ob, sm, rc);
    const u64 *p = in + c * 2 * N;
    u64 *o = out + c * 2 * N;
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const int pc = pz::pos_coef<NI_LOGN>(j, r);
      o[pc] = pz::reduce2(oa[r], q);
      o[N + pc] = pz::add_mod(pz::reduce2(ob[r], q), p[N + pc], q);  // elwise_add_mut(B', B)
    }
    __syncthreads();
  }
}

// out[c] = sample_extract(rlwe[idx[c] / N], idx[c] % N); an index past the
// batch leaves out[c] unchanged.
__global__ void extract_kernel(const u64 *rlwe, size_t rlwe_count, const u32 *idx, u64 *out, size_t count, u32 N,
                               u64 q) {
  for (size_t c = blockIdx.x; c < count; c += gridDim.x) {
    const u32 i = idx[c];
    const size_t ct = i / N, k = i % N;
    if (ct >= rlwe_count) continue;
    const u64 *a = rlwe + ct * 2 * N, *b = a + N;
    u64 *o = out + c * (size_t)(N + 1);
    for (u32 t = threadIdx.x; t <= N; t += blockDim.x) {
      if (t == 0) {
        o[0] = b[k];
      } else {
        const size_t ii = t - 1;
        o[t] = ii <= k ? a[k - ii] : q - a[N + k - ii];  // neg = q - x (modulus_u64.rs:147-149)
      }
    }
  }
}

pz_status ni_check(pz_ctx *c) {
  if (!c) return PZ_ERR_INVALID_ARGUMENT;
  if (c->P.variant != 2 || c->P.ni_ks_d == 0)
    return pz::fail(c, PZ_ERR_NOT_SUPPORTED, "not a non-interactive parameter set");
  if (c->logn != NI_LOGN) return pz::fail(c, PZ_ERR_NOT_SUPPORTED, "ring dimension other than 2048");
  return PZ_OK;
}

int grid_of(size_t n, int cap) { return (int)std::min<size_t>(std::max<size_t>(n, 1), (size_t)cap); }

// `streams` independent ChaCha8 streams (seeds[i]), `total` samples each,
// stream i written from dst + i * stream_stride.  Synchronous.
template <typename T>
pz_status seeded_fill(pz_ctx *c, const uint8_t (*seeds)[32], size_t streams, u64 q, u64 total, u64 row_len,
                      u64 row_stride, u64 row_off, T *dst, u64 stream_stride, cudaStream_t st) {
  if (total == 0 || streams == 0) return PZ_OK;
  const u64 nblocks = (total + UNSEED_MARGIN + 7) / 8;
  const size_t group = std::min<size_t>(streams, FILL_STREAMS);
  const u64 zone = pz::ni::uniform_zone(q);  // rand 0.8 UniformInt::new_inclusive(0, q - 1)
  // one scratch allocation: samples | off | totals | cnt | accept
  const size_t b_samples = group * nblocks * 64, b_off = group * (nblocks + 1) * 8, b_tot = group * 8,
               b_cnt = group * nblocks * 4, b_acc = group * nblocks;
  unsigned char *scratch = nullptr;
  cudaError_t e = cudaMallocAsync(&scratch, b_samples + b_off + b_tot + b_cnt + b_acc, st);
  u64 *samples = (u64 *)scratch, *off = (u64 *)(scratch + b_samples), *tot = (u64 *)(scratch + b_samples + b_off);
  u32 *cnt = (u32 *)(scratch + b_samples + b_off + b_tot);
  unsigned char *acc = scratch + b_samples + b_off + b_tot + b_cnt;
  std::vector<u64> accepted(streams, 0);
  for (size_t s0 = 0; s0 < streams && e == cudaSuccess; s0 += group) {
    const size_t m = std::min(group, streams - s0);
    ChaChaKeys keys{};
    for (size_t i = 0; i < m; i++) keys.k[i] = pz::ni::chacha_key(seeds[s0 + i]);
    const dim3 grid((unsigned)grid_of((nblocks + 255) / 256, 65535), (unsigned)m);
    unseed_candidates_kernel<<<grid, 256, 0, st>>>(keys, nblocks, q, zone, samples, acc, cnt);
    e = cudaGetLastError();
    if (e == cudaSuccess) {
      unseed_scan_kernel<<<(unsigned)m, 1024, 0, st>>>(cnt, nblocks, off, tot);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
      seeded_place_kernel<T><<<grid, 256, 0, st>>>(samples, acc, off, nblocks, total, row_len, row_stride, row_off,
                                                   dst + s0 * stream_stride, stream_stride);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&accepted[s0], tot, m * 8, cudaMemcpyDeviceToHost, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFreeAsync(scratch, st);
  if (e != cudaSuccess) return pz::cuda_fail(c, "seeded uniform fill", e);
  for (size_t i = 0; i < streams; i++)
    if (accepted[i] < total)  // more rejections than the margin covers (probability ~0)
      return pz::fail(c, PZ_ERR_NOT_SUPPORTED, "seeded fill: rejection margin exhausted");
  return PZ_OK;
}

}  // namespace

namespace pz {
pz_status seeded_fill_u64(pz_ctx *c, const uint8_t seed[32], u64 q, u64 total, u64 row_len, u64 row_stride,
                          u64 row_off, u64 *dst, cudaStream_t st) {
  return seeded_fill<u64>(c, (const uint8_t(*)[32])seed, 1, q, total, row_len, row_stride, row_off, dst, 0, st);
}
pz_status seeded_fill_u32(pz_ctx *c, const uint8_t seed[32], u64 q, u64 total, u64 row_len, u64 row_stride,
                          u64 row_off, u32 *dst, cudaStream_t st) {
  return seeded_fill<u32>(c, (const uint8_t(*)[32])seed, 1, q, total, row_len, row_stride, row_off, dst, 0, st);
}
pz_status seeded_fill_batch_u64(pz_ctx *c, const uint8_t (*seeds)[32], size_t streams, u64 q, u64 total, u64 *dst,
                                u64 stream_stride, cudaStream_t st) {
  return seeded_fill<u64>(c, seeds, streams, q, total, total, total, 0, dst, stream_stride, st);
}
}  // namespace pz

extern "C" {

pz_status pz_chacha_block(const uint32_t state[16], int rounds, uint32_t out[16]) {
  if (!state || !out) return PZ_ERR_INVALID_ARGUMENT;
  u32 s[16], o[16];
  for (int i = 0; i < 16; i++) s[i] = state[i];
  switch (rounds) {
    case 8: pz::ni::chacha_core<8>(s, o); break;
    case 12: pz::ni::chacha_core<12>(s, o); break;
    case 20: pz::ni::chacha_core<20>(s, o); break;
    default: return PZ_ERR_INVALID_ARGUMENT;
  }
  for (int i = 0; i < 16; i++) out[i] = o[i];
  return PZ_OK;
}

pz_status pz_uniform_mod_word(uint64_t q, uint64_t word, uint64_t *sample, int *accepted) {
  if (q == 0 || !sample || !accepted) return PZ_ERR_INVALID_ARGUMENT;
  u64 v = 0;
  *accepted = pz::ni::uniform_from_word(word, q, pz::ni::uniform_zone(q), v) ? 1 : 0;
  *sample = v;
  return PZ_OK;
}

pz_status pz_ni_ksk_upload(pz_ctx *c, const uint64_t *ksk, pz_ni_ksk **out) {
  pz_status s = ni_check(c);
  if (s != PZ_OK) return s;
  if (!ksk || !out) return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "pz_ni_ksk_upload: NULL argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lock(c->mu);
  PZ_CK(c, cudaSetDevice(c->device));
  const size_t N = c->P.rlwe_n, polys = 2 * (size_t)c->P.ni_ks_d;
  pz_ni_ksk *k = new pz_ni_ksk();
  k->ctx = c;
  k->d = c->P.ni_ks_d;
  k->bytes = polys * N * 8;
  u64 *stage = nullptr;
  cudaError_t e = cudaMalloc(&k->d_ksk, k->bytes);
  if (e == cudaSuccess) e = cudaMalloc(&stage, k->bytes);
  if (e == cudaSuccess) e = cudaMemcpyAsync(stage, ksk, k->bytes, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = pz::launch_key_convert((int)c->logn, stage, k->d_ksk, polys, c->rc, c->ni_conv_c, c->ni_conv_cs, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(stage);
  if (e != cudaSuccess) {
    cudaFree(k->d_ksk);
    delete k;
    return pz::cuda_fail(c, "pz_ni_ksk_upload", e);
  }
  *out = k;
  return PZ_OK;
}

pz_status pz_ni_ksk_upload_seeded(pz_ctx *c, const uint64_t *ksk_b, const uint8_t seed[32], pz_ni_ksk **out) {
  pz_status s = ni_check(c);
  if (s != PZ_OK) return s;
  if (!ksk_b || !seed || !out) return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "pz_ni_ksk_upload_seeded: NULL argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lock(c->mu);
  PZ_CK(c, cudaSetDevice(c->device));
  const size_t N = c->P.rlwe_n, d = c->P.ni_ks_d, polys = 2 * d;
  pz_ni_ksk *k = new pz_ni_ksk();
  k->ctx = c;
  k->d = (u32)d;
  k->bytes = polys * N * 8;
  u64 *stage = nullptr;
  cudaError_t e = cudaMalloc(&k->d_ksk, k->bytes);
  if (e == cudaSuccess) e = cudaMalloc(&stage, k->bytes);
  // keys.rs:965-1000: d A rows from the user's stream, then the B rows
  if (e == cudaSuccess) s = pz::seeded_fill_u64(c, seed, c->P.rlwe_q, (u64)d * N, d * N, 2 * d * N, 0, stage, c->stream);
  if (e == cudaSuccess && s == PZ_OK)
    e = cudaMemcpyAsync(stage + d * N, ksk_b, d * N * 8, cudaMemcpyDefault, c->stream);
  if (e == cudaSuccess && s == PZ_OK)
    e = pz::launch_key_convert((int)c->logn, stage, k->d_ksk, polys, c->rc, c->ni_conv_c, c->ni_conv_cs, c->stream);
  if (e == cudaSuccess && s == PZ_OK) e = cudaStreamSynchronize(c->stream);
  cudaFree(stage);
  if (e != cudaSuccess || s != PZ_OK) {
    cudaFree(k->d_ksk);
    delete k;
    return s != PZ_OK ? s : pz::cuda_fail(c, "pz_ni_ksk_upload_seeded", e);
  }
  *out = k;
  return PZ_OK;
}

void pz_ni_ksk_release(pz_ni_ksk *k) {
  if (!k) return;
  cudaSetDevice(k->ctx->device);
  cudaFree(k->d_ksk);
  delete k;
}

pz_status pz_ni_unseed_device(pz_ctx *c, const uint8_t seed[32], const uint64_t *d_b, uint64_t *d_rlwe, size_t count,
                              void *stream) {
  pz_status s = ni_check(c);
  if (s != PZ_OK) return s;
  if (!seed || (count && (!d_b || !d_rlwe))) return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "NULL argument");
  if (count == 0) return PZ_OK;
  PZ_CK(c, cudaSetDevice(c->device));
  cudaStream_t st = (cudaStream_t)stream;
  const u32 N = c->P.rlwe_n;
  // a-parts: sample k of the stream -> RLWE k / N, coefficient k % N; b-parts: row 1
  s = pz::seeded_fill_u64(c, seed, c->P.rlwe_q, (u64)count * N, N, 2 * N, 0, d_rlwe, st);
  if (s != PZ_OK) return s;
  PZ_CK(c, cudaMemcpy2DAsync(d_rlwe + N, 2 * N * 8, d_b, N * 8, N * 8, count, cudaMemcpyDeviceToDevice, st));
  return PZ_OK;
}

pz_status pz_ni_key_switch_device(pz_ctx *c, const pz_ni_ksk *k, const uint64_t *d_in, uint64_t *d_out, size_t count,
                                  void *stream) {
  pz_status s = ni_check(c);
  if (s != PZ_OK) return s;
  if (!k || k->ctx != c) return pz::fail(c, PZ_ERR_KEY_MISMATCH, "key-switching key does not belong to this context");
  if (count && (!d_in || !d_out)) return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "NULL argument");
  if (count == 0) return PZ_OK;
  PZ_CK(c, cudaSetDevice(c->device));
  const pz::Decomp dp = pz::decomposer(c->P.rlwe_q, c->P.ni_ks_logb, c->P.ni_ks_d);
  const size_t smem = 2 * (size_t)c->P.rlwe_n * 8;
  cudaStream_t st = (cudaStream_t)stream;
  // fewer RLWEs than two per SM: split each one's digit pairs over CTAs
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
  const u32 pairs = (k->d + 1) / 2;
  const size_t shares = std::min<size_t>(std::min<size_t>(8, pairs), (2 * (size_t)sms + count - 1) / count);
  if (shares <= 1) {
    ni_key_switch_kernel<<<grid_of(count, 65535), NI_T, smem, st>>>(c->rc, dp, k->d, k->d_ksk, d_in, d_out, count);
    PZ_CK(c, cudaGetLastError());
    return PZ_OK;
  }
  u64 *part = nullptr;
  PZ_CK(c, cudaMallocAsync(&part, count * shares * 2 * c->P.rlwe_n * 8, st));
  ni_ks_partial_kernel<<<dim3((unsigned)count, (unsigned)shares), NI_T, smem, st>>>(c->rc, dp, k->d, k->d_ksk, d_in,
                                                                                   part, count);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    ni_ks_finish_kernel<<<grid_of(count, 65535), NI_T, smem, st>>>(c->rc, part, (u32)shares, d_in, d_out, count);
    e = cudaGetLastError();
  }
  cudaFreeAsync(part, st);
  if (e != cudaSuccess) return pz::cuda_fail(c, "pz_ni_key_switch_device", e);
  return PZ_OK;
}

pz_status pz_sample_extract_device(pz_ctx *c, const uint64_t *d_rlwe, size_t rlwe_count, const uint32_t *d_index,
                                   uint64_t *d_lwe, size_t count, void *stream) {
  if (!c) return PZ_ERR_INVALID_ARGUMENT;
  if (count && (!d_rlwe || !d_index || !d_lwe)) return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "NULL argument");
  if (count == 0) return PZ_OK;
  PZ_CK(c, cudaSetDevice(c->device));
  extract_kernel<<<grid_of(count, 65535), 256, 0, (cudaStream_t)stream>>>(d_rlwe, rlwe_count, d_index, d_lwe, count,
                                                                          c->P.rlwe_n, c->P.rlwe_q);
  PZ_CK(c, cudaGetLastError());
  return PZ_OK;
}

pz_status pz_ni_ingest(pz_ctx *c, const pz_ni_ksk *k, const uint8_t seed[32], const uint64_t *b, size_t rlwe_count,
                       uint64_t *lwe_out, size_t nbools) {
  pz_status s = ni_check(c);
  if (s != PZ_OK) return s;
  if (!k || k->ctx != c) return pz::fail(c, PZ_ERR_KEY_MISMATCH, "key-switching key does not belong to this context");
  if (!seed || (rlwe_count && !b) || (nbools && !lwe_out))
    return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "NULL argument");
  const size_t N = c->P.rlwe_n;
  if (nbools > rlwe_count * N) return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "more bools than the batch holds");
  if (rlwe_count == 0) return PZ_OK;
  std::lock_guard<std::mutex> lock(c->mu);
  PZ_CK(c, cudaSetDevice(c->device));
  cudaStream_t st = c->stream;
  u64 *d_b = nullptr, *d_r = nullptr, *d_k = nullptr, *d_l = nullptr;
  u32 *d_i = nullptr;
  std::vector<u32> idx(nbools);
  for (size_t i = 0; i < nbools; i++) idx[i] = (u32)i;
  cudaError_t e = cudaMallocAsync(&d_b, rlwe_count * N * 8, st);
  if (e == cudaSuccess) e = cudaMallocAsync(&d_r, rlwe_count * 2 * N * 8, st);
  if (e == cudaSuccess) e = cudaMallocAsync(&d_k, rlwe_count * 2 * N * 8, st);
  if (e == cudaSuccess) e = cudaMallocAsync(&d_l, std::max<size_t>(nbools, 1) * (N + 1) * 8, st);
  if (e == cudaSuccess) e = cudaMallocAsync(&d_i, std::max<size_t>(nbools, 1) * 4, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_b, b, rlwe_count * N * 8, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && nbools) e = cudaMemcpyAsync(d_i, idx.data(), nbools * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) {
    s = pz_ni_unseed_device(c, seed, d_b, d_r, rlwe_count, st);
    if (s == PZ_OK) s = pz_ni_key_switch_device(c, k, d_r, d_k, rlwe_count, st);
    if (s == PZ_OK) s = pz_sample_extract_device(c, d_k, rlwe_count, d_i, d_l, nbools, st);
    if (s == PZ_OK && nbools) e = cudaMemcpyAsync(lwe_out, d_l, nbools * (N + 1) * 8, cudaMemcpyDeviceToHost, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFreeAsync(d_b, st);
  cudaFreeAsync(d_r, st);
  cudaFreeAsync(d_k, st);
  cudaFreeAsync(d_l, st);
  cudaFreeAsync(d_i, st);
  cudaStreamSynchronize(st);
  if (s != PZ_OK) return s;
  if (e != cudaSuccess) return pz::cuda_fail(c, "pz_ni_ingest", e);
  return PZ_OK;
}

}  // extern "C"
