// pz_ni_aggregate.cu -- non-interactive server-key aggregation on the device:
// aggregate_non_interactive_multi_party_server_key_shares (bool/evaluator.rs:
// 1222-1622).
//
//   ui_to_s keys   per user j: own B rows + every other user's zero
//                  encryptions for j (evaluator.rs:1269-1294); A rows from
//                  the user's CRS stream; the device key form of each is
//                  built once and read by every LWE index.
//   auto, LWE KSK  plain sums of the users' B rows (:1563-1605).
//   RGSWs          per LWE index l, in chunks of indices: the a_{l,i} rows
//                  from the index's CRS stream (all chunk streams in one
//                  batched seeded fill), the zero encryptions summed over
//                  users; each of these d_a + d_b values is decomposed (50
//                  one-bit digits) and transformed ONCE into HBM (the digit
//                  kernel), then every (value, user) pair is one CTA of the
//                  multiply-accumulate kernel: 50-digit MAC against that
//                  user's key, one inverse transform of both outputs, the
//                  user's NI RGSW row added (produce_rgsw_ciphertext_from_
//                  ni_rgsw, :480-608) and the row stored straight into its
//                  place in the leader's RGSW (rlwe x rgsw shape) or in the
//                  other users' RGSWs (rgsw x rgsw shape).  Then the batched
//                  RGSW x RGSW products (pz_aggregate_rgsw_device) multiply
//                  the leader's RGSW by the other users' in increasing id.
//
// Bytes per LWE index (NI_8P: d_a 20, d_b 18, 8 users): digits 38 x 50 x 16 KiB
// = 31 MB written once and read by 8 users (L2-resident when the users of one
// value run together, the grid's fastest index); key rows 1.6 MB per user,
// shared by every index.
#include <algorithm>
#include <cstring>
#include <vector>

#include "pz_internal.h"
#include "pz_ni.cuh"

using pz::u32;
using pz::u64;
using pz::ni::NI_LOGN;
using pz::ni::NI_T;

namespace {

struct NiUser {            // device view of one user's RGSW inputs
  const u64 *ksk;          // [2 d][N] device key form (A rows, then B rows)
  const u64 *self_leader;  // [segment][max_l][N]
  const u64 *not_leader;   // [n - segment][max_d][N]
  const u64 *zero_encs;    // [n][ra][N]
  u32 seg_b, seg_e;        // multi_party_user_id_lwe_segment
};

struct NiShape {
  u32 users, per_user, ra, rb, max_d, max_l, d;
};

// out[i] = sum_t src[t][i] mod q (elwise_add_mut over canonical rows)
__global__ void sum_mod_kernel(const u64 *const *src, u32 k, size_t len, u64 q, u64 *out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < len; i += (size_t)gridDim.x * blockDim.x) {
    u64 acc = 0;
    for (u32 t = 0; t < k; t++) {
      const u64 v = acc + src[t][i];
      acc = v >= q ? v - q : v;
    }
    out[i] = acc;
  }
}

// Values to key-switch for LWE indices idx0 .. idx0 + cnt - 1, [cnt][ra + rb][N]:
// row v < ra: sum over users of zero-enc row v (aggregated a_{l,v} s + e);
// row ra + r: q - a row (max_d - rb + r) of the index's stream (elwise_neg_mut,
// 0 -> q as in the reference).
__global__ void ni_values_kernel(const NiUser *users, NiShape sh, const u64 *arows, u32 idx0, u32 cnt, u64 q,
                                 u64 *vals) {
  constexpr u32 N = 1u << NI_LOGN;
  const u32 R = sh.ra + sh.rb;
  const size_t total = (size_t)cnt * R * N;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const u32 k = (u32)(i % N), v = (u32)((i / N) % R), c = (u32)(i / ((size_t)N * R));
    u64 x;
    if (v < sh.ra) {
      x = 0;
      for (u32 u = 0; u < sh.users; u++) {
        const u64 s = x + users[u].zero_encs[((size_t)(idx0 + c) * sh.ra + v) * N + k];
        x = s >= q ? s - q : s;
      }
    } else {
      x = q - arows[((size_t)c * sh.max_d + sh.max_d - sh.rb + (v - sh.ra)) * N + k];
    }
    vals[i] = x;
  }
}

// One value row per CTA: its d one-bit digits, transformed two at a time,
// stored [row][digit][N] in the thread-major order the MAC kernel reads back.
__global__ void __launch_bounds__(NI_T, 2)
    ni_digits_kernel(pz::RingConsts rc, pz::Decomp dp, u32 d, const u64 *vals, u64 *dig, size_t rows) {
  constexpr int N = 1 << NI_LOGN;
  extern __shared__ u64 sm[];  // 2N words: exchange buffer of the two-polynomial transforms
  const int j = threadIdx.x;
  for (size_t row = blockIdx.x; row < rows; row += gridDim.x) {
    const u64 *p = vals + row * N;
    u64 st[8];
#pragma unroll
    for (int r = 0; r < 8; r++) st[r] = pz::decomp_init(p[pz::pos_coef<NI_LOGN>(j, r)], dp);
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
      u64 *o = dig + (row * d + jd) * N;
#pragma unroll
      for (int r = 0; r < 8; r++) {
        o[r * NI_T + j] = x[r];
        if (two) o[N + r * NI_T + j] = y[r];
      }
    }
    __syncthreads();
  }
}

// One (index, value, user) item per CTA, user fastest.  The leader of an
// index only needs the last zero-enc value (ra - 1) and the last -a value
// (R - 1): its RGSW is in the rlwe x rgsw shape (d_a = d_b = 1), rows
// [A(-sm), B(-sm), A(m), B(m)] in leader_out[c].  Every other user t (in
// increasing id, the leader skipped) gets all R values: rows v / ra + v of
// others[t][c] for zero-enc values, 2 ra + r / 2 ra + rb + r for -a values.
__global__ void __launch_bounds__(NI_T, 2)
    ni_agg_mac_kernel(pz::RingConsts rc, NiShape sh, const u64 *dig, const NiUser *users, u32 idx0, u32 cnt,
                      u64 *leader_out, u64 *others) {
  constexpr int N = 1 << NI_LOGN;
  extern __shared__ u64 sm[];
  const int j = threadIdx.x;
  const u64 q = rc.q;
  const u32 R = sh.ra + sh.rb, rows1 = 2 * R, d = sh.d;
  const size_t items = (size_t)cnt * R * sh.users;
  for (size_t it = blockIdx.x; it < items; it += gridDim.x) {
    const u32 u = (u32)(it % sh.users), v = (u32)((it / sh.users) % R), c = (u32)(it / ((size_t)sh.users * R));
    const u32 idx = idx0 + c, L = idx / sh.per_user;
    const bool lead = u == L;
    if (lead && v != sh.ra - 1 && v != R - 1) continue;  // uniform over the CTA
    const NiUser U = users[u];
    const u64 *kk = U.ksk;
    const u64 *dv = dig + ((size_t)c * R + v) * d * N;
    u64 oa[8], ob[8];
#pragma unroll
    for (int r = 0; r < 8; r++) oa[r] = ob[r] = 0;
#pragma unroll 1
    for (u32 jd = 0; jd < d; jd += 2) {
      const bool two = jd + 1 < d;
      u64 x[8], y[8];
#pragma unroll
      for (int r = 0; r < 8; r++) {
        x[r] = dv[(size_t)jd * N + r * NI_T + j];
        y[r] = two ? dv[(size_t)(jd + 1) * N + r * NI_T + j] : 0;
      }
      pz::ni::ni_mac(oa, ob, x, y, kk + (size_t)jd * N, kk + (size_t)(d + jd) * N, kk + (size_t)(jd + 1) * N,
                     kk + (size_t)(d + jd + 1) * N, two, rc);
    }
    pz::ntt_inv<NI_LOGN, true>(oa, ob, sm, rc);
    const bool to_a = v < sh.ra;  // -sm rows add the NI row to A, m rows to B
    const u64 *ct;
    u64 *oA, *oB;
    if (lead) {
      ct = U.self_leader + ((size_t)(idx - U.seg_b) * sh.max_l + (sh.max_l - 1)) * N;
      oA = leader_out + ((size_t)c * 4 + (to_a ? 0 : 2)) * N;
      oB = oA + N;
    } else {
      const u32 pos = idx < U.seg_b ? idx : idx - (U.seg_e - U.seg_b);
      const u32 ctrow = to_a ? sh.max_d - sh.ra + v : sh.max_d - sh.rb + (v - sh.ra);
      ct = U.not_leader + ((size_t)pos * sh.max_d + ctrow) * N;
      const u32 t = u < L ? u : u - 1;
      u64 *base = others + ((size_t)t * cnt + c) * rows1 * N;
      oA = base + (size_t)(to_a ? v : 2 * sh.ra + (v - sh.ra)) * N;
      oB = base + (size_t)(to_a ? sh.ra + v : 2 * sh.ra + sh.rb + (v - sh.ra)) * N;
    }
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const int pc = pz::pos_coef<NI_LOGN>(j, r);
      u64 a = pz::reduce2(oa[r], q), b = pz::reduce2(ob[r], q);
      if (to_a) a = pz::add_mod(a, ct[pc], q);
      else b = pz::add_mod(b, ct[pc], q);
      oA[pc] = a;
      oB[pc] = b;
    }
    __syncthreads();
  }
}

int grid_cap(size_t n, int cap) { return (int)std::min<size_t>(std::max<size_t>(n, 1), (size_t)cap); }

void puncture(const uint8_t seed[32], size_t times, uint8_t out[32]) { pz::crs_puncture(seed, times, out); }

void segment(size_t user, size_t users, size_t n, u32 *b, u32 *e) {  // evaluator.rs:613-626
  const size_t per = (n + users - 1) / users;
  const size_t s = std::min(per * user, n), t = std::min(per * (user + 1), n);
  *b = (u32)s;
  *e = (u32)std::max(s, t);
}

}  // namespace

namespace pz {
// puncture_p_rng (utils.rs:219-228) with RandomFill<[u8; 32]> (random.rs:
// 162-175): the `times`-th 32-byte fill of ChaCha8(seed); each byte is the
// low byte of one u32 word, so fill t is words 32 (t - 1) .. 32 t - 1, i.e.
// blocks 2 (t - 1) and 2 (t - 1) + 1.
void crs_puncture(const uint8_t seed[32], size_t times, uint8_t out[32]) {
  const ni::ChaChaKey key = ni::chacha_key(seed);
  for (int h = 0; h < 2; h++) {
    u32 w[16];
    ni::chacha8_block(key, 2 * (u64)(times - 1) + h, w);
    for (int i = 0; i < 16; i++) out[16 * h + i] = (uint8_t)w[i];
  }
}
cudaError_t launch_sum_mod(const u64 *const *d_src, u32 k, size_t len, u64 q, u64 *out, cudaStream_t st) {
  if (len == 0) return cudaSuccess;
  sum_mod_kernel<<<grid_cap(len / 256, 1184), 256, 0, st>>>(d_src, k, len, q, out);
  return cudaGetLastError();
}
}  // namespace pz

extern "C" {

pz_status pz_interactive_crs_seed(const uint8_t crs[32], int what, uint8_t out[32]) {
  if (!crs || !out || what < 0 || what > 2) return PZ_ERR_INVALID_ARGUMENT;
  if (what == PZ_ICRS_PUBLIC_KEY) {
    pz::crs_puncture(crs, 1, out);
    return PZ_OK;
  }
  uint8_t key[32];
  pz::crs_puncture(crs, 2, key);  // key_seed
  pz::crs_puncture(key, what == PZ_ICRS_AUTO_KEYS ? 1 : 2, out);
  return PZ_OK;
}

pz_status pz_ni_crs_seed(const uint8_t crs[32], int what, size_t index, uint8_t out[32]) {
  if (!crs || !out || what < 0 || what > 3) return PZ_ERR_INVALID_ARGUMENT;
  uint8_t key[32], t[32];
  puncture(crs, 1, key);  // key_seed
  switch (what) {
    case PZ_CRS_AUTO_KEYS: puncture(key, 2, out); break;
    case PZ_CRS_LWE_KSK: puncture(key, 3, out); break;
    case PZ_CRS_UI_TO_S_KSK: puncture(crs, 2, t); puncture(t, index + 1, out); break;
    default: puncture(key, 1, t); puncture(t, index + 1, out); break;  // ni_rgsw_cts_main_seed
  }
  return PZ_OK;
}

pz_status pz_ni_aggregate_device(pz_ctx *c, const uint8_t crs[32], const pz_ni_server_key_share_view *shares,
                                 size_t users, uint64_t *d_ksk_b, uint64_t *d_rgsw, uint64_t *d_auto_b,
                                 uint64_t *d_lwe_b, void *stream) {
  if (!c) return PZ_ERR_INVALID_ARGUMENT;
  const pz_params &P = c->P;
  if (P.variant != 2 || P.ni_ks_d == 0 || !P.rgrg_logb)
    return pz::fail(c, PZ_ERR_NOT_SUPPORTED, "not a non-interactive parameter set");
  if (c->logn != NI_LOGN) return pz::fail(c, PZ_ERR_NOT_SUPPORTED, "ring dimension other than 2048");
  if (P.rlrg_d_a != 1 || P.rlrg_d_b != 1)
    return pz::fail(c, PZ_ERR_NOT_SUPPORTED, "rlwe x rgsw decomposition count other than 1");
  if (!crs || !shares || users == 0 || !d_ksk_b || !d_rgsw || !d_auto_b || !d_lwe_b)
    return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "pz_ni_aggregate_device: NULL argument or no users");
  for (size_t u = 0; u < users; u++) {
    const pz_ni_server_key_share_view &s = shares[u];
    if (!s.ui_to_s_ksk || (users > 1 && !s.ksk_zero_encs) || !s.rgsw_zero_encs || !s.auto_keys || !s.lwe_ksk)
      return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "pz_ni_aggregate_device: NULL share field");
  }
  PZ_CK(c, cudaSetDevice(c->device));
  cudaStream_t st = (cudaStream_t)stream;
  const size_t N = P.rlwe_n, n = P.lwe_n, d = P.ni_ks_d;
  const u32 ra = P.rgrg_d_a, rb = P.rgrg_d_b, max_d = std::max(ra, rb), R = ra + rb;
  const size_t rows1 = 2 * (size_t)R;
  NiShape sh{(u32)users, (u32)((n + users - 1) / users), ra, rb, max_d, 1, (u32)d};
  pz_status ps = PZ_OK;
  cudaError_t e = cudaSuccess;
  // ---- device buffers that live through the call
  u64 *d_keys = nullptr, *d_stage = nullptr;
  const u64 **d_src = nullptr;
  NiUser *d_users = nullptr;
  const size_t nsrc = users * users + 2 * users;  // ksk lists, auto list, lwe list
  if (e == cudaSuccess) e = cudaMallocAsync(&d_keys, users * 2 * d * N * 8, st);
  if (e == cudaSuccess) e = cudaMallocAsync(&d_stage, 2 * d * N * 8, st);
  if (e == cudaSuccess) e = cudaMallocAsync((void **)&d_src, nsrc * sizeof(u64 *), st);
  if (e == cudaSuccess) e = cudaMallocAsync(&d_users, users * sizeof(NiUser), st);
  // ---- ui_to_s key B rows (evaluator.rs:1269-1294), auto and LWE KSK sums
  std::vector<const u64 *> src(nsrc);
  for (size_t j = 0; j < users; j++) {
    src[j * users] = shares[j].ui_to_s_ksk;
    size_t t = 1;
    for (size_t k = 0; k < users; k++)
      if (k != j) src[j * users + t++] = shares[k].ksk_zero_encs + (j < k ? j : j - 1) * d * N;
  }
  for (size_t k = 0; k < users; k++) {
    src[users * users + k] = shares[k].auto_keys;
    src[users * users + users + k] = shares[k].lwe_ksk;
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_src, src.data(), nsrc * sizeof(u64 *), cudaMemcpyHostToDevice, st);
  for (size_t j = 0; j < users && e == cudaSuccess; j++) {
    sum_mod_kernel<<<grid_cap(d * N / 256, 1184), 256, 0, st>>>(d_src + j * users, (u32)users, d * N, P.rlwe_q,
                                                                 d_ksk_b + j * d * N);
    e = cudaGetLastError();
  }
  const size_t n_auto = (size_t)P.n_auto_keys * P.auto_d * N, n_lwe = (size_t)P.lwe_d * N;
  if (e == cudaSuccess) {
    sum_mod_kernel<<<grid_cap(n_auto / 256, 1184), 256, 0, st>>>(d_src + users * users, (u32)users, n_auto,
                                                                 P.rlwe_q, d_auto_b);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    sum_mod_kernel<<<grid_cap(n_lwe / 256, 1184), 256, 0, st>>>(d_src + users * users + users, (u32)users, n_lwe,
                                                                P.lwe_q, d_lwe_b);
    e = cudaGetLastError();
  }
  // ---- device key form of every user's Ksk(u_j -> s): A rows from the user's stream
  for (size_t j = 0; j < users && e == cudaSuccess && ps == PZ_OK; j++) {
    uint8_t seed[32];
    pz_ni_crs_seed(crs, PZ_CRS_UI_TO_S_KSK, j, seed);
    ps = pz::seeded_fill_u64(c, seed, P.rlwe_q, (u64)d * N, d * N, 2 * d * N, 0, d_stage, st);
    if (ps == PZ_OK) e = cudaMemcpyAsync(d_stage + d * N, d_ksk_b + j * d * N, d * N * 8, cudaMemcpyDeviceToDevice, st);
    if (ps == PZ_OK && e == cudaSuccess)
      e = pz::launch_key_convert(NI_LOGN, d_stage, d_keys + j * 2 * d * N, 2 * d, c->rc, c->ni_conv_c, c->ni_conv_cs, st);
  }
  std::vector<NiUser> hu(users);
  for (size_t u = 0; u < users; u++) {
    hu[u].ksk = d_keys + u * 2 * d * N;
    hu[u].self_leader = shares[u].self_leader_cts;
    hu[u].not_leader = shares[u].not_leader_cts;
    hu[u].zero_encs = shares[u].rgsw_zero_encs;
    segment(u, users, n, &hu[u].seg_b, &hu[u].seg_e);
    if ((hu[u].seg_e > hu[u].seg_b && !hu[u].self_leader) || (hu[u].seg_e - hu[u].seg_b < n && !hu[u].not_leader))
      ps = pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "pz_ni_aggregate_device: NULL NI RGSW ciphertexts");
  }
  if (e == cudaSuccess && ps == PZ_OK)
    e = cudaMemcpyAsync(d_users, hu.data(), users * sizeof(NiUser), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && ps == PZ_OK) e = cudaStreamSynchronize(st);  // hu, src leave scope only after this
  // ---- RGSWs, chunk by chunk of LWE indices
  const size_t per_index = ((size_t)R * d + R + max_d + (users - 1) * rows1) * N * 8;
  size_t chunk = std::min<size_t>(n, 64);
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess)
    chunk = std::max<size_t>(1, std::min(chunk, free_b / 2 / per_index));
  u64 *d_arows = nullptr, *d_vals = nullptr, *d_dig = nullptr, *d_others = nullptr;
  if (e == cudaSuccess && ps == PZ_OK) e = cudaMallocAsync(&d_arows, chunk * max_d * N * 8, st);
  if (e == cudaSuccess && ps == PZ_OK) e = cudaMallocAsync(&d_vals, chunk * R * N * 8, st);
  if (e == cudaSuccess && ps == PZ_OK) e = cudaMallocAsync(&d_dig, chunk * R * d * N * 8, st);
  if (e == cudaSuccess && ps == PZ_OK && users > 1)
    e = cudaMallocAsync(&d_others, (users - 1) * chunk * rows1 * N * 8, st);
  const pz::Decomp dp = pz::decomposer(P.rlwe_q, P.ni_ks_logb, (u32)d);
  const size_t smem = 2 * N * 8;
  std::vector<uint8_t> seeds(chunk * 32);
  for (size_t i0 = 0; i0 < n && e == cudaSuccess && ps == PZ_OK; i0 += chunk) {
    const size_t cnt = std::min(chunk, n - i0);
    for (size_t c0 = 0; c0 < cnt; c0++) pz_ni_crs_seed(crs, PZ_CRS_NI_RGSW, i0 + c0, &seeds[c0 * 32]);
    ps = pz::seeded_fill_batch_u64(c, (const uint8_t(*)[32])seeds.data(), cnt, P.rlwe_q, (u64)max_d * N, d_arows,
                                   (u64)max_d * N, st);
    if (ps != PZ_OK) break;
    ni_values_kernel<<<grid_cap(cnt * R * N / 256, 4736), 256, 0, st>>>(d_users, sh, d_arows, (u32)i0, (u32)cnt,
                                                                       P.rlwe_q, d_vals);
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    ni_digits_kernel<<<grid_cap(cnt * R, 65535), NI_T, smem, st>>>(c->rc, dp, (u32)d, d_vals, d_dig, cnt * R);
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    u64 *lead = d_rgsw + i0 * 4 * N;
    ni_agg_mac_kernel<<<grid_cap(cnt * R * users, 65535), NI_T, smem, st>>>(c->rc, sh, d_dig, d_users, (u32)i0,
                                                                           (u32)cnt, lead, d_others);
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    if (users > 1) ps = pz_aggregate_rgsw_device(c, lead, d_others, users - 1, cnt, st);
  }
  if (e == cudaSuccess && ps == PZ_OK) e = cudaStreamSynchronize(st);
  cudaFreeAsync(d_arows, st);
  cudaFreeAsync(d_vals, st);
  cudaFreeAsync(d_dig, st);
  cudaFreeAsync(d_others, st);
  cudaFreeAsync(d_keys, st);
  cudaFreeAsync(d_stage, st);
  cudaFreeAsync((void *)d_src, st);
  cudaFreeAsync(d_users, st);
  cudaStreamSynchronize(st);
  if (ps != PZ_OK) return ps;
  if (e != cudaSuccess) return pz::cuda_fail(c, "pz_ni_aggregate_device", e);
  return PZ_OK;
}

pz_status pz_ni_aggregate_server_key(pz_ctx *c, const uint8_t crs[32], const pz_ni_server_key_share_view *shares,
                                     size_t users, pz_key **key_out, pz_ni_ksk **ksks_out) {
  if (!c) return PZ_ERR_INVALID_ARGUMENT;
  if (!key_out || !ksks_out) return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "pz_ni_aggregate_server_key: NULL output");
  *key_out = nullptr;
  for (size_t u = 0; u < users; u++) ksks_out[u] = nullptr;
  const pz_params &P = c->P;
  const size_t N = P.rlwe_n, d = P.ni_ks_d;
  PZ_CK(c, cudaSetDevice(c->device));
  u64 *d_ksk = nullptr, *d_rgsw = nullptr, *d_auto = nullptr, *d_lwe = nullptr;
  cudaError_t e = cudaMalloc(&d_ksk, std::max<size_t>(users, 1) * d * N * 8);
  if (e == cudaSuccess) e = cudaMalloc(&d_rgsw, (size_t)P.lwe_n * 4 * N * 8);
  if (e == cudaSuccess) e = cudaMalloc(&d_auto, (size_t)P.n_auto_keys * P.auto_d * N * 8);
  if (e == cudaSuccess) e = cudaMalloc(&d_lwe, (size_t)P.lwe_d * N * 8);
  pz_status s = e == cudaSuccess ? PZ_OK : pz::cuda_fail(c, "pz_ni_aggregate_server_key", e);
  if (s == PZ_OK) s = pz_ni_aggregate_device(c, crs, shares, users, d_ksk, d_rgsw, d_auto, d_lwe, c->stream);
  if (s == PZ_OK) {
    pz_seeded_server_key_view v{};
    v.rgsw = d_rgsw;
    v.auto_b = d_auto;
    v.lwe_ksk_b = d_lwe;
    pz_ni_crs_seed(crs, PZ_CRS_AUTO_KEYS, 0, v.auto_seed);
    pz_ni_crs_seed(crs, PZ_CRS_LWE_KSK, 0, v.lwe_ksk_seed);
    s = pz_key_upload_seeded(c, &v, key_out);
  }
  for (size_t u = 0; u < users && s == PZ_OK; u++) {
    uint8_t seed[32];
    pz_ni_crs_seed(crs, PZ_CRS_UI_TO_S_KSK, u, seed);
    s = pz_ni_ksk_upload_seeded(c, d_ksk + u * d * N, seed, &ksks_out[u]);
  }
  cudaFree(d_ksk);
  cudaFree(d_rgsw);
  cudaFree(d_auto);
  cudaFree(d_lwe);
  if (s != PZ_OK) {
    pz_key_release(*key_out);
    *key_out = nullptr;
    for (size_t u = 0; u < users; u++) {
      pz_ni_ksk_release(ksks_out[u]);
      ksks_out[u] = nullptr;
    }
  }
  return s;
}

}  // extern "C"
