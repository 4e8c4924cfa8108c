// pz_aggregate.cu -- server-key aggregation on the device: batched
// rgsw_by_rgsw_inplace (rgsw/runtime.rs:883-985), the RGSW step of
// aggregate_interactive_multi_party_server_key_shares (bool/evaluator.rs:
// 1110-1200), which multiplies each LWE index's leader RGSW by every other
// user's RGSW for that index, one user after another.
//
// Each RLWE row pair of the leader's RGSW (rlwe x rgsw shape: d_a = d_b = 1
// for every production set, so the pairs are the contiguous row blocks
// (A(-sm), B(-sm)) and (A(m), B(m))) is one item of the external-product
// kernel in its general-decomposition form: the other user's RGSW (rgsw x rgsw
// shape, rgrg_decomposer_params: logb 2..7, up to 20/18 digits) is converted
// to the device evaluation form and plays the role of the key; digits of A
// and of B are transformed pairwise and accumulated lazily; one inverse
// transform per output; the result stays in the coefficient domain, like the
// reference's rgsw0 after its backward NTTs.
#include <algorithm>
#include <vector>

#include "pz_internal.h"

using pz::u32;
using pz::u64;

extern "C" {

pz_status pz_aggregate_rgsw_device(pz_ctx *c, uint64_t *d_rgsw0, const uint64_t *d_others, size_t steps,
                                   size_t count, void *stream) {
  if (!c) return PZ_ERR_INVALID_ARGUMENT;
  const pz_params &P = c->P;
  if (!P.rgrg_logb) return pz::fail(c, PZ_ERR_NOT_SUPPORTED, "parameter set without RGSW x RGSW");
  if (P.rlrg_d_a != 1 || P.rlrg_d_b != 1)
    return pz::fail(c, PZ_ERR_NOT_SUPPORTED, "rlwe x rgsw decomposition count other than 1");
  if ((steps && count) && (!d_rgsw0 || !d_others)) return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "NULL argument");
  if (steps == 0 || count == 0) return PZ_OK;
  PZ_CK(c, cudaSetDevice(c->device));
  cudaStream_t st = (cudaStream_t)stream;
  const size_t N = P.rlwe_n, ra = P.rgrg_d_a, rb = P.rgrg_d_b, rows1 = 2 * (ra + rb), rows0 = 4;
  const size_t chunk = std::min<size_t>(count, 4096);  // RGSWs per launch (item indices stay < 8192)
  pz::BrParams br = c->br;
  br.da = pz::decomposer(P.rlwe_q, P.rgrg_logb, (u32)ra);
  br.db = pz::decomposer(P.rlwe_q, P.rgrg_logb, (u32)rb);
  br.d_a = (u32)ra;
  br.d_b = (u32)rb;
  br.rgsw_rows = (u32)rows1;
  br.autos = nullptr;
  br.out_idx = nullptr;
  u64 *d_eval = nullptr;
  u32 *d_idx = nullptr;
  std::vector<u32> idx(2 * chunk);
  for (size_t i = 0; i < 2 * chunk; i++) idx[i] = (u32)(i / 2);  // two RLWEs per leader RGSW
  cudaError_t e = cudaMallocAsync(&d_eval, chunk * rows1 * N * 8, st);
  if (e == cudaSuccess) e = cudaMallocAsync(&d_idx, 2 * chunk * 4, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_idx, idx.data(), 2 * chunk * 4, cudaMemcpyHostToDevice, st);
  for (size_t t = 0; t < steps && e == cudaSuccess; t++) {  // the other users, in order
    for (size_t c0 = 0; c0 < count && e == cudaSuccess; c0 += chunk) {
      const size_t m = std::min(chunk, count - c0);
      const u64 *src = d_others + (t * count + c0) * rows1 * N;
      e = pz::launch_key_convert((int)c->logn, src, d_eval, m * rows1, c->rc, c->br_conv_c, c->br_conv_cs, st);
      if (e != cudaSuccess) break;
      br.rgsw = d_eval;
      br.n = (u32)m;
      e = pz::launch_ext_product((int)c->logn, false, br, d_rgsw0 + c0 * rows0 * N, d_idx, 2 * m, 0, st);
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFreeAsync(d_eval, st);
  cudaFreeAsync(d_idx, st);
  if (e != cudaSuccess) return pz::cuda_fail(c, "pz_aggregate_rgsw_device", e);
  return PZ_OK;
}

pz_status pz_rgsw_by_rgsw_device(pz_ctx *c, uint64_t *d_rgsw0, const uint64_t *d_rgsw1, size_t count,
                                 void *stream) {
  return pz_aggregate_rgsw_device(c, d_rgsw0, d_rgsw1, 1, count, stream);
}

// aggregate_interactive_multi_party_server_key_shares, whole: for each
// leader's segment of LWE indices its RGSWs are copied into place and the
// other users' RGSWs of the same indices (not_self_leader_rgsws, the offset
// of an earlier user's own segment removed) are gathered in increasing id
// into the [steps][count][rows][N] layout of pz_aggregate_rgsw_device; the
// auto keys and the LWE KSK are summed.
pz_status pz_aggregate_device(pz_ctx *c, const pz_server_key_share_view *shares, size_t users, uint64_t *d_rgsw,
                              uint64_t *d_auto_b, uint64_t *d_lwe_b, void *stream) {
  if (!c) return PZ_ERR_INVALID_ARGUMENT;
  const pz_params &P = c->P;
  if (!P.rgrg_logb) return pz::fail(c, PZ_ERR_NOT_SUPPORTED, "parameter set without RGSW x RGSW");
  if (P.rlrg_d_a != 1 || P.rlrg_d_b != 1)
    return pz::fail(c, PZ_ERR_NOT_SUPPORTED, "rlwe x rgsw decomposition count other than 1");
  if (!shares || users == 0 || !d_rgsw || !d_auto_b || !d_lwe_b)
    return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "pz_aggregate_device: NULL argument or no users");
  const size_t N = P.rlwe_n, n = P.lwe_n, rows0 = 4, rows1 = 2 * ((size_t)P.rgrg_d_a + P.rgrg_d_b);
  const size_t per = (n + users - 1) / users;
  std::vector<size_t> sb(users), se(users);
  size_t max_seg = 0;
  for (size_t u = 0; u < users; u++) {  // multi_party_user_id_lwe_segment (evaluator.rs:613-626)
    sb[u] = std::min(per * u, n);
    se[u] = std::max(sb[u], std::min(per * (u + 1), n));
    max_seg = std::max(max_seg, se[u] - sb[u]);
    const pz_server_key_share_view &v = shares[u];
    if (!v.auto_keys || !v.lwe_ksk || (se[u] > sb[u] && !v.self_leader_rgsws) ||
        (users > 1 && se[u] - sb[u] < n && !v.not_self_leader_rgsws))
      return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "pz_aggregate_device: NULL share field");
  }
  PZ_CK(c, cudaSetDevice(c->device));
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<const u64 *> src(2 * users);
  for (size_t u = 0; u < users; u++) {
    src[u] = shares[u].auto_keys;
    src[users + u] = shares[u].lwe_ksk;
  }
  const u64 **d_src = nullptr;
  u64 *d_others = nullptr;
  cudaError_t e = cudaMallocAsync((void **)&d_src, 2 * users * sizeof(u64 *), st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_src, src.data(), 2 * users * sizeof(u64 *), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = pz::launch_sum_mod(d_src, (u32)users, (size_t)P.n_auto_keys * P.auto_d * N, P.rlwe_q, d_auto_b, st);
  if (e == cudaSuccess) e = pz::launch_sum_mod(d_src + users, (u32)users, (size_t)P.lwe_d * N, P.lwe_q, d_lwe_b, st);
  if (e == cudaSuccess && users > 1) e = cudaMallocAsync(&d_others, (users - 1) * max_seg * rows1 * N * 8, st);
  pz_status ps = PZ_OK;
  for (size_t L = 0; L < users && e == cudaSuccess && ps == PZ_OK; L++) {
    const size_t b = sb[L], cnt = se[L] - sb[L];
    if (!cnt) continue;
    e = cudaMemcpyAsync(d_rgsw + b * rows0 * N, shares[L].self_leader_rgsws, cnt * rows0 * N * 8,
                        cudaMemcpyDeviceToDevice, st);
    for (size_t o = 0, t = 0; o < users && e == cudaSuccess; o++) {
      if (o == L) continue;
      const size_t pos = o < L ? b - (se[o] - sb[o]) : b;  // index in o's not_self_leader list
      e = cudaMemcpyAsync(d_others + t * cnt * rows1 * N, shares[o].not_self_leader_rgsws + pos * rows1 * N,
                          cnt * rows1 * N * 8, cudaMemcpyDeviceToDevice, st);
      t++;
    }
    if (e == cudaSuccess && users > 1) ps = pz_aggregate_rgsw_device(c, d_rgsw + b * rows0 * N, d_others, users - 1,
                                                                     cnt, st);
  }
  if (e == cudaSuccess && ps == PZ_OK) e = cudaStreamSynchronize(st);
  cudaFreeAsync((void *)d_src, st);
  cudaFreeAsync(d_others, st);
  cudaStreamSynchronize(st);
  if (ps != PZ_OK) return ps;
  if (e != cudaSuccess) return pz::cuda_fail(c, "pz_aggregate_device", e);
  return PZ_OK;
}

pz_status pz_aggregate_server_key(pz_ctx *c, const uint8_t crs[32], const pz_server_key_share_view *shares,
                                  size_t users, pz_key **key_out) {
  if (!c) return PZ_ERR_INVALID_ARGUMENT;
  if (!crs || !key_out) return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "pz_aggregate_server_key: NULL argument");
  *key_out = nullptr;
  const pz_params &P = c->P;
  const size_t N = P.rlwe_n;
  PZ_CK(c, cudaSetDevice(c->device));
  u64 *d_rgsw = nullptr, *d_auto = nullptr, *d_lwe = nullptr;
  cudaError_t e = cudaMalloc(&d_rgsw, (size_t)P.lwe_n * 4 * N * 8);
  if (e == cudaSuccess) e = cudaMalloc(&d_auto, (size_t)P.n_auto_keys * P.auto_d * N * 8);
  if (e == cudaSuccess) e = cudaMalloc(&d_lwe, (size_t)P.lwe_d * N * 8);
  pz_status s = e == cudaSuccess ? PZ_OK : pz::cuda_fail(c, "pz_aggregate_server_key", e);
  if (s == PZ_OK) s = pz_aggregate_device(c, shares, users, d_rgsw, d_auto, d_lwe, c->stream);
  if (s == PZ_OK) {
    pz_seeded_server_key_view v{};
    v.rgsw = d_rgsw;
    v.auto_b = d_auto;
    v.lwe_ksk_b = d_lwe;
    pz_interactive_crs_seed(crs, PZ_ICRS_AUTO_KEYS, v.auto_seed);
    pz_interactive_crs_seed(crs, PZ_ICRS_LWE_KSK, v.lwe_ksk_seed);
    s = pz_key_upload_seeded(c, &v, key_out);
  }
  cudaFree(d_rgsw);
  cudaFree(d_auto);
  cudaFree(d_lwe);
  return s;
}

}  // extern "C"
