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
      e = pz::launch_key_convert((int)c->logn, src, d_eval, m * rows1, c->rc, c->conv_c, c->conv_cs, st);
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

}  // extern "C"
