// pz_runtime.cu -- host runtime behind the C ABI (include/phantom_zone_b200.h).
//
// Owns per-context device tables (twiddles, dlog map, test vectors), device
// server keys, scratch, and the launch sequence of a gate batch:
//   ks kernel (prelude + mod-down + LWE key switch)  ->  pbs kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "pz_internal.h"

using pz::u32;
using pz::u64;
typedef unsigned __int128 u128;

namespace {

// bool/parameters.rs:526-726
const pz_params PARAMS[PZ_NUM_PARAMS] = {
    // rlwe_q, lwe_q, br_q, N, n, lwe_logb, lwe_d, rlrg_logb, d_a, d_b, auto_logb, auto_d, g, w, gauss, variant
    {18014398509404161ULL, 1ULL << 15, 1u << 11, 1u << 11, 580, 1, 12, 17, 1, 1, 24, 1, 5, 10, 0, 1, 0, 0, 0, 0},
    {18014398509404161ULL, 1ULL << 16, 1u << 11, 1u << 11, 620, 1, 13, 17, 1, 1, 24, 1, 5, 10, 0, 1, 0, 0, 0, 0},
    {18014398509404161ULL, 1ULL << 17, 1u << 12, 1u << 11, 660, 1, 14, 17, 1, 1, 24, 1, 5, 10, 0, 1, 0, 0, 0, 0},
    {18014398509404161ULL, 1ULL << 16, 1u << 12, 1u << 11, 520, 1, 13, 17, 1, 1, 24, 1, 5, 10, 1, 2, 0, 0, 0, 0},
    {18014398509404161ULL, 1ULL << 16, 1u << 11, 1u << 11, 620, 1, 13, 17, 1, 1, 24, 1, 5, 10, 0, 2, 0, 0, 0, 0},
    {18014398509404161ULL, 1ULL << 16, 1u << 12, 1u << 11, 620, 1, 13, 17, 1, 1, 24, 1, 5, 10, 0, 2, 0, 0, 0, 0},
    {18014398509404161ULL, 1ULL << 17, 1u << 12, 1u << 11, 660, 1, 14, 17, 1, 1, 24, 1, 5, 10, 0, 2, 0, 0, 0, 0},
    {268369921ULL, 1ULL << 16, 1u << 9, 1u << 9, 100, 4, 4, 7, 4, 4, 7, 4, 5, 5, 1, 0, 0, 0, 0, 0},
};

pz_params full_params(int id) {
  pz_params p = PARAMS[id];
  p.embedding_factor = 2 * p.rlwe_n / p.br_q;
  p.rgsw_rows = 2 * p.rlrg_d_a + 2 * p.rlrg_d_b;
  p.auto_rows = 2 * p.auto_d;
  p.n_auto_keys = p.w + 1;
  p.ni_ks_logb = p.variant == 2 ? 1 : 0;  // parameters.rs:616-697
  p.ni_ks_d = p.variant == 2 ? 50 : 0;
  // rgrg_decomposer_params, parameters.rs:539-695 (none for the single-party test set)
  static const uint32_t RGRG[PZ_NUM_PARAMS][3] = {{7, 6, 5}, {6, 7, 6}, {5, 9, 8}, {4, 10, 9},
                                                  {3, 13, 12}, {4, 10, 9}, {2, 20, 18}, {0, 0, 0}};
  p.rgrg_logb = RGRG[id][0];
  p.rgrg_d_a = RGRG[id][1];
  p.rgrg_d_b = RGRG[id][2];
  return p;
}

u64 mulmod(u64 a, u64 b, u64 q) { return (u64)(((u128)a * b) % q); }
u64 powmod(u64 a, u64 e, u64 q) {
  u64 r = 1 % q;
  a %= q;
  while (e) {
    if (e & 1) r = mulmod(r, a, q);
    a = mulmod(a, a, q);
    e >>= 1;
  }
  return r;
}
u64 invmod(u64 a, u64 q) { return powmod(a, q - 2, q); }  // q prime
u64 shoup(u64 v, u64 q) { return (u64)(((u128)v << 64) / q); }
// Second word of a twiddle-table entry: Shoup(w), or for the N = 2048 FP64-
// quotient butterflies the bits of w/Q rounded once to a double (the
// quotient in 80-bit long double first, error 2^-64 relative)
u64 tw_companion(u64 w, u64 q, u32 logn) {
  if (logn == 11 && pz::BFLY_FP64) {
    const double d = (double)((long double)w / (long double)q);
    u64 bits;
    memcpy(&bits, &d, 8);
    return bits;
  }
  return shoup(w, q);
}
u32 log2_exact(u64 v) { return 63 - __builtin_clzll(v); }
// utils.rs:230-237
u32 log2_ref(u64 v) { return (v & (v - 1)) == 0 ? 63 - __builtin_clzll(v) : 64 - __builtin_clzll(v); }

// A primitive 2N-th root of unity: c^((Q-1)/2N) for the smallest c >= 2
// whose power has order exactly 2N (omega^N = -1).
u64 default_root(u64 q, u64 two_n) {
  for (u64 c = 2; c < 1000000; c++) {
    u64 w = powmod(c, (q - 1) / two_n, q);
    if (powmod(w, two_n / 2, q) == q - 1) return w;
  }
  return 0;
}

pz::Decomp make_decomp(u64 q, u32 logb, u32 d) {  // decomposer.rs:158-178
  pz::Decomp dp;
  dp.q = q;
  dp.logb = logb;
  dp.d = d;
  dp.ignore_bits = log2_ref(q) - logb * d;
  dp.bmask = (1ull << logb) - 1;
  dp.bby2 = 1ull << (logb - 1);
  return dp;
}

}  // namespace

namespace pz {
Decomp decomposer(u64 q, u32 logb, u32 d) { return make_decomp(q, logb, d); }

pz_status fail(pz_ctx *ctx, pz_status s, const std::string &msg) {
  if (ctx) ctx->err = msg;
  return s;
}
pz_status cuda_fail(pz_ctx *ctx, const char *what, cudaError_t e) {
  pz_status s = (e == cudaErrorMemoryAllocation) ? PZ_ERR_OUT_OF_MEMORY : PZ_ERR_CUDA;
  return fail(ctx, s, std::string(what) + ": " + cudaGetErrorString(e));
}
u32 ks_stride(const pz_params &P) { return (P.lwe_n + 1 + 31) & ~31u; }
}  // namespace pz

namespace {
using pz::cuda_fail;
using pz::fail;
using pz::ks_stride;

cudaStream_t pick(pz_ctx *, void *stream) { return (cudaStream_t)stream; }

// evaluator.rs:664-673 dlog map; :688-726 test vectors; :728-743 auto elements
void build_tables(pz_ctx *c, std::vector<unsigned short> &dlog, std::vector<u64> &tv) {
  const pz_params &P = c->P;
  const u32 q = P.br_q, R = q / 2;
  const u64 Q = P.rlwe_q;
  dlog.assign(q, 0);
  for (u32 i = 0; i < q / 4; i++) {
    u64 v = powmod(P.g, i, q);
    dlog[v] = (unsigned short)i;
    dlog[q - v] = (unsigned short)(i + q / 4);
  }
  const u64 true_el = Q >> 3, false_el = Q - true_el;
  // X -> X^{-g} map on the br_q/2 ring (generate_auto_map, keygen.rs:16-41)
  std::vector<u32> idx(R);
  std::vector<unsigned char> sgn(R);
  const u64 k = 2ull * R - (P.g % (2ull * R));
  for (u32 i = 0; i < R; i++) {
    u64 t = ((u64)i * k) % (2ull * R);
    bool s = true;
    if (t >= R) { t -= R; s = false; }
    idx[i] = (u32)t;
    sgn[i] = s;
  }
  auto one = [&](u32 part, u64 before, u64 after, u64 *out) {
    for (u32 i = 0; i < R; i++) {
      u64 v = i < part ? before : after;
      out[idx[i]] = sgn[i] ? v : Q - v;
    }
  };
  tv.assign(6ull * R, 0);
  const u32 qby8 = q >> 3;
  one(3 * qby8, false_el, true_el, &tv[0 * R]);  // and
  one(3 * qby8, true_el, false_el, &tv[1 * R]);  // nand
  one(qby8, false_el, true_el, &tv[2 * R]);      // or
  one(qby8, true_el, false_el, &tv[3 * R]);      // nor
  one(qby8, false_el, true_el, &tv[4 * R]);      // xor
  one(qby8, true_el, false_el, &tv[5 * R]);      // xnor
  const u64 two_n = 2ull * P.rlwe_n;
  for (u32 s = 0; s <= P.w; s++) {
    u64 el = s == 0 ? two_n - (P.g % two_n) : (powmod(P.g, s, 1ull << 62) % q) % two_n;
    c->br.auto_k[s] = (u32)el;
  }
}

pz_status ensure_scratch(pz_ctx *c, size_t count) {
  if (count <= c->cap) return PZ_OK;
  size_t cap = std::max(count, c->cap * 2);
  const size_t L = (size_t)c->P.rlwe_n + 1;
  cudaFree(c->d_c0); cudaFree(c->d_c1); cudaFree(c->d_out); cudaFree(c->d_gates); cudaFree(c->d_ks);
  c->d_c0 = c->d_c1 = c->d_out = nullptr; c->d_gates = nullptr; c->d_ks = nullptr;
  c->cap = 0;
  PZ_CK(c, cudaMalloc(&c->d_c0, cap * L * 8));
  PZ_CK(c, cudaMalloc(&c->d_c1, cap * L * 8));
  PZ_CK(c, cudaMalloc(&c->d_out, cap * L * 8));
  PZ_CK(c, cudaMalloc(&c->d_gates, cap));
  PZ_CK(c, cudaMalloc(&c->d_ks, cap * ks_stride(c->P) * 4));
  c->cap = cap;
  return PZ_OK;
}

pz_status check_key(pz_ctx *c, const pz_key *k) {
  if (!k) return fail(c, PZ_ERR_INVALID_ARGUMENT, "key is NULL");
  if (k->ctx != c) return fail(c, PZ_ERR_KEY_MISMATCH, "key was uploaded through another context");
  return PZ_OK;
}

pz_status check_gates_host(pz_ctx *c, const uint8_t *gates, size_t count, bool raw) {
  for (size_t i = 0; i < count; i++)
    if ((gates[i] & 0x7f) > 5 || (!raw && (gates[i] & 0x80)))
      return fail(c, PZ_ERR_INVALID_ARGUMENT, "gate code out of range at index " + std::to_string(i));
  return PZ_OK;
}

}  // namespace

namespace pz {
void build_ksk8(pz_ctx *c, pz_key *k, cudaStream_t s) {
  const pz_params &P = c->P;
  const u32 rows = P.lwe_d * P.rlwe_n;
  if (!k->d_ksk || rows % 32 || P.rlwe_n % 32 || P.lwe_d > 16 || P.lwe_logb > 7) return;
  const u32 planes = ksk8_planes(c->ks.mask), cols = ksk8_cols(P.lwe_n);
  const size_t bytes = (size_t)planes * rows * cols;
  if (cudaMalloc(&k->d_ksk8, bytes) != cudaSuccess) {
    cudaGetLastError();
    k->d_ksk8 = nullptr;
    return;
  }
  if (launch_ksk_planes(k->d_ksk, rows, ks_stride(P), P.lwe_n, planes, k->d_ksk8, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(k->d_ksk8);
    k->d_ksk8 = nullptr;
    return;
  }
  k->bytes += bytes;
}

void free_key_arrays(pz_key *k) {
  cudaFree(k->d_rgsw);
  cudaFree(k->d_autos);
  cudaFree(k->d_ksk);
  cudaFree(k->d_ksk8);
}

void ks_bind_key(const pz_ctx *c, const pz_key *k, KsParams &ks) {
  ks.ksk = k->d_ksk;
  ks.ksk8 = k->d_ksk8;
  ks.planes = ksk8_planes(c->ks.mask);
  ks.ksk8_cols = ksk8_cols(c->P.lwe_n);
}

int effective_variant(pz_ctx *c, size_t count) {
  const bool d1 = c->P.rlrg_d_a == 1 && c->P.rlrg_d_b == 1 && c->P.auto_d == 1;
  if (c->logn != 11 || !d1) return c->pbs_variant;
  const pz_ctx::Tuned &t = c->tuned[size_bucket(count)];
  if (t.variant >= 0) return t.variant;
  if (c->split_below < 0) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    c->split_below = sms / 2;
  }
  return (count <= (size_t)c->split_below) ? pz::PBS_SPLIT : c->pbs_variant;
}

int effective_ks_ct(const pz_ctx *c, size_t count) {
  const pz_ctx::Tuned &t = c->tuned[size_bucket(count)];
  return t.ks_ct ? t.ks_ct : c->ks_ct;
}

pz_status run_gates(pz_ctx *c, const pz_key *k, const unsigned char *d_gates, const u64 *d_c0, const u64 *d_c1,
                    u64 *d_out, size_t count, u32 *d_ks_out, u64 *d_rlwe, cudaStream_t s, u32 *d_ks_scratch,
                    bool raw, const u32 *in0, const u32 *in1, const u32 *out_idx) {
  pz::BrParams br = c->br;
  br.rgsw = k->d_rgsw;
  br.autos = k->d_autos;
  br.out_idx = out_idx;
  pz::KsParams ks = c->ks;
  pz::ks_bind_key(c, k, ks);
  ks.raw = raw ? 1u : 0u;
  ks.in0 = in0;
  ks.in1 = in1;
  const u32 stride = ks_stride(c->P);
  u32 *d_ks = d_ks_out ? d_ks_out : d_ks_scratch;
  const u32 ks_out_stride = d_ks_out ? c->P.lwe_n + 1 : stride;
  ks.out_stride = ks_out_stride;
  cudaError_t e = pz::launch_ks(ks, d_gates, d_c0, d_c1, count, d_ks, s, d_ks_out != nullptr,
                                effective_ks_ct(c, count));
  if (e != cudaSuccess) return cuda_fail(c, "launch_ks", e);
  const bool d1 = c->P.rlrg_d_a == 1 && c->P.rlrg_d_b == 1 && c->P.auto_d == 1;
  e = pz::launch_pbs((int)c->logn, d1, br, d_ks, ks_out_stride, d_gates, d_out, count, d_rlwe, c->grid_limit, s,
                     effective_variant(c, count));
  if (e != cudaSuccess) return cuda_fail(c, "launch_pbs", e);
  return PZ_OK;
}

}  // namespace pz
using pz::run_gates;

extern "C" {

const char *pz_status_string(pz_status s) {
  switch (s) {
    case PZ_OK: return "ok";
    case PZ_ERR_INVALID_ARGUMENT: return "invalid argument";
    case PZ_ERR_CUDA: return "CUDA error";
    case PZ_ERR_OUT_OF_MEMORY: return "out of device memory";
    case PZ_ERR_NOT_SUPPORTED: return "not supported";
    case PZ_ERR_KEY_MISMATCH: return "key does not belong to this context";
  }
  return "unknown status";
}

pz_status pz_param_get(int id, pz_params *out) {
  if (id < 0 || id >= PZ_NUM_PARAMS || !out) return PZ_ERR_INVALID_ARGUMENT;
  *out = full_params(id);
  return PZ_OK;
}

pz_status pz_ctx_create(int id, int device, pz_ctx **out) { return pz_ctx_create_ex(id, device, 0, out); }

pz_status pz_ctx_create_ex(int id, int device, uint64_t root, pz_ctx **out) {
  if (!out) return PZ_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (id < 0 || id >= PZ_NUM_PARAMS) return PZ_ERR_INVALID_ARGUMENT;
  pz::noalloc_forget_device(device);
  pz_ctx *c = new pz_ctx();
  c->param_id = id;
  c->device = device;
  c->P = full_params(id);
  const pz_params &P = c->P;
  const u64 Q = P.rlwe_q;
  const u64 N = P.rlwe_n;
  c->logn = log2_exact(N);
  if (c->logn != 9 && c->logn != 11) { delete c; return PZ_ERR_NOT_SUPPORTED; }
  // the N = 2048 kernels reduce with the special form of this ring's prime
  if (c->logn == 11 && Q != pz::Q_N2048) { delete c; return PZ_ERR_NOT_SUPPORTED; }
  // ... and the one-digit decomposers of those sets (compile-time shapes)
  if (c->logn == 11 && P.rlrg_d_a == 1 && P.rlrg_d_b == 1 && P.auto_d == 1 &&
      (P.rlrg_logb != (u32)pz::RLRG_LOGB || P.auto_logb != (u32)pz::AUTO_LOGB ||
       log2_ref(Q) - P.rlrg_logb != (u32)pz::RLRG_IGN || log2_ref(Q) - P.auto_logb != (u32)pz::AUTO_IGN)) {
    delete c;
    return PZ_ERR_NOT_SUPPORTED;
  }
  if (root == 0) root = default_root(Q, 2 * N);
  if (root == 0 || powmod(root, N, Q) != Q - 1) { delete c; return PZ_ERR_INVALID_ARGUMENT; }
  c->root = root;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) { delete c; return PZ_ERR_CUDA; }
  // twiddles: psi^{bitrev(i)} and psi^{-bitrev(i)} (ntt.rs:337-369), each
  // interleaved with its companion: [w_0, ws_0, w_1, ws_1, ...] (the Shoup
  // companion, or w/Q as a double for the FP64-quotient butterflies)
  std::vector<u64> tw(4 * N);
  const u64 rinv = invmod(root, Q);
  u64 pw = 1, pwi = 1;
  for (u64 i = 0; i < N; i++) {
    u64 bo = 0;
    for (u32 b = 0; b < c->logn; b++) bo |= ((i >> b) & 1) << (c->logn - 1 - b);
    tw[2 * bo] = pw;
    tw[2 * bo + 1] = tw_companion(pw, Q, c->logn);
    tw[2 * N + 2 * bo] = pwi;
    tw[2 * N + 2 * bo + 1] = tw_companion(pwi, Q, c->logn);
    pw = mulmod(pw, root, Q);
    pwi = mulmod(pwi, rinv, Q);
  }
  std::vector<unsigned short> dlog;
  std::vector<u64> tv;
  build_tables(c, dlog, tv);
#define CK_CREATE(call)                                   \
  do {                                                    \
    cudaError_t _e = (call);                              \
    if (_e != cudaSuccess) { pz_ctx_destroy(c); return PZ_ERR_CUDA; } \
  } while (0)
  CK_CREATE(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  CK_CREATE(cudaMalloc(&c->d_tw, 4 * N * 8));
  CK_CREATE(cudaMemcpy(c->d_tw, tw.data(), 4 * N * 8, cudaMemcpyHostToDevice));
  CK_CREATE(cudaMalloc(&c->d_dlog, dlog.size() * 2));
  CK_CREATE(cudaMemcpy(c->d_dlog, dlog.data(), dlog.size() * 2, cudaMemcpyHostToDevice));
  CK_CREATE(cudaMalloc(&c->d_err, sizeof(u32)));
  CK_CREATE(cudaMemset(c->d_err, 0, sizeof(u32)));
  CK_CREATE(cudaMalloc(&c->d_tv, tv.size() * 8));
  CK_CREATE(cudaMemcpy(c->d_tv, tv.data(), tv.size() * 8, cudaMemcpyHostToDevice));
#undef CK_CREATE
  // Montgomery constant -Q^{-1} mod 2^64 (Newton iteration)
  u64 inv = Q;
  for (int i = 0; i < 6; i++) inv *= 2 - Q * inv;
  pz::RingConsts &rc = c->rc;
  rc.q = Q;
  rc.qinv_neg = 0 - inv;
  rc.n_inv = invmod(N, Q);
  rc.n_inv_s = shoup(rc.n_inv, Q);
  rc.one_s = shoup(1, Q);
  rc.iw1n = mulmod(tw[2 * N + 2], rc.n_inv, Q);  // psi^{-bitrev(1)} N^{-1}
  rc.iw1n_s = shoup(rc.iw1n, Q);
  rc.fw = c->d_tw;
  rc.iw = c->d_tw + 2 * N;
  const u64 r64 = (u64)(((u128)1 << 64) % Q);
  c->conv_c = mulmod(rc.n_inv, r64, Q);  // Montgomery-product keys: K * N^{-1} * 2^64
  c->conv_cs = shoup(c->conv_c, Q);
  // blind-rotation keys: K * N^{-1} where the multiply-accumulates fold (mac_reduce)
  // (every N = 2048 multiply-accumulate of the blind rotation and aggregation folds)
  const bool fold = c->logn == 11 && pz::MAC_FOLD_N2048;
  c->br_conv_c = fold ? rc.n_inv : c->conv_c;
  c->br_conv_cs = shoup(c->br_conv_c, Q);
  c->ni_conv_c = (c->logn == 11 && pz::MAC_FOLD_N2048) ? rc.n_inv : c->conv_c;
  c->ni_conv_cs = shoup(c->ni_conv_c, Q);
  pz::BrParams &br = c->br;
  br.rc = rc;
  br.err = c->d_err;
  br.da = make_decomp(Q, P.rlrg_logb, P.rlrg_d_a);
  br.db = make_decomp(Q, P.rlrg_logb, P.rlrg_d_b);
  br.dauto = make_decomp(Q, P.auto_logb, P.auto_d);
  br.d_a = P.rlrg_d_a;
  br.d_b = P.rlrg_d_b;
  br.d_auto = P.auto_d;
  br.rgsw_rows = P.rgsw_rows;
  br.auto_rows = P.auto_rows;
  br.n = P.lwe_n;
  br.br_q = P.br_q;
  br.w = P.w;
  br.g = P.g;
  br.emb = P.embedding_factor;
  br.q_ks_f = (double)P.lwe_q;
  br.ks_mask = (u32)(P.lwe_q - 1);
  br.br_q_f = (double)P.br_q;
  br.dlog = c->d_dlog;
  br.tv = c->d_tv;
  pz::KsParams &ks = c->ks;
  ks.Q = Q;
  ks.qby4 = Q >> 2;
  ks.mask = (u32)(P.lwe_q - 1);
  ks.q_ks_f = (double)P.lwe_q;
  ks.Q_f = (double)Q;
  ks.dks = make_decomp(P.lwe_q, P.lwe_logb, P.lwe_d);
  ks.d = P.lwe_d;
  ks.n = P.lwe_n;
  ks.N = P.rlwe_n;
  ks.ksk_stride = ks_stride(P);
  ks.out_stride = ks_stride(P);
  *out = c;
  return PZ_OK;
}

void pz_ctx_destroy(pz_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->d_tw); cudaFree(c->d_dlog); cudaFree(c->d_tv); cudaFree(c->d_err);
  cudaFree(c->d_c0); cudaFree(c->d_c1); cudaFree(c->d_out); cudaFree(c->d_gates); cudaFree(c->d_ks);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

const char *pz_last_error(const pz_ctx *c) { return c ? c->err.c_str() : "no context"; }

pz_status pz_ctx_device_error(pz_ctx *c, uint32_t *bits) {
  if (!c || !bits) return PZ_ERR_INVALID_ARGUMENT;
  PZ_CK(c, cudaSetDevice(c->device));
  PZ_CK(c, cudaDeviceSynchronize());
  u32 v = 0;
  PZ_CK(c, cudaMemcpy(&v, c->d_err, sizeof v, cudaMemcpyDeviceToHost));
  if (v) PZ_CK(c, cudaMemset(c->d_err, 0, sizeof v));
  *bits = v;
  return PZ_OK;
}

pz_status pz_ctx_params(const pz_ctx *c, pz_params *out) {
  if (!c || !out) return PZ_ERR_INVALID_ARGUMENT;
  *out = c->P;
  return PZ_OK;
}
uint64_t pz_ctx_ntt_root(const pz_ctx *c) { return c ? c->root : 0; }

pz_status pz_ctx_set_pbs_variant(pz_ctx *c, int v) {
  if (!c || v < 0 || v > pz::PBS_MAX_VARIANT) return PZ_ERR_INVALID_ARGUMENT;
  for (auto &t : c->tuned) t.variant = -1;
  c->pbs_variant = v;
  return PZ_OK;
}
pz_status pz_ctx_set_split_threshold(pz_ctx *c, int max_gates) {
  if (!c || max_gates < -1) return PZ_ERR_INVALID_ARGUMENT;
  c->split_below = max_gates;
  return PZ_OK;
}
int pz_ctx_pbs_variant(const pz_ctx *c) { return c ? c->pbs_variant : -1; }

pz_status pz_ctx_set_pbs_grid_limit(pz_ctx *c, int g) {
  if (!c || g < 0) return PZ_ERR_INVALID_ARGUMENT;
  c->grid_limit = g;
  return PZ_OK;
}

pz_status pz_key_upload(pz_ctx *c, const pz_server_key_view *v, pz_key **out) {
  if (!c || !v || !out || !v->rgsw || !v->autos || !v->lwe_ksk)
    return fail(c, PZ_ERR_INVALID_ARGUMENT, "pz_key_upload: NULL argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lock(c->mu);
  PZ_CK(c, cudaSetDevice(c->device));
  const pz_params &P = c->P;
  const size_t N = P.rlwe_n;
  const size_t rgsw_polys = (size_t)P.lwe_n * P.rgsw_rows;
  const size_t auto_polys = (size_t)P.n_auto_keys * P.auto_rows;
  const size_t ksk_rows = (size_t)P.lwe_d * N;
  const u32 stride = ks_stride(P);
  pz_key *k = new pz_key();
  k->ctx = c;
  auto cleanup = [&](pz_status s, const std::string &m) {
    pz::free_key_arrays(k);
    delete k;
    return fail(c, s, m);
  };
  cudaError_t e;
  if ((e = cudaMalloc(&k->d_rgsw, rgsw_polys * N * 8)) != cudaSuccess) return cleanup(PZ_ERR_OUT_OF_MEMORY, "rgsw alloc");
  if ((e = cudaMalloc(&k->d_autos, auto_polys * N * 8)) != cudaSuccess) return cleanup(PZ_ERR_OUT_OF_MEMORY, "auto alloc");
  if ((e = cudaMalloc(&k->d_ksk, ksk_rows * stride * 4)) != cudaSuccess) return cleanup(PZ_ERR_OUT_OF_MEMORY, "ksk alloc");
  k->bytes = (rgsw_polys + auto_polys) * N * 8 + ksk_rows * stride * 4;
  // coefficient rows -> device staging -> forward NTT + key form (br_conv_c) + device layout
  const size_t chunk = 1024;  // polynomials per staging copy
  u64 *d_stage = nullptr;
  if ((e = cudaMalloc(&d_stage, chunk * N * 8)) != cudaSuccess) return cleanup(PZ_ERR_OUT_OF_MEMORY, "staging alloc");
  auto convert = [&](const u64 *src, u64 *dst, size_t polys) -> cudaError_t {
    for (size_t p0 = 0; p0 < polys; p0 += chunk) {
      size_t m = std::min(chunk, polys - p0);
      cudaError_t e2 = cudaMemcpyAsync(d_stage, src + p0 * N, m * N * 8, cudaMemcpyHostToDevice, c->stream);
      if (e2 != cudaSuccess) return e2;
      e2 = pz::launch_key_convert((int)c->logn, d_stage, dst + p0 * N, m, c->rc, c->br_conv_c, c->br_conv_cs,
                                    c->stream);
      if (e2 != cudaSuccess) return e2;
      e2 = cudaStreamSynchronize(c->stream);
      if (e2 != cudaSuccess) return e2;
    }
    return cudaSuccess;
  };
  if ((e = convert(v->rgsw, k->d_rgsw, rgsw_polys)) != cudaSuccess ||
      (e = convert(v->autos, k->d_autos, auto_polys)) != cudaSuccess) {
    cudaFree(d_stage);
    return cleanup(PZ_ERR_CUDA, std::string("key conversion: ") + cudaGetErrorString(e));
  }
  cudaFree(d_stage);
  // LWE KSK: u64 rows mod q_ks -> u32 rows padded to `stride` words
  std::vector<u32> ksk32((size_t)ksk_rows * stride, 0);
  const size_t cols = P.lwe_n + 1;
  for (size_t r = 0; r < ksk_rows; r++)
    for (size_t col = 0; col < cols; col++) ksk32[r * stride + col] = (u32)(v->lwe_ksk[r * cols + col] & (P.lwe_q - 1));
  if ((e = cudaMemcpy(k->d_ksk, ksk32.data(), ksk32.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess)
    return cleanup(PZ_ERR_CUDA, std::string("ksk copy: ") + cudaGetErrorString(e));
  pz::build_ksk8(c, k, c->stream);
  *out = k;
  return PZ_OK;
}

pz_status pz_key_upload_seeded(pz_ctx *c, const pz_seeded_server_key_view *v, pz_key **out) {
  if (!c || !v || !out || !v->rgsw || !v->auto_b || !v->lwe_ksk_b)
    return fail(c, PZ_ERR_INVALID_ARGUMENT, "pz_key_upload_seeded: NULL argument");
  *out = nullptr;
  std::lock_guard<std::mutex> lock(c->mu);
  PZ_CK(c, cudaSetDevice(c->device));
  const pz_params &P = c->P;
  const size_t N = P.rlwe_n;
  const size_t rgsw_polys = (size_t)P.lwe_n * P.rgsw_rows;
  const size_t auto_polys = (size_t)P.n_auto_keys * P.auto_rows, d_auto = P.auto_d;
  const size_t ksk_rows = (size_t)P.lwe_d * N;
  const u32 stride = ks_stride(P);
  pz_key *k = new pz_key();
  k->ctx = c;
  u64 *d_stage = nullptr;
  auto cleanup = [&](pz_status s, const std::string &m) {
    cudaFree(d_stage);
    pz::free_key_arrays(k);
    delete k;
    return fail(c, s, m);
  };
  cudaError_t e;
  const size_t chunk = 1024;  // polynomials per staging copy (>= the auto keys)
  if ((e = cudaMalloc(&k->d_rgsw, rgsw_polys * N * 8)) != cudaSuccess) return cleanup(PZ_ERR_OUT_OF_MEMORY, "rgsw alloc");
  if ((e = cudaMalloc(&k->d_autos, auto_polys * N * 8)) != cudaSuccess) return cleanup(PZ_ERR_OUT_OF_MEMORY, "auto alloc");
  if ((e = cudaMalloc(&k->d_ksk, ksk_rows * stride * 4)) != cudaSuccess) return cleanup(PZ_ERR_OUT_OF_MEMORY, "ksk alloc");
  if ((e = cudaMalloc(&d_stage, std::max(chunk, auto_polys) * N * 8)) != cudaSuccess)
    return cleanup(PZ_ERR_OUT_OF_MEMORY, "staging alloc");
  k->bytes = (rgsw_polys + auto_polys) * N * 8 + ksk_rows * stride * 4;
  // RGSW ciphertexts: as pz_key_upload (keys.rs:738-757)
  for (size_t p0 = 0; p0 < rgsw_polys; p0 += chunk) {
    const size_t m = std::min(chunk, rgsw_polys - p0);
    if ((e = cudaMemcpyAsync(d_stage, v->rgsw + p0 * N, m * N * 8, cudaMemcpyDefault, c->stream)) != cudaSuccess ||
        (e = pz::launch_key_convert((int)c->logn, d_stage, k->d_rgsw + p0 * N, m, c->rc, c->br_conv_c, c->br_conv_cs,
                                    c->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(c->stream)) != cudaSuccess)
      return cleanup(PZ_ERR_CUDA, std::string("rgsw conversion: ") + cudaGetErrorString(e));
  }
  // auto keys (keys.rs:702-736): per slot d_auto A rows from the auto stream, then the B rows
  pz_status st = pz::seeded_fill_u64(c, v->auto_seed, P.rlwe_q, (u64)P.n_auto_keys * d_auto * N, d_auto * N,
                                     2 * d_auto * N, 0, d_stage, c->stream);
  if (st != PZ_OK) return cleanup(st, c->err);
  if ((e = cudaMemcpy2DAsync(d_stage + d_auto * N, 2 * d_auto * N * 8, v->auto_b, d_auto * N * 8, d_auto * N * 8,
                             P.n_auto_keys, cudaMemcpyDefault, c->stream)) != cudaSuccess ||
      (e = pz::launch_key_convert((int)c->logn, d_stage, k->d_autos, auto_polys, c->rc, c->br_conv_c, c->br_conv_cs,
                                  c->stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(c->stream)) != cudaSuccess)
    return cleanup(PZ_ERR_CUDA, std::string("auto key expansion: ") + cudaGetErrorString(e));
  // LWE KSK (keys.rs:759-772): per row n A words mod q_ks from the ksk stream, word 0 = b
  if ((e = cudaMemsetAsync(k->d_ksk, 0, ksk_rows * stride * 4, c->stream)) != cudaSuccess)
    return cleanup(PZ_ERR_CUDA, "ksk memset");
  st = pz::seeded_fill_u32(c, v->lwe_ksk_seed, P.lwe_q, (u64)ksk_rows * P.lwe_n, P.lwe_n, stride, 1, k->d_ksk,
                           c->stream);
  if (st != PZ_OK) return cleanup(st, c->err);
  std::vector<u64> b64(ksk_rows);  // host or device source
  if ((e = cudaMemcpy(b64.data(), v->lwe_ksk_b, ksk_rows * 8, cudaMemcpyDefault)) != cudaSuccess)
    return cleanup(PZ_ERR_CUDA, std::string("ksk b column: ") + cudaGetErrorString(e));
  std::vector<u32> b32(ksk_rows);
  for (size_t r = 0; r < ksk_rows; r++) b32[r] = (u32)(b64[r] & (P.lwe_q - 1));
  if ((e = cudaMemcpy2DAsync(k->d_ksk, stride * 4, b32.data(), 4, 4, ksk_rows, cudaMemcpyHostToDevice, c->stream)) !=
          cudaSuccess ||
      (e = cudaStreamSynchronize(c->stream)) != cudaSuccess)
    return cleanup(PZ_ERR_CUDA, std::string("ksk b column: ") + cudaGetErrorString(e));
  cudaFree(d_stage);
  d_stage = nullptr;
  pz::build_ksk8(c, k, c->stream);
  *out = k;
  return PZ_OK;
}

void pz_key_release(pz_key *k) {
  if (!k) return;
  cudaSetDevice(k->ctx->device);
  pz::free_key_arrays(k);
  delete k;
}
size_t pz_key_device_bytes(const pz_key *k) { return k ? k->bytes : 0; }

pz_status pz_gate_batch(pz_ctx *c, const pz_key *k, const uint8_t *gates, const uint64_t *c0,
                        const uint64_t *c1, uint64_t *out, size_t count) {
  if (!c) return PZ_ERR_INVALID_ARGUMENT;
  if (count == 0) return PZ_OK;
  if (!gates || !c0 || !c1 || !out) return fail(c, PZ_ERR_INVALID_ARGUMENT, "pz_gate_batch: NULL buffer");
  pz_status s = check_key(c, k);
  if (s != PZ_OK) return s;
  if ((s = check_gates_host(c, gates, count, false)) != PZ_OK) return s;
  std::lock_guard<std::mutex> lock(c->mu);
  PZ_CK(c, cudaSetDevice(c->device));
  if ((s = ensure_scratch(c, count)) != PZ_OK) return s;
  const size_t bytes = count * ((size_t)c->P.rlwe_n + 1) * 8;
  PZ_CK(c, cudaMemcpyAsync(c->d_gates, gates, count, cudaMemcpyHostToDevice, c->stream));
  PZ_CK(c, cudaMemcpyAsync(c->d_c0, c0, bytes, cudaMemcpyHostToDevice, c->stream));
  PZ_CK(c, cudaMemcpyAsync(c->d_c1, c1, bytes, cudaMemcpyHostToDevice, c->stream));
  if ((s = run_gates(c, k, c->d_gates, c->d_c0, c->d_c1, c->d_out, count, nullptr, nullptr, c->stream, c->d_ks,
                     false)) != PZ_OK)
    return s;
  PZ_CK(c, cudaMemcpyAsync(out, c->d_out, bytes, cudaMemcpyDeviceToHost, c->stream));
  PZ_CK(c, cudaStreamSynchronize(c->stream));
  return PZ_OK;
}

static pz_status gate_device_common(pz_ctx *c, const pz_key *k, const uint8_t *d_gates, const uint64_t *d_c0,
                                    const uint64_t *d_c1, uint64_t *d_out, size_t count, uint32_t *d_ks_out,
                                    uint64_t *d_rlwe, void *stream, bool raw) {
  if (!c) return PZ_ERR_INVALID_ARGUMENT;
  if (count == 0) return PZ_OK;
  if (!d_gates || !d_c0 || !d_out) return fail(c, PZ_ERR_INVALID_ARGUMENT, "NULL device buffer");
  pz_status s = check_key(c, k);
  if (s != PZ_OK) return s;
  PZ_CK(c, cudaSetDevice(c->device));
  cudaStream_t st = pick(c, stream);
  u32 *d_ks = nullptr;
  if (!d_ks_out) PZ_CK(c, cudaMallocAsync(&d_ks, count * ks_stride(c->P) * 4, st));
  s = run_gates(c, k, d_gates, d_c0, d_c1, d_out, count, d_ks_out, d_rlwe, st, d_ks, raw);
  if (d_ks) cudaFreeAsync(d_ks, st);
  return s;
}

pz_status pz_gate_batch_device(pz_ctx *c, const pz_key *k, const uint8_t *d_gates, const uint64_t *d_c0,
                               const uint64_t *d_c1, uint64_t *d_out, size_t count, void *stream) {
  if (c && count && !d_c1) return fail(c, PZ_ERR_INVALID_ARGUMENT, "NULL c1");
  return gate_device_common(c, k, d_gates, d_c0, d_c1, d_out, count, nullptr, nullptr, stream, false);
}

pz_status pz_gate_batch_debug_device(pz_ctx *c, const pz_key *k, const uint8_t *d_gates, const uint64_t *d_c0,
                                     const uint64_t *d_c1, uint64_t *d_out, size_t count, uint32_t *d_ks_out,
                                     uint64_t *d_rlwe_out, void *stream) {
  if (c && count && !d_c1) return fail(c, PZ_ERR_INVALID_ARGUMENT, "NULL c1");
  return gate_device_common(c, k, d_gates, d_c0, d_c1, d_out, count, d_ks_out, d_rlwe_out, stream, false);
}

pz_status pz_pbs_batch_device(pz_ctx *c, const pz_key *k, const uint8_t *d_test_vec, const uint64_t *d_lwe,
                              uint64_t *d_out, size_t count, void *stream) {
  return gate_device_common(c, k, d_test_vec, d_lwe, nullptr, d_out, count, nullptr, nullptr, stream, true);
}

pz_status pz_blind_rotate_batch_device(pz_ctx *c, const pz_key *k, const uint32_t *d_ks, const uint8_t *d_test_vec,
                                       uint64_t *d_out, size_t count, void *stream) {
  if (!c) return PZ_ERR_INVALID_ARGUMENT;
  if (count == 0) return PZ_OK;
  if (!d_ks || !d_test_vec || !d_out) return fail(c, PZ_ERR_INVALID_ARGUMENT, "NULL device buffer");
  pz_status s = check_key(c, k);
  if (s != PZ_OK) return s;
  PZ_CK(c, cudaSetDevice(c->device));
  pz::BrParams br = c->br;
  br.rgsw = k->d_rgsw;
  br.autos = k->d_autos;
  br.out_idx = nullptr;
  const bool d1 = c->P.rlrg_d_a == 1 && c->P.rlrg_d_b == 1 && c->P.auto_d == 1;
  PZ_CK(c, pz::launch_pbs((int)c->logn, d1, br, d_ks, c->P.lwe_n + 1, d_test_vec, d_out, count, nullptr,
                          c->grid_limit, pick(c, stream), pz::effective_variant(c, count)));
  return PZ_OK;
}

pz_status pz_ctx_autotune(pz_ctx *c, const pz_key *k, size_t batch, int *variant, double *ms) {
  if (!c || batch == 0) return PZ_ERR_INVALID_ARGUMENT;
  pz_status s = check_key(c, k);
  if (s != PZ_OK) return s;
  std::lock_guard<std::mutex> lock(c->mu);
  PZ_CK(c, cudaSetDevice(c->device));
  const bool d1 = c->P.rlrg_d_a == 1 && c->P.rlrg_d_b == 1 && c->P.auto_d == 1;
  const int nv = (c->logn == 11 && d1) ? pz::PBS_MAX_VARIANT + 1 : 1;
  // synthetic key-switched LWEs, uniform mod q_ks, and gate codes
  const u32 cols = c->P.lwe_n + 1;
  std::vector<u32> ks(batch * cols);
  std::vector<unsigned char> g(batch);
  u64 st = 0x9E3779B97F4A7C15ull;
  for (auto &v : ks) { st ^= st << 13; st ^= st >> 7; st ^= st << 17; v = (u32)(st % c->P.lwe_q); }
  for (size_t i = 0; i < batch; i++) g[i] = (unsigned char)(i % 6);
  u32 *d_ks = nullptr;
  unsigned char *d_g = nullptr;
  u64 *d_out = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  cudaError_t e = cudaMalloc(&d_ks, ks.size() * 4);
  if (e == cudaSuccess) e = cudaMalloc(&d_g, batch);
  if (e == cudaSuccess) e = cudaMalloc(&d_out, batch * (c->P.rlwe_n + 1) * 8);
  if (e == cudaSuccess) e = cudaMemcpy(d_ks, ks.data(), ks.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_g, g.data(), batch, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaEventCreate(&a);
  if (e == cudaSuccess) e = cudaEventCreate(&b);
  pz::BrParams br = c->br;
  br.rgsw = k->d_rgsw;
  br.autos = k->d_autos;
  br.out_idx = nullptr;
  double best = 1e30;
  int bv = c->pbs_variant;
  for (int v = 0; v < nv && e == cudaSuccess; v++) {
    // a batch of at least one wave is timed in whole waves of this shape (a
    // partial last wave would charge the shape for the batch's remainder):
    // the largest multiple of the shape's resident items not above the batch
    size_t slots = 1, items = batch;
    if ((e = pz::pbs_slots((int)c->logn, d1, c->P.br_q, c->P.lwe_n, v, &slots)) != cudaSuccess) break;
    if (batch >= slots) items = batch / slots * slots;
    auto launch = [&]() {
      return pz::launch_pbs((int)c->logn, d1, br, d_ks, cols, d_g, d_out, items, nullptr, c->grid_limit, c->stream, v);
    };
    if ((e = launch()) != cudaSuccess) break;  // warm-up
    if ((e = cudaEventRecord(a, c->stream)) != cudaSuccess) break;
    for (int r = 0; r < 2 && e == cudaSuccess; r++) e = launch();
    if (e == cudaSuccess) e = cudaEventRecord(b, c->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    float t = 0;
    if (e == cudaSuccess) cudaEventElapsedTime(&t, a, b);
    const double per_batch = t / 2.0 / (double)items * (double)batch;
    if (e == cudaSuccess && per_batch < best) {
      best = per_batch;
      bv = v;
    }
  }
  // key-switch tile: ciphertexts per CTA, timed on `batch` uniform inputs
  int bct = c->ks_ct;
  u64 *d_c01 = nullptr;
  const size_t L = (size_t)c->P.rlwe_n + 1;
  if (e == cudaSuccess) e = cudaMalloc(&d_c01, 2 * batch * L * 8);
  if (e == cudaSuccess) {
    std::vector<u64> c01(2 * batch * L);
    for (auto &v : c01) { st ^= st << 13; st ^= st >> 7; st ^= st << 17; v = st % c->P.rlwe_q; }
    e = cudaMemcpy(d_c01, c01.data(), c01.size() * 8, cudaMemcpyHostToDevice);
  }
  pz::KsParams ksp = c->ks;
  pz::ks_bind_key(c, k, ksp);
  ksp.raw = 0;
  ksp.out_stride = cols;
  double best_ks = 1e30;
  for (int ct : {8, 16, 32, pz::KS_CT_MMA}) {
    if (e != cudaSuccess) break;
    if (ct == pz::KS_CT_MMA && !k->d_ksk8) continue;
    auto launch = [&]() {
      return pz::launch_ks(ksp, d_g, d_c01, d_c01 + batch * L, batch, d_ks, c->stream, false, ct);
    };
    if ((e = launch()) != cudaSuccess) break;
    if ((e = cudaEventRecord(a, c->stream)) != cudaSuccess) break;
    for (int r = 0; r < 3 && e == cudaSuccess; r++) e = launch();
    if (e == cudaSuccess) e = cudaEventRecord(b, c->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    float t = 0;
    if (e == cudaSuccess) cudaEventElapsedTime(&t, a, b);
    if (e == cudaSuccess && t / 3 < best_ks) {
      best_ks = t / 3;
      bct = ct;
    }
  }
  cudaFree(d_c01);
  cudaFree(d_ks);
  cudaFree(d_g);
  cudaFree(d_out);
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (e != cudaSuccess) return cuda_fail(c, "pz_ctx_autotune", e);
  c->pbs_variant = bv;
  c->ks_ct = bct;
  c->tuned[pz::size_bucket(batch)] = pz_ctx::Tuned{bv, bct};
  if (variant) *variant = bv;
  if (ms) *ms = best;
  return PZ_OK;
}

pz_status pz_ctx_set_ks_tile(pz_ctx *c, int ciphertexts) {
  if (!c || (ciphertexts != 8 && ciphertexts != 16 && ciphertexts != 32 && ciphertexts != pz::KS_CT_MMA))
    return PZ_ERR_INVALID_ARGUMENT;
  c->ks_ct = ciphertexts;
  for (auto &t : c->tuned) t = pz_ctx::Tuned{};
  return PZ_OK;
}

pz_status pz_ctx_launch_shape(pz_ctx *c, size_t gates, int *variant, int *ks_tile) {
  if (!c) return PZ_ERR_INVALID_ARGUMENT;
  if (variant) *variant = pz::effective_variant(c, gates);
  if (ks_tile) *ks_tile = pz::effective_ks_ct(c, gates);
  return PZ_OK;
}

const char *pz_kernel_revision(void) { return pz::BR_KERNEL_REVISION; }

pz_status pz_ctx_pbs_slots(pz_ctx *c, int variant, size_t *slots) {
  if (!c || !slots) return PZ_ERR_INVALID_ARGUMENT;
  if (variant < 0) variant = c->pbs_variant;
  if (variant > pz::PBS_MAX_VARIANT) return fail(c, PZ_ERR_INVALID_ARGUMENT, "unknown launch shape");
  PZ_CK(c, cudaSetDevice(c->device));
  const bool d1 = c->P.rlrg_d_a == 1 && c->P.rlrg_d_b == 1 && c->P.auto_d == 1;
  PZ_CK(c, pz::pbs_slots((int)c->logn, d1, c->P.br_q, c->P.lwe_n, variant, slots));
  return PZ_OK;
}

pz_status pz_probe_imad_rate(int device, double *imad_per_second) {
  if (!imad_per_second) return PZ_ERR_INVALID_ARGUMENT;
  *imad_per_second = 0;
  if (cudaSetDevice(device) != cudaSuccess) return PZ_ERR_CUDA;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return PZ_ERR_CUDA;
  const int blocks = sms * 8, threads = 256;
  const u32 iters = 2048;
  u32 *sink = nullptr;
  cudaEvent_t e0, e1;
  if (cudaMalloc(&sink, blocks * 4) != cudaSuccess) return PZ_ERR_OUT_OF_MEMORY;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  pz_status st = PZ_OK;
  float best = 1e30f;
  for (int rep = 0; rep < 4 && st == PZ_OK; rep++) {
    cudaEventRecord(e0, 0);
    if (pz::launch_imad_probe(blocks, threads, iters, sink, 0) != cudaSuccess) st = PZ_ERR_CUDA;
    cudaEventRecord(e1, 0);
    if (cudaEventSynchronize(e1) != cudaSuccess) st = PZ_ERR_CUDA;
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;  // first launch is a warm-up
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (st == PZ_OK) *imad_per_second = (double)blocks * threads * iters * 16 * 8 / (best * 1e-3);
  return st;
}

pz_status pz_probe_pipe_rates(int device, double *rates, size_t n) {
  if (!rates) return PZ_ERR_INVALID_ARGUMENT;
  for (size_t i = 0; i < n; i++) rates[i] = 0;
  if (cudaSetDevice(device) != cudaSuccess) return PZ_ERR_CUDA;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return PZ_ERR_CUDA;
  const int blocks = sms * 8, threads = 256;
  const u32 iters = 1024;
  u32 *sink = nullptr;
  if (cudaMalloc(&sink, blocks * 4) != cudaSuccess) return PZ_ERR_OUT_OF_MEMORY;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  pz_status st = PZ_OK;
  for (size_t kind = 0; kind < n && kind < PZ_PIPE_PROBES && st == PZ_OK; kind++) {
    float best = 1e30f;
    for (int rep = 0; rep < 3 && st == PZ_OK; rep++) {
      cudaEventRecord(e0, 0);
      if (pz::launch_pipe_probe((int)kind, blocks, threads, iters, sink, 0) != cudaSuccess) st = PZ_ERR_CUDA;
      cudaEventRecord(e1, 0);
      if (cudaEventSynchronize(e1) != cudaSuccess) st = PZ_ERR_CUDA;
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0 && ms < best) best = ms;  // first launch is a warm-up
    }
    if (st == PZ_OK) rates[kind] = (double)blocks * threads * iters * 16 * 8 / (best * 1e-3);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  return st;
}

pz_status pz_not_batch_device(pz_ctx *c, const uint64_t *d_in, uint64_t *d_out, size_t words, void *stream) {
  if (!c) return PZ_ERR_INVALID_ARGUMENT;
  if (words == 0) return PZ_OK;
  if (!d_in || !d_out) return fail(c, PZ_ERR_INVALID_ARGUMENT, "NULL device buffer");
  PZ_CK(c, cudaSetDevice(c->device));
  PZ_CK(c, pz::launch_not(d_in, d_out, words, c->P.rlwe_q, pick(c, stream)));
  return PZ_OK;
}

pz_status pz_ntt_forward_device(pz_ctx *c, uint64_t *d, size_t count, void *stream) {
  if (!c || (count && !d)) return fail(c, PZ_ERR_INVALID_ARGUMENT, "NULL argument");
  PZ_CK(c, cudaSetDevice(c->device));
  PZ_CK(c, pz::launch_ntt_fwd((int)c->logn, d, count, c->rc, c->d_err, pick(c, stream)));
  return PZ_OK;
}

pz_status pz_ntt_backward_device(pz_ctx *c, uint64_t *d, size_t count, void *stream) {
  if (!c || (count && !d)) return fail(c, PZ_ERR_INVALID_ARGUMENT, "NULL argument");
  PZ_CK(c, cudaSetDevice(c->device));
  PZ_CK(c, pz::launch_ntt_inv((int)c->logn, d, count, c->rc, c->d_err, pick(c, stream)));
  return PZ_OK;
}

pz_status pz_rlwe_by_rgsw_device(pz_ctx *c, const pz_key *k, uint64_t *d_rlwe, const uint32_t *d_idx, size_t count,
                                 int trivial, void *stream) {
  if (!c || (count && (!d_rlwe || !d_idx))) return fail(c, PZ_ERR_INVALID_ARGUMENT, "NULL argument");
  pz_status s = check_key(c, k);
  if (s != PZ_OK) return s;
  PZ_CK(c, cudaSetDevice(c->device));
  pz::BrParams br = c->br;
  br.rgsw = k->d_rgsw;
  br.autos = k->d_autos;
  const bool d1 = c->P.rlrg_d_a == 1 && c->P.rlrg_d_b == 1 && c->P.auto_d == 1;
  PZ_CK(c, pz::launch_ext_product((int)c->logn, d1, br, d_rlwe, d_idx, count, trivial, pick(c, stream),
                                  c->pbs_variant));
  return PZ_OK;
}

pz_status pz_rlwe_auto_device(pz_ctx *c, const pz_key *k, uint64_t *d_rlwe, const uint32_t *d_slot, size_t count,
                              int trivial, void *stream) {
  if (!c || (count && (!d_rlwe || !d_slot))) return fail(c, PZ_ERR_INVALID_ARGUMENT, "NULL argument");
  pz_status s = check_key(c, k);
  if (s != PZ_OK) return s;
  PZ_CK(c, cudaSetDevice(c->device));
  pz::BrParams br = c->br;
  br.rgsw = k->d_rgsw;
  br.autos = k->d_autos;
  const bool d1 = c->P.rlrg_d_a == 1 && c->P.rlrg_d_b == 1 && c->P.auto_d == 1;
  PZ_CK(c, pz::launch_auto((int)c->logn, d1, br, d_rlwe, d_slot, count, trivial, pick(c, stream), c->pbs_variant));
  return PZ_OK;
}

pz_status pz_lwe_key_switch_device(pz_ctx *c, const pz_key *k, const uint64_t *d_in, uint32_t *d_out, size_t count,
                                   void *stream) {
  if (!c || (count && (!d_in || !d_out))) return fail(c, PZ_ERR_INVALID_ARGUMENT, "NULL argument");
  pz_status s = check_key(c, k);
  if (s != PZ_OK) return s;
  if (count == 0) return PZ_OK;
  PZ_CK(c, cudaSetDevice(c->device));
  cudaStream_t st = pick(c, stream);
  // raw inputs already mod q_ks: the mod-down step must be the identity, so
  // run the key-switch kernel with Q = q_ks and gate code GATE_RAW.
  pz::KsParams ks = c->ks;
  pz::ks_bind_key(c, k, ks);
  ks.Q = c->P.lwe_q;
  ks.Q_f = (double)c->P.lwe_q;
  ks.out_stride = c->P.lwe_n + 1;
  ks.raw = 1;
  cudaError_t e = pz::launch_ks(ks, nullptr, d_in, nullptr, count, d_out, st, true, pz::effective_ks_ct(c, count));
  if (e != cudaSuccess) return cuda_fail(c, "launch_ks", e);
  return PZ_OK;
}

}  // extern "C"
