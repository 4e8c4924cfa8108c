// pz_wire.cu -- wire formats (the reference has none): device-form server
// keys and circuits as flat byte strings, for checkpoint / restore and for
// handing work between processes of a serving deployment.
//
// Key blob: a 64-byte header followed by the device-form arrays exactly as
// they sit in device memory (RGSW and auto keys in the evaluation domain,
// scaled by the context's key-form constant -- N^{-1}, or N^{-1} 2^64 for
// Montgomery products -- in the per-thread layout; the LWE KSK as u32 rows
// of ks_stride words).  The evaluation domain depends on the NTT root and
// the scale on the build's multiply-accumulate reduction, so the header
// (version 2) records both and an import into a context with another root,
// key form or parameter set is refused.  Import is a plain copy: no forward
// NTT, no conversion.
//
// (The circuit blob lives with the circuit in pz_circuit.cu.)
#include <cstring>
#include <vector>

#include "pz_internal.h"

using pz::u32;
using pz::u64;

namespace {

constexpr u64 KEY_MAGIC = 0x31305945594b5a50ull;  // "PZKEY01"

struct KeyHeader {
  u64 magic;
  u32 version, param_id;
  u64 root;
  u64 rgsw_bytes, autos_bytes, ksk_bytes;
  u64 key_form;  // the scale of the RGSW and auto key rows (br_conv_c)
  u64 reserved;
};
static_assert(sizeof(KeyHeader) == 64, "key header is 64 bytes");

void key_sizes(const pz_ctx *c, size_t *rgsw, size_t *autos, size_t *ksk) {
  const pz_params &P = c->P;
  *rgsw = (size_t)P.lwe_n * P.rgsw_rows * P.rlwe_n * 8;
  *autos = (size_t)P.n_auto_keys * P.auto_rows * P.rlwe_n * 8;
  *ksk = (size_t)P.lwe_d * P.rlwe_n * pz::ks_stride(P) * 4;
}

}  // namespace

extern "C" {

pz_status pz_key_export(const pz_key *k, void *buf, size_t capacity, size_t *size) {
  if (!k || !size) return PZ_ERR_INVALID_ARGUMENT;
  pz_ctx *c = k->ctx;
  size_t rg, au, ks;
  key_sizes(c, &rg, &au, &ks);
  const size_t total = sizeof(KeyHeader) + rg + au + ks;
  *size = total;
  if (!buf) return PZ_OK;  // size query
  if (capacity < total) return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "pz_key_export: buffer too small");
  PZ_CK(c, cudaSetDevice(c->device));
  KeyHeader h{};
  h.magic = KEY_MAGIC;
  h.version = 2;
  h.key_form = c->br_conv_c;
  h.param_id = (u32)c->param_id;
  h.root = c->root;
  h.rgsw_bytes = rg;
  h.autos_bytes = au;
  h.ksk_bytes = ks;
  unsigned char *p = (unsigned char *)buf;
  memcpy(p, &h, sizeof h);
  p += sizeof h;
  PZ_CK(c, cudaMemcpy(p, k->d_rgsw, rg, cudaMemcpyDeviceToHost));
  PZ_CK(c, cudaMemcpy(p + rg, k->d_autos, au, cudaMemcpyDeviceToHost));
  PZ_CK(c, cudaMemcpy(p + rg + au, k->d_ksk, ks, cudaMemcpyDeviceToHost));
  return PZ_OK;
}

pz_status pz_key_import(pz_ctx *c, const void *buf, size_t size, pz_key **out) {
  if (!c || !buf || !out) return PZ_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  KeyHeader h;
  if (size < sizeof h) return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "pz_key_import: truncated blob");
  memcpy(&h, buf, sizeof h);
  size_t rg, au, ks;
  key_sizes(c, &rg, &au, &ks);
  if (h.magic != KEY_MAGIC || h.version < 1 || h.version > 2)
    return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "pz_key_import: not a key blob");
  // version 1 blobs carried Montgomery-form rows without recording it
  const u64 form = h.version == 1 ? c->conv_c : h.key_form;
  if (form != c->br_conv_c)
    return pz::fail(c, PZ_ERR_KEY_MISMATCH, "pz_key_import: key rows in another device form (other build)");
  if (h.param_id != (u32)c->param_id) return pz::fail(c, PZ_ERR_KEY_MISMATCH, "pz_key_import: other parameter set");
  if (h.root != c->root) return pz::fail(c, PZ_ERR_KEY_MISMATCH, "pz_key_import: exported under another NTT root");
  if (h.rgsw_bytes != rg || h.autos_bytes != au || h.ksk_bytes != ks || size != sizeof h + rg + au + ks)
    return pz::fail(c, PZ_ERR_INVALID_ARGUMENT, "pz_key_import: sizes do not match the parameter set");
  std::lock_guard<std::mutex> lock(c->mu);
  PZ_CK(c, cudaSetDevice(c->device));
  pz_key *k = new pz_key();
  k->ctx = c;
  k->bytes = rg + au + ks;
  const unsigned char *p = (const unsigned char *)buf + sizeof h;
  cudaError_t e = cudaMalloc(&k->d_rgsw, rg);
  if (e == cudaSuccess) e = cudaMalloc(&k->d_autos, au);
  if (e == cudaSuccess) e = cudaMalloc(&k->d_ksk, ks);
  if (e == cudaSuccess) e = cudaMemcpy(k->d_rgsw, p, rg, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(k->d_autos, p + rg, au, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(k->d_ksk, p + rg + au, ks, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    pz::free_key_arrays(k);
    delete k;
    return pz::cuda_fail(c, "pz_key_import", e);
  }
  pz::build_ksk8(c, k, c->stream);  // derived on the device; the blob carries only the u32 rows
  *out = k;
  return PZ_OK;
}

}  // extern "C"
