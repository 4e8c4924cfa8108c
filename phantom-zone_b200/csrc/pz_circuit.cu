// pz_circuit.cu -- boolean circuits (FheUint8 operations) as gate DAGs, and
// their levelized batched execution on the device.
//
// The builders restate the gate sequences of the reference's shortint
// circuits (shortint/ops.rs:5-356, shortint/mod.rs:42-292) call for call,
// with the same operand order: gate(c0, c1) and gate(c1, c0) give different
// ciphertext words for xor/xnor, so the order is part of bit-exactness.
// Instead of executing each gate when it is issued (the reference's
// BooleanGates calls), a builder records it; compile() assigns every gate to
// its ASAP level, and execution runs each level -- the gates of every
// circuit in the batch at that depth -- as one key-switch launch plus one
// blind-rotation launch over a device buffer holding every wire.
// not() is free: it flips a bit of the wire reference, applied (q - x) when
// the wire is read (evaluator.rs:2247-2250).
#include <algorithm>
#include <cstring>
#include <vector>

#include "pz_internal.h"

using pz::u32;
using pz::u64;

namespace {
constexpr u32 NONE = 0xffffffffu;
}

struct pz_circuit {
  // wire table: an input (kind 0, index) or a gate output (kind 1, gate index)
  std::vector<u32> wire_gate;  // NONE for inputs
  std::vector<u32> wire_input;  // input ordinal or NONE
  struct G {
    unsigned char type;
    u32 a, b;  // wire refs (bit 31 = not)
  };
  std::vector<G> gates;
  std::vector<u32> outputs;  // wire refs
  size_t n_inputs = 0;
  std::string err;
  // compiled schedule (host)
  bool compiled = false;
  // structure version: bumped by every added input, gate or output; the
  // device buffers and a captured graph belong to bound_version
  uint64_t version = 0, bound_version = ~0ull;
  std::vector<size_t> level_off;  // levels + 1 offsets into the per-gate arrays
  std::vector<unsigned char> h_type;
  std::vector<u32> h_in0, h_in1, h_out, h_outref;
  size_t max_width = 0;
  // device state (bound to one context)
  pz_ctx *dev_ctx = nullptr;
  size_t wire_cap = 0;
  u64 *d_wires = nullptr;
  unsigned char *d_type = nullptr;
  u32 *d_in0 = nullptr, *d_in1 = nullptr, *d_out = nullptr, *d_outref = nullptr, *d_ks = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;

  u32 new_wire(u32 gate, u32 input) {
    wire_gate.push_back(gate);
    wire_input.push_back(input);
    touch();
    return (u32)(wire_gate.size() - 1);
  }
  void touch() {
    compiled = false;
    version++;
  }
  bool valid(u32 ref) const { return ref != NONE && (ref & pz::WIRE_MASK) < wire_gate.size(); }
  u32 input() { return new_wire(NONE, (u32)n_inputs++); }
  u32 gate(int t, u32 a, u32 b) {
    if (t < 0 || t > 5 || !valid(a) || !valid(b)) return NONE;
    gates.push_back({(unsigned char)t, a, b});
    return new_wire((u32)(gates.size() - 1), NONE);
  }
  void free_device() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    graph_exec = nullptr;
    graph = nullptr;
    cudaFree(d_wires); cudaFree(d_type); cudaFree(d_in0); cudaFree(d_in1); cudaFree(d_out);
    cudaFree(d_outref); cudaFree(d_ks);
    d_wires = nullptr; d_type = nullptr; d_in0 = d_in1 = d_out = d_outref = d_ks = nullptr;
    wire_cap = 0;
    dev_ctx = nullptr;
    bound_version = ~0ull;
  }
  ~pz_circuit() { free_device(); }
};

namespace {

enum { AND = 0, NAND = 1, OR = 2, NOR = 3, XOR = 4, XNOR = 5 };

struct B {  // terse builder used by the shortint restatements
  pz_circuit *c;
  bool ok = true;
  u32 g(int t, u32 a, u32 b) {
    u32 w = c->gate(t, a, b);
    if (w == NONE) ok = false;
    return w;
  }
  u32 and_(u32 a, u32 b) { return g(AND, a, b); }
  u32 or_(u32 a, u32 b) { return g(OR, a, b); }
  u32 xor_(u32 a, u32 b) { return g(XOR, a, b); }
  u32 xnor_(u32 a, u32 b) { return g(XNOR, a, b); }
  static u32 not_(u32 a) { return a ^ pz::WIRE_NEG; }
};

// ops.rs:5-14 half_adder: a <- a ^ b, returns a & b
u32 half_adder(B &e, u32 &a, u32 b) {
  u32 carry = e.and_(a, b);
  a = e.xor_(a, b);
  return carry;
}
// ops.rs:16-44 full_adder_plain_carry_in
u32 full_adder_plain_carry_in(B &e, u32 &a, u32 b, bool carry_in) {
  u32 a_and_b = e.and_(a, b);
  a = e.xor_(a, b);
  if (carry_in) a_and_b = e.or_(a_and_b, a);
  if (carry_in) a = B::not_(a);
  return a_and_b;
}
// ops.rs:46-59 full_adder
u32 full_adder(B &e, u32 &a, u32 b, u32 carry_in) {
  u32 a_and_b = e.and_(a, b);
  a = e.xor_(a, b);
  u32 a_xor_b_and_c = e.and_(a, carry_in);
  a_and_b = e.or_(a_and_b, a_xor_b_and_c);
  a = e.xor_(a, carry_in);
  return a_and_b;
}
// ops.rs:61-91 arbitrary_bit_adder: a <- a + b, returns (carry_last, carry_last_last)
void arbitrary_bit_adder(B &e, u32 *a, const u32 *b, int n, bool carry_in, u32 &carry_last,
                         u32 &carry_last_last) {
  u32 carry = !carry_in ? half_adder(e, a[0], b[0]) : full_adder_plain_carry_in(e, a[0], b[0], true);
  for (int i = 1; i <= n - 3; i++) carry = full_adder(e, a[i], b[i], carry);
  carry_last_last = full_adder(e, a[n - 2], b[n - 2], carry);
  carry_last = full_adder(e, a[n - 1], b[n - 1], carry_last_last);
}
// ops.rs:93-105 arbitrary_bit_subtractor: out = !b + a + 1
void arbitrary_bit_subtractor(B &e, const u32 *a, const u32 *b, int n, u32 *out, u32 &carry_last,
                              u32 &carry_last_last) {
  for (int i = 0; i < n; i++) out[i] = B::not_(b[i]);
  arbitrary_bit_adder(e, out, a, n, true, carry_last, carry_last_last);
}
// ops.rs:123-141 arbitrary_bit_mux
void arbitrary_bit_mux(B &e, u32 selector, const u32 *if_true, const u32 *if_false, int n, u32 *out) {
  u32 not_selector = B::not_(selector);
  for (int i = 0; i < n; i++) {
    u32 s_and_a = e.and_(selector, if_true[i]);
    u32 s_and_b = e.and_(not_selector, if_false[i]);
    out[i] = e.or_(s_and_a, s_and_b);
  }
}
// ops.rs:143-187 eight_bit_mul
void eight_bit_mul(B &e, const u32 *a, const u32 *b, u32 *out) {
  std::vector<u32> carries;
  for (int i = 0; i < 8; i++) {
    if (i == 0) {
      out[0] = e.and_(a[0], b[0]);
    } else if (i == 1) {
      u32 tmp0 = e.and_(a[1], b[0]);
      u32 tmp1 = e.and_(a[0], b[1]);
      u32 carry = half_adder(e, tmp0, tmp1);
      carries.push_back(carry);
      out[1] = tmp0;
    } else {
      u32 sum = e.and_(a[i], b[0]);
      u32 tmp = e.and_(a[i - 1], b[1]);
      carries[0] = full_adder(e, sum, tmp, carries[0]);
      for (int j = 2; j < i; j++) {
        tmp = e.and_(a[i - j], b[j]);
        carries[j - 1] = full_adder(e, sum, tmp, carries[j - 1]);
      }
      tmp = e.and_(a[0], b[i]);
      u32 carry = half_adder(e, sum, tmp);
      carries.push_back(carry);
      out[i] = sum;
    }
  }
}
// ops.rs:189-259 arbitrary_bit_division_for_quotient_and_rem (restoring division)
void division(B &e, const u32 *a, const u32 *b, int n, u32 *quotient_out, u32 *remainder_out) {
  std::vector<u32> neg_b(n), remainder, quotient;
  for (int i = 0; i < n; i++) neg_b[i] = B::not_(b[i]);
  for (int i = 0; i < n; i++) {
    remainder.push_back(a[n - 1 - i]);
    std::vector<u32> subtract = remainder;
    u32 carry = full_adder_plain_carry_in(e, subtract[i], neg_b[0], true);
    for (int j = 1; j <= i; j++) carry = full_adder(e, subtract[i - j], neg_b[j], carry);
    for (int j = i + 1; j < n; j++) carry = e.and_(carry, neg_b[j]);
    u32 not_carry = B::not_(carry);
    for (size_t k = 0; k < remainder.size(); k++) {
      u32 s = e.and_(subtract[k], carry);
      u32 r = e.and_(remainder[k], not_carry);
      remainder[k] = e.or_(r, s);
    }
    quotient.push_back(carry);
  }
  std::reverse(remainder.begin(), remainder.end());
  std::reverse(quotient.begin(), quotient.end());
  for (int i = 0; i < n; i++) {
    quotient_out[i] = quotient[i];
    remainder_out[i] = remainder[i];
  }
}
// ops.rs:261-272 is_zero
u32 is_zero(B &e, const u32 *a, int n) {
  u32 out = B::not_(a[0]);
  for (int i = 1; i < n; i++) out = e.and_(out, B::not_(a[i]));
  return out;
}
// ops.rs:274-287 arbitrary_bit_equality
u32 equality(B &e, const u32 *a, const u32 *b, int n) {
  u32 out = e.xnor_(a[0], b[0]);
  for (int i = 1; i < n; i++) {
    u32 x = e.xnor_(a[i], b[i]);
    out = e.and_(out, x);
  }
  return out;
}
// ops.rs:292-321 and :341-356: a > b (unsigned)
u32 comparator(B &e, const u32 *a, const u32 *b, int n) {
  u32 comp = B::not_(b[n - 1]);
  comp = e.and_(comp, a[n - 1]);
  u32 casc = e.xnor_(a[n - 1], b[n - 1]);
  u32 tmp = B::not_(b[n - 2]);
  tmp = e.and_(tmp, a[n - 2]);
  tmp = e.and_(tmp, casc);
  comp = e.or_(comp, tmp);
  for (int i = 2; i < n; i++) {
    u32 tmp_casc = e.xnor_(a[n - i], b[n - i]);
    casc = e.and_(casc, tmp_casc);
    u32 t = B::not_(b[n - 1 - i]);
    t = e.and_(t, a[n - 1 - i]);
    t = e.and_(t, casc);
    comp = e.or_(comp, t);
  }
  return comp;
}

pz_status circ_fail(pz_circuit *c, const char *m) {
  if (c) c->err = m;
  return PZ_ERR_INVALID_ARGUMENT;
}

bool all_valid(pz_circuit *c, const u32 *w, int n) {
  if (!w) return false;
  for (int i = 0; i < n; i++)
    if (!c->valid(w[i])) return false;
  return true;
}

// ASAP levels; per level the gates in issue order.
void compile(pz_circuit *c) {
  if (c->compiled) return;
  const size_t G = c->gates.size();
  std::vector<u32> wlevel(c->wire_gate.size(), 0);
  std::vector<u32> glevel(G, 0);
  std::vector<u32> gate_wire(G, NONE);
  for (size_t w = 0; w < c->wire_gate.size(); w++)
    if (c->wire_gate[w] != NONE) gate_wire[c->wire_gate[w]] = (u32)w;
  // wires are created in issue order and a gate only reads earlier wires
  u32 depth = 0;
  for (size_t w = 0; w < c->wire_gate.size(); w++) {
    u32 g = c->wire_gate[w];
    if (g == NONE) { wlevel[w] = 0; continue; }
    const auto &x = c->gates[g];
    glevel[g] = std::max(wlevel[x.a & pz::WIRE_MASK], wlevel[x.b & pz::WIRE_MASK]) + 1;
    wlevel[w] = glevel[g];
    depth = std::max(depth, glevel[g]);
  }
  // physical slots: inputs first (input order), then gates (issue order)
  std::vector<u32> slot(c->wire_gate.size());
  for (size_t w = 0; w < c->wire_gate.size(); w++)
    slot[w] = c->wire_gate[w] == NONE ? c->wire_input[w] : (u32)(c->n_inputs + c->wire_gate[w]);
  auto phys = [&](u32 ref) { return slot[ref & pz::WIRE_MASK] | (ref & pz::WIRE_NEG); };
  std::vector<size_t> count(depth + 2, 0);
  for (size_t g = 0; g < G; g++) count[glevel[g]]++;
  c->level_off.assign(depth + 1, 0);  // level l (1..depth) -> [off[l-1], off[l])
  size_t acc = 0;
  c->max_width = 0;
  for (u32 l = 1; l <= depth; l++) {
    acc += count[l];
    c->level_off[l] = acc;
    c->max_width = std::max(c->max_width, count[l]);
  }
  c->h_type.assign(G, 0);
  c->h_in0.assign(G, 0);
  c->h_in1.assign(G, 0);
  c->h_out.assign(G, 0);
  std::vector<size_t> fillpos(depth + 1, 0);
  for (u32 l = 1; l <= depth; l++) fillpos[l] = c->level_off[l - 1];
  for (size_t g = 0; g < G; g++) {
    size_t p = fillpos[glevel[g]]++;
    c->h_type[p] = c->gates[g].type;
    c->h_in0[p] = phys(c->gates[g].a);
    c->h_in1[p] = phys(c->gates[g].b);
    c->h_out[p] = slot[gate_wire[g]];
  }
  c->h_outref.resize(c->outputs.size());
  for (size_t i = 0; i < c->outputs.size(); i++) c->h_outref[i] = phys(c->outputs[i]);
  c->compiled = true;
}

__global__ void gather_kernel(const u64 *wires, const u32 *refs, u64 *out, size_t count, size_t L, u64 q) {
  for (size_t i = blockIdx.x; i < count; i += gridDim.x) {
    const u32 r = refs[i];
    const u64 *src = wires + (size_t)(r & pz::WIRE_MASK) * L;
    u64 *dst = out + i * L;
    for (size_t k = threadIdx.x; k < L; k += blockDim.x) {
      const u64 x = src[k];
      dst[k] = (r & pz::WIRE_NEG) ? q - x : x;
    }
  }
}

// Device buffers sized for the circuit as it is now.  A circuit that gained
// inputs, gates or outputs since it was bound is re-uploaded (its old buffers
// and any captured graph are released).
pz_status bind_device(pz_ctx *ctx, pz_circuit *c) {
  compile(c);
  if (c->dev_ctx == ctx && c->d_type && c->bound_version == c->version) return PZ_OK;
  c->free_device();
  const size_t G = c->gates.size(), L = (size_t)ctx->P.rlwe_n + 1;
  const size_t W = c->n_inputs + G;
  PZ_CK(ctx, cudaMalloc(&c->d_wires, std::max<size_t>(W, 1) * L * 8));
  PZ_CK(ctx, cudaMalloc(&c->d_type, std::max<size_t>(G, 1)));
  PZ_CK(ctx, cudaMalloc(&c->d_in0, std::max<size_t>(G, 1) * 4));
  PZ_CK(ctx, cudaMalloc(&c->d_in1, std::max<size_t>(G, 1) * 4));
  PZ_CK(ctx, cudaMalloc(&c->d_out, std::max<size_t>(G, 1) * 4));
  PZ_CK(ctx, cudaMalloc(&c->d_outref, std::max<size_t>(c->outputs.size(), 1) * 4));
  PZ_CK(ctx, cudaMalloc(&c->d_ks, std::max<size_t>(c->max_width, 1) * pz::ks_stride(ctx->P) * 4));
  if (G) {
    PZ_CK(ctx, cudaMemcpy(c->d_type, c->h_type.data(), G, cudaMemcpyHostToDevice));
    PZ_CK(ctx, cudaMemcpy(c->d_in0, c->h_in0.data(), G * 4, cudaMemcpyHostToDevice));
    PZ_CK(ctx, cudaMemcpy(c->d_in1, c->h_in1.data(), G * 4, cudaMemcpyHostToDevice));
    PZ_CK(ctx, cudaMemcpy(c->d_out, c->h_out.data(), G * 4, cudaMemcpyHostToDevice));
  }
  if (!c->outputs.empty())
    PZ_CK(ctx, cudaMemcpy(c->d_outref, c->h_outref.data(), c->outputs.size() * 4, cudaMemcpyHostToDevice));
  c->wire_cap = W;
  c->dev_ctx = ctx;
  c->bound_version = c->version;
  return PZ_OK;
}

// Inputs -> wire slots, every level, outputs <- wires (all on stream s).
pz_status enqueue(pz_ctx *ctx, const pz_key *k, pz_circuit *c, const u64 *d_in, u64 *d_outp, cudaStream_t s) {
  const size_t L = (size_t)ctx->P.rlwe_n + 1;
  if (c->n_inputs) PZ_CK(ctx, cudaMemcpyAsync(c->d_wires, d_in, c->n_inputs * L * 8, cudaMemcpyDeviceToDevice, s));
  for (size_t l = 1; l < c->level_off.size(); l++) {
    const size_t o = c->level_off[l - 1], n = c->level_off[l] - o;
    pz_status st = pz::run_gates(ctx, k, c->d_type + o, c->d_wires, c->d_wires, c->d_wires, n, nullptr, nullptr, s,
                                 c->d_ks, false, c->d_in0 + o, c->d_in1 + o, c->d_out + o);
    if (st != PZ_OK) return st;
  }
  if (!c->outputs.empty()) {
    size_t blocks = std::min<size_t>(c->outputs.size(), 4096);
    gather_kernel<<<(unsigned)blocks, 256, 0, s>>>(c->d_wires, c->d_outref, d_outp, c->outputs.size(), L,
                                                   ctx->P.rlwe_q);
    PZ_CK(ctx, cudaGetLastError());
  }
  return PZ_OK;
}

}  // namespace

namespace pz {
bool circuit_view(pz_circuit *c, CircuitView *v) {
  if (!c || !v) return false;
  compile(c);
  v->n_inputs = c->n_inputs;
  v->n_gates = c->gates.size();
  v->n_outputs = c->outputs.size();
  v->levels = c->level_off.empty() ? 0 : c->level_off.size() - 1;
  v->level_off = c->level_off.data();
  v->type = c->h_type.data();
  v->in0 = c->h_in0.data();
  v->in1 = c->h_in1.data();
  v->out = c->h_out.data();
  v->outref = c->h_outref.data();
  return true;
}

cudaError_t launch_gather(const u64 *wires, const u32 *refs, u64 *out, size_t count, size_t L, u64 q,
                          cudaStream_t s) {
  if (count == 0) return cudaSuccess;
  const size_t blocks = std::min<size_t>(count, 4096);
  gather_kernel<<<(unsigned)blocks, 256, 0, s>>>(wires, refs, out, count, L, q);
  return cudaGetLastError();
}
}  // namespace pz

extern "C" {

pz_status pz_circuit_create(pz_circuit **out) {
  if (!out) return PZ_ERR_INVALID_ARGUMENT;
  *out = new pz_circuit();
  return PZ_OK;
}
void pz_circuit_destroy(pz_circuit *c) { delete c; }
const char *pz_circuit_last_error(const pz_circuit *c) { return c ? c->err.c_str() : "no circuit"; }

uint32_t pz_circuit_input(pz_circuit *c) { return c ? c->input() : NONE; }
uint32_t pz_circuit_gate(pz_circuit *c, int gate, uint32_t a, uint32_t b) { return c ? c->gate(gate, a, b) : NONE; }
uint32_t pz_circuit_not(pz_circuit *c, uint32_t a) { return (c && c->valid(a)) ? (a ^ pz::WIRE_NEG) : NONE; }
pz_status pz_circuit_output(pz_circuit *c, uint32_t w) {
  if (!c || !c->valid(w)) return circ_fail(c, "invalid wire");
  c->outputs.push_back(w);
  c->touch();
  return PZ_OK;
}

pz_status pz_circuit_info(pz_circuit *c, size_t *inputs, size_t *gates, size_t *outputs, size_t *levels,
                          size_t *max_width) {
  if (!c) return PZ_ERR_INVALID_ARGUMENT;
  compile(c);
  if (inputs) *inputs = c->n_inputs;
  if (gates) *gates = c->gates.size();
  if (outputs) *outputs = c->outputs.size();
  if (levels) *levels = c->level_off.empty() ? 0 : c->level_off.size() - 1;
  if (max_width) *max_width = c->max_width;
  return PZ_OK;
}

pz_status pz_circuit_level_sizes(pz_circuit *c, size_t *sizes, size_t cap) {
  if (!c || !sizes) return PZ_ERR_INVALID_ARGUMENT;
  compile(c);
  for (size_t l = 1; l < c->level_off.size() && l - 1 < cap; l++) sizes[l - 1] = c->level_off[l] - c->level_off[l - 1];
  return PZ_OK;
}

// FheUint8 operations -- shortint/mod.rs:63-292 over ops.rs
pz_status pz_u8_add(pz_circuit *c, const uint32_t *a, const uint32_t *b, uint32_t *out, uint32_t *overflow) {
  if (!c || !all_valid(c, a, 8) || !all_valid(c, b, 8) || !out) return circ_fail(c, "pz_u8_add: bad wires");
  B e{c};
  u32 x[8];
  std::copy(a, a + 8, x);
  u32 cl, cll;
  arbitrary_bit_adder(e, x, b, 8, false, cl, cll);
  std::copy(x, x + 8, out);
  if (overflow) *overflow = cl;  // overflowing_add (mod.rs:157-165)
  return e.ok ? PZ_OK : circ_fail(c, "pz_u8_add failed");
}

pz_status pz_u8_sub(pz_circuit *c, const uint32_t *a, const uint32_t *b, uint32_t *out, uint32_t *overflow) {
  if (!c || !all_valid(c, a, 8) || !all_valid(c, b, 8) || !out) return circ_fail(c, "pz_u8_sub: bad wires");
  B e{c};
  u32 cl, cll;
  arbitrary_bit_subtractor(e, a, b, 8, out, cl, cll);
  if (overflow) *overflow = B::not_(cl);  // overflowing_sub (mod.rs:171-179)
  return e.ok ? PZ_OK : circ_fail(c, "pz_u8_sub failed");
}

pz_status pz_u8_mul(pz_circuit *c, const uint32_t *a, const uint32_t *b, uint32_t *out) {
  if (!c || !all_valid(c, a, 8) || !all_valid(c, b, 8) || !out) return circ_fail(c, "pz_u8_mul: bad wires");
  B e{c};
  eight_bit_mul(e, a, b, out);
  return e.ok ? PZ_OK : circ_fail(c, "pz_u8_mul failed");
}

pz_status pz_u8_div_rem(pz_circuit *c, const uint32_t *a, const uint32_t *b, uint32_t *quotient, uint32_t *remainder,
                        uint32_t *div_zero_flag) {
  if (!c || !all_valid(c, a, 8) || !all_valid(c, b, 8) || !quotient || !remainder)
    return circ_fail(c, "pz_u8_div_rem: bad wires");
  B e{c};
  if (div_zero_flag) {  // set_div_by_zero_flag, shortint/mod.rs:42-56
    u32 z = is_zero(e, b, 8);
    *div_zero_flag = (*div_zero_flag == NONE) ? z : e.or_(*div_zero_flag, z);
  }
  division(e, a, b, 8, quotient, remainder);
  return e.ok ? PZ_OK : circ_fail(c, "pz_u8_div_rem failed");
}

// op: 0 eq, 1 neq, 2 lt, 3 gt, 4 le, 5 ge (shortint/mod.rs:214-270)
pz_status pz_u8_cmp(pz_circuit *c, int op, const uint32_t *a, const uint32_t *b, uint32_t *out) {
  if (!c || !all_valid(c, a, 8) || !all_valid(c, b, 8) || !out || op < 0 || op > 5)
    return circ_fail(c, "pz_u8_cmp: bad arguments");
  B e{c};
  switch (op) {
    case 0: *out = equality(e, a, b, 8); break;
    case 1: *out = B::not_(equality(e, a, b, 8)); break;
    case 2: *out = comparator(e, b, a, 8); break;
    case 3: *out = comparator(e, a, b, 8); break;
    case 4: *out = B::not_(comparator(e, a, b, 8)); break;
    case 5: *out = B::not_(comparator(e, b, a, 8)); break;
  }
  return e.ok ? PZ_OK : circ_fail(c, "pz_u8_cmp failed");
}

// mux(self=a, other=b, selector) -> selector ? a : b (shortint/mod.rs:273-279)
pz_status pz_u8_mux(pz_circuit *c, const uint32_t *a, const uint32_t *b, uint32_t selector, uint32_t *out) {
  if (!c || !all_valid(c, a, 8) || !all_valid(c, b, 8) || !c->valid(selector) || !out)
    return circ_fail(c, "pz_u8_mux: bad wires");
  B e{c};
  arbitrary_bit_mux(e, selector, a, b, 8, out);
  return e.ok ? PZ_OK : circ_fail(c, "pz_u8_mux failed");
}

// ---- wire format: header, wire table, gates, outputs (little-endian u32/u64)
namespace {
constexpr uint64_t CIRCUIT_MAGIC = 0x3130434952435a50ull;  // "PZCIRC01"
struct CircuitHeader {
  uint64_t magic;
  uint32_t version, reserved;
  uint64_t n_inputs, n_wires, n_gates, n_outputs;
};
}  // namespace

pz_status pz_circuit_serialize(const pz_circuit *c, void *buf, size_t capacity, size_t *size) {
  if (!c || !size) return PZ_ERR_INVALID_ARGUMENT;
  const size_t W = c->wire_gate.size(), G = c->gates.size(), O = c->outputs.size();
  const size_t total = sizeof(CircuitHeader) + W * 8 + G * 12 + O * 4;
  *size = total;
  if (!buf) return PZ_OK;
  if (capacity < total) return PZ_ERR_INVALID_ARGUMENT;
  CircuitHeader h{CIRCUIT_MAGIC, 1, 0, c->n_inputs, W, G, O};
  unsigned char *p = (unsigned char *)buf;
  memcpy(p, &h, sizeof h);
  p += sizeof h;
  memcpy(p, c->wire_gate.data(), W * 4);
  memcpy(p + W * 4, c->wire_input.data(), W * 4);
  p += W * 8;
  for (size_t g = 0; g < G; g++) {
    const u32 rec[3] = {c->gates[g].type, c->gates[g].a, c->gates[g].b};
    memcpy(p + g * 12, rec, 12);
  }
  p += G * 12;
  memcpy(p, c->outputs.data(), O * 4);
  return PZ_OK;
}

// Rebuilds a circuit from a blob, checking every index (a malformed blob is
// rejected, never read out of bounds).
pz_status pz_circuit_deserialize(const void *buf, size_t size, pz_circuit **out) {
  if (!buf || !out) return PZ_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  CircuitHeader h;
  if (size < sizeof h) return PZ_ERR_INVALID_ARGUMENT;
  memcpy(&h, buf, sizeof h);
  if (h.magic != CIRCUIT_MAGIC || h.version != 1) return PZ_ERR_INVALID_ARGUMENT;
  const uint64_t W = h.n_wires, G = h.n_gates, O = h.n_outputs;
  if (W > (1ull << 31) || G > W || O > (1ull << 31) || h.n_inputs > W) return PZ_ERR_INVALID_ARGUMENT;
  if (size != sizeof h + W * 8 + G * 12 + O * 4) return PZ_ERR_INVALID_ARGUMENT;
  const unsigned char *p = (const unsigned char *)buf + sizeof h;
  std::vector<u32> wg(W), wi(W), outs(O);
  memcpy(wg.data(), p, W * 4);
  memcpy(wi.data(), p + W * 4, W * 4);
  p += W * 8;
  pz_circuit *c = new pz_circuit();
  // replay the creation order: inputs and gates interleaved as recorded
  uint64_t next_gate = 0, next_input = 0;
  bool ok = true;
  for (uint64_t w = 0; w < W && ok; w++) {
    if (wg[w] == NONE) {
      ok = wi[w] == next_input;
      if (ok) { c->input(); next_input++; }
    } else {
      ok = wg[w] == next_gate && next_gate < G;
      if (ok) {
        u32 rec[3];
        memcpy(rec, p + next_gate * 12, 12);
        // operands must be earlier wires (valid() checks the range)
        ok = rec[0] <= 5 && (rec[1] & pz::WIRE_MASK) < w && (rec[2] & pz::WIRE_MASK) < w &&
             c->gate((int)rec[0], rec[1], rec[2]) == (u32)w;
        next_gate++;
      }
    }
  }
  ok = ok && next_gate == G && next_input == h.n_inputs;
  if (ok) {
    memcpy(outs.data(), p + G * 12, O * 4);
    for (uint64_t i = 0; i < O && ok; i++) {
      ok = c->valid(outs[i]);
      if (ok) c->outputs.push_back(outs[i]);
    }
  }
  if (!ok) {
    delete c;
    return PZ_ERR_INVALID_ARGUMENT;
  }
  *out = c;
  return PZ_OK;
}

pz_status pz_circuit_run_device(pz_ctx *ctx, const pz_key *k, pz_circuit *c, const uint64_t *d_inputs,
                                uint64_t *d_outputs, void *stream) {
  if (!ctx || !c) return PZ_ERR_INVALID_ARGUMENT;
  if (!k || k->ctx != ctx) return pz::fail(ctx, PZ_ERR_KEY_MISMATCH, "key does not belong to this context");
  if ((c->n_inputs && !d_inputs) || (!c->outputs.empty() && !d_outputs))
    return pz::fail(ctx, PZ_ERR_INVALID_ARGUMENT, "NULL circuit buffer");
  std::lock_guard<std::mutex> lock(ctx->mu);
  PZ_CK(ctx, cudaSetDevice(ctx->device));
  pz_status s = bind_device(ctx, c);
  if (s != PZ_OK) return s;
  return enqueue(ctx, k, c, d_inputs, d_outputs, (cudaStream_t)stream);
}

pz_status pz_circuit_run(pz_ctx *ctx, const pz_key *k, pz_circuit *c, const uint64_t *inputs, uint64_t *outputs) {
  if (!ctx || !c) return PZ_ERR_INVALID_ARGUMENT;
  if ((c->n_inputs && !inputs) || (!c->outputs.empty() && !outputs))
    return pz::fail(ctx, PZ_ERR_INVALID_ARGUMENT, "NULL circuit buffer");
  std::lock_guard<std::mutex> lock(ctx->mu);
  PZ_CK(ctx, cudaSetDevice(ctx->device));
  pz_status s = bind_device(ctx, c);
  if (s != PZ_OK) return s;
  const size_t L = (size_t)ctx->P.rlwe_n + 1;
  u64 *d_o = nullptr;
  PZ_CK(ctx, cudaMallocAsync(&d_o, std::max<size_t>(c->outputs.size(), 1) * L * 8, ctx->stream));
  // host inputs go straight into the input wire slots
  if (c->n_inputs)
    PZ_CK(ctx, cudaMemcpyAsync(c->d_wires, inputs, c->n_inputs * L * 8, cudaMemcpyHostToDevice, ctx->stream));
  s = enqueue(ctx, k, c, c->d_wires, d_o, ctx->stream);
  if (s == PZ_OK && !c->outputs.empty())
    s = (cudaMemcpyAsync(outputs, d_o, c->outputs.size() * L * 8, cudaMemcpyDeviceToHost, ctx->stream) == cudaSuccess)
            ? PZ_OK
            : pz::fail(ctx, PZ_ERR_CUDA, "output copy failed");
  cudaFreeAsync(d_o, ctx->stream);
  PZ_CK(ctx, cudaStreamSynchronize(ctx->stream));
  return s;
}

// Capture the whole circuit (input copy, every level, output gather) as one
// CUDA graph; pz_circuit_replay_graph then re-runs it with one launch.
pz_status pz_circuit_capture_graph(pz_ctx *ctx, const pz_key *k, pz_circuit *c, const uint64_t *d_inputs,
                                   uint64_t *d_outputs, void *stream) {
  if (!ctx || !c) return PZ_ERR_INVALID_ARGUMENT;
  if (!k || k->ctx != ctx) return pz::fail(ctx, PZ_ERR_KEY_MISMATCH, "key does not belong to this context");
  std::lock_guard<std::mutex> lock(ctx->mu);
  PZ_CK(ctx, cudaSetDevice(ctx->device));
  pz_status s = bind_device(ctx, c);
  if (s != PZ_OK) return s;
  cudaStream_t st = (cudaStream_t)stream;
  cudaStream_t cap = st;
  if (!cap) PZ_CK(ctx, cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  // kernel attributes are set by an uncaptured warm-up launch sequence
  if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
  if (c->graph) { cudaGraphDestroy(c->graph); c->graph = nullptr; }
  cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    if (!st) cudaStreamDestroy(cap);
    return pz::cuda_fail(ctx, "cudaStreamBeginCapture", e);
  }
  s = enqueue(ctx, k, c, d_inputs, d_outputs, cap);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(cap, &g);
  if (!st) cudaStreamDestroy(cap);
  if (s != PZ_OK) { if (g) cudaGraphDestroy(g); return s; }
  if (e != cudaSuccess) return pz::cuda_fail(ctx, "cudaStreamEndCapture", e);
  c->graph = g;
  e = cudaGraphInstantiate(&c->graph_exec, g, 0);
  if (e != cudaSuccess) return pz::cuda_fail(ctx, "cudaGraphInstantiate", e);
  return PZ_OK;
}

pz_status pz_circuit_replay_graph(pz_circuit *c, void *stream) {
  if (!c || !c->graph_exec || !c->dev_ctx) return circ_fail(c, "no captured graph");
  if (c->bound_version != c->version) return circ_fail(c, "circuit changed since its graph was captured");
  cudaError_t e = cudaGraphLaunch(c->graph_exec, (cudaStream_t)stream);
  if (e != cudaSuccess) return pz::cuda_fail(c->dev_ctx, "cudaGraphLaunch", e);
  return PZ_OK;
}

}  // extern "C"
