// pz_server.cu -- multi-session executor: continuous batching of circuits
// from many sessions (each with its own server key, any production parameter
// set) on one device.
//
// The reference evaluates one gate at a time, in the calling thread, against
// the one global server key of that thread's parameter set
// (bool/mp_api.rs:20-26, evaluator.rs:2136-2323).  Here every submitted
// circuit is a job bound to a session (a context + a device-resident server
// key).  A step
//   1. admits pending jobs in arrival order while their wires fit the device
//      arena and their session's server key is resident or can be made
//      resident within the key budget (admission by ciphertext + key bytes):
//      a managed session's key is imported from its device-form blob on
//      demand, evicting the keys of the least recently used sessions that
//      have no job in flight,
//   2. collects the next level of every admitted job, sorts the gates by
//      session and runs them as ONE ragged key-switch launch (tiles of one
//      session each) plus ONE ragged blind-rotation launch (each CTA loads
//      its gate's parameter set and key from a descriptor table), chunked at
//      max_items gates,
//   3. retires jobs whose last level ran: outputs are gathered (not() applied)
//      and copied out, their arena ranges are freed.
// Jobs admitted while others are mid-circuit join at their own level 1, so
// work of requests arriving at different times overlaps on the device.
// A dry-run server (device PZ_SERVER_DRY_RUN) runs the same admission and
// level bookkeeping without a GPU.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <random>
#include <unordered_map>
#include <vector>

#include "pz_internal.h"

using pz::u32;
using pz::u64;

namespace {
double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}
}  // namespace

struct pz_server {
  int device = 0;
  bool dry = false;
  cudaStream_t stream = nullptr;
  std::string err;

  struct Session {
    pz_ctx *ctx = nullptr;
    const pz_key *key = nullptr;  // the device key while resident (null: not resident)
    int param_id = 0;
    size_t key_bytes = 0;
    // managed: the server owns the device key, imported from the caller's
    // blob (the pz_key_export form) when a job needs it, released on eviction
    bool managed = false;
    const void *blob = nullptr;
    size_t blob_bytes = 0;
    pz_key *owned = nullptr;
    bool virt_resident = false;  // dry run: residency without a device key
    size_t jobs_in_flight = 0;   // admitted, unfinished jobs: they pin the key
    u64 last_use = 0;            // LRU clock of the last admission / step that used the key
  };
  std::vector<Session> sessions;
  // device bytes resident managed keys may hold (SIZE_MAX: no limit)
  size_t key_budget = SIZE_MAX, managed_bytes = 0;
  u64 use_clock = 0, key_imports = 0, key_evictions = 0;
  bool descs_dirty = false;
  bool ks_mma = false;  // every session with a resident key has its KSK byte planes: tensor-core key switch
  int logn = -1;
  bool d1 = true;
  size_t L = 0;
  u64 q = 0;
  u32 max_n = 0, max_br_q = 0, max_d = 0, ks_stride = 0;
  pz::BrParams *d_br = nullptr;
  pz::KsParams *d_ksp = nullptr;

  // wire arena: slots of L words
  u64 *d_arena = nullptr;
  size_t arena_slots = 0, slots_used = 0;
  std::map<size_t, size_t> free_ranges;  // start -> length

  // per-chunk staging (double-buffered host->device item arrays)
  size_t max_items = 0;
  size_t arena_bytes_req = 0;
  int flip = 0;
  u32 ksout_stride = 0;
  unsigned char *h_buf[2] = {nullptr, nullptr};
  unsigned char *d_buf[2] = {nullptr, nullptr};
  cudaEvent_t buf_free[2] = {nullptr, nullptr};
  u32 *d_ksout = nullptr;
  u64 *d_gather = nullptr;
  size_t gather_cap = 0;  // ciphertexts
  u32 *d_outref = nullptr;
  size_t outref_cap = 0;

  int pbs_variant = 0, grid_limit = 0;
  int schedule = PZ_SCHEDULE_ALL_READY;
  int sm_count = 148;  // the device's SMs (148 on B200; the dry-run server keeps this)

  struct Job {
    u64 id = 0;
    u32 session = 0;
    pz_circuit *c = nullptr;
    pz::CircuitView v;
    const u64 *in = nullptr;
    u64 *out = nullptr;
    int device_io = 0;
    size_t base = 0, slots = 0, level = 0;
    int state = 0;  // 0 pending, 1 running, 2 done, 3 failed
    double t_submit = 0, t_admit = 0, t_done = 0;
  };
  std::deque<Job *> pending;
  std::vector<Job *> active;
  std::unordered_map<u64, Job *> jobs;
  u64 next_id = 1;
  size_t n_done = 0, n_failed = 0;
  u64 steps = 0, gates = 0, launches = 0;

  pz_status fail(pz_status st, const std::string &m) {
    err = m;
    return st;
  }
  pz_status cuda(const char *what, cudaError_t e) {
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return PZ_ERR_CUDA;
  }

  // first fit over the free slot ranges
  bool alloc(size_t n, size_t *base) {
    for (auto it = free_ranges.begin(); it != free_ranges.end(); ++it) {
      if (it->second >= n) {
        *base = it->first;
        const size_t rest = it->second - n, start = it->first + n;
        free_ranges.erase(it);
        if (rest) free_ranges[start] = rest;
        slots_used += n;
        return true;
      }
    }
    return false;
  }
  void release(size_t base, size_t n) {
    if (!n) return;
    slots_used -= n;
    auto it = free_ranges.emplace(base, n).first;
    auto next = std::next(it);
    if (next != free_ranges.end() && it->first + it->second == next->first) {
      it->second += next->second;
      free_ranges.erase(next);
    }
    if (it != free_ranges.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == it->first) {
        prev->second += it->second;
        free_ranges.erase(it);
      }
    }
  }

  // packed item arrays of one chunk: gates | in0 | in1 | out | desc | tiles
  struct Layout {
    size_t gate, in0, in1, out, desc, tiles, total;
  };
  Layout layout(size_t cap) const {
    Layout l;
    size_t o = 0;
    auto take = [&](size_t bytes) {
      const size_t at = o;
      o += (bytes + 255) & ~(size_t)255;
      return at;
    };
    l.gate = take(cap);
    l.in0 = take(cap * 4);
    l.in1 = take(cap * 4);
    l.out = take(cap * 4);
    l.desc = take(cap * 4);
    l.tiles = take((cap + 1) * sizeof(pz::KsTile));
    l.total = o;
    return l;
  }

  bool resident(const Session &se) const { return !se.managed || se.owned || se.virt_resident; }

  ~pz_server() {
    for (auto &kv : jobs) delete kv.second;
    if (!dry) {
      cudaSetDevice(device);
      if (stream) cudaStreamSynchronize(stream);
      for (auto &se : sessions)
        if (se.owned) pz_key_release(se.owned);
      for (int b = 0; b < 2; b++) {
        if (h_buf[b]) cudaFreeHost(h_buf[b]);
        if (d_buf[b]) cudaFree(d_buf[b]);
        if (buf_free[b]) cudaEventDestroy(buf_free[b]);
      }
      cudaFree(d_arena);
      cudaFree(d_ksout);
      cudaFree(d_gather);
      cudaFree(d_outref);
      cudaFree(d_br);
      cudaFree(d_ksp);
      if (stream) cudaStreamDestroy(stream);
    }
  }
};

namespace {

size_t key_bytes_of(const pz_params &P) {
  // RGSW + auto keys (u64, device form) + KSK (u32 rows of ks_stride words)
  return (size_t)P.lwe_n * P.rgsw_rows * P.rlwe_n * 8 + (size_t)P.n_auto_keys * P.auto_rows * P.rlwe_n * 8 +
         (size_t)P.lwe_d * P.rlwe_n * pz::ks_stride(P) * 4;
}

// Re-upload the descriptor tables after a session was added.
pz_status upload_descs(pz_server *s) {
  if (s->dry) return PZ_OK;
  cudaError_t e = cudaStreamSynchronize(s->stream);  // no launch may still read the old tables
  if (e != cudaSuccess) return s->cuda("cudaStreamSynchronize", e);
  std::vector<pz::BrParams> br(s->sessions.size());
  std::vector<pz::KsParams> ks(s->sessions.size());
  for (size_t i = 0; i < s->sessions.size(); i++) {
    const auto &se = s->sessions[i];
    br[i] = se.ctx->br;  // a session without a resident key gets no items: null key pointers
    br[i].rgsw = se.key ? se.key->d_rgsw : nullptr;
    br[i].autos = se.key ? se.key->d_autos : nullptr;
    br[i].out_idx = nullptr;
    ks[i] = se.ctx->ks;
    ks[i].ksk = nullptr;
    if (se.key) pz::ks_bind_key(se.ctx, se.key, ks[i]);
  }
  bool mma = s->max_d <= 16;
  for (size_t i = 0; i < s->sessions.size(); i++)
    if (s->sessions[i].key && !s->sessions[i].key->d_ksk8) mma = false;
  s->ks_mma = mma;
  s->descs_dirty = false;
  cudaFree(s->d_br);
  cudaFree(s->d_ksp);
  s->d_br = nullptr;
  s->d_ksp = nullptr;
  if ((e = cudaMalloc(&s->d_br, br.size() * sizeof(pz::BrParams))) != cudaSuccess) return s->cuda("cudaMalloc", e);
  if ((e = cudaMalloc(&s->d_ksp, ks.size() * sizeof(pz::KsParams))) != cudaSuccess) return s->cuda("cudaMalloc", e);
  if ((e = cudaMemcpy(s->d_br, br.data(), br.size() * sizeof(pz::BrParams), cudaMemcpyHostToDevice)) != cudaSuccess)
    return s->cuda("cudaMemcpy", e);
  if ((e = cudaMemcpy(s->d_ksp, ks.data(), ks.size() * sizeof(pz::KsParams), cudaMemcpyHostToDevice)) != cudaSuccess)
    return s->cuda("cudaMemcpy", e);
  return PZ_OK;
}

pz_status add_session_common(pz_server *s, int param_id, pz_ctx *ctx, const pz_key *key, uint32_t *session,
                             const void *blob = nullptr, size_t blob_bytes = 0, bool managed = false) {
  pz_params P;
  if (pz_param_get(param_id, &P) != PZ_OK) return s->fail(PZ_ERR_INVALID_ARGUMENT, "bad parameter set");
  const int logn = (int)__builtin_ctzll(P.rlwe_n);
  const bool d1 = P.rlrg_d_a == 1 && P.rlrg_d_b == 1 && P.auto_d == 1;
  if (s->logn >= 0 && (logn != s->logn || d1 != s->d1 || P.rlwe_q != s->q))
    return s->fail(PZ_ERR_NOT_SUPPORTED, "all sessions of a server share the ring (N, Q) and decomposition shape");
  if (s->logn < 0) {
    s->logn = logn;
    s->d1 = d1;
    s->L = (size_t)P.rlwe_n + 1;
    s->q = P.rlwe_q;
  }
  pz_server::Session se;
  se.ctx = ctx;
  se.key = key;
  se.param_id = param_id;
  se.key_bytes = key ? key->bytes : key_bytes_of(P);
  se.managed = managed;
  se.blob = blob;
  se.blob_bytes = blob_bytes;
  s->sessions.push_back(se);
  s->max_n = std::max(s->max_n, P.lwe_n);
  s->max_br_q = std::max(s->max_br_q, P.br_q);
  s->max_d = std::max(s->max_d, P.lwe_d);
  s->ks_stride = std::max(s->ks_stride, pz::ks_stride(P));
  pz_status st = upload_descs(s);
  if (st != PZ_OK) {
    s->sessions.pop_back();
    return st;
  }
  if (session) *session = (uint32_t)(s->sessions.size() - 1);
  return PZ_OK;
}

pz_status ensure_arena(pz_server *s, size_t arena_bytes) {
  if (s->arena_slots) return PZ_OK;
  s->arena_slots = arena_bytes / (s->L * 8);
  if (s->arena_slots == 0) return s->fail(PZ_ERR_INVALID_ARGUMENT, "arena smaller than one ciphertext");
  s->free_ranges.clear();
  s->free_ranges[0] = s->arena_slots;
  if (s->dry) return PZ_OK;
  cudaError_t e = cudaMalloc(&s->d_arena, s->arena_slots * s->L * 8);
  if (e != cudaSuccess) {
    s->arena_slots = 0;
    return s->cuda("arena cudaMalloc", e);
  }
  return PZ_OK;
}

void evict(pz_server *s, pz_server::Session &se) {
  if (se.owned) pz_key_release(se.owned);
  se.owned = nullptr;
  se.key = nullptr;
  se.virt_resident = false;
  s->managed_bytes -= se.key_bytes;
  s->key_evictions++;
  s->descs_dirty = true;
}

// Make the key of session `sid` resident: evict the least recently used
// resident managed keys of sessions without jobs in flight until it fits the
// budget, then import it.  *fits = false: not now (the keys in the way are
// pinned by running jobs); a CUDA or blob error is returned as such.
pz_status make_resident(pz_server *s, u32 sid, bool *fits) {
  pz_server::Session &se = s->sessions[sid];
  *fits = true;
  if (s->resident(se)) return PZ_OK;
  while (s->managed_bytes + se.key_bytes > s->key_budget) {
    pz_server::Session *victim = nullptr;
    for (auto &o : s->sessions)
      if (&o != &se && o.managed && s->resident(o) && o.jobs_in_flight == 0 &&
          (!victim || o.last_use < victim->last_use))
        victim = &o;
    if (!victim) {
      *fits = false;
      return PZ_OK;
    }
    evict(s, *victim);
  }
  if (s->dry) {
    se.virt_resident = true;
  } else {
    pz_key *k = nullptr;
    pz_status st = pz_key_import(se.ctx, se.blob, se.blob_bytes, &k);
    if (st != PZ_OK) return s->fail(st, std::string("managed session key import: ") + pz_last_error(se.ctx));
    se.owned = k;
    se.key = k;
  }
  s->managed_bytes += se.key_bytes;
  s->key_imports++;
  s->descs_dirty = true;
  return PZ_OK;
}

void fail_job(pz_server *s, pz_server::Job *j) {
  j->state = 3;
  j->t_done = now_ms();
  s->n_failed++;
  s->pending.pop_front();
}

// The wire arena and the key-switch scratch for the widest session so far.
pz_status ensure_device_buffers(pz_server *s) {
  pz_status st = ensure_arena(s, s->arena_bytes_req);
  if (st != PZ_OK) return st;
  if (s->ks_stride > s->ksout_stride) {
    cudaStreamSynchronize(s->stream);
    cudaFree(s->d_ksout);
    s->d_ksout = nullptr;
    s->ksout_stride = 0;
    cudaError_t e = cudaMalloc(&s->d_ksout, s->max_items * (size_t)s->ks_stride * 4);
    if (e != cudaSuccess) return s->cuda("cudaMalloc", e);
    s->ksout_stride = s->ks_stride;
  }
  return PZ_OK;
}

// Admit pending jobs in arrival order while their wires fit the arena and
// their session's key is (or can be made) resident.  Resident managed keys
// over the budget (it may have been lowered) are evicted first, least
// recently used idle ones, as far as idle ones go.
pz_status admit(pz_server *s) {
  while (s->managed_bytes > s->key_budget) {
    pz_server::Session *victim = nullptr;
    for (auto &o : s->sessions)
      if (o.managed && s->resident(o) && o.jobs_in_flight == 0 && (!victim || o.last_use < victim->last_use))
        victim = &o;
    if (!victim) break;
    evict(s, *victim);
  }
  while (!s->pending.empty()) {
    pz_server::Job *j = s->pending.front();
    const size_t need = j->v.n_inputs + j->v.n_gates;
    pz_server::Session &se = s->sessions[j->session];
    if (need > s->arena_slots || (se.managed && se.key_bytes > s->key_budget)) {  // can never fit
      fail_job(s, j);
      continue;
    }
    bool fits = true;
    pz_status st = make_resident(s, j->session, &fits);
    if (st != PZ_OK) return st;
    if (!fits) break;
    size_t base;
    if (!s->alloc(std::max<size_t>(need, 1), &base)) break;
    se.jobs_in_flight++;
    se.last_use = ++s->use_clock;
    j->base = base;
    j->slots = std::max<size_t>(need, 1);
    j->level = 0;
    j->state = 1;
    j->t_admit = now_ms();
    if (!s->dry && j->v.n_inputs) {
      cudaError_t e = cudaMemcpyAsync(s->d_arena + base * s->L, j->in, j->v.n_inputs * s->L * 8,
                                      j->device_io ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s->stream);
      if (e != cudaSuccess) return s->cuda("input copy", e);
    }
    s->pending.pop_front();
    s->active.push_back(j);
  }
  return s->descs_dirty ? upload_descs(s) : PZ_OK;
}

struct Item {
  u32 session;
  unsigned char gate;
  u32 in0, in1, out;
};

// Run the sorted items of one step, in chunks of max_items.
pz_status run_items(pz_server *s, const std::vector<Item> &items) {
  if (s->dry || items.empty()) return PZ_OK;
  const pz_server::Layout lay = s->layout(s->max_items);
  for (size_t c0 = 0; c0 < items.size(); c0 += s->max_items) {
    const size_t n = std::min(s->max_items, items.size() - c0);
    const int b = s->flip;
    s->flip ^= 1;
    cudaError_t e = cudaEventSynchronize(s->buf_free[b]);  // its previous chunk has been read
    if (e != cudaSuccess) return s->cuda("cudaEventSynchronize", e);
    unsigned char *h = s->h_buf[b];
    unsigned char *hg = h + lay.gate;
    u32 *h0 = (u32 *)(h + lay.in0), *h1 = (u32 *)(h + lay.in1), *ho = (u32 *)(h + lay.out);
    u32 *hd = (u32 *)(h + lay.desc);
    pz::KsTile *ht = (pz::KsTile *)(h + lay.tiles);
    size_t ntiles = 0;
    const u32 tile_cap = s->ks_mma ? (u32)pz::KSM_ROWS : (u32)pz::KS_TILE_CT;
    for (size_t i = 0; i < n; i++) {
      const Item &it = items[c0 + i];
      hg[i] = it.gate;
      h0[i] = it.in0;
      h1[i] = it.in1;
      ho[i] = it.out;
      hd[i] = it.session;
      if (ntiles == 0 || ht[ntiles - 1].desc != it.session || ht[ntiles - 1].count == tile_cap)
        ht[ntiles++] = pz::KsTile{it.session, (u32)i, 0};
      ht[ntiles - 1].count++;
    }
    unsigned char *d = s->d_buf[b];
    if ((e = cudaMemcpyAsync(d, h, lay.total, cudaMemcpyHostToDevice, s->stream)) != cudaSuccess)
      return s->cuda("item upload", e);
    if ((e = cudaEventRecord(s->buf_free[b], s->stream)) != cudaSuccess) return s->cuda("cudaEventRecord", e);
    e = (s->ks_mma ? pz::launch_ks_mma_ragged : pz::launch_ks_ragged)(
        s->d_ksp, (const pz::KsTile *)(d + lay.tiles), ntiles, n, s->max_n, (u32)(s->L - 1), s->max_d, d + lay.gate,
        s->d_arena, (const u32 *)(d + lay.in0), (const u32 *)(d + lay.in1), s->d_ksout, s->ks_stride, s->stream);
    if (e != cudaSuccess) return s->cuda("launch_ks_ragged", e);
    // a step of at most half the SMs' gates: one cluster of two CTAs per gate (the latency form)
    const int variant = (s->logn == 11 && s->d1 && n <= (size_t)s->sm_count / 2) ? pz::PBS_SPLIT : s->pbs_variant;
    e = pz::launch_pbs_ragged(s->logn, s->d1, s->d_br, (const u32 *)(d + lay.desc), s->max_br_q, s->max_n,
                              s->d_ksout, s->ks_stride, d + lay.gate, s->d_arena, (const u32 *)(d + lay.out), n,
                              s->grid_limit, s->stream, variant);
    if (e != cudaSuccess) return s->cuda("launch_pbs_ragged", e);
    s->launches += 2;
  }
  return PZ_OK;
}

// The jobs that advance one level this step.  PZ_SCHEDULE_ALL_READY: every
// admitted job with a level left.  PZ_SCHEDULE_CRITICAL_PATH: the jobs with
// the most levels left always advance (they set the number of steps the
// batch needs); the others, most levels left first, fill the step only up to
// the launch-time tier the mandatory gates already pay for -- one CTA per SM,
// two, ... up to the variant's CTAs per SM, then whole waves -- so work with
// slack moves into steps that would otherwise leave SMs idle.  A job waits
// at most until its remaining depth is the largest, so the batch still ends
// after (deepest circuit) steps.
size_t level_width(const pz_server::Job *j) { return j->v.level_off[j->level + 1] - j->v.level_off[j->level]; }

void select_jobs(pz_server *s, std::vector<pz_server::Job *> &run) {
  run.clear();
  if (s->schedule != PZ_SCHEDULE_CRITICAL_PATH) {
    for (auto *j : s->active)
      if (j->level < j->v.levels) run.push_back(j);
    return;
  }
  size_t depth = 0;
  for (auto *j : s->active)
    if (j->level < j->v.levels) depth = std::max(depth, j->v.levels - j->level);
  std::vector<pz_server::Job *> opt;
  size_t g = 0;
  for (auto *j : s->active) {
    if (j->level >= j->v.levels) continue;
    if (j->v.levels - j->level == depth) {
      run.push_back(j);
      g += level_width(j);
    } else {
      opt.push_back(j);
    }
  }
  const size_t sms = (size_t)std::max(1, s->sm_count);
  const size_t cps = (s->pbs_variant == 0 || s->pbs_variant == pz::PBS_BULK) ? 2 : s->pbs_variant == 2 ? 4 : 3;
  const size_t wave = sms * cps;
  const size_t cap = g <= wave ? std::max<size_t>(1, (g + sms - 1) / sms) * sms : (g + wave - 1) / wave * wave;
  std::stable_sort(opt.begin(), opt.end(), [](const pz_server::Job *a, const pz_server::Job *b) {
    return a->v.levels - a->level > b->v.levels - b->level;
  });
  for (auto *j : opt) {
    const size_t w = level_width(j);
    if (g + w <= cap) {
      run.push_back(j);
      g += w;
    }
  }
}

// Gather the outputs of finished jobs (on the stream; copies complete at the
// step's final synchronisation).
pz_status finish_outputs(pz_server *s, const std::vector<pz_server::Job *> &fin) {
  if (s->dry || fin.empty()) return PZ_OK;
  size_t host_outs = 0, refs = 0;
  for (auto *j : fin) {
    refs += j->v.n_outputs;
    if (!j->device_io) host_outs += j->v.n_outputs;
  }
  cudaError_t e;
  if (refs > s->outref_cap) {
    if ((e = cudaStreamSynchronize(s->stream)) != cudaSuccess) return s->cuda("cudaStreamSynchronize", e);
    cudaFree(s->d_outref);
    s->d_outref = nullptr;
    s->outref_cap = 0;
    if ((e = cudaMalloc(&s->d_outref, refs * 4)) != cudaSuccess) return s->cuda("cudaMalloc", e);
    s->outref_cap = refs;
  }
  if (host_outs > s->gather_cap) {
    if ((e = cudaStreamSynchronize(s->stream)) != cudaSuccess) return s->cuda("cudaStreamSynchronize", e);
    cudaFree(s->d_gather);
    s->d_gather = nullptr;
    s->gather_cap = 0;
    if ((e = cudaMalloc(&s->d_gather, host_outs * s->L * 8)) != cudaSuccess) return s->cuda("cudaMalloc", e);
    s->gather_cap = host_outs;
  }
  std::vector<u32> h(refs);
  size_t r = 0;
  for (auto *j : fin)
    for (size_t i = 0; i < j->v.n_outputs; i++) {
      const u32 ref = j->v.outref[i];
      h[r++] = (u32)(j->base + (ref & pz::WIRE_MASK)) | (ref & pz::WIRE_NEG);
    }
  if (refs && (e = cudaMemcpyAsync(s->d_outref, h.data(), refs * 4, cudaMemcpyHostToDevice, s->stream)) != cudaSuccess)
    return s->cuda("outref upload", e);
  size_t ro = 0, go = 0;
  for (auto *j : fin) {
    const size_t no = j->v.n_outputs;
    if (!no) continue;
    u64 *dst = j->device_io ? j->out : s->d_gather + go * s->L;
    if ((e = pz::launch_gather(s->d_arena, s->d_outref + ro, dst, no, s->L, s->q, s->stream)) != cudaSuccess)
      return s->cuda("gather", e);
    if (!j->device_io) {
      if ((e = cudaMemcpyAsync(j->out, dst, no * s->L * 8, cudaMemcpyDeviceToHost, s->stream)) != cudaSuccess)
        return s->cuda("output copy", e);
      go += no;
    }
    ro += no;
  }
  return PZ_OK;  // complete at the step's stream synchronisation
}

}  // namespace

extern "C" {

pz_status pz_server_create(int device, size_t arena_bytes, size_t max_items, pz_server **out) {
  if (!out || max_items == 0) return PZ_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  pz_server *s = new pz_server();
  s->dry = device == PZ_SERVER_DRY_RUN;
  s->device = s->dry ? 0 : device;
  if (!s->dry) cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, device);
  s->max_items = max_items;
  s->arena_slots = 0;
  s->arena_bytes_req = arena_bytes;  // slots are sized by the first session's ring (L words)
  if (!s->dry) {
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
      s->dry = true;  // nothing device-side to release
      delete s;
      return PZ_ERR_CUDA;
    }
    const pz_server::Layout lay = s->layout(max_items);
    for (int b = 0; b < 2; b++) {
      if (cudaMallocHost(&s->h_buf[b], lay.total) != cudaSuccess || cudaMalloc(&s->d_buf[b], lay.total) != cudaSuccess ||
          cudaEventCreateWithFlags(&s->buf_free[b], cudaEventDisableTiming) != cudaSuccess ||
          cudaEventRecord(s->buf_free[b], s->stream) != cudaSuccess) {
        delete s;
        return PZ_ERR_OUT_OF_MEMORY;
      }
    }
  }
  *out = s;
  return PZ_OK;
}

void pz_server_destroy(pz_server *s) { delete s; }

const char *pz_server_last_error(const pz_server *s) { return s ? s->err.c_str() : "no server"; }

pz_status pz_server_add_session(pz_server *s, pz_ctx *ctx, const pz_key *key, uint32_t *session) {
  if (!s || !ctx || !key) return PZ_ERR_INVALID_ARGUMENT;
  if (s->dry) return s->fail(PZ_ERR_INVALID_ARGUMENT, "dry-run server: use pz_server_add_virtual_session");
  if (key->ctx != ctx) return s->fail(PZ_ERR_KEY_MISMATCH, "key does not belong to this context");
  if (ctx->device != s->device) return s->fail(PZ_ERR_INVALID_ARGUMENT, "context is on another device");
  cudaSetDevice(s->device);
  pz_status st = add_session_common(s, ctx->param_id, ctx, key, session);
  if (st != PZ_OK) return st;
  return ensure_device_buffers(s);
}

pz_status pz_server_add_managed_session(pz_server *s, pz_ctx *ctx, const void *key_blob, size_t blob_bytes,
                                        uint32_t *session) {
  if (!s || !ctx || !key_blob || !blob_bytes) return PZ_ERR_INVALID_ARGUMENT;
  if (s->dry) return s->fail(PZ_ERR_INVALID_ARGUMENT, "dry-run server: use pz_server_add_virtual_managed_session");
  if (ctx->device != s->device) return s->fail(PZ_ERR_INVALID_ARGUMENT, "context is on another device");
  if (blob_bytes != 64 + key_bytes_of(ctx->P))
    return s->fail(PZ_ERR_INVALID_ARGUMENT, "managed session: blob size does not match the parameter set");
  cudaSetDevice(s->device);
  pz_status st = add_session_common(s, ctx->param_id, ctx, nullptr, session, key_blob, blob_bytes, true);
  if (st != PZ_OK) return st;
  return ensure_device_buffers(s);
}

pz_status pz_server_add_virtual_managed_session(pz_server *s, int param_id, uint32_t *session) {
  if (!s) return PZ_ERR_INVALID_ARGUMENT;
  if (!s->dry) return s->fail(PZ_ERR_INVALID_ARGUMENT, "virtual sessions exist only on a dry-run server");
  pz_status st = add_session_common(s, param_id, nullptr, nullptr, session, nullptr, 0, true);
  if (st != PZ_OK) return st;
  return ensure_arena(s, s->arena_bytes_req);
}

pz_status pz_server_set_key_budget(pz_server *s, size_t bytes) {
  if (!s) return PZ_ERR_INVALID_ARGUMENT;
  s->key_budget = bytes ? bytes : SIZE_MAX;
  return PZ_OK;
}

pz_status pz_server_session_resident(pz_server *s, uint32_t session, int *resident) {
  if (!s || !resident) return PZ_ERR_INVALID_ARGUMENT;
  if (session >= s->sessions.size()) return s->fail(PZ_ERR_INVALID_ARGUMENT, "unknown session");
  *resident = s->resident(s->sessions[session]) ? 1 : 0;
  return PZ_OK;
}

pz_status pz_server_add_virtual_session(pz_server *s, int param_id, uint32_t *session) {
  if (!s) return PZ_ERR_INVALID_ARGUMENT;
  if (!s->dry) return s->fail(PZ_ERR_INVALID_ARGUMENT, "virtual sessions exist only on a dry-run server");
  pz_status st = add_session_common(s, param_id, nullptr, nullptr, session);
  if (st != PZ_OK) return st;
  return ensure_arena(s, s->arena_bytes_req);
}

pz_status pz_server_submit(pz_server *s, uint32_t session, pz_circuit *c, const uint64_t *inputs,
                           uint64_t *outputs, int device_io, uint64_t *job) {
  if (!s || !c) return PZ_ERR_INVALID_ARGUMENT;
  if (session >= s->sessions.size()) return s->fail(PZ_ERR_INVALID_ARGUMENT, "unknown session");
  pz_server::Job *j = new pz_server::Job();
  if (!pz::circuit_view(c, &j->v)) {
    delete j;
    return s->fail(PZ_ERR_INVALID_ARGUMENT, "bad circuit");
  }
  if (!s->dry && ((j->v.n_inputs && !inputs) || (j->v.n_outputs && !outputs))) {
    delete j;
    return s->fail(PZ_ERR_INVALID_ARGUMENT, "NULL job buffer");
  }
  j->id = s->next_id++;
  j->session = session;
  j->c = c;
  j->in = inputs;
  j->out = outputs;
  j->device_io = device_io;
  j->t_submit = now_ms();
  s->jobs[j->id] = j;
  s->pending.push_back(j);
  if (job) *job = j->id;
  return PZ_OK;
}

pz_status pz_server_step(pz_server *s, size_t *gates_run) {
  if (!s) return PZ_ERR_INVALID_ARGUMENT;
  if (gates_run) *gates_run = 0;
  if (!s->dry) cudaSetDevice(s->device);
  pz_status st = admit(s);
  if (st != PZ_OK) return st;
  std::vector<pz_server::Job *> run;
  select_jobs(s, run);
  // next level of every selected job, sorted by session (counting sort)
  std::vector<size_t> per(s->sessions.size() + 1, 0);
  for (auto *j : run) per[j->session + 1] += j->v.level_off[j->level + 1] - j->v.level_off[j->level];
  for (size_t i = 1; i < per.size(); i++) per[i] += per[i - 1];
  const size_t total = per.back();
  std::vector<Item> items(total);
  for (auto *j : run) {
    s->sessions[j->session].last_use = ++s->use_clock;
    const size_t a = j->v.level_off[j->level], b = j->v.level_off[j->level + 1];
    size_t &pos = per[j->session];
    for (size_t g = a; g < b; g++) {
      Item &it = items[pos++];
      it.session = j->session;
      it.gate = j->v.type[g];
      it.in0 = (u32)(j->base + (j->v.in0[g] & pz::WIRE_MASK)) | (j->v.in0[g] & pz::WIRE_NEG);
      it.in1 = (u32)(j->base + (j->v.in1[g] & pz::WIRE_MASK)) | (j->v.in1[g] & pz::WIRE_NEG);
      it.out = (u32)(j->base + j->v.out[g]);
    }
    j->level++;
  }
  st = run_items(s, items);
  if (st != PZ_OK) return st;
  std::vector<pz_server::Job *> fin, still;
  for (auto *j : s->active) (j->level >= j->v.levels ? fin : still).push_back(j);
  st = finish_outputs(s, fin);
  if (st != PZ_OK) return st;
  if (!s->dry) {
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return s->cuda("step", e);
  }
  const double t = now_ms();
  for (auto *j : fin) {
    j->state = 2;
    j->t_done = t;
    s->release(j->base, j->slots);
    s->sessions[j->session].jobs_in_flight--;
    s->n_done++;
  }
  s->active.swap(still);
  s->steps++;
  s->gates += total;
  if (gates_run) *gates_run = total;
  return PZ_OK;
}

pz_status pz_server_job_status(pz_server *s, uint64_t job, int *state, double *latency_ms, double *queue_ms) {
  if (!s) return PZ_ERR_INVALID_ARGUMENT;
  auto it = s->jobs.find(job);
  if (it == s->jobs.end()) return s->fail(PZ_ERR_INVALID_ARGUMENT, "unknown job");
  const pz_server::Job *j = it->second;
  if (state) *state = j->state;
  if (latency_ms) *latency_ms = j->state >= 2 ? j->t_done - j->t_submit : -1.0;
  if (queue_ms) *queue_ms = j->state >= 1 && j->state != 3 ? j->t_admit - j->t_submit : -1.0;
  return PZ_OK;
}

pz_status pz_server_forget(pz_server *s, uint64_t job) {
  if (!s) return PZ_ERR_INVALID_ARGUMENT;
  auto it = s->jobs.find(job);
  if (it == s->jobs.end()) return s->fail(PZ_ERR_INVALID_ARGUMENT, "unknown job");
  if (it->second->state < 2) return s->fail(PZ_ERR_INVALID_ARGUMENT, "job not finished");
  delete it->second;
  s->jobs.erase(it);
  return PZ_OK;
}

pz_status pz_server_stats_get(pz_server *s, pz_server_stats *out) {
  if (!s || !out) return PZ_ERR_INVALID_ARGUMENT;
  std::memset(out, 0, sizeof(*out));
  out->pending = s->pending.size();
  out->active = s->active.size();
  out->done = s->n_done;
  out->failed = s->n_failed;
  out->arena_slots = s->arena_slots;
  out->arena_slots_used = s->slots_used;
  out->arena_bytes = s->arena_slots * s->L * 8;
  out->sessions = s->sessions.size();
  for (auto &se : s->sessions) {
    out->key_bytes += se.key_bytes;
    if (s->resident(se)) out->resident_key_bytes += se.key_bytes;
  }
  out->key_budget = s->key_budget == SIZE_MAX ? 0 : s->key_budget;
  out->key_imports = s->key_imports;
  out->key_evictions = s->key_evictions;
  out->steps = s->steps;
  out->gates = s->gates;
  out->launches = s->launches;
  return PZ_OK;
}

pz_status pz_server_set_launch(pz_server *s, int pbs_variant, int grid_limit) {
  if (!s || pbs_variant < 0 || pbs_variant > pz::PBS_MAX_VARIANT || pbs_variant == pz::PBS_SPLIT || grid_limit < 0)
    return PZ_ERR_INVALID_ARGUMENT;
  s->pbs_variant = pbs_variant;
  s->grid_limit = grid_limit;
  return PZ_OK;
}

pz_status pz_server_set_schedule(pz_server *s, int policy) {
  if (!s) return PZ_ERR_INVALID_ARGUMENT;
  if (policy != PZ_SCHEDULE_ALL_READY && policy != PZ_SCHEDULE_CRITICAL_PATH)
    return s->fail(PZ_ERR_INVALID_ARGUMENT, "pz_server_set_schedule: unknown policy");
  s->schedule = policy;
  return PZ_OK;
}

pz_status pz_server_autotune(pz_server *s, size_t batch, int *variant, int *grid_limit, double *best_ms) {
  if (!s || batch == 0) return PZ_ERR_INVALID_ARGUMENT;
  if (s->dry) return s->fail(PZ_ERR_NOT_SUPPORTED, "dry-run server");
  if (s->sessions.empty()) return s->fail(PZ_ERR_INVALID_ARGUMENT, "no session");
  if (!s->active.empty()) return s->fail(PZ_ERR_INVALID_ARGUMENT, "autotune needs an idle server");
  batch = std::min(batch, std::min(s->max_items, s->arena_slots));
  cudaSetDevice(s->device);
  // synthetic key-switched LWEs (uniform mod each session's q_ks), gates
  // spread over the sessions, outputs into arena slots [0, batch)
  std::mt19937_64 rng(0x7A11u);
  std::vector<u32> ks((size_t)batch * s->ks_stride, 0), desc(batch), outi(batch);
  std::vector<unsigned char> g(batch);
  std::vector<u32> live;  // sessions whose key is on the device now
  for (u32 i = 0; i < (u32)s->sessions.size(); i++)
    if (s->sessions[i].key) live.push_back(i);
  if (live.empty()) return s->fail(PZ_ERR_INVALID_ARGUMENT, "autotune needs a session with a resident key");
  for (size_t i = 0; i < batch; i++) {
    desc[i] = live[i % live.size()];
    const pz_params &P = s->sessions[desc[i]].ctx->P;
    for (u32 c = 0; c <= P.lwe_n; c++) ks[i * s->ks_stride + c] = (u32)(rng() % P.lwe_q);
    g[i] = (unsigned char)(rng() % 6);
    outi[i] = (u32)i;
  }
  u32 *d_ks = nullptr, *d_desc = nullptr, *d_out = nullptr;
  unsigned char *d_g = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  pz_status st = PZ_OK;
  double best = 1e30;
  int bv = s->pbs_variant, bg = s->grid_limit;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
  const int grids[2] = {0, 2 * sms};
  auto CK = [&](cudaError_t e, const char *w) {
    if (e != cudaSuccess && st == PZ_OK) st = s->cuda(w, e);
    return e == cudaSuccess;
  };
  if (CK(cudaMalloc(&d_ks, ks.size() * 4), "cudaMalloc") && CK(cudaMalloc(&d_desc, batch * 4), "cudaMalloc") &&
      CK(cudaMalloc(&d_out, batch * 4), "cudaMalloc") && CK(cudaMalloc(&d_g, batch), "cudaMalloc") &&
      CK(cudaMemcpy(d_ks, ks.data(), ks.size() * 4, cudaMemcpyHostToDevice), "cudaMemcpy") &&
      CK(cudaMemcpy(d_desc, desc.data(), batch * 4, cudaMemcpyHostToDevice), "cudaMemcpy") &&
      CK(cudaMemcpy(d_out, outi.data(), batch * 4, cudaMemcpyHostToDevice), "cudaMemcpy") &&
      CK(cudaMemcpy(d_g, g.data(), batch, cudaMemcpyHostToDevice), "cudaMemcpy") &&
      CK(cudaEventCreate(&a), "cudaEventCreate") && CK(cudaEventCreate(&b), "cudaEventCreate")) {
    // one-CTA shapes (register caps 2/3/4 CTAs per SM) and the staged-key shape
    const int shapes[4] = {0, 1, 2, pz::PBS_BULK};
    const int nv = (s->logn == 11 && s->d1) ? 4 : 1;
    for (int vi = 0; vi < nv && st == PZ_OK; vi++) {
      const int v = shapes[vi];
      for (int gi = 0; gi < 2 && st == PZ_OK; gi++) {
        auto launch = [&]() {
          return pz::launch_pbs_ragged(s->logn, s->d1, s->d_br, d_desc, s->max_br_q, s->max_n, d_ks, s->ks_stride,
                                       d_g, s->d_arena, d_out, batch, grids[gi], s->stream, v);
        };
        if (!CK(launch(), "launch_pbs_ragged")) break;  // warm-up
        if (!CK(cudaEventRecord(a, s->stream), "cudaEventRecord")) break;
        for (int r = 0; r < 2; r++)
          if (!CK(launch(), "launch_pbs_ragged")) break;
        if (!CK(cudaEventRecord(b, s->stream), "cudaEventRecord")) break;
        if (!CK(cudaEventSynchronize(b), "cudaEventSynchronize")) break;
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        if (ms / 2 < best) {
          best = ms / 2;
          bv = v;
          bg = grids[gi];
        }
      }
    }
  }
  cudaStreamSynchronize(s->stream);
  cudaFree(d_ks);
  cudaFree(d_desc);
  cudaFree(d_out);
  cudaFree(d_g);
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (st != PZ_OK) return st;
  s->pbs_variant = bv;
  s->grid_limit = bg;
  if (variant) *variant = bv;
  if (grid_limit) *grid_limit = bg;
  if (best_ms) *best_ms = best;
  return PZ_OK;
}

}  // extern "C"
