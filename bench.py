#!/usr/bin/env python
"""Gate-bootstrap throughput of the B200 engine (one JSON line on rank 0).

Workload (one step): the batched circuit wavefront at NonInteractiveLTE8Party
parameters -- 1024 independent FheUint8 a*b (155 gates each) and 1024 a<b (35
gates each), 194,560 gate bootstraps.  Every circuit level (the gates of all
2048 circuits at that depth) is one key-switch launch plus one blind-rotation
launch; the whole circuit is one CUDA graph replayed per step.

  value   gate bootstraps/s with inputs resident in HBM (graph replay, CUDA events)
  e2e     the same through pz_circuit_run: host buffers in pinned memory,
          host->device inputs and device->host outputs inside the timed region
  plain   InteractiveLTE2Party, 128 NAND gates, one gate per launch
  roofline  blind-rotation kernel: algorithmic 32-bit multiply instructions
          (10 per 64-bit modmul, the roofline convention) per second / the IMAD
          rate measured on this GPU by pz_probe_imad_rate
  cpu_baseline  the CPU oracle (a C++ restatement of the reference's pbs path)
          on all host threads, bounded sample of the same gates

Keys and ciphertexts are seeded synthetic data with the reference's shapes and
value distribution (uniform mod Q / mod q_ks): RLWE/RGSW/LWE ciphertexts are
pseudo-random, so the bootstrap schedule and work equal those of real keys.
Inputs (537 MB of ciphertexts per step) exceed L2; the server key stays
L2/HBM resident across steps as in steady-state serving.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PARAM = "NI_8P"
N_MUL = 1024
N_LT = 1024
C_MM = 10  # 32-bit multiply instructions per 64-bit Shoup modmul (roofline convention)
GATE_NAMES = ["and", "nand", "or", "nor", "xor", "xnor"]
REF_STEP_SECONDS = 10.0  # wall time of one timed step of the CPU reference arm
ROOFLINE_WAVES = 8  # whole waves of the blind-rotation launch timed for the roofline
WORKLOAD_CONFIG = {
    "workload": "batched circuit wavefront: NI_8P, 1024 FheUint8 a*b + 1024 a<b, "
                "each level one launch, whole circuit one CUDA graph",
    "param_set": PARAM,
}


def pz():
    import importlib
    return importlib.import_module("phantom-zone_b200")


# ---------------------------------------------------------------------------
def synthetic_key(p, seed):
    rng = np.random.default_rng(seed)
    N, n = p.rlwe_n, p.lwe_n
    rgsw = rng.integers(0, p.rlwe_q, (n, p.rgsw_rows, N), dtype=np.uint64)
    autos = rng.integers(0, p.rlwe_q, (p.n_auto_keys, p.auto_rows, N), dtype=np.uint64)
    ksk = rng.integers(0, p.lwe_q, (p.lwe_d * N, n + 1), dtype=np.uint64)
    return rgsw, autos, ksk


def wavefront_circuit(P):
    C = P.Circuit()
    pairs = [(C.input_u8(), C.input_u8()) for _ in range(N_MUL + N_LT)]
    for a, b in pairs[:N_MUL]:
        C.outputs(C.u8_mul(a, b))
    for a, b in pairs[N_MUL:]:
        C.output(C.u8_cmp("lt", a, b))
    return C


def schedule_work(p, ks):
    """Exact counts of the blind rotation's work per ciphertext (pbs.rs:240-414)
    from key-switched LWEs ks [count][n+1]: returns modmuls by the roofline
    convention M = F (N/2) logN + I ((N/2) logN + N) + MAC."""
    br_q, n, N, g, w = p.br_q, p.lwe_n, p.rlwe_n, p.g, p.w
    dlog = np.zeros(br_q, np.int64)
    for i in range(br_q // 4):
        v = pow(g, i, br_q)
        dlog[v] = i
        dlog[br_q - v] = i + br_q // 4
    shift = int(np.log2(p.lwe_q)) - int(np.log2(br_q))
    q4 = br_q // 4
    logn = int(np.log2(N))
    total = 0
    for row in ks:
        odd = (row[1:].astype(np.int64) >> shift)
        odd = odd + ((odd & 1) ^ 1)
        cnt = np.bincount(dlog[odd], minlength=br_q // 2)
        trivial, autos_nt = True, 0

        def bucket(b):
            nonlocal trivial
            if cnt[b]:
                trivial = False

        v = 0
        for i in range(q4 - 1, 0, -1):
            bucket(q4 + i)
            v += 1
            if cnt[q4 + i - 1] or v == w or i == 1:
                autos_nt += 0 if trivial else 1
                v = 0
        bucket(q4)
        autos_nt += 0 if trivial else 1
        v = 0
        for i in range(q4 - 1, 0, -1):
            bucket(i)
            v += 1
            if cnt[i - 1] or v == w or i == 1:
                autos_nt += 0 if trivial else 1
                v = 0
        A = autos_nt
        F, I = 2 * n - 1 + A, 2 * n + 2 * A
        MAC = (4 * n - 2) * N + 2 * A * N
        total += F * (N // 2) * logn + I * ((N // 2) * logn + N) + MAC
    return total


def measured_hbm_gbs():
    """HBM copy bandwidth: MEASURED_PEAKS.json's when the file is present,
    else the fallback figure measured earlier on this pool's B200s."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        rec = json.load(open(path))
        for k in ("hbm_gbs", "hbm_copy_gbs"):
            if k in rec:
                return {"gbs": float(rec[k]), "source": f"MEASURED_PEAKS.json {k}"}
    except (OSError, ValueError):
        pass
    return {"gbs": 6650.0, "source": "fallback (no MEASURED_PEAKS.json): 6.65 TB/s measured earlier on this pool"}


def traffic_record(P, variant, B):
    """DRAM bytes per launch of B bootstraps from the committed ncu capture
    (profiles/pbs_kernel_traffic.json, bytes per bootstrap of a warm launch),
    used only when it was taken on the blind-rotation revision this library
    reports and on the same launch shape; None otherwise."""
    path = os.path.join(ROOT, "profiles", "pbs_kernel_traffic.json")
    rev = P.kernel_revision()
    try:
        rec = json.load(open(path))
    except (OSError, ValueError):
        return None, "no ncu capture on record"
    if rec.get("kernel_revision") != rev or rec.get("variant") != variant:
        return None, (f"ncu capture on record is of {rec.get('kernel_revision')} variant {rec.get('variant')}, "
                      f"not {rev} variant {variant}")
    return int(rec["bytes_per_bootstrap"] * B), (f"ncu capture of {rev} variant {variant}: "
                                                  f"{rec['bytes_per_bootstrap']} B per bootstrap x {B}")


def wavefront_parity_check(p, okey, h_in, h_out, d_out, mul_ids=(0,), lt_ids=(N_MUL, N_MUL + N_LT - 1)):
    """The measured wavefront checked after the timed region: the graph
    replay's outputs equal the host-buffer run's word for word, and the
    outputs of a few circuits equal the oracle's sequential gate-by-gate
    evaluation of the same FheUint8 ops (shortint/ops.rs) on the same inputs
    and synthetic key, word for word."""
    from concurrent.futures import ThreadPoolExecutor
    L = p.rlwe_n + 1
    replay = d_out.cpu().numpy().view(np.uint64)
    host = h_out.numpy().view(np.uint64)
    same_paths = bool(np.array_equal(replay, host))
    inp = h_in.numpy().view(np.uint64)

    def job(kind_i):
        kind, i = kind_i
        a, b = inp[16 * i:16 * i + 8], inp[16 * i + 8:16 * i + 16]
        if kind == "mul":
            return kind, i, okey.u8_op("mul", a, b)[0], replay[8 * i:8 * i + 8]
        return kind, i, okey.u8_op("lt", a, b)[0], replay[8 * N_MUL + (i - N_MUL)][None, :]

    jobs = [("mul", i) for i in mul_ids] + [("lt", i) for i in lt_ids]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
        res = list(ex.map(job, jobs))
    ok = same_paths and all(np.array_equal(want.reshape(-1, L), got.reshape(-1, L)) for _, _, want, got in res)
    return {"parity_checked": bool(ok), "replay_equals_host_run": same_paths,
            "circuits_checked": [f"{k} #{i}" for k, i, _, _ in res],
            "ciphertexts_checked": int(sum(g.size // L for _, _, _, g in res)),
            "oracle_seconds": time.perf_counter() - t0,
            "what": "every output of the graph replay == the C-ABI host-buffer run; the listed circuits' outputs == "
                    "the oracle's sequential evaluation, word for word"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl" if args.impl != "reference" else "gloo",
                                timeout=datetime.timedelta(seconds=600))
        return dist, int(os.environ["RANK"]), world, int(os.environ.get("LOCAL_RANK", "0"))
    return None, 0, 1, 0


def max_over_ranks(dist, x, device=None):
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
def host_cores():
    """Logical CPUs this process may run on, and the physical cores behind them
    (distinct (package, core) pairs in the sysfs topology)."""
    cpus = sorted(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else list(range(os.cpu_count() or 1))
    phys = set()
    for c in cpus:
        base = f"/sys/devices/system/cpu/cpu{c}/topology/"
        try:
            phys.add((open(base + "physical_package_id").read().strip(), open(base + "core_id").read().strip()))
        except OSError:
            phys.add(("?", str(c)))
    return len(cpus), len(phys)


def wavefront_gate_mix(ev):
    """Gate codes (and, nand, or, nor, xor, xnor) of the wavefront -- 1024
    FheUint8 a*b and 1024 a<b -- tallied from the oracle's own restatement of
    the reference's circuits (a dry run, nothing bootstrapped)."""
    return N_MUL * ev.u8_gate_mix("mul") + N_LT * ev.u8_gate_mix("lt")


def mix_gates(mix, count, rng):
    """`count` gate codes in the proportions of `mix` (largest remainder), shuffled."""
    mix = np.asarray(mix, np.float64)
    want = mix / mix.sum() * count
    n = np.floor(want).astype(np.int64)
    for i in np.argsort(-(want - n))[:count - int(n.sum())]:
        n[i] += 1
    codes = np.repeat(np.arange(6, dtype=np.uint8), n)
    rng.shuffle(codes)
    return codes


def cpu_gate_sample(p, key_arrays, threads, count, mix, seed=11, okey=None):
    """Time the oracle (CPU restatement of the reference's gate path) on `count`
    independent gates of the gate mix `mix`, spread over `threads` threads."""
    from oracle import oracle as O
    if okey is None:
        okey = O.Evaluator(PARAM).key(O.ServerKeyCoeff(*key_arrays))
    rng = np.random.default_rng(seed)
    c0 = rng.integers(0, p.rlwe_q, (count, p.rlwe_n + 1), dtype=np.uint64)
    c1 = rng.integers(0, p.rlwe_q, (count, p.rlwe_n + 1), dtype=np.uint64)
    gates = mix_gates(mix, count, rng)
    t0 = time.perf_counter()
    okey.gate_batch(gates, c0, c1, threads=threads)
    dt = time.perf_counter() - t0
    return count / dt, count, dt


def cpu_reference_setup(key_arrays=None):
    """The oracle side of the workload: parameter record, synthetic key (the
    same words the GPU arm uploads, unless given), oracle key and the
    wavefront's gate mix.  Uses the oracle only -- the product library is not
    loaded."""
    from oracle import oracle as O
    p = O.param_info(PARAM)
    if key_arrays is None:
        key_arrays = synthetic_key(p, 0x5EED)
    ev = O.Evaluator(PARAM)
    okey = ev.key(O.ServerKeyCoeff(*key_arrays))
    return p, key_arrays, okey, wavefront_gate_mix(ev)


def cpu_calibrated_sample(p, key_arrays, okey, mix, threads, seconds):
    """Gates per sample sized to about `seconds` of wall time on `threads`
    threads (calibrated on two gates per thread)."""
    rate0, _, _ = cpu_gate_sample(p, key_arrays, threads, 2 * threads, mix, seed=10, okey=okey)
    return max(threads, int(round(seconds * rate0 / threads)) * threads)


def run_reference(args):
    """--impl reference: the CPU restatement of the reference's gate path (the
    oracle, a port: the Rust crate cannot be built here) on all host threads,
    on independent gates in the wavefront's gate mix.  Rank 0 alone under
    torchrun; the product library is never loaded on this arm."""
    dist, rank, world, _ = dist_setup(args)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    threads, physical = host_cores()
    p, key_arrays, okey, mix = cpu_reference_setup()
    count = cpu_calibrated_sample(p, key_arrays, okey, mix, threads, args.ref_step_seconds)
    per_step = []
    for s in range(args.warmup + args.steps):
        # warm-up steps: one gate per thread; timed steps: the calibrated sample
        n = threads if s < args.warmup else count
        _, _, dt = cpu_gate_sample(p, key_arrays, threads, n, mix, seed=100 + s, okey=okey)
        if s >= args.warmup:
            per_step.append(dt)
    value = count * len(per_step) / sum(per_step)
    mix_s = ", ".join(f"{g} {int(c)}" for g, c in zip(GATE_NAMES, mix) if c)
    sample = (f"{count} independent NI_8P gates per step in the wavefront's gate mix ({mix_s} per 1024 a*b + "
              f"1024 a<b), {threads} threads on {physical} physical cores, "
              f"{sum(per_step) / len(per_step):.1f} s wall per step")
    line = {
        "impl": "reference", "metric": "gate bootstraps/sec", "value": value, "unit": "gate bootstraps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(per_step) / len(per_step), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": dict(WORKLOAD_CONFIG, sample=sample),
        "cpu_baseline": {"value": value, "unit": "gate bootstraps/s", "cores": threads, "physical_cores": physical,
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "gate bootstraps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def plain_form(P, torch, device, seed=7):
    """Plain form at InteractiveLTE2Party: 128 NAND bootstraps, one gate per launch."""
    p = P.params("I_2P_LB_SR")
    eng = P.Engine("I_2P_LB_SR", device=device)
    key = eng.upload_key(*synthetic_key(p, seed))
    rng = np.random.default_rng(seed)
    L = p.rlwe_n + 1
    c0 = torch.from_numpy(rng.integers(0, p.rlwe_q, (128, L), dtype=np.uint64).view(np.int64)).cuda()
    c1 = torch.from_numpy(rng.integers(0, p.rlwe_q, (128, L), dtype=np.uint64).view(np.int64)).cuda()
    g = torch.full((128,), 1, dtype=torch.uint8, device="cuda")
    out = torch.empty_like(c0)
    for i in range(3):
        eng.gate_batch_device(key, g[i:i + 1], c0[i], c1[i], out[i])
    torch.cuda.synchronize()
    lat = []
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(128)]
    for i in range(128):
        ev[i][0].record()
        eng.gate_batch_device(key, g[i:i + 1], c0[i], c1[i], out[i])
        ev[i][1].record()
    torch.cuda.synchronize()
    lat = [a.elapsed_time(b) for a, b in ev]
    total = sum(lat)
    key.release()
    eng.close()
    return {"value": 128 / (total / 1e3), "unit": "gate bootstraps/s", "p50_ms": statistics.median(lat),
            "p99_ms": float(np.percentile(lat, 99)), "config": "I_2P_LB_SR, 128 NAND, one gate per launch"}


SERVING_PARAMS = ["I_2P_LB_SR", "I_4P", "I_8P", "NI_2P", "NI_4P_HB_FR", "NI_8P"]


def microbench(P, torch, device, count=4096, reps=5):
    """Kernel microbench: forward+inverse negacyclic NTT of `count` polynomials
    (N = 2048, mod Q, seeded uniform), and `count` RLWE x RGSW external
    products at InteractiveLTE2Party (key index i mod n)."""
    p = P.params("I_2P_LB_SR")
    N = p.rlwe_n
    eng = P.Engine("I_2P_LB_SR", device=device)
    rng = np.random.default_rng(0x11)
    x = torch.from_numpy(rng.integers(0, p.rlwe_q, (count, N), dtype=np.uint64).view(np.int64)).cuda()
    t = x.clone()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    eng.ntt_forward_device(t)
    eng.ntt_backward_device(t)
    torch.cuda.synchronize()
    roundtrip_ok = bool(torch.equal(t, x))
    ev[0].record()
    for _ in range(reps):
        eng.ntt_forward_device(t)
    ev[1].record()
    for _ in range(reps):
        eng.ntt_backward_device(t)
    ev[2].record()
    torch.cuda.synchronize()
    fwd_ms = ev[0].elapsed_time(ev[1]) / reps
    inv_ms = ev[1].elapsed_time(ev[2]) / reps
    logn = int(np.log2(N))
    mm = count * ((N // 2) * logn + (N // 2) * logn + N)  # fwd + inv (N^-1 scaling counted as in the convention)
    key = eng.upload_key(*synthetic_key(p, 0x5EED))
    rl = torch.from_numpy(rng.integers(0, p.rlwe_q, (count, 2, N), dtype=np.uint64).view(np.int64)).cuda()
    idx = torch.arange(count, dtype=torch.int32, device="cuda") % p.lwe_n
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ep_by_shape = {}
    for v in (0, 1, 2):  # register caps of 2 / 3 / 4 CTAs per SM
        eng.pbs_variant = v
        eng.rlwe_by_rgsw_device(key, rl, idx)
        torch.cuda.synchronize()
        a.record()
        for _ in range(reps):
            eng.rlwe_by_rgsw_device(key, rl, idx)
        b.record()
        torch.cuda.synchronize()
        ep_by_shape[v] = a.elapsed_time(b) / reps
    ep_variant = min(ep_by_shape, key=ep_by_shape.get)
    ep_ms = ep_by_shape[ep_variant]
    key.release()
    eng.close()
    peak_imad = P.probe_imad_rate(device)
    hbm = measured_hbm_gbs()
    ntt_mm_s = mm / ((fwd_ms + inv_ms) / 1e3)
    ntt_gbs = 4 * count * N * 8 / ((fwd_ms + inv_ms) / 1e3) / 1e9
    ep_mm_s = count * 57344 / (ep_ms / 1e3)
    return {"config": f"{count} polys N={N} mod Q fwd+inv NTT; {count} RLWE x RGSW at I_2P_LB_SR (index i mod n)",
            "ntt_fwd_ms": fwd_ms, "ntt_inv_ms": inv_ms, "ntt_roundtrip_exact": roundtrip_ok,
            "ntt_polys_per_s": count / ((fwd_ms + inv_ms) / 1e3),
            "ntt_modmul_per_s": ntt_mm_s, "ntt_hbm_gbs": ntt_gbs,
            "ntt_int_frac": ntt_mm_s * C_MM / peak_imad,
            "ntt_hbm_frac": ntt_gbs / hbm["gbs"] if hbm["gbs"] else None,
            "ext_product_ms": ep_ms, "ext_products_per_s": count / (ep_ms / 1e3),
            "ext_product_modmul_per_s": ep_mm_s, "ext_product_int_frac": ep_mm_s * C_MM / peak_imad,
            "ext_product_ms_by_variant": ep_by_shape, "ext_product_variant": ep_variant,
            "roof": {"int_peak_imad_per_s": peak_imad, "int_peak_source": "pz_probe_imad_rate on this GPU",
                     "hbm_gbs": hbm["gbs"], "hbm_source": hbm["source"],
                     "what": "fractions: algorithmic modmuls x 10 IMAD / the IMAD peak; bytes in + out of both "
                             "passes / the HBM copy bandwidth"}}


def ni_ingest_bench(P, torch, device, count=64, reps=3):
    """Non-interactive input path at NonInteractiveLTE8Party: `count` seeded
    RLWEs (count x N bools) unseeded, key-switched u_j -> s and extracted,
    device buffers, CUDA events; plus the key switch alone."""
    prm = "NI_8P"
    p = P.params(prm)
    N = p.rlwe_n
    eng = P.Engine(prm, device=device)
    rng = np.random.default_rng(0x33)
    ksk = eng.upload_ni_ksk(rng.integers(0, p.rlwe_q, (2 * p.ni_ks_d, N), dtype=np.uint64))
    d_b = torch.from_numpy(rng.integers(0, p.rlwe_q, (count, N), dtype=np.uint64).view(np.int64)).cuda()
    d_r = torch.empty((count, 2, N), dtype=torch.int64, device="cuda")
    d_k = torch.empty_like(d_r)
    idx = torch.arange(count * N, dtype=torch.int32, device="cuda")
    d_l = torch.empty((count * N, N + 1), dtype=torch.int64, device="cuda")
    seed = bytes(range(32))

    def run():
        eng.ni_unseed_device(seed, d_b, d_r)
        eng.ni_key_switch_device(ksk, d_r, d_k)
        eng.sample_extract_device(d_k, idx, d_l)

    run()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    a.record()
    for _ in range(reps):
        run()
    b.record()
    for _ in range(reps):
        eng.ni_key_switch_device(ksk, d_r, d_k)
    c.record()
    torch.cuda.synchronize()
    all_ms = a.elapsed_time(b) / reps
    ks_ms = b.elapsed_time(c) / reps
    logn = int(np.log2(N))
    per_rlwe = p.ni_ks_d * (N // 2) * logn + 2 * ((N // 2) * logn + N) + 2 * p.ni_ks_d * N
    mm = count * per_rlwe
    del d_l
    # the key switch alone at a serving-sized batch (the extraction of that
    # many bools would not fit: N + 1 words per bool)
    big = 1024
    d_rb = torch.from_numpy(rng.integers(0, p.rlwe_q, (big, 2, N), dtype=np.uint64).view(np.int64)).cuda()
    d_kb = torch.empty_like(d_rb)
    eng.ni_key_switch_device(ksk, d_rb, d_kb)
    torch.cuda.synchronize()
    a.record()
    for _ in range(reps):
        eng.ni_key_switch_device(ksk, d_rb, d_kb)
    b.record()
    torch.cuda.synchronize()
    big_ms = a.elapsed_time(b) / reps
    peak = P.probe_imad_rate(device)
    ksk.release()
    eng.close()
    return {"config": f"NI_8P, {count} seeded RLWEs = {count * N} bools: unseed + rlwe_key_switch (d=50) + extract; "
                      f"key switch alone also at {big} RLWEs",
            "ingest_ms": all_ms, "bools_per_s": count * N / (all_ms / 1e3), "key_switch_ms": ks_ms,
            "rlwe_key_switches_per_s": count / (ks_ms / 1e3), "key_switch_modmul_per_s": mm / (ks_ms / 1e3),
            "key_switch_int_frac": mm / (ks_ms / 1e3) * C_MM / peak,
            f"key_switch_{big}_ms": big_ms, f"rlwe_key_switches_per_s_{big}": big / (big_ms / 1e3),
            f"key_switch_int_frac_{big}": big * per_rlwe / (big_ms / 1e3) * C_MM / peak}


def key_upload_bench(P, device):
    """Server-key upload at NonInteractiveLTE8Party: the full expanded key from
    the host vs the seeded form (auto-key B rows and LWE-KSK column 0 plus two
    seeds, A parts regenerated on the device)."""
    prm = "NI_8P"
    p = P.params(prm)
    rgsw, autos, ksk = synthetic_key(p, 0x5EED)
    auto_b = np.ascontiguousarray(autos[:, p.auto_d:, :])
    lwe_b = np.ascontiguousarray(ksk[:, 0])
    eng = P.Engine(prm, device=device)
    eng.upload_key(rgsw, autos, ksk).release()  # warm-up
    t0 = time.perf_counter()
    k1 = eng.upload_key(rgsw, autos, ksk)
    t1 = time.perf_counter()
    k2 = eng.upload_key_seeded(rgsw, auto_b, b"\x01" * 32, lwe_b, b"\x02" * 32)
    t2 = time.perf_counter()
    blob = k1.export()
    t3 = time.perf_counter()
    k3 = eng.import_key(blob)
    t4 = time.perf_counter()
    for k in (k1, k2, k3):
        k.release()
    eng.close()
    return {"config": "NI_8P server key, host -> device, wall clock", "full_ms": (t1 - t0) * 1e3,
            "seeded_ms": (t2 - t1) * 1e3, "full_host_bytes": int(rgsw.nbytes + autos.nbytes + ksk.nbytes),
            "seeded_host_bytes": int(rgsw.nbytes + auto_b.nbytes + lwe_b.nbytes + 64),
            "export_ms": (t3 - t2) * 1e3, "import_ms": (t4 - t3) * 1e3, "device_form_bytes": len(blob)}


def aggregate_bench(P, torch, device, prm="I_8P"):
    """Interactive server-key aggregation at InteractiveLTE8Party: the RGSW step
    for all n LWE indices and the 7 other users (n x 7 RGSW x RGSW products,
    rgrg decomposition logb 5, 9/8 digits), synthetic ciphertexts on the device."""
    p = P.params(prm)
    N, n = p.rlwe_n, p.lwe_n
    steps = 7
    eng = P.Engine(prm, device=device)
    g = torch.Generator(device="cuda").manual_seed(5)
    rows1 = 2 * (p.rgrg_d_a + p.rgrg_d_b)
    lead = torch.randint(0, p.rlwe_q, (n, 4, N), dtype=torch.int64, device="cuda", generator=g)
    others = torch.randint(0, p.rlwe_q, (steps, n, rows1, N), dtype=torch.int64, device="cuda", generator=g)
    work = lead.clone()
    eng.aggregate_rgsw_device(work, others[:1])  # warm-up: one step
    torch.cuda.synchronize()
    work.copy_(lead)
    t0 = time.perf_counter()
    eng.aggregate_rgsw_device(work, others)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    products = n * steps
    # the whole aggregation from 8 parties' shares (pz_aggregate_device: RGSW placement and gathers
    # per leader segment, the same products, auto / LWE-KSK sums)
    users, per = steps + 1, -(-n // (steps + 1))
    shares = []
    for u in range(users):
        seg = min(per * (u + 1), n) - min(per * u, n)
        shares.append(dict(
            self_leader_rgsws=torch.randint(0, p.rlwe_q, (seg, 4, N), dtype=torch.int64, device="cuda", generator=g),
            not_self_leader_rgsws=torch.randint(0, p.rlwe_q, (n - seg, rows1, N), dtype=torch.int64, device="cuda",
                                                generator=g),
            auto_keys=torch.randint(0, p.rlwe_q, (p.n_auto_keys, p.auto_d, N), dtype=torch.int64, device="cuda",
                                    generator=g),
            lwe_ksk=torch.randint(0, p.lwe_q, (p.lwe_d * N,), dtype=torch.int64, device="cuda", generator=g)))
    o_rgsw = torch.empty((n, 4, N), dtype=torch.int64, device="cuda")
    o_auto = torch.empty((p.n_auto_keys, p.auto_d, N), dtype=torch.int64, device="cuda")
    o_lwe = torch.empty((p.lwe_d * N,), dtype=torch.int64, device="cuda")
    eng.aggregate_device(shares, o_rgsw, o_auto, o_lwe)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    eng.aggregate_device(shares, o_rgsw, o_auto, o_lwe)
    torch.cuda.synchronize()
    whole_ms = (time.perf_counter() - t1) * 1e3
    del shares
    logn = int(np.log2(N))
    ntt = (N // 2) * logn
    # per RGSW x RGSW: key conversion (rows1 forward NTTs) + 2 RLWE x RGSW (digit NTTs, MAC rows, 2 inverse)
    mm = products * (rows1 * ntt + 2 * ((p.rgrg_d_a + p.rgrg_d_b) * ntt + 2 * (ntt + N) +
                                        2 * (p.rgrg_d_a + p.rgrg_d_b) * N))
    eng.close()
    return {"config": f"{prm}: {n} LWE indices x {steps} other users = {products} RGSW x RGSW "
                      f"(rgrg logb {p.rgrg_logb}, {p.rgrg_d_a}/{p.rgrg_d_b} digits), device buffers",
            "ms": dt * 1e3, "rgsw_products_per_s": products / dt, "modmul_per_s": mm / dt,
            "whole_aggregation_ms": whole_ms}


def ni_aggregate_bench(P, torch, device, prm="NI_8P", users=8):
    """Non-interactive server-key aggregation at NonInteractiveLTE8Party with 8
    users: ui_to_s keys, auto / LWE KSK sums and the RGSWs of all n LWE indices
    (per index 38 values x 50 digits transformed once, 38 x 7 + 2 key-switch
    MACs, 7 RGSW x RGSW products), synthetic canonical shares on the device."""
    p = P.params(prm)
    N, n, Q = p.rlwe_n, p.lwe_n, p.rlwe_q
    ra, rb = p.rgrg_d_a, p.rgrg_d_b
    mx, ml = max(ra, rb), max(p.rlrg_d_a, p.rlrg_d_b)
    eng = P.Engine(prm, device=device)
    g = torch.Generator(device="cuda").manual_seed(9)

    def U(*shape, q=Q):
        return torch.randint(0, q, shape, dtype=torch.int64, device="cuda", generator=g)

    per = -(-n // users)
    shares = []
    for j in range(users):
        b, e = min(per * j, n), min(per * (j + 1), n)
        shares.append(dict(ui_to_s_ksk=U(50, N), ksk_zero_encs=U(users - 1, 50, N), self_leader_cts=U(e - b, ml, N),
                           not_leader_cts=U(n - (e - b), mx, N), rgsw_zero_encs=U(n, ra, N),
                           auto_keys=U(p.n_auto_keys, p.auto_d, N), lwe_ksk=U(p.lwe_d * N, q=p.lwe_q)))
    ksk = torch.empty((users, 50, N), dtype=torch.int64, device="cuda")
    rgsw = torch.empty((n, 4, N), dtype=torch.int64, device="cuda")
    auto = torch.empty((p.n_auto_keys, p.auto_d, N), dtype=torch.int64, device="cuda")
    lwe = torch.empty(p.lwe_d * N, dtype=torch.int64, device="cuda")
    crs = bytes(range(32))
    eng.ni_aggregate_device(crs, shares, ksk, rgsw, auto, lwe)  # warm-up (allocator, module load)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    eng.ni_aggregate_device(crs, shares, ksk, rgsw, auto, lwe)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    R = ra + rb
    ntt = (N // 2) * int(np.log2(N))
    ks_macs = n * (R * (users - 1) + 2)
    products = n * (users - 1)
    share_bytes = sum(int(t.numel()) * 8 for sh in shares for t in sh.values())
    eng.close()
    return {"config": f"{prm}, {users} users: {n} LWE indices, {n * R} values x 50 digits, {ks_macs} key-switch "
                      f"MACs, {products} RGSW x RGSW (rgrg logb {p.rgrg_logb}, {ra}/{rb} digits), device shares",
            "ms": dt * 1e3, "share_bytes": share_bytes, "digit_ntts_per_s": n * R * 50 / dt,
            "ks_macs_per_s": ks_macs / dt, "butterflies_per_s": (n * R * 50 + ks_macs * 2) * ntt / dt}


def u8_job(P, op):
    C = P.Circuit()
    a, b = C.input_u8(), C.input_u8()
    if op == "add":
        C.outputs(C.u8_add(a, b))
    elif op == "mul":
        C.outputs(C.u8_mul(a, b))
    elif op == "lt":
        C.output(C.u8_cmp("lt", a, b))
    elif op == "div_rem":
        q, r, f = C.u8_div_rem(a, b)
        C.outputs(q)
        C.outputs(r)
        C.output(f)
    return C


def ragged_batch(P, device, per_session=64, params=("I_2P_LB_SR", "I_4P", "I_8P"), seed=4):
    """Ragged batch: sessions of the 2-, 4- and 8-party interactive sets in
    one server; per session `per_session` FheUint8 ops (add, mul, div_rem,
    lt; 20 % of the div_rem jobs with divisor 0) submitted at once; every step is one ragged key-switch launch
    plus one ragged blind-rotation launch across the sessions; the launch
    shape comes from the server's autotuner.  The zero divisors are trivial
    encryptions of 0 (every bit a = 0, b = -Q/8), valid under every key."""
    S = P.Server(device=device, arena_bytes=4 << 30, max_items=16384)
    keep = []
    for i, prm in enumerate(params):
        p = P.params(prm)
        eng = P.Engine(prm, device=device)
        key = eng.upload_key(*synthetic_key(p, 0x5EED + i))
        keep.append((eng, key, S.add_session(eng, key), p))
    tune = S.autotune(2368)
    S.set_schedule(P.server.SCHEDULE_CRITICAL_PATH)  # all jobs arrive together: deepest first, fill the rest
    rng = np.random.default_rng(seed)
    ops = ["add", "mul", "div_rem", "lt"]
    templates = {op: u8_job(P, op) for op in ops}
    L = keep[0][3].rlwe_n + 1
    pool = rng.integers(0, keep[0][3].rlwe_q, (64, L), dtype=np.uint64)
    gates = 0
    jobs = []
    for eng, key, sid, p in keep:
        for k in range(per_session):
            op = ops[k % 4]
            C = templates[op]
            inp = pool[rng.integers(0, 64 - 16):][:16].copy()
            if op == "div_rem" and rng.random() < 0.2:
                # divisor 0: every bit a noiseless encryption of false under any
                # key -- a = 0, b = -Q/8 (false_el, evaluator.rs:239-242)
                inp[8:16] = 0
                inp[8:16, 0] = keep[0][3].rlwe_q - (keep[0][3].rlwe_q >> 3)
            jobs.append(S.submit(sid, C, inp))
            gates += C.info()["gates"]
    t0 = time.perf_counter()
    steps = S.run_until_idle()
    dt = time.perf_counter() - t0
    st = S.stats()
    S.close()
    for eng, key, _, _ in keep:
        key.release()
        eng.close()
    return {"value": gates / dt, "unit": "gate bootstraps/s", "gates": gates, "jobs": len(jobs), "steps": steps,
            "launches": st["launches"], "seconds": dt, "autotune": tune,
            "schedule": "critical path",
            "config": f"sessions {list(params)}, {per_session} jobs each (add/mul/div_rem/lt), all submitted at once"}


def serving_circuit(P, target, rng):
    """A circuit of about `target` gates composed of FheUint8 ops chained on
    an accumulator (single gates fill the remainder)."""
    C = P.Circuit()
    acc = C.input_u8()
    sizes = [("mul", 155), ("sub", 38), ("add", 37), ("lt", 35), ("mux", 24), ("eq", 15)]
    made = 0
    while made < target:
        fit = [o for o, g in sizes if g <= target - made]
        if not fit:
            x = C.input()
            w = C.gate(["nand", "xor", "or"][int(rng.integers(0, 3))], acc[made % 8], x)
            acc[made % 8] = w
            made += 1
            continue
        op = fit[int(rng.integers(0, len(fit)))]
        b = C.input_u8()
        if op == "mul":
            acc = C.u8_mul(acc, b)
        elif op == "sub":
            acc = C.u8_sub(acc, b)
        elif op == "add":
            acc = C.u8_add(acc, b)
        elif op == "lt":
            acc[0] = C.u8_cmp("lt", acc, b)
        elif op == "mux":
            acc = C.u8_mux(acc, b, C.input())
        elif op == "eq":
            acc[0] = C.u8_cmp("eq", acc, b)
        made = C.info()["gates"]
    C.outputs(acc)
    return C


SERVING_RATES = [40.0, 80.0, 160.0, 320.0, 640.0]  # offered loads of the sweep, circuits/s


def serving_point(S, sids, templates, pool, rate, n_arr, rng):
    """Poisson arrivals at `rate` circuits/s (n_arr circuits, random sessions
    and templates) served by continuous batching; throughput = gates done /
    (last completion - first arrival); latency = completion - arrival."""
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_arr))
    st0 = S.stats()
    lat, inflight, gates_done = [], {}, 0
    idx, t0 = 0, time.perf_counter()
    steps, max_active, step_gates = 0, 0, []
    while idx < n_arr or inflight:
        now = time.perf_counter() - t0
        while idx < n_arr and arrivals[idx] <= now:
            C = templates[int(rng.integers(0, len(templates)))]
            ni = C.info()["inputs"]
            off = int(rng.integers(0, len(pool) - ni)) if ni < len(pool) else 0
            j = S.submit(sids[int(rng.integers(0, len(sids)))], C, pool[off:off + ni])
            inflight[j] = (arrivals[idx], C.info()["gates"])
            idx += 1
        if not inflight:
            time.sleep(max(0.0, arrivals[idx] - (time.perf_counter() - t0)))
            continue
        step_gates.append(S.step())
        steps += 1
        max_active = max(max_active, S.stats()["active"])
        tdone = time.perf_counter() - t0
        for j in list(inflight):
            if S.status(j)["state"] == 2:
                a, g = inflight.pop(j)
                lat.append((tdone - a) * 1e3)
                gates_done += g
                S.forget(j)
    total = time.perf_counter() - t0 - arrivals[0]
    st = S.stats()
    lat = np.array(lat)
    return {"offered_circuits_per_s": rate, "circuits": len(lat), "value": gates_done / total,
            "unit": "gate bootstraps/s", "gates": gates_done, "seconds": total,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)), "steps": steps,
            "mean_gates_per_step": float(np.mean(step_gates)), "max_active_jobs": max_active,
            "key_imports": st["key_imports"] - st0["key_imports"],
            "key_evictions": st["key_evictions"] - st0["key_evictions"]}


def serving(P, device, sessions=64, rates=SERVING_RATES, arrivals=480, tight_keys=16, seed=8):
    """Serving: `sessions` managed sessions (cycling over the 2/4/8-party
    interactive and non-interactive sets), each with its device-form key
    blob; the server imports a session's key when a job needs it and admits
    jobs by ciphertext + key bytes.  Poisson arrivals of FheUint8 circuits of
    U[1, 300] gates, continuous batching (one ragged launch pair per step).
    A load sweep at `rates` circuits/s (`arrivals` circuits each) with every
    key resident after a warm-up job per session, then one point at the
    sweep's second rate with a key budget of `tight_keys` keys (jobs of cold
    sessions import their key, evicting the least recently used idle one)."""
    S = P.Server(device=device, arena_bytes=8 << 30, max_items=16384)
    rng = np.random.default_rng(seed)
    engines, blobs = {}, {}
    for i, prm in enumerate(SERVING_PARAMS):
        eng = P.Engine(prm, device=device)
        key = eng.upload_key(*synthetic_key(P.params(prm), 0x5EED + i))
        engines[prm], blobs[prm] = eng, key.export()
        key.release()
    sids, kbytes = [], []
    for k in range(sessions):
        prm = SERVING_PARAMS[k % len(SERVING_PARAMS)]
        sids.append(S.add_managed_session(engines[prm], blobs[prm]))
        kbytes.append(len(blobs[prm]) - 64)
    templates = [serving_circuit(P, int(rng.integers(1, 301)), rng) for _ in range(48)]
    L = engines[SERVING_PARAMS[0]].L
    pool = rng.integers(0, engines[SERVING_PARAMS[0]].Q, (512, L), dtype=np.uint64)
    Cw = P.Circuit()
    Cw.output(Cw.gate("nand", Cw.input(), Cw.input()))
    t_imp = time.perf_counter()
    for sid in sids:  # warm-up: one gate per session imports every key
        S.submit(sid, Cw, pool[:2])
    S.run_until_idle()
    import_all_s = time.perf_counter() - t_imp
    tune = S.autotune(2368)
    key_bytes = S.stats()["resident_key_bytes"]
    points = [serving_point(S, sids, templates, pool, r, arrivals, rng) for r in rates]
    # the knee: the first offered load at which queueing takes over (median
    # latency over twice the lightest load's)
    mean_gates = sum(c.info()["gates"] for c in templates) / len(templates)
    for pt in points:
        pt["offered_gates_per_s"] = pt["offered_circuits_per_s"] * mean_gates
    knee = next((pt["offered_circuits_per_s"] for pt in points if pt["p50_ms"] > 2 * points[0]["p50_ms"]), None)
    S.set_key_budget(tight_keys * max(kbytes))
    tight = serving_point(S, sids, templates, pool, rates[1], arrivals, rng)
    tight["key_budget_bytes"] = tight_keys * max(kbytes)
    S.set_key_budget(0)
    # one client alone: an FheUint8 add (37 gates over its levels) on an idle server, five times
    Ca = P.Circuit()
    a_in, b_in = Ca.input_u8(), Ca.input_u8()
    Ca.outputs(Ca.u8_add(a_in, b_in))
    alone = []
    for r in range(6):
        ta = time.perf_counter()
        ja = S.submit(sids[0], Ca, pool[r:r + 16])
        while S.status(ja)["state"] != 2:
            S.step()
        if r:
            alone.append((time.perf_counter() - ta) * 1e3)
        S.forget(ja)
    S.close()
    for eng in engines.values():
        eng.close()
    best = max(points, key=lambda pt: pt["value"])
    return {"value": best["value"], "unit": "gate bootstraps/s", "saturation_rate": best["offered_circuits_per_s"],
            "p50_ms": best["p50_ms"], "p99_ms": best["p99_ms"], "knee_circuits_per_s": knee,
            "mean_gates_per_circuit": mean_gates, "points": points, "tight_key_budget": tight,
            "device_key_bytes": key_bytes, "import_all_keys_s": import_all_s, "autotune": tune,
            "alone_add_ms": float(np.median(alone)), "alone_add_levels": Ca.info()["levels"],
            "config": f"{sessions} managed sessions over {SERVING_PARAMS}, Poisson arrivals of circuits of "
                      f"U[1,300] gates from FheUint8 ops, {arrivals} per offered load {rates} circuits/s, admission "
                      f"by ciphertext + key bytes; tight point: key budget of {tight_keys} keys"}


def kernels_case(P, torch, device, count=296):
    """Small profiling case: each kernel of the path once after one warm-up
    (NI_8P, synthetic key): NTT forward/inverse, external product,
    automorphism, batched key switch, blind rotation, and one ragged step of
    the multi-session executor (key switch + blind rotation over 2 sessions)."""
    prm = "NI_8P"
    p = P.params(prm)
    N, L = p.rlwe_n, p.rlwe_n + 1
    eng = P.Engine(prm, device=device)
    key = eng.upload_key(*synthetic_key(p, 0x5EED))
    rng = np.random.default_rng(21)
    polys = torch.from_numpy(rng.integers(0, p.rlwe_q, (count, N), dtype=np.uint64).view(np.int64)).cuda()
    rl = torch.from_numpy(rng.integers(0, p.rlwe_q, (count, 2, N), dtype=np.uint64).view(np.int64)).cuda()
    idx = torch.arange(count, dtype=torch.int32, device="cuda") % p.lwe_n
    slots = torch.arange(count, dtype=torch.int32, device="cuda") % p.n_auto_keys
    lwe = torch.from_numpy(rng.integers(0, p.lwe_q, (count, L), dtype=np.uint64).view(np.int64)).cuda()
    ks_out = torch.empty((count, p.lwe_n + 1), dtype=torch.int32, device="cuda")
    ks = torch.from_numpy(rng.integers(0, p.lwe_q, (count, p.lwe_n + 1), dtype=np.uint64).astype(np.uint32)
                          .view(np.int32)).cuda()
    tv = torch.from_numpy(rng.integers(0, 6, count).astype(np.uint8)).cuda()
    br_out = torch.empty((count, L), dtype=torch.int64, device="cuda")
    S = P.Server(device=device, arena_bytes=1 << 28, max_items=count)
    eng2 = P.Engine("I_2P_LB_SR", device=device)
    key2 = eng2.upload_key(*synthetic_key(P.params("I_2P_LB_SR"), 0x5EEE))
    sids = [S.add_session(eng, key), S.add_session(eng2, key2)]
    C = P.Circuit()
    ins = [C.input() for _ in range(2 * count)]
    for i in range(count):
        C.output(C.gate("nand", ins[2 * i], ins[2 * i + 1]))
    inp = rng.integers(0, p.rlwe_q, (2 * count, L), dtype=np.uint64)
    for rep in range(2):  # warm-up, then the profiled launch of each kernel
        eng.ntt_forward_device(polys)
        eng.ntt_backward_device(polys)
        eng.rlwe_by_rgsw_device(key, rl, idx)
        eng.rlwe_auto_device(key, rl, slots)
        eng.lwe_key_switch_device(key, lwe, ks_out)
        eng.blind_rotate_device(key, ks, tv, br_out)
        S.submit(sids[0], C, inp[:2 * count])
        S.run_until_idle()
    torch.cuda.synchronize()
    S.close()
    for k, e in ((key, eng), (key2, eng2)):
        k.release()
        e.close()
    return {"mode": "kernels", "count": count, "param_set": prm}


def kernel_only(args):
    """One kernel on a batch of synthetic items, --warmup + --steps launches,
    printing the mean launch time (the small case profiled with ncu)."""
    import torch
    P = pz()
    p = P.params(args.param)
    L = p.rlwe_n + 1
    eng = P.Engine(args.param)
    if args.variant is not None:
        eng.pbs_variant = args.variant
    key = eng.upload_key(*synthetic_key(p, 0x5EED))
    rng = np.random.default_rng(99)
    B = args.batch
    if args.mode == "br-kernel":
        ks = rng.integers(0, p.lwe_q, (B, p.lwe_n + 1), dtype=np.uint64).astype(np.uint32)
        d_ks = torch.from_numpy(ks.view(np.int32)).cuda()
        d_tv = torch.from_numpy(rng.integers(0, 6, B).astype(np.uint8)).cuda()
        d_out = torch.empty((B, L), dtype=torch.int64, device="cuda")

        def launch():
            eng.blind_rotate_device(key, d_ks, d_tv, d_out)
    else:
        eng.set_ks_tile(args.ks_tile)
        lwe = torch.from_numpy(rng.integers(0, p.lwe_q, (B, L), dtype=np.uint64).view(np.int64)).cuda()
        d_out = torch.empty((B, p.lwe_n + 1), dtype=torch.int32, device="cuda")

        def launch():
            eng.lwe_key_switch_device(key, lwe, d_out)
    for _ in range(args.warmup):
        launch()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(args.steps):
        launch()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / max(args.steps, 1)
    out = {"mode": args.mode, "param_set": args.param, "batch": B, "variant": eng.pbs_variant,
           "ms_per_launch": ms, "items_per_s": B / ms * 1e3}
    if args.mode == "ks-kernel":
        out["ks_tile"] = args.ks_tile
    if args.mode == "br-kernel":
        out["modmuls_per_item"] = schedule_work(p, ks) / B
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity-check", action="store_true",
                    help="skip the oracle check of the measured wavefront's outputs")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the microbench / ragged / serving sub-results")
    ap.add_argument("--mode", default="wavefront",
                    choices=["wavefront", "br-kernel", "ks-kernel", "microbench", "ragged", "serving", "kernels",
                             "ni", "key-upload", "aggregate", "ni-aggregate"],
                    help="br-kernel / ks-kernel: only that kernel on --batch items (profiling case)")
    ap.add_argument("--batch", type=int, default=296)
    ap.add_argument("--param", default=PARAM)
    ap.add_argument("--variant", type=int, default=None,
                    help="blind-rotation launch-shape variant (wavefront mode: fixed instead of autotuned)")
    ap.add_argument("--ks-tile", type=int, default=64,
                    help="key-switch ciphertexts per CTA (8, 16, 32; 64 = tensor cores) with --variant or ks-kernel")
    ap.add_argument("--users", type=int, default=8, help="users of the ni-aggregate mode")
    ap.add_argument("--ref-step-seconds", type=float, default=REF_STEP_SECONDS,
                    help="wall time of one timed step of the CPU reference arm")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.mode in ("microbench", "ragged", "serving", "kernels", "ni", "key-upload", "aggregate", "ni-aggregate"):
        import torch
        P = pz()
        fn = {"microbench": lambda: microbench(P, torch, 0), "ragged": lambda: ragged_batch(P, 0),
              "serving": lambda: serving(P, 0), "kernels": lambda: kernels_case(P, torch, 0),
              "ni": lambda: ni_ingest_bench(P, torch, 0), "key-upload": lambda: key_upload_bench(P, 0),
              "aggregate": lambda: aggregate_bench(P, torch, 0),
              "ni-aggregate": lambda: ni_aggregate_bench(P, torch, 0, prm=args.param, users=args.users)}[args.mode]
        print(json.dumps({"mode": args.mode, **fn()}), flush=True)
        return
    if args.mode != "wavefront":
        return kernel_only(args)

    import torch
    dist, rank, world, local = dist_setup(args)
    torch.cuda.set_device(local)
    P = pz()
    p = P.params(PARAM)
    L = p.rlwe_n + 1

    eng = P.Engine(PARAM, device=local)
    key_arrays = synthetic_key(p, 0x5EED + rank)
    key = eng.upload_key(*key_arrays)
    C = wavefront_circuit(P)
    info = C.info()
    gates_per_step = info["gates"]
    rng = np.random.default_rng(1234 + rank)
    h_in = torch.from_numpy(rng.integers(0, p.rlwe_q, (info["inputs"], L), dtype=np.uint64).view(np.int64))
    h_in = h_in.pin_memory()
    h_out = torch.empty((info["outputs"], L), dtype=torch.int64).pin_memory()
    d_in = h_in.cuda()
    d_out = torch.empty((info["outputs"], L), dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()

    if args.variant is None:
        tune = eng.autotune(key, 2368)  # blind-rotation launch shape and key-switch tile for this GPU
    else:  # a fixed launch shape (profiling: the same kernels with and without a profiler)
        eng.pbs_variant = args.variant
        eng.set_ks_tile(args.ks_tile)
        tune = {"variant": args.variant, "ms": None, "ks_tile": args.ks_tile, "fixed": True}
    # warm-up step 1 is a direct run (sets kernel attributes, binds the
    # circuit to the device); the circuit is then captured and replayed
    C.run_device(eng, key, d_in, d_out)
    torch.cuda.synchronize()
    C.capture_graph(eng, key, d_in, d_out)
    for _ in range(max(args.warmup - 1, 0)):
        C.replay_graph()
    torch.cuda.synchronize()

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clocks:
        for i in range(args.steps):
            evs[i][0].record()
            C.replay_graph()
            evs[i][1].record()
        torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    if dist:
        dist.barrier()
    total_ms = max_over_ranks(dist, sum(step_ms), "cuda")
    value = world * gates_per_step * args.steps / (total_ms / 1e3)

    # e2e: host buffers through the synchronous C-ABI call (copies inside)
    e2e_ms = []
    for i in range(args.steps):
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        P._lib.check(P._lib.lib().pz_circuit_run(eng.h, key.h, C.h,
                                                 P._lib.ctypes.cast(h_in.data_ptr(), P._lib.u64p),
                                                 P._lib.ctypes.cast(h_out.data_ptr(), P._lib.u64p)),
                     eng.h, "pz_circuit_run")
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_total = max_over_ranks(dist, sum(e2e_ms), "cuda")
    e2e_value = world * gates_per_step * args.steps / (e2e_total / 1e3)

    # dominant kernel: blind rotation alone on whole waves of the autotuned
    # launch shape (ROOFLINE_WAVES x the items resident at once)
    B = ROOFLINE_WAVES * eng.pbs_slots()
    ks = rng.integers(0, p.lwe_q, (B, p.lwe_n + 1), dtype=np.uint64).astype(np.uint32)
    d_ks = torch.from_numpy(ks.view(np.int32)).cuda()
    d_tv = torch.from_numpy(rng.integers(0, 6, B).astype(np.uint8)).cuda()
    d_br = torch.empty((B, L), dtype=torch.int64, device="cuda")
    eng.blind_rotate_device(key, d_ks, d_tv, d_br)
    torch.cuda.synchronize()
    reps = 3
    ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ea.record()
    for _ in range(reps):
        eng.blind_rotate_device(key, d_ks, d_tv, d_br)
    eb.record()
    torch.cuda.synchronize()
    br_ms = ea.elapsed_time(eb) / reps
    modmuls = schedule_work(p, ks)
    achieved = modmuls * C_MM / (br_ms / 1e3) / 1e12  # T IMAD/s
    peak = P.probe_imad_rate(local) / 1e12
    # the other pipes the butterflies use (the quotient runs on the FP64 pipe and the conversion unit)
    pipes = {k: v / 1e12 for k, v in P.probe_pipe_rates(local).items()}
    traffic, traffic_source = traffic_record(P, tune["variant"], B)

    plain = None
    if not args.no_plain and rank == 0:
        plain = plain_form(P, torch, local)

    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        extras["microbench"] = microbench(P, torch, local)
        extras["ragged"] = ragged_batch(P, local)
        extras["serving"] = serving(P, local)
        extras["ni_ingest"] = ni_ingest_bench(P, torch, local)
        extras["key_upload"] = key_upload_bench(P, local)
        extras["aggregate"] = aggregate_bench(P, torch, local)
        extras["ni_aggregate"] = ni_aggregate_bench(P, torch, local)

    cpu, parity = None, None
    okey_c = mix = None
    if rank == 0 and (not args.no_cpu_baseline or not args.no_parity_check):
        _, _, okey_c, mix = cpu_reference_setup(key_arrays)
    if rank == 0 and not args.no_parity_check:
        parity = wavefront_parity_check(p, okey_c, h_in, h_out, d_out)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads, physical = host_cores()
        count = cpu_calibrated_sample(p, key_arrays, okey_c, mix, threads, 12.0)
        rate, count, dt = cpu_gate_sample(p, key_arrays, threads, count, mix, okey=okey_c)
        cpu = {"value": rate, "unit": "gate bootstraps/s", "cores": threads, "physical_cores": physical,
               "kind": "port",
               "sample": f"{count} independent NI_8P gates in the wavefront's gate mix, {threads} threads on "
                         f"{physical} physical cores, {dt:.1f} s"}

    if rank == 0:
        launches_per_step = 2 * info["levels"] + 1
        line = {
            "metric": "gate bootstraps/sec", "value": value, "unit": "gate bootstraps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded uniform keys and ciphertexts with the reference's shapes)",
            "config": {**WORKLOAD_CONFIG, "gates_per_step": gates_per_step, "levels": info["levels"],
                       "max_level_width": info["max_level_width"],
                       "l2": "inputs (537 MB/step) larger than L2; server key resident",
                       "pbs_variant": tune["variant"], "ks_tile": tune["ks_tile"]},
            "latency_ms": {"p50": statistics.median(step_ms), "p99": float(np.percentile(step_ms, 99)),
                           "what": "completion time of every circuit in the wavefront"},
            "e2e": {"value": e2e_value, "unit": "gate bootstraps/s",
                    "h2d_bytes_per_step": int(info["inputs"] * L * 8),
                    "d2h_bytes_per_step": int(info["outputs"] * L * 8)},
            "gpu_launches": launches_per_step * args.steps,
            "roofline": {"bound": "int", "kernel": "pbs_kernel (blind rotation)", "achieved": achieved,
                         "peak": peak, "unit": "TIMAD/s", "frac": achieved / peak, "traffic": traffic,
                         "traffic_source": traffic_source,
                         "peak_source": "pz_probe_imad_rate on this GPU (MEASURED_PEAKS.json has no integer peak)",
                         "launch_ms": br_ms, "bootstraps_per_launch": B,
                         "modmuls_per_bootstrap": modmuls / B,
                         "pipe_rates_tips": pipes,
                         "convention": "10 IMAD per 64-bit modmul; the butterflies' quotient runs on the FP64 "
                                       "pipe and the conversion unit, so part of the work is off the IMAD pipe"},
            "plain": plain,
            "parity": parity,
            **extras,
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    C.close()
    key.release()
    eng.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
