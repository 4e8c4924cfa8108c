"""Multi-session executor on the GPU: ragged launches mixing parameter sets
and server keys, continuous batching, admission by device bytes.  Every job's
output must equal, word for word, the same circuit run alone on its own
session (the single-session path, itself pinned to the oracle), decrypt to
the plaintext result, and -- for one job -- equal the oracle's sequential
gate-by-gate evaluation."""
import numpy as np
import pytest

from conftest import oracle, oracle_setup, pz

pytestmark = pytest.mark.gpu

_SESS = {}


def session(param):
    """Engine + device key from the oracle's client secrets (decryptable)."""
    if param not in _SESS:
        ev, secrets, coeff, okey = oracle_setup(param)
        eng = pz().Engine(param)
        key = eng.upload_key(coeff.rgsw, coeff.autos, coeff.ksk)
        _SESS[param] = (eng, key, ev, secrets[0], okey)
    return _SESS[param]


def synthetic_session(param, seed):
    """Engine + a uniform synthetic key: a second user of the same parameter set."""
    eng = pz().Engine(param)
    p = eng.p
    rng = np.random.default_rng(seed)
    N, n = p.rlwe_n, p.lwe_n
    rgsw = rng.integers(0, p.rlwe_q, (n, p.rgsw_rows, N), dtype=np.uint64)
    autos = rng.integers(0, p.rlwe_q, (p.n_auto_keys, p.auto_rows, N), dtype=np.uint64)
    ksk = rng.integers(0, p.lwe_q, (p.lwe_d * N, n + 1), dtype=np.uint64)
    return eng, eng.upload_key(rgsw, autos, ksk)


def circuit(op):
    C = pz().Circuit()
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


def enc_pair(ev, s, x, y, seed):
    r = oracle().Rng(bytes([seed & 0xFF]) * 32)
    bits = np.array([(v >> i) & 1 for v in (x, y) for i in range(8)])
    return ev.encrypt_bool(r, s, bits).reshape(16, ev.L)


def dec_u8(ev, s, cts):
    bits = ev.decrypt_bool(s, cts.reshape(-1, ev.L))
    return sum(int(b) << i for i, b in enumerate(bits[:8]))


def expect(op, ev, s, out, x, y):
    if op == "add":
        assert dec_u8(ev, s, out) == (x + y) % 256
    elif op == "mul":
        assert dec_u8(ev, s, out) == (x * y) % 256
    elif op == "lt":
        assert ev.decrypt_bool(s, out.reshape(-1, ev.L))[0] == int(x < y)
    elif op == "div_rem":
        q = 255 if y == 0 else x // y
        r = x if y == 0 else x % y
        assert dec_u8(ev, s, out[:8]) == q
        assert dec_u8(ev, s, out[8:16]) == r
        assert ev.decrypt_bool(s, out[16:17])[0] == int(y == 0)


@pytest.mark.parametrize("policy", [0, 1])
def test_ragged_mixed_parameter_sets(gpu_available, policy):
    """One step mixes I_2P, I_4P, I_8P and NI_8P sessions (n = 580/620/660/660,
    d_ks = 12/13/14/14, br_q = 2^11/2^11/2^12/2^12) running add, lt and
    div_rem (divisor 0 in one job); every output equals the job run alone and
    decrypts right, under both step schedules (all ready levels; critical path
    first)."""
    P = pz()
    params = ["I_2P_LB_SR", "I_4P", "I_8P", "NI_8P"]
    S = P.Server(device=0, arena_bytes=1 << 29, max_items=4096)
    S.set_schedule(policy)
    sids = {p: S.add_session(*session(p)[:2]) for p in params}
    rng = np.random.default_rng(3)
    jobs = []
    for k, p in enumerate(params):
        eng, key, ev, s, _ = session(p)
        for op in ["add", "lt", "div_rem"]:
            x, y = (int(v) for v in rng.integers(0, 256, 2))
            if op == "div_rem" and k == 0:
                y = 0
            C = circuit(op)
            inp = enc_pair(ev, s, x, y, 17 * k + len(jobs))
            jobs.append((p, op, x, y, C, inp, S.submit(sids[p], C, inp)))
    S.run_until_idle()
    st = S.stats()
    assert st["done"] == len(jobs) and st["failed"] == 0 and st["arena_slots_used"] == 0
    # every step was one ragged launch pair: steps == deepest circuit
    assert st["steps"] == max(C.info()["levels"] for *_, C, _, _ in jobs)
    for p, op, x, y, C, inp, j in jobs:
        eng, key, ev, s, _ = session(p)
        got = S.result(j)
        alone = C.run(eng, key, inp)
        assert np.array_equal(got, alone), f"{p} {op}: mixed-batch words differ from the job alone"
        expect(op, ev, s, got, x, y)


def test_ragged_job_matches_sequential_oracle(gpu_available):
    """An I_2P addition run in a mixed batch equals the oracle's gate-by-gate
    evaluation of shortint add (ops.rs) word for word."""
    P = pz()
    S = P.Server(device=0, arena_bytes=1 << 27, max_items=1024)
    e2, k2, ev, s, okey = session("I_2P_LB_SR")
    s_i2 = S.add_session(e2, k2)
    s_n8 = S.add_session(*session("NI_8P")[:2])
    inp = enc_pair(ev, s, 201, 77, 99)
    j = S.submit(s_i2, circuit("add"), inp)
    ev8, s8 = session("NI_8P")[2:4]
    S.submit(s_n8, circuit("lt"), enc_pair(ev8, s8, 3, 4, 5))
    S.run_until_idle()
    want = okey.u8_op("add", inp[:8], inp[8:16])[0]
    assert np.array_equal(S.result(j), want)
    assert dec_u8(ev, s, S.result(j)) == (201 + 77) % 256


def test_continuous_batching_same_alone_and_in_the_mix(gpu_available):
    """Jobs of three sessions (two users of NI_8P with different keys, one of
    I_2P) arrive over several steps; results equal each job run alone."""
    P = pz()
    S = P.Server(device=0, arena_bytes=1 << 28, max_items=2048)
    e8, k8, ev8, s8, _ = session("NI_8P")
    e8b, k8b = synthetic_session("NI_8P", 11)
    e2, k2, ev2, s2, _ = session("I_2P_LB_SR")
    sess = [(S.add_session(e8, k8), e8, k8), (S.add_session(e8b, k8b), e8b, k8b), (S.add_session(e2, k2), e2, k2)]
    rng = np.random.default_rng(5)
    plan = []  # (arrival step, session index, op)
    for t in range(10):
        for _ in range(int(rng.poisson(0.8))):
            plan.append((t, int(rng.integers(0, 3)), ["add", "lt", "mul"][int(rng.integers(0, 3))]))
    assert len(plan) >= 4
    jobs, step, pi = [], 0, 0
    while pi < len(plan) or S.stats()["active"] or S.stats()["pending"]:
        while pi < len(plan) and plan[pi][0] <= step:
            _, si, op = plan[pi]
            sid, eng, key = sess[si]
            L = eng.L
            inp = np.random.default_rng(1000 + pi).integers(0, eng.Q, (16, L), dtype=np.uint64)
            C = circuit(op)
            jobs.append((si, op, C, inp, S.submit(sid, C, inp)))
            pi += 1
        S.step()
        step += 1
    for si, op, C, inp, j in jobs:
        _, eng, key = sess[si]
        assert np.array_equal(S.result(j), C.run(eng, key, inp)), f"job {j} ({op}) differs in the mix"
        assert S.status(j)["latency_ms"] > 0


def test_admission_waits_for_device_bytes(gpu_available):
    """An arena with room for two multiplications at a time: the rest queue,
    results are unchanged."""
    P = pz()
    e2, k2, ev, s, _ = session("I_2P_LB_SR")
    C = circuit("mul")
    need = C.info()["inputs"] + C.info()["gates"]
    S = P.Server(device=0, arena_bytes=(2 * need + 10) * e2.L * 8, max_items=512)
    sid = S.add_session(e2, k2)
    vals = [(13, 17), (250, 3), (0, 99), (128, 2)]
    ins = [enc_pair(ev, s, x, y, 40 + i) for i, (x, y) in enumerate(vals)]
    jobs = [S.submit(sid, circuit("mul"), inp) for inp in ins]
    S.step()
    assert [S.status(j)["state"] for j in jobs] == [1, 1, 0, 0]
    S.run_until_idle()
    for (x, y), inp, j in zip(vals, ins, jobs):
        assert np.array_equal(S.result(j), C.run(e2, k2, inp))
        assert dec_u8(ev, s, S.result(j)) == (x * y) % 256
    assert S.status(jobs[3])["queue_ms"] > 0


def test_autotune_then_run(gpu_available):
    P = pz()
    S = P.Server(device=0, arena_bytes=1 << 28, max_items=1024)
    e8, k8, ev8, s8, _ = session("NI_8P")
    e2, k2, ev2, s2, _ = session("I_2P_LB_SR")
    a, b = S.add_session(e8, k8), S.add_session(e2, k2)
    t = S.autotune(296)
    assert t["variant"] in (0, 1, 2, 4) and t["ms"] > 0 and t["grid_limit"] >= 0
    inp = enc_pair(ev2, s2, 9, 200, 7)
    C = circuit("lt")
    j = S.submit(b, C, inp)
    S.submit(a, circuit("add"), enc_pair(ev8, s8, 1, 2, 3))
    S.run_until_idle()
    assert np.array_equal(S.result(j), C.run(e2, k2, inp))
    assert ev2.decrypt_bool(s2, S.result(j))[0] == 1


def test_managed_sessions_evict_and_reimport_keys(gpu_available):
    """Managed sessions with a key budget of one I_2P key: every job brings
    its session's key in (evicting the other, idle one) from the device-form
    blob; a session whose key was evicted and imported again gives the same
    words as the job run alone, and every output decrypts right."""
    P = pz()
    eng, key, ev, s, _ = session("I_2P_LB_SR")
    blob = key.export()
    S = P.Server(device=0, arena_bytes=1 << 27, max_items=1024)
    a = S.add_managed_session(eng, blob)
    b = S.add_managed_session(eng, blob)
    S.set_key_budget(len(blob) - 64)
    C = circuit("add")
    outs = []
    for k, sid in enumerate([a, b, a]):
        x, y = 17 * k + 5, 250 - 9 * k
        inp = enc_pair(ev, s, x, y, 40 + k)
        j = S.submit(sid, C, inp)
        S.run_until_idle()
        assert S.resident(sid) and not S.resident(b if sid == a else a)
        got = S.result(j)
        assert np.array_equal(got, C.run(eng, key, inp)), f"job {k}: words differ from the job alone"
        expect("add", ev, s, got, x, y)
        outs.append(got)
    st = S.stats()
    assert st["key_imports"] == 3 and st["key_evictions"] == 2 and st["failed"] == 0
    assert eng.device_error() == 0


@pytest.mark.parametrize("grid_limit", [0, 5])
def test_staged_key_ragged_shape(gpu_available, grid_limit):
    """The staged-key ragged blind rotation (launch shape 4: every operation's
    key rows come into shared memory by bulk copy, each item with its own
    session's key) -- one CTA per gate, and a grid of 5 CTAs that each run
    many items in turn -- gives the words of every job run alone."""
    P = pz()
    S = P.Server(device=0, arena_bytes=1 << 28, max_items=4096)
    S.set_launch(4, grid_limit)
    params = ["I_2P_LB_SR", "I_8P", "NI_8P"]
    sids = {p: S.add_session(*session(p)[:2]) for p in params}
    jobs = []
    for k, p in enumerate(params):
        eng, key, ev, s, _ = session(p)
        for op in ["mul", "lt"]:
            x, y = 31 * k + 7, 200 - 13 * k
            C = circuit(op)
            inp = enc_pair(ev, s, x, y, 60 + 2 * k + (op == "lt"))
            jobs.append((p, op, x, y, C, inp, S.submit(sids[p], C, inp)))
    S.run_until_idle()
    assert S.stats()["failed"] == 0
    for p, op, x, y, C, inp, j in jobs:
        eng, key, ev, s, _ = session(p)
        got = S.result(j)
        assert np.array_equal(got, C.run(eng, key, inp)), f"{p} {op}: words differ from the job alone"
        expect(op, ev, s, got, x, y)
    assert session("NI_8P")[0].device_error() == 0
