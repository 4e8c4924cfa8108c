"""Multi-session executor bookkeeping on the host (dry-run server, no GPU):
admission by device bytes in arrival order, one circuit level per job per
step, continuous batching of late arrivals, latency accounting."""
import pytest

from conftest import pz


def u8_circuit(op):
    P = pz()
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


def slots(C):
    i = C.info()
    return i["inputs"] + i["gates"]


def L_of(param):
    return pz().params(param).rlwe_n + 1


def make_server(arena_slots, params=("I_2P_LB_SR", "NI_8P"), max_items=4096):
    P = pz()
    S = P.Server(device=P.DRY_RUN, arena_bytes=arena_slots * L_of(params[0]) * 8, max_items=max_items)
    sids = [S.add_virtual_session(P.param_id(p)) for p in params]
    return S, sids


def test_levels_advance_one_per_step():
    S, (s0, s1) = make_server(1 << 16)
    circs = [u8_circuit("add"), u8_circuit("lt"), u8_circuit("mul")]
    jobs = [S.submit(s0 if i % 2 == 0 else s1, c) for i, c in enumerate(circs)]
    sizes = [c.level_sizes() for c in circs]
    depth = max(len(s) for s in sizes)
    for step in range(depth):
        ran = S.step()
        assert ran == sum(s[step] for s in sizes if step < len(s))
        for j, s in zip(jobs, sizes):
            want = pz().server.DONE if step + 1 >= len(s) else pz().server.RUNNING
            assert S.status(j)["state"] == want
    st = S.stats()
    assert st["done"] == 3 and st["active"] == 0 and st["pending"] == 0
    assert st["arena_slots_used"] == 0
    assert st["gates"] == sum(c.info()["gates"] for c in circs)


def test_admission_by_device_bytes_fifo():
    a = u8_circuit("mul")
    need = slots(a)
    S, (s0, _) = make_server(2 * need + need // 2)  # room for two such jobs, not three
    jobs = [S.submit(s0, a) for _ in range(3)]
    S.step()
    states = [S.status(j)["state"] for j in jobs]
    assert states == [pz().server.RUNNING, pz().server.RUNNING, pz().server.PENDING]
    assert S.stats()["arena_slots_used"] == 2 * need
    S.run_until_idle()
    assert all(S.status(j)["state"] == pz().server.DONE for j in jobs)
    # the third job waited for a whole circuit: it queued, the first two did not
    assert S.status(jobs[2])["queue_ms"] >= S.status(jobs[0])["queue_ms"]
    assert S.stats()["arena_slots_used"] == 0


def test_job_larger_than_arena_fails_without_blocking_others():
    big, small = u8_circuit("mul"), u8_circuit("lt")
    S, (s0, s1) = make_server(slots(big) - 1)
    jb = S.submit(s0, big)
    js = S.submit(s1, small)
    S.run_until_idle()
    assert S.status(jb)["state"] == pz().server.FAILED
    assert S.status(js)["state"] == pz().server.DONE
    assert S.stats()["failed"] == 1


def test_late_arrival_joins_running_batch():
    m, l = u8_circuit("mul"), u8_circuit("lt")
    ms, ls = m.level_sizes(), l.level_sizes()
    S, (s0, s1) = make_server(1 << 16)
    S.submit(s0, m)
    for k in range(3):
        assert S.step() == ms[k]
    S.submit(s1, l)  # arrives while the multiplication is mid-circuit
    assert S.step() == ms[3] + ls[0]  # one step carries both sessions' gates
    assert S.step() == ms[4] + ls[1]


def test_stats_and_forget():
    S, (s0, s1) = make_server(1 << 14)
    st = S.stats()
    assert st["sessions"] == 2
    P = pz()
    assert st["key_bytes"] > 2 * P.params("I_2P_LB_SR").lwe_n * 4 * 2048 * 8
    j = S.submit(s0, u8_circuit("add"))
    with pytest.raises(RuntimeError):
        S.forget(j)  # not finished
    S.run_until_idle()
    lat = S.status(j)["latency_ms"]
    assert lat >= 0
    S.forget(j)
    with pytest.raises(RuntimeError):
        S.status(j)


def test_mixed_ring_rejected():
    P = pz()
    S = P.Server(device=P.DRY_RUN, arena_bytes=1 << 24, max_items=64)
    S.add_virtual_session(P.param_id("NI_8P"))
    with pytest.raises(RuntimeError):
        S.add_virtual_session(P.param_id("SP_TEST"))  # N = 512: another ring


def _ragged_mix(S, sids, per_op):
    ops = ["add", "mul", "div_rem", "lt"]
    circs = {op: u8_circuit(op) for op in ops}
    for sid in sids:
        for k in range(4 * per_op):
            S.submit(sid, circs[ops[k % 4]])
    return circs


def _run_counts(S):
    counts = []
    while S.stats()["active"] or S.stats()["pending"]:
        counts.append(S.step())
    return counts


def test_critical_path_schedule_keeps_depth_and_fills_tiers():
    """CRITICAL_PATH: the batch still ends after (deepest circuit) steps and
    runs every gate once; the wide first levels of the short jobs are spread
    over steps the deep jobs leave part-empty, so fewer waves are launched
    (tiers: 148 SMs, 3 CTAs per SM at the default launch variant)."""
    P = pz()
    waves = {}
    for policy in (P.server.SCHEDULE_ALL_READY, P.server.SCHEDULE_CRITICAL_PATH):
        S, sids = make_server(1 << 22, params=("I_2P_LB_SR", "I_4P", "I_8P"), max_items=16384)
        S.set_launch(1)
        S.set_schedule(policy)
        circs = _ragged_mix(S, sids, 16)
        counts = _run_counts(S)
        depth = max(c.info()["levels"] for c in circs.values())
        assert len(counts) == depth
        assert sum(counts) == sum(c.info()["gates"] for c in circs.values()) * 16 * len(sids)
        assert S.stats()["done"] == 4 * 16 * len(sids)
        # launch-time model: partial waves by their SM tier, whole waves of 444
        w = 0.0
        for g in counts:
            full, rem = divmod(g, 444)
            w += full + (0 if rem == 0 else (1 / 3 if rem <= 148 else 2 / 3 if rem <= 296 else 1))
        waves[policy] = w
    assert waves[P.server.SCHEDULE_CRITICAL_PATH] < 0.85 * waves[P.server.SCHEDULE_ALL_READY]


def test_schedule_policy_rejects_unknown():
    S, _ = make_server(1 << 16)
    with pytest.raises(Exception):
        S.set_schedule(7)


def key_bytes(param):
    p = pz().params(param)
    stride = (p.lwe_n + 1 + 31) // 32 * 32
    return (p.lwe_n * p.rgsw_rows * p.rlwe_n * 8 + p.n_auto_keys * p.auto_rows * p.rlwe_n * 8 +
            p.lwe_d * p.rlwe_n * stride * 4)


def test_managed_keys_admission_and_lru_eviction():
    """Admission by ciphertext + key bytes: with a key budget for two NI_8P
    keys and three managed sessions, a job of the third session evicts the
    least recently used idle key; a session with a job in flight is never
    evicted (a job waits instead, in arrival order); a key larger than the
    budget fails its job."""
    P = pz()
    S = P.Server(device=P.DRY_RUN, arena_bytes=(1 << 16) * L_of("NI_8P") * 8, max_items=4096)
    kb = key_bytes("NI_8P")
    a, b, c = (S.add_virtual_managed_session(P.param_id("NI_8P")) for _ in range(3))
    S.set_key_budget(2 * kb)
    assert not any(S.resident(x) for x in (a, b, c))
    add = u8_circuit("add")
    ja = S.submit(a, add)
    S.run_until_idle()
    jb = S.submit(b, add)
    S.run_until_idle()
    st = S.stats()
    assert st["key_imports"] == 2 and st["key_evictions"] == 0 and st["resident_key_bytes"] == 2 * kb
    # a was used least recently: the first job of c evicts it
    jc = S.submit(c, add)
    S.step()
    assert S.resident(c) and S.resident(b) and not S.resident(a)
    assert S.stats()["key_evictions"] == 1
    # while c and b both have jobs in flight, a new job of a cannot get its key: it waits
    S.submit(b, u8_circuit("mul"))
    S.step()
    ja2 = S.submit(a, add)
    S.step()
    assert S.status(ja2)["state"] == P.server.PENDING and not S.resident(a)
    S.run_until_idle()
    # c finished first (15 levels vs mul's), so c's idle key made room for a
    assert S.status(ja2)["state"] == P.server.DONE and S.resident(a) and not S.resident(c)
    for j in (ja, jb, jc, ja2):
        assert S.status(j)["state"] == P.server.DONE
    st = S.stats()
    assert st["key_imports"] == 4 and st["key_evictions"] == 2 and st["resident_key_bytes"] <= 2 * kb
    # a key that can never fit the budget fails its job
    S.set_key_budget(kb // 2)
    jx = S.submit(c, add)
    S.step()
    assert S.status(jx)["state"] == P.server.FAILED


def test_unmanaged_sessions_ignore_the_key_budget():
    """Sessions added with a resident key are always resident; the key budget
    governs managed sessions only."""
    P = pz()
    S, (s0, s1) = make_server(1 << 16)
    S.set_key_budget(1)
    j = S.submit(s0, u8_circuit("lt"))
    S.run_until_idle()
    assert S.status(j)["state"] == P.server.DONE and S.resident(s0) and S.resident(s1)
    assert S.stats()["key_imports"] == 0


def test_lowering_the_key_budget_evicts_idle_keys():
    """Keys already resident over a lowered budget are evicted at the next
    step, least recently used first, idle sessions only."""
    P = pz()
    S = P.Server(device=P.DRY_RUN, arena_bytes=(1 << 16) * L_of("NI_8P") * 8, max_items=4096)
    kb = key_bytes("NI_8P")
    sids = [S.add_virtual_managed_session(P.param_id("NI_8P")) for _ in range(4)]
    for sid in sids:  # all four resident, used in order
        S.submit(sid, u8_circuit("lt"))
        S.run_until_idle()
    assert all(S.resident(x) for x in sids)
    j = S.submit(sids[0], u8_circuit("mul"))  # sids[0] busy, most recently used
    S.step()
    S.set_key_budget(2 * kb)
    S.step()
    # sids[1] and sids[2] were the least recently used idle keys
    assert [S.resident(x) for x in sids] == [True, False, False, True]
    assert S.stats()["resident_key_bytes"] == 2 * kb and S.stats()["key_evictions"] == 2
    S.run_until_idle()
    assert S.status(j)["state"] == P.server.DONE
