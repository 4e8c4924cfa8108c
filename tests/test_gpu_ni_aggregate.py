"""Non-interactive server-key aggregation on the GPU vs the oracle, word for
word (aggregate_non_interactive_multi_party_server_key_shares, bool/
evaluator.rs:1222-1622), and the aggregated key evaluating gates on inputs
ingested with the aggregated ui_to_s keys."""
import numpy as np
import pytest

from conftest import oracle, pz, to_dev, to_host

pytestmark = pytest.mark.gpu

# device share field -> oracle share field
FIELDS = dict(ui_to_s_ksk="ui_to_s_ksk", ksk_zero_encs="ksk_zero_encs", self_leader_cts="self_leader",
              not_leader_cts="not_leader", rgsw_zero_encs="zero_encs", auto_keys="auto_keys", lwe_ksk="lwe_ksk")


def random_shares(ev, users, seed):
    """Uniform canonical share arrays of the reference's shapes (parity only)."""
    g = np.random.default_rng(seed)
    i = ev.info
    N, n, Q = ev.N, ev.n, ev.Q
    mx, ml = max(i.rgrg_d_a, i.rgrg_d_b), max(i.rlrg_d_a, i.rlrg_d_b)
    out = []
    for j in range(users):
        b, e = ev.lwe_segment(j, users)
        out.append(dict(ui_to_s_ksk=g.integers(0, Q, (50, N), dtype=np.uint64),
                        ksk_zero_encs=g.integers(0, Q, (users - 1, 50, N), dtype=np.uint64),
                        self_leader=g.integers(0, Q, (e - b, ml, N), dtype=np.uint64),
                        not_leader=g.integers(0, Q, (n - (e - b), mx, N), dtype=np.uint64),
                        zero_encs=g.integers(0, Q, (n, i.rgrg_d_a, N), dtype=np.uint64),
                        auto_keys=g.integers(0, Q, (i.w + 1, i.auto_d, N), dtype=np.uint64),
                        lwe_ksk=g.integers(0, i.lwe_q, i.lwe_d * N, dtype=np.uint64)))
    return out


def to_device(shares):
    return [{k: to_dev(sh[v]) for k, v in FIELDS.items()} for sh in shares]


def device_aggregate(eng, ev, crs, dshares):
    import torch
    i, N = ev.info, ev.N
    users = len(dshares)
    ksk = torch.zeros((users, 50, N), dtype=torch.int64, device="cuda")
    rgsw = torch.zeros((ev.n, 4, N), dtype=torch.int64, device="cuda")
    auto = torch.zeros((i.w + 1, i.auto_d, N), dtype=torch.int64, device="cuda")
    lwe = torch.zeros(i.lwe_d * N, dtype=torch.int64, device="cuda")
    eng.ni_aggregate_device(crs, dshares, ksk, rgsw, auto, lwe)
    torch.cuda.synchronize()
    return to_host(ksk), to_host(rgsw), to_host(auto), to_host(lwe)


def check_against_oracle(ev, crs, shares, got, ranges):
    ksk, rgsw, auto, lwe = got
    for i0, i1 in ranges:
        w_ksk, w_rgsw, w_auto, w_lwe = ev.ni_aggregate(crs, shares, i0, i1)
        assert np.array_equal(rgsw[i0:i1], w_rgsw), (i0, i1)
    assert np.array_equal(ksk, w_ksk)
    assert np.array_equal(auto, w_auto)
    assert np.array_equal(lwe, w_lwe)


@pytest.mark.parametrize("param,users", [("NI_4P_LB_SR", 3), ("NI_8P", 4)])
def test_ni_aggregate_matches_oracle(gpu_available, param, users):
    """Random shares: every aggregated word equals the oracle's, at indices led
    by each user and across the segment boundaries."""
    O = oracle()
    ev = O.Evaluator(param)
    crs = bytes(range(100, 132))
    shares = random_shares(ev, users, 5)
    eng = pz().Engine(param)
    got = device_aggregate(eng, ev, crs, to_device(shares))
    per = -(-ev.n // users)
    ranges = [(0, 1), (per - 1, per + 1), (ev.n - 1, ev.n)]
    check_against_oracle(ev, crs, shares, got, ranges)


def test_ni_aggregated_key_runs_gates(gpu_available):
    """Two users' genuine NI shares (NI_2P): device aggregation == oracle; the
    server key and ui_to_s keys from pz_ni_aggregate_server_key ingest each
    user's NI-encrypted bools (decrypting under the ideal secret) and evaluate
    NAND gates across the two users' inputs."""
    O = oracle()
    ev = O.Evaluator("NI_2P")
    users, N = 2, ev.N
    crs = b"\x5a" * 32
    s, z, sp, zp = ev.client_keys(users)
    up = ev.client_keys(users, seed_base=7)[2]
    auto_b, lwe_b = ev.gen_seeded_auto_lwe(s, z, O.ni_crs_seed(crs, 0), O.ni_crs_seed(crs, 1))
    shares = []
    for j in range(users):
        sh = ev.ni_gen_share(crs, j, users, sp[j], up[j], zp[j], bytes([j + 1]) * 32)
        sh["auto_keys"] = auto_b if j == 0 else np.zeros_like(auto_b)
        sh["lwe_ksk"] = lwe_b if j == 0 else np.zeros_like(lwe_b)
        shares.append(sh)
    eng = pz().Engine("NI_2P")
    dshares = to_device(shares)
    got = device_aggregate(eng, ev, crs, dshares)
    check_against_oracle(ev, crs, shares, got, [(0, 2), (ev.n // 2 - 1, ev.n // 2 + 1), (ev.n - 1, ev.n)])
    key, ksks = eng.ni_aggregate_server_key(crs, dshares)
    g = np.random.default_rng(12)
    k = 24
    lwes = []
    for j in range(users):
        bits = g.integers(0, 2, k).astype(np.uint8)
        seed = bytes([0x30 + j]) * 32
        b = ev.ni_encrypt_bools(up[j], bits, seed)
        lw = eng.ni_ingest(ksks[j], seed, b, k)
        assert np.array_equal(ev.decrypt_bool(s, lw), bits)
        lwes.append((bits, lw))
    (b0, l0), (b1, l1) = lwes
    out = eng.gate_batch(key, np.full(k, O.GATES["nand"], np.uint8), l0, l1)
    assert np.array_equal(ev.decrypt_bool(s, out), 1 - (b0 & b1))
