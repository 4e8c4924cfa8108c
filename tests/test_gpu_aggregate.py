"""Server-key aggregation on the GPU: batched rgsw_by_rgsw_inplace
(runtime.rs:883-985) and the sequential RGSW step of the interactive
aggregation (evaluator.rs:1110-1200), word for word against the oracle, and
the aggregated RGSW still decrypts to the product."""
import numpy as np
import pytest

from conftest import oracle, oracle_setup, pz, to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("param", ["I_2P_LB_SR", "I_8P", "NI_8P"])
def test_rgsw_by_rgsw_matches_oracle(gpu_available, param):
    ev, _, _, _ = oracle_setup(param)
    eng = pz().Engine(param)
    rng = np.random.default_rng(21)
    count = 3
    r0 = rng.integers(0, ev.Q, (count, ev.rgsw_rows(0), ev.N), dtype=np.uint64)
    r1 = rng.integers(0, ev.Q, (count, ev.rgsw_rows(1), ev.N), dtype=np.uint64)
    r0[1, 0, :11] = 0
    want = np.stack([ev.rgsw_by_rgsw(r0[c], r1[c]) for c in range(count)])
    d0 = to_dev(r0)
    eng.rgsw_by_rgsw_device(d0, to_dev(r1))
    assert np.array_equal(to_host(d0).reshape(want.shape), want)


def test_aggregate_sequence_matches_oracle_and_decrypts(gpu_available):
    O = oracle()
    param = "I_4P"
    ev, (s, _, _, _), _, _ = oracle_setup(param)
    eng = pz().Engine(param)
    N, Q = ev.N, ev.Q

    def mono(k):
        m = np.zeros(N, np.uint64)
        m[k] = 1
        return m

    count, exps = 2, [5, 7, 2]  # three other users after the leader's X^3
    lead = np.stack([ev.rgsw_encrypt(s, mono(3), 0, bytes([0x80 + c]) * 32) for c in range(count)])
    others = np.stack([np.stack([ev.rgsw_encrypt(s, mono(k), 1, bytes([0x90 + 8 * t + c]) * 32)
                                 for c in range(count)]) for t, k in enumerate(exps)])
    want = lead.copy()
    for t in range(len(exps)):
        want = np.stack([ev.rgsw_by_rgsw(want[c], others[t, c]) for c in range(count)])
    d0 = to_dev(lead)
    eng.aggregate_rgsw_device(d0, to_dev(others))
    got = to_host(d0).reshape(want.shape)
    assert np.array_equal(got, want)
    # the m rows of RGSW(X^17) decrypt to beta X^17
    s_mod = np.array([int(x) % Q for x in s], dtype=np.uint64)
    out = np.empty(N, np.uint64)
    O.lib().orc_negacyclic_mul(Q, O._p(np.ascontiguousarray(got[0, 2])), O._p(s_mod), O._p(out), N)
    beta = 1 << (54 - ev.info.rlrg_logb)
    noise = (got[0, 3].astype(object) - out.astype(object) - mono(17).astype(object) * beta) % Q
    centred = np.array([int(v) if v < Q // 2 else int(v) - Q for v in noise])
    assert np.max(np.abs(centred)) < (1 << 34)


def _random_interactive_shares(ev, users, seed):
    g = np.random.default_rng(seed)
    i, N, Q = ev.info, ev.N, ev.Q
    out = []
    for j in range(users):
        b, e = ev.lwe_segment(j, users)
        out.append(dict(self_leader=g.integers(0, Q, (e - b, 4, N), dtype=np.uint64),
                        not_leader=g.integers(0, Q, (ev.n - (e - b), ev.rgsw_rows(1), N), dtype=np.uint64),
                        auto_keys=g.integers(0, Q, (i.w + 1, i.auto_d, N), dtype=np.uint64),
                        lwe_ksk=g.integers(0, i.lwe_q, i.lwe_d * N, dtype=np.uint64)))
    return out


def _to_device(shares):
    names = dict(self_leader_rgsws="self_leader", not_self_leader_rgsws="not_leader", auto_keys="auto_keys",
                 lwe_ksk="lwe_ksk")
    return [{k: to_dev(sh[v]) for k, v in names.items()} for sh in shares]


@pytest.mark.parametrize("param,users", [("I_2P_LB_SR", 2), ("I_8P", 3)])
def test_whole_aggregation_matches_oracle(gpu_available, param, users):
    """pz_aggregate_device (aggregate_interactive_multi_party_server_key_shares,
    evaluator.rs:1050-1200) on random shares == the oracle word for word: RGSWs at
    each segment boundary (leader changes), auto-key and LWE-KSK sums."""
    import torch
    O = oracle()
    ev = O.Evaluator(param)
    shares = _random_interactive_shares(ev, users, 3)
    eng = pz().Engine(param)
    i, N = ev.info, ev.N
    rgsw = torch.zeros((ev.n, 4, N), dtype=torch.int64, device="cuda")
    auto = torch.zeros((i.w + 1, i.auto_d, N), dtype=torch.int64, device="cuda")
    lwe = torch.zeros(i.lwe_d * N, dtype=torch.int64, device="cuda")
    eng.aggregate_device(_to_device(shares), rgsw, auto, lwe)
    torch.cuda.synchronize()
    got = to_host(rgsw)
    per = -(-ev.n // users)
    for i0, i1 in [(0, 1), (per - 1, per + 1), (ev.n - 1, ev.n)]:
        want, w_auto, w_lwe = ev.aggregate(shares, i0, i1)
        assert np.array_equal(got[i0:i1], want), (i0, i1)
    assert np.array_equal(to_host(auto), w_auto)
    assert np.array_equal(to_host(lwe), w_lwe)


def test_aggregated_server_key_runs_gates(gpu_available):
    """Two users' shares (RGSWs of X^{emb z_j[l]} under the ideal secret, CRS-seeded
    auto / LWE-KSK parts): pz_aggregate_server_key gives a key whose NAND gates
    decrypt correctly and equal the oracle's gates on the oracle's aggregate."""
    from test_oracle import interactive_shares
    O = oracle()
    ev = O.Evaluator("I_2P_LB_SR")
    crs = b"\x2a" * 32
    s, shares = interactive_shares(ev, crs, 2)
    eng = pz().Engine("I_2P_LB_SR")
    key = eng.aggregate_server_key(crs, _to_device(shares))
    rgsw, auto, lwe = ev.aggregate(shares)
    autos, ksk = ev.expand_seeded_key(auto, O.interactive_crs_seed(crs, 1), lwe, O.interactive_crs_seed(crs, 2))
    okey = ev.key(O.ServerKeyCoeff(rgsw, autos, ksk))
    r = O.Rng(b"\x09" * 32)
    bits0, bits1 = np.array([0, 1, 1, 0, 1, 0, 1, 1]), np.array([0, 0, 1, 1, 1, 1, 0, 1])
    c0, c1 = ev.encrypt_bool(r, s, bits0), ev.encrypt_bool(r, s, bits1)
    gates = np.full(8, O.GATES["nand"], np.uint8)
    out = eng.gate_batch(key, gates, c0, c1)
    assert np.array_equal(out, okey.gate_batch(gates, c0, c1, threads=4))
    assert np.array_equal(ev.decrypt_bool(s, out), 1 - (bits0 & bits1))
