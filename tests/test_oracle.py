"""Pins of the CPU oracle against the reference's own tests (no GPU).

The reference ships no golden vectors (all its tests draw from entropy-seeded
RNGs), so the oracle is pinned by restating those tests' properties:
  ntt.rs:474-508      forward/backward round trip and output ranges
  ntt.rs:510-540      NTT product == schoolbook negacyclic product (25..60-bit primes)
  modulus_u64.rs:284-336   shoup_matrix_fma == naive u128 arithmetic
  decomposer.rs:325-370    signed decomposition recomposes within +-1 after rounding
  rgsw/mod.rs:526-686      Shoup external product == non-Shoup, bit for bit; decrypts to m0*m1
  rgsw/mod.rs:688-831      Shoup automorphism == non-Shoup, bit for bit; decrypts to m(X^k)
  mp_api.rs:662-695        bool gates under (multi-party) decryption
plus the committed fixtures of tests/golden/ (oracle regression vectors).
"""
import numpy as np
import pytest

from conftest import combine, oracle, oracle_setup

O = oracle()


def _rng(tag):
    return O.Rng(bytes([tag]) * 32)


def test_generate_prime_matches_reference_rule():
    N = 1 << 4
    for bits in [25, 40, 50, 60]:
        p = O.lib().orc_generate_prime(bits, 2 * N, 1 << bits)
        assert p != 0 and p % (2 * N) == 1 and p.bit_length() == bits


@pytest.mark.parametrize("bits", [25, 40, 50, 60])
def test_ntt_negacyclic_mul(bits):
    """ntt.rs:510-540 (N = 16, K = 128 in the reference; 32 samples here)."""
    N = 1 << 4
    p = O.lib().orc_generate_prime(bits, 2 * N, 1 << bits)
    h = O.lib().orc_ntt_custom_new(p, N)
    r = _rng(bits)
    try:
        for _ in range(32):
            a = r.uniform_mod(p, N)
            b = r.uniform_mod(p, N)
            fa, fb = a.copy(), b.copy()
            O.lib().orc_ntt_custom_forward(h, O._p(fa), 1)
            O.lib().orc_ntt_custom_forward(h, O._p(fb), 1)
            prod = np.array([O.lib().orc_mul_mod_barrett(p, int(x), int(y)) for x, y in zip(fa, fb)],
                            np.uint64)
            O.lib().orc_ntt_custom_backward(h, O._p(prod), 0)
            want = np.empty(N, np.uint64)
            O.lib().orc_negacyclic_mul(p, O._p(a), O._p(b), O._p(want), N)
            assert np.array_equal(prod, want)
    finally:
        O.lib().orc_ntt_custom_free(h)


@pytest.mark.parametrize("param", ["SP_TEST", "I_2P_LB_SR"])
def test_ntt_roundtrip_and_ranges(param):
    """ntt.rs:474-508 at the parameter set's own ring."""
    ev, _, _, _ = oracle_setup(param)
    r = _rng(3)
    for _ in range(4):
        a = r.uniform_mod(ev.Q, ev.N)
        f = ev.ntt_forward(a)
        assert (f < ev.Q).all() and not np.array_equal(f, a)
        assert np.array_equal(ev.ntt_backward(f), a)
        fl = ev.ntt_forward(a, lazy=True)
        assert (fl < 2 * ev.Q).all()
        assert np.array_equal(ev.ntt_backward(fl), a)
        bl = ev.ntt_backward(f, lazy=True)
        assert (bl < 2 * ev.Q).all()
        assert np.array_equal(np.where(bl >= ev.Q, bl - np.uint64(ev.Q), bl), a)


def test_shoup_matrix_fma():
    """modulus_u64.rs:284-336: prime 36028797017456641, ring 8, d = 2."""
    p = 36028797017456641
    r = _rng(5)
    for _ in range(64):
        a = r.uniform_mod(p, 16)
        b = r.uniform_mod(p, 16)
        a_sh = np.array([O.lib().orc_shoup_repr(int(v), p) for v in a], np.uint64)
        out = np.zeros(8, np.uint64)
        O.lib().orc_shoup_matrix_fma(p, O._p(out), O._p(a), O._p(a_sh), O._p(b), 2, 8)
        got = np.where(out >= p, out - np.uint64(p), out)
        want = [(int(a[i]) * int(b[i]) + int(a[8 + i]) * int(b[8 + i])) % p for i in range(8)]
        assert list(map(int, got)) == want


@pytest.mark.parametrize("logq", [37, 55])
@pytest.mark.parametrize("prime", [True, False])
def test_decomposition_recomposes(logq, prime):
    """decomposer.rs:325-370 (logb 11, d 3; 10^6 samples there, 4000 here)."""
    logb, d = 11, 3
    q = O.lib().orc_generate_prime(logq, 2 << 11, 1 << logq) if prime else 1 << logq
    r = _rng(logq + prime)
    vals = r.uniform_mod(q, 4000)
    limbs = np.zeros(8, np.uint64)
    for v in vals:
        ib = O.lib().orc_decompose_custom(q, logb, d, int(v), O._p(limbs))
        back = O.lib().orc_round_value(O.lib().orc_recompose(q, logb, d, O._p(limbs)), ib)
        rounded = O.lib().orc_round_value(int(v), ib)
        assert abs(int(rounded) - int(back)) <= 1


def test_decompose_edge_values():
    """Q and 0 decompose identically (the wrapping !(q - v) + 1 of decomposer.rs:219-221)."""
    ev, _, _, _ = oracle_setup("I_2P_LB_SR")
    for which in range(4):
        assert np.array_equal(ev.decompose(which, ev.Q if which else ev.info.lwe_q),
                              ev.decompose(which, 0))


def _rlwe_decrypt(ev, s, rl):
    """b - a s (negacyclic, mod Q) for an RLWE [a | b] under secret s."""
    N, Q = ev.N, ev.Q
    a, b = rl[:N], rl[N:]
    sq = np.array([(int(x) % Q) if x >= 0 else Q + int(x) for x in s], np.uint64)
    prod = np.empty(N, np.uint64)
    O.lib().orc_negacyclic_mul(Q, O._p(np.ascontiguousarray(a)), O._p(sq), O._p(prod), N)
    return np.array([(int(bb) - int(pp)) % Q for bb, pp in zip(b, prod)], np.uint64)


def _signed(v, Q):
    v = int(v) % Q
    return v - Q if v > Q // 2 else v


@pytest.mark.parametrize("param", ["SP_TEST", "I_2P_LB_SR"])
def test_rlwe_by_rgsw_shoup_equals_plain_and_decrypts(param):
    """rgsw/mod.rs:526-686: Shoup == non-Shoup; RLWE(m) x RGSW(X^{emb z_i}) decrypts to m X^{emb z_i}."""
    ev, (s, z, _, _), _, key = oracle_setup(param)
    r = _rng(7)
    N, Q = ev.N, ev.Q
    delta = Q // 8
    for trial in range(3):
        i = [0, ev.n // 2, ev.n - 1][trial]
        m = r.uniform_mod(4, N)
        a = r.uniform_mod(Q, N)
        rl = np.concatenate([a, np.zeros(N, np.uint64)])
        sa = _rlwe_decrypt(ev, s, np.concatenate([a, np.zeros(N, np.uint64)]))  # = -a s
        b = np.array([(int(m[k]) * delta - int(sa[k])) % Q for k in range(N)], np.uint64)
        rl[N:] = b
        x = key.rlwe_by_rgsw(rl, i, shoup=True)
        y = key.rlwe_by_rgsw(rl, i, shoup=False)
        assert np.array_equal(x, y)
        dec = _rlwe_decrypt(ev, s, x)
        e = int(z[i]) * ev.info.embedding_factor
        want = np.zeros(N, np.int64)
        for k in range(N):  # m(X) * X^e, negacyclic
            t = k + e
            sign = 1
            while t >= N:
                t -= N
                sign = -sign
            while t < 0:
                t += N
                sign = -sign
            want[t] += sign * int(m[k])
        got = np.array([round(_signed(v, Q) / delta) for v in dec])
        assert np.array_equal(got, want)


@pytest.mark.parametrize("param", ["SP_TEST", "I_2P_LB_SR"])
def test_rlwe_auto_shoup_equals_plain_and_decrypts(param):
    """rgsw/mod.rs:688-831: Shoup == non-Shoup; decrypts to m(X^k)."""
    ev, (s, _, _, _), _, key = oracle_setup(param)
    r = _rng(9)
    N, Q = ev.N, ev.Q
    delta = Q // 8
    for slot in [0, 1, ev.info.w]:
        m = r.uniform_mod(4, N)
        a = r.uniform_mod(Q, N)
        sa = _rlwe_decrypt(ev, s, np.concatenate([a, np.zeros(N, np.uint64)]))
        b = np.array([(int(m[k]) * delta - int(sa[k])) % Q for k in range(N)], np.uint64)
        rl = np.concatenate([a, b])
        x = key.rlwe_auto(rl, slot, shoup=True)
        y = key.rlwe_auto(rl, slot, shoup=False)
        assert np.array_equal(x, y)
        idx, sgn = ev.auto_map(slot)
        want = np.zeros(N, np.int64)
        for k in range(N):
            want[idx[k]] = int(m[k]) if sgn[k] else -int(m[k])
        got = np.array([round(_signed(v, Q) / delta) for v in _rlwe_decrypt(ev, s, x)])
        assert np.array_equal(np.mod(got, 8), np.mod(want, 8))


def test_lwe_key_switch_preserves_message():
    """lwe.rs:14-44: the key-switched LWE decrypts (under z, mod q_ks) like the input (under s)."""
    ev, (s, z, _, _), _, key = oracle_setup("I_2P_LB_SR")
    qk = ev.info.lwe_q
    r = _rng(11)
    for bit in [0, 1, 1, 0]:
        ct = ev.encrypt_bool(r, s, [bit])[0]
        down = np.array([int(np.round(float(v) * qk / float(ev.Q))) for v in ct], np.uint64)
        out = key.lwe_key_switch(down)
        m_in = (int(down[0]) - sum(int(a) * int(x) for a, x in zip(down[1:], s))) % qk
        m_out = (int(out[0]) - sum(int(a) * int(x) for a, x in zip(out[1:], z))) % qk
        diff = (m_in - m_out) % qk
        assert min(diff, qk - diff) < qk // 16


TRUTH = {
    "and": lambda a, b: a & b, "nand": lambda a, b: 1 - (a & b), "or": lambda a, b: a | b,
    "nor": lambda a, b: 1 - (a | b), "xor": lambda a, b: a ^ b, "xnor": lambda a, b: 1 - (a ^ b),
}


@pytest.mark.parametrize("param", ["SP_TEST", "I_2P_LB_SR"])
def test_gates_decrypt_correctly(param):
    """mp_api.rs:662-695: every gate on all four input pairs, single- and multi-party decryption."""
    ev, (s, _, sp, _), _, key = oracle_setup(param)
    r = _rng(13)
    a = np.array([0, 0, 1, 1])
    b = np.array([0, 1, 0, 1])
    c0 = ev.encrypt_bool(r, s, a)
    c1 = ev.encrypt_bool(r, s, b)
    for g, f in TRUTH.items():
        out = np.stack([key.gate(g, c0[i], c1[i]) for i in range(4)])
        assert list(ev.decrypt_bool(s, out)) == list(f(a, b))
        assert list(ev.mp_decrypt_bool(r, sp, out)) == list(f(a, b))
    assert list(ev.decrypt_bool(s, np.stack([ev.not_(c) for c in c0]))) == list(1 - a)


def test_gate_batch_threads_equal_single():
    ev, (s, _, _, _), _, key = oracle_setup("SP_TEST")
    r = _rng(15)
    c0 = ev.encrypt_bool(r, s, [0, 1, 1, 0, 1, 0])
    c1 = ev.encrypt_bool(r, s, [1, 1, 0, 0, 1, 1])
    gates = np.array([0, 1, 2, 3, 4, 5], np.uint8)
    single = np.stack([key.gate(int(g), c0[i], c1[i]) for i, g in enumerate(gates)])
    assert np.array_equal(key.gate_batch(gates, c0, c1, threads=3), single)


def test_pbs_prelude_is_the_gate():
    """gate(c0, c1) == pbs(combine(c0, c1)) (evaluator.rs:2163-2245)."""
    ev, (s, _, _, _), _, key = oracle_setup("SP_TEST")
    r = _rng(17)
    c0 = ev.encrypt_bool(r, s, [1])[0]
    c1 = ev.encrypt_bool(r, s, [0])[0]
    for g in TRUTH:
        out, _, _, _ = key.pbs(g, combine(ev, g, c0, c1))
        assert np.array_equal(out, key.gate(g, c0, c1))


@pytest.mark.parametrize("param", ["NI_2P", "NI_8P"])
def test_ni_input_path_round_trip(param):
    """Non-interactive inputs (ni_mp_api.rs:248-440): bools encrypted as seeded
    RLWEs under a user's secret u, unseeded, key-switched u -> s with Ksk(u -> s)
    and extracted decrypt under s; a wrong seed does not."""
    O = oracle()
    ev, (s, z, sp, zp), _, _ = oracle_setup(param)
    u = sp[-1]
    ksk = ev.ni_ksk_gen(u, s)
    bits = np.random.default_rng(5).integers(0, 2, ev.N + 300).astype(np.uint8)  # two RLWEs, ragged
    b = ev.ni_encrypt_bools(u, bits, b"\x07" * 32)
    assert b.shape == (2, ev.N)
    lwes = ev.ni_ingest(ksk, b"\x07" * 32, b, len(bits))
    assert np.array_equal(ev.decrypt_bool(s, lwes), bits)
    bad = ev.ni_ingest(ksk, b"\x08" * 32, b, 64)
    assert not np.array_equal(ev.decrypt_bool(s, bad), bits[:64])


@pytest.mark.parametrize("param", ["I_2P_LB_SR", "NI_8P"])
def test_seeded_key_expansion_stream_order(param):
    """keys.rs:687-781: auto A rows slot by slot (auto_element_dlogs order), then
    LWE-KSK A words row by row, each from its own ChaCha8 stream."""
    O = oracle()
    ev, _, coeff, _ = oracle_setup(param)
    i = ev.info
    d, N, n = i.auto_d, ev.N, ev.n
    auto_b = coeff.autos[:, d:, :]
    lwe_b = coeff.ksk[:, 0]
    sa, sl = b"\x61" * 32, b"\x62" * 32
    autos, ksk = ev.expand_seeded_key(auto_b, sa, lwe_b, sl)
    a_stream = O.Rng(sa).uniform_mod(ev.Q, i.n_auto_keys * d * N).reshape(i.n_auto_keys, d, N)
    assert np.array_equal(autos[:, :d, :], a_stream)
    assert np.array_equal(autos[:, d:, :], auto_b)
    k_stream = O.Rng(sl).uniform_mod(i.lwe_q, i.lwe_d * N * n).reshape(i.lwe_d * N, n)
    assert np.array_equal(ksk[:, 1:], k_stream)
    assert np.array_equal(ksk[:, 0], lwe_b)


@pytest.mark.parametrize("param", ["I_2P_LB_SR", "NI_8P"])
def test_rgsw_by_rgsw_decrypts_to_product(param):
    """rgsw_by_rgsw_inplace (runtime.rs:883-985): RGSW(X^3) x RGSW(X^5) is an
    RGSW(X^8) -- its m rows decrypt to beta X^8 and its -sm rows to -beta s X^8."""
    O = oracle()
    ev, (s, _, _, _), _, _ = oracle_setup(param)
    N, Q = ev.N, ev.Q

    def mono(k):
        m = np.zeros(N, np.uint64)
        m[k] = 1
        return m

    r0 = ev.rgsw_encrypt(s, mono(3), 0, b"\x71" * 32)
    r1 = ev.rgsw_encrypt(s, mono(5), 1, b"\x72" * 32)
    prod = ev.rgsw_by_rgsw(r0, r1)
    s_mod = np.array([int(x) % Q for x in s], dtype=np.uint64)

    def mul(a, b):
        out = np.empty(N, np.uint64)
        O.lib().orc_negacyclic_mul(Q, O._p(np.ascontiguousarray(a)), O._p(np.ascontiguousarray(b)), O._p(out), N)
        return out

    beta = 1 << (54 - ev.info.rlrg_logb)  # gadget 0 of the d = 1 rlwe x rgsw decomposer: 2^ignore_bits
    s8 = mul(s_mod, mono(8))
    for row_a, row_b, want in [(2, 3, mono(8)), (0, 1, (Q - s8) % Q)]:
        noise = (mul(prod[row_a], s_mod).astype(object) * -1 + prod[row_b].astype(object)
                 - want.astype(object) * beta) % Q
        centred = np.array([int(v) if v < Q // 2 else int(v) - Q for v in noise])
        assert np.max(np.abs(centred)) < (1 << 34), (row_a, np.max(np.abs(centred)))


def test_ni_crs_seeds_are_punctured_streams():
    """NonInteractiveMultiPartyCrs (evaluator.rs:115-172): every seed is the
    t-th 32-byte fill of a ChaCha8 stream (puncture_p_rng, utils.rs:219-228),
    a byte being the low byte of one u32 word (random.rs:162-175)."""
    O = oracle()

    def puncture(seed, times):
        r = O.Rng(seed)
        out = b""
        for _ in range(times):
            out = b""
            for _ in range(16):  # two u32 words per next_u64, low word first
                v = int(O.lib().orc_rng_next_u64(r.h))
                out += bytes([v & 0xFF, (v >> 32) & 0xFF])
        return out

    crs = bytes(range(7, 39))
    key = puncture(crs, 1)
    assert O.ni_crs_seed(crs, 0) == puncture(key, 2)
    assert O.ni_crs_seed(crs, 1) == puncture(key, 3)
    ks = puncture(crs, 2)
    for j in (0, 3):
        assert O.ni_crs_seed(crs, 2, j) == puncture(ks, j + 1)
    main = puncture(key, 1)
    for i in (0, 1, 9):
        assert O.ni_crs_seed(crs, 3, i) == puncture(main, i + 1)
    # InteractiveMultiPartyCrs (evaluator.rs:78-100): public key 1, key seed 2 -> auto 1, lwe 2
    assert O.interactive_crs_seed(crs, 0) == puncture(crs, 1)
    ikey = puncture(crs, 2)
    assert O.interactive_crs_seed(crs, 1) == puncture(ikey, 1)
    assert O.interactive_crs_seed(crs, 2) == puncture(ikey, 2)


def _ni_shares(ev, crs, users, seed_base=0):
    """Client-side NI key shares (evaluator.rs:1624-1975) for `users` users, with
    random auto / LWE KSK rows (the aggregation only sums those)."""
    s, z, sp, zp = ev.client_keys(users, seed_base=seed_base)
    up = ev.client_keys(users, seed_base=seed_base + 7)[2]
    info = ev.info
    g = np.random.default_rng(31 + seed_base)
    shares = []
    for j in range(users):
        sh = ev.ni_gen_share(crs, j, users, sp[j], up[j], zp[j], bytes([j + 1]) * 32)
        sh["auto_keys"] = g.integers(0, ev.Q, (info.w + 1, info.auto_d, ev.N), dtype=np.uint64)
        sh["lwe_ksk"] = g.integers(0, info.lwe_q, info.lwe_d * ev.N, dtype=np.uint64)
        shares.append(sh)
    return s, z, up, shares


def test_ni_aggregation_decrypts():
    """aggregate_non_interactive_multi_party_server_key_shares (evaluator.rs:
    1222-1622) restated: the aggregated RGSW of LWE index l encrypts
    X^{emb z[l]} (z the ideal LWE secret) under the ideal RLWE secret s -- its
    m rows decrypt to beta X^{emb z[l]}, its -sm rows to -beta s X^{emb z[l]} --
    for indices led by each user; each user's Ksk(u_j -> s) decrypts to its
    gadget multiples of u_j; the auto / LWE KSK parts are the sums."""
    O = oracle()
    ev = O.Evaluator("NI_2P")
    N, Q, users = ev.N, ev.Q, 2
    crs = b"\x5a" * 32
    s, z, up, shares = _ni_shares(ev, crs, users)
    emb = 2 * N // ev.info.br_q
    s_mod = np.array([int(x) % Q for x in s], dtype=np.uint64)

    def mul(a, b):
        out = np.empty(N, np.uint64)
        O.lib().orc_negacyclic_mul(Q, O._p(np.ascontiguousarray(a)), O._p(np.ascontiguousarray(b)), O._p(out), N)
        return out

    def centred_max(v):
        v = np.asarray(v).astype(object) % Q
        return max(abs(int(x) if x < Q // 2 else int(x) - Q) for x in v)

    beta = 1 << (54 - ev.info.rlrg_logb)
    for i0 in (0, ev.n - 2):  # user 0 leads the first, user 1 the last indices
        ksk, rgsw, auto, lwe = ev.ni_aggregate(crs, shares, i0, i0 + 2)
        for k in range(2):
            li = i0 + k
            m = np.zeros(N, np.uint64)
            e = int(z[li]) * emb
            if e < 0:
                m[N + e] = Q - 1
            else:
                m[e] = 1
            sm = mul(s_mod, m)
            r = rgsw[k]
            for row_a, row_b, want in [(2, 3, m), (0, 1, (Q - sm) % Q)]:
                noise = (r[row_b].astype(object) - mul(r[row_a], s_mod).astype(object)
                         - want.astype(object) * beta)
                assert centred_max(noise) < (1 << 34), (li, row_a, centred_max(noise))
    assert np.array_equal(auto, sum(sh["auto_keys"].astype(object) for sh in shares) % Q)
    assert np.array_equal(lwe, sum(sh["lwe_ksk"].astype(object) for sh in shares) % ev.info.lwe_q)
    for j in range(users):  # B - A s = e + beta_i u_j, A from the user's CRS stream
        a_rows = O.Rng(O.ni_crs_seed(crs, 2, j)).uniform_mod(Q, 50 * N).reshape(50, N)
        u_mod = np.array([int(x) % Q for x in up[j]], dtype=np.uint64)
        for i in (0, 25, 49):
            g = 1 << (4 + i)  # one-bit digits over the top 50 of the 54 bits: beta_i = 2^(4 + i)
            noise = (ksk[j, i].astype(object) - mul(a_rows[i], s_mod).astype(object)
                     - u_mod.astype(object) * g)
            assert centred_max(noise) < (1 << 12), (j, i)


def test_ni_protocol_end_to_end():
    """The whole non-interactive server side on the oracle: genuine shares of
    two users (auto / LWE-KSK parts seeded from the CRS) -> aggregation of all
    LWE indices -> seeded expansion (keys.rs:869-1004) -> each user's bools
    ingested with its aggregated ui_to_s key -> NAND gates across the two
    users' inputs decrypt correctly under the ideal secret."""
    O = oracle()
    ev = O.Evaluator("NI_2P")
    users = 2
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
    ksk_b, rgsw, auto, lwe = ev.ni_aggregate(crs, shares, threads=8)
    autos, ksk = ev.expand_seeded_key(auto, O.ni_crs_seed(crs, 0), lwe, O.ni_crs_seed(crs, 1))
    key = ev.key(O.ServerKeyCoeff(rgsw, autos, ksk))
    g = np.random.default_rng(12)
    k = 6
    ins = []
    for j in range(users):
        bits = g.integers(0, 2, k).astype(np.uint8)
        seed = bytes([0x30 + j]) * 32
        b = ev.ni_encrypt_bools(up[j], bits, seed)
        lw = ev.ni_ingest(ev.expand_ni_ksk(ksk_b[j], O.ni_crs_seed(crs, 2, j)), seed, b, k)
        assert np.array_equal(ev.decrypt_bool(s, lw), bits)
        ins.append((bits, lw))
    (b0, l0), (b1, l1) = ins
    out = key.gate_batch(np.full(k, O.GATES["nand"], np.uint8), l0, l1, threads=4)
    assert np.array_equal(ev.decrypt_bool(s, out), 1 - (b0 & b1))


def interactive_shares(ev, crs, users, seed_base=0):
    """Interactive server key shares (keys.rs:334-360) built from RGSW encryptions of
    X^{emb z_j[l]} under the ideal secret (what the collective public key encrypts to):
    the leader's in the rlwe x rgsw shape, the others' in the rgsw x rgsw shape; auto /
    LWE-KSK B parts under (s, z) with CRS-seeded A parts, all in user 0's share."""
    O = oracle()
    s, z, sp, zp = ev.client_keys(users, seed_base=seed_base)
    N, Q = ev.N, ev.Q
    emb = 2 * N // ev.info.br_q
    auto_b, lwe_b = ev.gen_seeded_auto_lwe(s, z, O.interactive_crs_seed(crs, 1), O.interactive_crs_seed(crs, 2))

    def mono(v):
        m = np.zeros(N, np.uint64)
        e = int(v) * emb
        if e < 0:
            m[N + e] = Q - 1
        else:
            m[e] = 1
        return m

    shares = []
    for j in range(users):
        b, e = ev.lwe_segment(j, users)
        lead = [ev.rgsw_encrypt(s, mono(zp[j][li]), 0, bytes([j, li % 256, li // 256]) + b"\x01" * 29)
                for li in range(b, e)]
        other = [ev.rgsw_encrypt(s, mono(zp[j][li]), 1, bytes([j, li % 256, li // 256]) + b"\x02" * 29)
                 for li in list(range(0, b)) + list(range(e, ev.n))]
        shares.append(dict(self_leader=np.stack(lead) if lead else np.zeros((0, 4, N), np.uint64),
                           not_leader=np.stack(other) if other else np.zeros((0, ev.rgsw_rows(1), N), np.uint64),
                           auto_keys=auto_b if j == 0 else np.zeros_like(auto_b),
                           lwe_ksk=lwe_b if j == 0 else np.zeros_like(lwe_b)))
    return s, shares


def test_interactive_aggregation_end_to_end():
    """aggregate_interactive_multi_party_server_key_shares (evaluator.rs:1050-1200) on the
    oracle: two users' shares -> aggregated RGSWs (leader x other) + summed auto / LWE
    KSK -> seeded expansion with the interactive CRS seeds -> gates decrypt correctly."""
    O = oracle()
    ev = O.Evaluator("I_2P_LB_SR")
    crs = b"\x2a" * 32
    s, shares = interactive_shares(ev, crs, 2)
    rgsw, auto, lwe = ev.aggregate(shares)
    autos, ksk = ev.expand_seeded_key(auto, O.interactive_crs_seed(crs, 1), lwe, O.interactive_crs_seed(crs, 2))
    key = ev.key(O.ServerKeyCoeff(rgsw, autos, ksk))
    r = O.Rng(b"\x07" * 32)
    bits0, bits1 = np.array([0, 1, 1, 0, 1, 0]), np.array([0, 0, 1, 1, 1, 1])
    c0, c1 = ev.encrypt_bool(r, s, bits0), ev.encrypt_bool(r, s, bits1)
    out = key.gate_batch(np.full(6, O.GATES["nand"], np.uint8), c0, c1, threads=4)
    assert np.array_equal(ev.decrypt_bool(s, out), 1 - (bits0 & bits1))
