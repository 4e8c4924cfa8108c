"""Bit-exact parity of the CUDA path with the CPU oracle (through the C ABI).

Every comparison here is exact equality of u64 words: the kernels must
produce the same ciphertext words as the oracle's restatement of the
reference on the same key bytes and inputs.
"""
import numpy as np
import pytest

from conftest import combine, oracle, oracle_setup, pz, to_dev, to_host

pytestmark = pytest.mark.gpu

PARAMS = ["SP_TEST", "I_2P_LB_SR", "I_4P", "I_8P", "NI_2P", "NI_4P_HB_FR", "NI_4P_LB_SR", "NI_8P"]
FAST = ["SP_TEST", "I_2P_LB_SR", "NI_8P"]

_ENGINES = {}


def engine_and_key(param):
    if param not in _ENGINES:
        ev, secrets, coeff, okey = oracle_setup(param)
        eng = pz().Engine(param, ntt_root=ev.psi())
        dkey = eng.upload_key(coeff.rgsw, coeff.autos, coeff.ksk)
        _ENGINES[param] = (eng, dkey)
    return _ENGINES[param]


def rng(tag):
    return oracle().Rng(bytes([tag]) * 32)


@pytest.mark.parametrize("param", PARAMS)
def test_ntt_matches_oracle(gpu_available, param):
    ev, _, _, _ = oracle_setup(param)
    eng, _ = engine_and_key(param)
    assert eng.ntt_root == ev.psi()
    count = 64
    x = rng(0x11).uniform_mod(ev.Q, count * ev.N).reshape(count, ev.N)
    want = np.stack([ev.ntt_forward(r) for r in x])
    t = to_dev(x)
    eng.ntt_forward_device(t)
    got = to_host(t).reshape(count, ev.N)
    assert np.array_equal(got, want)
    eng.ntt_backward_device(t)
    assert np.array_equal(to_host(t).reshape(count, ev.N), x)


def test_ntt_batch_many_pairs_odd_count(gpu_available):
    """The persistent batched NTT: more polynomial pairs than resident CTAs
    (each CTA streams several pairs through its double-buffered stage), an
    odd count (a last pair of one), forward and inverse each equal to the
    oracle's transforms, and no device error raised."""
    ev, _, _, _ = oracle_setup("NI_8P")
    eng, _ = engine_and_key("NI_8P")
    count = 4 * 148 + 3
    r = rng(0x13)
    x = r.uniform_mod(ev.Q, count * ev.N).reshape(count, ev.N)
    t = to_dev(x)
    eng.ntt_forward_device(t)
    assert np.array_equal(to_host(t).reshape(count, ev.N), np.stack([ev.ntt_forward(v) for v in x]))
    y = r.uniform_mod(ev.Q, count * ev.N).reshape(count, ev.N)  # arbitrary evaluation-domain words
    t = to_dev(y)
    eng.ntt_backward_device(t)
    assert np.array_equal(to_host(t).reshape(count, ev.N), np.stack([ev.ntt_backward(v) for v in y]))
    assert eng.device_error() == 0


@pytest.mark.parametrize("param", ["SP_TEST", "I_2P_LB_SR"])
def test_ntt_negacyclic_product_default_root(gpu_available, param):
    """ntt.rs:510-540 pin: NTT product == schoolbook product (library's own root)."""
    O = oracle()
    ev, _, _, _ = oracle_setup(param)
    eng = pz().Engine(param)
    r = rng(0x12)
    a = r.uniform_mod(ev.Q, ev.N)
    b = r.uniform_mod(ev.Q, ev.N)
    ta, tb = to_dev(a), to_dev(b)
    eng.ntt_forward_device(ta)
    eng.ntt_forward_device(tb)
    fa, fb = to_host(ta), to_host(tb)
    prod = np.array([(int(u) * int(v)) % ev.Q for u, v in zip(fa, fb)], dtype=np.uint64)
    tp = to_dev(prod)
    eng.ntt_backward_device(tp)
    want = np.empty(ev.N, np.uint64)
    O.lib().orc_negacyclic_mul(ev.Q, O._p(a), O._p(b), O._p(want), ev.N)
    assert np.array_equal(to_host(tp), want)


@pytest.mark.parametrize("param", PARAMS)
@pytest.mark.parametrize("trivial", [False, True])
def test_rlwe_by_rgsw(gpu_available, param, trivial):
    ev, _, _, okey = oracle_setup(param)
    eng, dkey = engine_and_key(param)
    count = 24
    r = rng(0x21 + trivial)
    rl = r.uniform_mod(ev.Q, count * 2 * ev.N).reshape(count, 2, ev.N)
    if trivial:
        rl[:, 0, :] = 0
    idx = (r.uniform_mod(ev.n, count)).astype(np.uint32)
    idx[0], idx[-1] = 0, ev.n - 1
    want = np.stack([okey.rlwe_by_rgsw(rl[i].reshape(-1), int(idx[i]), trivial=trivial) for i in range(count)])
    t = to_dev(rl)
    eng.rlwe_by_rgsw_device(dkey, t, to_dev(idx), trivial=trivial)
    got = to_host(t).reshape(count, -1)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("param", PARAMS)
@pytest.mark.parametrize("trivial", [False, True])
def test_rlwe_auto(gpu_available, param, trivial):
    ev, _, _, okey = oracle_setup(param)
    eng, dkey = engine_and_key(param)
    slots = np.arange(ev.info.w + 1, dtype=np.uint32)
    count = len(slots) * 2
    slots = np.concatenate([slots, slots])
    r = rng(0x31 + trivial)
    rl = r.uniform_mod(ev.Q, count * 2 * ev.N).reshape(count, 2, ev.N)
    rl[1, 0, :7] = 0  # zeros exercise neg(0) = Q on the a-part
    if trivial:
        rl[:, 0, :] = 0
        rl[2, 1, :5] = 0
        rl[3, 1, :5] = ev.Q  # trivial autos may carry Q (neg(0)) in b
    want = np.stack([okey.rlwe_auto(rl[i].reshape(-1), int(slots[i]), trivial=trivial) for i in range(count)])
    t = to_dev(rl)
    eng.rlwe_auto_device(dkey, t, to_dev(slots), trivial=trivial)
    assert np.array_equal(to_host(t).reshape(count, -1), want)


@pytest.mark.parametrize("param", PARAMS)
def test_lwe_key_switch(gpu_available, param):
    ev, _, _, okey = oracle_setup(param)
    eng, dkey = engine_and_key(param)
    qk = ev.info.lwe_q
    count = 20
    r = rng(0x41)
    x = r.uniform_mod(qk + 1, count * ev.L).reshape(count, ev.L)  # [0, q_ks] (mod-down may give q_ks)
    x[0, :] = qk
    x[1, :] = 0
    want = np.stack([okey.lwe_key_switch(x[i]) for i in range(count)])
    out = to_dev(np.zeros((count, ev.n + 1), np.uint32))
    eng.lwe_key_switch_device(dkey, to_dev(x), out)
    got = to_host(out, np.uint32).astype(np.uint64)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("param", ["I_2P_LB_SR", "NI_8P"])
@pytest.mark.parametrize("tile", [8, 16, 32, 64])
def test_lwe_key_switch_every_tile(gpu_available, param, tile):
    """The key switch with 8, 16 and 32 ciphertexts per CTA and the
    tensor-core form (64: s8 digits x u8 KSK byte planes) -- the shapes the
    autotuner picks from -- equals the oracle, on a batch that leaves a
    partial last tile and on one large enough to run unsplit (grid.z = 1);
    the inputs include the q_ks edge value."""
    ev, _, _, okey = oracle_setup(param)
    eng, dkey = engine_and_key(param)
    qk = ev.info.lwe_q
    r = rng(0x42 + tile)
    try:
        eng.set_ks_tile(tile)
        # the second count leaves one share per tile (grid.z = 1): 4 x 148 CTAs of
        # 128 threads for the IMAD tiles, 4 x 148 / 3 row tiles of 64 for the tensor cores
        big = 4 * 148 * tile // 8 + 3 if tile < 64 else 64 * (4 * 148 // 3 + 1) + 3
        for count in (tile + 5, big):
            x = r.uniform_mod(qk + 1, count * ev.L).reshape(count, ev.L)
            x[0, :] = qk
            idx = np.concatenate([np.arange(min(count, 24)), count - 1 - np.arange(8)])
            want = np.stack([okey.lwe_key_switch(x[i]) for i in idx])
            out = to_dev(np.zeros((count, ev.n + 1), np.uint32))
            eng.lwe_key_switch_device(dkey, to_dev(x), out)
            got = to_host(out, np.uint32).astype(np.uint64).reshape(count, -1)
            assert np.array_equal(got[idx], want), (tile, count)
            assert eng.launch_shape(count)["ks_tile"] == tile
    finally:
        eng.set_ks_tile(64)


def _gate_inputs(ev, secrets, count, tag):
    s = secrets[0]
    r = rng(tag)
    bits0 = (r.uniform_mod(2, count)).astype(np.int64)
    bits1 = (r.uniform_mod(2, count)).astype(np.int64)
    c0 = ev.encrypt_bool(r, s, bits0)
    c1 = ev.encrypt_bool(r, s, bits1)
    return bits0, bits1, c0, c1


TRUTH = {
    "and": lambda a, b: a & b, "nand": lambda a, b: 1 - (a & b), "or": lambda a, b: a | b,
    "nor": lambda a, b: 1 - (a | b), "xor": lambda a, b: a ^ b, "xnor": lambda a, b: 1 - (a ^ b),
}


@pytest.mark.parametrize("param", PARAMS)
def test_gate_batch_bit_exact(gpu_available, param):
    O = oracle()
    ev, secrets, _, okey = oracle_setup(param)
    eng, dkey = engine_and_key(param)
    names = list(TRUTH)
    count = 12 if param in FAST else 6
    bits0, bits1, c0, c1 = _gate_inputs(ev, secrets, count, 0x51)
    gates = np.array([O.GATES[names[i % 6]] for i in range(count)], np.uint8)
    out = to_dev(np.zeros((count, ev.L), np.uint64))
    ks = to_dev(np.zeros((count, ev.n + 1), np.uint32))
    rl = to_dev(np.zeros((count, 2 * ev.N), np.uint64))
    eng.gate_batch_device(dkey, to_dev(gates), to_dev(c0), to_dev(c1), out, ks_out=ks, rlwe_out=rl)
    got_out, got_ks, got_rl = to_host(out), to_host(ks, np.uint32), to_host(rl)
    for i in range(count):
        g = names[i % 6]
        comb = combine(ev, g, c0[i], c1[i])
        w_out, w_ks, w_rl, _ = okey.pbs(g, comb)
        assert np.array_equal(got_ks[i].astype(np.uint64), w_ks), f"key switch mismatch at {i} ({g})"
        assert np.array_equal(got_rl[i], w_rl), f"blind rotation mismatch at {i} ({g})"
        assert np.array_equal(got_out[i], w_out), f"output mismatch at {i} ({g})"
    dec = ev.decrypt_bool(secrets[0], got_out)
    want = np.array([TRUTH[names[i % 6]](bits0[i], bits1[i]) for i in range(count)])
    assert np.array_equal(dec, want)


@pytest.mark.parametrize("param", PARAMS)
def test_gate_batch_tensor_core_key_switch(gpu_available, param):
    """Gates whose key switch runs on the tensor cores (tile 64: the gate
    prelude and mod-down feed s8 digits, the KSK comes as u8 byte planes)
    give the oracle's key-switched LWEs and outputs, across a partial second
    row tile (70 gates)."""
    O = oracle()
    ev, secrets, _, okey = oracle_setup(param)
    eng, dkey = engine_and_key(param)
    names = list(TRUTH)
    count = 70
    bits0, bits1, c0, c1 = _gate_inputs(ev, secrets, count, 0x57)
    gates = np.array([O.GATES[names[i % 6]] for i in range(count)], np.uint8)
    out = to_dev(np.zeros((count, ev.L), np.uint64))
    ks = to_dev(np.zeros((count, ev.n + 1), np.uint32))
    try:
        eng.set_ks_tile(64)
        eng.gate_batch_device(dkey, to_dev(gates), to_dev(c0), to_dev(c1), out, ks_out=ks)
    finally:
        eng.set_ks_tile(64)
    got_out, got_ks = to_host(out), to_host(ks, np.uint32)
    for i in list(range(4)) + list(range(63, 70)):
        g = names[i % 6]
        w_out, w_ks, _, _ = okey.pbs(g, combine(ev, g, c0[i], c1[i]))
        assert np.array_equal(got_ks[i].astype(np.uint64), w_ks), f"key switch mismatch at {i} ({g})"
        assert np.array_equal(got_out[i], w_out), f"output mismatch at {i} ({g})"
    dec = ev.decrypt_bool(secrets[0], got_out)
    want = np.array([TRUTH[names[i % 6]](bits0[i], bits1[i]) for i in range(count)])
    assert np.array_equal(dec, want)


@pytest.mark.parametrize("param", ["SP_TEST", "I_2P_LB_SR"])
def test_gate_batch_host_api(gpu_available, param):
    """pz_gate_batch (host buffers, synchronous) == oracle gates."""
    O = oracle()
    ev, secrets, _, okey = oracle_setup(param)
    eng, dkey = engine_and_key(param)
    count = 8
    bits0, bits1, c0, c1 = _gate_inputs(ev, secrets, count, 0x61)
    gates = np.array([O.GATES["nand"]] * count, np.uint8)
    got = eng.gate_batch(dkey, gates, c0, c1)
    want = okey.gate_batch(gates, c0, c1, threads=4)
    assert np.array_equal(got, want)
    assert np.array_equal(ev.decrypt_bool(secrets[0], got), 1 - (bits0 & bits1))


@pytest.mark.parametrize("param", ["I_2P_LB_SR", "NI_8P"])
@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4])
def test_pbs_variants_bit_exact(gpu_available, param, variant):
    """Every launch-shape variant of the blind rotation (3: one ciphertext on a
    cluster of two CTAs; 4: keys streamed into shared memory by bulk copies)
    gives the oracle's words."""
    O = oracle()
    ev, secrets, _, okey = oracle_setup(param)
    eng, dkey = engine_and_key(param)
    count = 4
    bits0, bits1, c0, c1 = _gate_inputs(ev, secrets, count, 0x71 + variant)
    gates = np.array([O.GATES[g] for g in ["nand", "xor", "or", "xnor"]], np.uint8)
    old = eng.pbs_variant
    eng.pbs_variant = variant
    eng.set_split_threshold(0)  # the variant under test, not the small-batch default
    try:
        out = to_dev(np.zeros((count, ev.L), np.uint64))
        eng.gate_batch_device(dkey, to_dev(gates), to_dev(c0), to_dev(c1), out)
        got = to_host(out)
    finally:
        eng.pbs_variant = old
        eng.set_split_threshold(-1)
    want = okey.gate_batch(gates, c0, c1, threads=4)
    assert np.array_equal(got, want)
    assert eng.device_error() == 0


def test_ctx_autotune_keeps_results(gpu_available):
    """pz_ctx_autotune picks a launch variant; the gate words do not change."""
    O = oracle()
    ev, secrets, _, okey = oracle_setup("NI_8P")
    eng, dkey = engine_and_key("NI_8P")
    old = eng.pbs_variant
    try:
        t = eng.autotune(dkey, 296)
        assert t["variant"] in (0, 1, 2, 3, 4) and t["ms"] > 0 and eng.pbs_variant == t["variant"]
        assert t["ks_tile"] in (8, 16, 32, 64)
        assert eng.launch_shape(296) == {"variant": t["variant"], "ks_tile": t["ks_tile"]}
        bits0, bits1, c0, c1 = _gate_inputs(ev, secrets, 4, 0x7F)
        gates = np.array([O.GATES[g] for g in ["and", "nand", "xor", "nor"]], np.uint8)
        assert np.array_equal(eng.gate_batch(dkey, gates, c0, c1), okey.gate_batch(gates, c0, c1, threads=4))
    finally:
        eng.pbs_variant = old
        eng.set_ks_tile(64)


def test_split_kernel_many_items_per_cluster(gpu_available):
    """The two-CTA kernel with fewer clusters than ciphertexts (each cluster
    bootstraps several in turn, reusing its digit slots) and the staged-key
    kernel with fewer CTAs than ciphertexts == the one-CTA kernel."""
    O = oracle()
    ev, secrets, _, okey = oracle_setup("NI_8P")
    eng, dkey = engine_and_key("NI_8P")
    count = 24
    r = rng(0x7E)
    c0 = r.uniform_mod(ev.Q, count * ev.L).reshape(count, ev.L)
    c1 = r.uniform_mod(ev.Q, count * ev.L).reshape(count, ev.L)
    gates = (np.arange(count) % 6).astype(np.uint8)
    outs = []
    old = eng.pbs_variant
    try:
        for v, limit in [(0, 0), (3, 5), (4, 5)]:
            eng.pbs_variant = v
            eng.set_split_threshold(0)
            eng.set_pbs_grid_limit(limit)
            out = to_dev(np.zeros((count, ev.L), np.uint64))
            eng.gate_batch_device(dkey, to_dev(gates), to_dev(c0), to_dev(c1), out)
            outs.append(to_host(out))
    finally:
        eng.pbs_variant = old
        eng.set_split_threshold(-1)
        eng.set_pbs_grid_limit(0)
    assert np.array_equal(outs[0], outs[1])
    assert np.array_equal(outs[0], outs[2])  # staged keys: each CTA runs ~5 items, its mbarrier phases carry over
    assert np.array_equal(outs[1][:3], okey.gate_batch(gates[:3], c0[:3], c1[:3], threads=3))
    assert eng.device_error() == 0


def test_pbs_slots_whole_waves(gpu_available):
    """pz_ctx_pbs_slots: every launch shape reports its resident ciphertexts
    (a multiple of the SM count for the one-CTA shapes, more CTAs per SM for
    tighter register caps), and the autotuner times whole waves of them."""
    import torch
    eng, dkey = engine_and_key("NI_8P")
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    slots = [eng.pbs_slots(v) for v in range(5)]
    assert all(s > 0 for s in slots)
    for v in range(3):
        assert slots[v] % sms == 0
    assert slots[0] <= slots[1] <= slots[2]
    assert eng.pbs_slots(-1) == slots[eng.pbs_variant]
    old = eng.pbs_variant
    try:
        t = eng.autotune(dkey, 2 * slots[2])
        assert t["variant"] in (0, 1, 2, 3, 4) and t["ms"] > 0
    finally:
        eng.pbs_variant = old
