"""Seeded server keys expanded on the device (keys.rs:687-781, 869-1004):
uploading the seeded form gives, word for word, the same gate bootstraps,
LWE key switches, automorphisms and NI key switches as uploading the
oracle's expansion of the same seeds in full."""
import numpy as np
import pytest

from conftest import oracle, oracle_setup, pz, to_dev, to_host

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("param", ["I_2P_LB_SR", "NI_8P"])
def test_seeded_upload_equals_full_upload(gpu_available, param):
    O = oracle()
    ev, _, coeff, _ = oracle_setup(param)
    d = ev.info.auto_d
    auto_b = np.ascontiguousarray(coeff.autos[:, d:, :])
    lwe_b = np.ascontiguousarray(coeff.ksk[:, 0])
    sa, sl = b"\x61" * 32, b"\x62" * 32
    autos2, ksk2 = ev.expand_seeded_key(auto_b, sa, lwe_b, sl)
    eng = pz().Engine(param)
    k_full = eng.upload_key(coeff.rgsw, autos2, ksk2)
    k_seed = eng.upload_key_seeded(coeff.rgsw, auto_b, sa, lwe_b, sl)
    okey2 = ev.key(O.ServerKeyCoeff(coeff.rgsw, autos2, ksk2))
    rng = np.random.default_rng(12)
    count = 8
    c0 = rng.integers(0, ev.Q, (count, ev.L), dtype=np.uint64)
    c1 = rng.integers(0, ev.Q, (count, ev.L), dtype=np.uint64)
    gates = (np.arange(count) % 6).astype(np.uint8)
    got_seed = eng.gate_batch(k_seed, gates, c0, c1)
    assert np.array_equal(got_seed, eng.gate_batch(k_full, gates, c0, c1))
    assert np.array_equal(got_seed, okey2.gate_batch(gates, c0, c1, threads=4))
    # the LWE key switch reads only the KSK, the automorphisms only the auto keys
    x = rng.integers(0, ev.info.lwe_q, (6, ev.L), dtype=np.uint64)
    outs = []
    for k in (k_seed, k_full):
        o = to_dev(np.zeros((6, ev.n + 1), np.uint32))
        eng.lwe_key_switch_device(k, to_dev(x), o)
        outs.append(to_host(o, np.uint32))
    assert np.array_equal(outs[0], outs[1])
    slots = np.arange(ev.info.w + 1, dtype=np.uint32)
    rl = rng.integers(0, ev.Q, (len(slots), 2, ev.N), dtype=np.uint64)
    res = []
    for k in (k_seed, k_full):
        t = to_dev(rl)
        eng.rlwe_auto_device(k, t, to_dev(slots))
        res.append(to_host(t))
    assert np.array_equal(res[0], res[1])
    assert np.array_equal(res[0].reshape(len(slots), -1),
                          np.stack([okey2.rlwe_auto(rl[i].reshape(-1), int(slots[i])) for i in range(len(slots))]))


def test_seeded_ni_ksk_upload(gpu_available):
    ev, (s, _, sp, _), _, _ = oracle_setup("NI_8P")
    ksk = ev.ni_ksk_gen(sp[0], s)
    b = np.ascontiguousarray(ksk[ev.NI_KS_D:])
    seed = b"\x63" * 32
    full = ev.expand_ni_ksk(b, seed)
    eng = pz().Engine("NI_8P")
    k1, k2 = eng.upload_ni_ksk_seeded(b, seed), eng.upload_ni_ksk(full)
    rl = np.random.default_rng(13).integers(0, ev.Q, (4, 2, ev.N), dtype=np.uint64)
    outs = []
    for k in (k1, k2):
        o = to_dev(np.zeros_like(rl))
        eng.ni_key_switch_device(k, to_dev(rl), o)
        outs.append(to_host(o).reshape(rl.shape))
    assert np.array_equal(outs[0], outs[1])
    assert np.array_equal(outs[0][2], ev.ni_key_switch(full, rl[2]))
