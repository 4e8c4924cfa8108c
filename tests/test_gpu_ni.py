"""Non-interactive input path on the GPU vs the oracle, word for word:
unseed (ni_mp_api.rs:248-280), rlwe_key_switch u_j -> s (runtime.rs:1001-1063),
extract (ni_mp_api.rs:217-236), and the whole ingestion feeding a gate."""
import numpy as np
import pytest

from conftest import oracle, oracle_setup, pz, to_dev, to_host

pytestmark = pytest.mark.gpu

NI = ["NI_2P", "NI_8P"]
_S = {}


def setup_ni(param):
    if param not in _S:
        ev, (s, z, sp, zp), coeff, okey = oracle_setup(param)
        u = sp[-1]
        ksk = ev.ni_ksk_gen(u, s)
        eng = pz().Engine(param)
        _S[param] = (ev, s, u, ksk, okey, eng, eng.upload_ni_ksk(ksk), eng.upload_key(coeff.rgsw, coeff.autos,
                                                                                       coeff.ksk))
    return _S[param]


@pytest.mark.parametrize("param", NI)
def test_unseed_matches_oracle(gpu_available, param):
    ev, s, u, ksk, _, eng, _, _ = setup_ni(param)
    seed = bytes(range(32))
    b = np.random.default_rng(3).integers(0, ev.Q, (3, ev.N), dtype=np.uint64)
    want = ev.ni_unseed(seed, b)
    d_r = to_dev(np.zeros((3, 2, ev.N), np.uint64))
    eng.ni_unseed_device(seed, to_dev(b), d_r)
    assert np.array_equal(to_host(d_r).reshape(3, 2, ev.N), want)


@pytest.mark.parametrize("param,count", [("NI_2P", 6), ("NI_8P", 6), ("NI_8P", 1), ("NI_8P", 300)])
def test_ni_key_switch_matches_oracle(gpu_available, param, count):
    """Small batches split each RLWE's digits over CTAs (1, 6 RLWEs); large
    ones run one CTA per RLWE (300)."""
    ev, s, u, ksk, _, eng, dksk, _ = setup_ni(param)
    rl = np.random.default_rng(4).integers(0, ev.Q, (count, 2, ev.N), dtype=np.uint64)
    rl[0, 0, :9] = 0  # -0 = q in the reference's elwise_neg_mut
    rl[-1, 0, :] = 0
    want = np.stack([ev.ni_key_switch(ksk, r) for r in rl])
    d_out = to_dev(np.zeros_like(rl))
    eng.ni_key_switch_device(dksk, to_dev(rl), d_out)
    assert np.array_equal(to_host(d_out).reshape(count, 2, ev.N), want)


def test_sample_extract_at_index(gpu_available):
    ev, s, u, ksk, _, eng, _, _ = setup_ni("NI_8P")
    rl = np.random.default_rng(6).integers(0, ev.Q, (2, 2, ev.N), dtype=np.uint64)
    rl[0, 0, 5] = 0  # neg(0) = q in the extracted a
    N = ev.N
    idx = np.array([0, 1, 7, N - 1, N, N + 3, 2 * N - 1, 1234], np.uint32)
    want = np.stack([ev.sample_extract(rl[i // N], i % N) for i in idx])
    d_l = to_dev(np.zeros((len(idx), ev.L), np.uint64))
    eng.sample_extract_device(to_dev(rl), to_dev(idx), d_l)
    assert np.array_equal(to_host(d_l).reshape(len(idx), ev.L), want)


@pytest.mark.parametrize("param", NI)
def test_ingest_end_to_end_and_gate(gpu_available, param):
    """Client bools under u_j -> server ingestion (one call) == oracle, decrypt
    under s, and the ingested LWEs feed a NAND gate bootstrap correctly."""
    O = oracle()
    ev, s, u, ksk, okey, eng, dksk, dkey = setup_ni(param)
    bits = np.random.default_rng(9).integers(0, 2, ev.N + 100).astype(np.uint8)
    seed = b"\x2a" * 32
    b = ev.ni_encrypt_bools(u, bits, seed)
    got = eng.ni_ingest(dksk, seed, b, len(bits))
    want = ev.ni_ingest(ksk, seed, b, len(bits))
    assert np.array_equal(got, want)
    assert np.array_equal(ev.decrypt_bool(s, got), bits)
    k = 16
    gates = np.full(k, O.GATES["nand"], np.uint8)
    out = eng.gate_batch(dkey, gates, got[:k], got[k:2 * k])
    assert np.array_equal(out, okey.gate_batch(gates, got[:k], got[k:2 * k], threads=4))
    assert np.array_equal(ev.decrypt_bool(s, out), 1 - (bits[:k] & bits[k:2 * k]))
