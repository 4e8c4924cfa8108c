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
