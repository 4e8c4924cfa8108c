"""FheUint8 circuits on the GPU (levelized, batched) vs the oracle's sequential
gate-by-gate evaluation, bit for bit, and their plaintext semantics under
decryption (mp_api.rs:491-660: +, -, *, div/rem incl. division by zero,
==, !=, <, >, <=, >=, mux)."""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from conftest import oracle, oracle_setup, pz, to_dev, to_host

pytestmark = pytest.mark.gpu

_ENG = {}


def eng_key(param):
    if param not in _ENG:
        ev, _, coeff, _ = oracle_setup(param)
        eng = pz().Engine(param)
        _ENG[param] = (eng, eng.upload_key(coeff.rgsw, coeff.autos, coeff.ksk))
    return _ENG[param]


def enc_u8(ev, r, s, vals):
    bits = np.array([[(v >> i) & 1 for i in range(8)] for v in vals]).reshape(-1)
    return ev.encrypt_bool(r, s, bits).reshape(len(vals), 8, ev.L)


def dec_u8(ev, s, cts):
    bits = ev.decrypt_bool(s, cts.reshape(-1, ev.L)).reshape(-1, 8)
    return np.array([sum(int(b) << i for i, b in enumerate(row)) for row in bits])


def build_all_ops(C, n_pairs):
    """Every FheUint8 operator on n_pairs (a, b, selector) triples."""
    ins, outs = [], {}
    for p in range(n_pairs):
        a, b = C.input_u8(), C.input_u8()
        sel = C.input()
        ins.append((a, b, sel))
    names = ["add", "sub", "mul", "q", "r", "flag", "eq", "neq", "lt", "gt", "le", "ge", "mux"]
    for k in names:
        outs[k] = []
    for p, (a, b, sel) in enumerate(ins):
        o = {"add": C.u8_add(a, b), "sub": C.u8_sub(a, b), "mul": C.u8_mul(a, b)}
        q, r, f = C.u8_div_rem(a, b)
        o.update(q=q, r=r, flag=[f])
        for op in ["eq", "neq", "lt", "gt", "le", "ge"]:
            o[op] = [C.u8_cmp(op, a, b)]
        o["mux"] = C.u8_mux(a, b, sel)
        for k in names:
            outs[k].append(o[k])
    order = []
    for k in names:
        for p in range(n_pairs):
            C.outputs(outs[k][p])
            order.append((k, p, len(outs[k][p])))
    return order


def split_outputs(order, out):
    res, i = {}, 0
    for k, p, w in order:
        res.setdefault(k, {})[p] = out[i:i + w]
        i += w
    return res


def plaintext(a, b, s):
    q = 255 if b == 0 else a // b
    r = a if b == 0 else a % b
    return {"add": (a + b) % 256, "sub": (a - b) % 256, "mul": (a * b) % 256, "q": q, "r": r,
            "flag": int(b == 0), "eq": int(a == b), "neq": int(a != b), "lt": int(a < b), "gt": int(a > b),
            "le": int(a <= b), "ge": int(a >= b), "mux": a if s else b}


def run_ops(param, vals):
    ev, (s, _, _, _), _, _ = oracle_setup(param)
    eng, key = eng_key(param)
    C = pz().Circuit()
    order = build_all_ops(C, len(vals))
    r = oracle().Rng(b"\x05" * 32)
    inputs = []
    for a, b, sel in vals:
        inputs.append(enc_u8(ev, r, s, [a])[0])
        inputs.append(enc_u8(ev, r, s, [b])[0])
        inputs.append(ev.encrypt_bool(r, s, [sel]))
    inputs = np.concatenate([x.reshape(-1, ev.L) for x in inputs])
    out = C.run(eng, key, inputs)
    return ev, s, inputs, order, split_outputs(order, out)


def test_u8_ops_bit_exact_vs_sequential_oracle(gpu_available):
    param = "SP_TEST"
    vals = [(200, 7, 1), (13, 0, 0)]  # second pair divides by zero
    ev, s, inputs, order, got = run_ops(param, vals)
    _, _, _, okey = oracle_setup(param)

    def check_pair(p):
        a_ct = inputs[p * 17:p * 17 + 8]
        b_ct = inputs[p * 17 + 8:p * 17 + 16]
        sel = inputs[p * 17 + 16]
        want = {}
        want["add"] = okey.u8_op("add", a_ct, b_ct)[0]
        want["sub"] = okey.u8_op("sub", a_ct, b_ct)[0]
        want["mul"] = okey.u8_op("mul", a_ct, b_ct)[0]
        q, r, f = okey.u8_op("div_rem", a_ct, b_ct, flag=None)
        # the circuit's flag starts from "no flag yet": is_zero(b) itself
        want["q"], want["r"], want["flag"] = q, r, f.reshape(1, -1)
        for op in ["eq", "neq", "lt", "gt", "le", "ge"]:
            want[op] = okey.u8_op(op, a_ct, b_ct)[0]
        want["mux"] = okey.u8_op("mux", a_ct, b_ct, sel=sel)[0]
        return want

    with ThreadPoolExecutor(max_workers=len(vals)) as ex:
        wants = list(ex.map(check_pair, range(len(vals))))
    for p in range(len(vals)):
        for k, w in wants[p].items():
            assert np.array_equal(got[k][p], w), f"pair {p} op {k} differs from the sequential oracle"
    for p, (a, b, sel) in enumerate(vals):
        exp = plaintext(a, b, sel)
        for k in exp:
            v = dec_u8(ev, s, got[k][p]) [0] if got[k][p].shape[0] == 8 else ev.decrypt_bool(s, got[k][p])[0]
            assert v == exp[k], (a, b, k, v, exp[k])


def test_u8_semantics_random_pairs(gpu_available):
    """Plaintext semantics of every operator on random pairs, 20% with divisor 0."""
    r = np.random.default_rng(7)
    n = 48
    a = r.integers(0, 256, n)
    b = r.integers(0, 256, n)
    b[r.random(n) < 0.2] = 0
    sel = r.integers(0, 2, n)
    vals = list(zip(a.tolist(), b.tolist(), sel.tolist()))
    ev, s, _, _, got = run_ops("SP_TEST", vals)
    for p, (x, y, z) in enumerate(vals):
        exp = plaintext(x, y, z)
        for k in exp:
            ct = got[k][p]
            v = dec_u8(ev, s, ct)[0] if ct.shape[0] == 8 else ev.decrypt_bool(s, ct)[0]
            assert v == exp[k], (x, y, k, v, exp[k])


@pytest.mark.parametrize("param", ["I_2P_LB_SR", "NI_8P"])
def test_wavefront_mul_lt_graph_replay(gpu_available, param):
    """a*b and a<b batched per level, captured as one CUDA graph and replayed;
    outputs equal the direct run, the sequential oracle (one pair) and plaintext."""
    import torch
    ev, (s, _, _, _), _, okey = oracle_setup(param)
    eng, key = eng_key(param)
    vals = [(37, 201), (255, 255), (0, 9), (128, 3)]
    C = pz().Circuit()
    pairs = [(C.input_u8(), C.input_u8()) for _ in vals]
    for a, b in pairs:
        C.outputs(C.u8_mul(a, b))
    for a, b in pairs:
        C.output(C.u8_cmp("lt", a, b))
    r = oracle().Rng(b"\x09" * 32)
    inp = np.concatenate([np.concatenate([enc_u8(ev, r, s, [x])[0], enc_u8(ev, r, s, [y])[0]]) for x, y in vals])
    d_in = to_dev(inp)
    d_out = to_dev(np.zeros((C.n_outputs, ev.L), np.uint64))
    C.run_device(eng, key, d_in, d_out)
    torch.cuda.synchronize()
    direct = to_host(d_out).reshape(-1, ev.L).copy()
    d_out.zero_()
    C.capture_graph(eng, key, d_in, d_out)
    C.replay_graph()
    torch.cuda.synchronize()
    assert np.array_equal(to_host(d_out).reshape(-1, ev.L), direct)
    muls = direct[:8 * len(vals)].reshape(len(vals), 8, ev.L)
    lts = direct[8 * len(vals):]
    for p, (x, y) in enumerate(vals):
        assert dec_u8(ev, s, muls[p])[0] == (x * y) % 256
        assert ev.decrypt_bool(s, lts[p])[0] == int(x < y)
    # one pair against the sequential oracle, word for word
    a_ct, b_ct = inp[0:8], inp[8:16]
    assert np.array_equal(lts[0], okey.u8_op("lt", a_ct, b_ct)[0][0])
    assert np.array_equal(muls[0], okey.u8_op("mul", a_ct, b_ct)[0])


@pytest.mark.parametrize("param", ["I_2P_LB_SR", "NI_8P"])
def test_mul_and_lt_multi_party_decryption(gpu_available, param):
    """FheUint8 a*b and a<b on the GPU, each output bit decrypted by the
    parties' decryption shares and their aggregation (multi-party decryption,
    mp_api.rs:491-660) with the 2 / 8 parties of the parameter set."""
    O = oracle()
    ev, (s, _, sp, _), _, _ = oracle_setup(param)
    eng, key = eng_key(param)
    C = pz().Circuit()
    a, b = C.input_u8(), C.input_u8()
    C.outputs(C.u8_mul(a, b))
    C.output(C.u8_cmp("lt", a, b))
    r = O.Rng(b"\x05" * 32)
    for x, y in [(201, 77), (13, 250), (0, 0)]:
        inp = np.concatenate([enc_u8(ev, r, s, [x])[0], enc_u8(ev, r, s, [y])[0]])
        out = C.run(eng, key, inp)
        bits = ev.mp_decrypt_bool(r, sp, out)
        assert sum(int(v) << i for i, v in enumerate(bits[:8])) == (x * y) % 256
        assert int(bits[8]) == int(x < y)


def test_circuit_grown_after_a_run_is_rebound(gpu_available):
    """A circuit that gains inputs, gates and outputs after it ran (and after
    its graph was captured) is re-uploaded on its next run: the stale graph is
    refused, and every output of the grown circuit equals the oracle's gate
    evaluation, word for word."""
    import torch
    param = "SP_TEST"
    ev, (s, _, _, _), _, okey = oracle_setup(param)
    eng, key = eng_key(param)
    r = oracle().Rng(b"\x0b" * 32)
    bits = [1, 0, 1, 1, 0]
    cts = ev.encrypt_bool(r, s, bits)
    C = pz().Circuit()
    a, b = C.input(), C.input()
    w0 = C.gate("nand", a, b)
    C.output(w0)
    first = C.run(eng, key, cts[:2])
    assert np.array_equal(first[0], okey.gate("nand", cts[0], cts[1]))
    d_in = to_dev(cts[:2])
    d_out = to_dev(np.zeros((1, ev.L), np.uint64))
    C.capture_graph(eng, key, d_in, d_out)
    # grow: three more inputs, gates reading old and new wires, two more outputs
    c, d, e = C.input(), C.input(), C.input()
    w1 = C.gate("xor", w0, c)
    w2 = C.gate("or", C.not_(w1), d)
    w3 = C.gate("and", w2, e)
    C.output(w1)
    C.output(w3)
    with pytest.raises(RuntimeError):
        C.replay_graph()
    got = C.run(eng, key, cts)
    v0 = okey.gate("nand", cts[0], cts[1])
    v1 = okey.gate("xor", v0, cts[2])
    v2 = okey.gate("or", ev.not_(v1), cts[3])
    v3 = okey.gate("and", v2, cts[4])
    assert np.array_equal(got, np.stack([v0, v1, v3]))
    # the device path binds the grown circuit too
    d_in = to_dev(cts)
    d_out = to_dev(np.zeros((3, ev.L), np.uint64))
    C.run_device(eng, key, d_in, d_out)
    torch.cuda.synchronize()
    assert np.array_equal(to_host(d_out).reshape(3, ev.L), got)
    truth = [1 - (bits[0] & bits[1])]
    truth.append(truth[0] ^ bits[2])
    truth.append(((1 - truth[1]) | bits[3]) & bits[4])
    assert list(ev.decrypt_bool(s, got)) == truth
