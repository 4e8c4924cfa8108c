"""FheUint8 plaintext semantics at the strength of the reference's own test
(bool/mp_api.rs:491-660 `all_uint8_apis`: + - * / % == > < >= <= and mux over
encrypted u8 pairs, division by zero giving quotient 255, remainder = the
dividend and the error flag set).

The reference walks all 256 x 256 pairs one gate at a time on the CPU at its
single-party test set SP_TEST_BOOL_PARAMS.  That set (LWE dimension 100 with
a Gaussian secret, blind-rotation modulus 512) bootstraps a gate wrongly
about once in 10^4 in the restated algorithm -- measured on the oracle, and
what the odd mod switch's noise against the test vector's 64/512 margin
predicts -- so an exhaustive run there meets wrong bits whatever the
implementation.  Here each operator is one batched circuit on the GPU at the
production InteractiveLTE2Party set (keys under the parties' summed secret,
every output decrypted):

* div_rem: every divisor 0..255 against the dividends 0, 1, 127, 128, 255
  (1,280 pairs, 256 of them with divisor 0 -- quotient, remainder and flag);
* + - * and the six comparisons: the 16 x 16 grid of edge values below
  (256 pairs each);
* mux: the same grid, selector alternating.
"""
import numpy as np
import pytest

from conftest import oracle, oracle_setup, pz

pytestmark = pytest.mark.gpu

PARAM = "I_2P_LB_SR"
EDGE = [0, 1, 2, 3, 7, 8, 15, 16, 31, 64, 127, 128, 129, 200, 254, 255]
DIVIDENDS = [0, 1, 127, 128, 255]

_ENG = {}


def eng_key():
    if PARAM not in _ENG:
        ev, _, coeff, _ = oracle_setup(PARAM)
        eng = pz().Engine(PARAM)
        _ENG[PARAM] = (eng, eng.upload_key(coeff.rgsw, coeff.autos, coeff.ksk))
    return _ENG[PARAM]


def encrypt_pairs(ev, s, pairs, seed, with_sel=False):
    """Input ciphertexts [a bits, b bits (, selector)] per pair, LSB first."""
    bits = []
    for k, (a, b) in enumerate(pairs):
        bits += [(a >> i) & 1 for i in range(8)] + [(b >> i) & 1 for i in range(8)]
        if with_sel:
            bits.append(k & 1)
    return ev.encrypt_bool(oracle().Rng(bytes([seed]) * 32), s, np.array(bits))


def decrypt_u8(ev, s, cts):
    bits = ev.decrypt_bool(s, cts.reshape(-1, ev.L)).reshape(-1, 8).astype(np.int64)
    return (bits << np.arange(8)).sum(axis=1)


def run(C, inputs):
    eng, key = eng_key()
    return C.run(eng, key, inputs)


def test_div_rem_every_divisor(gpu_available):
    ev, (s, _, _, _), _, _ = oracle_setup(PARAM)
    pairs = [(a, b) for b in range(256) for a in DIVIDENDS]
    C = pz().Circuit()
    outs = []
    for _ in pairs:
        a, b = C.input_u8(), C.input_u8()
        outs.append(C.u8_div_rem(a, b))  # each with its own flag: is_zero(b)
    for q, r, f in outs:
        C.outputs(q)
        C.outputs(r)
        C.output(f)
    got = run(C, encrypt_pairs(ev, s, pairs, 0x21)).reshape(len(pairs), 17, ev.L)
    quo = decrypt_u8(ev, s, got[:, :8])
    rem = decrypt_u8(ev, s, got[:, 8:16])
    flag = ev.decrypt_bool(s, np.ascontiguousarray(got[:, 16]))
    for k, (a, b) in enumerate(pairs):
        if b == 0:  # mp_api.rs:553-589: quotient 255, remainder a, flag set
            assert (quo[k], rem[k], flag[k]) == (255, a, 1), (a, b, quo[k], rem[k], flag[k])
        else:
            assert (quo[k], rem[k], flag[k]) == (a // b, a % b, 0), (a, b, quo[k], rem[k], flag[k])


GRID = [(a, b) for a in EDGE for b in EDGE]


@pytest.mark.parametrize("op", ["add", "sub", "mul"])
def test_arithmetic_edge_grid(gpu_available, op):
    ev, (s, _, _, _), _, _ = oracle_setup(PARAM)
    C = pz().Circuit()
    for _ in GRID:
        a, b = C.input_u8(), C.input_u8()
        C.outputs({"add": C.u8_add, "sub": C.u8_sub, "mul": C.u8_mul}[op](a, b))
    got = decrypt_u8(ev, s, run(C, encrypt_pairs(ev, s, GRID, 0x22)))
    want = {"add": lambda a, b: (a + b) % 256, "sub": lambda a, b: (a - b) % 256,
            "mul": lambda a, b: (a * b) % 256}[op]
    for k, (a, b) in enumerate(GRID):
        assert got[k] == want(a, b), (op, a, b, got[k])


def test_comparisons_edge_grid(gpu_available):
    ev, (s, _, _, _), _, _ = oracle_setup(PARAM)
    ops = {"eq": lambda a, b: a == b, "neq": lambda a, b: a != b, "lt": lambda a, b: a < b,
           "gt": lambda a, b: a > b, "le": lambda a, b: a <= b, "ge": lambda a, b: a >= b}
    C = pz().Circuit()
    for _ in GRID:
        a, b = C.input_u8(), C.input_u8()
        for op in ops:
            C.output(C.u8_cmp(op, a, b))
    got = ev.decrypt_bool(s, run(C, encrypt_pairs(ev, s, GRID, 0x23))).reshape(len(GRID), len(ops))
    for k, (a, b) in enumerate(GRID):
        for i, (op, f) in enumerate(ops.items()):
            assert got[k, i] == int(f(a, b)), (op, a, b)


def test_mux_edge_grid(gpu_available):
    ev, (s, _, _, _), _, _ = oracle_setup(PARAM)
    C = pz().Circuit()
    for _ in GRID:
        a, b = C.input_u8(), C.input_u8()
        sel = C.input()
        C.outputs(C.u8_mux(a, b, sel))  # selector ? a : b (shortint/mod.rs:273-279)
    got = decrypt_u8(ev, s, run(C, encrypt_pairs(ev, s, GRID, 0x24, with_sel=True)))
    for k, (a, b) in enumerate(GRID):
        assert got[k] == (a if k & 1 else b), (a, b, k & 1, got[k])
