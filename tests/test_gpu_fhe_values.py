"""Eager FheBool / FheUint8 operators on the GPU (bool/mod.rs:120-200,
shortint/mod.rs:16-292) at the production InteractiveLTE2Party set: chained
operators decrypt to the plaintext results, single operators are bit-exact
with the oracle's sequential gates, and the division-by-zero flag follows
the reference (OR-accumulated by / and div_rem, untouched by %, cleared by
reset_error_flags)."""
import numpy as np
import pytest

from conftest import oracle, oracle_setup, pz

pytestmark = pytest.mark.gpu

PARAM = "I_2P_LB_SR"


@pytest.fixture(scope="module")
def ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    P = pz()
    ev, (s, _, _, _), coeff, okey = oracle_setup(PARAM)
    eng = P.Engine(PARAM)
    key = eng.upload_key(coeff.rgsw, coeff.autos, coeff.ksk)
    P.clear_server_key()
    P.set_server_key(eng, key)
    rng = oracle().Rng(b"\x61" * 32)

    def enc(v):
        return P.FheUint8(ev.encrypt_bool(rng, s, np.array([(v >> i) & 1 for i in range(8)])))

    def encb(bit):
        return P.FheBool(ev.encrypt_bool(rng, s, np.array([bit]))[0])

    def dec(x):
        if isinstance(x, P.FheBool):
            return int(ev.decrypt_bool(s, x.lwe().reshape(1, -1))[0])
        bits = ev.decrypt_bool(s, x.lwe()).astype(np.int64)
        return int((bits << np.arange(8)).sum())

    yield P, ev, okey, enc, encb, dec
    P.reset_error_flags()
    P.clear_server_key()


def test_chained_arithmetic(ctx):
    P, _, _, enc, _, dec = ctx
    for a, b in [(200, 7), (13, 0), (255, 255), (0, 1), (128, 3)]:
        x, y = enc(a), enc(b)
        z = x + y
        z += y
        assert dec(z) == (a + 2 * b) % 256
        w = x * y - z
        assert dec(w) == (a * b - (a + 2 * b)) % 256
        s, ov = x.overflowing_add(y)
        assert (dec(s), dec(ov)) == ((a + b) % 256, int(a + b > 255))
        d, ov = x.overflowing_sub(y)
        assert (dec(d), dec(ov)) == ((a - b) % 256, int(a < b))
        t = enc(a)
        ov = t.overflowing_add_assign(y)
        assert (dec(t), dec(ov)) == ((a + b) % 256, int(a + b > 255))


def test_division_and_flag(ctx):
    P, _, _, enc, _, dec = ctx
    P.reset_error_flags()
    assert P.div_zero_error_flag() is None
    x, y, zero = enc(200), enc(7), enc(0)
    assert dec(x / y) == 28 and dec(x // y) == 28
    assert dec(P.div_zero_error_flag()) == 0
    assert dec(x % zero) == 200  # remainder leaves the flag alone
    assert dec(P.div_zero_error_flag()) == 0
    q, r = x.div_rem(zero)
    assert (dec(q), dec(r)) == (255, 200)
    assert dec(P.div_zero_error_flag()) == 1
    q, r = x.div_rem(y)  # OR-accumulated: stays set
    assert (dec(q), dec(r)) == (28, 4)
    assert dec(P.div_zero_error_flag()) == 1
    P.reset_error_flags()
    assert P.div_zero_error_flag() is None
    assert dec(x % y) == 4
    assert P.div_zero_error_flag() is None


def test_comparisons_and_selection(ctx):
    P, _, _, enc, encb, dec = ctx
    for a, b in [(5, 9), (9, 5), (77, 77), (0, 255)]:
        x, y = enc(a), enc(b)
        got = [dec(getattr(x, op)(y)) for op in ["eq", "neq", "lt", "gt", "le", "ge"]]
        assert got == [int(a == b), int(a != b), int(a < b), int(a > b), int(a <= b), int(a >= b)]
        assert dec(x.max(y)) == max(a, b) and dec(x.min(y)) == min(a, b)
        for sel in (0, 1):
            assert dec(x.mux(y, encb(sel))) == (a if sel else b)


def test_bool_operators(ctx):
    P, _, _, _, encb, dec = ctx
    for p in (0, 1):
        for q in (0, 1):
            x, y = encb(p), encb(q)
            assert dec(x & y) == (p & q) and dec(x | y) == (p | q) and dec(x ^ y) == (p ^ q)
            assert dec(x.nand(y)) == 1 - (p & q) and dec(x.nor(y)) == 1 - (p | q)
            assert dec(x.xnor(y)) == 1 - (p ^ q) and dec(~x) == 1 - p
            z = encb(p)
            z &= y
            z |= x
            z ^= y
            assert dec(z) == (((p & q) | p) ^ q)


def test_bytes_compose(ctx):
    P, _, _, enc, encb, dec = ctx
    x = enc(0b10110010)
    bits = x.bits()
    assert [dec(b) for b in bits] == [(0b10110010 >> i) & 1 for i in range(8)]
    assert dec(P.FheUint8.from_bools(bits[::-1])) == 0b01001101


def test_operators_bit_exact_with_oracle(ctx):
    """One operator each: the eager path gives the oracle's ciphertexts."""
    P, ev, okey, enc, _, _ = ctx
    x, y = enc(150), enc(3)
    a, b = x.lwe(), y.lwe()
    assert np.array_equal((x + y).lwe(), okey.u8_op("add", a, b)[0])
    assert np.array_equal(x.lt(y).lwe(), okey.u8_op("lt", a, b)[0][0])
    P.reset_error_flags()
    zero = enc(0)
    q0, _ = x.div_rem(zero)
    flag0 = P.div_zero_error_flag().lwe()
    q, r = x.div_rem(y)  # with the flag of the first division OR'd in
    want_q0, _, want_f0 = okey.u8_op("div_rem", a, zero.lwe(), flag=None)
    assert np.array_equal(q0.lwe(), want_q0) and np.array_equal(flag0, want_f0)
    want_q, want_r, want_f = okey.u8_op("div_rem", a, b, flag=flag0)
    assert np.array_equal(q.lwe(), want_q) and np.array_equal(r.lwe(), want_r)
    assert np.array_equal(P.div_zero_error_flag().lwe(), want_f)
    P.reset_error_flags()
