"""Known-answer pins of the seed expansion, for the product and the oracle.

The reference expands every seeded key part and unseeds client ciphertexts
with rand_chacha 0.3.1's ChaCha8Rng and rand 0.8.5's
Uniform::new_inclusive(0, q - 1) (random.rs:93-110; call sites
bool/keys.rs:711-718,763-771, bool/enc_dec.rs:82-96).  Neither crate is in
this image, so these pins come from published vectors: the ChaCha block
function of RFC 8439 (section 2.3.2 and appendix A.1, 20 rounds), the
published ChaCha8 vector for an all-zero 256-bit key and IV, and hand-worked
cases of the uniform sampler's rejection zone.  The product's block function
(the same template runs on the device in the seeded fill) and the oracle's are
checked separately, so a mistake shared by both restatements would fail here.
"""
import ctypes

import numpy as np

from conftest import oracle, pz

SIGMA = [0x61707865, 0x3320646E, 0x79622D32, 0x6B206574]

# RFC 8439 section 2.3.2: key 00:01:..:1f, counter 1, nonce 00:00:00:09:00:00:00:4a:00:00:00:00
RFC_STATE = SIGMA + [0x03020100, 0x07060504, 0x0B0A0908, 0x0F0E0D0C, 0x13121110, 0x17161514, 0x1B1A1918,
                     0x1F1E1D1C, 0x00000001, 0x09000000, 0x4A000000, 0x00000000]
RFC_OUT = [0xE4E7F110, 0x15593BD1, 0x1FDD0F50, 0xC47120A3, 0xC7F4D1C7, 0x0368C033, 0x9AAA2204, 0x4E6CD4C3,
           0x466482D2, 0x09AA9F07, 0x05D7C214, 0xA2028BD9, 0xD19C12B5, 0xB94E16DE, 0xE883D0CB, 0x4E3C50A2]
ZERO_STATE = SIGMA + [0] * 12
# RFC 8439 appendix A.1, test vector 1: all-zero key and nonce, block 0, 20 rounds
ZERO_OUT_20 = bytes.fromhex("76b8e0ada0f13d90405d6ae55386bd28bdd219b8a08ded1aa836efcc8b770dc7"
                            "da41597c5157488d7724e03fb8d84a376a43b8f41518a11cc387b669b2ee6586")
# ChaCha with 8 rounds, all-zero 256-bit key and all-zero IV, first block (the
# published reduced-round ChaCha test vectors, 256-bit key case)
ZERO_OUT_8 = bytes.fromhex("3e00ef2f895f40d67f5bb8e81f09a5a12c840ec3ce9a7f3b181be188ef711a1e"
                           "984ce172b9216f419f445367456d5619314a42a3da86b001387bfdb80e0cfe42")


def product_block(state, rounds):
    P = pz()
    s = (ctypes.c_uint32 * 16)(*state)
    out = (ctypes.c_uint32 * 16)()
    assert P._lib.lib().pz_chacha_block(s, rounds, out) == 0
    return list(out)


def words_le(b):
    return list(np.frombuffer(b, dtype="<u4"))


def test_chacha20_rfc8439_block():
    assert product_block(RFC_STATE, 20) == RFC_OUT
    assert list(oracle().chacha_block(RFC_STATE, 20)) == RFC_OUT


def test_chacha20_zero_key_rfc8439_a1():
    assert product_block(ZERO_STATE, 20) == words_le(ZERO_OUT_20)
    assert list(oracle().chacha_block(ZERO_STATE, 20)) == words_le(ZERO_OUT_20)


def test_chacha8_zero_key_and_rand_chacha_layout():
    """8 rounds against the published zero-key vector; the oracle's ChaCha8Rng
    (rand_chacha layout: 64-bit block counter in words 12-13, stream id 0 in
    words 14-15, seed = key) emits that block's words for the all-zero seed,
    low word first in each u64 (rand_core's BlockRng::next_u64)."""
    want = words_le(ZERO_OUT_8)
    assert product_block(ZERO_STATE, 8) == want
    assert list(oracle().chacha_block(ZERO_STATE, 8)) == want
    O = oracle()
    r = O.Rng(bytes(32))
    got = [O.lib().orc_rng_next_u64(r.h) for _ in range(8)]
    assert got == [int(want[2 * i]) | (int(want[2 * i + 1]) << 32) for i in range(8)]


def test_bad_round_count_is_rejected():
    s = (ctypes.c_uint32 * 16)(*ZERO_STATE)
    out = (ctypes.c_uint32 * 16)()
    assert pz()._lib.lib().pz_chacha_block(s, 7, out) != 0


def product_uniform(q, word):
    v, acc = ctypes.c_uint64(), ctypes.c_int()
    assert pz()._lib.lib().pz_uniform_mod_word(q, word, ctypes.byref(v), ctypes.byref(acc)) == 0
    return bool(acc.value), v.value


# (q, word, accepted, sample), worked by hand from rand 0.8's UniformInt:
# zone = 2^64 - 1 - (2^64 - q) mod q; accept iff lo64(word q) <= zone;
# sample = hi64(word q).
#   q = 2^63 + 1: (2^64 - q) mod q = 2^63 - 1, zone = 2^63;
#     word 2^63 -> lo = 2^63 (= zone: accepted), hi = 2^62
#     word 1    -> lo = 2^63 + 1 (zone + 1: rejected)
#     word 2    -> lo = 2, hi = 1;  word 2^63 + 1 -> lo = 1, hi = 2^62 + 1
#     word 2^63 - 1 -> lo = 2^64 - 1 (rejected)
#   q = 3: 2^64 = 1 (mod 3), zone = 2^64 - 2;
#     word 0xAAAAAAAAAAAAAAAA -> 3 word = 2^65 - 2: lo = 2^64 - 2 (= zone), hi = 1
#     word 0x5555555555555555 -> 3 word = 2^64 - 1: lo = 2^64 - 1 (rejected)
#     word 0xAAAAAAAAAAAAAAAB -> 3 word = 2^65 + 1: lo = 1, hi = 2
UNIFORM_CASES = [
    (2**63 + 1, 2**63, True, 2**62),
    (2**63 + 1, 1, False, None),
    (2**63 + 1, 2, True, 1),
    (2**63 + 1, 2**63 + 1, True, 2**62 + 1),
    (2**63 + 1, 2**63 - 1, False, None),
    (3, 0xAAAAAAAAAAAAAAAA, True, 1),
    (3, 0x5555555555555555, False, None),
    (3, 0xAAAAAAAAAAAAAAAB, True, 2),
]


def test_uniform_rejection_zone_hand_worked():
    O = oracle()
    for q, w, acc, sample in UNIFORM_CASES:
        for got in (product_uniform(q, w), O.uniform_mod_word(q, w)):
            assert got[0] == acc, (q, w)
            if acc:
                assert got[1] == sample, (q, w)


def test_uniform_rejection_zone_at_the_rlwe_prime():
    """Q = 2^54 - 77823: (2^64 - Q) mod Q = 2^64 mod Q = 2^10 * 77823, so the
    zone's complement holds 79,691,776 of the 2^64 words; the words whose
    product with Q lands just on either side of the zone decide the same way in
    the product and the oracle."""
    Q = 18014398509404161
    rej = (2**64 - Q) % Q
    assert rej == 1024 * 77823
    zone = 2**64 - 1 - rej
    O = oracle()
    # lo64(w Q) walks through every residue class as w varies; find words whose
    # low product sits at zone and zone + 1 (w = t Q^-1 mod 2^64)
    qinv = pow(Q, -1, 2**64)
    for lo, acc in [(zone, True), (zone + 1, False), (2**64 - 1, False), (0, True)]:
        w = (lo * qinv) % 2**64
        assert (w * Q) % 2**64 == lo
        for got in (product_uniform(Q, w), O.uniform_mod_word(Q, w)):
            assert got[0] == acc
            if acc:
                assert got[1] == (w * Q) >> 64
