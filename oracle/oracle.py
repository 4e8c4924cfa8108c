"""ctypes wrapper over the CPU oracle (oracle/_build/liboracle_pz.so).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA product.  Only tests/,
``__graft_entry__.smoke()`` and ``bench.py``'s cpu_baseline / reference legs
may import this module.  The oracle restates the reference's Rust path
(see pz_oracle.h for the file:line map); its equality with the Rust binary
is unpinned because the Rust reference cannot be built here.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle_pz.so")

u64p = ctypes.POINTER(ctypes.c_uint64)
u32p = ctypes.POINTER(ctypes.c_uint32)
u8p = ctypes.POINTER(ctypes.c_uint8)
i32p = ctypes.POINTER(ctypes.c_int32)
vp = ctypes.c_void_p

PARAM_IDS = {
    "I_2P_LB_SR": 0, "I_4P": 1, "I_8P": 2, "NI_2P": 3,
    "NI_4P_HB_FR": 4, "NI_4P_LB_SR": 5, "NI_8P": 6, "SP_TEST": 7,
}
GATES = {"and": 0, "nand": 1, "or": 2, "nor": 3, "xor": 4, "xnor": 5}


class ParamInfo(ctypes.Structure):
    _fields_ = [
        ("rlwe_q", ctypes.c_uint64), ("lwe_q", ctypes.c_uint64),
        ("br_q", ctypes.c_uint32), ("rlwe_n", ctypes.c_uint32), ("lwe_n", ctypes.c_uint32),
        ("lwe_logb", ctypes.c_uint32), ("lwe_d", ctypes.c_uint32),
        ("rlrg_logb", ctypes.c_uint32), ("rlrg_d_a", ctypes.c_uint32), ("rlrg_d_b", ctypes.c_uint32),
        ("auto_logb", ctypes.c_uint32), ("auto_d", ctypes.c_uint32),
        ("g", ctypes.c_uint32), ("w", ctypes.c_uint32),
        ("lwe_secret_gaussian", ctypes.c_uint32), ("variant", ctypes.c_uint32),
        ("embedding_factor", ctypes.c_uint32), ("rgsw_rows", ctypes.c_uint32),
        ("auto_rows", ctypes.c_uint32), ("n_auto_keys", ctypes.c_uint32),
        ("ni_ks_logb", ctypes.c_uint32), ("ni_ks_d", ctypes.c_uint32),
        ("rgrg_logb", ctypes.c_uint32), ("rgrg_d_a", ctypes.c_uint32), ("rgrg_d_b", ctypes.c_uint32),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise RuntimeError(f"oracle library missing: {_LIB_PATH} (run `make -C oracle`)")
        L = ctypes.CDLL(_LIB_PATH)
        sig = {
            "orc_param_info_get": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ParamInfo)]),
            "orc_eval_new": (vp, [ctypes.c_int]),
            "orc_eval_free": (None, [vp]),
            "orc_eval_psi": (ctypes.c_uint64, [vp]),
            "orc_eval_tables": (None, [vp, u64p, u64p, u64p]),
            "orc_eval_test_vec": (None, [vp, ctypes.c_int, u64p]),
            "orc_eval_dlog_map": (None, [vp, u32p]),
            "orc_eval_auto_map": (None, [vp, ctypes.c_int, u32p, u8p]),
            "orc_ntt_forward": (None, [vp, u64p, ctypes.c_int]),
            "orc_ntt_backward": (None, [vp, u64p, ctypes.c_int]),
            "orc_decompose": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_uint64, u64p]),
            "orc_shoup_matrix_fma": (None, [ctypes.c_uint64, u64p, u64p, u64p, u64p, ctypes.c_size_t, ctypes.c_size_t]),
            "orc_shoup_repr": (ctypes.c_uint64, [ctypes.c_uint64, ctypes.c_uint64]),
            "orc_barrett_mul": (ctypes.c_uint64, [vp, ctypes.c_uint64, ctypes.c_uint64]),
            "orc_negacyclic_mul": (None, [ctypes.c_uint64, u64p, u64p, u64p, ctypes.c_size_t]),
            "orc_key_new": (vp, [vp, u64p, u64p, u64p]),
            "orc_key_free": (None, [vp]),
            "orc_rlwe_by_rgsw": (None, [vp, vp, u64p, ctypes.c_uint32, ctypes.c_int, ctypes.c_int]),
            "orc_rlwe_auto": (None, [vp, vp, u64p, ctypes.c_uint32, ctypes.c_int, ctypes.c_int]),
            "orc_lwe_key_switch": (None, [vp, vp, u64p, u64p]),
            "orc_pbs": (ctypes.c_int, [vp, vp, ctypes.c_int, u64p, u64p, u64p]),
            "orc_gate": (None, [vp, vp, ctypes.c_int, u64p, u64p]),
            "orc_not": (None, [vp, u64p]),
            "orc_gate_batch": (None, [vp, vp, u8p, u64p, u64p, u64p, ctypes.c_size_t, ctypes.c_int]),
            "orc_sample_extract": (None, [vp, u64p, u64p, ctypes.c_uint32]),
            "orc_ni_unseed": (None, [vp, u8p, u64p, ctypes.c_size_t, u64p]),
            "orc_ni_key_switch": (None, [vp, u64p, u64p, u64p]),
            "orc_ni_encrypt_bools": (None, [vp, i32p, u8p, u8p, u8p, ctypes.c_size_t, u64p]),
            "orc_ni_ksk_gen": (None, [vp, i32p, i32p, u8p, u64p]),
            "orc_expand_seeded_key": (None, [vp, u64p, u8p, u64p, u8p, u64p, u64p]),
            "orc_expand_ni_ksk": (None, [vp, u64p, u8p, u64p]),
            "orc_rgsw_by_rgsw": (None, [vp, u64p, u64p]),
            "orc_rgsw_encrypt": (None, [vp, i32p, u64p, ctypes.c_int, u8p, u64p]),
            "orc_ni_crs_seed": (None, [u8p, ctypes.c_int, ctypes.c_size_t, u8p]),
            "orc_interactive_crs_seed": (None, [u8p, ctypes.c_int, u8p]),
            "orc_ni_aggregate": (None, [vp, u8p, ctypes.c_int] + [ctypes.POINTER(u64p)] * 7 +
                                 [ctypes.c_size_t, ctypes.c_size_t, u64p, u64p, u64p, u64p]),
            "orc_gen_seeded_auto_lwe": (None, [vp, i32p, i32p, u8p, u8p, u8p, u64p, u64p]),
            "orc_ni_gen_share": (None, [vp, u8p, ctypes.c_int, ctypes.c_int, i32p, i32p, i32p, u8p, u64p, u64p,
                                        u64p, u64p, u64p]),
            "orc_u8_op": (ctypes.c_int, [vp, vp, ctypes.c_int, u64p, u64p, u64p, u64p, u64p, u64p, ctypes.POINTER(ctypes.c_int)]),
            "orc_u8_gate_mix": (ctypes.c_int, [vp, ctypes.c_int, u64p]),
            "orc_generate_prime": (ctypes.c_uint64, [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64]),
            "orc_ntt_custom_new": (vp, [ctypes.c_uint64, ctypes.c_size_t]),
            "orc_ntt_custom_free": (None, [vp]),
            "orc_ntt_custom_forward": (None, [vp, u64p, ctypes.c_int]),
            "orc_ntt_custom_backward": (None, [vp, u64p, ctypes.c_int]),
            "orc_mul_mod_barrett": (ctypes.c_uint64, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]),
            "orc_decompose_custom": (ctypes.c_uint32, [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, u64p]),
            "orc_round_value": (ctypes.c_uint64, [ctypes.c_uint64, ctypes.c_uint32]),
            "orc_recompose": (ctypes.c_uint64, [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, u64p]),
            "orc_chacha_block": (None, [u32p, ctypes.c_int, u32p]),
            "orc_uniform_mod_word": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint64, u64p]),
            "orc_rng_new": (vp, [u8p]),
            "orc_rng_free": (None, [vp]),
            "orc_rng_next_u64": (ctypes.c_uint64, [vp]),
            "orc_rng_uniform_mod": (None, [vp, ctypes.c_uint64, u64p, ctypes.c_size_t]),
            "orc_client_keys": (None, [vp, ctypes.c_int, ctypes.c_int, i32p, i32p, i32p, i32p]),
            "orc_gen_server_key": (None, [vp, i32p, i32p, u8p, u64p, u64p, u64p]),
            "orc_encrypt_bool": (None, [vp, vp, i32p, ctypes.c_int, u64p]),
            "orc_decrypt_bool": (ctypes.c_int, [vp, i32p, u64p]),
            "orc_mp_decryption_share": (ctypes.c_uint64, [vp, vp, i32p, u64p]),
            "orc_mp_aggregate_decrypt": (ctypes.c_int, [vp, u64p, u64p, ctypes.c_int]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a, t=u64p):
    return a.ctypes.data_as(t)


def ni_crs_seed(crs, what, index=0):
    """NonInteractiveMultiPartyCrs seed (evaluator.rs:115-172): what 0 auto keys, 1 LWE KSK,
    2 ui_to_s KSK of user `index`, 3 NI RGSW of LWE index `index`."""
    out = (ctypes.c_uint8 * 32)()
    lib().orc_ni_crs_seed((ctypes.c_uint8 * 32)(*bytes(crs)), int(what), int(index), out)
    return bytes(out)


def interactive_crs_seed(crs, what):
    """InteractiveMultiPartyCrs seed (evaluator.rs:78-100): what 0 public-key share, 1 auto keys, 2 LWE KSK."""
    out = (ctypes.c_uint8 * 32)()
    lib().orc_interactive_crs_seed((ctypes.c_uint8 * 32)(*bytes(crs)), int(what), out)
    return bytes(out)


def param_info(name_or_id):
    pid = PARAM_IDS[name_or_id] if isinstance(name_or_id, str) else int(name_or_id)
    info = ParamInfo()
    if lib().orc_param_info_get(pid, ctypes.byref(info)) != 0:
        raise ValueError(f"unknown parameter set {name_or_id}")
    return info


def chacha_block(state, rounds):
    """The ChaCha block function on a 16-word input state (out = rounds(state) + state)."""
    s = np.ascontiguousarray(state, np.uint32)
    out = np.zeros(16, np.uint32)
    lib().orc_chacha_block(_p(s, u32p), int(rounds), _p(out, u32p))
    return out


def uniform_mod_word(q, word):
    """rand 0.8's uniform sampler for [0, q) on one 64-bit word: (accepted, sample)."""
    v = ctypes.c_uint64()
    ok = lib().orc_uniform_mod_word(int(q), int(word), ctypes.byref(v))
    return bool(ok), v.value


class Rng:
    """ChaCha8 stream; seed is 32 bytes."""

    def __init__(self, seed):
        seed = bytes(seed)
        assert len(seed) == 32
        self._seed = (ctypes.c_uint8 * 32)(*seed)
        self.h = lib().orc_rng_new(self._seed)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None and lib is not None:
            _lib.orc_rng_free(self.h)
            self.h = None

    def uniform_mod(self, q, n):
        out = np.empty(n, dtype=np.uint64)
        lib().orc_rng_uniform_mod(self.h, q, _p(out), n)
        return out


class ServerKeyCoeff:
    """Coefficient-domain expanded server key (layout of orc_key_new)."""

    def __init__(self, rgsw, autos, ksk):
        self.rgsw, self.autos, self.ksk = rgsw, autos, ksk


class Evaluator:
    """Oracle BoolEvaluator for one parameter set."""

    def __init__(self, param):
        self.pid = PARAM_IDS[param] if isinstance(param, str) else int(param)
        self.info = param_info(self.pid)
        self.h = lib().orc_eval_new(self.pid)
        i = self.info
        self.N, self.n, self.Q = i.rlwe_n, i.lwe_n, i.rlwe_q
        self.L = self.N + 1

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_eval_free(self.h)
            self.h = None

    # --- tables -------------------------------------------------------------
    def psi(self):
        return lib().orc_eval_psi(self.h)

    def tables(self):
        a = np.empty(self.N, np.uint64)
        b = np.empty(self.N, np.uint64)
        ni = (ctypes.c_uint64 * 1)()
        lib().orc_eval_tables(self.h, _p(a), _p(b), ni)
        return a, b, int(ni[0])

    def test_vec(self, gate):
        out = np.empty(self.info.br_q // 2, np.uint64)
        lib().orc_eval_test_vec(self.h, GATES[gate] if isinstance(gate, str) else gate, _p(out))
        return out

    def dlog_map(self):
        out = np.empty(self.info.br_q, np.uint32)
        lib().orc_eval_dlog_map(self.h, _p(out, u32p))
        return out

    def auto_map(self, k):
        idx = np.empty(self.N, np.uint32)
        sgn = np.empty(self.N, np.uint8)
        lib().orc_eval_auto_map(self.h, k, _p(idx, u32p), _p(sgn, u8p))
        return idx, sgn

    # --- arithmetic -------------------------------------------------------------
    def ntt_forward(self, poly, lazy=False):
        a = np.ascontiguousarray(poly, dtype=np.uint64).copy()
        lib().orc_ntt_forward(self.h, _p(a), int(lazy))
        return a

    def ntt_backward(self, poly, lazy=False):
        a = np.ascontiguousarray(poly, dtype=np.uint64).copy()
        lib().orc_ntt_backward(self.h, _p(a), int(lazy))
        return a

    def decompose(self, which, value):
        out = np.zeros(64, np.uint64)
        d = lib().orc_decompose(self.h, which, int(value), _p(out))
        return out[:d]

    def barrett_mul(self, a, b):
        return lib().orc_barrett_mul(self.h, int(a), int(b))

    # --- keys ---------------------------------------------------------------
    def client_keys(self, parties, seed_base=0):
        N, n = self.N, self.n
        s = np.empty(N, np.int32)
        z = np.empty(n, np.int32)
        sp = np.empty((parties, N), np.int32)
        zp = np.empty((parties, n), np.int32)
        lib().orc_client_keys(self.h, parties, seed_base, _p(s, i32p), _p(z, i32p),
                              _p(sp, i32p), _p(zp, i32p))
        return s, z, sp, zp

    def gen_server_key(self, s, z, err_seed=b"\x33" * 32):
        i = self.info
        N, n = self.N, self.n
        rgsw = np.empty((n, i.rgsw_rows, N), np.uint64)
        autos = np.empty((i.n_auto_keys, i.auto_rows, N), np.uint64)
        ksk = np.empty((i.lwe_d * N, n + 1), np.uint64)
        seed = (ctypes.c_uint8 * 32)(*bytes(err_seed))
        lib().orc_gen_server_key(self.h, _p(np.ascontiguousarray(s, np.int32), i32p),
                                 _p(np.ascontiguousarray(z, np.int32), i32p), seed,
                                 _p(rgsw), _p(autos), _p(ksk))
        return ServerKeyCoeff(rgsw, autos, ksk)

    def key(self, coeff):
        return OracleKey(self, coeff)

    # --- client -----------------------------------------------------------------
    def encrypt_bool(self, rng, s, bits):
        bits = np.atleast_1d(np.asarray(bits, dtype=np.int64))
        out = np.empty((len(bits), self.L), np.uint64)
        sp = _p(np.ascontiguousarray(s, np.int32), i32p)
        for k, b in enumerate(bits):
            row = out[k]
            lib().orc_encrypt_bool(self.h, rng.h, sp, int(b), _p(row))
        return out

    def u8_gate_mix(self, op):
        """Gates the FheUint8 operation `op` issues, by gate code (and, nand,
        or, nor, xor, xnor), from a dry run of the sequential restatement."""
        counts = np.zeros(6, np.uint64)
        assert lib().orc_u8_gate_mix(self.h, OracleKey.U8_OPS[op], _p(counts)) == 0
        return counts.astype(np.int64)

    def decrypt_bool(self, s, cts):
        cts = np.atleast_2d(np.ascontiguousarray(cts, np.uint64))
        sp = _p(np.ascontiguousarray(s, np.int32), i32p)
        return np.array([lib().orc_decrypt_bool(self.h, sp, _p(np.ascontiguousarray(c))) for c in cts])

    def mp_decrypt_bool(self, rng, s_parts, cts):
        cts = np.atleast_2d(np.ascontiguousarray(cts, np.uint64))
        out = []
        P = len(s_parts)
        for c in cts:
            c = np.ascontiguousarray(c)
            shares = np.array([lib().orc_mp_decryption_share(
                self.h, rng.h, _p(np.ascontiguousarray(s_parts[p], np.int32), i32p), _p(c))
                for p in range(P)], dtype=np.uint64)
            out.append(lib().orc_mp_aggregate_decrypt(self.h, _p(c), _p(shares), P))
        return np.array(out)

    def sample_extract(self, rlwe, index=0):
        r = np.ascontiguousarray(rlwe, np.uint64)
        out = np.empty(self.L, np.uint64)
        lib().orc_sample_extract(self.h, _p(r), _p(out), index)
        return out

    def not_(self, c):
        a = np.ascontiguousarray(c, np.uint64).copy()
        lib().orc_not(self.h, _p(a))
        return a

    # --- non-interactive input path (NI parameter sets) ---------------------------
    NI_KS_D = 50  # ui_to_s key switch decomposition count (logb 1)

    def ni_encrypt_bools(self, u, bits, seed, err_seed=b"\x44" * 32):
        """Client: seeded RLWEs of `bits` under the user's RLWE secret u -> b [count][N]."""
        bits = np.ascontiguousarray(bits, np.uint8)
        count = (len(bits) + self.N - 1) // self.N
        out = np.empty((count, self.N), np.uint64)
        lib().orc_ni_encrypt_bools(self.h, _p(np.ascontiguousarray(u, np.int32), i32p),
                                   (ctypes.c_uint8 * 32)(*bytes(seed)), (ctypes.c_uint8 * 32)(*bytes(err_seed)),
                                   _p(bits, u8p), len(bits), _p(out))
        return out

    def ni_ksk_gen(self, u, s, err_seed=b"\x55" * 32):
        out = np.empty((2 * self.NI_KS_D, self.N), np.uint64)
        lib().orc_ni_ksk_gen(self.h, _p(np.ascontiguousarray(u, np.int32), i32p),
                             _p(np.ascontiguousarray(s, np.int32), i32p), (ctypes.c_uint8 * 32)(*bytes(err_seed)),
                             _p(out))
        return out

    def ni_unseed(self, seed, b):
        b = np.ascontiguousarray(b, np.uint64).reshape(-1, self.N)
        out = np.empty((len(b), 2, self.N), np.uint64)
        lib().orc_ni_unseed(self.h, (ctypes.c_uint8 * 32)(*bytes(seed)), _p(b), len(b), _p(out))
        return out

    def ni_key_switch(self, ksk, rlwe):
        ksk = np.ascontiguousarray(ksk, np.uint64)
        r = np.ascontiguousarray(rlwe, np.uint64)
        out = np.empty(2 * self.N, np.uint64)
        lib().orc_ni_key_switch(self.h, _p(ksk), _p(r), _p(out))
        return out.reshape(2, self.N)

    def expand_seeded_key(self, auto_b, auto_seed, lwe_b, lwe_seed):
        """Seeded server key -> coefficient-domain autos and LWE KSK (keys.rs:687-781)."""
        i = self.info
        autos = np.empty((i.n_auto_keys, i.auto_rows, self.N), np.uint64)
        ksk = np.empty((i.lwe_d * self.N, self.n + 1), np.uint64)
        lib().orc_expand_seeded_key(self.h, _p(np.ascontiguousarray(auto_b, np.uint64)),
                                    (ctypes.c_uint8 * 32)(*bytes(auto_seed)),
                                    _p(np.ascontiguousarray(lwe_b, np.uint64)),
                                    (ctypes.c_uint8 * 32)(*bytes(lwe_seed)), _p(autos), _p(ksk))
        return autos, ksk

    def expand_ni_ksk(self, b, seed):
        out = np.empty((2 * self.NI_KS_D, self.N), np.uint64)
        lib().orc_expand_ni_ksk(self.h, _p(np.ascontiguousarray(b, np.uint64)), (ctypes.c_uint8 * 32)(*bytes(seed)),
                                _p(out))
        return out

    def rgsw_rows(self, which):
        i = self.info
        return 2 * (i.rlrg_d_a + i.rlrg_d_b) if which == 0 else 2 * (i.rgrg_d_a + i.rgrg_d_b)

    def rgsw_by_rgsw(self, rgsw0, rgsw1):
        r0 = np.ascontiguousarray(rgsw0, np.uint64).copy()
        lib().orc_rgsw_by_rgsw(self.h, _p(r0), _p(np.ascontiguousarray(rgsw1, np.uint64)))
        return r0

    def rgsw_encrypt(self, s, m, which, seed=b"\x71" * 32):
        out = np.empty((self.rgsw_rows(which), self.N), np.uint64)
        lib().orc_rgsw_encrypt(self.h, _p(np.ascontiguousarray(s, np.int32), i32p),
                               _p(np.ascontiguousarray(m, np.uint64)), int(which),
                               (ctypes.c_uint8 * 32)(*bytes(seed)), _p(out))
        return out

    def lwe_segment(self, user, users):
        """multi_party_user_id_lwe_segment (evaluator.rs:613-626)."""
        per = -(-self.n // users)
        b, e = per * user, min(per * (user + 1), self.n)
        return b, max(b, e)

    def ni_gen_share(self, crs, user, users, s, u, z, err_seed):
        """RGSW / KSK parts of one user's NI server key share (evaluator.rs:1624-1975)
        -> dict of arrays (coefficient domain)."""
        N, n, d = self.N, self.n, self.NI_KS_D
        info = param_info(self.pid)
        ra, rb = info.rgrg_d_a, info.rgrg_d_b
        mx, ml = max(ra, rb), max(info.rlrg_d_a, info.rlrg_d_b)
        b, e = self.lwe_segment(user, users)
        out = dict(ui_to_s_ksk=np.empty((d, N), np.uint64),
                   ksk_zero_encs=np.empty((max(users - 1, 1), d, N), np.uint64),
                   self_leader=np.empty((max(e - b, 1), ml, N), np.uint64),
                   not_leader=np.empty((max(n - (e - b), 1), mx, N), np.uint64),
                   zero_encs=np.empty((n, ra, N), np.uint64))
        lib().orc_ni_gen_share(self.h, (ctypes.c_uint8 * 32)(*bytes(crs)), int(user), int(users),
                               _p(np.ascontiguousarray(s, np.int32), i32p), _p(np.ascontiguousarray(u, np.int32), i32p),
                               _p(np.ascontiguousarray(z, np.int32), i32p), (ctypes.c_uint8 * 32)(*bytes(err_seed)),
                               *[_p(out[k]) for k in ("ui_to_s_ksk", "ksk_zero_encs", "self_leader", "not_leader",
                                                      "zero_encs")])
        out["self_leader"] = out["self_leader"][:e - b]
        out["not_leader"] = out["not_leader"][:n - (e - b)]
        out["ksk_zero_encs"] = out["ksk_zero_encs"][:users - 1]
        return out

    def gen_seeded_auto_lwe(self, s, z, auto_seed, lwe_seed, err_seed=b"\x44" * 32):
        """Auto-key B rows [w+1][d_auto][N] and LWE-KSK column 0 [d_ks N] under (s, z), A parts
        from the two seeds' streams (the seeded server key's form)."""
        info = self.info
        auto_b = np.empty((info.w + 1, info.auto_d, self.N), np.uint64)
        lwe_b = np.empty(info.lwe_d * self.N, np.uint64)
        lib().orc_gen_seeded_auto_lwe(self.h, _p(np.ascontiguousarray(s, np.int32), i32p),
                                      _p(np.ascontiguousarray(z, np.int32), i32p),
                                      (ctypes.c_uint8 * 32)(*bytes(auto_seed)), (ctypes.c_uint8 * 32)(*bytes(lwe_seed)),
                                      (ctypes.c_uint8 * 32)(*bytes(err_seed)), _p(auto_b), _p(lwe_b))
        return auto_b, lwe_b

    def aggregate(self, shares, i0=0, i1=None):
        """aggregate_interactive_multi_party_server_key_shares (evaluator.rs:1050-1200) composed from
        the restated pieces: auto-key and LWE-KSK sums, and per LWE index l the leader's RGSW
        (rlwe x rgsw shape) times every other user's RGSW (rgsw x rgsw shape) in increasing id
        (rgsw_by_rgsw_inplace).  shares: dicts self_leader [segment][rows0][N], not_leader
        [n - segment][rows1][N], auto_keys [w+1][d_auto][N], lwe_ksk [d_ks N] (user id order).
        -> (rgsw [i1-i0][rows0][N], auto, lwe)."""
        info = self.info
        users = len(shares)
        i1 = self.n if i1 is None else i1
        auto = np.zeros_like(shares[0]["auto_keys"], dtype=object)
        lwe = np.zeros_like(shares[0]["lwe_ksk"], dtype=object)
        for sh in shares:
            auto = (auto + sh["auto_keys"].astype(object)) % self.Q
            lwe = (lwe + sh["lwe_ksk"].astype(object)) % info.lwe_q
        segs = [self.lwe_segment(u, users) for u in range(users)]
        out = []
        for li in range(i0, i1):
            lead = next(u for u, (b, e) in enumerate(segs) if b <= li < e)
            r = shares[lead]["self_leader"][li - segs[lead][0]].copy()
            for o in range(users):
                if o == lead:
                    continue
                b, e = segs[o]
                pos = li if li < b else li - (e - b)
                r = self.rgsw_by_rgsw(r, shares[o]["not_leader"][pos])
            out.append(r)
        return np.stack(out), auto.astype(np.uint64), lwe.astype(np.uint64)

    def ni_aggregate(self, crs, shares, i0=0, i1=None, threads=1):
        """aggregate_non_interactive_multi_party_server_key_shares (evaluator.rs:1222-1622).
        shares: list (user id order) of dicts with ui_to_s_ksk, ksk_zero_encs, self_leader,
        not_leader, zero_encs, auto_keys [w+1][d_auto][N], lwe_ksk [lwe_d N].
        -> (ksk_b [users][50][N], rgsw [i1-i0][rows][N], auto [w+1][d_auto][N], lwe [lwe_d N])."""
        info = param_info(self.pid)
        i1 = self.n if i1 is None else i1
        users, N = len(shares), self.N
        keep = []

        def ptrs(key):
            arrs = [np.ascontiguousarray(sh[key], np.uint64) for sh in shares]
            keep.extend(arrs)
            return (u64p * users)(*[_p(a) for a in arrs])

        fields = [ptrs(k) for k in ("ui_to_s_ksk", "ksk_zero_encs", "self_leader", "not_leader", "zero_encs",
                                    "auto_keys", "lwe_ksk")]
        rows = 2 * info.rlrg_d_a + 2 * info.rlrg_d_b
        ksk = np.empty((users, self.NI_KS_D, N), np.uint64)
        rgsw = np.empty((max(i1 - i0, 1), rows, N), np.uint64)
        auto = np.empty((info.w + 1, info.auto_d, N), np.uint64)
        lwe = np.empty(info.lwe_d * N, np.uint64)
        cs = (ctypes.c_uint8 * 32)(*bytes(crs))
        if threads <= 1 or i1 - i0 < 2:
            lib().orc_ni_aggregate(self.h, cs, users, *fields, i0, i1, _p(ksk), _p(rgsw), _p(auto), _p(lwe))
            return ksk, rgsw[:i1 - i0], auto, lwe
        from concurrent.futures import ThreadPoolExecutor  # ctypes calls run without the GIL

        step = -(-(i1 - i0) // threads)
        parts = [(a, min(a + step, i1)) for a in range(i0, i1, step)]

        def run(ab):
            a, b = ab
            k2, a2, l2 = np.empty_like(ksk), np.empty_like(auto), np.empty_like(lwe)
            view = rgsw[a - i0:b - i0]
            lib().orc_ni_aggregate(self.h, cs, users, *fields, a, b, _p(k2), _p(view), _p(a2), _p(l2))
            return k2, a2, l2

        with ThreadPoolExecutor(len(parts)) as ex:
            res = list(ex.map(run, parts))
        ksk[:], auto[:], lwe[:] = res[0]
        return ksk, rgsw[:i1 - i0], auto, lwe

    def ni_ingest(self, ksk, seed, b, nbits):
        """unseed -> key switch -> extract every bool (the server's NI input path)."""
        rl = self.ni_unseed(seed, b)
        ks = [self.ni_key_switch(ksk, r) for r in rl]
        return np.stack([self.sample_extract(ks[i // self.N], i % self.N) for i in range(nbits)])


class OracleKey:
    def __init__(self, ev, coeff):
        self.ev = ev
        self.coeff = coeff
        self.h = lib().orc_key_new(ev.h, _p(np.ascontiguousarray(coeff.rgsw)),
                                   _p(np.ascontiguousarray(coeff.autos)),
                                   _p(np.ascontiguousarray(coeff.ksk)))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_key_free(self.h)
            self.h = None

    def rlwe_by_rgsw(self, rlwe, lwe_index, trivial=False, shoup=True):
        a = np.ascontiguousarray(rlwe, np.uint64).copy()
        lib().orc_rlwe_by_rgsw(self.ev.h, self.h, _p(a), lwe_index, int(trivial), int(shoup))
        return a

    def rlwe_auto(self, rlwe, k, trivial=False, shoup=True):
        a = np.ascontiguousarray(rlwe, np.uint64).copy()
        lib().orc_rlwe_auto(self.ev.h, self.h, _p(a), k, int(trivial), int(shoup))
        return a

    def lwe_key_switch(self, lwe_in):
        a = np.ascontiguousarray(lwe_in, np.uint64)
        out = np.empty(self.ev.n + 1, np.uint64)
        lib().orc_lwe_key_switch(self.ev.h, self.h, _p(a), _p(out))
        return out

    def pbs(self, gate, lwe):
        a = np.ascontiguousarray(lwe, np.uint64).copy()
        ks = np.empty(self.ev.n + 1, np.uint64)
        rl = np.empty(2 * self.ev.N, np.uint64)
        autos = lib().orc_pbs(self.ev.h, self.h, GATES[gate] if isinstance(gate, str) else gate,
                              _p(a), _p(ks), _p(rl))
        return a, ks, rl, autos

    def gate(self, gate, c0, c1):
        a = np.ascontiguousarray(c0, np.uint64).copy()
        b = np.ascontiguousarray(c1, np.uint64)
        lib().orc_gate(self.ev.h, self.h, GATES[gate] if isinstance(gate, str) else gate, _p(a), _p(b))
        return a

    U8_OPS = {"add": 0, "sub": 1, "mul": 2, "div_rem": 3, "eq": 4, "neq": 5, "lt": 6, "gt": 7,
              "le": 8, "ge": 9, "mux": 10, "overflowing_add": 11, "overflowing_sub": 12}

    def u8_op(self, op, a, b, sel=None, flag=None):
        """FheUint8 op, sequential gates.  Returns (out, out2, flag)."""
        L = self.ev.L
        a = np.ascontiguousarray(a, np.uint64).reshape(8, L)
        b = np.ascontiguousarray(b, np.uint64).reshape(8, L)
        code = self.U8_OPS[op]
        nout = 1 if code in (4, 5, 6, 7, 8, 9) else 8
        out = np.zeros((nout, L), np.uint64)
        out2 = np.zeros((8, L), np.uint64)
        fl = np.zeros(L, np.uint64) if flag is None else np.ascontiguousarray(flag, np.uint64).copy()
        fs = ctypes.c_int(0 if flag is None else 1)
        sp = _p(np.ascontiguousarray(sel, np.uint64)) if sel is not None else None
        rc = lib().orc_u8_op(self.ev.h, self.h, code, _p(a), _p(b), sp, _p(out), _p(out2), _p(fl),
                             ctypes.byref(fs))
        assert rc == 0
        return out, out2, (fl if fs.value else None)

    def gate_batch(self, gates, c0, c1, threads=1):
        gates = np.ascontiguousarray(gates, np.uint8)
        c0 = np.ascontiguousarray(c0, np.uint64)
        c1 = np.ascontiguousarray(c1, np.uint64)
        out = np.empty_like(c0)
        lib().orc_gate_batch(self.ev.h, self.h, _p(gates, u8p), _p(c0), _p(c1), _p(out),
                             len(gates), threads)
        return out


def setup(param, parties=2, seed_base=0, err_seed=b"\x33" * 32):
    """Evaluator + client keys + server key for a parameter set."""
    ev = Evaluator(param)
    s, z, sp, zp = ev.client_keys(parties, seed_base)
    coeff = ev.gen_server_key(s, z, err_seed)
    key = ev.key(coeff)
    return ev, (s, z, sp, zp), coeff, key
