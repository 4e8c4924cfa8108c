"""ctypes binding of the C ABI in include/phantom_zone_b200.h.

The engine is the CUDA library ``libpz_b200.so`` built in this package
directory (``make -C phantom-zone_b200``).  There is no CPU fallback: if the
library is missing or a call fails, an exception is raised.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpz_b200.so")

u64p = ctypes.POINTER(ctypes.c_uint64)
u32p = ctypes.POINTER(ctypes.c_uint32)
u8p = ctypes.POINTER(ctypes.c_uint8)
vp = ctypes.c_void_p
st = ctypes.c_int


class PzParams(ctypes.Structure):
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


class PzServerKeyView(ctypes.Structure):
    _fields_ = [("rgsw", u64p), ("autos", u64p), ("lwe_ksk", u64p)]


class PzSeededServerKeyView(ctypes.Structure):
    _fields_ = [("rgsw", u64p), ("auto_b", u64p), ("lwe_ksk_b", u64p),
                ("auto_seed", ctypes.c_uint8 * 32), ("lwe_ksk_seed", ctypes.c_uint8 * 32)]


class PzNiShareView(ctypes.Structure):
    _fields_ = [(n, vp) for n in ("ui_to_s_ksk", "ksk_zero_encs", "self_leader_cts", "not_leader_cts",
                                  "rgsw_zero_encs", "auto_keys", "lwe_ksk")]


class PzServerKeyShareView(ctypes.Structure):
    _fields_ = [(n, vp) for n in ("self_leader_rgsws", "not_self_leader_rgsws", "auto_keys", "lwe_ksk")]


class PzServerStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_size_t) for n in ("pending", "active", "done", "failed", "arena_slots",
                                                "arena_slots_used", "arena_bytes", "sessions", "key_bytes")] + \
               [(n, ctypes.c_uint64) for n in ("steps", "gates", "launches")] + \
               [(n, ctypes.c_size_t) for n in ("resident_key_bytes", "key_budget")] + \
               [(n, ctypes.c_uint64) for n in ("key_imports", "key_evictions")]


# name -> (restype, argtypes); every symbol declared in the public header
SIGNATURES = {
    "pz_status_string": (ctypes.c_char_p, [st]),
    "pz_param_get": (st, [ctypes.c_int, ctypes.POINTER(PzParams)]),
    "pz_ctx_create": (st, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]),
    "pz_ctx_create_ex": (st, [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(vp)]),
    "pz_ctx_destroy": (None, [vp]),
    "pz_last_error": (ctypes.c_char_p, [vp]),
    "pz_ctx_params": (st, [vp, ctypes.POINTER(PzParams)]),
    "pz_ctx_ntt_root": (ctypes.c_uint64, [vp]),
    "pz_key_upload": (st, [vp, ctypes.POINTER(PzServerKeyView), ctypes.POINTER(vp)]),
    "pz_key_release": (None, [vp]),
    "pz_key_device_bytes": (ctypes.c_size_t, [vp]),
    "pz_gate_batch": (st, [vp, vp, u8p, u64p, u64p, u64p, ctypes.c_size_t]),
    "pz_gate_batch_device": (st, [vp, vp, vp, vp, vp, vp, ctypes.c_size_t, vp]),
    "pz_gate_batch_device_noalloc": (st, [vp, vp, vp, vp, vp, vp, ctypes.c_size_t, vp]),
    "pz_gate_batch_debug_device": (st, [vp, vp, vp, vp, vp, vp, ctypes.c_size_t, vp, vp, vp]),
    "pz_pbs_batch_device": (st, [vp, vp, vp, vp, vp, ctypes.c_size_t, vp]),
    "pz_not_batch_device": (st, [vp, vp, vp, ctypes.c_size_t, vp]),
    "pz_blind_rotate_batch_device": (st, [vp, vp, vp, vp, vp, ctypes.c_size_t, vp]),
    "pz_probe_imad_rate": (st, [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "pz_probe_pipe_rates": (st, [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_size_t]),
    "pz_ntt_forward_device": (st, [vp, vp, ctypes.c_size_t, vp]),
    "pz_ntt_backward_device": (st, [vp, vp, ctypes.c_size_t, vp]),
    "pz_rlwe_by_rgsw_device": (st, [vp, vp, vp, vp, ctypes.c_size_t, ctypes.c_int, vp]),
    "pz_rlwe_auto_device": (st, [vp, vp, vp, vp, ctypes.c_size_t, ctypes.c_int, vp]),
    "pz_lwe_key_switch_device": (st, [vp, vp, vp, vp, ctypes.c_size_t, vp]),
    "pz_ctx_set_pbs_grid_limit": (st, [vp, ctypes.c_int]),
    "pz_ctx_set_pbs_variant": (st, [vp, ctypes.c_int]),
    "pz_ctx_pbs_variant": (ctypes.c_int, [vp]),
    "pz_ctx_pbs_slots": (st, [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]),
    "pz_kernel_revision": (ctypes.c_char_p, []),
    "pz_ctx_set_ks_tile": (st, [vp, ctypes.c_int]),
    "pz_ctx_launch_shape": (st, [vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "pz_ctx_device_error": (st, [vp, ctypes.POINTER(ctypes.c_uint32)]),
    "pz_chacha_block": (st, [ctypes.POINTER(ctypes.c_uint32), ctypes.c_int, ctypes.POINTER(ctypes.c_uint32)]),
    "pz_uniform_mod_word": (st, [ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64),
                                 ctypes.POINTER(ctypes.c_int)]),
    "pz_ni_ksk_upload": (st, [vp, u64p, ctypes.POINTER(vp)]),
    "pz_ni_ksk_release": (None, [vp]),
    "pz_ni_ksk_upload_seeded": (st, [vp, u64p, u8p, ctypes.POINTER(vp)]),
    "pz_key_upload_seeded": (st, [vp, ctypes.POINTER(PzSeededServerKeyView), ctypes.POINTER(vp)]),
    "pz_ni_unseed_device": (st, [vp, u8p, vp, vp, ctypes.c_size_t, vp]),
    "pz_ni_key_switch_device": (st, [vp, vp, vp, vp, ctypes.c_size_t, vp]),
    "pz_sample_extract_device": (st, [vp, vp, ctypes.c_size_t, vp, vp, ctypes.c_size_t, vp]),
    "pz_ni_ingest": (st, [vp, vp, u8p, u64p, ctypes.c_size_t, u64p, ctypes.c_size_t]),
    "pz_rgsw_by_rgsw_device": (st, [vp, vp, vp, ctypes.c_size_t, vp]),
    "pz_aggregate_rgsw_device": (st, [vp, vp, vp, ctypes.c_size_t, ctypes.c_size_t, vp]),
    "pz_server_set_schedule": (st, [vp, ctypes.c_int]),
    "pz_interactive_crs_seed": (st, [u8p, ctypes.c_int, u8p]),
    "pz_aggregate_device": (st, [vp, ctypes.POINTER(PzServerKeyShareView), ctypes.c_size_t, vp, vp, vp, vp]),
    "pz_aggregate_server_key": (st, [vp, u8p, ctypes.POINTER(PzServerKeyShareView), ctypes.c_size_t,
                                     ctypes.POINTER(vp)]),
    "pz_ni_crs_seed": (st, [u8p, ctypes.c_int, ctypes.c_size_t, u8p]),
    "pz_ni_aggregate_device": (st, [vp, u8p, ctypes.POINTER(PzNiShareView), ctypes.c_size_t, vp, vp, vp, vp, vp]),
    "pz_ni_aggregate_server_key": (st, [vp, u8p, ctypes.POINTER(PzNiShareView), ctypes.c_size_t,
                                        ctypes.POINTER(vp), ctypes.POINTER(vp)]),
    "pz_ctx_autotune": (st, [vp, vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]),
    "pz_ctx_set_split_threshold": (st, [vp, ctypes.c_int]),
    "pz_key_export": (st, [vp, vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "pz_key_import": (st, [vp, vp, ctypes.c_size_t, ctypes.POINTER(vp)]),
    "pz_circuit_serialize": (st, [vp, vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "pz_circuit_deserialize": (st, [vp, ctypes.c_size_t, ctypes.POINTER(vp)]),
    "pz_server_create": (st, [ctypes.c_int, ctypes.c_size_t, ctypes.c_size_t, ctypes.POINTER(vp)]),
    "pz_server_destroy": (None, [vp]),
    "pz_server_last_error": (ctypes.c_char_p, [vp]),
    "pz_server_add_session": (st, [vp, vp, vp, u32p]),
    "pz_server_add_virtual_session": (st, [vp, ctypes.c_int, u32p]),
    "pz_server_add_managed_session": (st, [vp, vp, ctypes.c_void_p, ctypes.c_size_t, u32p]),
    "pz_server_add_virtual_managed_session": (st, [vp, ctypes.c_int, u32p]),
    "pz_server_set_key_budget": (st, [vp, ctypes.c_size_t]),
    "pz_server_session_resident": (st, [vp, ctypes.c_uint32, ctypes.POINTER(ctypes.c_int)]),
    "pz_server_submit": (st, [vp, ctypes.c_uint32, vp, vp, vp, ctypes.c_int, u64p]),
    "pz_server_step": (st, [vp, ctypes.POINTER(ctypes.c_size_t)]),
    "pz_server_job_status": (st, [vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "pz_server_forget": (st, [vp, ctypes.c_uint64]),
    "pz_server_stats_get": (st, [vp, ctypes.POINTER(PzServerStats)]),
    "pz_server_set_launch": (st, [vp, ctypes.c_int, ctypes.c_int]),
    "pz_server_autotune": (st, [vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                ctypes.POINTER(ctypes.c_double)]),
    "pz_circuit_create": (st, [ctypes.POINTER(vp)]),
    "pz_circuit_destroy": (None, [vp]),
    "pz_circuit_last_error": (ctypes.c_char_p, [vp]),
    "pz_circuit_input": (ctypes.c_uint32, [vp]),
    "pz_circuit_gate": (ctypes.c_uint32, [vp, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32]),
    "pz_circuit_not": (ctypes.c_uint32, [vp, ctypes.c_uint32]),
    "pz_circuit_output": (st, [vp, ctypes.c_uint32]),
    "pz_circuit_info": (st, [vp] + [ctypes.POINTER(ctypes.c_size_t)] * 5),
    "pz_circuit_level_sizes": (st, [vp, ctypes.POINTER(ctypes.c_size_t), ctypes.c_size_t]),
    "pz_u8_add": (st, [vp, u32p, u32p, u32p, u32p]),
    "pz_u8_sub": (st, [vp, u32p, u32p, u32p, u32p]),
    "pz_u8_mul": (st, [vp, u32p, u32p, u32p]),
    "pz_u8_div_rem": (st, [vp, u32p, u32p, u32p, u32p, u32p]),
    "pz_u8_cmp": (st, [vp, ctypes.c_int, u32p, u32p, u32p]),
    "pz_u8_mux": (st, [vp, u32p, u32p, ctypes.c_uint32, u32p]),
    "pz_circuit_run_device": (st, [vp, vp, vp, vp, vp, vp]),
    "pz_circuit_run": (st, [vp, vp, vp, u64p, u64p]),
    "pz_circuit_capture_graph": (st, [vp, vp, vp, vp, vp, vp]),
    "pz_circuit_replay_graph": (st, [vp, vp]),
}

_lib = None


def lib():
    """Load libpz_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"CUDA engine not built: {LIB_PATH} is missing (run `make -C phantom-zone_b200`)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class PzError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{msg} (status {status})")
        self.status = status


def check(status, ctx=None, what=""):
    if status != 0:
        L = lib()
        detail = L.pz_last_error(ctx).decode() if ctx else L.pz_status_string(status).decode()
        raise PzError(status, f"{what}: {L.pz_status_string(status).decode()}: {detail}")
