"""Python handle over the C ABI: one ``Engine`` per (parameter set, device).

Host-memory calls take and return numpy arrays; ``*_device`` calls take
torch CUDA tensors (any 8-byte integer dtype for u64 words) and run
asynchronously on the given stream (default: torch's current stream).
"""
import ctypes

import numpy as np

from ._lib import PzNiShareView, PzParams, PzServerKeyShareView, PzSeededServerKeyView, PzServerKeyView, check, lib, u8p, u64p, vp

PARAMETER_SETS = {
    "I_2P_LB_SR": 0, "I_4P": 1, "I_8P": 2, "NI_2P": 3,
    "NI_4P_HB_FR": 4, "NI_4P_LB_SR": 5, "NI_8P": 6, "SP_TEST": 7,
}
# ParameterSelector names of the reference (bool/mp_api.rs:28-32,
# bool/ni_mp_api.rs:39-47) -> parameter sets.
SELECTORS = {
    "InteractiveLTE2Party": "I_2P_LB_SR",
    "InteractiveLTE4Party": "I_4P",
    "InteractiveLTE8Party": "I_8P",
    "NonInteractiveLTE2Party": "NI_2P",
    "NonInteractiveLTE4Party": "NI_4P_HB_FR",
    "NonInteractiveLTE8Party": "NI_8P",
}
GATES = {"and": 0, "nand": 1, "or": 2, "nor": 3, "xor": 4, "xnor": 5}


def param_id(param):
    if isinstance(param, int):
        return param
    if param in SELECTORS:
        param = SELECTORS[param]
    return PARAMETER_SETS[param]


def params(param):
    p = PzParams()
    check(lib().pz_param_get(param_id(param), ctypes.byref(p)), None, "pz_param_get")
    return p


def probe_imad_rate(device=0):
    """32-bit IMAD instructions per second measured on `device`."""
    v = ctypes.c_double()
    check(lib().pz_probe_imad_rate(device, ctypes.byref(v)), None, "pz_probe_imad_rate")
    return v.value


PIPE_PROBES = ["imad", "imad_wide", "imad_hi", "dfma", "cvt_f64_u64", "cvt_u64_f64", "imad_with_dfma"]


def probe_pipe_rates(device=0):
    """Instructions per second of the pipes the butterflies use, by name."""
    arr = (ctypes.c_double * len(PIPE_PROBES))()
    check(lib().pz_probe_pipe_rates(device, arr, len(PIPE_PROBES)), None, "pz_probe_pipe_rates")
    return dict(zip(PIPE_PROBES, list(arr)))


def kernel_revision():
    """Revision tag of the blind-rotation kernel in the loaded library (a
    profile on record applies only to the revision it was taken on)."""
    return lib().pz_kernel_revision().decode()


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream(stream):
    if stream is None:
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, int):
        return ctypes.c_void_p(stream)
    return ctypes.c_void_p(stream.cuda_stream)


class DeviceKey:
    """A server key resident on the engine's device."""

    def __init__(self, engine, handle):
        self.engine = engine
        self.h = handle

    @property
    def device_bytes(self):
        return lib().pz_key_device_bytes(self.h)

    def export(self):
        """Device-form key as bytes (checkpoint / hand-over between processes)."""
        size = ctypes.c_size_t()
        check(lib().pz_key_export(self.h, None, 0, ctypes.byref(size)), self.engine.h, "pz_key_export")
        buf = ctypes.create_string_buffer(size.value)
        check(lib().pz_key_export(self.h, buf, size.value, ctypes.byref(size)), self.engine.h, "pz_key_export")
        return buf.raw

    def release(self):
        if self.h:
            lib().pz_key_release(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class NiKsk:
    """A user's ui_to_s key-switching key resident on the engine's device."""

    def __init__(self, engine, handle):
        self.engine = engine
        self.h = handle

    def release(self):
        if self.h:
            lib().pz_ni_ksk_release(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


CRS_AUTO_KEYS, CRS_LWE_KSK, CRS_UI_TO_S_KSK, CRS_NI_RGSW = 0, 1, 2, 3
NI_SHARE_FIELDS = ("ui_to_s_ksk", "ksk_zero_encs", "self_leader_cts", "not_leader_cts", "rgsw_zero_encs",
                   "auto_keys", "lwe_ksk")


def ni_crs_seed(crs, what, index=0):
    """NonInteractiveMultiPartyCrs seed (bool/evaluator.rs:115-172), host only."""
    out = (ctypes.c_uint8 * 32)()
    check(lib().pz_ni_crs_seed(_seed(crs), int(what), int(index), out), None, "pz_ni_crs_seed")
    return bytes(out)


ICRS_PUBLIC_KEY, ICRS_AUTO_KEYS, ICRS_LWE_KSK = 0, 1, 2
SHARE_FIELDS = ("self_leader_rgsws", "not_self_leader_rgsws", "auto_keys", "lwe_ksk")


def interactive_crs_seed(crs, what):
    """InteractiveMultiPartyCrs seed (bool/evaluator.rs:78-100), host only."""
    out = (ctypes.c_uint8 * 32)()
    check(lib().pz_interactive_crs_seed(_seed(crs), int(what), out), None, "pz_interactive_crs_seed")
    return bytes(out)


def _seed(seed):
    seed = bytes(seed)
    if len(seed) != 32:
        raise ValueError("seed must be 32 bytes")
    return (ctypes.c_uint8 * 32)(*seed)


class Engine:
    def __init__(self, param, device=0, ntt_root=0):
        self.param_id = param_id(param)
        h = vp()
        check(lib().pz_ctx_create_ex(self.param_id, device, int(ntt_root), ctypes.byref(h)), None,
              "pz_ctx_create")
        self.h = h
        self.device = device
        self.p = PzParams()
        check(lib().pz_ctx_params(self.h, ctypes.byref(self.p)), self.h, "pz_ctx_params")
        self.N, self.n, self.Q = self.p.rlwe_n, self.p.lwe_n, self.p.rlwe_q
        self.L = self.N + 1

    def close(self):
        if getattr(self, "h", None):
            lib().pz_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ntt_root(self):
        return lib().pz_ctx_ntt_root(self.h)

    def set_pbs_grid_limit(self, g):
        check(lib().pz_ctx_set_pbs_grid_limit(self.h, int(g)), self.h, "set_pbs_grid_limit")

    def set_split_threshold(self, max_gates):
        """Launches of at most max_gates gates use the two-CTA low-latency kernel (-1: default)."""
        check(lib().pz_ctx_set_split_threshold(self.h, int(max_gates)), self.h, "set_split_threshold")

    @property
    def pbs_variant(self):
        return lib().pz_ctx_pbs_variant(self.h)

    @pbs_variant.setter
    def pbs_variant(self, v):
        check(lib().pz_ctx_set_pbs_variant(self.h, int(v)), self.h, "set_pbs_variant")

    def device_error(self):
        """Error bits set by this context's kernels on the device (bounded waits
        that ran out); synchronizes the device and clears them."""
        v = ctypes.c_uint32()
        check(lib().pz_ctx_device_error(self.h, ctypes.byref(v)), self.h, "pz_ctx_device_error")
        return v.value

    def pbs_slots(self, variant=-1):
        """Ciphertexts a blind-rotation launch of shape `variant` (-1: the
        current one) holds resident at once; multiples run in whole waves."""
        n = ctypes.c_size_t()
        check(lib().pz_ctx_pbs_slots(self.h, int(variant), ctypes.byref(n)), self.h, "pz_ctx_pbs_slots")
        return n.value

    def autotune(self, key, batch=2368):
        """Pick the fastest blind-rotation variant and key-switch tile for
        this context on `batch` gates (cached for batches of that size bucket)."""
        v, ms = ctypes.c_int(), ctypes.c_double()
        check(lib().pz_ctx_autotune(self.h, key.h, int(batch), ctypes.byref(v), ctypes.byref(ms)), self.h,
              "pz_ctx_autotune")
        return {"variant": v.value, "ms": ms.value, "ks_tile": self.launch_shape(batch)["ks_tile"]}

    def set_ks_tile(self, ciphertexts):
        """Key-switch ciphertexts per CTA (8, 16, 32; 64 = the tensor-core form);
        clears the tuned choices."""
        check(lib().pz_ctx_set_ks_tile(self.h, int(ciphertexts)), self.h, "pz_ctx_set_ks_tile")

    def launch_shape(self, gates):
        """The blind-rotation variant and key-switch tile a batch of `gates` uses."""
        v, t = ctypes.c_int(), ctypes.c_int()
        check(lib().pz_ctx_launch_shape(self.h, int(gates), ctypes.byref(v), ctypes.byref(t)), self.h,
              "pz_ctx_launch_shape")
        return {"variant": v.value, "ks_tile": t.value}

    # -- keys --------------------------------------------------------------
    def upload_key(self, rgsw, autos, lwe_ksk):
        """Upload a coefficient-domain server key (layouts of pz_server_key_view)."""
        p = self.p
        rgsw = np.ascontiguousarray(rgsw, dtype=np.uint64)
        autos = np.ascontiguousarray(autos, dtype=np.uint64)
        lwe_ksk = np.ascontiguousarray(lwe_ksk, dtype=np.uint64)
        if rgsw.size != p.lwe_n * p.rgsw_rows * p.rlwe_n:
            raise ValueError("rgsw has the wrong size for this parameter set")
        if autos.size != p.n_auto_keys * p.auto_rows * p.rlwe_n:
            raise ValueError("auto keys have the wrong size for this parameter set")
        if lwe_ksk.size != p.lwe_d * p.rlwe_n * (p.lwe_n + 1):
            raise ValueError("lwe ksk has the wrong size for this parameter set")
        view = PzServerKeyView(rgsw.ctypes.data_as(u64p), autos.ctypes.data_as(u64p),
                               lwe_ksk.ctypes.data_as(u64p))
        h = vp()
        check(lib().pz_key_upload(self.h, ctypes.byref(view), ctypes.byref(h)), self.h, "pz_key_upload")
        return DeviceKey(self, h)

    def import_key(self, blob):
        """A key exported by DeviceKey.export() under the same parameter set and NTT root."""
        blob = bytes(blob)
        h = vp()
        check(lib().pz_key_import(self.h, blob, len(blob), ctypes.byref(h)), self.h, "pz_key_import")
        return DeviceKey(self, h)

    def upload_key_seeded(self, rgsw, auto_b, auto_seed, lwe_ksk_b, lwe_ksk_seed):
        """Upload a seeded server key: RGSW in full, auto-key B rows [w+1][d_auto][N]
        and LWE-KSK column 0 [d_ks N]; the A parts are regenerated on the device
        from the two CRS-derived seeds (keys.rs:687-781)."""
        p = self.p
        rgsw = np.ascontiguousarray(rgsw, dtype=np.uint64)
        auto_b = np.ascontiguousarray(auto_b, dtype=np.uint64)
        lwe_ksk_b = np.ascontiguousarray(lwe_ksk_b, dtype=np.uint64)
        if rgsw.size != p.lwe_n * p.rgsw_rows * p.rlwe_n:
            raise ValueError("rgsw has the wrong size for this parameter set")
        if auto_b.size != p.n_auto_keys * p.auto_d * p.rlwe_n:
            raise ValueError("auto B rows have the wrong size for this parameter set")
        if lwe_ksk_b.size != p.lwe_d * p.rlwe_n:
            raise ValueError("lwe ksk column has the wrong size for this parameter set")
        v = PzSeededServerKeyView(rgsw.ctypes.data_as(u64p), auto_b.ctypes.data_as(u64p),
                                  lwe_ksk_b.ctypes.data_as(u64p), _seed(auto_seed), _seed(lwe_ksk_seed))
        h = vp()
        check(lib().pz_key_upload_seeded(self.h, ctypes.byref(v), ctypes.byref(h)), self.h, "pz_key_upload_seeded")
        return DeviceKey(self, h)

    def upload_ni_ksk_seeded(self, ksk_b, seed):
        ksk_b = np.ascontiguousarray(ksk_b, dtype=np.uint64)
        if ksk_b.size != self.p.ni_ks_d * self.N or self.p.ni_ks_d == 0:
            raise ValueError("ui_to_s B rows have the wrong size (or the set is not non-interactive)")
        h = vp()
        check(lib().pz_ni_ksk_upload_seeded(self.h, ksk_b.ctypes.data_as(u64p), _seed(seed), ctypes.byref(h)), self.h,
              "pz_ni_ksk_upload_seeded")
        return NiKsk(self, h)

    # -- gates, host memory --------------------------------------------------
    def gate_batch(self, key, gates, c0, c1):
        gates = np.ascontiguousarray(gates, dtype=np.uint8)
        c0 = np.ascontiguousarray(c0, dtype=np.uint64).reshape(-1, self.L)
        c1 = np.ascontiguousarray(c1, dtype=np.uint64).reshape(-1, self.L)
        if not (len(gates) == len(c0) == len(c1)):
            raise ValueError("gates, c0 and c1 must have the same count")
        out = np.empty_like(c0)
        check(lib().pz_gate_batch(self.h, key.h, gates.ctypes.data_as(u8p), c0.ctypes.data_as(u64p),
                                  c1.ctypes.data_as(u64p), out.ctypes.data_as(u64p), len(gates)),
              self.h, "pz_gate_batch")
        return out

    # -- device memory ---------------------------------------------------------
    def gate_batch_device(self, key, gates, c0, c1, out, stream=None, ks_out=None, rlwe_out=None):
        count = gates.numel()
        if ks_out is None and rlwe_out is None:
            check(lib().pz_gate_batch_device(self.h, key.h, _ptr(gates), _ptr(c0), _ptr(c1), _ptr(out),
                                             count, _stream(stream)), self.h, "pz_gate_batch_device")
        else:
            check(lib().pz_gate_batch_debug_device(self.h, key.h, _ptr(gates), _ptr(c0), _ptr(c1),
                                                   _ptr(out), count, _ptr(ks_out), _ptr(rlwe_out),
                                                   _stream(stream)), self.h, "pz_gate_batch_debug_device")

    def gate_batch_device_noalloc(self, key, gates, c0, c1, out, stream=None):
        """gate_batch_device without any device allocation (fixed in-library
        scratch; bounded batch size; concurrent calls must not overlap)."""
        check(lib().pz_gate_batch_device_noalloc(self.h, key.h, _ptr(gates), _ptr(c0), _ptr(c1), _ptr(out),
                                                 gates.numel(), _stream(stream)), self.h,
              "pz_gate_batch_device_noalloc")

    def pbs_batch_device(self, key, test_vec, lwe, out, stream=None):
        check(lib().pz_pbs_batch_device(self.h, key.h, _ptr(test_vec), _ptr(lwe), _ptr(out),
                                        test_vec.numel(), _stream(stream)), self.h, "pz_pbs_batch_device")

    def blind_rotate_device(self, key, ks, test_vec, out, stream=None):
        check(lib().pz_blind_rotate_batch_device(self.h, key.h, _ptr(ks), _ptr(test_vec), _ptr(out),
                                                 test_vec.numel(), _stream(stream)), self.h,
              "pz_blind_rotate_batch_device")

    def not_device(self, x, out, stream=None):
        check(lib().pz_not_batch_device(self.h, _ptr(x), _ptr(out), x.numel(), _stream(stream)),
              self.h, "pz_not_batch_device")

    def ntt_forward_device(self, polys, stream=None):
        check(lib().pz_ntt_forward_device(self.h, _ptr(polys), polys.numel() // self.N, _stream(stream)),
              self.h, "pz_ntt_forward_device")

    def ntt_backward_device(self, polys, stream=None):
        check(lib().pz_ntt_backward_device(self.h, _ptr(polys), polys.numel() // self.N, _stream(stream)),
              self.h, "pz_ntt_backward_device")

    def rlwe_by_rgsw_device(self, key, rlwe, lwe_index, trivial=False, stream=None):
        check(lib().pz_rlwe_by_rgsw_device(self.h, key.h, _ptr(rlwe), _ptr(lwe_index), lwe_index.numel(),
                                           int(trivial), _stream(stream)), self.h, "pz_rlwe_by_rgsw_device")

    def rlwe_auto_device(self, key, rlwe, slot, trivial=False, stream=None):
        check(lib().pz_rlwe_auto_device(self.h, key.h, _ptr(rlwe), _ptr(slot), slot.numel(), int(trivial),
                                        _stream(stream)), self.h, "pz_rlwe_auto_device")

    # -- non-interactive input path ---------------------------------------------
    def upload_ni_ksk(self, ksk):
        """ui_to_s key of one user: [2 * ni_ks_d][N] coefficient domain (rows A then B)."""
        ksk = np.ascontiguousarray(ksk, dtype=np.uint64)
        if ksk.size != 2 * self.p.ni_ks_d * self.N or self.p.ni_ks_d == 0:
            raise ValueError("ui_to_s key has the wrong size (or the set is not non-interactive)")
        h = vp()
        check(lib().pz_ni_ksk_upload(self.h, ksk.ctypes.data_as(u64p), ctypes.byref(h)), self.h, "pz_ni_ksk_upload")
        return NiKsk(self, h)

    def ni_unseed_device(self, seed, d_b, d_rlwe, stream=None):
        check(lib().pz_ni_unseed_device(self.h, _seed(seed), _ptr(d_b), _ptr(d_rlwe), d_b.numel() // self.N,
                                        _stream(stream)), self.h, "pz_ni_unseed_device")

    def ni_key_switch_device(self, ksk, d_in, d_out, stream=None):
        check(lib().pz_ni_key_switch_device(self.h, ksk.h, _ptr(d_in), _ptr(d_out), d_in.numel() // (2 * self.N),
                                            _stream(stream)), self.h, "pz_ni_key_switch_device")

    def sample_extract_device(self, d_rlwe, d_index, d_lwe, stream=None):
        check(lib().pz_sample_extract_device(self.h, _ptr(d_rlwe), d_rlwe.numel() // (2 * self.N), _ptr(d_index),
                                             _ptr(d_lwe), d_index.numel(), _stream(stream)), self.h,
              "pz_sample_extract_device")

    def ni_ingest(self, ksk, seed, b, nbools):
        """Host buffers: seeded RLWE b-parts [count][N] -> LWEs [nbools][N+1] under s."""
        b = np.ascontiguousarray(b, dtype=np.uint64).reshape(-1, self.N)
        out = np.zeros((nbools, self.L), np.uint64)
        check(lib().pz_ni_ingest(self.h, ksk.h, _seed(seed), b.ctypes.data_as(u64p), len(b),
                                 out.ctypes.data_as(u64p), nbools), self.h, "pz_ni_ingest")
        return out

    # -- server-key aggregation ----------------------------------------------------
    def rgsw_by_rgsw_device(self, rgsw0, rgsw1, stream=None):
        """rgsw0 [count][4][N] <- rgsw0 x rgsw1 (rgsw1 [count][2 rgrg_d_a + 2 rgrg_d_b][N]), both coefficient domain."""
        count = rgsw0.numel() // (4 * self.N)
        check(lib().pz_rgsw_by_rgsw_device(self.h, _ptr(rgsw0), _ptr(rgsw1), count, _stream(stream)), self.h,
              "pz_rgsw_by_rgsw_device")

    def aggregate_rgsw_device(self, rgsw0, others, stream=None):
        """rgsw0[c] <- rgsw0[c] x others[0][c] x ... (others [steps][count][rows][N])."""
        count = rgsw0.numel() // (4 * self.N)
        steps = others.numel() // (count * 2 * (self.p.rgrg_d_a + self.p.rgrg_d_b) * self.N) if count else 0
        check(lib().pz_aggregate_rgsw_device(self.h, _ptr(rgsw0), _ptr(others), steps, count, _stream(stream)),
              self.h, "pz_aggregate_rgsw_device")

    def _share_views(self, shares):
        """shares: list (user id order) of dicts SHARE_FIELDS -> device tensors (u64 as int64)."""
        views = (PzServerKeyShareView * len(shares))()
        for v, sh in zip(views, shares):
            for f in SHARE_FIELDS:
                t = sh.get(f)
                setattr(v, f, t.data_ptr() if t is not None and t.numel() else None)
        return views

    def aggregate_device(self, shares, rgsw, auto_b, lwe_b, stream=None):
        """aggregate_interactive_multi_party_server_key_shares (bool/evaluator.rs:1050-1200) on
        device shares; outputs (device tensors) in the seeded server key's coefficient form."""
        check(lib().pz_aggregate_device(self.h, self._share_views(shares), len(shares), _ptr(rgsw), _ptr(auto_b),
                                        _ptr(lwe_b), _stream(stream)), self.h, "pz_aggregate_device")

    def aggregate_server_key(self, crs, shares):
        """Aggregation + seeded expansion -> DeviceKey; shares on the device."""
        kh = vp()
        check(lib().pz_aggregate_server_key(self.h, _seed(crs), self._share_views(shares), len(shares),
                                            ctypes.byref(kh)), self.h, "pz_aggregate_server_key")
        return DeviceKey(self, kh)

    def _ni_share_views(self, shares):
        """shares: list (user id order) of dicts NI_SHARE_FIELDS -> device tensors (u64 as int64)."""
        views = (PzNiShareView * len(shares))()
        for v, sh in zip(views, shares):
            for f in NI_SHARE_FIELDS:
                t = sh.get(f)
                setattr(v, f, t.data_ptr() if t is not None and t.numel() else None)
        return views

    def ni_aggregate_device(self, crs, shares, ksk_b, rgsw, auto_b, lwe_b, stream=None):
        """aggregate_non_interactive_multi_party_server_key_shares (bool/evaluator.rs:1222-1622)
        on device shares; outputs (device tensors) in the seeded server key's coefficient form."""
        views = self._ni_share_views(shares)
        check(lib().pz_ni_aggregate_device(self.h, _seed(crs), views, len(shares), _ptr(ksk_b), _ptr(rgsw),
                                           _ptr(auto_b), _ptr(lwe_b), _stream(stream)), self.h,
              "pz_ni_aggregate_device")

    def ni_aggregate_server_key(self, crs, shares):
        """Aggregation + expansion: -> (DeviceKey, [NiKsk per user]); shares on the device."""
        views = self._ni_share_views(shares)
        kh = vp()
        ks = (vp * len(shares))()
        check(lib().pz_ni_aggregate_server_key(self.h, _seed(crs), views, len(shares), ctypes.byref(kh), ks),
              self.h, "pz_ni_aggregate_server_key")
        return DeviceKey(self, kh), [NiKsk(self, vp(h)) for h in ks]

    def lwe_key_switch_device(self, key, lwe_in, out, stream=None):
        count = lwe_in.numel() // self.L
        check(lib().pz_lwe_key_switch_device(self.h, key.h, _ptr(lwe_in), _ptr(out), count,
                                             _stream(stream)), self.h, "pz_lwe_key_switch_device")
