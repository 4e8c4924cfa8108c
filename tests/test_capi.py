"""C ABI library: loads and exports every symbol include/*.h declares (no GPU calls)."""
import ctypes
import glob
import os
import re

from conftest import ROOT, pz


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(pz_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ["pz_ctx_create", "pz_key_upload", "pz_gate_batch", "pz_gate_batch_device",
                 "pz_ntt_forward_device", "pz_rlwe_by_rgsw_device", "pz_rlwe_auto_device",
                 "pz_lwe_key_switch_device", "pz_last_error"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(pz()._lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header():
    bound = set(pz()._lib.SIGNATURES)
    assert set(declared_functions()) <= bound


def test_param_table_matches_oracle():
    """The product's parameter table equals the oracle's (parameters.rs:526-726)."""
    from oracle import oracle as O
    P = pz()
    for name, pid in P.PARAMETER_SETS.items():
        a = P.params(pid)
        b = O.param_info(pid)
        for f, _ in a._fields_:
            assert getattr(a, f) == getattr(b, f), (name, f)


def test_invalid_arguments_rejected_without_gpu():
    L = pz()._lib.lib()
    h = ctypes.c_void_p()
    assert L.pz_ctx_create(99, 0, ctypes.byref(h)) == 1  # PZ_ERR_INVALID_ARGUMENT
    assert L.pz_param_get(-1, None) == 1
    assert L.pz_status_string(0) == b"ok"
    # NULL context / seed / share arguments are refused before any device work
    assert L.pz_ni_aggregate_device(None, None, None, 0, None, None, None, None, None) == 1
    assert L.pz_ni_aggregate_server_key(None, None, None, 0, None, None) == 1
    out = (ctypes.c_uint8 * 32)()
    assert L.pz_ni_crs_seed(None, 0, 0, out) == 1
    assert L.pz_ni_crs_seed((ctypes.c_uint8 * 32)(), 4, 0, out) == 1  # unknown seed kind
    assert L.pz_aggregate_device(None, None, 0, None, None, None, None) == 1
    assert L.pz_aggregate_server_key(None, None, None, 0, None) == 1
    assert L.pz_interactive_crs_seed((ctypes.c_uint8 * 32)(), 3, out) == 1


def test_ni_crs_seeds_host_matches_oracle():
    """pz_ni_crs_seed (host code, block-indexed ChaCha8) == the oracle's
    sequential puncturing (evaluator.rs:115-172), every kind of seed."""
    from conftest import oracle
    O = oracle()
    eng = pz().engine
    crs = bytes(range(3, 35))
    for what, idx in [(0, 0), (1, 0), (2, 0), (2, 7), (3, 0), (3, 1), (3, 659)]:
        assert eng.ni_crs_seed(crs, what, idx) == O.ni_crs_seed(crs, what, idx)


def test_interactive_crs_seeds_host_matches_oracle():
    """pz_interactive_crs_seed == the oracle's InteractiveMultiPartyCrs (evaluator.rs:78-100)."""
    from conftest import oracle
    O = oracle()
    crs = bytes(range(5, 37))
    for what in range(3):
        assert pz().engine.interactive_crs_seed(crs, what) == O.interactive_crs_seed(crs, what)
