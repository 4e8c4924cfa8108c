import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def pz():
    """The product package (directory name contains a hyphen)."""
    return importlib.import_module("phantom-zone_b200")


def oracle():
    from oracle import oracle as O
    return O


_SETUPS = {}

# parties each parameter set is designed for (SP_TEST_BOOL_PARAMS is single-party)
PARTIES = {"SP_TEST": 1, "I_2P_LB_SR": 2, "I_4P": 4, "I_8P": 8, "NI_2P": 2, "NI_4P_HB_FR": 4,
           "NI_4P_LB_SR": 4, "NI_8P": 8}


def oracle_setup(param, parties=None):
    """Oracle evaluator + client secrets + coefficient-domain server key (cached)."""
    parties = PARTIES[param] if parties is None else parties
    key = (param, parties)
    if key not in _SETUPS:
        O = oracle()
        ev, secrets, coeff, okey = O.setup(param, parties=parties)
        _SETUPS[key] = (ev, secrets, coeff, okey)
    return _SETUPS[key]


def to_dev(a):
    import torch
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        return torch.from_numpy(a.view(np.int64).copy()).cuda()
    if a.dtype == np.uint32:
        return torch.from_numpy(a.view(np.int32).copy()).cuda()
    return torch.from_numpy(a.copy()).cuda()


def to_host(t, dtype=np.uint64):
    return t.cpu().numpy().view(dtype)


def combine(ev, gate, c0, c1):
    """Gate prelude of evaluator.rs:2118-2133 in numpy (add/sub_mod_fast)."""
    Q = np.uint64(ev.Q)
    c0 = np.asarray(c0, np.uint64)
    c1 = np.asarray(c1, np.uint64)

    def red(x):  # x < 2Q -> [0, Q) without computing the negative branch
        x = np.array(x, np.uint64, copy=True)
        x[x >= Q] -= Q
        return x

    if gate in ("xor", "xnor", 4, 5):
        d = (Q + c0) - c1
        d = red(d)
        return red(d + d)
    s = red(c0 + c1)
    s[..., 0] = red(s[..., 0] + np.uint64(ev.Q >> 2))
    return s


@pytest.fixture
def gpu_available():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
