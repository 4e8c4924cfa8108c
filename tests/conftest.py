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


def oracle_setup(param, parties=2):
    """Oracle evaluator + client secrets + coefficient-domain server key (cached)."""
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
    if gate in ("xor", "xnor", 4, 5):
        d = np.where(c0 >= c1, c0 - c1, (Q + c0) - c1)
        s = d + d
        return np.where(s >= Q, s - Q, s)
    s = c0 + c1
    s = np.where(s >= Q, s - Q, s)
    s = s.copy()
    b = s[..., 0] + np.uint64(ev.Q >> 2)
    s[..., 0] = np.where(b >= Q, b - Q, b)
    return s


@pytest.fixture
def gpu_available():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True
