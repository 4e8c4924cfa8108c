"""phantom-zone_b200: B200-native server-side gate bootstrap for phantom-zone.

The hot path (LWE key switch -> automorphism-based blind rotation -> sample
extraction) runs in hand-written CUDA kernels for sm_100a behind the C ABI
declared in include/phantom_zone_b200.h; this package is the Python host side
(ctypes) mirroring the reference's BoolEvaluator / BooleanGates / FheUint8
interface.  Import it with ``importlib.import_module("phantom-zone_b200")``.
"""
from . import _lib
from .engine import (GATES, PARAMETER_SETS, SELECTORS, DeviceKey, Engine, kernel_revision, param_id, params,
                     probe_imad_rate, probe_pipe_rates)
from .circuits import Circuit
from .server import DRY_RUN, Server
from .fhe import (FheBool, FheUint8, clear_server_key, div_zero_error_flag, reset_error_flags,
                  set_server_key)

__all__ = ["FheBool", "FheUint8", "set_server_key", "clear_server_key", "div_zero_error_flag",
           "reset_error_flags", "Circuit", "Server", "DRY_RUN", "Engine", "DeviceKey", "GATES", "PARAMETER_SETS", "SELECTORS", "kernel_revision", "param_id", "params",
           "probe_imad_rate", "probe_pipe_rates", "_lib"]
