"""Eager FheBool / FheUint8 values: the reference's operator front end
(bool/mod.rs:120-200 for FheBool, shortint/mod.rs:16-292 for FheUint8) over
the engine.

Each operator runs one cached circuit (circuits.Circuit, levelized: one
batched key switch + blind rotation launch per level) on the device with the
operands' ciphertexts already resident in HBM; values stay on the device
between operators and reach the host only through ``lwe()``.

State mirrors the reference:

* the server key is process-global and set once (``set_server_key``,
  bool/mp_api.rs:136-145 / 183-185: "Attempted to set server key twice.");
* the division-by-zero flag is thread-local (shortint/mod.rs:10-28): ``/``
  and ``div_rem`` OR ``is_zero(divisor)`` into it (shortint/mod.rs:42-56),
  ``%`` leaves it alone (shortint/mod.rs:123-137), ``reset_error_flags``
  clears it;
* circuits (and their device wire buffers) are cached per thread, like the
  reference's thread-local BoolEvaluator.

Ciphertexts are LWE vectors of N + 1 u64 words (a[0..N) then b, under the
ideal RLWE secret); an FheUint8 is 8 of them, LSB first
(shortint/enc_dec.rs:11-29).  Encryption and decryption are client-side and
not part of this server library.
"""
import threading

import numpy as np

from .circuits import Circuit
from .engine import GATES

_KEY = {}
_KEY_LOCK = threading.Lock()
_TLS = threading.local()


def set_server_key(engine, key):
    """Make (engine, key) the server key every operator uses.  A second call
    raises, as the reference's OnceLock does (bool/mp_api.rs:136-145)."""
    with _KEY_LOCK:
        if _KEY:
            raise RuntimeError("Attempted to set server key twice.")
        _KEY["engine"], _KEY["key"] = engine, key


def clear_server_key():
    """Drop the global server key (the reference has no such call: a process
    there sets its key once; this lets one process serve several key sets in
    turn).  Cached circuits of the old engine are dropped with it on their
    thread's next operator."""
    with _KEY_LOCK:
        _KEY.clear()


def _server():
    if not _KEY:
        raise RuntimeError("Server key not set!")  # bool/mp_api.rs:183-185
    return _KEY["engine"], _KEY["key"]


def div_zero_error_flag():
    """FheBool: whether a division since the last reset had divisor 0; None
    when no division ran (shortint/mod.rs:14-18)."""
    return getattr(_TLS, "div_zero", None)


def reset_error_flags():
    """Clear this thread's error flags (shortint/mod.rs:20-28)."""
    _TLS.div_zero = None


# -- cached circuits -------------------------------------------------------------------
def _build(name):
    """Circuit for one operator: (circuit, outputs as (kind, width) groups)."""
    C = Circuit()
    if name in GATES:
        a, b = C.input(), C.input()
        C.output(C.gate(name, a, b))
        return C
    a, b = C.input_u8(), C.input_u8()
    if name in ("add", "sub"):
        C.outputs(getattr(C, "u8_" + name)(a, b))
    elif name in ("overflowing_add", "overflowing_sub"):
        out, ov = getattr(C, "u8_" + name.split("_")[1])(a, b, overflow=True)
        C.outputs(out)
        C.output(ov)
    elif name == "mul":
        C.outputs(C.u8_mul(a, b))
    elif name in ("div", "div_or", "div_rem", "div_rem_or", "rem"):
        flag = C.input() if name.endswith("_or") else None
        q, r, f = C.u8_div_rem(a, b, flag=flag, track_flag=name != "rem")
        if name.startswith("div"):
            C.outputs(q)
        if name != "div" and name != "div_or":
            C.outputs(r)
        if name != "rem":
            C.output(f)
    elif name in ("eq", "neq", "lt", "gt", "le", "ge"):
        C.output(C.u8_cmp(name, a, b))
    elif name == "mux":
        C.outputs(C.u8_mux(a, b, C.input()))
    elif name in ("max", "min"):
        C.outputs(getattr(C, "u8_" + name)(a, b))
    else:
        raise KeyError(name)
    return C


def _circuit(engine, name):
    cache = getattr(_TLS, "circuits", None)
    if cache is None or cache[0] is not engine:
        cache = _TLS.circuits = (engine, {})
    c = cache[1].get(name)
    if c is None:
        c = cache[1][name] = _build(name)
    return c


def _run(name, *operands):
    """Run operator `name` on device operands ([k][L] int64 tensors, in input
    order); returns the [outputs][L] device tensor."""
    import torch
    engine, key = _server()
    c = _circuit(engine, name)
    inp = torch.cat([o.reshape(-1, engine.L) for o in operands])
    if inp.shape[0] != c.n_inputs:
        raise ValueError(f"{name}: {inp.shape[0]} input ciphertexts, circuit takes {c.n_inputs}")
    out = torch.empty((c.n_outputs, engine.L), dtype=torch.int64, device=inp.device)
    c.run_device(engine, key, inp, out)
    return out


def _device(ct, rows):
    """Host u64 array or device int64 tensor -> contiguous [rows][L] device tensor."""
    import torch
    engine, _ = _server()
    if isinstance(ct, torch.Tensor):
        t = ct.to(device=f"cuda:{engine.device}", dtype=torch.int64)
    else:
        a = np.ascontiguousarray(ct, np.uint64)
        t = torch.from_numpy(a.view(np.int64).copy()).to(f"cuda:{engine.device}")
    t = t.reshape(rows, -1).contiguous()
    if t.shape[1] != engine.L:
        raise ValueError(f"ciphertext length {t.shape[1]}, expected N + 1 = {engine.L}")
    return t


def _fold_div_zero(flag_now):
    """The thread's flag becomes flag_now (first division) -- the circuits
    with an ``_or`` suffix already OR'd the previous flag in."""
    _TLS.div_zero = FheBool._wrap(flag_now)


class FheBool:
    """Encrypted bit (bool/mod.rs:120-200: & | ^ and their assign forms, !)."""

    __slots__ = ("data",)

    def __init__(self, lwe):
        self.data = _device(lwe, 1)[0]

    @classmethod
    def _wrap(cls, t):
        v = cls.__new__(cls)
        v.data = t.reshape(-1)
        return v

    def lwe(self):
        """The ciphertext on the host: u64[N + 1]."""
        return self.data.cpu().numpy().view(np.uint64)

    def _gate(self, name, other):
        return FheBool._wrap(_run(name, self.data, other.data)[0])

    def __and__(self, other):
        return self._gate("and", other)

    def __or__(self, other):
        return self._gate("or", other)

    def __xor__(self, other):
        return self._gate("xor", other)

    def __iand__(self, other):
        self.data = _run("and", self.data, other.data)[0]
        return self

    def __ior__(self, other):
        self.data = _run("or", self.data, other.data)[0]
        return self

    def __ixor__(self, other):
        self.data = _run("xor", self.data, other.data)[0]
        return self

    def nand(self, other):
        return self._gate("nand", other)

    def nor(self, other):
        return self._gate("nor", other)

    def xnor(self, other):
        return self._gate("xnor", other)

    def __invert__(self):
        """NOT: negation mod Q, no bootstrap (evaluator.rs:2247-2250)."""
        import torch
        engine, _ = _server()
        out = torch.empty_like(self.data)
        engine.not_device(self.data, out)
        return FheBool._wrap(out)


class FheUint8:
    """Encrypted u8 as 8 FheBool, LSB first (shortint/mod.rs:63-292)."""

    __slots__ = ("data",)

    def __init__(self, lwes):
        """lwes: u64[8][N + 1] (host) or a [8][N + 1] device tensor."""
        self.data = _device(lwes, 8)

    @classmethod
    def from_bools(cls, bits):
        import torch
        if len(bits) != 8:
            raise ValueError("FheUint8 takes 8 FheBool, LSB first")
        return cls._wrap(torch.stack([b.data for b in bits]))

    @classmethod
    def _wrap(cls, t):
        v = cls.__new__(cls)
        v.data = t.reshape(8, -1)
        return v

    def bits(self):
        return [FheBool._wrap(self.data[i]) for i in range(8)]

    def lwe(self):
        """The ciphertexts on the host: u64[8][N + 1], LSB first."""
        return self.data.cpu().numpy().view(np.uint64)

    # -- arithmetic (shortint/mod.rs:63-205) ---------------------------------------------
    def __add__(self, other):
        return FheUint8._wrap(_run("add", self.data, other.data))

    def __iadd__(self, other):
        self.data = _run("add", self.data, other.data)
        return self

    def __sub__(self, other):
        return FheUint8._wrap(_run("sub", self.data, other.data))

    def __mul__(self, other):
        return FheUint8._wrap(_run("mul", self.data, other.data))

    def __floordiv__(self, other):
        """Quotient; sets the division-by-zero flag (shortint/mod.rs:103-121)."""
        prev = div_zero_error_flag()
        if prev is None:
            out = _run("div", self.data, other.data)
        else:
            out = _run("div_or", self.data, other.data, prev.data)
        _fold_div_zero(out[8])
        return FheUint8._wrap(out[:8])

    __truediv__ = __floordiv__  # Rust's `/` on integers

    def __mod__(self, other):
        """Remainder; the flag is not touched (shortint/mod.rs:123-137)."""
        return FheUint8._wrap(_run("rem", self.data, other.data))

    def div_rem(self, other):
        """(quotient, remainder); divisor 0 gives (255, self) and sets the
        flag (shortint/mod.rs:178-205)."""
        prev = div_zero_error_flag()
        if prev is None:
            out = _run("div_rem", self.data, other.data)
        else:
            out = _run("div_rem_or", self.data, other.data, prev.data)
        _fold_div_zero(out[16])
        return FheUint8._wrap(out[:8]), FheUint8._wrap(out[8:16])

    def overflowing_add(self, other):
        """(self + other, overflow) (shortint/mod.rs:152-164)."""
        out = _run("overflowing_add", self.data, other.data)
        return FheUint8._wrap(out[:8]), FheBool._wrap(out[8])

    def overflowing_add_assign(self, other):
        """self += other; returns overflow (shortint/mod.rs:139-150)."""
        out = _run("overflowing_add", self.data, other.data)
        self.data = out[:8]
        return FheBool._wrap(out[8])

    def overflowing_sub(self, other):
        """(self - other, overflow) (shortint/mod.rs:166-176)."""
        out = _run("overflowing_sub", self.data, other.data)
        return FheUint8._wrap(out[:8]), FheBool._wrap(out[8])

    # -- comparison and selection (shortint/mod.rs:207-292) -------------------------------
    def _cmp(self, op, other):
        return FheBool._wrap(_run(op, self.data, other.data)[0])

    def eq(self, other):
        return self._cmp("eq", other)

    def neq(self, other):
        return self._cmp("neq", other)

    def lt(self, other):
        return self._cmp("lt", other)

    def gt(self, other):
        return self._cmp("gt", other)

    def le(self, other):
        return self._cmp("le", other)

    def ge(self, other):
        return self._cmp("ge", other)

    def mux(self, other, selector):
        """selector ? self : other (shortint/mod.rs:272-279)."""
        return FheUint8._wrap(_run("mux", self.data, other.data, selector.data))

    def max(self, other):
        return FheUint8._wrap(_run("max", self.data, other.data))

    def min(self, other):
        return FheUint8._wrap(_run("min", self.data, other.data))
