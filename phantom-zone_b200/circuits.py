"""Circuit builder over the C ABI: FheUint8 operations recorded as gate DAGs
and executed level by level (one batched launch per level).

Wires are integer handles; an FheUint8 is a list of 8 wires, LSB first
(shortint/enc_dec.rs:11-29).  Operators follow shortint/mod.rs:63-292.
"""
import ctypes

import numpy as np

from ._lib import check, lib, u32p, u64p, vp
from .engine import GATES, _ptr, _stream

WIRE_NONE = 0xFFFFFFFF
CMP_OPS = {"eq": 0, "neq": 1, "lt": 2, "gt": 3, "le": 4, "ge": 5}


def _arr(ws):
    a = (ctypes.c_uint32 * len(ws))(*ws)
    return a


class Circuit:
    def __init__(self):
        h = vp()
        check(lib().pz_circuit_create(ctypes.byref(h)), None, "pz_circuit_create")
        self.h = h
        self.n_inputs = 0
        self.n_outputs = 0

    def close(self):
        if getattr(self, "h", None):
            lib().pz_circuit_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _err(self, what):
        raise RuntimeError(f"{what}: {lib().pz_circuit_last_error(self.h).decode()}")

    def _chk(self, status, what):
        if status != 0:
            self._err(what)

    # -- wires -----------------------------------------------------------------
    def input(self):
        self.n_inputs += 1
        return lib().pz_circuit_input(self.h)

    def input_u8(self):
        return [self.input() for _ in range(8)]

    def gate(self, name, a, b):
        w = lib().pz_circuit_gate(self.h, GATES[name], a, b)
        if w == WIRE_NONE:
            self._err("gate")
        return w

    def not_(self, a):
        return lib().pz_circuit_not(self.h, a)

    def output(self, w):
        self._chk(lib().pz_circuit_output(self.h, w), "output")
        self.n_outputs += 1

    def outputs(self, ws):
        for w in ws:
            self.output(w)

    # -- FheUint8 operators ------------------------------------------------------
    def u8_add(self, a, b, overflow=False):
        out = (ctypes.c_uint32 * 8)()
        ov = ctypes.c_uint32(WIRE_NONE)
        self._chk(lib().pz_u8_add(self.h, _arr(a), _arr(b), out, ctypes.byref(ov) if overflow else None), "u8_add")
        return (list(out), ov.value) if overflow else list(out)

    def u8_sub(self, a, b, overflow=False):
        out = (ctypes.c_uint32 * 8)()
        ov = ctypes.c_uint32(WIRE_NONE)
        self._chk(lib().pz_u8_sub(self.h, _arr(a), _arr(b), out, ctypes.byref(ov) if overflow else None), "u8_sub")
        return (list(out), ov.value) if overflow else list(out)

    def u8_mul(self, a, b):
        out = (ctypes.c_uint32 * 8)()
        self._chk(lib().pz_u8_mul(self.h, _arr(a), _arr(b), out), "u8_mul")
        return list(out)

    def u8_div_rem(self, a, b, flag=None, track_flag=True):
        """Returns (quotient, remainder, div_by_zero_flag)."""
        q = (ctypes.c_uint32 * 8)()
        r = (ctypes.c_uint32 * 8)()
        f = ctypes.c_uint32(WIRE_NONE if flag is None else flag)
        self._chk(lib().pz_u8_div_rem(self.h, _arr(a), _arr(b), q, r, ctypes.byref(f) if track_flag else None),
                  "u8_div_rem")
        return list(q), list(r), (f.value if track_flag else None)

    def u8_cmp(self, op, a, b):
        out = ctypes.c_uint32(WIRE_NONE)
        self._chk(lib().pz_u8_cmp(self.h, CMP_OPS[op], _arr(a), _arr(b), ctypes.byref(out)), "u8_cmp")
        return out.value

    def u8_mux(self, a, b, selector):
        out = (ctypes.c_uint32 * 8)()
        self._chk(lib().pz_u8_mux(self.h, _arr(a), _arr(b), selector, out), "u8_mux")
        return list(out)

    def u8_max(self, a, b):  # shortint/mod.rs:282-285
        return self.u8_mux(a, b, self.u8_cmp("gt", a, b))

    def u8_min(self, a, b):  # shortint/mod.rs:288-291
        return self.u8_mux(a, b, self.u8_cmp("lt", a, b))

    # -- wire format -----------------------------------------------------------------
    def serialize(self):
        size = ctypes.c_size_t()
        check(lib().pz_circuit_serialize(self.h, None, 0, ctypes.byref(size)), None, "pz_circuit_serialize")
        buf = ctypes.create_string_buffer(max(size.value, 1))
        check(lib().pz_circuit_serialize(self.h, buf, size.value, ctypes.byref(size)), None, "pz_circuit_serialize")
        return buf.raw[:size.value]

    @classmethod
    def deserialize(cls, blob):
        blob = bytes(blob)
        c = cls.__new__(cls)
        h = vp()
        check(lib().pz_circuit_deserialize(blob, len(blob), ctypes.byref(h)), None, "pz_circuit_deserialize")
        c.h = h
        info = c.info()
        c.n_inputs, c.n_outputs = info["inputs"], info["outputs"]
        return c

    # -- structure -----------------------------------------------------------------
    def info(self):
        v = [ctypes.c_size_t() for _ in range(5)]
        check(lib().pz_circuit_info(self.h, *[ctypes.byref(x) for x in v]), None, "pz_circuit_info")
        keys = ["inputs", "gates", "outputs", "levels", "max_level_width"]
        return {k: x.value for k, x in zip(keys, v)}

    def level_sizes(self):
        n = self.info()["levels"]
        arr = (ctypes.c_size_t * max(n, 1))()
        check(lib().pz_circuit_level_sizes(self.h, arr, n), None, "pz_circuit_level_sizes")
        return list(arr)[:n]

    # -- execution -------------------------------------------------------------------
    def run(self, engine, key, inputs):
        """Host buffers: inputs [n_inputs][N+1] -> outputs [n_outputs][N+1]."""
        inputs = np.ascontiguousarray(inputs, np.uint64).reshape(-1, engine.L)
        if len(inputs) != self.n_inputs:
            raise ValueError(f"expected {self.n_inputs} input ciphertexts, got {len(inputs)}")
        out = np.zeros((self.n_outputs, engine.L), np.uint64)
        check(lib().pz_circuit_run(engine.h, key.h, self.h, inputs.ctypes.data_as(u64p),
                                   out.ctypes.data_as(u64p)), engine.h, "pz_circuit_run")
        return out

    def run_device(self, engine, key, d_inputs, d_outputs, stream=None):
        check(lib().pz_circuit_run_device(engine.h, key.h, self.h, _ptr(d_inputs), _ptr(d_outputs),
                                          _stream(stream)), engine.h, "pz_circuit_run_device")

    def capture_graph(self, engine, key, d_inputs, d_outputs, stream=None):
        check(lib().pz_circuit_capture_graph(engine.h, key.h, self.h, _ptr(d_inputs), _ptr(d_outputs),
                                             _stream(stream)), engine.h, "pz_circuit_capture_graph")

    def replay_graph(self, stream=None):
        self._chk(lib().pz_circuit_replay_graph(self.h, _stream(stream)), "replay_graph")
