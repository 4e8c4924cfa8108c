"""Multi-session executor over the C ABI (pz_server_*): continuous batching of
circuits from many sessions, each with its own device-resident server key and
parameter set, on one device.

Each ``step()`` admits pending jobs in arrival order while their wires fit the
device arena, runs the next circuit level of every admitted job -- all
sessions together -- as one ragged key-switch launch and one ragged
blind-rotation launch, and retires finished jobs.  One host thread drives a
server.  ``device=DRY_RUN`` gives a host-only server (admission and level
bookkeeping without GPU work).
"""
import ctypes

import numpy as np

from ._lib import PzServerStats, lib, u32p, u64p, vp
from .engine import _ptr

DRY_RUN = -1
PENDING, RUNNING, DONE, FAILED = 0, 1, 2, 3


SCHEDULE_ALL_READY, SCHEDULE_CRITICAL_PATH = 0, 1


class Server:
    def __init__(self, device=0, arena_bytes=1 << 30, max_items=8192):
        h = vp()
        st = lib().pz_server_create(int(device), int(arena_bytes), int(max_items), ctypes.byref(h))
        if st != 0:
            raise RuntimeError(f"pz_server_create failed ({lib().pz_status_string(st).decode()})")
        self.h = h
        self.device = device
        self._keep = {}  # job -> buffers that must outlive the job
        self.L = None

    def close(self):
        if getattr(self, "h", None):
            lib().pz_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, status, what):
        if status != 0:
            raise RuntimeError(f"{what}: {lib().pz_server_last_error(self.h).decode()}")

    def add_session(self, engine, key):
        sid = ctypes.c_uint32()
        self._chk(lib().pz_server_add_session(self.h, engine.h, key.h, ctypes.byref(sid)), "add_session")
        self.L = engine.L
        return sid.value

    def add_managed_session(self, engine, key_blob):
        """A session whose device key the server imports from `key_blob` (the
        bytes of DeviceKey.export(), kept referenced here) when a job needs it
        and evicts when the key budget calls for room (least recently used,
        no job in flight).  Sessions may share one blob object."""
        sid = ctypes.c_uint32()
        blob = key_blob if isinstance(key_blob, bytes) else bytes(key_blob)
        self._blobs = getattr(self, "_blobs", {})
        self._blobs[id(blob)] = blob  # the server reads it on every import: keep it alive
        self._chk(lib().pz_server_add_managed_session(self.h, engine.h, blob, len(blob), ctypes.byref(sid)),
                  "add_managed_session")
        self.L = engine.L
        return sid.value

    def add_virtual_managed_session(self, param_id):
        """Dry-run servers: a managed session (residency bookkeeping only)."""
        sid = ctypes.c_uint32()
        self._chk(lib().pz_server_add_virtual_managed_session(self.h, int(param_id), ctypes.byref(sid)),
                  "add_virtual_managed_session")
        return sid.value

    def set_key_budget(self, nbytes):
        """Device bytes resident managed keys may hold (0: no limit)."""
        self._chk(lib().pz_server_set_key_budget(self.h, int(nbytes)), "set_key_budget")

    def resident(self, session):
        r = ctypes.c_int()
        self._chk(lib().pz_server_session_resident(self.h, int(session), ctypes.byref(r)), "session_resident")
        return bool(r.value)

    def add_virtual_session(self, param_id):
        sid = ctypes.c_uint32()
        self._chk(lib().pz_server_add_virtual_session(self.h, int(param_id), ctypes.byref(sid)),
                  "add_virtual_session")
        return sid.value

    def submit(self, session, circuit, inputs=None, device_outputs=None):
        """Host inputs (numpy [n_inputs][N+1]) -> returns the job id; the
        outputs array is available from ``result(job)`` once done.  With
        torch CUDA tensors for inputs and device_outputs the job reads and
        writes device memory directly."""
        job = ctypes.c_uint64()
        if device_outputs is not None:
            self._chk(lib().pz_server_submit(self.h, session, circuit.h, _ptr(inputs), _ptr(device_outputs), 1,
                                             ctypes.byref(job)), "submit")
            self._keep[job.value] = (circuit, inputs, device_outputs)
            return job.value
        if inputs is None:  # dry run: no buffers
            self._chk(lib().pz_server_submit(self.h, session, circuit.h, None, None, 0, ctypes.byref(job)), "submit")
            self._keep[job.value] = (circuit, None, None)
            return job.value
        inputs = np.ascontiguousarray(inputs, np.uint64)
        L = inputs.shape[-1]
        out = np.zeros((circuit.n_outputs, L), np.uint64)
        self._chk(lib().pz_server_submit(self.h, session, circuit.h, inputs.ctypes.data_as(u64p),
                                         out.ctypes.data_as(u64p), 0, ctypes.byref(job)), "submit")
        self._keep[job.value] = (circuit, inputs, out)
        return job.value

    def step(self):
        n = ctypes.c_size_t()
        self._chk(lib().pz_server_step(self.h, ctypes.byref(n)), "step")
        return n.value

    def run_until_idle(self, max_steps=1 << 30):
        steps = 0
        while steps < max_steps:
            s = self.stats()
            if s["pending"] == 0 and s["active"] == 0:
                break
            self.step()
            steps += 1
        return steps

    def status(self, job):
        st, lat, qu = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
        self._chk(lib().pz_server_job_status(self.h, job, ctypes.byref(st), ctypes.byref(lat), ctypes.byref(qu)),
                  "job_status")
        return {"state": st.value, "latency_ms": lat.value, "queue_ms": qu.value}

    def result(self, job):
        if self.status(job)["state"] != DONE:
            raise RuntimeError(f"job {job} is not done")
        return self._keep[job][2]

    def forget(self, job):
        self._chk(lib().pz_server_forget(self.h, job), "forget")
        self._keep.pop(job, None)

    def stats(self):
        s = PzServerStats()
        self._chk(lib().pz_server_stats_get(self.h, ctypes.byref(s)), "stats")
        return {n: getattr(s, n) for n, _ in PzServerStats._fields_}

    def set_launch(self, pbs_variant, grid_limit=0):
        self._chk(lib().pz_server_set_launch(self.h, int(pbs_variant), int(grid_limit)), "set_launch")

    def set_schedule(self, policy):
        """ALL_READY (0, default) or CRITICAL_PATH (1): see pz_server_set_schedule."""
        self._chk(lib().pz_server_set_schedule(self.h, int(policy)), "set_schedule")

    def autotune(self, batch):
        v, g, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self._chk(lib().pz_server_autotune(self.h, int(batch), ctypes.byref(v), ctypes.byref(g), ctypes.byref(ms)),
                  "autotune")
        return {"variant": v.value, "grid_limit": g.value, "ms": ms.value}
