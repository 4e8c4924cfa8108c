"""The allocation-free gate entry point (pz_gate_batch_device_noalloc).

Hosts that cannot allocate device memory on their gate path -- a process
whose GPU memory is reserved up front by another allocator, or a serving
thread that must not make allocating CUDA calls -- use this variant; its
key-switch scratch is a fixed array inside the library.  It must give the
same ciphertext words as pz_gate_batch_device (exact equality, like every
parity check in this suite) on consecutive calls, since all calls share and
reuse that array.  This file is collected last on purpose.
"""
import numpy as np
import pytest

from conftest import pz, to_dev, to_host

pytestmark = pytest.mark.gpu


def _setup(param, count, seed):
    P = pz()
    p = P.params(param)
    rng = np.random.default_rng(seed)
    N, n, L = p.rlwe_n, p.lwe_n, p.rlwe_n + 1
    eng = P.Engine(param)
    key = eng.upload_key(rng.integers(0, p.rlwe_q, (n, p.rgsw_rows, N), dtype=np.uint64),
                         rng.integers(0, p.rlwe_q, (p.n_auto_keys, p.auto_rows, N), dtype=np.uint64),
                         rng.integers(0, p.lwe_q, (p.lwe_d * N, n + 1), dtype=np.uint64))
    return eng, key, p, rng, L


class _DefaultPool:
    """The device's default stream-ordered memory pool (the one
    cudaMallocAsync draws from), read through the driver API: used and
    reserved bytes and their high watermarks."""
    RESERVED_CURRENT, RESERVED_HIGH, USED_CURRENT, USED_HIGH = 5, 6, 7, 8  # CUmemPool_attribute

    def __init__(self, ordinal=0):
        import ctypes
        self.ct = ctypes
        self.cu = ctypes.CDLL("libcuda.so.1")
        dev = ctypes.c_int()
        assert self.cu.cuDeviceGet(ctypes.byref(dev), ordinal) == 0
        self.pool = ctypes.c_void_p()
        assert self.cu.cuDeviceGetDefaultMemPool(ctypes.byref(self.pool), dev) == 0

    def get(self, attr):
        v = self.ct.c_uint64()
        assert self.cu.cuMemPoolGetAttribute(self.pool, attr, self.ct.byref(v)) == 0
        return v.value

    def reset_highs(self):  # a high watermark set to 0 restarts from the current value
        zero = self.ct.c_uint64(0)
        for attr in (self.USED_HIGH, self.RESERVED_HIGH):
            assert self.cu.cuMemPoolSetAttribute(self.pool, attr, self.ct.byref(zero)) == 0


def test_noalloc_matches_gate_batch_device_on_two_calls(gpu_available):
    """Two calls in a row equal pz_gate_batch_device word for word, and
    neither draws anything from the default memory pool (no cudaMallocAsync)
    or from torch's caching allocator."""
    import torch
    eng, key, p, rng, L = _setup("I_2P_LB_SR", 0, 2024)
    pool = _DefaultPool(torch.cuda.current_device())
    for call in range(2):  # the second call reuses the shared scratch left by the first
        count = 40 + 17 * call
        c0 = to_dev(rng.integers(0, p.rlwe_q, (count, L), dtype=np.uint64))
        c1 = to_dev(rng.integers(0, p.rlwe_q, (count, L), dtype=np.uint64))
        gates = to_dev(rng.integers(0, 6, count).astype(np.uint8))
        want = torch.empty_like(c0)
        got = torch.zeros_like(c0)
        eng.gate_batch_device(key, gates, c0, c1, want)  # this one allocates its scratch from the pool
        torch.cuda.synchronize()
        pool.reset_highs()
        used, reserved = pool.get(pool.USED_CURRENT), pool.get(pool.RESERVED_CURRENT)
        torch_reserved = torch.cuda.memory_reserved()
        eng.gate_batch_device_noalloc(key, gates, c0, c1, got)
        torch.cuda.synchronize()
        assert pool.get(pool.USED_HIGH) == used and pool.get(pool.RESERVED_HIGH) == reserved, \
            f"call {call}: the no-alloc path drew from the default memory pool"
        assert torch.cuda.memory_reserved() == torch_reserved
        assert np.array_equal(to_host(got), to_host(want)), f"call {call}: outputs differ"


def test_noalloc_rejects_batches_beyond_its_scratch(gpu_available):
    import torch
    eng, key, p, rng, L = _setup("SP_TEST", 0, 7)
    stride = (p.lwe_n + 1 + 31) // 32 * 32
    too_many = (4096 * 672) // stride + 1
    c0 = torch.zeros((too_many, L), dtype=torch.int64, device="cuda")
    gates = torch.zeros(too_many, dtype=torch.uint8, device="cuda")
    with pytest.raises(RuntimeError, match="exceed the fixed scratch"):
        eng.gate_batch_device_noalloc(key, gates, c0, c0, c0)
