"""demsph_build_hash_start_end_noalloc against buildHashStartEnd.

The non-allocating entry point exists for callers that cannot allocate
device memory while they run: for example a host loop that reserved its
whole GPU memory budget before starting, or code that issues work where a
cudaMalloc is not allowed because it may synchronise the device or fail
under memory pressure.  It does the same sort as buildHashStartEnd with a
fixed scratch array inside the library instead of a per-call allocation.

Two calls in a row with different inputs must give exactly the results of
the allocating entry point (the outputs are integers, so the tolerance is
zero), must leave the device's memory pool and free memory where they were
(nothing allocated, not even for the length of the call), and a size beyond
the fixed scratch must be rejected with a message.  One case holds keys at
or above the start / end table size, which the table skips.  This file is
named to be collected last; it also runs alone.
"""
import ctypes as C

import numpy as np
import pytest

from this_studio_b200 import _lib

from .test_gpu_compat import expected

pytestmark = pytest.mark.gpu

MAX_KEYS = 262144  # DEMSPH_NOALLOC_MAX_KEYS in include/demsph.h


def _buffers(torch, keys, ncell):
    dev = torch.device("cuda")
    hv = torch.tensor(keys, dtype=torch.int32, device=dev)
    hi = torch.full((len(keys),), -5, dtype=torch.int32, device=dev)
    st = torch.full((ncell,), -1, dtype=torch.int32, device=dev)
    en = torch.full((ncell,), -1, dtype=torch.int32, device=dev)
    return hv, hi, st, en


def _call(torch, fn, bufs, ncell):
    hv, hi, st, en = bufs
    s = torch.cuda.current_stream().cuda_stream
    L = _lib.lib()
    if fn == "noalloc":
        return L.demsph_build_hash_start_end_noalloc(st.data_ptr(), en.data_ptr(), hi.data_ptr(), hv.data_ptr(),
                                                     ncell, hv.numel(), s)
    L.buildHashStartEnd(st.data_ptr(), en.data_ptr(), hi.data_ptr(), hv.data_ptr(), ncell, hv.numel(), 0, 0, s)
    return 0


def _sort(torch, fn, keys, ncell):
    bufs = _buffers(torch, keys, ncell)
    rc = _call(torch, fn, bufs, ncell)
    torch.cuda.synchronize()
    return rc, [t.cpu().numpy() for t in bufs]


class _Pool:
    """The current device's default stream-ordered memory pool (the one
    cudaMallocAsync draws from) and the device's free memory, through the
    driver API."""

    USED, USED_HIGH, RESERVED = 7, 8, 5  # CU_MEMPOOL_ATTR_*

    def __init__(self):
        self.cu = C.CDLL("libcuda.so.1")
        dev = C.c_int()
        assert self.cu.cuCtxGetDevice(C.byref(dev)) == 0
        self.pool = C.c_void_p()
        assert self.cu.cuDeviceGetDefaultMemPool(C.byref(self.pool), dev) == 0

    def attr(self, a):
        v = C.c_uint64()
        assert self.cu.cuMemPoolGetAttribute(self.pool, a, C.byref(v)) == 0
        return v.value

    def reset_high(self):
        z = C.c_uint64(0)  # resets the watermark to the current use
        assert self.cu.cuMemPoolSetAttribute(self.pool, self.USED_HIGH, C.byref(z)) == 0

    def free(self):
        f, t = C.c_size_t(), C.c_size_t()
        assert self.cu.cuMemGetInfo_v2(C.byref(f), C.byref(t)) == 0
        return f.value


def test_noalloc_matches_allocating_entry_point(gpu):
    import torch

    rng = np.random.default_rng(42)
    cases = [(100_000, 30_000, 0), (MAX_KEYS, 50_000, 1)]
    inputs = []
    for n, ncell, above in cases:
        keys = rng.integers(-1, ncell + (ncell // 10 if above else 0), size=n)
        keys[rng.random(n) < 0.25] = -1
        inputs.append((keys, ncell))
    assert (inputs[1][0] >= inputs[1][1]).sum() > 1000  # keys the start / end table skips
    # the first call on a device may load the library's module (which holds
    # the fixed array); make it before measuring
    rc, _ = _sort(torch, "noalloc", inputs[0][0][:1000], 16)
    assert rc == _lib.OK, _lib.lib().demsph_last_error()
    torch.cuda.synchronize()
    bufs = [_buffers(torch, keys, ncell) for keys, ncell in inputs]
    torch.cuda.synchronize()
    pool = _Pool()
    pool.reset_high()
    used0, res0, free0 = pool.attr(pool.USED), pool.attr(pool.RESERVED), pool.free()
    for b, (keys, ncell) in zip(bufs, inputs):  # two calls in a row on the shared scratch
        rc = _call(torch, "noalloc", b, ncell)
        assert rc == _lib.OK, _lib.lib().demsph_last_error()
    torch.cuda.synchronize()
    assert pool.attr(pool.USED) == used0 and pool.attr(pool.USED_HIGH) == used0
    assert pool.attr(pool.RESERVED) == res0
    assert pool.free() == free0
    got = [[t.cpu().numpy() for t in b] for b in bufs]
    for (keys, ncell), out in zip(inputs, got):
        _, ref = _sort(torch, "alloc", keys, ncell)
        for a, b in zip(out, ref):
            np.testing.assert_array_equal(a, b)
        # and on its own against numpy: stable order, start / end of each cell
        for a, b in zip(out, expected(keys, ncell)):
            np.testing.assert_array_equal(a, b)


def test_noalloc_rejects_oversize(gpu):
    import torch

    keys = np.zeros(MAX_KEYS + 1, np.int64)
    rc, _ = _sort(torch, "noalloc", keys, 4)
    assert rc == _lib.ERR_INVALID
    assert b"exceed" in _lib.lib().demsph_last_error()
