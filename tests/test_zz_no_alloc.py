"""demsph_build_hash_start_end_noalloc against buildHashStartEnd.

The non-allocating entry point exists for callers that cannot allocate
device memory while they run: for example a host loop that reserved its
whole GPU memory budget before starting, or code that issues work where a
cudaMalloc is not allowed because it may synchronise the device or fail
under memory pressure.  It does the same sort as buildHashStartEnd with a
fixed scratch array inside the library instead of a per-call allocation.

Two calls in a row with different inputs must give exactly the results of
the allocating entry point (the outputs are integers, so the tolerance is
zero), and a size beyond the fixed scratch must be rejected with a message.
This file is named to be collected last; it also runs alone.
"""
import numpy as np
import pytest

from this_studio_b200 import _lib

pytestmark = pytest.mark.gpu

MAX_KEYS = 262144  # DEMSPH_NOALLOC_MAX_KEYS in include/demsph.h


def _sort(torch, fn, keys, ncell):
    dev = torch.device("cuda")
    hv = torch.tensor(keys, dtype=torch.int32, device=dev)
    hi = torch.full((len(keys),), -5, dtype=torch.int32, device=dev)
    st = torch.full((ncell,), -1, dtype=torch.int32, device=dev)
    en = torch.full((ncell,), -1, dtype=torch.int32, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    L = _lib.lib()
    if fn == "noalloc":
        rc = L.demsph_build_hash_start_end_noalloc(st.data_ptr(), en.data_ptr(), hi.data_ptr(), hv.data_ptr(),
                                                   ncell, len(keys), s)
    else:
        L.buildHashStartEnd(st.data_ptr(), en.data_ptr(), hi.data_ptr(), hv.data_ptr(), ncell, len(keys), 0, 0, s)
        rc = 0
    torch.cuda.synchronize()
    return rc, [t.cpu().numpy() for t in (hv, hi, st, en)]


def test_noalloc_matches_allocating_entry_point(gpu):
    import torch

    rng = np.random.default_rng(42)
    cases = [(100_000, 30_000), (MAX_KEYS, 50_000)]
    for n, ncell in cases:  # two calls in a row on the shared scratch
        keys = rng.integers(-1, ncell, size=n)
        keys[rng.random(n) < 0.25] = -1
        rc, got = _sort(torch, "noalloc", keys, ncell)
        assert rc == _lib.OK, _lib.lib().demsph_last_error()
        _, ref = _sort(torch, "alloc", keys, ncell)
        for a, b in zip(got, ref):
            np.testing.assert_array_equal(a, b)


def test_noalloc_rejects_oversize(gpu):
    import torch

    keys = np.zeros(MAX_KEYS + 1, np.int64)
    rc, _ = _sort(torch, "noalloc", keys, 4)
    assert rc == _lib.ERR_INVALID
    assert b"exceed" in _lib.lib().demsph_last_error()
