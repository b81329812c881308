"""The reference's sort / scan launchers (buildHashStartEnd, buildPrefixSum)
through the C ABI, against numpy: stable sort order, start / end tables and
the inclusive scan are integer results, so they must match exactly."""
import numpy as np
import pytest

from this_studio_b200 import _lib

pytestmark = pytest.mark.gpu


def _ptr(t):
    return t.data_ptr()


def run_hash_sort(torch, keys, ncell, fn="buildHashStartEnd"):
    dev = torch.device("cuda")
    hv = torch.tensor(keys, dtype=torch.int32, device=dev)
    hi = torch.full((len(keys),), -7, dtype=torch.int32, device=dev)
    st = torch.full((ncell,), -1, dtype=torch.int32, device=dev)
    en = torch.full((ncell,), -1, dtype=torch.int32, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    rc = getattr(_lib.lib(), fn)(_ptr(st), _ptr(en), _ptr(hi), _ptr(hv), ncell, len(keys), 0, 0, s)
    torch.cuda.synchronize()
    return rc, hv.cpu().numpy(), hi.cpu().numpy(), st.cpu().numpy(), en.cpu().numpy()


def expected(keys, ncell):
    keys = np.asarray(keys, np.int64)
    order = np.argsort(keys, kind="stable")
    sk = keys[order]
    st = np.full(ncell, -1, np.int64)
    en = np.full(ncell, -1, np.int64)
    for i, h in enumerate(sk):
        if 0 <= h < ncell:
            if i == 0 or sk[i - 1] != h:
                st[h] = i
            if i == len(sk) - 1 or sk[i + 1] != h:
                en[h] = i + 1
    return sk, order, st, en


@pytest.mark.parametrize("n,ncell", [(1, 4), (1000, 37), (70000, 5000), (300000, 40000)])
def test_build_hash_start_end(gpu, n, ncell):
    import torch

    rng = np.random.default_rng(n)
    keys = rng.integers(-1, ncell, size=n)
    keys[rng.random(n) < 0.3] = -1  # the dummy-hash case: many -1 keys
    _, hv, hi, st, en = run_hash_sort(torch, keys, ncell)
    sk, order, est, een = expected(keys, ncell)
    np.testing.assert_array_equal(hv, sk)
    np.testing.assert_array_equal(hi, order)
    np.testing.assert_array_equal(st, est)
    np.testing.assert_array_equal(en, een)


def test_build_hash_start_end_wide_keys(gpu):
    import torch

    rng = np.random.default_rng(2)
    keys = rng.integers(-2**31, 2**31 - 1, size=5000)
    keys[:100] = 7
    _, hv, hi, st, en = run_hash_sort(torch, keys, 16)
    sk, order, est, een = expected(keys, 16)
    np.testing.assert_array_equal(hv, sk)
    np.testing.assert_array_equal(hi, order)


@pytest.mark.parametrize("n", [1, 4096, 4097, 1_000_003])
def test_build_prefix_sum(gpu, n):
    import torch

    rng = np.random.default_rng(n)
    cnt = rng.integers(0, 9, size=n).astype(np.int32)
    dev = torch.device("cuda")
    c = torch.tensor(cnt, device=dev)
    out = torch.zeros(n, dtype=torch.int32, device=dev)
    _lib.lib().buildPrefixSum(out.data_ptr(), c.data_ptr(), n, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), np.cumsum(cnt, dtype=np.int64).astype(np.int32))
