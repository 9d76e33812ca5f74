"""The allocation-free radix sort (ys_radix_sort_pairs_noalloc) against the
regular one, through the C ABI.

Some callers cannot call cudaMalloc -- graph-capturing code, allocation-free
real-time loops, hosts that own all device memory -- so the library offers a
sort whose scratch is a fixed __device__ array.  Two calls in a row must give
exactly the regular sort's keys and values (bit-exact: the sort is integer
work), which also shows that a call does not depend on what the previous call
left in the shared array.  Named to run last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sorted_regular(lib, keys, vals):
    import torch
    from ysim_b200 import _lib
    dk = torch.from_numpy(keys.view(np.int32).copy()).cuda()
    dv = torch.from_numpy(vals.view(np.int32).copy()).cuda()
    scratch = torch.empty(int(lib.ys_radix_sort_scratch_bytes(len(keys))) + 16, dtype=torch.uint8, device="cuda")
    _lib.check(lib.ys_radix_sort_pairs(C.c_void_p(dk.data_ptr()), C.c_void_p(dv.data_ptr()), len(keys),
                                       C.c_void_p(scratch.data_ptr()), None))
    return dk.cpu().numpy().view(np.uint32), dv.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_regular_sort_twice_in_a_row(cuda_lib):
    import torch
    from ysim_b200 import _lib
    rng = np.random.default_rng(2024)
    for n in (300_001, 1 << 20):  # two calls: a ragged size, then the maximum
        keys = rng.integers(0, 1 << 30, n, dtype=np.uint32)
        keys[: n // 4] = keys[7]  # long runs of equal keys: stability matters
        vals = np.arange(n, dtype=np.uint32)
        want_k, want_v = _sorted_regular(cuda_lib, keys, vals)
        dk = torch.from_numpy(keys.view(np.int32).copy()).cuda()
        dv = torch.from_numpy(vals.view(np.int32).copy()).cuda()
        torch.cuda.synchronize()
        _lib.check(cuda_lib.ys_radix_sort_pairs_noalloc(C.c_void_p(dk.data_ptr()), C.c_void_p(dv.data_ptr()), n,
                                                        None), "ys_radix_sort_pairs_noalloc")
        torch.cuda.synchronize()
        assert np.array_equal(dk.cpu().numpy().view(np.uint32), want_k)
        assert np.array_equal(dv.cpu().numpy().view(np.uint32), want_v)


def test_noalloc_sort_rejects_sizes_beyond_its_scratch(cuda_lib):
    from ysim_b200 import _lib
    st = cuda_lib.ys_radix_sort_pairs_noalloc(C.c_void_p(16), C.c_void_p(16), (1 << 20) + 1, None)
    assert st == -4  # YS_ERR_CAPACITY, before any device access
    assert b"exceeds" in cuda_lib.ys_last_error()
