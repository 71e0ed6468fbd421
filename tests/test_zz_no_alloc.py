"""SortByKeyNoAlloc, the allocation-free variant of SortByKey.

Some callers cannot let a library allocate device memory: a host that owns
all device memory through its own pool, or a time-critical loop where a
cudaMalloc (which can synchronise the device or fail under memory pressure)
is not acceptable.  SortByKeyNoAlloc keeps its scratch in a fixed array of
about 2.4 MB inside the library instead, so it accepts at most 262,144
pairs.  These checks call it through the C ABI and compare it, bit for bit,
with SortByKey on the same input, twice in a row (the fixed array keeps the
previous call's contents).  This file is collected last so that a run that
stops at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from sphpc_b200 import _lib

pytestmark = pytest.mark.gpu

MAX_PAIRS = 1 << 18


def _u32(t):
    return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_uint))


def test_no_alloc_sort_matches_sort_by_key_twice():
    import torch
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(2024)
    for n, maxkey in ((200_003, 1 << 21), (MAX_PAIRS, 1 << 30), (4097, 37)):
        keys = rng.integers(0, maxkey, size=n, dtype=np.int64).astype(np.uint32)
        vals = rng.permutation(n).astype(np.uint32)
        ka = torch.from_numpy(keys.view(np.int32)).cuda()
        va = torch.from_numpy(vals.view(np.int32)).cuda()
        kb, vb = ka.clone(), va.clone()
        _lib.call("SortByKey", _u32(ka), _u32(va), n, stream)
        _lib.call("SortByKeyNoAlloc", _u32(kb), _u32(vb), n, stream)
        torch.cuda.synchronize()
        assert torch.equal(ka, kb)
        assert torch.equal(va, vb)
        # pinned by an independent stable sort as well, not only by SortByKey
        order = np.argsort(keys, kind="stable")
        np.testing.assert_array_equal(kb.cpu().numpy().view(np.uint32), keys[order])
        np.testing.assert_array_equal(vb.cpu().numpy().view(np.uint32), vals[order])


def test_no_alloc_sort_rejects_counts_above_its_limit():
    import torch
    n = MAX_PAIRS + 1
    k = torch.zeros(n, dtype=torch.int32, device="cuda")
    v = torch.zeros(n, dtype=torch.int32, device="cuda")
    rc = _lib.load().SortByKeyNoAlloc(_u32(k), _u32(v), n, None)
    assert rc == -1
    assert "262144" in _lib.load().sphpc_last_error().decode()
