"""The allocation-free counting sort (pbpic_counting_sort_keys_static).

Some callers cannot call cudaMalloc: a host code whose GPU memory is already
owned by another allocator, or a time loop that must not pay for an
allocation's synchronisation. For them the library offers the stateless
counting sort with its scratch in a static device array. These tests call it
through the C ABI and check its permutation and counts against the allocating
entry point, on two calls in a row (the second smaller than the first, so that
anything left in the shared scratch by the first call would show), and check
that sizes beyond the array's limit are refused. This file runs last so that a
failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(name, keys, ncells):
    import torch

    from pbpic_b200 import _lib as L
    n = keys.numel()
    perm = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    counts = torch.full((ncells,), -1, dtype=torch.int32, device="cuda")
    fn = getattr(L.lib(), name)
    L.check(fn(ctypes.c_void_p(keys.data_ptr()), n, ncells, ctypes.c_void_p(perm.data_ptr()),
               ctypes.c_void_p(counts.data_ptr()), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    return perm[:n].cpu().numpy(), counts.cpu().numpy()


def test_static_sort_matches_the_allocating_sort(gpu_lib):
    import torch
    g = torch.Generator().manual_seed(2024)
    cases = [(900_000, 70_000), (5_000, 300)]  # second call smaller: stale scratch would show
    for n, ncells in cases:
        keys = torch.randint(0, ncells, (n,), generator=g, dtype=torch.int32)
        keys[: n // 4] = 7  # a heavy cell
        kd = keys.cuda()
        p_static, c_static = _call("pbpic_counting_sort_keys_static", kd, ncells)
        p_alloc, c_alloc = _call("pbpic_counting_sort_keys", kd, ncells)
        assert np.array_equal(p_static, p_alloc)
        assert np.array_equal(c_static, c_alloc)
        assert np.array_equal(p_static, np.argsort(keys.numpy(), kind="stable"))


def test_static_sort_refuses_sizes_beyond_its_scratch(gpu_lib):
    import torch

    import pbpic_b200
    from pbpic_b200 import _lib as L
    n = L.STATIC_SORT_MAX_KEYS + 1
    kd = torch.zeros(n, dtype=torch.int32, device="cuda")
    with pytest.raises(pbpic_b200.PbpicError) as e:
        _call("pbpic_counting_sort_keys_static", kd, 4)
    assert e.value.code == -4 and "limit" in str(e.value)
    # the largest allowed size still works after the refusal
    kd = torch.randint(0, 4, (L.STATIC_SORT_MAX_KEYS,), dtype=torch.int32, device="cuda")
    p, c = _call("pbpic_counting_sort_keys_static", kd, 4)
    assert np.array_equal(p, np.argsort(kd.cpu().numpy(), kind="stable"))
