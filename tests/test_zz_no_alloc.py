"""gk_tc_count_noalloc: the triangle count for callers that cannot let the
library allocate GPU memory (their framework already holds the device's memory,
or their host forbids allocations while it runs).  It must give the same count
as gk_tc_count, call after call, although every call reuses the same fixed
device array; graphs beyond the array's row limit and host-resident inputs are
refused.  Collected last so that a run stopping at its first failure has run
everything else."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def noalloc_count(gk, L, sched=0):
    lib = gk.load()
    out = ctypes.c_uint64(0)
    g = L.as_gk()
    status = lib.gk_tc_count_noalloc(ctypes.byref(g), ctypes.addressof(out), sched, None)
    return status, int(out.value)


def test_noalloc_matches_tc_count_twice(gk, orc, cuda):
    import torch
    for scale, seed in [(16, 3), (12, 1), (20, 2)]:
        A = gk.gen_rmat(scale, 16, seed=seed, device="cuda")
        L = gk.extract_lower(A)
        torch.cuda.synchronize()
        want = gk.tc_count(L)
        for _ in range(2):  # the second call sees the first call's leftovers in the shared array
            status, got = noalloc_count(gk, L)
            assert status == 0, gk.load().gk_last_error_string()
            assert got == want
    # a small graph after a large one, then against the oracle
    A = gk.gen_rmat(10, 16, seed=7, device="cuda")
    L = gk.extract_lower(A)
    status, got = noalloc_count(gk, L)
    assert status == 0 and got == gk.tc_count(L) == orc.tc_lower(L.numpy())


def test_noalloc_device_output(gk, cuda):
    import torch
    lib = gk.load()
    A = gk.gen_rmat(14, 16, seed=1, device="cuda")
    L = gk.extract_lower(A)
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    g = L.as_gk()
    assert lib.gk_tc_count_noalloc(ctypes.byref(g), ctypes.c_void_p(out.data_ptr()), 0,
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
    torch.cuda.synchronize()
    assert int(out.item()) == gk.tc_count(L)


def test_noalloc_empty_graphs(gk, cuda):
    """An empty graph gives 0; its one-entry row pointer must still be in
    device memory, since the content check reads it on the device."""
    import torch
    from tests import graphs as G
    for n in (0, 5):
        E = G.empty(n)
        status, got = noalloc_count(gk, E.to("cuda"))
        assert status == 0 and got == 0, gk.load().gk_last_error_string()
        status, _ = noalloc_count(gk, E)  # host rowptr {0, ...}
        assert status == 1 and b"device memory" in gk.load().gk_last_error_string()
    torch.cuda.synchronize()
    # the library still works after the refusals
    A = gk.gen_rmat(8, 16, seed=2, device="cuda")
    L = gk.extract_lower(A)
    status, got = noalloc_count(gk, L)
    assert status == 0 and got == gk.tc_count(L)


def test_noalloc_refuses_what_it_cannot_hold(gk, cuda):
    A = gk.gen_rmat(21, 4, seed=1, device="cuda")  # 2,097,152 rows > 1,048,576
    L = gk.extract_lower(A)
    status, _ = noalloc_count(gk, L)
    assert status == 1 and b"1048576" in gk.load().gk_last_error_string()
    H = gk.lower_host(gk.gen_rmat(8, 16, seed=1))  # host arrays would need staging
    status, _ = noalloc_count(gk, H)
    assert status == 1 and b"device memory" in gk.load().gk_last_error_string()
