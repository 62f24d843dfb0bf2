"""cpra_b200_converge_error_noalloc: ConvergeError for callers that cannot
allocate GPU memory while they run (their device memory is reserved by another
allocator or pool, or cudaFree's device-wide synchronisation would stall their
other streams).  It keeps its partial sums in a fixed scratch array compiled
into the library instead of allocating, needs no context, and must give what
the regular entry point gives.  This file is collected last so that a run that
stops at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F32, F64 = 0, 1


def _run_both(torch, cb, M, N, L, B, dtype, seed):
    """(old, err) from the context entry point and from the no-alloc one on
    the same inputs."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    cdt = torch.complex64 if dtype == np.float32 else torch.complex128
    n = M * N * L * B
    old = torch.randn(n, dtype=cdt, device="cuda", generator=g)
    new = torch.randn(n, dtype=cdt, device="cuda", generator=g)

    impl = cb.B200Impl(M, N, L, B, dtype=np.dtype(dtype).name)
    old_a = old.clone()
    err_a = np.zeros(B, dtype)
    assert impl.ConvergeError(old_a, new, err_a, M, N, L, B)
    impl.close()

    old_b = old.clone()
    err_b = np.full(B, -1, dtype)
    torch.cuda.synchronize()
    rc = cb.lib().cpra_b200_converge_error_noalloc(F64 if dtype == np.float64 else F32, old_b.data_ptr(),
                                                   new.data_ptr(), err_b.ctypes.data_as(ctypes.c_void_p),
                                                   M, N, L, B, None)
    assert rc == cb.OK, cb.last_error()
    return old_a.cpu().numpy(), err_a, old_b.cpu().numpy(), err_b


def test_noalloc_converge_error_matches_regular_entry(cuda):
    import torch
    import cpra_b200 as cb
    # several calls in a row share the static scratch; each must stand alone
    for k, (M, N, L, B, dt) in enumerate([(32, 32, 2, 3, np.float32), (16, 8, 1, 7, np.float32),
                                          (8, 8, 4, 2, np.float64), (64, 64, 1, 256, np.float32)]):
        old_a, err_a, old_b, err_b = _run_both(torch, cb, M, N, L, B, dt, seed=11 + k)
        np.testing.assert_array_equal(old_b, old_a)   # old <- new - old, element-wise exact
        # both take IEEE double square roots and a division of the same FP64 sums
        np.testing.assert_array_equal(err_b, err_a)
        assert np.all(np.isfinite(err_b)) and np.all(err_b > 0)


def test_noalloc_converge_error_allocates_nothing(cuda):
    """After the first call on the device (which loads the library's device
    code and with it the scratch array), further calls leave the device's free
    memory unchanged."""
    import torch
    import cpra_b200 as cb
    M, N, L, B = 64, 64, 1, 256
    g = torch.Generator(device="cuda").manual_seed(5)
    new = torch.randn(M * N * L * B, dtype=torch.complex64, device="cuda", generator=g)
    olds = [torch.randn(M * N * L * B, dtype=torch.complex64, device="cuda", generator=g) for _ in range(3)]
    errs = [np.zeros(B, np.float32) for _ in range(4)]

    def call(old, err):
        rc = cb.lib().cpra_b200_converge_error_noalloc(F32, old.data_ptr(), new.data_ptr(),
                                                       err.ctypes.data_as(ctypes.c_void_p), M, N, L, B, None)
        assert rc == cb.OK, cb.last_error()

    first = olds[0].clone()
    torch.cuda.synchronize()
    call(first, errs[3])
    free_before = torch.cuda.mem_get_info()[0]
    for old, err in zip(olds, errs):
        call(old, err)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    np.testing.assert_array_equal(errs[0], errs[3])   # same inputs, same bits


def test_noalloc_converge_error_refuses_batches_above_the_limit(cuda):
    import torch
    import cpra_b200 as cb
    B = 257
    x = torch.zeros(4 * B, dtype=torch.complex64, device="cuda")
    err = np.zeros(B, np.float32)
    rc = cb.lib().cpra_b200_converge_error_noalloc(F32, x.data_ptr(), x.data_ptr(),
                                                   err.ctypes.data_as(ctypes.c_void_p), 2, 2, 1, B, None)
    assert rc == cb.EARG
    assert "limit of 256" in cb.last_error()
