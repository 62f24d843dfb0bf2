"""Raw-file I/O of the reference program on the B200 backend (GPU).

The reference reads its constraint planes with Cpra::ReadMatrixFromFile and
writes one reconstruction file and one error file per start
(include/detail/CPRA.inl:8-48, src/CPRA_MKL.cpp:156-225).  Files are raw
elements with no header, so numpy's tofile/fromfile are the reference format.
Everything here is bit-exact: the I/O entries only move and select data, and
cpra_files must write what Initialize + cpra_run produce batch by batch.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tb(cuda):
    import torch
    import cpra_b200
    return torch, cpra_b200


def test_read_matrix_into_any_memory(tb, tmp_path):
    torch, cb = tb
    rng = np.random.default_rng(1)
    data = rng.standard_normal(100_003).astype(np.float32)
    f = tmp_path / "a.f32"
    data.tofile(f)
    impl = cb.B200Impl(8, 8, 1, 1)
    assert impl.set_option(cb.OPT_IO_CHUNK, 4096)  # 98 chunks through the two pinned buffers
    assert impl.get_option(cb.OPT_IO_CHUNK) == 4096
    d = torch.empty(data.size, dtype=torch.float32, device="cuda")
    assert impl.read_matrix(f, d, data.size)
    np.testing.assert_array_equal(d.cpu().numpy(), data)
    pinned = torch.empty(data.size, dtype=torch.float32).pin_memory()
    assert impl.read_matrix(f, pinned, data.size)
    np.testing.assert_array_equal(pinned.numpy(), data)
    pageable = np.zeros(data.size, np.float32)
    assert impl.read_matrix(f, pageable, data.size)
    np.testing.assert_array_equal(pageable, data)
    managed = impl.alloc(data.nbytes, managed=True)
    assert impl.read_matrix(f, managed, data.size) and impl.Sync()
    got = np.ctypeslib.as_array((ctypes.c_float * data.size).from_address(managed))
    np.testing.assert_array_equal(got, data)
    impl.free(managed)
    # a prefix of the file, and f64 elements by the context's type
    part = torch.zeros(777, dtype=torch.float32, device="cuda")
    assert impl.read_matrix(f, part, 777)
    np.testing.assert_array_equal(part.cpu().numpy(), data[:777])
    d64 = rng.standard_normal(5000)
    d64.tofile(tmp_path / "b.f64")
    impl64 = cb.B200Impl(8, 8, 1, 1, "float64")
    t64 = torch.empty(5000, dtype=torch.float64, device="cuda")
    assert impl64.read_matrix(tmp_path / "b.f64", t64, 5000)
    np.testing.assert_array_equal(t64.cpu().numpy(), d64)


def test_read_matrix_errors(tb, tmp_path):
    """A missing file and a zero size are errors (include/detail/CPRA.inl:11-21);
    so is a short file."""
    torch, cb = tb
    impl = cb.B200Impl(8, 8, 1, 1)
    d = torch.zeros(64, dtype=torch.float32, device="cuda")
    assert not impl.read_matrix(tmp_path / "missing.f32", d, 64)
    assert "cannot open" in cb.last_error()
    np.arange(10, dtype=np.float32).tofile(tmp_path / "short.f32")
    assert not impl.read_matrix(tmp_path / "short.f32", d, 64)
    assert "short file" in cb.last_error()
    assert not impl.read_matrix(tmp_path / "short.f32", d, 0)
    assert not impl.set_option(cb.OPT_IO_CHUNK, 100)
    # the context stays usable
    assert impl.read_matrix(tmp_path / "short.f32", d, 10)
    np.testing.assert_array_equal(d[:10].cpu().numpy(), np.arange(10, dtype=np.float32))


def test_write_matrix_round_trip(tb, tmp_path):
    torch, cb = tb
    impl = cb.B200Impl(8, 8, 1, 1)
    assert impl.set_option(cb.OPT_IO_CHUNK, 8192)
    src = torch.randn(65_537, device="cuda")
    f = tmp_path / "w.f32"
    assert impl.write_matrix(f, src, src.numel())
    np.testing.assert_array_equal(np.fromfile(f, np.float32), src.cpu().numpy())
    # overwrite with fewer elements from host memory: the file is replaced
    h = np.arange(3, dtype=np.float32)
    assert impl.write_matrix(f, h, 3)
    np.testing.assert_array_equal(np.fromfile(f, np.float32), h)
    assert not impl.write_matrix(f, src, 0)


@pytest.mark.parametrize("M,N,P,B,count,dtype", [(16, 16, 3, 4, 3, "float32"), (6, 10, 2, 3, 3, "float32"),
                                                 (8, 8, 3, 2, 2, "float64")])
def test_write_starts_files(tb, tmp_path, M, N, P, B, count, dtype):
    """Start i's files: the real parts of its P planes and its P errors
    (src/CPRA_MKL.cpp:186-209), numbered from file_index."""
    torch, cb = tb
    rdt, cdt = (np.float32, np.complex64) if dtype == "float32" else (np.float64, np.complex128)
    rng = np.random.default_rng(M * N + P)
    x = (rng.standard_normal((P, B, M, N)) + 1j * rng.standard_normal((P, B, M, N))).astype(cdt)
    err = rng.uniform(0, 1, P * B).astype(rdt)
    impl = cb.B200Impl(M, N, 1, B, dtype)
    assert impl.set_option(cb.OPT_IO_CHUNK, 4096)
    xd = torch.from_numpy(x.ravel()).cuda()
    rec, erp = tmp_path / "rec", tmp_path / "err"
    assert impl.write_starts(rec, erp, 5, xd, err, P, B, count)
    for i in range(count):
        got = np.fromfile(f"{rec}.{5 + i}", rdt)
        np.testing.assert_array_equal(got, x[:, i].real.ravel())
        np.testing.assert_array_equal(np.fromfile(f"{erp}.{5 + i}", rdt), err.reshape(P, B)[:, i])
    assert not (tmp_path / f"rec.{5 + count}").exists()
    # reconstructions only
    assert impl.write_starts(tmp_path / "only", None, 1, xd, None, P, B, 1)
    np.testing.assert_array_equal(np.fromfile(tmp_path / "only.1", rdt), x[:, 0].real.ravel())
    assert not impl.write_starts(rec, erp, 1, xd, err, P, B, B + 1)
    assert not impl.write_starts(rec, None, 1, xd, err, P, B, 1)


@pytest.mark.parametrize("L,P,B,total,epi,it,pre", [(64, 4, 3, 7, 2, 2, 1), (128, 3, 2, 0, 1, 2, 0),
                                                    (256, 3, 2, 3, 1, 2, 1)])
def test_cpra_files_matches_batches(tb, tmp_path, L, P, B, total, epi, it, pre):
    """cpra_files (src/CPRA_MKL.cpp:156-225 without the parser) writes, for
    max(batch, total) starts in batches, exactly what Initialize + cpra_run +
    write_starts give batch by batch on a context with the same seed."""
    torch, cb = tb
    rng = np.random.default_rng(L + total)
    A = (rng.uniform(0, 30, (P, L, L)) * (rng.uniform(0, 1, (P, L, L)) > 0.1)).astype(np.float32)
    S = (rng.uniform(0, 1, (P, L, L)) > 0.45).astype(np.float32)
    A.tofile(tmp_path / "A.f32")
    S.tofile(tmp_path / "S.f32")
    run = cb.B200Impl(L, L, 1, B)
    assert run.set_option(cb.OPT_SEED, 77)
    assert run.cpra_files(tmp_path / "A.f32", tmp_path / "S.f32", tmp_path / "rec", tmp_path / "err", P, total, epi,
                          it, pre, 0.9)
    ref = cb.B200Impl(L, L, 1, B)
    assert ref.set_option(cb.OPT_SEED, 77)
    Ad = torch.from_numpy(A.ravel()).cuda()
    Sd = torch.from_numpy(S.ravel()).cuda()
    x = torch.empty(P * B * L * L, dtype=torch.complex64, device="cuda")
    n_total = max(B, total)
    done = 0
    while done < n_total:
        n = min(B, n_total - done)
        err = np.zeros(P * B, np.float32)
        assert ref.Initialize(torch.view_as_real(x), 2 * x.numel())
        assert ref.cpra_run(x, Ad, Sd, P, B, epi, it, pre, 0.9, final_step=True, err=err) and ref.Sync()
        xr = x.cpu().numpy().reshape(P, B, L, L)
        for i in range(n):
            k = done + i + 1
            np.testing.assert_array_equal(np.fromfile(tmp_path / f"rec.{k}", np.float32), xr[:, i].real.ravel())
            np.testing.assert_array_equal(np.fromfile(tmp_path / f"err.{k}", np.float32), err.reshape(P, B)[:, i])
        done += n
    assert not (tmp_path / f"rec.{n_total + 1}").exists()
    assert not run.cpra_files(tmp_path / "nope.f32", tmp_path / "S.f32", tmp_path / "rec", tmp_path / "err", P,
                              total, epi, it, pre, 0.9)


@pytest.mark.parametrize("M,N,L,B,total,iters", [(16, 16, 16, 2, 3, 2), (32, 16, 8, 3, 0, 1)])
def test_conv_files_matches_batches(tb, tmp_path, M, N, L, B, total, iters):
    """conv_files (src/CONV_MKL.cpp:103-172 without the parser) writes, for
    every start of max(batch, total), its volume's real parts and its error,
    exactly as Initialize + conv_run give them batch by batch."""
    torch, cb = tb
    rng = np.random.default_rng(M + N + L + total)
    vol = M * N * L
    A = (rng.uniform(0, 40, vol) * (rng.uniform(0, 1, vol) > 0.1)).astype(np.float32)
    S = (rng.uniform(0, 1, vol) > 0.5).astype(np.float32)
    A.tofile(tmp_path / "A.f32")
    S.tofile(tmp_path / "S.f32")
    run = cb.B200Impl(M, N, L, B)
    assert run.set_option(cb.OPT_SEED, 5)
    assert run.conv_files(tmp_path / "A.f32", tmp_path / "S.f32", tmp_path / "rec", tmp_path / "err", total, iters,
                          0.9)
    ref = cb.B200Impl(M, N, L, B)
    assert ref.set_option(cb.OPT_SEED, 5)
    Ad, Sd = torch.from_numpy(A).cuda(), torch.from_numpy(S).cuda()
    x = torch.empty(B * vol, dtype=torch.complex64, device="cuda")
    n_total = max(B, total)
    done = 0
    while done < n_total:
        n = min(B, n_total - done)
        err = np.zeros(B, np.float32)
        assert ref.Initialize(torch.view_as_real(x), 2 * x.numel())
        assert ref.conv_run(x, Ad, Sd, iters, 0.9, final_step=True, err=err) and ref.Sync()
        xr = x.cpu().numpy().reshape(B, vol)
        for i in range(n):
            k = done + i + 1
            np.testing.assert_array_equal(np.fromfile(tmp_path / f"rec.{k}", np.float32), xr[i].real)
            np.testing.assert_array_equal(np.fromfile(tmp_path / f"err.{k}", np.float32), err[i:i + 1])
        done += n
    assert not (tmp_path / f"rec.{n_total + 1}").exists()
