"""Parity of the B200 backend with the oracle and the reference build (GPU).

Every operator is called through the C ABI (cpra_b200 -> libcpra_b200.so) on
seeded inputs and compared with the golden fixtures produced by the
reference's own MklImpl<T> source (tests/golden/make_golden.py) and with the
oracle.  Tolerances: integer/permutation/element-wise arithmetic bit-exact;
one FP32 transform 1e-6 relative L2; difference-map iterations 1e-5 relative
L2 per iteration (the stated per-iteration bound); FP64 transforms 1e-13.
"""
import numpy as np
import pytest

import cpra_oracle as O
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

G = np.load(GOLDEN / "ref_golden.npz")
FP32_FFT_TOL = 1e-6
FP32_DM_TOL = 1e-5


@pytest.fixture(scope="module")
def tb(cuda):
    import torch
    import cpra_b200
    return torch, cpra_b200


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.detach().cpu().numpy()


# ---- reference unit tests, on the B200 backend ---------------------------------------
def test_kat_merge_norm_mkl(tb):
    """test/unitest_mkl.cpp:15-40 on the B200 backend."""
    torch, cb = tb
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, 1, 1, 1, 1)
    x = dev(torch, np.full(1000, 10 + 10j, np.complex64))
    assert impl.MergeAddData(x, x, 0.5, 0.5, 1000)
    assert impl.Sync()
    np.testing.assert_array_equal(host(x), np.full(1000, 10 + 10j, np.complex64))
    assert impl.Normalization(x, 10, 1000)
    assert impl.Sync()
    np.testing.assert_array_equal(host(x), np.full(1000, 1 + 1j, np.complex64))


def test_kat_merge_norm_cuda_managed(tb):
    """test/unitest_cuda.cu:13-41: managed memory written and read by the host."""
    torch, cb = tb
    import ctypes
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, 1, 1, 1, 1)
    p = impl.alloc(8 * 10, managed=True)
    buf = (ctypes.c_float * 20).from_address(p)
    for i in range(20):
        buf[i] = 10.0
    assert impl.MergeAddData(p, p, 1, 1, 10)
    assert impl.Sync()
    assert all(buf[i] == 20.0 for i in range(20))
    assert impl.Normalization(p, 20, 10)
    assert impl.Sync()
    assert all(buf[i] == 1.0 for i in range(20))
    assert impl.free(p)


def test_kat_initialize(tb):
    """test/unitest_cuda.cu:4-11 (values in [0, 1]) plus determinism per seed."""
    torch, cb = tb
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, 1, 1, 1, 1)
    a = torch.full((1000,), -1.0, device="cuda")
    assert impl.Initialize(a, 1000) and impl.Sync()
    v = host(a)
    assert np.all((v >= 0) & (v <= 1)) and v.std() > 0.2
    impl2 = cb.NewCpraImpl(cb.IMPL_TYPE.B200, 1, 1, 1, 1)
    b = torch.zeros(1000, device="cuda")
    impl2.Initialize(b, 1000); impl2.Sync()
    np.testing.assert_array_equal(v, host(b))
    assert not impl.Initialize(a, 0)


def test_kat_2d_dft_double(tb):
    """test/unitest_mkl.cpp:42-71 (10x10 ones, double, 1e-14)."""
    torch, cb = tb
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, 10, 10, 1, 1, dtype="float64")
    x = dev(torch, np.ones(100, np.complex128))
    assert impl.Forward2D(x) and impl.Sync()
    want = np.zeros(100, np.complex128)
    want[55] = 100
    assert np.max(np.abs(host(x) - want)) <= 1e-14
    assert impl.Backward2D(x) and impl.Sync()
    assert np.max(np.abs(host(x) - 1)) <= 1e-14


# ---- transforms --------------------------------------------------------------------
@pytest.mark.parametrize("tag,T,M,N,B", [("f32_64", np.float32, 64, 64, 2), ("f64_32", np.float64, 32, 32, 2),
                                         ("f32_128", np.float32, 128, 128, 1), ("f32_16x8", np.float32, 16, 8, 3)])
def test_transforms_vs_reference(tb, tag, T, M, N, B):
    torch, cb = tb
    tol = FP32_FFT_TOL if T == np.float32 else 1e-13
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, 1, B, dtype=np.dtype(T).name)
    x = G[f"{tag}_x"]
    y = dev(torch, x)
    assert impl.Forward2D(y) and impl.Sync()
    assert O.rel_l2(host(y), G[f"{tag}_fwd"]) < tol
    y = dev(torch, x)
    assert impl.Backward2D(y) and impl.Sync()
    assert O.rel_l2(host(y), G[f"{tag}_bwd"]) < tol
    y = dev(torch, x)
    assert impl.FFTShift2D(y, M, N, B) and impl.Sync()
    np.testing.assert_array_equal(host(y), G[f"{tag}_shift"])


@pytest.mark.parametrize("M,N,B", [(256, 256, 2), (512, 512, 1), (64, 256, 2), (160, 160, 1), (2, 4, 3)])
def test_transforms_other_sizes_vs_oracle(tb, M, N, B):
    torch, cb = tb
    rng = np.random.default_rng(M * 1000 + N)
    x = (rng.standard_normal(M * N * B) + 1j * rng.standard_normal(M * N * B)).astype(np.complex64)
    o = O.OracleImpl(np.float32, M, N, 1, B)
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, 1, B)
    tol = FP32_FFT_TOL * (4 if max(M, N) > 128 else 1) * (20 if (M & (M - 1)) else 1)
    for fn in ("Forward2D", "Backward2D"):
        a = x.copy(); getattr(o, fn)(a)
        y = dev(torch, x)
        assert getattr(impl, fn)(y) and impl.Sync()
        assert O.rel_l2(host(y), a) < tol, fn


def test_forward_backward_roundtrip_large(tb):
    """Size-independent property at the full pattern size of the 512^2 case."""
    torch, cb = tb
    M = N = 512
    B = 4
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, 1, B)
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn(M * N * B, dtype=torch.complex64, device="cuda", generator=g)
    y = x.clone()
    assert impl.Forward2D(y) and impl.Backward2D(y) and impl.Sync()
    assert (torch.linalg.vector_norm(y - x) / torch.linalg.vector_norm(x)).item() < 2e-6
    # Parseval: ||F x||^2 = MN ||x||^2
    y = x.clone()
    impl.Forward2D(y); impl.Sync()
    r = (torch.linalg.vector_norm(y) ** 2 / (M * N * torch.linalg.vector_norm(x) ** 2)).item()
    assert abs(r - 1) < 1e-5


def test_shift3d_vs_reference(tb):
    torch, cb = tb
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, 6, 8, 4, 2)
    y = dev(torch, G["shift3d_x"])
    assert impl.FFTShift3D(y, 6, 8, 4, 2) and impl.Sync()
    np.testing.assert_array_equal(host(y), G["shift3d_out"])


@pytest.mark.parametrize("T,n,B", [(np.float32, 8, 2), (np.float32, 32, 1), (np.float32, 128, 1),
                                   (np.float64, 16, 1), (np.float32, 10, 1)])
def test_transforms_3d_vs_oracle(tb, T, n, B):
    torch, cb = tb
    rng = np.random.default_rng(n)
    C = O.complex_dtype(T)
    x = (rng.standard_normal(n ** 3 * B) + 1j * rng.standard_normal(n ** 3 * B)).astype(C)
    o = O.OracleImpl(T, n, n, n, B)
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, n, n, n, B, dtype=np.dtype(T).name)
    tol = (5e-6 if n % 2 == 0 and (n & (n - 1)) == 0 else 2e-5) if T == np.float32 else 1e-13
    for fn in ("Forward3D", "Backward3D"):
        a = x.copy(); getattr(o, fn)(a)
        y = dev(torch, x)
        assert getattr(impl, fn)(y) and impl.Sync()
        assert O.rel_l2(host(y), a) < tol, fn


# ---- element-wise operators ----------------------------------------------------------
def test_elementwise_vs_reference(tb):
    torch, cb = tb
    M = N = 32
    B = 3
    num = M * N * B
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, 1, B)
    x = G["ew_x"]
    A, S, Cc = dev(torch, G["ew_A"]), dev(torch, G["ew_S"]), dev(torch, G["ew_C"])
    y = dev(torch, x); assert impl.SpaceConstraint(y, S, num, B) and impl.Sync()
    np.testing.assert_array_equal(host(y), G["ew_sc"])
    y = dev(torch, x); assert impl.DataConstraint(y, Cc, num, B) and impl.Sync()
    np.testing.assert_array_equal(host(y), G["ew_dc_complex"])
    beta = np.float32(0.9)
    y = dev(torch, x)
    assert impl.MergeAddData(dev(torch, G["ew_src"]), y, -1.0 / beta, 1.0 + 1.0 / beta, num) and impl.Sync()
    np.testing.assert_array_equal(host(y), G["ew_merge"])
    y = dev(torch, x); assert impl.Normalization(y, 3.0, num) and impl.Sync()
    np.testing.assert_array_equal(host(y), G["ew_norm3"])
    y = dev(torch, x); assert impl.DataConstraint(y, A, num, B) and impl.Sync()
    got, ref = host(y), G["ew_dc_real"]
    assert np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-30)) < 4e-7
    Af = np.tile(G["ew_A"], B)
    np.testing.assert_array_equal(got[Af == 0], x[Af == 0])
    assert got[5] == 0


def test_elementwise_cuda_modes(tb):
    """The reference CUDA kernels' semantics behind the mode options
    (CUDA_Impl_Kernel.cuh:16-38)."""
    torch, cb = tb
    M = N = 32
    B = 3
    num = M * N * B
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, 1, B)
    assert impl.set_option(cb.OPT_SPACE_MODE, 1) and impl.set_option(cb.OPT_DATA_MODE, 1)
    o = O.OracleImpl(np.float32, M, N, 1, B, space_mode="cuda")
    x = G["ew_x"]
    a = x.copy(); o.SpaceConstraint(a, G["ew_S"], num, B)
    y = dev(torch, x); impl.SpaceConstraint(y, dev(torch, G["ew_S"]), num, B); impl.Sync()
    np.testing.assert_array_equal(host(y), a)
    y = dev(torch, x); impl.DataConstraint(y, dev(torch, G["ew_A"]), num, B); impl.Sync()
    got = host(y)
    Af = np.tile(G["ew_A"], B)
    nz = (Af == 0) & (np.abs(x) > 0)
    assert np.all(got[nz] == 0)   # no A == 0 skip: polar(0, arg z) = 0


def test_argument_errors(tb):
    torch, cb = tb
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, 8, 8, 1, 2)
    x = torch.zeros(128, dtype=torch.complex64, device="cuda")
    s = torch.zeros(64, device="cuda")
    assert not impl.MergeAddData(x, x, 0.0, 1.0, 128)
    assert not impl.MergeAddData(x, x, 1.0, 1.0, 0)
    assert not impl.Normalization(x, 0.0, 128)
    assert not impl.SpaceConstraint(x, s, 0, 2)
    assert not impl.SpaceConstraint(x, s, 128, 0)
    assert not impl.DataConstraint(x, s, 1, 2)      # empty plane
    assert not impl.FFTShift2D(x, 7, 8, 1)          # odd: not a shift in the reference either
    assert not impl.Initialize(s, 0)
    assert impl.Sync()
    odd = cb.NewCpraImpl(cb.IMPL_TYPE.B200, 7, 8, 1, 1)
    with pytest.raises(cb.CpraB200Error):
        odd.Forward2D(x)


def test_merge_broadcast_ragged_batch(tb):
    """num not a multiple of batch: element i uses plane element i % (num/batch)."""
    torch, cb = tb
    rng = np.random.default_rng(11)
    num, batch = 1000, 3
    x = (rng.standard_normal(num) + 1j * rng.standard_normal(num)).astype(np.complex64)
    S = rng.uniform(0, 1, num // batch).astype(np.float32)
    o = O.OracleImpl(np.float32, 1, 1, 1, 1)
    a = x.copy(); o.SpaceConstraint(a, S, num, batch)
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, 1, 1, 1, 1)
    y = dev(torch, x); impl.SpaceConstraint(y, dev(torch, S), num, batch); impl.Sync()
    np.testing.assert_array_equal(host(y), a)


# ---- difference-map iterations --------------------------------------------------------
def dm_per_call(impl, x, t1, t2, A, S, num, B, beta):
    """src/CPRA_MKL.cpp:94-110, one interface call at a time."""
    b = float(np.float32(beta))
    impl.Forward2D(t1)
    impl.DataConstraint(t1, A, num, B)
    impl.Backward2D(t1)
    impl.MergeAddData(x, t1, -1.0 / b, 1.0 + 1.0 / b, num)
    impl.SpaceConstraint(t1, S, num, B)
    impl.SpaceConstraint(t2, S, num, B)
    impl.MergeAddData(x, t2, 1.0 / b, 1.0 - 1.0 / b, num)
    impl.Forward2D(t2)
    impl.DataConstraint(t2, A, num, B)
    impl.Backward2D(t2)
    impl.MergeAddData(t1, x, b, 1.0, num)
    impl.MergeAddData(t2, x, -1.0 * b, 1.0, num)


@pytest.mark.parametrize("iters", [1, 5])
@pytest.mark.parametrize("fusion", [0, 1])
def test_dm_iterations_vs_reference(tb, iters, fusion):
    torch, cb = tb
    M = N = 64
    B = 2
    num = M * N * B
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, 1, B)
    impl.set_option(cb.OPT_FUSION, fusion)
    x, t1, t2 = (dev(torch, G["dm_x0"]) for _ in range(3))
    A, S = dev(torch, G["dm_A"]), dev(torch, G["dm_S"])
    for _ in range(iters):
        dm_per_call(impl, x, t1, t2, A, S, num, B, 0.9)
    assert impl.Sync()
    for name, v in (("x", x), ("t1", t1), ("t2", t2)):
        assert O.rel_l2(host(v), G[f"dm{iters}_{name}"]) < FP32_DM_TOL * iters, name


@pytest.mark.parametrize("L,B,iters", [(128, 3, 4), (64, 5, 3), (32, 2, 6), (256, 2, 3), (512, 1, 2)])
def test_fused_equals_per_call_bitwise(tb, L, B, iters):
    """One fused launch, the recorder-fused call stream and the per-call kernels
    write identical bits."""
    torch, cb = tb
    rng = np.random.default_rng(L + B)
    num = L * L * B
    amps = (rng.uniform(0, 40, L * L) * (rng.uniform(0, 1, L * L) > 0.1)).astype(np.float32)
    sup = (rng.uniform(0, 1, L * L) > 0.5).astype(np.float32)
    x0 = (rng.uniform(0, 1, num) + 1j * rng.uniform(0, 1, num)).astype(np.complex64)
    outs = []
    for mode in ("per_call", "recorded", "dm_api"):
        impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
        impl.set_option(cb.OPT_FUSION, 0 if mode == "per_call" else 1)
        x, t1, t2 = (dev(torch, x0) for _ in range(3))
        A, S = dev(torch, amps), dev(torch, sup)
        if mode == "dm_api":
            assert impl.dm_iterations(x, t1, t2, A, S, B, 0.9, iters)
        else:
            for _ in range(iters):
                dm_per_call(impl, x, t1, t2, A, S, num, B, 0.9)
        assert impl.Sync()
        outs.append([host(v) for v in (x, t1, t2)])
    for k in (1, 2):
        for a, b in zip(outs[0], outs[k]):
            np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("L,B,iters", [(256, 2, 3), (512, 1, 2)])
def test_dm_large_vs_oracle(tb, L, B, iters):
    """The 256 / 512 line-pass iterations against the float64-inside oracle:
    <= 1e-5 relative L2 per iteration for x, t1 and t2."""
    torch, cb = tb
    rng = np.random.default_rng(L)
    num = L * L * B
    amps = (rng.uniform(0, 40, L * L) * (rng.uniform(0, 1, L * L) > 0.1)).astype(np.float32)
    sup = (rng.uniform(0, 1, L * L) > 0.5).astype(np.float32)
    x0 = (rng.uniform(0, 1, num) + 1j * rng.uniform(0, 1, num)).astype(np.complex64)
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    x, t1, t2 = (dev(torch, x0) for _ in range(3))
    assert impl.dm_iterations(x, t1, t2, dev(torch, amps), dev(torch, sup), B, 0.9, iters) and impl.Sync()
    o = O.OracleImpl(np.float32, L, L, 1, B)
    xo, t1o, t2o = x0.copy(), x0.copy(), x0.copy()
    for _ in range(iters):
        O.dm_iteration(o, xo, t1o, t2o, amps, sup, num, B, 0.9)
    for got, want in ((x, xo), (t1, t1o), (t2, t2o)):
        assert O.rel_l2(host(got), want) < FP32_DM_TOL * iters


@pytest.mark.parametrize("L,B,iters", [(64, 4, 3), (256, 2, 2)])
def test_fused_per_pattern_constraints(tb, L, B, iters):
    """dm_iterations with per-pattern modulus/support planes equals running each
    pattern on its own with a shared plane."""
    torch, cb = tb
    rng = np.random.default_rng(5)
    A = rng.uniform(0, 10, (B, L * L)).astype(np.float32)
    S = (rng.uniform(0, 1, (B, L * L)) > 0.4).astype(np.float32)
    x0 = (rng.uniform(0, 1, (B, L * L)) + 1j * rng.uniform(0, 1, (B, L * L))).astype(np.complex64)
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    x, t1, t2 = (dev(torch, x0.ravel()) for _ in range(3))
    assert impl.dm_iterations(x, t1, t2, dev(torch, A.ravel()), dev(torch, S.ravel()), B, 0.9, iters,
                              a_stride=L * L, s_stride=L * L) and impl.Sync()
    one = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, 1)
    for b in range(B):
        xb, t1b, t2b = (dev(torch, x0[b]) for _ in range(3))
        one.dm_iterations(xb, t1b, t2b, dev(torch, A[b]), dev(torch, S[b]), 1, 0.9, iters)
        one.Sync()
        np.testing.assert_array_equal(host(xb), host(x)[b * L * L:(b + 1) * L * L])


def cpra_driver(impl, torch, M, N, L, P, B, A, S, x, epi, iters, pre_iter, beta, err):
    """src/CPRA_MKL.cpp:35-140 issued through the interface, unchanged."""
    MNB = M * N * B
    t1 = torch.empty(MNB, dtype=x.dtype, device=x.device)
    t2 = torch.empty_like(t1)
    old = torch.empty_like(t1)
    nb = MNB * x.element_size()
    b = float(np.float32(beta))
    impl.Memcpy(t1, x, nb)
    impl.Memcpy(t2, x, nb)
    for _ in range(pre_iter):
        dm_per_call(impl, x[:MNB], t1, t2, A, S, MNB, B, beta)
    impl.Sync()
    for e in range(epi):
        for p in range(P):
            xp = x[MNB * p: MNB * (p + 1)]
            if p == P - 1:
                impl.MergeAddData(x[MNB * (p - 1): MNB * p], xp, 0.5, 0.5, MNB)
            elif p == 0:
                impl.MergeAddData(x[MNB * (p + 1): MNB * (p + 2)], xp, 0.5, 0.5, MNB)
            else:
                impl.MergeAddData(x[MNB * (p - 1): MNB * p], xp, 0.5, 0, MNB)
                impl.MergeAddData(x[MNB * (p + 1): MNB * (p + 2)], xp, 0.5, 1, MNB)
            impl.Memcpy(t1, xp, nb)
            impl.Memcpy(t2, xp, nb)
            Ap, Sp = A[M * N * p: M * N * (p + 1)], S[M * N * p: M * N * (p + 1)]
            for i in range(iters):
                last = (i == iters - 1 and e == epi - 1)
                if last:
                    impl.Memcpy(old, xp, nb)
                dm_per_call(impl, xp, t1, t2, Ap, Sp, MNB, B, beta)
                if last:
                    impl.Memcpy(t1, xp, nb)
                    impl.Forward2D(old)
                    impl.Forward2D(t1)
                    impl.ConvergeError(old, t1, err[B * p: B * (p + 1)], M, N, 1, B)
    for p in range(P):
        xp = x[MNB * p: MNB * (p + 1)]
        Ap, Sp = A[M * N * p: M * N * (p + 1)], S[M * N * p: M * N * (p + 1)]
        impl.Memcpy(t1, xp, nb)
        impl.Forward2D(t1)
        impl.DataConstraint(t1, Ap, MNB, B)
        impl.Backward2D(t1)
        impl.MergeAddData(xp, t1, -1.0 / b, 1.0 + 1.0 / b, MNB)
        impl.SpaceConstraint(t1, Sp, MNB, B)
        impl.Memcpy(xp, t1, nb)
    impl.Sync()


@pytest.mark.parametrize("fusion", [0, 1])
def test_cpra_episode_driver_vs_reference(tb, fusion):
    torch, cb = tb
    M, N, L, P, B, epi, it, pre = (int(v) for v in G["cpra_cfg"])
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, L, B)
    impl.set_option(cb.OPT_FUSION, fusion)
    x = dev(torch, G["cpra_x0"])
    err = np.zeros(P * B, np.float32)
    cpra_driver(impl, torch, M, N, L, P, B, dev(torch, G["cpra_A"]), dev(torch, G["cpra_S"]), x, epi, it, pre,
                0.9, err)
    assert O.rel_l2(host(x), G["cpra_x"]) < 1e-3
    _, err_o = O.cpra_sample(np.float32, M, N, L, P, B, G["cpra_A"], G["cpra_S"], G["cpra_x0"], epi, it, pre, 0.9)
    assert np.all(np.isfinite(err)) and np.max(np.abs(err - err_o) / np.abs(err_o)) < 1e-2


def test_converge_error_vs_oracle(tb):
    torch, cb = tb
    rng = np.random.default_rng(2)
    M, N, L, B = 16, 16, 4, 3
    n = M * N * L * B
    old = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    new = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    o = O.OracleImpl(np.float32, M, N, L, B)
    a = old.copy(); err_o = np.zeros(B, np.float32)
    o.ConvergeError(a, new, err_o, M, N, L, B)
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, L, B)
    y = dev(torch, old)
    err = np.zeros(B, np.float32)
    assert impl.ConvergeError(y, dev(torch, new), err, M, N, L, B)
    np.testing.assert_array_equal(host(y), a)     # old <- new - old, element-wise exact
    np.testing.assert_allclose(err, err_o, rtol=1e-6)


def test_real2d_to_3d_vs_oracle(tb):
    torch, cb = tb
    rng = np.random.default_rng(9)
    M = N = L = 32
    P = 12
    src = rng.uniform(0, 1, P * M * N).astype(np.float32)
    ang = np.deg2rad(np.linspace(0, 165, P)).astype(np.float32)
    want = O.real2d_to_3d(np.float32, src, ang, M, N, P, L)
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, L, 1)
    dst = torch.zeros(M * N * L, device="cuda")
    assert impl.Real2DTo3DInterpolation(dev(torch, src), dst, dev(torch, ang), M, N, P, L) and impl.Sync()
    got = host(dst)
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-6)
    assert (want != 0).sum() > 0.05 * want.size


@pytest.mark.parametrize("L,P,B,epi,it,pre", [(32, 4, 2, 2, 3, 4), (128, 5, 3, 2, 3, 2), (64, 3, 2, 1, 1, 0),
                                              (256, 3, 2, 2, 2, 1)])
def test_cpra_run_equals_driver_bitwise(tb, L, P, B, epi, it, pre):
    """cpra_b200_cpra_run (carousel mix and t1 = t2 = x fused into each angle's
    launch) writes the same bits as the reference driver's call sequence issued
    one call at a time (src/CPRA_MKL.cpp:35-140)."""
    torch, cb = tb
    rng = np.random.default_rng(L * 7 + P)
    A = (rng.uniform(0, 30, (P, L * L)) * (rng.uniform(0, 1, (P, L * L)) > 0.1)).astype(np.float32)
    S = (rng.uniform(0, 1, (P, L * L)) > 0.45).astype(np.float32)
    x0 = (rng.uniform(0, 1, P * B * L * L) + 1j * rng.uniform(0, 1, P * B * L * L)).astype(np.complex64)
    Ad, Sd = dev(torch, A.ravel()), dev(torch, S.ravel())
    ref = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    ref.set_option(cb.OPT_FUSION, 0)
    xr = dev(torch, x0)
    err_r = np.zeros(P * B, np.float32)
    cpra_driver(ref, torch, L, L, 1, P, B, Ad, Sd, xr, epi, it, pre, 0.9, err_r)
    run = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    xf = dev(torch, x0)
    err_f = np.zeros(P * B, np.float32)
    assert run.cpra_run(xf, Ad, Sd, P, B, epi, it, pre, 0.9, final_step=True, err=err_f) and run.Sync()
    np.testing.assert_array_equal(host(xf), host(xr))
    np.testing.assert_array_equal(err_f, err_r)


def test_cpra_run_vs_reference(tb):
    torch, cb = tb
    M, N, L, P, B, epi, it, pre = (int(v) for v in G["cpra_cfg"])
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, L, B)
    x = dev(torch, G["cpra_x0"])
    assert impl.cpra_run(x, dev(torch, G["cpra_A"]), dev(torch, G["cpra_S"]), P, B, epi, it, pre, 0.9) and impl.Sync()
    assert O.rel_l2(host(x), G["cpra_x"]) < 1e-3
    # argument errors of the driver entry
    assert not impl.cpra_run(x, dev(torch, G["cpra_A"]), dev(torch, G["cpra_S"]), 1, B, epi, it, pre, 0.9)
    assert not impl.cpra_run(x, dev(torch, G["cpra_A"]), dev(torch, G["cpra_S"]), P, B + 1, epi, it, pre, 0.9)


@pytest.mark.parametrize("L,P,B,epi,it,pre,final,pinned,dtype",
                         [(64, 4, 2, 2, 3, 1, True, True, "float32"), (128, 5, 3, 1, 2, 0, True, False, "float32"),
                          (256, 3, 2, 2, 2, 1, False, True, "float32"), (32, 3, 2, 0, 2, 2, True, True, "float32"),
                          (32, 4, 2, 2, 2, 1, True, True, "float64")])
def test_cpra_run_host_bitwise(tb, L, P, B, epi, it, pre, final, pinned, dtype):
    """cpra_b200_cpra_run_host (per-angle uploads overlapped with the first
    episode, per-angle read-back after the final projection) writes the same
    bits and the same errors as cpra_b200_cpra_run on device buffers, twice in
    a row on one context, from pinned or pageable host memory."""
    torch, cb = tb
    rdt, cdt = (np.float32, np.complex64) if dtype == "float32" else (np.float64, np.complex128)
    rng = np.random.default_rng(L + 11 * P + epi)
    A = (rng.uniform(0, 30, (P, L * L)) * (rng.uniform(0, 1, (P, L * L)) > 0.1)).astype(rdt)
    S = (rng.uniform(0, 1, (P, L * L)) > 0.45).astype(rdt)
    x0 = (rng.uniform(0, 1, P * B * L * L) + 1j * rng.uniform(0, 1, P * B * L * L)).astype(cdt)
    ref = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B, dtype)
    xr = dev(torch, x0)
    err_r = np.zeros(P * B, rdt)
    assert ref.cpra_run(xr, dev(torch, A.ravel()), dev(torch, S.ravel()), P, B, epi, it, pre, 0.9,
                        final_step=final, err=err_r if epi else None) and ref.Sync()
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B, dtype)

    def hbuf(a):
        t = torch.from_numpy(np.ascontiguousarray(a).view(rdt).copy())
        return t.pin_memory() if pinned else t

    Ah, Sh = hbuf(A.ravel()), hbuf(S.ravel())
    for _ in range(2):
        xh = hbuf(x0)
        err = np.zeros(P * B, rdt)
        assert impl.cpra_run_host(xh, Ah, Sh, P, B, epi, it, pre, 0.9, final_step=final, err=err if epi else None)
        np.testing.assert_array_equal(xh.numpy().view(cdt), host(xr))
        np.testing.assert_array_equal(err, err_r)
    assert not impl.cpra_run_host(hbuf(x0), Ah, Sh, 1, B, epi, it, pre, 0.9)
    assert not impl.cpra_run_host(hbuf(x0), Ah, Sh, P, B + 1, epi, it, pre, 0.9)


@pytest.mark.parametrize("L,P,B,epi,it,pre,lanes,final,dtype",
                         [(64, 7, 2, 3, 2, 1, 2, True, "float32"), (64, 6, 3, 4, 3, 0, 3, False, "float32"),
                          (32, 5, 2, 5, 2, 1, 0, True, "float32"), (128, 3, 2, 4, 2, 1, 4, True, "float32"),
                          (256, 5, 2, 3, 2, 1, 2, True, "float32"), (512, 3, 1, 2, 2, 0, 0, True, "float32"),
                          (32, 4, 2, 3, 2, 1, 2, True, "float64"), (64, 3, 2, 0, 2, 1, 4, True, "float32"),
                          (64, 3, 2, 1, 2, 1, 4, True, "float32")])
def test_cpra_run_lanes_bitwise(tb, L, P, B, epi, it, pre, lanes, final, dtype):
    """cpra_run's wavefront schedule (episode e on lane e mod W, angle p of
    episode e beside angle p-2 of episode e+1) writes the same bits and the
    same errors as one stream taking the angles in order: directly, replayed
    from a CUDA graph, and through the host-buffer entry."""
    torch, cb = tb
    rdt, cdt = (np.float32, np.complex64) if dtype == "float32" else (np.float64, np.complex128)
    rng = np.random.default_rng(L + 3 * P + 17 * epi)
    A = (rng.uniform(0, 30, (P, L * L)) * (rng.uniform(0, 1, (P, L * L)) > 0.1)).astype(rdt)
    S = (rng.uniform(0, 1, (P, L * L)) > 0.45).astype(rdt)
    x0 = (rng.uniform(0, 1, P * B * L * L) + 1j * rng.uniform(0, 1, P * B * L * L)).astype(cdt)
    Ad, Sd = dev(torch, A.ravel()), dev(torch, S.ravel())
    ref = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B, dtype)
    assert ref.set_option(cb.OPT_LANES, 1)
    xr = dev(torch, x0)
    err_r = np.zeros(P * B, rdt)
    assert ref.cpra_run(xr, Ad, Sd, P, B, epi, it, pre, 0.9, final_step=final, err=err_r) and ref.Sync()
    run = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B, dtype)
    assert run.set_option(cb.OPT_LANES, lanes)
    for graph in (0, 1, 1):
        assert run.set_option(cb.OPT_GRAPH, graph)
        x = dev(torch, x0)
        err = np.zeros(P * B, rdt)
        assert run.cpra_run(x, Ad, Sd, P, B, epi, it, pre, 0.9, final_step=final, err=err) and run.Sync()
        np.testing.assert_array_equal(host(x), host(xr))
        np.testing.assert_array_equal(err, err_r)
    assert run.set_option(cb.OPT_GRAPH, 0)
    xh = torch.from_numpy(x0.view(rdt).copy()).pin_memory()
    err = np.zeros(P * B, rdt)
    assert run.cpra_run_host(xh, torch.from_numpy(A.ravel().copy()).pin_memory(),
                             torch.from_numpy(S.ravel().copy()).pin_memory(), P, B, epi, it, pre, 0.9,
                             final_step=final, err=err)
    np.testing.assert_array_equal(xh.numpy().view(cdt), host(xr))
    np.testing.assert_array_equal(err, err_r)
    assert not run.set_option(cb.OPT_LANES, 17)


@pytest.mark.parametrize("L,P,B,epi", [(64, 6, 3, 5), (256, 3, 2, 3)])
def test_cpra_run_autotune_bitwise(tb, L, P, B, epi):
    """CPRA_B200_OPT_AUTOTUNE: the first run of a key times the lane counts
    on a copy of x and caches the fastest.  The tuning run, a later run (which
    launches only its own kernels) and a host-buffer run all write the bits
    and errors of one stream taking the angles in order."""
    torch, cb = tb
    it, pre = 2, 1
    rng = np.random.default_rng(L + P + epi)
    A = (rng.uniform(0, 30, (P, L * L)) * (rng.uniform(0, 1, (P, L * L)) > 0.1)).astype(np.float32)
    S = (rng.uniform(0, 1, (P, L * L)) > 0.45).astype(np.float32)
    x0 = (rng.uniform(0, 1, P * B * L * L) + 1j * rng.uniform(0, 1, P * B * L * L)).astype(np.complex64)
    Ad, Sd = dev(torch, A.ravel()), dev(torch, S.ravel())
    ref = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    assert ref.set_option(cb.OPT_LANES, 1)
    xr, err_r = dev(torch, x0), np.zeros(P * B, np.float32)
    assert ref.cpra_run(xr, Ad, Sd, P, B, epi, it, pre, 0.9, final_step=True, err=err_r) and ref.Sync()
    run = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    assert run.get_option(cb.OPT_AUTOTUNE) == 0
    assert run.set_option(cb.OPT_AUTOTUNE, 1) and run.get_option(cb.OPT_AUTOTUNE) == 1
    launched = []
    for _ in range(2):
        x, err = dev(torch, x0), np.zeros(P * B, np.float32)
        n0 = cb.kernels_launched()
        assert run.cpra_run(x, Ad, Sd, P, B, epi, it, pre, 0.9, final_step=True, err=err) and run.Sync()
        launched.append(cb.kernels_launched() - n0)
        np.testing.assert_array_equal(host(x), host(xr))
        np.testing.assert_array_equal(err, err_r)
        assert 1 <= run.get_option(cb.OPT_LANES) <= 16
    assert launched[1] < launched[0]  # the first run also ran the trials
    xh = torch.from_numpy(x0.view(np.float32).copy()).pin_memory()
    err = np.zeros(P * B, np.float32)
    assert run.cpra_run_host(xh, torch.from_numpy(A.ravel().copy()).pin_memory(),
                             torch.from_numpy(S.ravel().copy()).pin_memory(), P, B, epi, it, pre, 0.9,
                             final_step=True, err=err)
    np.testing.assert_array_equal(xh.numpy().view(np.complex64), host(xr))
    np.testing.assert_array_equal(err, err_r)


@pytest.mark.parametrize("name", ["drop_in_standalone", "drop_in_ref_iface"])
def test_cpp_drop_in_driver(tb, tmp_path, name):
    """The reference driver's call sequence through CpraImpl<float>* on
    B200Impl<float> (C++, managed memory, recorder fusion on) writes the same
    bits as the per-call Python driver, and matches the reference build."""
    import subprocess
    from conftest import REPO
    torch, cb = tb
    exe = REPO / "tests" / "cpp" / "_bin" / name
    # build() compiles both drivers (the second against the reference's own
    # interface header); a missing binary is a failure, not a vanished test
    assert exe.exists(), f"{exe} is not built (python tests/cpp/build.py)"
    M, N, L, P, B, epi, it, pre = (int(v) for v in G["cpra_cfg"])
    (tmp_path / "cfg.txt").write_text(f"{M} {N} {L} {P} {B} {epi} {it} {pre} 0.9\n")
    G["cpra_A"].astype(np.float32).tofile(tmp_path / "A.f32")
    G["cpra_S"].astype(np.float32).tofile(tmp_path / "S.f32")
    G["cpra_x0"].astype(np.complex64).tofile(tmp_path / "x0.c64")
    out = tmp_path / "out.bin"
    r = subprocess.run([str(exe), str(tmp_path), str(out)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    raw = np.fromfile(out, dtype=np.uint8)
    nx = P * B * M * N
    x = raw[: nx * 8].view(np.complex64)
    err = raw[nx * 8:].view(np.float32)
    ref = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, L, B)
    ref.set_option(cb.OPT_FUSION, 0)
    xr = dev(torch, G["cpra_x0"])
    err_r = np.zeros(P * B, np.float32)
    cpra_driver(ref, torch, M, N, L, P, B, dev(torch, G["cpra_A"]), dev(torch, G["cpra_S"]), xr, epi, it, pre, 0.9,
                err_r)
    np.testing.assert_array_equal(x, host(xr))
    np.testing.assert_array_equal(err, err_r)
    assert O.rel_l2(x, G["cpra_x"]) < 1e-3


@pytest.mark.parametrize("L,B,shared", [(128, 3, True), (64, 4, False), (160, 2, False)])
def test_rfactor_vs_oracle(tb, L, B, shared):
    """Project-defined R-factor (FP64 sums on the GPU) against the float64 oracle."""
    torch, cb = tb
    rng = np.random.default_rng(L + B)
    x = (rng.standard_normal(B * L * L) + 1j * rng.standard_normal(B * L * L)).astype(np.complex64)
    A = rng.uniform(0, 20, (1 if shared else B) * L * L).astype(np.float32)
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    xd = dev(torch, x)
    r = impl.rfactor(xd, dev(torch, A), B, a_stride=0 if shared else L * L)
    want = O.rfactor(x, A, L, L, B, a_stride=0 if shared else L * L)
    np.testing.assert_allclose(r, want, rtol=1e-5)
    np.testing.assert_array_equal(host(xd), x)   # input untouched


@pytest.mark.parametrize("M,P,tol", [(24, 10, 1e-5), (64, 40, 1e-4), (18, 12, 1e-5)])
def test_complex_merge_vs_oracle(tb, M, P, tol):
    """Project-defined trilinear gather merge (Complex2DTo3DInterpolation)
    against the float64 oracle.  Coordinates and weights are float: their
    rounding (about M/2 * 2^-23 absolute) bounds the relative L2 error at
    1e-5 for 24^3 and 1e-4 for 64^3.  At 24^3 and 64^3 a work item is four
    voxels along the tilt axis; 18 is no multiple of 4, so 18^3 runs one
    voxel per item."""
    torch, cb = tb
    rng = np.random.default_rng(21)
    N = L = M
    src = (rng.standard_normal(P * M * N) + 1j * rng.standard_normal(P * M * N)).astype(np.complex64)
    ang = np.deg2rad(np.linspace(0, 170, P) + 0.37).astype(np.float32)
    want = O.complex2d_to_3d(np.float32, src, ang, M, N, P, L)
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, L, 1)
    dst = torch.zeros(M * N * L, dtype=torch.complex64, device="cuda")
    assert impl.Complex2DTo3DInterpolation(dev(torch, src), dst, dev(torch, ang), M, N, P, L) and impl.Sync()
    got = host(dst)
    assert O.rel_l2(got, want) < tol
    assert (np.abs(want) > 0).mean() > 0.3


# ---- hybrid input-output with shrinkwrap (project-defined) -----------------------------
def _hio_inputs(L, B, seed):
    from cpra_b200 import synth
    d = synth.patterns_2d(count=B, n=L, radius=int(0.19 * L), seed=seed)
    S0 = synth.autocorrelation_support(d["A"])
    x0 = synth.random_phase_start(d["A"], seed=seed + 1)
    return d["A"], S0, x0


@pytest.mark.parametrize("L,B,iters,pos,tmem", [(64, 3, 1, False, 1), (64, 3, 5, False, 1), (128, 2, 3, True, 1),
                                                 (128, 2, 5, False, 0), (128, 3, 5, False, 1),
                                                 (256, 2, 3, False, 1), (512, 1, 2, True, 1)])
def test_hio_iterations_vs_oracle(tb, L, B, iters, pos, tmem):
    """HIO iterations (no support update) against the oracle, 1e-5 relative L2
    per iteration; at 128^2 both the tensor-memory kernel (tmem 1) and the
    L2 kernel (tmem 0), at 256^2 and 512^2 the line passes (the cluster
    kernel has its own tests below)."""
    torch, cb = tb
    A, S0, x0 = _hio_inputs(L, B, seed=L + iters)
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    assert impl.set_option(cb.OPT_TMEM, tmem) and impl.set_option(cb.OPT_HIO_CLUSTER, 0)
    x, S = dev(torch, x0.ravel()), dev(torch, S0.ravel())
    assert impl.hio_shrinkwrap(x, dev(torch, A.ravel()), S, B, iters, beta=0.9, sw_every=0, positivity=pos)
    assert impl.Sync()
    xo, So, _ = O.hio_shrinkwrap(x0, A, S0, L, B, iters, 0.9, sw_every=0, positivity=pos)
    assert O.rel_l2(host(x), xo) < FP32_DM_TOL * iters
    np.testing.assert_array_equal(host(S), So.astype(np.float32))   # no update: support unchanged


@pytest.mark.parametrize("L,tmem,cluster", [(32, 1, 0), (64, 1, 0), (128, 1, 0), (128, 0, 0), (128, 1, 8),
                                            (256, 1, 8)])
def test_hio_fused_split_calls_bitwise(tb, L, tmem, cluster):
    """The fused HIO kernels carry x on chip from one iteration to the next
    and write it to memory only after their last iteration: 7 iterations in
    one call equal 3 + 4 iterations in two calls (which restart from memory),
    bit for bit, with and without positivity; the one-CTA kernels and the
    cluster kernel (8 CTAs per pattern)."""
    torch, cb = tb
    B = 3
    A, S0, x0 = _hio_inputs(L, B, seed=L + 11)
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    assert impl.set_option(cb.OPT_TMEM, tmem) and impl.set_option(cb.OPT_HIO_CLUSTER, cluster)
    Ad = dev(torch, A.ravel())
    for pos in (False, True):
        x1, S1 = dev(torch, x0.ravel()), dev(torch, S0.ravel())
        assert impl.hio_shrinkwrap(x1, Ad, S1, B, 7, beta=0.9, sw_every=0, positivity=pos) and impl.Sync()
        x2, S2 = dev(torch, x0.ravel()), dev(torch, S0.ravel())
        assert impl.hio_shrinkwrap(x2, Ad, S2, B, 3, beta=0.9, sw_every=0, positivity=pos)
        assert impl.hio_shrinkwrap(x2, Ad, S2, B, 4, beta=0.9, sw_every=0, positivity=pos) and impl.Sync()
        assert torch.equal(torch.view_as_real(x1), torch.view_as_real(x2)), (L, pos)
        assert torch.equal(S1, S2)


def test_hio_shrinkwrap_support_vs_oracle(tb):
    """Support masks after shrinkwrap updates differ in <= 0.1% of pixels."""
    torch, cb = tb
    L, B = 128, 4
    A, S0, x0 = _hio_inputs(L, B, seed=3)
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    x, S = dev(torch, x0.ravel()), dev(torch, S0.ravel())
    assert impl.hio_shrinkwrap(x, dev(torch, A.ravel()), S, B, 20, beta=0.9, sw_every=10) and impl.Sync()
    xo, So, _ = O.hio_shrinkwrap(x0, A, S0, L, B, 20, 0.9, sw_every=10)
    diff = (host(S) != So.astype(np.float32)).mean()
    assert diff <= 1e-3, diff
    # HIO is chaotic and a support pixel that flips on the threshold separates
    # the trajectories, so x itself is only checked loosely here; the bars are
    # the support masks (above) and the R-factor after a full run (below)
    assert O.rel_l2(host(x), xo) < 5e-2


def test_hio_shrinkwrap_full_run_rfactor(tb):
    """The plain 2D configuration: 16 patterns of 128x128, HIO beta 0.9, 200
    iterations, shrinkwrap every 20 (sigma 3 -> 1.5, threshold 0.1), random
    phase starts.  The reconstruction (support times modulus projection of the
    final iterate) has a mean R-factor within 2% (relative) of the float64
    oracle's.  HIO from random starts is chaotic: the float64 oracle itself,
    started from the same starts perturbed by 1e-7 (relative, below float
    rounding), moves its 16-pattern mean R-factor by 0.1% to 1.6% (six
    perturbations), its per-pattern median difference by 1.1% to 2.5% and its
    worst pattern by 7% to 12%; single patterns of an FP32 run drift further
    (up to ~18% seen).  So the mean is bounded at 2%, the per-pattern median
    difference at 4% and the worst pattern at 25%."""
    torch, cb = tb
    L, B = 128, 16
    A, S0, x0 = _hio_inputs(L, B, seed=0)
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    x, S, Ad = dev(torch, x0.ravel()), dev(torch, S0.ravel()), dev(torch, A.ravel())
    est = torch.empty_like(x)
    assert impl.hio_shrinkwrap(x, Ad, S, B, 200, beta=0.9, sw_every=20, sigma_start=3.0, sigma_end=1.5,
                               threshold=0.1, estimate=est) and impl.Sync()
    r = impl.rfactor(est, Ad, B, a_stride=L * L)
    xo, So, eo = O.hio_shrinkwrap(x0, A, S0, L, B, 200, 0.9, sw_every=20, sigma_start=3.0, sigma_end=1.5,
                                  threshold=0.1)
    ro = O.rfactor(eo, A, L, L, B, a_stride=L * L)
    rel = np.abs(r - ro) / ro
    assert abs(r.mean() - ro.mean()) / ro.mean() < 0.02, (r, ro)
    assert np.median(rel) < 0.04 and np.max(rel) < 0.25, (r, ro)
    # the estimate is the modulus projection inside the final support, zero outside
    e = host(est).reshape(B, -1)
    assert np.all(e[host(S).reshape(B, -1) < 0.5] == 0)


# ---- 256 and 512: the same iteration as line passes over chunks of patterns --------------
def test_hio_large_chunking_is_exact(tb):
    """Patterns are independent, so the chunk size (patterns per pass) of the
    line passes must not change a bit of x, S or the estimate."""
    torch, cb = tb
    L, B = 256, 3
    A, S0, x0 = _hio_inputs(L, B, seed=7)
    out = []
    for chunk in (0, 1, 2):
        impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
        assert impl.set_option(cb.OPT_HIO_CHUNK, chunk) and impl.set_option(cb.OPT_HIO_CLUSTER, 0)
        x, S = dev(torch, x0.ravel()), dev(torch, S0.ravel())
        est = torch.empty_like(x)
        assert impl.hio_shrinkwrap(x, dev(torch, A.ravel()), S, B, 12, beta=0.9, sw_every=5, estimate=est)
        assert impl.Sync()
        out.append((host(x), host(S), host(est)))
    for o in out[1:]:
        for a, b in zip(out[0], o):
            np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("L,cluster", [(256, 0), (512, 0), (256, 8)])
def test_hio_large_shrinkwrap_support_vs_oracle(tb, L, cluster):
    """Support masks after shrinkwrap updates differ in <= 0.1% of pixels
    (line passes; at 256 also the cluster kernel, 8 CTAs per pattern)."""
    torch, cb = tb
    B = 2
    A, S0, x0 = _hio_inputs(L, B, seed=11)
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    assert impl.set_option(cb.OPT_HIO_CLUSTER, cluster)
    x, S = dev(torch, x0.ravel()), dev(torch, S0.ravel())
    assert impl.hio_shrinkwrap(x, dev(torch, A.ravel()), S, B, 20, beta=0.9, sw_every=10) and impl.Sync()
    xo, So, _ = O.hio_shrinkwrap(x0, A, S0, L, B, 20, 0.9, sw_every=10)
    diff = (host(S) != So.astype(np.float32)).mean()
    assert diff <= 1e-3, diff
    assert O.rel_l2(host(x), xo) < 5e-2


def test_hio_large_estimate_only(tb):
    """iters = 0 with an estimate: S (.) P_M(x) of the input, S binarised."""
    torch, cb = tb
    L, B = 512, 1
    A, S0, x0 = _hio_inputs(L, B, seed=5)
    S0 = S0 * 0.75   # inside values 0.75: still inside, written back as 1
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    x, S = dev(torch, x0.ravel()), dev(torch, S0.ravel())
    est = torch.empty_like(x)
    assert impl.hio_shrinkwrap(x, dev(torch, A.ravel()), S, B, 0, sw_every=0, estimate=est) and impl.Sync()
    _, _, eo = O.hio_shrinkwrap(x0, A, (S0 > 0.5).astype(np.float32), L, B, 0, 0.9, sw_every=0)
    assert O.rel_l2(host(est), eo) < FP32_DM_TOL
    np.testing.assert_array_equal(host(S), (S0 > 0.5).astype(np.float32).ravel())
    np.testing.assert_array_equal(host(x), x0.ravel())


@pytest.mark.parametrize("cluster", [0, 8])
def test_hio_large_full_run_rfactor(tb, cluster):
    """The uneven-size configuration's 256x256 bucket shape: HIO beta 0.9, 100
    iterations, shrinkwrap every 20 (sigma 3 -> 1.5, threshold 0.1), support
    radius ~0.19 of the side; line passes (cluster 0) and the cluster kernel
    (8 CTAs per pattern).  Bars as for the 128x128 run (chaotic iteration):
    mean R-factor of the reconstructions within 2% (relative) of the float64
    oracle's, median per-pattern difference < 4%, worst < 25%."""
    torch, cb = tb
    L, B = 256, 8
    A, S0, x0 = _hio_inputs(L, B, seed=2)
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    assert impl.set_option(cb.OPT_HIO_CLUSTER, cluster)
    x, S, Ad = dev(torch, x0.ravel()), dev(torch, S0.ravel()), dev(torch, A.ravel())
    est = torch.empty_like(x)
    assert impl.hio_shrinkwrap(x, Ad, S, B, 100, beta=0.9, sw_every=20, sigma_start=3.0, sigma_end=1.5,
                               threshold=0.1, estimate=est) and impl.Sync()
    r = impl.rfactor(est, Ad, B, a_stride=L * L)
    xo, So, eo = O.hio_shrinkwrap(x0, A, S0, L, B, 100, 0.9, sw_every=20, sigma_start=3.0, sigma_end=1.5,
                                  threshold=0.1)
    ro = O.rfactor(eo, A, L, L, B, a_stride=L * L)
    rel = np.abs(r - ro) / ro
    assert abs(r.mean() - ro.mean()) / ro.mean() < 0.02, (r, ro)
    assert np.median(rel) < 0.04 and np.max(rel) < 0.25, (r, ro)
    e = host(est).reshape(B, -1)
    assert np.all(e[host(S).reshape(B, -1) < 0.5] == 0)


# ---- one pattern over a thread-block cluster -----------------------------------------------
@pytest.mark.parametrize("cluster", [2, 4, 8])
@pytest.mark.parametrize("pos", [False, True])
def test_hio_cluster_128_equals_tmem_kernel_bitwise(tb, cluster, pos):
    """At 128^2 the cluster kernel runs the tensor-memory kernel's line
    transforms and per-element steps in the same order, with the rows and
    the columns of a pattern owned by different CTAs: x, the support and the
    estimate are the same bits for 2, 4 and 8 CTAs per pattern, through two
    shrinkwrap updates."""
    torch, cb = tb
    L, B = 128, 3
    A, S0, x0 = _hio_inputs(L, B, seed=40 + cluster)
    out = []
    for cl in (0, cluster):
        impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
        assert impl.set_option(cb.OPT_TMEM, 1) and impl.set_option(cb.OPT_HIO_CLUSTER, cl)
        x, S = dev(torch, x0.ravel()), dev(torch, S0.ravel())
        est = torch.empty_like(x)
        assert impl.hio_shrinkwrap(x, dev(torch, A.ravel()), S, B, 25, beta=0.9, sw_every=10, positivity=pos,
                                   estimate=est)
        assert impl.Sync()
        out.append((host(x), host(S), host(est)))
        impl.close()
    for a, b in zip(*out):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("cluster,pos", [(8, False), (16, True)])
def test_hio_cluster_256_vs_oracle(tb, cluster, pos):
    """256^2 over 8 or 16 CTAs per pattern: HIO iterations (no support
    update) against the oracle, 1e-5 relative L2 per iteration."""
    torch, cb = tb
    L, B, iters = 256, 2, 3
    A, S0, x0 = _hio_inputs(L, B, seed=50 + cluster)
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    assert impl.set_option(cb.OPT_HIO_CLUSTER, cluster)
    x, S = dev(torch, x0.ravel()), dev(torch, S0.ravel())
    assert impl.hio_shrinkwrap(x, dev(torch, A.ravel()), S, B, iters, beta=0.9, sw_every=0, positivity=pos)
    assert impl.Sync()
    xo, So, _ = O.hio_shrinkwrap(x0, A, S0, L, B, iters, 0.9, sw_every=0, positivity=pos)
    assert O.rel_l2(host(x), xo) < FP32_DM_TOL * iters
    np.testing.assert_array_equal(host(S), So.astype(np.float32))


def test_hio_cluster_256_sizes_bitwise(tb):
    """8 and 16 CTAs per 256^2 pattern run the same line transforms: the same
    bits of x, the support and the estimate through two shrinkwrap updates."""
    torch, cb = tb
    L, B = 256, 3
    A, S0, x0 = _hio_inputs(L, B, seed=61)
    out = []
    for cl in (8, 16):
        impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
        assert impl.set_option(cb.OPT_HIO_CLUSTER, cl)
        x, S = dev(torch, x0.ravel()), dev(torch, S0.ravel())
        est = torch.empty_like(x)
        assert impl.hio_shrinkwrap(x, dev(torch, A.ravel()), S, B, 25, beta=0.9, sw_every=10, estimate=est)
        assert impl.Sync()
        out.append((host(x), host(S), host(est)))
        impl.close()
    for a, b in zip(*out):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("B", [4, 40])
def test_autotune_hio_cluster_bitwise(tb, B):
    """With CPRA_B200_OPT_AUTOTUNE and the automatic cluster choice, a 128^2
    call measures one CTA per pattern against clusters of 2, 4 and 8 (on
    copies of x and S); whatever it picks, x, the support and the estimate
    are the bits of the tensor-memory kernel, on the measuring call and on
    the cached one; the automatic choice without the tuner gives them too."""
    torch, cb = tb
    L, iters, sw = 128, 12, 5
    A, S0, x0 = _hio_inputs(L, B, seed=90 + B)
    res = []
    for tune, cluster in ((0, 0), (0, 1), (1, 1)):
        impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
        assert impl.set_option(cb.OPT_AUTOTUNE, tune) and impl.set_option(cb.OPT_HIO_CLUSTER, cluster)
        for _ in range(2 if tune else 1):
            x, Sd = dev(torch, x0.ravel()), dev(torch, S0.ravel())
            est = torch.empty_like(x)
            assert impl.hio_shrinkwrap(x, dev(torch, A.ravel()), Sd, B, iters, beta=0.9, sw_every=sw, estimate=est)
            assert impl.Sync()
            res.append((host(x), host(Sd), host(est)))
        impl.close()
    for r in res[1:]:
        for a, b in zip(r, res[0]):
            np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("B,iters,sw,cluster", [(2, 0, 0, 8), (3, 20, 10, 4), (18, 10, 5, 1), (1, 7, 7, 2)])
def test_hio_cluster_128_edges_bitwise(tb, B, iters, sw, cluster):
    """Edge cases of the cluster kernel against the one-CTA tensor-memory
    kernel, bit for bit: the estimate alone (no iteration), a support update
    after the last iteration (then the estimate), the automatic choice at its
    boundary (18 patterns x 8 CTAs = 144 SMs), a single pattern."""
    torch, cb = tb
    L = 128
    A, S0, x0 = _hio_inputs(L, B, seed=300 + B + iters)
    out = []
    for cl in (0, cluster):
        impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
        assert impl.set_option(cb.OPT_HIO_CLUSTER, cl)
        x, S = dev(torch, x0.ravel()), dev(torch, S0.ravel())
        est = torch.empty_like(x)
        assert impl.hio_shrinkwrap(x, dev(torch, A.ravel()), S, B, iters, beta=0.9, sw_every=sw, estimate=est)
        assert impl.Sync()
        out.append((host(x), host(S), host(est)))
        impl.close()
    for a, b in zip(*out):
        np.testing.assert_array_equal(a, b)


def test_hio_cluster_256_estimate_only_vs_oracle(tb):
    """iters = 0 with an estimate at 256^2 over 8 CTAs: S (.) P_M(x) of the
    input within the per-iteration bar, x untouched, S binarised."""
    torch, cb = tb
    L, B = 256, 2
    A, S0, x0 = _hio_inputs(L, B, seed=17)
    S0 = S0 * 0.75
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    assert impl.set_option(cb.OPT_HIO_CLUSTER, 8)
    x, S = dev(torch, x0.ravel()), dev(torch, S0.ravel())
    est = torch.empty_like(x)
    assert impl.hio_shrinkwrap(x, dev(torch, A.ravel()), S, B, 0, sw_every=0, estimate=est) and impl.Sync()
    _, _, eo = O.hio_shrinkwrap(x0, A, (S0 > 0.5).astype(np.float32), L, B, 0, 0.9, sw_every=0)
    assert O.rel_l2(host(est), eo) < FP32_DM_TOL
    np.testing.assert_array_equal(host(S), (S0 > 0.5).astype(np.float32).ravel())
    np.testing.assert_array_equal(host(x), x0.ravel())


def test_hio_cluster_wait_runs_out_reports_error(tb):
    """The cluster kernel's waits for its peers' blocks are bounded.  With the
    failure test armed the launch's first CTA withholds its first row blocks;
    its peers' waits run out after about a second, the launch marks itself
    failed and Sync raises.  The context stays usable: the same call again
    gives the bits of a fresh context."""
    import time
    torch, cb = tb
    L, B, iters = 128, 2, 3
    A, S0, x0 = _hio_inputs(L, B, seed=71)
    Ad = dev(torch, A.ravel())
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    assert impl.set_option(cb.OPT_HIO_CLUSTER, 8) and impl.set_option(cb.OPT_FAILURE_TEST, 1)
    x, S = dev(torch, x0.ravel()), dev(torch, S0.ravel())
    t0 = time.monotonic()
    assert impl.hio_shrinkwrap(x, Ad, S, B, iters, beta=0.9, sw_every=0)
    with pytest.raises(cb.CpraB200Error, match="ran out"):
        impl.Sync()
    assert 0.9 < time.monotonic() - t0 < 60
    assert impl.get_option(cb.OPT_FAILURE_TEST) == 0   # cleared by the launch
    x, S = dev(torch, x0.ravel()), dev(torch, S0.ravel())
    assert impl.hio_shrinkwrap(x, Ad, S, B, iters, beta=0.9, sw_every=0) and impl.Sync()
    fresh = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    assert fresh.set_option(cb.OPT_HIO_CLUSTER, 8)
    xf, Sf = dev(torch, x0.ravel()), dev(torch, S0.ravel())
    assert fresh.hio_shrinkwrap(xf, Ad, Sf, B, iters, beta=0.9, sw_every=0) and fresh.Sync()
    np.testing.assert_array_equal(host(x), host(xf))
    np.testing.assert_array_equal(host(S), host(Sf))
    impl.close()
    fresh.close()


def test_hio_cluster_option_checked(tb):
    torch, cb = tb
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, 128, 128, 1, 1)
    assert impl.get_option(cb.OPT_HIO_CLUSTER) == 1   # automatic by default
    for v in (0, 1, 2, 4, 8, 16):
        assert impl.set_option(cb.OPT_HIO_CLUSTER, v)
        assert impl.get_option(cb.OPT_HIO_CLUSTER) == v
    for v in (-1, 3, 32):
        assert not impl.set_option(cb.OPT_HIO_CLUSTER, v)
    impl.close()


# ---- uneven sizes in one call --------------------------------------------------------------
@pytest.mark.parametrize("own_sigma,cluster", [(False, 0), (True, 0), (True, 8)])
def test_hio_batched_matches_per_size_calls(tb, own_sigma, cluster):
    """Each bucket of the uneven-size call gives the same bits as a
    single-size call with the same patterns (the buckets only share the
    device, not data); with own_sigma each bucket has its own blur schedule
    (3 -> 1.5 px times side / 128) and the CUDA backend's DataConstraint;
    with cluster 8 the 128 and 256 buckets run on the cluster kernel."""
    torch, cb = tb
    sizes = [(64, 3), (128, 2), (256, 2), (512, 3)]
    iters, sw = 12, 5
    data = {L: _hio_inputs(L, B, seed=L) for L, B in sizes}
    sig = {L: ((3.0 * L / 128, 1.5 * L / 128) if own_sigma else (3.0, 1.5)) for L, _ in sizes}
    buckets, keep = [], []
    for L, B in sizes:
        A, S0, x0 = data[L]
        b = {"side": L, "count": B, "x": dev(torch, x0.ravel()), "A": dev(torch, A.ravel()),
             "S": dev(torch, S0.ravel())}
        if own_sigma:
            b["sigma_start"], b["sigma_end"] = sig[L]
        b["estimate"] = torch.empty_like(b["x"])
        buckets.append(b)
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, 64, 64, 1, 1)
    assert impl.set_option(cb.OPT_DATA_MODE, 1 if own_sigma else 0)
    assert impl.set_option(cb.OPT_HIO_CLUSTER, cluster)
    assert impl.hio_batched(buckets, iters, beta=0.9, sw_every=sw) and impl.Sync()
    for (L, B), b in zip(sizes, buckets):
        A, S0, x0 = data[L]
        one = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
        assert one.set_option(cb.OPT_DATA_MODE, 1 if own_sigma else 0)
        assert one.set_option(cb.OPT_HIO_CLUSTER, cluster)
        x, S = dev(torch, x0.ravel()), dev(torch, S0.ravel())
        est = torch.empty_like(x)
        assert one.hio_shrinkwrap(x, dev(torch, A.ravel()), S, B, iters, beta=0.9, sw_every=sw,
                                  sigma_start=sig[L][0], sigma_end=sig[L][1], estimate=est)
        assert one.Sync()
        np.testing.assert_array_equal(host(b["x"]), host(x))
        np.testing.assert_array_equal(host(b["S"]), host(S))
        np.testing.assert_array_equal(host(b["estimate"]), host(est))


def test_hio_batched_rejects_bad_buckets(tb):
    torch, cb = tb
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, 64, 64, 1, 1)
    x = torch.zeros(96 * 96, dtype=torch.complex64, device="cuda")
    A = torch.zeros(96 * 96, dtype=torch.float32, device="cuda")
    with pytest.raises(cb.CpraB200Error):
        impl.hio_batched([{"side": 96, "count": 1, "x": x, "A": A, "S": A}], 2)
    assert not impl.hio_batched([], 2)


# ---- CUDA graphs of whole runs --------------------------------------------------------------
@pytest.mark.parametrize("L", [64, 256])
def test_cpra_run_graph_replay_bitwise(tb, L):
    """With CPRA_B200_OPT_GRAPH the first cpra_run call is captured and later
    identical calls replay the graph: same bits, same error output and the
    same kernel count as running without graphs."""
    torch, cb = tb
    P, B, epi, it, pre = 3, 2, 2, 2, 1
    rng = np.random.default_rng(L)
    A = (rng.uniform(0, 30, (P, L * L)) * (rng.uniform(0, 1, (P, L * L)) > 0.1)).astype(np.float32)
    S = (rng.uniform(0, 1, (P, L * L)) > 0.45).astype(np.float32)
    x0 = (rng.uniform(0, 1, P * B * L * L) + 1j * rng.uniform(0, 1, P * B * L * L)).astype(np.complex64)
    Ad, Sd = dev(torch, A.ravel()), dev(torch, S.ravel())
    plain = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    xr = dev(torch, x0)
    err_r = np.zeros(P * B, np.float32)
    n0 = cb.kernels_launched()
    assert plain.cpra_run(xr, Ad, Sd, P, B, epi, it, pre, 0.9, final_step=True, err=err_r) and plain.Sync()
    n_plain = cb.kernels_launched() - n0
    g = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    assert g.set_option(cb.OPT_GRAPH, 1)
    x = dev(torch, x0)
    for rep in range(3):
        x.copy_(dev(torch, x0))
        err = np.zeros(P * B, np.float32)
        n0 = cb.kernels_launched()
        assert g.cpra_run(x, Ad, Sd, P, B, epi, it, pre, 0.9, final_step=True, err=err) and g.Sync()
        assert cb.kernels_launched() - n0 == n_plain
        np.testing.assert_array_equal(host(x), host(xr))
        np.testing.assert_array_equal(err, err_r)


def test_graph_recaptured_after_buffers_move(tb):
    """A call that grows a context buffer invalidates the cached graphs (they
    hold its old address); the next run captures anew and stays exact."""
    torch, cb = tb
    L, P, B = 64, 3, 2
    rng = np.random.default_rng(3)
    A = rng.uniform(0, 30, (P, L * L)).astype(np.float32)
    S = (rng.uniform(0, 1, (P, L * L)) > 0.45).astype(np.float32)
    x0 = (rng.uniform(0, 1, P * B * L * L) + 1j * rng.uniform(0, 1, P * B * L * L)).astype(np.complex64)
    Ad, Sd = dev(torch, A.ravel()), dev(torch, S.ravel())
    ref = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    xr = dev(torch, x0)
    assert ref.cpra_run(xr, Ad, Sd, P, B, 1, 2, 0, 0.9) and ref.Sync()
    g = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
    assert g.set_option(cb.OPT_GRAPH, 1)
    x = dev(torch, x0)
    assert g.cpra_run(x, Ad, Sd, P, B, 1, 2, 0, 0.9) and g.Sync()
    # rfactor over many patterns grows the context's work buffer
    big = torch.zeros(64 * L * L, dtype=torch.complex64, device="cuda")
    g.rfactor(big, Ad, 64)
    x.copy_(dev(torch, x0))
    assert g.cpra_run(x, Ad, Sd, P, B, 1, 2, 0, 0.9) and g.Sync()
    np.testing.assert_array_equal(host(x), host(xr))


def test_hio_batched_graph_replay_bitwise(tb):
    torch, cb = tb
    sizes = [(64, 2), (256, 1)]
    data = {L: _hio_inputs(L, B, seed=L + 3) for L, B in sizes}

    def buckets():
        out = []
        for L, B in sizes:
            A, S0, x0 = data[L]
            out.append({"side": L, "count": B, "x": dev(torch, x0.ravel()), "A": dev(torch, A.ravel()),
                        "S": dev(torch, S0.ravel())})
        return out

    plain = cb.NewCpraImpl(cb.IMPL_TYPE.B200, 64, 64, 1, 1)
    want = buckets()
    assert plain.hio_batched(want, 10, sw_every=5) and plain.Sync()
    g = cb.NewCpraImpl(cb.IMPL_TYPE.B200, 64, 64, 1, 1)
    assert g.set_option(cb.OPT_GRAPH, 1)
    bk = buckets()
    for rep in range(2):
        for (L, B), b in zip(sizes, bk):
            A, S0, x0 = data[L]
            b["x"].copy_(dev(torch, x0.ravel()))
            b["S"].copy_(dev(torch, S0.ravel()))
        assert g.hio_batched(bk, 10, sw_every=5) and g.Sync()
        for b, w in zip(bk, want):
            np.testing.assert_array_equal(host(b["x"]), host(w["x"]))
            np.testing.assert_array_equal(host(b["S"]), host(w["S"]))


# ---- the benchmark's 3D step, fused ---------------------------------------------------------
@pytest.mark.parametrize("T,M,N,L,B,mode", [(np.float32, 32, 32, 32, 2, 0), (np.float32, 64, 64, 64, 1, 1),
                                            (np.float64, 16, 16, 16, 1, 0), (np.float32, 8, 16, 32, 2, 0),
                                            (np.float32, 24, 24, 24, 1, 0)])
def test_constraint3d_equals_operator_calls(tb, T, M, N, L, B, mode):
    """constraint3d (five axis passes per iteration) writes the same bits as
    Forward3D, DataConstraint (complex), Backward3D, SpaceConstraint called one
    at a time (src/benchmark_mkl.cpp:164-170), and follows the oracle."""
    torch, cb = tb
    rng = np.random.default_rng(M * N + L)
    cdt = np.complex64 if T == np.float32 else np.complex128
    vol = M * N * L
    x0 = (rng.standard_normal(B * vol) + 1j * rng.standard_normal(B * vol)).astype(cdt)
    C = (rng.standard_normal(vol) + 1j * rng.standard_normal(vol)).astype(cdt)
    C[rng.uniform(size=vol) < 0.3] = 0
    S = (rng.uniform(size=vol) > 0.4).astype(T)
    dtype = "float32" if T == np.float32 else "float64"
    outs = []
    # the operator calls; constraint3d on its default path (the operator
    # kernels); constraint3d as fused axis passes (CPRA_B200_OPT_FUSED3D)
    for fused, fused3d in ((False, 0), (True, 0), (True, 1)):
        impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, L, B, dtype=dtype)
        assert impl.set_option(cb.OPT_SPACE_MODE, mode)
        assert impl.set_option(cb.OPT_FUSED3D, fused3d)
        x = dev(torch, x0)
        Cd, Sd = dev(torch, C), dev(torch, S)
        for _ in range(2):
            if fused:
                assert impl.constraint3d(x, Cd, Sd, 1)
            else:
                assert impl.Forward3D(x)
                assert impl.DataConstraint(x, Cd, B * vol, B)
                assert impl.Backward3D(x)
                assert impl.SpaceConstraint(x, Sd, B * vol, B)
        assert impl.Sync()
        outs.append(host(x))
    np.testing.assert_array_equal(outs[0], outs[1])
    np.testing.assert_array_equal(outs[0], outs[2])
    if mode == 0:
        o = O.OracleImpl(T, M, N, L, B)
        xo = x0.copy()
        for _ in range(2):
            o.Forward3D(xo)
            o.DataConstraint(xo, C, B * vol, B)
            o.Backward3D(xo)
            o.SpaceConstraint(xo, S, B * vol, B)
        assert O.rel_l2(outs[1], xo) < (1e-5 if T == np.float32 else 1e-12)


# ---- the conventional 3D difference map (src/CONV_MKL.cpp:37-88) through the recorder ------
def dm3d_per_call(impl, x, t1, t2, A, S, num, B, beta):
    """src/CONV_MKL.cpp:47-61, one interface call at a time."""
    b = float(np.float32(beta)) if x.dtype == __import__("torch").complex64 else float(beta)
    impl.Forward3D(t1)
    impl.DataConstraint(t1, A, num, B)
    impl.Backward3D(t1)
    impl.MergeAddData(x, t1, -1.0 / b, 1.0 + 1.0 / b, num)
    impl.SpaceConstraint(t1, S, num, B)
    impl.SpaceConstraint(t2, S, num, B)
    impl.MergeAddData(x, t2, 1.0 / b, 1.0 - 1.0 / b, num)
    impl.Forward3D(t2)
    impl.DataConstraint(t2, A, num, B)
    impl.Backward3D(t2)
    impl.MergeAddData(t1, x, b, 1.0, num)
    impl.MergeAddData(t2, x, -1.0 * b, 1.0, num)


def conv_driver_per_call(impl, torch, x, A, S, M, N, L, B, iters, beta, err, final):
    """ShrinkWrap_CONV_MKL_Sample (src/CONV_MKL.cpp:30-88) one interface call
    at a time, from the guesses already in x."""
    num = M * N * L * B
    nbytes = x.numel() * x.element_size()
    b = float(np.float32(beta)) if x.dtype == torch.complex64 else float(beta)
    t1, t2, old = (torch.empty_like(x) for _ in range(3))
    impl.Memcpy(t1, x, nbytes)
    impl.Memcpy(t2, x, nbytes)
    for i in range(iters):
        if err is not None and i == iters - 1:
            impl.Memcpy(old, x, nbytes)
        dm3d_per_call(impl, x, t1, t2, A, S, num, B, beta)
        if err is not None and i == iters - 1:
            impl.Memcpy(t1, x, nbytes)
            impl.Forward3D(old)
            impl.Forward3D(t1)
            impl.ConvergeError(old, t1, err, M, N, L, B)
    if final:
        impl.Memcpy(t1, x, nbytes)
        impl.Forward3D(t1)
        impl.DataConstraint(t1, A, num, B)
        impl.Backward3D(t1)
        impl.MergeAddData(x, t1, -1.0 / b, 1.0 + 1.0 / b, num)
        impl.SpaceConstraint(t1, S, num, B)
        impl.Memcpy(x, t1, nbytes)
    assert impl.Sync()


@pytest.mark.parametrize("T,M,N,L,B,iters,with_err,final",
                         [(np.float32, 16, 16, 16, 2, 3, True, True), (np.float32, 32, 16, 8, 2, 2, False, True),
                          (np.float64, 16, 16, 16, 1, 2, True, True), (np.float32, 12, 12, 12, 1, 2, True, True),
                          (np.float32, 16, 16, 16, 2, 1, True, False), (np.float32, 16, 16, 16, 1, 0, False, True)])
def test_conv_run_equals_driver(tb, T, M, N, L, B, iters, with_err, final):
    """cpra_b200_conv_run writes the same bits and errors as the reference's
    conventional driver issued one call at a time with fusion off, directly
    and replayed from a CUDA graph; and agrees with the oracle."""
    torch, cb = tb
    rng = np.random.default_rng(M * N * L + B + iters)
    vol = M * N * L
    cdt = np.complex64 if T == np.float32 else np.complex128
    dtype = "float32" if T == np.float32 else "float64"
    amps = (rng.uniform(0, 40, vol) * (rng.uniform(0, 1, vol) > 0.1)).astype(T)
    sup = (rng.uniform(0, 1, vol) > 0.5).astype(T)
    x0 = (rng.uniform(0, 1, vol * B) + 1j * rng.uniform(0, 1, vol * B)).astype(cdt)
    A, S = dev(torch, amps), dev(torch, sup)
    ref = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, L, B, dtype=dtype)
    ref.set_option(cb.OPT_FUSION, 0)
    xr = dev(torch, x0)
    err_r = np.zeros(B, T) if with_err else None
    conv_driver_per_call(ref, torch, xr, A, S, M, N, L, B, iters, 0.9, err_r, final)
    run = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, L, B, dtype=dtype)
    for graph, fused3d in ((0, 0), (1, 0), (1, 0), (0, 1), (1, 1), (1, 1)):
        assert run.set_option(cb.OPT_GRAPH, graph)
        assert run.set_option(cb.OPT_FUSED3D, fused3d)
        x = dev(torch, x0)
        err = np.zeros(B, T) if with_err else None
        assert run.conv_run(x, A, S, iters, 0.9, final_step=final, err=err) and run.Sync()
        np.testing.assert_array_equal(host(x), host(xr))
        if with_err:
            np.testing.assert_array_equal(err, err_r)
    # the oracle: the same driver on the FP64/FP32 restatement
    o = O.OracleImpl(T, M, N, L, B)
    xo, t1o, t2o = x0.copy(), x0.copy(), x0.copy()
    bb = float(np.float32(0.9)) if T == np.float32 else 0.9
    num = vol * B
    for _ in range(iters):
        o.Forward3D(t1o); o.DataConstraint(t1o, amps, num, B); o.Backward3D(t1o)
        o.MergeAddData(xo, t1o, -1.0 / bb, 1.0 + 1.0 / bb, num); o.SpaceConstraint(t1o, sup, num, B)
        o.SpaceConstraint(t2o, sup, num, B); o.MergeAddData(xo, t2o, 1.0 / bb, 1.0 - 1.0 / bb, num)
        o.Forward3D(t2o); o.DataConstraint(t2o, amps, num, B); o.Backward3D(t2o)
        o.MergeAddData(t1o, xo, bb, 1.0, num); o.MergeAddData(t2o, xo, -1.0 * bb, 1.0, num)
    if final:
        t1o = xo.copy()
        o.Forward3D(t1o); o.DataConstraint(t1o, amps, num, B); o.Backward3D(t1o)
        o.MergeAddData(xo, t1o, -1.0 / bb, 1.0 + 1.0 / bb, num); o.SpaceConstraint(t1o, sup, num, B)
        xo = t1o
    tol = (FP32_DM_TOL if T == np.float32 else 1e-12) * max(iters + final, 1)
    assert O.rel_l2(host(xr), xo) < tol
    assert not run.conv_run(x, A, S, -1, 0.9)
    assert not run.conv_run(x, A, S, 0, 0.9, err=np.zeros(B, T))


@pytest.mark.parametrize("T,M,N,L,B,iters", [(np.float32, 16, 16, 16, 1, 3), (np.float32, 32, 16, 8, 2, 2),
                                             (np.float64, 16, 16, 16, 1, 2), (np.float32, 12, 12, 12, 1, 2)])
def test_dm3d_recorder_equals_per_call(tb, T, M, N, L, B, iters):
    """The 12-call iteration with the 3D transforms, issued one call at a time,
    runs as ten fused axis passes per iteration (power-of-two sizes, with
    CPRA_B200_OPT_FUSED3D) and writes the same bits as with fusion off; other
    sizes run per call."""
    torch, cb = tb
    rng = np.random.default_rng(M * N * L + B)
    vol = M * N * L
    num = vol * B
    cdt = np.complex64 if T == np.float32 else np.complex128
    amps = (rng.uniform(0, 40, vol) * (rng.uniform(0, 1, vol) > 0.1)).astype(T)
    sup = (rng.uniform(0, 1, vol) > 0.5).astype(T)
    x0 = (rng.uniform(0, 1, num) + 1j * rng.uniform(0, 1, num)).astype(cdt)
    dtype = "float32" if T == np.float32 else "float64"
    outs = []
    for fusion in (0, 1):
        impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, L, B, dtype=dtype)
        impl.set_option(cb.OPT_FUSION, fusion)
        impl.set_option(cb.OPT_FUSED3D, fusion)
        x, t1, t2 = (dev(torch, x0) for _ in range(3))
        A, S = dev(torch, amps), dev(torch, sup)
        for _ in range(iters):
            dm3d_per_call(impl, x, t1, t2, A, S, num, B, 0.9)
        assert impl.Sync()
        outs.append([host(v) for v in (x, t1, t2)])
    for a, b in zip(outs[0], outs[1]):
        np.testing.assert_array_equal(a, b)
    o = O.OracleImpl(T, M, N, L, B)
    xo, t1o, t2o = x0.copy(), x0.copy(), x0.copy()
    bb = float(np.float32(0.9)) if T == np.float32 else 0.9
    for _ in range(iters):
        o.Forward3D(t1o); o.DataConstraint(t1o, amps, num, B); o.Backward3D(t1o)
        o.MergeAddData(xo, t1o, -1.0 / bb, 1.0 + 1.0 / bb, num); o.SpaceConstraint(t1o, sup, num, B)
        o.SpaceConstraint(t2o, sup, num, B); o.MergeAddData(xo, t2o, 1.0 / bb, 1.0 - 1.0 / bb, num)
        o.Forward3D(t2o); o.DataConstraint(t2o, amps, num, B); o.Backward3D(t2o)
        o.MergeAddData(t1o, xo, bb, 1.0, num); o.MergeAddData(t2o, xo, -1.0 * bb, 1.0, num)
    tol = (FP32_DM_TOL if T == np.float32 else 1e-12) * iters
    for got, want in zip(outs[1], (xo, t1o, t2o)):
        assert O.rel_l2(got, want) < tol


# ---- the autotuner's other choices: the path of the 3D step and the HIO chunk ------------------
def test_autotune_constraint3d_and_hio_chunk_bitwise(tb):
    """With CPRA_B200_OPT_AUTOTUNE the 3D step measures its two paths and the
    256^2 HIO passes their chunk (on copies of the inputs, once per shape);
    whatever each picks, the results equal those of every candidate, on the
    measuring call and on the cached one."""
    torch, cb = tb
    rng = np.random.default_rng(77)
    n = 32
    vol = n ** 3
    x0 = (rng.standard_normal(vol) + 1j * rng.standard_normal(vol)).astype(np.complex64)
    C = (rng.standard_normal(vol) + 1j * rng.standard_normal(vol)).astype(np.complex64)
    C[rng.uniform(size=vol) < 0.3] = 0
    S = (rng.uniform(size=vol) > 0.4).astype(np.float32)
    outs = []
    for tune, fused3d in ((0, 0), (0, 1), (1, 0), (1, 1)):
        impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, n, n, n, 1)
        assert impl.set_option(cb.OPT_AUTOTUNE, tune) and impl.set_option(cb.OPT_FUSED3D, fused3d)
        for _ in range(2):   # the first tuned call measures, the second uses the cache
            x = dev(torch, x0)
            assert impl.constraint3d(x, dev(torch, C), dev(torch, S), 3) and impl.Sync()
            outs.append(host(x))
    for o in outs[1:]:
        np.testing.assert_array_equal(o, outs[0])

    L, B, iters, sw = 256, 4, 12, 5
    A, S0, x0 = _hio_inputs(L, B, seed=5)
    res = []
    for tune, chunk in ((0, 4), (0, 2), (0, 1), (1, 0)):
        impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, L, L, 1, B)
        assert impl.set_option(cb.OPT_AUTOTUNE, tune) and impl.set_option(cb.OPT_HIO_CHUNK, chunk)
        assert impl.set_option(cb.OPT_HIO_CLUSTER, 0)   # the line passes
        for _ in range(2 if tune else 1):
            x, Sd = dev(torch, x0.ravel()), dev(torch, S0.ravel())
            est = torch.empty_like(x)
            assert impl.hio_shrinkwrap(x, dev(torch, A.ravel()), Sd, B, iters, beta=0.9, sw_every=sw, estimate=est)
            assert impl.Sync()
            res.append((host(x), host(Sd), host(est)))
    for r in res[1:]:
        for a, b in zip(r, res[0]):
            np.testing.assert_array_equal(a, b)
