"""Pins the CPU oracle (oracle/cpra_oracle.py) before it is trusted.

1. The reference's own known-answer tests, restated (test/unitest_mkl.cpp:4-71).
2. The golden fixtures in tests/golden/ref_golden.npz, produced by the
   reference's MklImpl<T> source compiled here (tests/golden/make_golden.py).
3. When oracle/_ref is built in this checkout, seeded cases run live against it.
"""
import numpy as np
import pytest

import cpra_oracle as O
from conftest import GOLDEN

G = np.load(GOLDEN / "ref_golden.npz")

FP32_FFT_TOL = 1e-6   # one FP32 transform vs the float64-rounded oracle
FP32_DM_TOL = 1e-5    # per difference-map iteration, relative L2


# ---- test/unitest_mkl.cpp -------------------------------------------------------
def test_kat_initialize_range():
    """MKLTEST.Test_MKL_Initialize (unitest_mkl.cpp:4-12): values in [0, 1]."""
    impl = O.OracleImpl(np.float32, 1, 1, 1, 1)
    buf = np.full(1000, -1, np.float32)
    assert impl.Initialize(buf, 1000)
    assert np.all((buf >= 0) & (buf <= 1))
    assert not impl.Initialize(buf, 0)


def test_kat_norm_merge():
    """MKLTEST.Test_Norm_Merge (unitest_mkl.cpp:15-40): exact values."""
    impl = O.OracleImpl(np.float32, 1, 1, 1, 1)
    x = np.full(1000, 10 + 10j, np.complex64)
    assert impl.MergeAddData(x, x, 0.5, 0.5, 1000)
    assert np.all(x.real == 10) and np.all(x.imag == 10)
    assert impl.Normalization(x, 10, 1000)
    assert np.all(x.real == 1) and np.all(x.imag == 1)
    np.testing.assert_array_equal(G["kat_merge_half"], np.full(1000, 10 + 10j, np.complex64))
    np.testing.assert_array_equal(G["kat_norm10"], np.full(1000, 1 + 1j, np.complex64))


def test_kat_2d_dft_double():
    """MKLTEST.Test_2D_DFT (unitest_mkl.cpp:42-71): 10x10 ones, double."""
    impl = O.OracleImpl(np.float64, 10, 10, 1, 1)
    x = np.ones(100, np.complex128)
    assert impl.Forward2D(x)
    want = np.zeros(100, np.complex128)
    want[5 * 10 + 5] = 100
    assert np.max(np.abs(x - want)) <= 1e-14
    assert np.max(np.abs(G["kat_dft10_fwd"] - want)) <= 1e-14   # the reference build passes too
    assert impl.Backward2D(x)
    assert np.max(np.abs(x - 1)) <= 1e-14
    assert np.max(np.abs(G["kat_dft10_bwd"] - 1)) <= 1e-14


def test_argument_errors_match_reference():
    impl = O.OracleImpl(np.float32, 4, 4, 1, 1)
    x = np.zeros(16, np.complex64)
    s = np.zeros(16, np.float32)
    assert not impl.MergeAddData(x, x, 0.0, 1.0, 16)   # MKL_Impl.inl:34
    assert not impl.MergeAddData(x, x, 1.0, 1.0, 0)
    assert not impl.Normalization(x, 0.0, 16)          # :55
    assert not impl.SpaceConstraint(x, s, 0, 1)         # :73
    assert not impl.DataConstraint(x, s, 16, 0)         # :89


# ---- golden fixtures from the compiled reference ----------------------------------
@pytest.mark.parametrize("tag,T,M,N,B", [("f32_64", np.float32, 64, 64, 2), ("f64_32", np.float64, 32, 32, 2),
                                         ("f32_128", np.float32, 128, 128, 1), ("f32_16x8", np.float32, 16, 8, 3)])
def test_oracle_transforms_vs_reference(tag, T, M, N, B):
    tol = FP32_FFT_TOL if T == np.float32 else 1e-13
    impl = O.OracleImpl(T, M, N, 1, B)
    x = G[f"{tag}_x"]
    y = x.copy(); impl.Forward2D(y)
    assert O.rel_l2(y, G[f"{tag}_fwd"]) < tol
    y = x.copy(); impl.Backward2D(y)
    assert O.rel_l2(y, G[f"{tag}_bwd"]) < tol
    y = x.copy(); impl.FFTShift2D(y, M, N, B)
    np.testing.assert_array_equal(y, G[f"{tag}_shift"])


def test_oracle_shift3d_vs_reference():
    impl = O.OracleImpl(np.float32, 6, 8, 4, 2)
    y = G["shift3d_x"].copy()
    impl.FFTShift3D(y, 6, 8, 4, 2)
    np.testing.assert_array_equal(y, G["shift3d_out"])


def test_oracle_elementwise_vs_reference():
    M = N = 32
    B = 3
    num = M * N * B
    impl = O.OracleImpl(np.float32, M, N, 1, B)
    x = G["ew_x"]
    y = x.copy(); impl.SpaceConstraint(y, G["ew_S"], num, B)
    np.testing.assert_array_equal(y, G["ew_sc"])
    y = x.copy(); impl.DataConstraint(y, G["ew_C"], num, B)
    np.testing.assert_array_equal(y, G["ew_dc_complex"])
    beta = np.float32(0.9)
    y = x.copy(); impl.MergeAddData(G["ew_src"], y, -1.0 / beta, 1.0 + 1.0 / beta, num)
    np.testing.assert_array_equal(y, G["ew_merge"])
    y = x.copy(); impl.Normalization(y, 3.0, num)
    np.testing.assert_array_equal(y, G["ew_norm3"])
    # the modulus projection goes through polar/arg in the reference: ulp-level
    y = x.copy(); impl.DataConstraint(y, G["ew_A"], num, B)
    ref = G["ew_dc_real"]
    assert np.max(np.abs(y - ref) / np.maximum(np.abs(ref), 1e-30)) < 4e-7
    # A == 0 and z == 0 are left untouched in both
    A = np.tile(G["ew_A"], B)
    np.testing.assert_array_equal(y[A == 0], x[A == 0])
    assert y[5] == 0 and ref[5] == 0


def test_oracle_threshold_edge():
    """S < 0.9 compares a float against the double 0.9 (MKL_Impl.inl:83):
    S = 0.9f is below it and is zeroed, nextafter(0.9f, 1) is kept."""
    S = G["ew_S"][:4]
    assert list(O._threshold_mask(S)) == [True, False, True, False]
    out = G["ew_sc"][:4]
    assert out[0] == 0 and out[2] == 0
    assert out[1] == G["ew_x"][1].real and out[3] == G["ew_x"][3].real


@pytest.mark.parametrize("iters", [1, 5])
def test_oracle_dm_iterations_vs_reference(iters):
    M = N = 64
    B = 2
    impl = O.OracleImpl(np.float32, M, N, 1, B)
    x0 = G["dm_x0"]
    x, t1, t2 = x0.copy(), x0.copy(), x0.copy()
    for _ in range(iters):
        O.dm_iteration(impl, x, t1, t2, G["dm_A"], G["dm_S"], M * N * B, B, 0.9)
    for name, v in (("x", x), ("t1", t1), ("t2", t2)):
        assert O.rel_l2(v, G[f"dm{iters}_{name}"]) < FP32_DM_TOL * iters, name


def test_oracle_cpra_episode_vs_reference():
    M, N, L, P, B, epi, it, pre = (int(v) for v in G["cpra_cfg"])
    x, _ = O.cpra_sample(np.float32, M, N, L, P, B, G["cpra_A"], G["cpra_S"], G["cpra_x0"], epi, it, pre, 0.9)
    # 4 + 2*4*3 + 1 = 29 chained iterations per start: drift is bounded, not ulp-level
    assert O.rel_l2(x, G["cpra_x"]) < 1e-3


# ---- live, when the reference build is present -----------------------------------
def _ref():
    import ref_lib
    if not ref_lib.available():
        pytest.skip("oracle/_ref not built (make -C oracle)")
    return ref_lib


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_oracle_live_vs_reference(T):
    R = _ref()
    rng = np.random.default_rng(7)
    M, N, B = 32, 16, 2
    C = O.complex_dtype(T)
    x = (rng.standard_normal(M * N * B) + 1j * rng.standard_normal(M * N * B)).astype(C)
    o, r = O.OracleImpl(T, M, N, 1, B), R.RefImpl(T, M, N, 1, B)
    tol = FP32_FFT_TOL if T == np.float32 else 1e-13
    a, b = x.copy(), x.copy()
    o.Forward2D(a); r.Forward2D(b)
    assert O.rel_l2(a, b) < tol
    a, b = x.copy(), x.copy()
    o.Backward2D(a); r.Backward2D(b)
    assert O.rel_l2(a, b) < tol
