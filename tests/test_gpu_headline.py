"""Parity at the carousel configuration's full size, against the reference build.

The carousel configuration: 128 x 128 patterns of a 128^3 ellipsoid volume's
projections at 90 angles (2 degree steps, 1e7 photons, Poisson), 10 episodes x
10 difference-map iterations per angle, the carousel mix, the last episode's
convergence error and the final projection (src/CPRA_MKL.cpp:35-140).  The
same seeded starts run through cpra_b200_cpra_run on the GPU and through the
reference's own MklImpl<float> operators in the reference driver's call order
(oracle/_ref, oracle/ref_capi.cpp `cpra_sample`).

Difference-map iterations from random starts are chaotic: 100 iterations per
angle amplify rounding differences, so single trajectories cannot agree
element by element.  The reference's own float and double builds, from the
same starts, already differ by up to 2.6 % in a start's R-factor (1.7 % in
the mean over 4 starts) and by about 3 % of the pixels in the support of the
final projection.  The results are therefore compared through what the
iteration is for, with the reference's double build as the anchor:
  * R-factor  sum | |Forward2D(x)| - A | / sum A  (float64, averaged over the
    90 angles): the mean over the starts within 1 % of the double build's and
    within 2 % of the float build's; each start within 2.5 % of the double
    build's;
  * support of the final projection, |x| > 0.1 max|x| per plane: differs from
    the double build's in no more pixels than the float build's does (25 %
    slack for 4 starts, plus 0.2 % of the pixels).
Per iteration the bound is 1e-5 relative L2 (one and five iterations at
128 x 128 against the reference operators on the same inputs).
"""
import numpy as np
import pytest

import cpra_oracle as O

pytestmark = pytest.mark.gpu

M = N = 128
P, EPI, ITERS, BETA = 90, 10, 10, 0.9
STARTS = 4
RFACTOR_MEAN_TOL_F64 = 0.01     # mean over the starts, against the double build
RFACTOR_MEAN_TOL_F32 = 0.02     # mean over the starts, against the float build
RFACTOR_START_TOL_F64 = 0.025   # any single start, against the double build
FP32_DM_TOL = 1e-5


@pytest.fixture(scope="module")
def ref():
    import ref_lib
    # the reference build is part of build(): its absence is a failure, not a skip
    assert ref_lib.available(), "oracle/_ref/libcpra_mklref.so is not built (make -C oracle)"
    ref_lib.QUIET = True
    return ref_lib


@pytest.fixture(scope="module")
def carousel_data():
    from cpra_b200 import synth
    return synth.carousel(n=M, P=P, seed=1)


def _support(x, frac=0.1):
    a = np.abs(np.asarray(x).reshape(-1, M * N))
    return a > frac * a.max(axis=1, keepdims=True)


def _rfactor_per_start(x, A):
    """[STARTS] mean over the angles of the per-pattern R-factor (float64)."""
    xs = np.asarray(x).reshape(P, STARTS, M * N)
    r = np.zeros((P, STARTS))
    for p in range(P):
        r[p] = O.rfactor(xs[p].ravel(), A[p].ravel(), M, N, STARTS)
    return r.mean(axis=0), r


def test_carousel_full_episode_vs_reference(cuda, ref, carousel_data):
    import torch
    import cpra_b200 as cb
    d = carousel_data
    A = np.ascontiguousarray(d["A"], np.float32)
    S = np.ascontiguousarray(d["S"], np.float32)
    rng = np.random.default_rng(2024)
    # Initialize's distribution (uniform [0, 1) real and imaginary parts), seeded
    x0 = (rng.uniform(0, 1, P * STARTS * M * N) + 1j * rng.uniform(0, 1, P * STARTS * M * N)).astype(np.complex64)

    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, 1, STARTS)
    xg = torch.from_numpy(x0.copy()).cuda()
    err = np.zeros(P * STARTS, np.float32)
    ok = impl.cpra_run(xg, torch.from_numpy(A.ravel()).cuda(), torch.from_numpy(S.ravel()).cuda(), P, STARTS,
                       EPI, ITERS, 0, BETA, final_step=True, err=err)
    assert ok and impl.Sync()
    x_b200 = xg.cpu().numpy()
    impl.close()

    x_ref = ref.cpra_sample(np.float32, M, N, 1, P, STARTS, A, S, x0, EPI, ITERS, 0, BETA)
    # the reference's double build from the same starts: how far float results
    # of this chaotic iteration are from double ones at all
    x_ref64 = ref.cpra_sample(np.float64, M, N, 1, P, STARTS, A, S, x0, EPI, ITERS, 0, BETA)

    r_b200, _ = _rfactor_per_start(x_b200, A)
    r_ref, _ = _rfactor_per_start(x_ref, A)
    r_64, _ = _rfactor_per_start(x_ref64, A)
    rel32 = np.abs(r_b200 - r_ref) / r_ref
    rel64 = np.abs(r_b200 - r_64) / r_64
    ref32_vs_64 = np.abs(r_ref - r_64) / r_64
    mean32 = abs(r_b200.mean() - r_ref.mean()) / r_ref.mean()
    mean64 = abs(r_b200.mean() - r_64.mean()) / r_64.mean()
    sup64 = np.mean(_support(x_b200) != _support(x_ref64))
    sup32 = np.mean(_support(x_b200) != _support(x_ref))
    sup_ref = np.mean(_support(x_ref) != _support(x_ref64))
    report = (f"carousel 128^2 x 90 angles x 10x10, {STARTS} starts: R-factor b200 {r_b200}, reference f32 {r_ref}, "
              f"reference f64 {r_64}; b200 vs f64 per start {rel64} (mean {mean64:.2e}); b200 vs f32 per start "
              f"{rel32} (mean {mean32:.2e}); reference f32 vs f64 per start {ref32_vs_64}; support differs: b200 vs "
              f"f64 {sup64:.2e}, b200 vs f32 {sup32:.2e}, reference f32 vs f64 {sup_ref:.2e}")
    print("\n" + report)
    assert mean64 < RFACTOR_MEAN_TOL_F64, report
    assert mean32 < RFACTOR_MEAN_TOL_F32, report
    assert np.all(rel64 < RFACTOR_START_TOL_F64), report
    assert sup64 <= 1.25 * sup_ref + 0.002, report
    # the final projection is real in all three (MKL_Impl.inl:70-84)
    assert np.all(x_b200.imag == 0) and np.all(x_ref.imag == 0) and np.all(x_ref64.imag == 0)
    assert np.all(np.isfinite(err))


@pytest.mark.parametrize("iters", [1, 5])
def test_dm_iterations_128_vs_reference(cuda, ref, carousel_data, iters):
    """The fused 128 x 128 kernel (one launch of `iters` iterations) against the
    reference operators, per iteration within 1e-5 relative L2."""
    import torch
    import cpra_b200 as cb
    B = 2
    A = np.ascontiguousarray(carousel_data["A"][7].ravel(), np.float32)
    S = np.ascontiguousarray(carousel_data["S"][7].ravel(), np.float32)
    rng = np.random.default_rng(iters)
    x0 = (rng.uniform(0, 1, B * M * N) + 1j * rng.uniform(0, 1, B * M * N)).astype(np.complex64)
    r = ref.RefImpl(np.float32, M, N, 1, B)
    xr, t1r, t2r = x0.copy(), x0.copy(), x0.copy()
    assert r.dm_iterations(xr, t1r, t2r, A, S, M * N * B, B, BETA, iters)
    impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, 1, B)
    x, t1, t2 = (torch.from_numpy(x0.copy()).cuda() for _ in range(3))
    assert impl.dm_iterations(x, t1, t2, torch.from_numpy(A).cuda(), torch.from_numpy(S).cuda(), B, BETA, iters)
    assert impl.Sync()
    for name, g, w in (("x", x, xr), ("t1", t1, t1r), ("t2", t2, t2r)):
        e = O.rel_l2(g.cpu().numpy(), w)
        assert e < FP32_DM_TOL * iters, f"{name}: rel L2 {e:.3e}"
    impl.close()


@pytest.mark.parametrize("init", [0, 1])
def test_tmem_kernel_equals_l2_kernel_bitwise(cuda, carousel_data, init):
    """k_dm_tm (x and t2 in tensor memory) writes the same bits as k_dm (x and
    t2 through L2): through the dm_iterations entry (t1, t2 from their
    buffers), and through cpra_run's angle launches (t1 = t2 = x after each of
    the three carousel mixes: first, middle and last angle)."""
    import torch
    import cpra_b200 as cb
    B, Pp, iters = 5, 3, 4
    rng = np.random.default_rng(100 + init)
    A = np.ascontiguousarray(carousel_data["A"][:Pp].ravel(), np.float32)
    S = np.ascontiguousarray(carousel_data["S"][:Pp].ravel(), np.float32)
    x0 = (rng.uniform(0, 1, Pp * B * M * N) + 1j * rng.uniform(0, 1, Pp * B * M * N)).astype(np.complex64)
    outs = []
    for tm in (0, 1):
        impl = cb.NewCpraImpl(cb.IMPL_TYPE.B200, M, N, 1, B)
        impl.set_option(cb.OPT_TMEM, tm)
        x = torch.from_numpy(x0.copy()).cuda()
        Ad, Sd = torch.from_numpy(A).cuda(), torch.from_numpy(S).cuda()
        if init:
            err = np.zeros(Pp * B, np.float32)
            assert impl.cpra_run(x, Ad, Sd, Pp, B, 2, iters, 0, BETA, final_step=True, err=err)
            assert impl.Sync()
            outs.append((x.cpu().numpy(), err.copy()))
        else:
            t1 = torch.from_numpy(x0[: B * M * N][::-1].copy()).cuda()
            t2 = torch.from_numpy((x0[: B * M * N] * 0.5).copy()).cuda()
            xv = x[: B * M * N]
            assert impl.dm_iterations(xv, t1, t2, Ad[: M * N], Sd[: M * N], B, BETA, iters) and impl.Sync()
            outs.append((xv.cpu().numpy(), t1.cpu().numpy(), t2.cpu().numpy()))
        impl.close()
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)
