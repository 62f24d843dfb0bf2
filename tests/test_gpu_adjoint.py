"""Hand-written adjoints of the amplitude loss through the slice operator
(project-defined): against the float64 oracle, against central finite
differences, and through a test-side torch.autograd.Function."""
import numpy as np
import pytest

import cpra_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tb(cuda):
    import torch
    import cpra_b200
    return torch, cpra_b200


def _problem(M, P, L, seed, dtype=np.complex64):
    rng = np.random.default_rng(seed)
    N = M
    V = (rng.standard_normal(L * N * M) + 1j * rng.standard_normal(L * N * M)).astype(dtype)
    ang = np.deg2rad(rng.uniform(3, 177, P)).astype(np.float64 if dtype == np.complex128 else np.float32)
    A = rng.uniform(0.2, 2.0, P * N * M).astype(np.float64 if dtype == np.complex128 else np.float32)
    return V, ang, A


def test_slice_vs_oracle(tb):
    torch, cb = tb
    M, P, L = 16, 5, 16
    V, ang, _ = _problem(M, P, L, 1)
    impl = cb.B200Impl(M, M, L, 1)
    out = torch.zeros(P * M * M, dtype=torch.complex64, device="cuda")
    assert impl.slice(torch.from_numpy(V).cuda(), torch.from_numpy(ang).cuda(), M, M, P, L, out) and impl.Sync()
    want = O.slice_volume(V, ang, M, M, P, L).ravel()
    assert O.rel_l2(out.cpu().numpy(), want) < 1e-6


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_loss_grad_vs_oracle(tb, dtype):
    torch, cb = tb
    M, P, L = 16, 6, 16
    cdt = np.complex64 if dtype == "float32" else np.complex128
    V, ang, A = _problem(M, P, L, 2, cdt)
    impl = cb.B200Impl(M, M, L, 1, dtype=dtype)
    gV = torch.zeros(V.size, dtype=torch.complex64 if dtype == "float32" else torch.complex128, device="cuda")
    loss, ga = impl.slice_loss_grad(torch.from_numpy(V).cuda(), torch.from_numpy(ang).cuda(),
                                    torch.from_numpy(A).cuda(), M, M, P, L, gV)
    lo, gVo, gao = O.slice_loss_grad(V, ang, A, M, M, P, L)
    tol = 1e-5 if dtype == "float32" else 1e-12
    assert abs(loss - lo) / lo < tol
    assert O.rel_l2(gV.cpu().numpy(), gVo.ravel()) < tol
    np.testing.assert_allclose(ga, gao, rtol=10 * tol, atol=10 * tol * np.abs(gao).max())


def test_loss_grad_vs_finite_differences(tb):
    """Central differences in float64: h = 1e-3 on the volume (the loss is smooth
    where |s| > 0); h = 1e-6 on the angles (bilinear weights have kinks where a
    sample point crosses a voxel plane, so a small step keeps both evaluations
    on one side of them).  Relative agreement 1e-4."""
    torch, cb = tb
    M, P, L = 12, 4, 12
    V, ang, A = _problem(M, P, L, 3, np.complex128)
    impl = cb.B200Impl(M, M, L, 1, dtype="float64")
    Vd, Ad = torch.from_numpy(V).cuda(), torch.from_numpy(A).cuda()
    gV = torch.zeros_like(Vd)
    _, ga = impl.slice_loss_grad(Vd, torch.from_numpy(ang).cuda(), Ad, M, M, P, L, gV)
    g = gV.cpu().numpy()

    def loss_at(Vh, angh):
        tmp = torch.zeros_like(Vd)
        l, _ = impl.slice_loss_grad(torch.from_numpy(Vh).cuda(), torch.from_numpy(angh).cuda(), Ad, M, M, P, L, tmp)
        return l

    rng = np.random.default_rng(0)
    # voxels that some slice samples (others have a zero gradient)
    touched = np.nonzero(np.abs(g) > 1e-6 * np.abs(g).max())[0]
    for k in rng.choice(touched, 8, replace=False):
        for unit, part in ((1.0, np.real), (1j, np.imag)):
            h = 1e-3
            Vp, Vm = V.copy(), V.copy()
            Vp[k] += unit * h
            Vm[k] -= unit * h
            fd = (loss_at(Vp, ang) - loss_at(Vm, ang)) / (2 * h)
            assert abs(fd - part(g[k])) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(g).max()), (k, fd, part(g[k]))
    for p in range(P):
        h = 1e-6
        ap, am = ang.copy(), ang.copy()
        ap[p] += h
        am[p] -= h
        fd = (loss_at(V, ap) - loss_at(V, am)) / (2 * h)
        assert abs(fd - ga[p]) <= 1e-4 * abs(fd), (p, fd, ga[p])


def test_autograd_function_and_refinement(tb):
    """A test-side torch.autograd.Function over the C ABI; a few gradient steps
    on the volume and the angles lower the loss of perturbed orientations."""
    torch, cb = tb
    M, P, L = 16, 8, 16
    impl = cb.B200Impl(M, M, L, 1)

    class SliceLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, Vr, ang, A):
            V = torch.view_as_complex(Vr.contiguous())
            gV = torch.zeros_like(V)
            loss, ga = impl.slice_loss_grad(V, ang.contiguous(), A, M, M, P, L, gV)
            ctx.save_for_backward(torch.view_as_real(gV), torch.from_numpy(ga).to(ang))
            return Vr.new_tensor(loss)

        @staticmethod
        def backward(ctx, gout):
            gVr, ga = ctx.saved_tensors
            return gout * gVr, gout * ga, None

    rng = np.random.default_rng(5)
    Vt = (rng.standard_normal(L * M * M) + 1j * rng.standard_normal(L * M * M)).astype(np.complex64)
    ang_t = np.deg2rad(np.linspace(10, 170, P)).astype(np.float32)
    out = torch.zeros(P * M * M, dtype=torch.complex64, device="cuda")
    impl.slice(torch.from_numpy(Vt).cuda(), torch.from_numpy(ang_t).cuda(), M, M, P, L, out)
    impl.Sync()
    A = out.abs().contiguous()
    Vr = torch.view_as_real(torch.from_numpy(Vt).cuda()).clone().requires_grad_(True)
    ang = (torch.from_numpy(ang_t).cuda() + torch.from_numpy(np.deg2rad(rng.normal(0, 0.5, P)).astype(np.float32)).cuda())
    ang.requires_grad_(True)
    opt = torch.optim.Adam([{"params": [ang], "lr": 1e-3}, {"params": [Vr], "lr": 1e-3}])
    losses = []
    for _ in range(25):
        opt.zero_grad()
        loss = SliceLoss.apply(Vr, ang, A)
        loss.backward()
        assert ang.grad is not None and Vr.grad is not None
        opt.step()
        losses.append(loss.item())
    assert losses[-1] < 0.5 * losses[0], losses


def test_refine_matches_torch_adam(tb):
    """cpra_b200_refine (device-side Adam over the adjoints) follows the same
    trajectory as torch.optim.Adam driven by the same gradients, and lowers the
    loss of perturbed orientations."""
    torch, cb = tb
    M, P, L, steps = 16, 8, 16, 25
    impl = cb.B200Impl(M, M, L, 1)
    rng = np.random.default_rng(5)
    Vt = (rng.standard_normal(L * M * M) + 1j * rng.standard_normal(L * M * M)).astype(np.complex64)
    ang_t = np.deg2rad(np.linspace(10, 170, P)).astype(np.float32)
    out = torch.zeros(P * M * M, dtype=torch.complex64, device="cuda")
    impl.slice(torch.from_numpy(Vt).cuda(), torch.from_numpy(ang_t).cuda(), M, M, P, L, out)
    impl.Sync()
    A = out.abs().contiguous()
    ang0 = (ang_t + np.deg2rad(rng.normal(0, 0.5, P))).astype(np.float32)

    # torch Adam over the same C-ABI gradients
    Vr = torch.view_as_real(torch.from_numpy(Vt).cuda()).clone().requires_grad_(True)
    ang = torch.from_numpy(ang0).cuda().clone().requires_grad_(True)
    opt = torch.optim.Adam([{"params": [ang], "lr": 1e-3}, {"params": [Vr], "lr": 1e-3}])
    want = []
    for _ in range(steps):
        opt.zero_grad()
        V = torch.view_as_complex(Vr.detach().contiguous())
        gV = torch.zeros_like(V)
        loss, ga = impl.slice_loss_grad(V, ang.detach().contiguous(), A, M, M, P, L, gV)
        Vr.grad = torch.view_as_real(gV).clone()
        ang.grad = torch.from_numpy(ga).to(ang)
        opt.step()
        want.append(loss)

    V = torch.from_numpy(Vt).cuda().clone()
    a = torch.from_numpy(ang0).cuda().clone()
    got = impl.refine(V, a, A, M, M, P, L, steps, lr_volume=1e-3, lr_angle=1e-3)
    assert got.shape == (steps,)
    np.testing.assert_allclose(got, want, rtol=1e-4)
    assert got[-1] < 0.5 * got[0], got
    Vw = torch.view_as_complex(Vr.detach().contiguous()).cpu().numpy()
    assert np.linalg.norm(V.cpu().numpy() - Vw) / np.linalg.norm(Vw) < 1e-4
    np.testing.assert_allclose(a.cpu().numpy(), ang.detach().cpu().numpy(), rtol=0, atol=1e-6)


def test_best_start(tb):
    """The start whose planes produced the modulus data wins (R = 0); the
    scores are the mean per-angle R-factors; best_out gathers its planes."""
    torch, cb = tb
    L, P, B, best = 64, 3, 5, 2
    rng = np.random.default_rng(11)
    x = (rng.standard_normal((P, B, L, L)) + 1j * rng.standard_normal((P, B, L, L))).astype(np.complex64)
    A = np.stack([np.abs(np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(x[p, best])))) for p in range(P)])
    A = A.astype(np.float32)
    impl = cb.B200Impl(L, L, 1, B)
    xd = torch.from_numpy(x.ravel()).cuda()
    out = torch.zeros(P * L * L, dtype=torch.complex64, device="cuda")
    b, scores = impl.best_start(xd, torch.from_numpy(A.ravel()).cuda(), P, B, best_out=out)
    impl.Sync()
    assert b == best
    want = [np.mean([O.rfactor(x[p, k].ravel(), A[p].ravel(), L, L, 1) for p in range(P)]) for k in range(B)]
    np.testing.assert_allclose(scores, want, rtol=1e-5, atol=1e-6)
    np.testing.assert_array_equal(out.cpu().numpy().reshape(P, L, L), x[:, best])


@pytest.mark.parametrize("P", [37, 4100])
def test_gathers_any_angles_vs_oracle(tb, P):
    """The gathers over slices (merge adjoint and trilinear merge) visit only the
    slices whose direction can reach a voxel (sorted table, up to 4096 slices)
    or all of them (above): both match the float64 oracle for angles over
    several turns, negative, beyond pi, repeated, and on 0 and pi exactly."""
    torch, cb = tb
    M, L = 8, 8
    rng = np.random.default_rng(P)
    V = (rng.standard_normal(L * M * M) + 1j * rng.standard_normal(L * M * M)).astype(np.complex128)
    ang = rng.uniform(-7.0, 9.0, P)
    ang[:4] = [0.0, np.pi, -np.pi, 2 * np.pi]
    ang[4:8] = ang[8:12]
    A = rng.uniform(0.2, 2.0, P * M * M)
    impl = cb.B200Impl(M, M, L, 1, dtype="float64")
    gV = torch.zeros(V.size, dtype=torch.complex128, device="cuda")
    loss, ga = impl.slice_loss_grad(torch.from_numpy(V).cuda(), torch.from_numpy(ang).cuda(),
                                    torch.from_numpy(A).cuda(), M, M, P, L, gV)
    lo, gVo, gao = O.slice_loss_grad(V, ang, A, M, M, P, L)
    assert abs(loss - lo) / lo < 1e-12
    assert O.rel_l2(gV.cpu().numpy(), gVo.ravel()) < 1e-12
    src = (rng.standard_normal(P * M * M) + 1j * rng.standard_normal(P * M * M)).astype(np.complex128)
    dst = torch.zeros(L * M * M, dtype=torch.complex128, device="cuda")
    assert impl.Complex2DTo3DInterpolation(torch.from_numpy(src).cuda(), dst, torch.from_numpy(ang).cuda(),
                                           M, M, P, L) and impl.Sync()
    want = O.complex2d_to_3d(np.float64, src, ang, M, M, P, L)
    assert O.rel_l2(dst.cpu().numpy(), want) < 1e-12


# ---- two orientation parameters per slice and the real-space volume -------------------
def _orient_problem(M, P, L, seed, dtype=np.complex64, rot_deg=3.0):
    V, ang, A = _problem(M, P, L, seed, dtype)
    rng = np.random.default_rng(seed + 100)
    rot = np.deg2rad(rng.uniform(-rot_deg, rot_deg, P)).astype(ang.dtype)
    return V, ang, rot, A


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_slice_orient_vs_oracle(tb, dtype):
    """Trilinear slices with tilt and in-plane rotation against the float64
    oracle: 1e-6 relative L2 in float (coordinates and weights in float,
    16^3 volume), 1e-13 in double; a null rotation array is the one-angle
    slice, bit for bit."""
    torch, cb = tb
    M, P, L = 16, 5, 16
    cdt = np.complex64 if dtype == "float32" else np.complex128
    V, ang, rot, _ = _orient_problem(M, P, L, 7, cdt)
    impl = cb.B200Impl(M, M, L, 1, dtype=dtype)
    tdt = torch.complex64 if dtype == "float32" else torch.complex128
    out = torch.zeros(P * M * M, dtype=tdt, device="cuda")
    Vd, ad = torch.from_numpy(V).cuda(), torch.from_numpy(ang).cuda()
    assert impl.slice_orient(Vd, ad, torch.from_numpy(rot).cuda(), M, M, P, L, out) and impl.Sync()
    want = O.slice_volume_orient(V, ang, rot, M, M, P, L).ravel()
    assert O.rel_l2(out.cpu().numpy(), want) < (1e-6 if dtype == "float32" else 1e-13)
    a = torch.zeros_like(out)
    b = torch.zeros_like(out)
    assert impl.slice_orient(Vd, ad, None, M, M, P, L, a) and impl.slice(Vd, ad, M, M, P, L, b) and impl.Sync()
    np.testing.assert_array_equal(a.cpu().numpy(), b.cpu().numpy())


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_loss_grad_orient_vs_oracle(tb, dtype):
    torch, cb = tb
    M, P, L = 16, 6, 16
    cdt = np.complex64 if dtype == "float32" else np.complex128
    V, ang, rot, A = _orient_problem(M, P, L, 8, cdt)
    impl = cb.B200Impl(M, M, L, 1, dtype=dtype)
    gV = torch.zeros(V.size, dtype=torch.complex64 if dtype == "float32" else torch.complex128, device="cuda")
    loss, ga, gr = impl.slice_loss_grad_orient(torch.from_numpy(V).cuda(), torch.from_numpy(ang).cuda(),
                                               torch.from_numpy(rot).cuda(), torch.from_numpy(A).cuda(),
                                               M, M, P, L, gV)
    lo, gVo, gao, gro = O.slice_loss_grad_orient(V, ang, rot, A, M, M, P, L)
    tol = 1e-5 if dtype == "float32" else 1e-12
    assert abs(loss - lo) / lo < tol
    assert O.rel_l2(gV.cpu().numpy(), gVo.ravel()) < tol
    np.testing.assert_allclose(ga, gao, rtol=10 * tol, atol=10 * tol * np.abs(gao).max())
    np.testing.assert_allclose(gr, gro, rtol=10 * tol, atol=10 * tol * np.abs(gro).max())


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_loss_grad_orient_dense_slices_vs_oracle(tb, dtype):
    """400 slices (dense: the adjoint gather takes two voxels along the tilt
    axis per work item from 360 slices on) against the float64 oracle, at
    the same tolerances as the sparse case."""
    torch, cb = tb
    M, P, L = 16, 400, 16
    cdt = np.complex64 if dtype == "float32" else np.complex128
    V, ang, rot, A = _orient_problem(M, P, L, 41, cdt)
    impl = cb.B200Impl(M, M, L, 1, dtype=dtype)
    gV = torch.zeros(V.size, dtype=torch.complex64 if dtype == "float32" else torch.complex128, device="cuda")
    loss, ga, gr = impl.slice_loss_grad_orient(torch.from_numpy(V).cuda(), torch.from_numpy(ang).cuda(),
                                               torch.from_numpy(rot).cuda(), torch.from_numpy(A).cuda(),
                                               M, M, P, L, gV)
    lo, gVo, gao, gro = O.slice_loss_grad_orient(V, ang, rot, A, M, M, P, L)
    tol = 1e-5 if dtype == "float32" else 1e-12
    assert abs(loss - lo) / lo < tol
    assert O.rel_l2(gV.cpu().numpy(), gVo.ravel()) < tol


def test_loss_grad_orient_vs_finite_differences(tb):
    """Central differences in float64: h = 1e-3 on the volume, h = 1e-6 on the
    tilts and rotations (trilinear weights have kinks where a sample point
    crosses a voxel plane; a small step stays on one side).  1e-4 relative."""
    torch, cb = tb
    M, P, L = 12, 4, 12
    V, ang, rot, A = _orient_problem(M, P, L, 9, np.complex128)
    impl = cb.B200Impl(M, M, L, 1, dtype="float64")
    Vd, Ad = torch.from_numpy(V).cuda(), torch.from_numpy(A).cuda()
    gV = torch.zeros_like(Vd)
    _, ga, gr = impl.slice_loss_grad_orient(Vd, torch.from_numpy(ang).cuda(), torch.from_numpy(rot).cuda(), Ad,
                                            M, M, P, L, gV)
    g = gV.cpu().numpy()

    def loss_at(Vh, angh, roth):
        tmp = torch.zeros_like(Vd)
        return impl.slice_loss_grad_orient(torch.from_numpy(Vh).cuda(), torch.from_numpy(angh).cuda(),
                                           torch.from_numpy(roth).cuda(), Ad, M, M, P, L, tmp)[0]

    rng = np.random.default_rng(1)
    touched = np.nonzero(np.abs(g) > 1e-6 * np.abs(g).max())[0]
    for k in rng.choice(touched, 6, replace=False):
        for unit, part in ((1.0, np.real), (1j, np.imag)):
            h = 1e-3
            Vp, Vm = V.copy(), V.copy()
            Vp[k] += unit * h
            Vm[k] -= unit * h
            fd = (loss_at(Vp, ang, rot) - loss_at(Vm, ang, rot)) / (2 * h)
            assert abs(fd - part(g[k])) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(g).max()), (k, fd, part(g[k]))
    for p in range(P):
        h = 1e-6
        for which, grad in ((0, ga), (1, gr)):
            ap, am, rp, rm = ang.copy(), ang.copy(), rot.copy(), rot.copy()
            if which == 0:
                ap[p] += h
                am[p] -= h
            else:
                rp[p] += h
                rm[p] -= h
            fd = (loss_at(V, ap, rp) - loss_at(V, am, rm)) / (2 * h)
            assert abs(fd - grad[p]) <= 1e-4 * abs(fd), (p, which, fd, grad[p])


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_volume_loss_grad_vs_oracle_and_finite_differences(tb, dtype):
    """The real-space chain (Forward3D, slice, modulus loss) and its adjoint
    (the slice adjoint, then the transform's adjoint) against the float64
    oracle (float: 1e-5; double: 1e-11) and, in double, central differences
    h = 1e-3 on single voxels (1e-4 relative)."""
    torch, cb = tb
    M = P = L = 16
    P = 6
    rng = np.random.default_rng(12)
    T = np.float32 if dtype == "float32" else np.float64
    vol = rng.standard_normal(L * M * M).astype(T)
    ang = np.deg2rad(rng.uniform(3, 177, P)).astype(T)
    rot = np.deg2rad(rng.uniform(-2, 2, P)).astype(T)
    A = rng.uniform(0.2, 40.0, P * M * M).astype(T)
    impl = cb.B200Impl(M, M, L, 1, dtype=dtype)
    vd, ad, rd, Ad = (torch.from_numpy(v).cuda() for v in (vol, ang, rot, A))
    g = torch.zeros_like(vd)
    loss, ga, gr = impl.volume_loss_grad(vd, ad, rd, Ad, M, M, P, L, g)
    lo, go, gao, gro = O.volume_loss_grad(vol, ang, rot, A, M, M, P, L)
    tol = 1e-5 if dtype == "float32" else 1e-11
    assert abs(loss - lo) / lo < tol
    assert O.rel_l2(g.cpu().numpy(), go.ravel()) < tol
    np.testing.assert_allclose(ga, gao, rtol=10 * tol, atol=10 * tol * np.abs(gao).max())
    np.testing.assert_allclose(gr, gro, rtol=10 * tol, atol=10 * tol * np.abs(gro).max())
    if dtype == "float64":
        gg = g.cpu().numpy()
        tmp = torch.zeros_like(vd)
        for k in rng.choice(vol.size, 6, replace=False):
            h = 1e-3
            vp, vm = vol.copy(), vol.copy()
            vp[k] += h
            vm[k] -= h
            lp = impl.volume_loss_grad(torch.from_numpy(vp).cuda(), ad, rd, Ad, M, M, P, L, tmp)[0]
            lm = impl.volume_loss_grad(torch.from_numpy(vm).cuda(), ad, rd, Ad, M, M, P, L, tmp)[0]
            fd = (lp - lm) / (2 * h)
            assert abs(fd - gg[k]) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(gg).max()), (k, fd, gg[k])


def test_refine_orient_recovers_tilt_and_rotation(tb):
    """Slices of a known real-space volume at jittered orientations (tilt and
    in-plane rotation, 1 degree rms): refining both from the nominal
    orientations through the hand-written adjoints, with the volume held
    (lr_volume 0), brings the rms orientation error below a third of the
    jitter; the loss falls."""
    torch, cb = tb
    M = L = 32
    P = 24
    rng = np.random.default_rng(21)
    z, y, x = np.meshgrid(*(np.arange(M) - M / 2,) * 3, indexing="ij")
    vol = np.zeros((L, M, M), np.float32)
    for _ in range(6):
        c = rng.uniform(-6, 6, 3)
        a = rng.uniform(2, 5, 3)
        vol[(((z - c[0]) / a[0]) ** 2 + ((y - c[1]) / a[1]) ** 2 + ((x - c[2]) / a[2]) ** 2) <= 1] += rng.uniform(0.3, 1)
    vol = vol.ravel()
    nominal = np.deg2rad(np.arange(P) * 180.0 / P).astype(np.float32)
    jit = np.deg2rad(1.0)
    a_true = (nominal + rng.normal(0, jit, P)).astype(np.float32)
    r_true = rng.normal(0, jit, P).astype(np.float32)
    impl = cb.B200Impl(M, M, L, 1)
    VF = torch.from_numpy(vol.astype(np.complex64)).cuda()
    assert impl.Forward3D(VF) and impl.Sync()
    out = torch.zeros(P * M * M, dtype=torch.complex64, device="cuda")
    assert impl.slice_orient(VF, torch.from_numpy(a_true).cuda(), torch.from_numpy(r_true).cuda(), M, M, P, L, out)
    impl.Sync()
    A = out.abs().contiguous()
    v = torch.from_numpy(vol).cuda()
    a = torch.from_numpy(nominal).cuda()
    r = torch.zeros(P, dtype=torch.float32, device="cuda")
    rms0 = np.sqrt(np.mean((nominal - a_true) ** 2 + r_true ** 2))
    losses = impl.refine_orient(v, a, r, A, M, M, P, L, 150, real_space=True, lr_volume=0.0, lr_angle=2e-3,
                                lr_rot=2e-3)
    rms1 = np.sqrt(np.mean((a.cpu().numpy() - a_true) ** 2 + (r.cpu().numpy() - r_true) ** 2))
    assert losses[-1] < 0.1 * losses[0], losses[[0, -1]]
    assert rms1 < rms0 / 3, (np.rad2deg(rms0), np.rad2deg(rms1))
    np.testing.assert_array_equal(v.cpu().numpy(), vol)   # lr_volume 0 holds the volume


@pytest.mark.parametrize("P", [90, 400])
def test_gathers_deterministic_with_dynamic_voxels(tb, P):
    """The merge and the adjoint gather hand their work to the resident
    warps from a counter, in whatever order the warps come; each voxel is
    still summed by one thread in a fixed order, so repeated calls (the
    counter reused, the context fresh or not) give the same bits (at 400
    slices the adjoint takes two voxels per work item)."""
    torch, cb = tb
    M, L = 64, 64
    V, ang, A = _problem(M, P, L, 31)
    rot = (np.random.default_rng(32).standard_normal(P) * 0.005).astype(np.float32)
    Vd, angd, Ad, rotd = (torch.from_numpy(a).cuda() for a in (V, ang, A, rot))
    src = torch.from_numpy(
        (np.random.default_rng(33).standard_normal(P * M * M) * (1 + 1j)).astype(np.complex64)).cuda()
    outs = []
    for fresh in (True, False, True):
        impl = cb.B200Impl(M, M, L, 1) if fresh or not outs else impl
        gV = torch.zeros_like(Vd)
        impl.slice_loss_grad_orient(Vd, angd, rotd, Ad, M, M, P, L, gV)
        merged = torch.zeros_like(Vd)
        assert impl.Complex2DTo3DInterpolation(src, merged, angd, M, M, P, L) and impl.Sync()
        outs.append((gV.cpu().numpy(), merged.cpu().numpy()))
    for o in outs[1:]:
        for a, b in zip(outs[0], o):
            np.testing.assert_array_equal(a, b)
