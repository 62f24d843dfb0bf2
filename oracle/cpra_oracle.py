"""CPU oracle for the carousel phase-retrieval hot path (test infrastructure only).

This module is the CHECKER, not the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may import it.  The B200 backend never routes through it.

It restates, in numpy, the arithmetic of the reference's operator backend
``MklImpl<T>`` (``include/MKL_Impl.hpp``, ``include/detail/MKL_Impl.inl``) and
the call sequences of its driver programs (``src/CPRA_MKL.cpp``,
``src/CONV_MKL.cpp``, ``src/benchmark_mkl.cpp``), with each function citing the
reference file:line it follows.  Arrays are flat numpy arrays (views allowed),
mutated in place exactly like the reference mutates its raw pointers, so the
restated drivers read like the reference's own.

Precision model: ``T`` is ``np.float32`` or ``np.float64``.  Every operator
takes T-rounded inputs, evaluates in float64 where the reference calls a
library (DFTI FFT, polar/arg) and rounds its result to T once, which is the
correctly-rounded-per-operator reading of the reference.  Element-wise
arithmetic that the reference spells out (axpby, scaling, the 0.9 threshold
compare) is evaluated in T with the same operation order and no fused
multiply-add.

Pinning: ``tests/test_oracle_pins.py`` checks this module against the
reference's own known-answer tests (``test/unitest_mkl.cpp:15-71``) and against
the reference ``MklImpl<T>`` source compiled here (``oracle/_ref``) on seeded
inputs; ``tests/golden/`` holds fixtures produced by that compiled reference.
The FFT itself is pinned to oneMKL 2024.1 DFTI only through the 10x10 KAT
(oneMKL is not installable here).
"""
from __future__ import annotations

import math
import numpy as np

__all__ = [
    "OracleImpl", "cpra_sample", "conv_sample", "dm_iteration",
    "rel_l2", "complex_dtype",
]


def complex_dtype(T):
    return np.complex64 if np.dtype(T) == np.float32 else np.complex128


def rel_l2(a, b):
    """Relative L2 distance ||a-b|| / ||b|| evaluated in float64."""
    a = np.asarray(a).astype(np.complex128).ravel()
    b = np.asarray(b).astype(np.complex128).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def _threshold_mask(S):
    """``S < 0.9`` with S promoted to double, as in MKL_Impl.inl:83
    (``flat_constr_data[...] < 0.9`` compares a T against a double literal)."""
    return np.asarray(S).astype(np.float64) < 0.9


class OracleImpl:
    """numpy restatement of ``CpraImpl<T>`` as implemented by ``MklImpl<T>``.

    Construction mirrors ``MklImpl(m, n, l, batch_size)``
    (``include/MKL_Impl.hpp:14-121``): the 2D/3D transform shapes and batch are
    fixed here, element-wise operators take explicit sizes.  Methods return
    ``bool`` with the reference's argument checks (``MKL_Impl.inl:11,34,55,73,
    89,112``).
    """

    def __init__(self, T, m, n, l, batch_size, space_mode="mkl"):
        self.T = np.dtype(T).type
        self.C = complex_dtype(T)
        self.m, self.n, self.l, self.batch = int(m), int(n), int(l), int(batch_size)
        # "mkl": MKL_Impl.inl:70-84 (threshold 0.9, no positivity);
        # "cuda": CUDA_Impl_Kernel.cuh:16-28 (positivity times mask value).
        self.space_mode = space_mode

    # -- MKL_Impl.inl:7-29 -------------------------------------------------
    def Initialize(self, flat, num, seed=0):
        """Uniform [0,1) fill.  The reference seeds a thread_local mt19937 per
        OpenMP thread (MKL_Impl.inl:16), so its values are not reproducible;
        the oracle uses a seeded numpy generator and tests check only range."""
        if num < 1:
            return False
        rng = np.random.default_rng(seed)
        flat[:num] = rng.random(num, dtype=np.float64).astype(self.T)
        return True

    # -- MKL_Impl.inl:180-209 ----------------------------------------------
    def FFTShift2D(self, x, M, N, Batch):
        """Quadrant swap of each MxN plane (even M, N), MKL_Impl.inl:180-209."""
        a = x[: M * N * Batch].reshape(Batch, M, N)
        a[...] = np.roll(a, (M // 2, N // 2), axis=(1, 2))
        return True

    # -- MKL_Impl.inl:212-251 ----------------------------------------------
    def FFTShift3D(self, x, M, N, L, Batch):
        """Octant swap of each [L][M][N] volume (even sizes), MKL_Impl.inl:212-251
        (index ``dep*M*N + row*N + col``)."""
        a = x[: M * N * L * Batch].reshape(Batch, L, M, N)
        a[...] = np.roll(a, (L // 2, M // 2, N // 2), axis=(1, 2, 3))
        return True

    # -- MKL_Impl.inl:128-139, MKL_Impl.hpp:24-44 ---------------------------
    def _fft(self, x, shape, inverse):
        a = x[: int(np.prod(shape)) * self.batch].reshape((self.batch,) + shape)
        axes = tuple(range(1, len(shape) + 1))
        v = a.astype(np.complex128)
        if inverse:
            # DFTI backward with DFTI_BACKWARD_SCALE = 1/(prod shape),
            # MKL_Impl.hpp:40 (scale stored as T)
            scale = float(self.T(1.0) / self.T(int(np.prod(shape))))
            v = np.fft.ifftn(v, axes=axes) * (np.prod(shape) * scale)
        else:
            v = np.fft.fftn(v, axes=axes)
        a[...] = v.astype(self.C)

    def Forward2D(self, x):
        """fftshift -> unscaled forward DFT -> fftshift (MKL_Impl.inl:128-139)."""
        self.FFTShift2D(x, self.m, self.n, self.batch)
        self._fft(x, (self.m, self.n), inverse=False)
        self.FFTShift2D(x, self.m, self.n, self.batch)
        return True

    def Backward2D(self, x):
        """fftshift -> backward DFT scaled by 1/(MN) -> fftshift (MKL_Impl.inl:141-152)."""
        self.FFTShift2D(x, self.m, self.n, self.batch)
        self._fft(x, (self.m, self.n), inverse=True)
        self.FFTShift2D(x, self.m, self.n, self.batch)
        return True

    def Forward3D(self, x):
        """3D analogue on [L][M][N] volumes (MKL_Impl.inl:154-165).  The
        reference's 3D descriptor is built from the 2-element ``dim2D``
        (MKL_Impl.hpp:46-47, undefined behaviour); this restates the intended
        rank-3 DFT over (L, M, N)."""
        self.FFTShift3D(x, self.m, self.n, self.l, self.batch)
        self._fft(x, (self.l, self.m, self.n), inverse=False)
        self.FFTShift3D(x, self.m, self.n, self.l, self.batch)
        return True

    def Backward3D(self, x):
        """MKL_Impl.inl:167-178 with scale 1/(MNL) (MKL_Impl.hpp:62)."""
        self.FFTShift3D(x, self.m, self.n, self.l, self.batch)
        self._fft(x, (self.l, self.m, self.n), inverse=True)
        self.FFTShift3D(x, self.m, self.n, self.l, self.batch)
        return True

    # -- MKL_Impl.inl:70-84 --------------------------------------------------
    def SpaceConstraint(self, x, S, num, batch_size):
        if num == 0 or batch_size == 0:
            return False
        plane = num // batch_size
        idx = np.arange(num) % plane
        s = np.asarray(S)[idx]
        v = x[:num]
        if self.space_mode == "mkl":
            re = v.real.copy()
            re[_threshold_mask(s)] = 0
        else:  # CUDA_Impl_Kernel.cuh:16-28
            re = v.real.copy()
            neg = re < 0
            re = (re * s).astype(self.T)
            re[neg] = 0
        v.real = re
        v.imag = 0
        return True

    # -- MKL_Impl.inl:86-106 -------------------------------------------------
    def DataConstraint(self, x, A, num, batch_size):
        """Real (modulus) or complex constraint, chosen by A's dtype like the
        reference's two overloads (MKL_Impl.inl:86-106 and :108-126)."""
        if num == 0 or batch_size == 0:
            return False
        plane = num // batch_size
        idx = np.arange(num) % plane
        a = np.asarray(A)[idx]
        v = x[:num]
        if np.iscomplexobj(a):
            # MKL_Impl.inl:108-126: if |C|^2 != 0: z = C
            cr, ci = a.real.astype(self.T), a.imag.astype(self.T)
            keep = (cr * cr + ci * ci) != 0
            v[keep] = a[keep]
            return True
        re, im = v.real.astype(self.T), v.imag.astype(self.T)
        nrm = re * re + im * im                      # std::norm in T
        upd = (a != 0) & (nrm > 0)                    # A==0 unconstrained (:98-104)
        r64, i64 = re[upd].astype(np.float64), im[upd].astype(np.float64)
        mag = np.hypot(r64, i64)
        amp = a[upd].astype(np.float64)
        # std::polar(A, std::arg(z)) == A * z / |z|
        v[upd] = ((amp * r64 / mag) + 1j * (amp * i64 / mag)).astype(self.C)
        return True

    # -- MKL_Impl.inl:31-50 --------------------------------------------------
    def MergeAddData(self, src, dst, alpha, beta, num):
        """dst = alpha*src + beta*dst (cblas_?axpby with real coefficients)."""
        if alpha == 0 or num == 0:
            return False
        a, b = self.T(alpha), self.T(beta)
        s = src[:num].copy()          # src may alias dst (unitest_mkl.cpp:33)
        d = dst[:num]
        sv = s.view(self.T)
        dv = d.view(self.T)
        dv[...] = (a * sv).astype(self.T) + (b * dv).astype(self.T)
        return True

    # -- MKL_Impl.inl:52-68 --------------------------------------------------
    def Normalization(self, x, norm, num):
        """x *= 1/norm (cblas_?scal with T(1.0/norm))."""
        if norm == 0 or num == 0:
            return False
        a = self.T(1.0 / float(norm))
        xv = x[:num].view(self.T)
        xv[...] = (xv * a).astype(self.T)
        return True

    # -- CUDA_Impl.inl:145-172 (the MKL backend's version is a stub) --------
    def ConvergeError(self, old, new, err, m, n, l=1, batch_size=1):
        """old <- new - old over m*n*l*batch; err[i] = ||old_i|| / ||new_i||,
        each norm over the first m*n elements of member i (stride m*n*l),
        as CUDA_Impl.inl:157-158 computes it."""
        num = m * n * l * batch_size
        self.MergeAddData(new, old, 1.0, -1.0, num)
        for i in range(batch_size):
            o = old[i * m * n * l: i * m * n * l + m * n].astype(np.complex128)
            w = new[i * m * n * l: i * m * n * l + m * n].astype(np.complex128)
            err[i] = self.T(np.linalg.norm(o) / np.linalg.norm(w))
        return True

    def Memcpy(self, dst, src, nbytes):
        """MKL_Impl.hpp:159-162 copies with std::memcpy (its missing return is
        a reference defect; the oracle returns True)."""
        cnt = nbytes // np.dtype(self.C).itemsize
        dst[:cnt] = src[:cnt]
        return True

    def Sync(self):
        return True


def dm_iteration(impl, x, t1, t2, A, S, num, batch, beta):
    """One difference-map iteration, src/CPRA_MKL.cpp:94-110 (same call order,
    same coefficient expressions evaluated in double then passed as T).
    ``beta`` is first rounded to T: the driver's Beta parameter is a T."""
    b = float(impl.T(beta))
    impl.Forward2D(t1)
    impl.DataConstraint(t1, A, num, batch)
    impl.Backward2D(t1)
    impl.MergeAddData(x, t1, -1.0 / b, 1.0 + 1.0 / b, num)
    impl.SpaceConstraint(t1, S, num, batch)
    impl.SpaceConstraint(t2, S, num, batch)
    impl.MergeAddData(x, t2, 1.0 / b, 1.0 - 1.0 / b, num)
    impl.Forward2D(t2)
    impl.DataConstraint(t2, A, num, batch)
    impl.Backward2D(t2)
    impl.MergeAddData(t1, x, b, 1.0, num)
    impl.MergeAddData(t2, x, -1.0 * b, 1.0, num)


def cpra_sample(T, M, N, L, P, B, A, S, x0, epi, iters, pre_iter, beta,
                t1_0=None, t2_0=None, with_error=True):
    """Restated ``ShrinkWrap_CPRA_MKL_Sample`` (src/CPRA_MKL.cpp:10-154).

    ``x0`` replaces the reference's ``Initialize`` fill (:21-23) by a seeded
    initial guess of shape [P][B][M][N]; t1/t2 initial contents are overwritten
    by the Memcpy at :35-36 before first use, so they do not matter.
    Returns (x [P*B*M*N] complex, err [P*B] T).
    """
    T = np.dtype(T).type
    C = complex_dtype(T)
    impl = OracleImpl(T, M, N, L, B)
    beta = float(T(beta))
    MNB = M * N * B
    x = np.ascontiguousarray(np.asarray(x0, dtype=C).ravel()).copy()
    t1 = np.zeros(MNB, C) if t1_0 is None else np.asarray(t1_0, C).ravel().copy()
    t2 = np.zeros(MNB, C) if t2_0 is None else np.asarray(t2_0, C).ravel().copy()
    old = np.zeros(MNB, C)
    err = np.zeros(P * B, T)
    A = np.asarray(A, T).ravel()
    S = np.asarray(S, T).ravel()
    nbytes = np.dtype(C).itemsize * MNB
    # Step A, pre-reconstruction on angle 0 (:35-55)
    impl.Memcpy(t1, x, nbytes)
    impl.Memcpy(t2, x, nbytes)
    for _ in range(pre_iter):
        dm_iteration(impl, x[:MNB], t1, t2, A, S, MNB, B, beta)
    impl.Sync()
    # Step B, episodes over the carousel angles, Gauss-Seidel order (:59-124)
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
            impl.Memcpy(t1, xp, nbytes)
            impl.Memcpy(t2, xp, nbytes)
            Ap = A[M * N * p: M * N * (p + 1)]
            Sp = S[M * N * p: M * N * (p + 1)]
            for i in range(iters):
                last = with_error and (i == iters - 1 and e == epi - 1)
                if last:
                    impl.Memcpy(old, xp, nbytes)
                dm_iteration(impl, xp, t1, t2, Ap, Sp, MNB, B, beta)
                if last:
                    impl.Memcpy(t1, xp, nbytes)
                    impl.Forward2D(old)
                    impl.Forward2D(t1)
                    impl.ConvergeError(old, t1, err[B * p: B * (p + 1)], M, N, 1, B)
    # Final projection (:126-140)
    for p in range(P):
        xp = x[MNB * p: MNB * (p + 1)]
        Ap = A[M * N * p: M * N * (p + 1)]
        Sp = S[M * N * p: M * N * (p + 1)]
        impl.Memcpy(t1, xp, nbytes)
        impl.Forward2D(t1)
        impl.DataConstraint(t1, Ap, MNB, B)
        impl.Backward2D(t1)
        impl.MergeAddData(xp, t1, -1.0 / beta, 1.0 + 1.0 / beta, MNB)
        impl.SpaceConstraint(t1, Sp, MNB, B)
        impl.Memcpy(xp, t1, nbytes)
    impl.Sync()
    return x, err


def conv_sample(T, M, N, L, B, A, S, x0, iters, beta):
    """Restated ``ShrinkWrap_CONV_MKL_Sample`` (src/CONV_MKL.cpp:10-101): the
    same DM update on [L][M][N] volumes with the 3D transforms and the real
    modulus constraint.  Returns (x, err[B])."""
    T = np.dtype(T).type
    C = complex_dtype(T)
    impl = OracleImpl(T, M, N, L, B)
    num = M * N * L * B
    x = np.asarray(x0, C).ravel().copy()
    t1 = np.zeros(num, C)
    t2 = np.zeros(num, C)
    old = np.zeros(num, C)
    err = np.zeros(B, T)
    A = np.asarray(A, T).ravel()
    S = np.asarray(S, T).ravel()
    nbytes = np.dtype(C).itemsize * num
    b = float(T(beta))
    impl.Memcpy(t1, x, nbytes)
    impl.Memcpy(t2, x, nbytes)
    for i in range(iters):
        if i == iters - 1:
            impl.Memcpy(old, x, nbytes)
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
        if i == iters - 1:
            impl.Memcpy(t1, x, nbytes)
            impl.Forward3D(old)
            impl.Forward3D(t1)
            impl.ConvergeError(old, t1, err, M, N, L, B)
    impl.Memcpy(t1, x, nbytes)
    impl.Forward3D(t1)
    impl.DataConstraint(t1, A, num, B)
    impl.Backward3D(t1)
    impl.MergeAddData(x, t1, -1.0 / b, 1.0 + 1.0 / b, num)
    impl.SpaceConstraint(t1, S, num, B)
    impl.Memcpy(x, t1, nbytes)
    return x, err


def real2d_to_3d(T, src, angles, m, n, p, l):
    """Deterministic restatement of ``ker_Real2DTo3DInterpolation`` +
    ``ker_NormRealInterpolation`` (CUDA_Impl_Kernel.cuh:68-119, launched by
    CUDA_Impl.inl:174-197).

    Slice pixel i of P column-major MxN slices maps to a 3D point rotated about
    the y axis by angles[z]; its nearest voxel receives weight 50 (distance
    <= 0.02) or 1/distance, pixels with distance >= 0.5 or an out-of-range
    flat index are skipped.  The reference's ``return`` (:94-95) drops the rest
    of a thread's grid-stride items and its ``+=`` races (:99-105); here every
    pixel is visited once and contributions are summed in float64 before the
    T-rounded division by the weight, which is the kernel's intended result.
    """
    T = np.dtype(T).type
    M, N, P, L = int(m), int(n), int(p), int(l)
    src = np.asarray(src, T).ravel()[: M * N * P]
    ang = np.asarray(angles, T).ravel()[:P].astype(np.float64)
    i = np.arange(M * N * P, dtype=np.int64)
    zin = i // (M * N)
    xin = (i - M * N * zin) // M
    yin = (i - M * N * zin) - M * xin
    xr = xin.astype(np.float64) - N / 2.0
    yr = -yin.astype(np.float64) + M / 2.0
    a = ang[zin]
    x3 = yr * np.sin(a)
    y3 = xr
    z3 = yr * np.cos(a)
    j = np.rint(x3)            # round-half-even differs from C round() only at .5
    k = np.rint(y3)
    ll = np.rint(z3)
    # C round(): half away from zero
    j = np.where(np.abs(x3 - np.trunc(x3)) == 0.5, np.trunc(x3) + np.sign(x3), j)
    k = np.where(np.abs(y3 - np.trunc(y3)) == 0.5, np.trunc(y3) + np.sign(y3), k)
    ll = np.where(np.abs(z3 - np.trunc(z3)) == 0.5, np.trunc(z3) + np.sign(z3), ll)
    j, k, ll = j.astype(np.int64), k.astype(np.int64), ll.astype(np.int64)
    z = L // 2 - j
    x = N // 2 + k
    y = M // 2 - ll
    index = z * M * N + x * M + y
    dist = np.sqrt((x3 - j) ** 2 + (y3 - k) ** 2 + (z3 - ll) ** 2)
    ok = (index < M * N * L) & (index >= 0) & (dist < 0.5)
    w = np.where(dist <= 0.02, 50.0, 1.0 / np.maximum(dist, 1e-300))
    acc = np.zeros(M * N * L, np.float64)
    wt = np.zeros(M * N * L, np.float64)
    np.add.at(acc, index[ok], (w * src.astype(np.float64))[ok])
    np.add.at(wt, index[ok], w[ok])
    out = acc.astype(T)
    nz = wt > 0
    out[nz] = (acc[nz] / wt[nz]).astype(T)
    return out


def rfactor(x, A, M, N, batch, a_stride=0):
    """Project-defined R-factor (no counterpart in the reference, whose only
    metric is ConvergeError): for pattern b,
        R_b = sum | |Forward2D(x_b)| - A_b | / sum A_b
    with Forward2D the reference's shift-DFT-shift (MKL_Impl.inl:128-139),
    evaluated here entirely in float64."""
    x = np.asarray(x).astype(np.complex128).ravel()[: batch * M * N].copy()
    impl = OracleImpl(np.float64, M, N, 1, batch)
    impl.Forward2D(x)
    F = np.abs(x.reshape(batch, M * N))
    A = np.asarray(A, np.float64).ravel()
    out = np.zeros(batch)
    for b in range(batch):
        a = A[b * a_stride: b * a_stride + M * N]
        out[b] = np.abs(F[b] - a).sum() / a.sum()
    return out


def complex2d_to_3d(T, src, angles, m, n, p, l):
    """Project-defined trilinear gather merge of P complex central slices into
    a [L][N][M] volume (the reference's Complex2DTo3DInterpolation is a stub,
    include/CUDA_Impl.cuh:89), in the geometry of the real merge
    (CUDA_Impl_Kernel.cuh:68-119): voxel (z, x, y) is the point
    (j, k, l) = (L/2 - z, x - N/2, M/2 - y); slice p at angle a sees it at
    in-plane row yIn = M/2 - (j sin a + l cos a), column xIn = x, and at
    distance d = j cos a - l sin a from its plane.  Slices with |d| < 1 add
    (1 - |d|) times the slice sampled linearly in yIn; the voxel is the
    weight-normalised sum (0 where nothing reaches it)."""
    T = np.dtype(T).type
    M, N, P, L = int(m), int(n), int(p), int(l)
    src = np.asarray(src).astype(np.complex128).reshape(P, N, M)
    ang = np.asarray(angles, T).astype(np.float64)[:P]
    z, x, y = np.meshgrid(np.arange(L), np.arange(N), np.arange(M), indexing="ij")
    j = (L // 2 - z).astype(np.float64)
    ll = (M // 2 - y).astype(np.float64)
    acc = np.zeros((L, N, M), np.complex128)
    wsum = np.zeros((L, N, M))
    for q in range(P):
        sa, ca = np.sin(ang[q]), np.cos(ang[q])
        d = j * ca - ll * sa
        wd = 1.0 - np.abs(d)
        yin = (M // 2) - (j * sa + ll * ca)
        y0 = np.floor(yin)
        fy = yin - y0
        y0 = y0.astype(np.int64)
        s = np.zeros_like(acc)
        sw = np.zeros_like(wsum)
        for dy in (0, 1):
            yy = y0 + dy
            wy = fy if dy else 1.0 - fy
            ok = (yy >= 0) & (yy < M) & (wy != 0)
            v = np.zeros_like(acc)
            v[ok] = src[q, x[ok], yy[ok]]
            s += np.where(ok, wy, 0.0) * v
            sw += np.where(ok, wy, 0.0)
        use = (wd > 0) & (sw > 0)
        acc[use] += wd[use] * s[use]
        wsum[use] += wd[use] * sw[use]
    out = np.zeros((L, N, M), np.complex128)
    nz = wsum > 0
    out[nz] = acc[nz] / wsum[nz]
    return out.astype(complex_dtype(T)).ravel()


def gaussian_transfer(L, sigma):
    """DFT of the normalised periodic Gaussian g[n] ~ exp(-min(n, L-n)^2 /
    (2 sigma^2)), real and even (float64)."""
    n = np.arange(L)
    d = np.minimum(n, L - n).astype(np.float64)
    g = np.exp(-d * d / (2.0 * sigma * sigma))
    g /= g.sum()
    return np.real(np.fft.fft(g))


def hio_shrinkwrap(x0, A, S0, L, batch, iters, beta, sw_every=0, sigma_start=3.0, sigma_end=1.5, threshold=0.1,
                   positivity=False, a_stride=None, s_stride=None):
    """Project-defined hybrid input-output with shrinkwrap, float64 (the
    reference has neither; its operator composition supplies the modulus
    projection y = Backward2D(DataConstraint(Forward2D(x))),
    MKL_Impl.inl:86-152).  Per iteration: x <- y inside the support (and
    Re y >= 0 with positivity), x <- x - beta*y elsewhere.  Every sw_every
    iterations the support becomes {v > threshold * max v}, v = |x| circularly
    blurred by a normalised periodic Gaussian, sigma linear from sigma_start at
    the first update to sigma_end at the last.  Returns (x, S, estimate) with
    estimate = S (.) y of the final x."""
    plane = L * L
    a_stride = plane if a_stride is None else a_stride
    s_stride = plane if s_stride is None else s_stride
    x0 = np.asarray(x0).astype(np.complex128).ravel()
    A = np.asarray(A, np.float64).ravel()
    S0 = np.asarray(S0, np.float64).ravel()
    updates = iters // sw_every if sw_every else 0
    impl = OracleImpl(np.float64, L, L, 1, 1)
    xs, ss, es = [], [], []
    for b in range(batch):
        x = x0[b * plane:(b + 1) * plane].copy()
        a = A[b * a_stride: b * a_stride + plane]
        S = S0[b * s_stride: b * s_stride + plane] > 0.5
        k = 0
        for it in range(iters):
            y = x.copy()
            impl.Forward2D(y)
            impl.DataConstraint(y, a, plane, 1)
            impl.Backward2D(y)
            inside = S & (y.real >= 0) if positivity else S
            x = np.where(inside, y, x - beta * y)
            if updates and (it + 1) % sw_every == 0:
                sg = sigma_start + (sigma_end - sigma_start) * k / (updates - 1) if updates > 1 else sigma_start
                k += 1
                g = gaussian_transfer(L, sg)
                v = np.real(np.fft.ifft2(np.fft.fft2(np.abs(x).reshape(L, L)) * np.outer(g, g))).ravel()
                S = v > threshold * v.max()
        y = x.copy()
        impl.Forward2D(y)
        impl.DataConstraint(y, a, plane, 1)
        impl.Backward2D(y)
        xs.append(x)
        ss.append(S.astype(np.float64))
        es.append(np.where(S, y, 0))
    return np.concatenate(xs), np.concatenate(ss), np.concatenate(es)


def _orient_weights(M, N, L, a, r=0.0):
    """Trilinear sampling of one slice with tilt a and in-plane rotation r
    (the slice operator's geometry, project-defined; r = 0 is the merges'
    bilinear sample on the plane x = xIn): for every slice pixel, [N][M] with
    yIn fastest, the (z, x, y) of its up to eight voxels, their weights and the
    weights' derivatives in a and r (float64).  xr = xIn - N/2, yr = M/2 - yIn,
    xq = xr cos r - yr sin r, yq = xr sin r + yr cos r; the point is
    z = L/2 - yq sin a, x = N/2 + xq, y = M/2 - yq cos a."""
    xIn, yIn = np.meshgrid(np.arange(N), np.arange(M), indexing="ij")
    xr, yr = (xIn - N // 2).astype(np.float64), (M // 2 - yIn).astype(np.float64)
    sa, ca, sr, cr = np.sin(a), np.cos(a), np.sin(r), np.cos(r)
    xq, yq = cr * xr - sr * yr, sr * xr + cr * yr
    pts = (L // 2 - yq * sa, N // 2 + xq, M // 2 - yq * ca)
    d_a = (-yq * ca, np.zeros_like(yq), yq * sa)
    d_r = (-xq * sa, -yq, -xq * ca)
    lo = [np.floor(q).astype(np.int64) for q in pts]
    out = []
    for cz in (0, 1):
        for cx in (0, 1):
            for cy in (0, 1):
                idx, w, ga, gr = [], [], [], []
                for q, l0, c, da, dr in zip(pts, lo, (cz, cx, cy), d_a, d_r):
                    v = l0 + c
                    u = q - v
                    idx.append(v)
                    w.append(np.maximum(0.0, 1.0 - np.abs(u)))
                    sg = np.where(u >= 0, -1.0, 1.0)
                    ga.append(sg * da)
                    gr.append(sg * dr)
                z, x, y = idx
                ok = (z >= 0) & (z < L) & (x >= 0) & (x < N) & (y >= 0) & (y < M) & (w[0] > 0) & (w[1] > 0) & (w[2] > 0)
                wt = w[0] * w[1] * w[2]
                dwa = ga[0] * w[1] * w[2] + w[0] * ga[1] * w[2] + w[0] * w[1] * ga[2]
                dwr = gr[0] * w[1] * w[2] + w[0] * gr[1] * w[2] + w[0] * w[1] * gr[2]
                out.append((np.where(ok, z, 0), np.where(ok, x, 0), np.where(ok, y, 0), ok, np.where(ok, wt, 0.0),
                            np.where(ok, dwa, 0.0), np.where(ok, dwr, 0.0)))
    return out


def slice_volume_orient(V, angles, rot, M, N, P, L):
    """Central slices ([P][N][M] complex128) of the [L][N][M] Fourier volume V
    at tilts `angles` and in-plane rotations `rot` (None: zero), float64."""
    V = np.asarray(V).astype(np.complex128).reshape(L, N, M)
    out = np.zeros((P, N, M), np.complex128)
    for p in range(P):
        r = 0.0 if rot is None else float(rot[p])
        for z, x, y, ok, w, _, _ in _orient_weights(M, N, L, float(angles[p]), r):
            out[p] += w * V[z, x, y]
    return out


def slice_loss_grad_orient(V, angles, rot, A, M, N, P, L):
    """Loss sum (|slice| - A)^2 and its gradients in float64: (loss,
    dL/dRe V + i dL/dIm V as [L][N][M], dL/da [P], dL/dr [P])."""
    V = np.asarray(V).astype(np.complex128).reshape(L, N, M)
    A = np.asarray(A, np.float64).reshape(P, N, M)
    gV = np.zeros_like(V)
    ga, gr = np.zeros(P), np.zeros(P)
    loss = 0.0
    for p in range(P):
        ws = _orient_weights(M, N, L, float(angles[p]), 0.0 if rot is None else float(rot[p]))
        s = np.zeros((N, M), np.complex128)
        dsa = np.zeros((N, M), np.complex128)
        dsr = np.zeros((N, M), np.complex128)
        for z, x, y, ok, w, dwa, dwr in ws:
            vals = V[z, x, y]
            s += w * vals
            dsa += dwa * vals
            dsr += dwr * vals
        mag = np.abs(s)
        d = mag - A[p]
        loss += float((d * d).sum())
        G = np.where(mag > 0, 2 * d * s / np.where(mag > 0, mag, 1), 0)
        ga[p] = float(np.real(np.conj(G) * dsa).sum())
        gr[p] = float(np.real(np.conj(G) * dsr).sum())
        for z, x, y, ok, w, _, _ in ws:
            np.add.at(gV, (z[ok], x[ok], y[ok]), (w * G)[ok])
    return loss, gV, ga, gr


def volume_loss_grad(vol, angles, rot, A, M, N, P, L):
    """The loss of a real-space volume through the shifted 3D transform
    (Forward3D, MKL_Impl.inl:154-178 with fftshifts; cube volumes) and the
    slice operator, float64: (loss, dL/dvol [L][N][M] real, dL/da, dL/dr).
    dL/dvol = Re(Forward3D^H dL/dV), the adjoint transform being the inverse
    transform without its normalisation."""
    assert M == N == L
    vol = np.asarray(vol, np.float64).reshape(L, N, M)
    impl = OracleImpl(np.float64, M, N, L, 1)
    VF = vol.astype(np.complex128).ravel().copy()
    impl.Forward3D(VF)
    loss, gV, ga, gr = slice_loss_grad_orient(VF, angles, rot, A, M, N, P, L)
    g = gV.ravel().copy()
    impl.Backward3D(g)
    return loss, np.real(g).reshape(L, N, M) * float(M * N * L), ga, gr


def _slice_weights(M, N, L, a):
    """Bilinear sampling of one slice (the merges' geometry): for every slice
    pixel (xIn, yIn) the (z, y) of its up to four voxels on the plane x = xIn,
    their weights and the weights' derivatives in the angle (float64)."""
    yIn = np.arange(M)
    yr = (M // 2 - yIn).astype(np.float64)
    zf = (L // 2) - yr * np.sin(a)
    yf = (M // 2) - yr * np.cos(a)
    dz, dy = -yr * np.cos(a), yr * np.sin(a)
    z0, y0 = np.floor(zf).astype(np.int64), np.floor(yf).astype(np.int64)
    fz, fy = zf - z0, yf - y0
    out = []
    for da in (0, 1):
        for db in (0, 1):
            z, y = z0 + da, y0 + db
            wz, dwz = (fz, dz) if da else (1 - fz, -dz)
            wy, dwy = (fy, dy) if db else (1 - fy, -dy)
            ok = (z >= 0) & (z < L) & (y >= 0) & (y < M)
            out.append((z, y, ok, wz * wy, dwz * wy + wz * dwy))
    return out


def slice_volume(V, angles, M, N, P, L):
    """Project-defined central slices ([P][N][M] complex128) of the [L][N][M]
    Fourier volume V: pixel (xIn, yIn) of angle a samples V bilinearly at
    z = L/2 - yr sin a, x = xIn, y = M/2 - yr cos a, yr = M/2 - yIn."""
    V = np.asarray(V).astype(np.complex128).reshape(L, N, M)
    out = np.zeros((P, N, M), np.complex128)
    for p in range(P):
        for z, y, ok, w, _ in _slice_weights(M, N, L, float(angles[p])):
            zz, yy = np.where(ok, z, 0), np.where(ok, y, 0)
            out[p] += np.where(ok, w, 0.0)[None, :] * V[zz, :, yy].T
    return out


def slice_loss_grad(V, angles, A, M, N, P, L):
    """Loss sum (|slice| - A)^2 and its gradients in float64:
    (loss, dL/dRe V + i dL/dIm V as [L][N][M], dL/da as [P])."""
    V = np.asarray(V).astype(np.complex128).reshape(L, N, M)
    A = np.asarray(A, np.float64).reshape(P, N, M)
    gV = np.zeros_like(V)
    ga = np.zeros(P)
    loss = 0.0
    for p in range(P):
        ws = _slice_weights(M, N, L, float(angles[p]))
        s = np.zeros((N, M), np.complex128)
        ds = np.zeros((N, M), np.complex128)
        for z, y, ok, w, dw in ws:
            zz, yy = np.where(ok, z, 0), np.where(ok, y, 0)
            vals = V[zz, :, yy].T
            s += np.where(ok, w, 0.0)[None, :] * vals
            ds += np.where(ok, dw, 0.0)[None, :] * vals
        mag = np.abs(s)
        d = mag - A[p]
        loss += float((d * d).sum())
        G = np.where(mag > 0, 2 * d * s / np.where(mag > 0, mag, 1), 0)
        ga[p] = float(np.real(np.conj(G) * ds).sum())
        for z, y, ok, w, _ in ws:
            for yi in np.nonzero(ok)[0]:
                gV[z[yi], :, y[yi]] += w[yi] * G[:, yi]
    return loss, gV, ga
