"""Seeded synthetic carousel data with the shapes and statistics of the
benchmark configurations (no dataset is involved; all inputs are generated).

* ``carousel(...)``: a real volume of random ellipsoids inside a sphere,
  projected at P angles about one tilt axis (the slice's column axis, the
  y axis of the reference's merge geometry, CUDA_Impl_Kernel.cuh:80-90); each
  projection's far-field intensity |FFT|^2, scaled to a photon budget with
  Poisson noise, gives the modulus plane A = sqrt(I) (DC at (M/2, N/2), the
  reference's centred layout) and the support plane S (1 inside the projected
  sphere, 0 outside).
* ``patterns_2d(...)``: independent 2D objects (Gaussian blobs in a disc,
  phase in [-0.3, 0.3]) with their noisy moduli and supports.
* ``carousel_gpu(...)``: the large carousel on the GPU, its moduli taken with
  the slice operator itself (tilt and in-plane rotation per pattern), so that
  the data match the model of the orientation refinement.

Data preparation only: nothing here is on the benchmarked path.
"""
from __future__ import annotations

import numpy as np


def _ellipsoid_volume(rng, n, count, axes_range, radius, dens_range=(0.2, 1.0)):
    z, y, x = np.meshgrid(*(np.arange(n) - n / 2,) * 3, indexing="ij")
    vol = np.zeros((n, n, n), np.float32)
    for _ in range(count):
        a = rng.uniform(*axes_range, size=3)
        r = rng.uniform(0, radius - a.max())
        d = rng.standard_normal(3)
        c = d / np.linalg.norm(d) * r
        q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        pts = np.stack([z - c[0], y - c[1], x - c[2]], -1) @ q
        inside = ((pts / a) ** 2).sum(-1) <= 1.0
        vol[inside] += rng.uniform(*dens_range)
    vol[(z ** 2 + y ** 2 + x ** 2) > radius ** 2] = 0
    return vol


def _project(vol, angles):
    """Parallel projections about the axis of array dim 1 (rows of a slice are
    the rotated direction, columns the tilt axis)."""
    n = vol.shape[0]
    z, y, x = np.nonzero(vol)
    w = vol[z, y, x].astype(np.float64)
    zc, yc, xc = z - n / 2, y - n / 2, x - n / 2
    out = np.zeros((len(angles), n, n), np.float64)
    for p, a in enumerate(angles):
        # rotate (z, x) about the y axis; the detector row is the rotated x
        u = np.cos(a) * xc - np.sin(a) * zc
        ru = np.clip(np.rint(u + n / 2).astype(np.int64), 0, n - 1)
        col = yc.astype(np.int64) + n // 2
        np.add.at(out[p], (ru, col), w)
    return out


def _modulus(proj, photons, rng):
    F = np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(proj, axes=(-2, -1))), axes=(-2, -1))
    I = np.abs(F) ** 2
    I *= photons / I.sum(axis=(-2, -1), keepdims=True)
    I = rng.poisson(I).astype(np.float64)
    return np.sqrt(I).astype(np.float32)


def carousel(n=128, P=90, step_deg=2.0, ellipsoids=32, axes=(4, 16), radius=40, photons=1e7, seed=1):
    """Returns dict(A=[P][n][n] f32, S=[P][n][n] f32, angles=[P] f32 radians,
    volume=[n][n][n] f32)."""
    rng = np.random.default_rng(seed)
    vol = _ellipsoid_volume(rng, n, ellipsoids, axes, radius)
    angles = np.deg2rad(np.arange(P) * step_deg)
    proj = _project(vol, angles)
    A = _modulus(proj, photons, rng)
    yy, xx = np.mgrid[0:n, 0:n]
    disc = (((yy - n / 2) ** 2 + (xx - n / 2) ** 2) <= (radius + 2) ** 2).astype(np.float32)
    S = np.broadcast_to(disc, (P, n, n)).copy()
    return {"A": A, "S": S, "angles": angles.astype(np.float32), "volume": vol}


def patterns_2d(count=16, n=128, radius=24, blobs=8, photons=1e6, seed=0):
    """Independent 2D objects as in the plain 2D configuration.  Returns
    dict(A, S, obj) with A, S [count][n][n] f32 and obj complex64."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:n, 0:n] - n / 2
    disc = (yy ** 2 + xx ** 2) <= radius ** 2
    objs = np.zeros((count, n, n), np.complex64)
    for k in range(count):
        amp = np.zeros((n, n))
        for _ in range(blobs):
            r, t = radius * np.sqrt(rng.uniform()), rng.uniform(0, 2 * np.pi)
            cy, cx = r * np.sin(t), r * np.cos(t)
            s = rng.uniform(2, 6)
            amp += rng.uniform(0, 1) * np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) / (2 * s * s))
        amp *= disc
        phase = rng.uniform(-0.3, 0.3, (n, n))
        objs[k] = (amp * np.exp(1j * phase)).astype(np.complex64)
    F = np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(objs, axes=(-2, -1))), axes=(-2, -1))
    I = np.abs(F) ** 2
    I *= photons / I.sum(axis=(-2, -1), keepdims=True)
    A = np.sqrt(rng.poisson(I)).astype(np.float32)
    S = np.broadcast_to(disc.astype(np.float32), (count, n, n)).copy()
    return {"A": A, "S": S, "obj": objs}


def r_factor(x_plane, A_plane):
    """R = sum | |F x| - A | / sum A in float64 for one centred plane
    (project-defined metric; the reference reports only ConvergeError)."""
    F = np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(np.asarray(x_plane, np.complex128))))
    A = np.asarray(A_plane, np.float64)
    return float(np.abs(np.abs(F) - A).sum() / max(A.sum(), 1e-300))


def autocorrelation_support(A, frac=0.04):
    """Initial support from the autocorrelation |IFFT(A^2)| > frac * max, per
    plane ([count][n][n] float32 of 0/1): the autocorrelation's extent bounds
    twice the object's."""
    A = np.asarray(A, np.float64)
    ac = np.abs(np.fft.fftshift(np.fft.ifft2(np.fft.ifftshift(A * A, axes=(-2, -1))), axes=(-2, -1)))
    mx = ac.reshape(ac.shape[0], -1).max(axis=1)[:, None, None]
    return (ac > frac * mx).astype(np.float32)


def random_phase_start(A, seed=0):
    """Starting guesses: the centred inverse transform of A with uniform random
    phases, [count][n][n] complex64 (seeded)."""
    rng = np.random.default_rng(seed)
    A = np.asarray(A, np.float64)
    ph = np.exp(2j * np.pi * rng.uniform(size=A.shape))
    x = np.fft.fftshift(np.fft.ifft2(np.fft.ifftshift(A * ph, axes=(-2, -1))), axes=(-2, -1))
    return x.astype(np.complex64)


def carousel_gpu(torch, n=256, P=180, step_deg=1.0, jitter_deg=0.3, ellipsoids=64, axes=(4, 16), radius=None,
                 photons=1e8, seed=3, device="cuda"):
    """The carousel synthesis at sizes where numpy is too slow (256^3 and up),
    on the GPU, with the slice operator's own geometry so that the data match
    the model the refinement fits: a real volume of random ellipsoids inside a
    sphere, its Fourier volume (Forward3D), central slices at P tilts step_deg
    apart, each tilt and each in-plane rotation jittered by N(0, jitter_deg)
    (cpra_b200_slice_orient: the merges' geometry with the detector grid turned
    in its plane), intensities |slice|^2 scaled to `photons` per pattern on
    average, Poisson noise, and disc supports.  Returns dict(A [P][n][n]
    float32 in the 2D stage's pattern layout (row: the tilted coordinate,
    column: the tilt axis), A_slices [P][n][n] in the slice layout (the
    transpose), S, angles_true, rot_true, angles_nominal [P] float32 radians,
    volume [n][n][n] float32 in the data's units, i.e. the real-space volume
    whose slices the noise-free A are), all on `device`."""
    import cpra_b200
    g = torch.Generator(device=device).manual_seed(seed)
    radius = radius if radius is not None else 0.3125 * n
    ax = torch.arange(n, device=device, dtype=torch.float32) - n / 2
    z, y, x = torch.meshgrid(ax, ax, ax, indexing="ij")
    vol = torch.zeros((n, n, n), device=device)
    for _ in range(ellipsoids):
        a = axes[0] + (axes[1] - axes[0]) * torch.rand(3, device=device, generator=g)
        r = (radius - float(a.max())) * float(torch.rand(1, device=device, generator=g))
        d = torch.randn(3, device=device, generator=g)
        c = d / d.norm() * r
        q, _ = torch.linalg.qr(torch.randn(3, 3, device=device, generator=g))
        pts = torch.stack([z - c[0], y - c[1], x - c[2]], -1) @ q
        inside = ((pts / a) ** 2).sum(-1) <= 1.0
        vol += inside * (0.2 + 0.8 * float(torch.rand(1, device=device, generator=g)))
        del pts, inside
    vol[(z * z + y * y + x * x) > radius * radius] = 0
    del z, y, x
    nominal = torch.deg2rad(torch.arange(P, device=device, dtype=torch.float64) * step_deg)
    true = nominal + torch.deg2rad(jitter_deg * torch.randn(P, device=device, generator=g, dtype=torch.float64))
    rot = torch.deg2rad(jitter_deg * torch.randn(P, device=device, generator=g, dtype=torch.float64))
    impl = cpra_b200.B200Impl(n, n, n, 1)
    VF = vol.reshape(-1).to(torch.complex64)
    impl.Forward3D(VF)
    sl = torch.empty(P * n * n, dtype=torch.complex64, device=device)
    impl.slice_orient(VF, true.float().contiguous(), rot.float().contiguous(), n, n, P, n, sl)
    impl.Sync()
    impl.close()
    del VF
    I = sl.abs().double().reshape(P, n, n) ** 2
    del sl
    scale = photons * P / float(I.sum())
    I = I * scale
    A_sl = torch.sqrt(torch.poisson(I, generator=g)).float()
    del I
    yy, xx = torch.meshgrid(ax, ax, indexing="ij")
    disc = ((yy * yy + xx * xx) <= (radius + 2) ** 2).float()
    S = disc.expand(P, n, n).contiguous()
    return {"A": A_sl.transpose(1, 2).contiguous(), "A_slices": A_sl.contiguous(), "S": S,
            "angles_true": true.float(), "rot_true": rot.float(), "angles_nominal": nominal.float(),
            "volume": vol * float(scale) ** 0.5}
