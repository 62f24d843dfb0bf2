"""Generates tests/golden/ref_golden.npz from the reference's own operator code.

The outputs come from ``oracle/_ref/libcpra_mklref.so``: the reference's
``MklImpl<T>`` source (include/MKL_Impl.hpp, include/detail/MKL_Impl.inl)
compiled unchanged against the project's DFTI/CBLAS shim (``make -C oracle``).
Inputs are seeded synthetic data.  Run from the repository root:

    make -C oracle && python tests/golden/make_golden.py

The fixture travels with the repository, so the GPU tests can check the B200
backend against reference outputs without the reference being present.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO / "oracle"))
import ref_lib as R  # noqa: E402

OUT = Path(__file__).resolve().parent / "ref_golden.npz"


def cplx(rng, n, dtype=np.complex64):
    return (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(dtype)


def object_planes(rng, M, N, count, radius_frac=0.25):
    """Small seeded test objects: Gaussian blobs inside a disc, returned with
    their centred Fourier modulus and support mask (float32 [count][M][N])."""
    yy, xx = np.mgrid[0:M, 0:N]
    amps, sups = [], []
    for _ in range(count):
        r = radius_frac * min(M, N)
        disc = ((yy - M / 2) ** 2 + (xx - N / 2) ** 2) <= r * r
        obj = np.zeros((M, N))
        for _ in range(6):
            cy, cx = rng.uniform(M / 2 - r / 2, M / 2 + r / 2), rng.uniform(N / 2 - r / 2, N / 2 + r / 2)
            s = rng.uniform(1.0, 3.0)
            obj += rng.uniform(0.2, 1.0) * np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) / (2 * s * s))
        obj *= disc
        F = np.fft.fftshift(np.fft.fft2(np.fft.ifftshift(obj)))
        amps.append(np.abs(F).astype(np.float32))
        sups.append(disc.astype(np.float32))
    return np.stack(amps), np.stack(sups)


def main():
    if not R.available():
        raise SystemExit("build the reference first: make -C oracle")
    rng = np.random.default_rng(20261203)
    g = {}

    # reference KATs (test/unitest_mkl.cpp:15-71), as the reference computes them
    r = R.RefImpl(np.float64, 10, 10, 1, 1)
    x = np.ones(100, np.complex128)
    g["kat_dft10_in"] = x.copy()
    r.Forward2D(x)
    g["kat_dft10_fwd"] = x.copy()
    r.Backward2D(x)
    g["kat_dft10_bwd"] = x.copy()
    r = R.RefImpl(np.float32, 1, 1, 1, 1)
    x = np.full(1000, 10 + 10j, np.complex64)
    r.MergeAddData(x, x, 0.5, 0.5, 1000)
    g["kat_merge_half"] = x.copy()
    r.Normalization(x, 10, 1000)
    g["kat_norm10"] = x.copy()

    # 2D transforms and shifts
    for T, M, N, B, tag in ((np.float32, 64, 64, 2, "f32_64"), (np.float64, 32, 32, 2, "f64_32"),
                            (np.float32, 128, 128, 1, "f32_128"), (np.float32, 16, 8, 3, "f32_16x8")):
        C = np.complex64 if T == np.float32 else np.complex128
        r = R.RefImpl(T, M, N, 1, B)
        x = cplx(rng, M * N * B, C)
        g[f"{tag}_x"] = x.copy()
        y = x.copy(); r.Forward2D(y); g[f"{tag}_fwd"] = y
        y = x.copy(); r.Backward2D(y); g[f"{tag}_bwd"] = y
        y = x.copy(); r.FFTShift2D(y, M, N, B); g[f"{tag}_shift"] = y

    # 3D shift ([L][M][N], index dep*M*N + row*N + col)
    r = R.RefImpl(np.float32, 6, 8, 4, 2)
    x = cplx(rng, 6 * 8 * 4 * 2)
    g["shift3d_x"] = x.copy()
    r.FFTShift3D(x, 6, 8, 4, 2)
    g["shift3d_out"] = x.copy()

    # element-wise operators, batch of 3 planes of 32x32 sharing one constraint
    M = N = 32
    B = 3
    r = R.RefImpl(np.float32, M, N, 1, B)
    x = cplx(rng, M * N * B) * 100
    x[5] = 0  # |z| == 0 stays 0
    A = rng.uniform(0, 50, M * N).astype(np.float32)
    A[::9] = 0  # A == 0: unconstrained (MKL_Impl.inl:98-104)
    S = rng.uniform(0.0, 1.0, M * N).astype(np.float32)
    S[:4] = np.array([0.9, np.nextafter(np.float32(0.9), np.float32(1)), np.nextafter(np.float32(0.9), np.float32(0)),
                      1.0], np.float32)
    Cc = cplx(rng, M * N) * 3
    Cc[::7] = 0  # |C| == 0: unconstrained (MKL_Impl.inl:121)
    g["ew_x"], g["ew_A"], g["ew_S"], g["ew_C"] = x.copy(), A, S, Cc
    y = x.copy(); r.DataConstraint(y, A, M * N * B, B); g["ew_dc_real"] = y
    y = x.copy(); r.DataConstraint(y, Cc, M * N * B, B); g["ew_dc_complex"] = y
    y = x.copy(); r.SpaceConstraint(y, S, M * N * B, B); g["ew_sc"] = y
    src = cplx(rng, M * N * B)
    g["ew_src"] = src
    beta = np.float32(0.9)
    y = x.copy(); r.MergeAddData(src, y, -1.0 / beta, 1.0 + 1.0 / beta, M * N * B); g["ew_merge"] = y
    y = x.copy(); r.Normalization(y, 3.0, M * N * B); g["ew_norm3"] = y

    # difference-map iterations (src/CPRA_MKL.cpp:94-110), 64x64, batch 2
    M = N = 64
    B = 2
    amps, sups = object_planes(rng, M, N, 1)
    A, S = amps[0].ravel(), sups[0].ravel()
    x0 = (rng.uniform(0, 1, M * N * B) + 1j * rng.uniform(0, 1, M * N * B)).astype(np.complex64)
    g["dm_A"], g["dm_S"], g["dm_x0"] = A, S, x0
    for iters in (1, 5):
        r = R.RefImpl(np.float32, M, N, 1, B)
        x, t1, t2 = x0.copy(), x0.copy(), x0.copy()
        r.dm_iterations(x, t1, t2, A, S, M * N * B, B, 0.9, iters)
        g[f"dm{iters}_x"], g[f"dm{iters}_t1"], g[f"dm{iters}_t2"] = x, t1, t2

    # restated carousel episode driver on the reference operators
    M = N = 32
    P, B = 4, 2
    amps, sups = object_planes(rng, M, N, P)
    x0 = (rng.uniform(0, 1, P * B * M * N) + 1j * rng.uniform(0, 1, P * B * M * N)).astype(np.complex64)
    g["cpra_A"], g["cpra_S"], g["cpra_x0"] = amps.ravel(), sups.ravel(), x0
    g["cpra_cfg"] = np.array([M, N, 1, P, B, 2, 3, 4], np.int64)  # M N L P B epi iter preit
    g["cpra_x"] = R.cpra_sample(np.float32, M, N, 1, P, B, amps, sups, x0, 2, 3, 4, 0.9)

    np.savez_compressed(OUT, **g)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(g)} arrays)")


if __name__ == "__main__":
    main()
