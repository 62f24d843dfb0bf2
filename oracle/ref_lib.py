"""ctypes access to ``oracle/_ref/libcpra_mklref.so`` (test infrastructure only).

The library is the reference's own ``MklImpl<T>`` operator source compiled
unchanged against the project-written DFTI/CBLAS shim (``oracle/Makefile``).
Each method mirrors one ``CpraImpl<T>`` virtual (include/CPRA_Impl.hpp:23-60)
and operates in place on contiguous numpy arrays.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
import sys
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "_ref" / "libcpra_mklref.so"
_lib = None
# True: the reference's constructor/destructor status lines (below) are
# discarded instead of going to stderr
QUIET = False


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} is not built (run: make -C oracle)")
        L = C.CDLL(str(LIB_PATH))
        u64, i32, vp, f64 = C.c_uint64, C.c_int, C.c_void_p, C.c_double
        L.cpra_ref_create.restype = vp
        L.cpra_ref_create.argtypes = [i32, u64, u64, u64, u64]
        L.cpra_ref_destroy.argtypes = [i32, vp]
        L.cpra_ref_set_threads.argtypes = [i32]
        L.cpra_ref_set_threads.restype = i32
        for name in ("forward2d", "backward2d"):
            f = getattr(L, f"cpra_ref_{name}")
            f.argtypes = [i32, vp, vp]
            f.restype = i32
        L.cpra_ref_fftshift2d.argtypes = [i32, vp, vp, u64, u64, u64]
        L.cpra_ref_fftshift3d.argtypes = [i32, vp, vp, u64, u64, u64, u64]
        for name in ("space_constraint", "data_constraint_real", "data_constraint_complex"):
            f = getattr(L, f"cpra_ref_{name}")
            f.argtypes = [i32, vp, vp, vp, u64, u64]
            f.restype = i32
        L.cpra_ref_merge_add.argtypes = [i32, vp, vp, vp, f64, f64, u64]
        L.cpra_ref_normalization.argtypes = [i32, vp, vp, f64, u64]
        L.cpra_ref_initialize.argtypes = [i32, vp, vp, u64]
        L.cpra_ref_dm_iterations.argtypes = [i32, vp, vp, vp, vp, vp, vp, u64, u64, f64, i32]
        L.cpra_ref_cpra_sample.argtypes = [i32, u64, u64, u64, u64, u64, vp, vp, vp, i32, i32, i32, f64, vp]
        for f in (L.cpra_ref_fftshift2d, L.cpra_ref_fftshift3d, L.cpra_ref_merge_add,
                  L.cpra_ref_normalization, L.cpra_ref_initialize, L.cpra_ref_dm_iterations,
                  L.cpra_ref_cpra_sample):
            f.restype = i32
        _lib = L
    return _lib


def set_threads(n: int) -> int:
    return lib().cpra_ref_set_threads(int(n))


@contextlib.contextmanager
def _c_stdout_to_stderr():
    """The reference's constructor and destructor report DFTI failures with
    printf (include/MKL_Impl.hpp:28-79, 167-179; its 3D descriptor is built
    from the 2D length array and the shim refuses it, "shim DFTI: unsupported
    configuration").  Those lines go to stderr here, so that a caller's stdout
    carries only its own output, or nowhere with QUIET set."""
    libc = C.CDLL(None)
    sys.stdout.flush()
    libc.fflush(None)
    saved = os.dup(1)
    sink = os.open(os.devnull, os.O_WRONLY) if QUIET else 2
    try:
        os.dup2(sink, 1)
        yield
    finally:
        libc.fflush(None)
        os.dup2(saved, 1)
        os.close(saved)
        if QUIET:
            os.close(sink)


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"], "reference wrappers need contiguous arrays"
    return a.ctypes.data_as(C.c_void_p)


class RefImpl:
    """The reference ``MklImpl<T>`` behind a numpy-array interface."""

    def __init__(self, T, m, n, l, batch_size):
        self.T = np.dtype(T).type
        self.dbl = 1 if self.T == np.float64 else 0
        self.m, self.n, self.l, self.batch = int(m), int(n), int(l), int(batch_size)
        L = lib()
        with _c_stdout_to_stderr():
            self.h = L.cpra_ref_create(self.dbl, self.m, self.n, self.l, self.batch)

    def __del__(self):
        # the reference's destructor prints its last DFTI status twice
        # (include/MKL_Impl.hpp:167-179): routed to stderr like the constructor's
        try:
            if self.h:
                L = lib()
                with _c_stdout_to_stderr():
                    L.cpra_ref_destroy(self.dbl, self.h)
                self.h = None
        except Exception:
            pass

    def Forward2D(self, x):
        return bool(lib().cpra_ref_forward2d(self.dbl, self.h, _p(x)))

    def Backward2D(self, x):
        return bool(lib().cpra_ref_backward2d(self.dbl, self.h, _p(x)))

    def FFTShift2D(self, x, M, N, B):
        return bool(lib().cpra_ref_fftshift2d(self.dbl, self.h, _p(x), M, N, B))

    def FFTShift3D(self, x, M, N, L, B):
        return bool(lib().cpra_ref_fftshift3d(self.dbl, self.h, _p(x), M, N, L, B))

    def SpaceConstraint(self, x, S, num, batch):
        return bool(lib().cpra_ref_space_constraint(self.dbl, self.h, _p(x), _p(S), num, batch))

    def DataConstraint(self, x, A, num, batch):
        if np.iscomplexobj(A):
            return bool(lib().cpra_ref_data_constraint_complex(self.dbl, self.h, _p(x), _p(A), num, batch))
        return bool(lib().cpra_ref_data_constraint_real(self.dbl, self.h, _p(x), _p(A), num, batch))

    def MergeAddData(self, src, dst, alpha, beta, num):
        return bool(lib().cpra_ref_merge_add(self.dbl, self.h, _p(src), _p(dst), float(alpha), float(beta), num))

    def Normalization(self, x, norm, num):
        return bool(lib().cpra_ref_normalization(self.dbl, self.h, _p(x), float(norm), num))

    def Initialize(self, x, num):
        return bool(lib().cpra_ref_initialize(self.dbl, self.h, _p(x), num))

    def dm_iterations(self, x, t1, t2, A, S, num, batch, beta, iters):
        return bool(lib().cpra_ref_dm_iterations(self.dbl, self.h, _p(x), _p(t1), _p(t2), _p(A), _p(S),
                                                 num, batch, float(beta), int(iters)))


def cpra_sample(T, M, N, L, P, B, A, S, x0, epi, iters, pre_iter, beta):
    """Reference driver order (src/CPRA_MKL.cpp:35-140) on the reference
    operators.  Returns x [P*B*M*N] complex (the MKL error output is a stub)."""
    T = np.dtype(T).type
    dbl = 1 if T == np.float64 else 0
    Cx = np.complex128 if dbl else np.complex64
    x = np.ascontiguousarray(np.asarray(x0, Cx).ravel()).copy()
    A = np.ascontiguousarray(np.asarray(A, T).ravel())
    S = np.ascontiguousarray(np.asarray(S, T).ravel())
    err = np.zeros(P * B, T)
    with _c_stdout_to_stderr():
        ok = lib().cpra_ref_cpra_sample(dbl, M, N, L, P, B, _p(A), _p(S), _p(x), epi, iters, pre_iter,
                                        float(beta), _p(err))
    if not ok:
        raise ValueError("cpra_ref_cpra_sample rejected its arguments")
    return x
