"""Python bindings of the B200 carousel phase-retrieval backend.

Mirrors the reference's operator interface ``CPRA::CpraImpl<T>``
(include/CPRA_Impl.hpp:18-63) and its factory ``NewCpraImpl``
(include/Impl_Factory.hpp:14-30) over the C ABI of ``libcpra_b200.so``
(include/cpra_b200.h): same method names, same argument meaning, ``False`` for
argument errors (the reference's ``return false``) and an exception for CUDA
failures (the reference throws ``CPRA::cuda_error``).

Data arguments are CUDA tensors (``torch``) or raw device addresses (``int``).
There is no CPU path: importing this module fails if the CUDA library is not
built, and every operator runs on the GPU.
"""
from __future__ import annotations

import ctypes as C
import enum
import os
from pathlib import Path

__all__ = [
    "IMPL_TYPE", "CpraB200Error", "B200Impl", "NewCpraImpl", "library_path", "lib",
    "OK", "EARG", "ECUDA", "EUNSUP", "OPT_FUSION", "OPT_SPACE_MODE", "OPT_DATA_MODE", "OPT_SEED",
    "OPT_KERNEL_TIMING", "OPT_HIO_CHUNK", "OPT_GRAPH", "OPT_LANES", "OPT_IO_CHUNK", "OPT_AUTOTUNE", "OPT_TMEM",
    "OPT_FUSED3D", "OPT_HIO_CLUSTER", "OPT_FAILURE_TEST",
]

OK, EARG, ECUDA, EUNSUP = 0, 1, 2, 3
F32, F64 = 0, 1
OPT_FUSION, OPT_SPACE_MODE, OPT_DATA_MODE, OPT_SEED, OPT_KERNEL_TIMING, OPT_HIO_CHUNK, OPT_GRAPH, OPT_LANES = \
    1, 2, 3, 4, 5, 6, 7, 8
OPT_IO_CHUNK = 9
OPT_AUTOTUNE = 10
OPT_TMEM = 11
OPT_FUSED3D = 12
OPT_HIO_CLUSTER = 13
OPT_FAILURE_TEST = 14

_HERE = Path(__file__).resolve().parent


def library_path() -> Path:
    return Path(os.environ.get("CPRA_B200_LIB", _HERE / "libcpra_b200.so"))


class CpraB200Error(RuntimeError):
    """A CUDA runtime failure or an unsupported shape reported by the backend."""


class IMPL_TYPE(enum.IntEnum):
    """``enum IMPL_TYPE`` of include/CPRA_Impl.hpp:15 with the B200 entry added."""
    CUDA = 0
    MKL = 1
    B200 = 2


_lib = None

# name -> (argtypes) ; every entry point returns int
class HioBucket(C.Structure):
    """cpra_b200_hio_bucket (include/cpra_b200.h)."""
    _fields_ = [("side", C.c_uint64), ("count", C.c_uint64), ("x", C.c_void_p), ("A", C.c_void_p),
                ("S", C.c_void_p), ("estimate", C.c_void_p), ("sigma_start", C.c_double), ("sigma_end", C.c_double)]


_SIGS = {
    "cpra_b200_create": [C.POINTER(C.c_void_p), C.c_int, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64],
    "cpra_b200_destroy": [C.c_void_p],
    "cpra_b200_set_option": [C.c_void_p, C.c_int, C.c_int64],
    "cpra_b200_get_option": [C.c_void_p, C.c_int, C.POINTER(C.c_int64)],
    "cpra_b200_get_stream": [C.c_void_p, C.POINTER(C.c_void_p)],
    "cpra_b200_alloc": [C.c_void_p, C.POINTER(C.c_void_p), C.c_uint64, C.c_int],
    "cpra_b200_free": [C.c_void_p, C.c_void_p],
    "cpra_b200_initialize": [C.c_void_p, C.c_void_p, C.c_uint64],
    "cpra_b200_forward2d": [C.c_void_p, C.c_void_p],
    "cpra_b200_backward2d": [C.c_void_p, C.c_void_p],
    "cpra_b200_fftshift2d": [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64],
    "cpra_b200_forward3d": [C.c_void_p, C.c_void_p],
    "cpra_b200_backward3d": [C.c_void_p, C.c_void_p],
    "cpra_b200_fftshift3d": [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64],
    "cpra_b200_space_constraint": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64],
    "cpra_b200_data_constraint_real": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64],
    "cpra_b200_data_constraint_complex": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64],
    "cpra_b200_merge_add": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_uint64],
    "cpra_b200_normalization": [C.c_void_p, C.c_void_p, C.c_double, C.c_uint64],
    "cpra_b200_real2d_to_3d": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p] + [C.c_uint64] * 4,
    "cpra_b200_complex2d_to_3d": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p] + [C.c_uint64] * 4,
    "cpra_b200_converge_error": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p] + [C.c_uint64] * 4,
    "cpra_b200_memcpy": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64],
    "cpra_b200_sync": [C.c_void_p],
    "cpra_b200_dm_iterations": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                C.c_void_p, C.c_uint64, C.c_uint64, C.c_double, C.c_int],
    "cpra_b200_cpra_run": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_int,
                           C.c_int, C.c_int, C.c_double, C.c_int, C.c_void_p],
    "cpra_b200_cpra_run_host": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_int,
                                C.c_int, C.c_int, C.c_double, C.c_int, C.c_void_p],
    "cpra_b200_read_matrix": [C.c_void_p, C.c_char_p, C.c_void_p, C.c_uint64, C.c_uint64],
    "cpra_b200_write_matrix": [C.c_void_p, C.c_char_p, C.c_void_p, C.c_uint64, C.c_uint64],
    "cpra_b200_write_starts": [C.c_void_p, C.c_char_p, C.c_char_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_uint64,
                               C.c_uint64, C.c_uint64],
    "cpra_b200_cpra_files": [C.c_void_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_uint64, C.c_uint64,
                             C.c_int, C.c_int, C.c_int, C.c_double],
    "cpra_b200_conv_run": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_int,
                           C.c_void_p],
    "cpra_b200_conv_files": [C.c_void_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_uint64, C.c_int,
                             C.c_double],
    "cpra_b200_kernel_timing": [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)],
    "cpra_b200_hio_shrinkwrap": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_uint64,
                                 C.c_int, C.c_double, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                                 C.c_void_p],
    "cpra_b200_constraint3d": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int],
    "cpra_b200_refine": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p] + [C.c_uint64] * 4 +
                        [C.c_int, C.c_double, C.c_double, C.c_void_p],
    "cpra_b200_best_start": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p,
                             C.c_void_p],
    "cpra_b200_hio_batched": [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int, C.c_double,
                              C.c_double, C.c_double, C.c_int],
    "cpra_b200_slice": [C.c_void_p, C.c_void_p, C.c_void_p] + [C.c_uint64] * 4 + [C.c_void_p],
    "cpra_b200_slice_loss_grad": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p] + [C.c_uint64] * 4
                                 + [C.c_void_p, C.c_void_p, C.c_void_p],
    "cpra_b200_slice_orient": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p] + [C.c_uint64] * 4 + [C.c_void_p],
    "cpra_b200_slice_loss_grad_orient": [C.c_void_p] + [C.c_void_p] * 4 + [C.c_uint64] * 4 + [C.c_void_p] * 4,
    "cpra_b200_volume_loss_grad": [C.c_void_p] + [C.c_void_p] * 4 + [C.c_uint64] * 4 + [C.c_void_p] * 4,
    "cpra_b200_refine_orient": [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
                               + [C.c_uint64] * 4 + [C.c_int, C.c_double, C.c_double, C.c_double, C.c_void_p],
    "cpra_b200_rfactor": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p],
    "cpra_b200_converge_error_noalloc": [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p] + [C.c_uint64] * 4
                                        + [C.c_void_p],
}


def lib():
    """Load libcpra_b200.so (fails loudly if it is not built)."""
    global _lib
    if _lib is None:
        path = library_path()
        if not path.exists():
            raise ImportError(f"{path} not found: build it with "
                              "`python carousel-phase-retrieval-algorithm_b200/build.py`")
        L = C.CDLL(str(path))
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.cpra_b200_last_error.argtypes = []
        L.cpra_b200_last_error.restype = C.c_char_p
        L.cpra_b200_kernels_launched.argtypes = []
        L.cpra_b200_kernels_launched.restype = C.c_uint64
        _lib = L
    return _lib


def kernels_launched() -> int:
    """Kernels launched by libcpra_b200.so in this process so far."""
    return int(lib().cpra_b200_kernels_launched())


def last_error() -> str:
    return lib().cpra_b200_last_error().decode(errors="replace")


def _addr(a) -> int:
    """Device address of a tensor / integer address (None -> 0)."""
    if a is None:
        return 0
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):
        if hasattr(a, "is_cuda") and not a.is_cuda and a.numel() > 0:
            raise ValueError("B200 operators take CUDA tensors (there is no CPU path)")
        return a.data_ptr()
    if hasattr(a, "ctypes"):  # numpy array: host pointer (ConvergeError's output only)
        return a.ctypes.data
    raise TypeError(f"cannot take the address of {type(a).__name__}")


def _any_addr(a) -> int:
    """Address of device, managed or host memory (the file I/O entries take any)."""
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    if hasattr(a, "ctypes"):
        return a.ctypes.data
    raise TypeError(f"cannot take the address of {type(a).__name__}")


def _check(rc: int, what: str) -> bool:
    if rc == OK:
        return True
    if rc == EARG:
        return False
    raise CpraB200Error(f"{what}: {last_error()}")


class B200Impl:
    """``CpraImpl<T>`` implemented by the B200 backend (``T`` = float32 or
    float64), constructed like ``CudaImpl(m, n, l, batch_size)``
    (include/CUDA_Impl.cuh:16-52)."""

    def __init__(self, m: int, n: int, l: int, batch_size: int, dtype: str = "float32"):
        self.dtype = dtype
        self.dbl = dtype in ("float64", "double")
        self.m, self.n, self.l, self.batch = int(m), int(n), int(l), int(batch_size)
        h = C.c_void_p()
        rc = lib().cpra_b200_create(C.byref(h), F64 if self.dbl else F32, self.m, self.n, self.l, self.batch)
        if rc != OK:
            raise CpraB200Error(f"cpra_b200_create: {last_error()}")
        self._h = h

    # -- lifetime -------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().cpra_b200_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_option(self, option: int, value: int) -> bool:
        return _check(lib().cpra_b200_set_option(self._h, option, int(value)), "set_option")

    def get_option(self, option: int) -> int:
        v = C.c_int64()
        _check(lib().cpra_b200_get_option(self._h, option, C.byref(v)), "get_option")
        return v.value

    def stream(self) -> int:
        s = C.c_void_p()
        _check(lib().cpra_b200_get_stream(self._h, C.byref(s)), "get_stream")
        return s.value or 0

    # -- CpraImpl<T> (include/CPRA_Impl.hpp:23-60) ----------------------------
    def Initialize(self, flat_data_ptr, num) -> bool:
        return _check(lib().cpra_b200_initialize(self._h, _addr(flat_data_ptr), int(num)), "Initialize")

    def Forward2D(self, flat_input) -> bool:
        return _check(lib().cpra_b200_forward2d(self._h, _addr(flat_input)), "Forward2D")

    def Backward2D(self, flat_input) -> bool:
        return _check(lib().cpra_b200_backward2d(self._h, _addr(flat_input)), "Backward2D")

    def FFTShift2D(self, flat_input, M, N, Batch) -> bool:
        return _check(lib().cpra_b200_fftshift2d(self._h, _addr(flat_input), int(M), int(N), int(Batch)),
                      "FFTShift2D")

    def Forward3D(self, flat_input) -> bool:
        return _check(lib().cpra_b200_forward3d(self._h, _addr(flat_input)), "Forward3D")

    def Backward3D(self, flat_input) -> bool:
        return _check(lib().cpra_b200_backward3d(self._h, _addr(flat_input)), "Backward3D")

    def FFTShift3D(self, flat_input, M, N, L, Batch) -> bool:
        return _check(lib().cpra_b200_fftshift3d(self._h, _addr(flat_input), int(M), int(N), int(L), int(Batch)),
                      "FFTShift3D")

    def SpaceConstraint(self, flat_src_data, flat_constr_data, num, batch_size) -> bool:
        return _check(lib().cpra_b200_space_constraint(self._h, _addr(flat_src_data), _addr(flat_constr_data),
                                                       int(num), int(batch_size)), "SpaceConstraint")

    def DataConstraint(self, flat_src_data, flat_constr_data, num, batch_size) -> bool:
        """Real (modulus) or complex overload, chosen by the constraint's dtype
        like the reference's two overloads (include/CPRA_Impl.hpp:39,41)."""
        cplx = getattr(flat_constr_data, "is_complex", lambda: False)()
        f = lib().cpra_b200_data_constraint_complex if cplx else lib().cpra_b200_data_constraint_real
        return _check(f(self._h, _addr(flat_src_data), _addr(flat_constr_data), int(num), int(batch_size)),
                      "DataConstraint")

    def DataConstraintComplex(self, flat_src_data, flat_constr_data, num, batch_size) -> bool:
        return _check(lib().cpra_b200_data_constraint_complex(self._h, _addr(flat_src_data), _addr(flat_constr_data),
                                                              int(num), int(batch_size)), "DataConstraint")

    def MergeAddData(self, flat_src, flat_dst, alpha, beta, num) -> bool:
        return _check(lib().cpra_b200_merge_add(self._h, _addr(flat_src), _addr(flat_dst), float(alpha),
                                                float(beta), int(num)), "MergeAddData")

    def Normalization(self, flat_src, norm, num) -> bool:
        return _check(lib().cpra_b200_normalization(self._h, _addr(flat_src), float(norm), int(num)),
                      "Normalization")

    def Real2DTo3DInterpolation(self, flat_2d_src, flat_3d_dst, angles, m, n, p, l) -> bool:
        return _check(lib().cpra_b200_real2d_to_3d(self._h, _addr(flat_2d_src), _addr(flat_3d_dst), _addr(angles),
                                                   int(m), int(n), int(p), int(l)), "Real2DTo3DInterpolation")

    def Complex2DTo3DInterpolation(self, flat_2d_src, flat_3d_dst, angles, m, n, p, l) -> bool:
        return _check(lib().cpra_b200_complex2d_to_3d(self._h, _addr(flat_2d_src), _addr(flat_3d_dst),
                                                      _addr(angles), int(m), int(n), int(p), int(l)),
                      "Complex2DTo3DInterpolation")

    def ConvergeError(self, flat_old, flat_new, flat_error, m, n, l=1, batch_size=1) -> bool:
        """``flat_error`` is host memory (numpy array of T, or a CPU tensor),
        as include/CPRA_Impl.hpp:55 requires."""
        return _check(lib().cpra_b200_converge_error(self._h, _addr(flat_old), _addr(flat_new),
                                                     _host_addr(flat_error), int(m), int(n), int(l),
                                                     int(batch_size)), "ConvergeError")

    def Memcpy(self, dst, src, nbytes) -> bool:
        return _check(lib().cpra_b200_memcpy(self._h, _addr(dst), _addr(src), int(nbytes)), "Memcpy")

    def Sync(self) -> bool:
        return _check(lib().cpra_b200_sync(self._h), "Sync")

    # -- extensions -------------------------------------------------------------
    def dm_iterations(self, x, t1, t2, A, S, batch, beta, iters, a_stride=0, s_stride=0) -> bool:
        """``iters`` fused difference-map iterations (src/CPRA_MKL.cpp:94-110)."""
        return _check(lib().cpra_b200_dm_iterations(self._h, _addr(x), _addr(t1), _addr(t2), _addr(A),
                                                    int(a_stride), _addr(S), int(s_stride), int(batch),
                                                    float(beta), int(iters)), "dm_iterations")

    def cpra_run(self, x, A, S, P, batch, epi, iters, pre_iter, beta, final_step=True, err=None) -> bool:
        """The carousel driver of src/CPRA_MKL.cpp:35-140 on resident buffers;
        ``err`` (host array of P*batch, optional) receives the last episode's
        convergence errors."""
        return _check(lib().cpra_b200_cpra_run(self._h, _addr(x), _addr(A), _addr(S), int(P), int(batch), int(epi),
                                               int(iters), int(pre_iter), float(beta), 1 if final_step else 0,
                                               _host_addr(err) if err is not None else 0), "cpra_run")

    def conv_run(self, x, A, S, iters, beta, final_step=True, err=None) -> bool:
        """The conventional 3D driver of src/CONV_MKL.cpp:10-88 on resident
        volumes; ``err`` (host array of batch, optional) receives the last
        iteration's convergence errors."""
        return _check(lib().cpra_b200_conv_run(self._h, _addr(x), _addr(A), _addr(S), int(iters), float(beta),
                                               1 if final_step else 0,
                                               _host_addr(err) if err is not None else 0), "conv_run")

    def cpra_run_host(self, x, A, S, P, batch, epi, iters, pre_iter, beta, final_step=True, err=None) -> bool:
        """``cpra_run`` on host arrays (numpy or CPU tensors; pinned ones let the
        per-angle copies overlap the computation); ``x`` is overwritten."""
        return _check(lib().cpra_b200_cpra_run_host(self._h, _host_addr(x), _host_addr(A), _host_addr(S), int(P),
                                                    int(batch), int(epi), int(iters), int(pre_iter), float(beta),
                                                    1 if final_step else 0,
                                                    _host_addr(err) if err is not None else 0), "cpra_run_host")

    # -- raw-file I/O (include/detail/CPRA.inl:8-48, src/CPRA_MKL.cpp:156-225) ------
    def read_matrix(self, path, dst, count, elem_bytes=None) -> bool:
        """ReadMatrixFromFile: ``count`` elements of a raw file into ``dst``
        (device, managed or host); element size from the context's type."""
        eb = (8 if self.dbl else 4) if elem_bytes is None else int(elem_bytes)
        return _check(lib().cpra_b200_read_matrix(self._h, os.fsencode(path), _any_addr(dst), int(count), eb),
                      "read_matrix")

    def write_matrix(self, path, src, count, elem_bytes=None) -> bool:
        """WriteMatrixToFile: ``count`` elements of ``src`` to a raw file."""
        eb = (8 if self.dbl else 4) if elem_bytes is None else int(elem_bytes)
        return _check(lib().cpra_b200_write_matrix(self._h, os.fsencode(path), _any_addr(src), int(count), eb),
                      "write_matrix")

    def write_starts(self, recon_prefix, err_prefix, file_index, x, err, P, batch, count=None) -> bool:
        """The per-start output files of src/CPRA_MKL.cpp:186-209 for starts
        0..count-1 of ``x`` [P][batch][m][n] (device) and host errors ``err``
        [P][batch] (both prefixes' files, or only the reconstructions when
        ``err_prefix`` and ``err`` are None)."""
        count = batch if count is None else count
        return _check(lib().cpra_b200_write_starts(
            self._h, os.fsencode(recon_prefix), os.fsencode(err_prefix) if err_prefix is not None else None,
            int(file_index), _addr(x), _host_addr(err) if err is not None else None, int(P), int(batch),
            int(count)), "write_starts")

    def cpra_files(self, a_path, s_path, recon_prefix, err_prefix, P, total, epi, iters, pre_iter, beta) -> bool:
        """The reference program's main loop (src/CPRA_MKL.cpp:156-225) from
        the constraint files to the per-start output files."""
        return _check(lib().cpra_b200_cpra_files(self._h, os.fsencode(a_path), os.fsencode(s_path),
                                                 os.fsencode(recon_prefix), os.fsencode(err_prefix), int(P),
                                                 int(total), int(epi), int(iters), int(pre_iter), float(beta)),
                      "cpra_files")

    def conv_files(self, a_path, s_path, recon_prefix, err_prefix, total, iters, beta) -> bool:
        """The conventional program's main loop (src/CONV_MKL.cpp:103-172) from
        the constraint volumes' files to per-start output files."""
        return _check(lib().cpra_b200_conv_files(self._h, os.fsencode(a_path), os.fsencode(s_path),
                                                 os.fsencode(recon_prefix), os.fsencode(err_prefix), int(total),
                                                 int(iters), float(beta)), "conv_files")

    def hio_shrinkwrap(self, x, A, S, batch, iters, beta=0.9, sw_every=20, sigma_start=3.0, sigma_end=1.5,
                       threshold=0.1, positivity=False, a_stride=None, s_stride=None, estimate=None) -> bool:
        """Fused HIO iterations with shrinkwrap support updates (project-defined);
        per-pattern planes by default (stride m*n); ``estimate`` (optional
        device buffer) receives S (.) P_M(x) of the final x."""
        plane = self.m * self.n
        a_stride = plane if a_stride is None else a_stride
        s_stride = plane if s_stride is None else s_stride
        return _check(lib().cpra_b200_hio_shrinkwrap(self._h, _addr(x), _addr(A), int(a_stride), _addr(S),
                                                     int(s_stride), int(batch), int(iters), float(beta),
                                                     int(sw_every), float(sigma_start), float(sigma_end),
                                                     float(threshold), 1 if positivity else 0, _addr(estimate)),
                      "hio_shrinkwrap")

    def hio_batched(self, buckets, iters, beta=0.9, sw_every=20, sigma_start=3.0, sigma_end=1.5, threshold=0.1,
                    positivity=False) -> bool:
        """HIO + shrinkwrap over patterns of uneven sizes in one call
        (project-defined): ``buckets`` is a list of dicts with keys side,
        count, x, A, S and optionally estimate (device buffers, per-pattern
        contiguous) and sigma_start, sigma_end (the bucket's own blur
        schedule); each bucket runs on its own stream."""
        arr = (HioBucket * len(buckets))()
        for i, b in enumerate(buckets):
            arr[i] = HioBucket(int(b["side"]), int(b["count"]), _addr(b["x"]), _addr(b["A"]), _addr(b["S"]),
                               _addr(b.get("estimate")), float(b.get("sigma_start", 0.0)),
                               float(b.get("sigma_end", 0.0)))
        return _check(lib().cpra_b200_hio_batched(self._h, C.cast(arr, C.c_void_p), len(buckets), int(iters),
                                                  float(beta), int(sw_every), float(sigma_start), float(sigma_end),
                                                  float(threshold), 1 if positivity else 0), "hio_batched")

    def slice(self, V, angles, m, n, p, l, out) -> bool:
        """Central slices of the Fourier volume V at the given angles (project-defined)."""
        return _check(lib().cpra_b200_slice(self._h, _addr(V), _addr(angles), int(m), int(n), int(p), int(l),
                                            _addr(out)), "slice")

    def slice_loss_grad(self, V, angles, A, m, n, p, l, grad_V):
        """Amplitude loss of the slices against A and its adjoints; returns
        (loss, dL/dangles as a numpy float64 array); grad_V is written."""
        import numpy as np
        loss = np.zeros(1, np.float64)
        ga = np.zeros(int(p), np.float64)
        _check(lib().cpra_b200_slice_loss_grad(self._h, _addr(V), _addr(angles), _addr(A), int(m), int(n), int(p),
                                               int(l), _addr(grad_V), loss.ctypes.data_as(C.c_void_p),
                                               ga.ctypes.data_as(C.c_void_p)), "slice_loss_grad")
        return float(loss[0]), ga

    def slice_orient(self, V, angles, rot, m, n, p, l, out) -> bool:
        """Central slices at tilts `angles` and in-plane rotations `rot`
        (None: none) (project-defined)."""
        return _check(lib().cpra_b200_slice_orient(self._h, _addr(V), _addr(angles), _addr(rot), int(m), int(n),
                                                   int(p), int(l), _addr(out)), "slice_orient")

    def slice_loss_grad_orient(self, V, angles, rot, A, m, n, p, l, grad_V):
        """(loss, dL/dangles, dL/drot) for the two-parameter orientations;
        grad_V is written."""
        import numpy as np
        loss = np.zeros(1, np.float64)
        ga = np.zeros(int(p), np.float64)
        gr = np.zeros(int(p), np.float64)
        _check(lib().cpra_b200_slice_loss_grad_orient(self._h, _addr(V), _addr(angles), _addr(rot), _addr(A), int(m),
                                                      int(n), int(p), int(l), _addr(grad_V),
                                                      loss.ctypes.data_as(C.c_void_p), ga.ctypes.data_as(C.c_void_p),
                                                      gr.ctypes.data_as(C.c_void_p)), "slice_loss_grad_orient")
        return float(loss[0]), ga, gr

    def volume_loss_grad(self, vol, angles, rot, A, m, n, p, l, grad_vol):
        """(loss, dL/dangles, dL/drot) of a real-space volume through
        Forward3D, the slice operator and the modulus loss; grad_vol (real,
        device) is written."""
        import numpy as np
        loss = np.zeros(1, np.float64)
        ga = np.zeros(int(p), np.float64)
        gr = np.zeros(int(p), np.float64)
        _check(lib().cpra_b200_volume_loss_grad(self._h, _addr(vol), _addr(angles), _addr(rot), _addr(A), int(m),
                                                int(n), int(p), int(l), _addr(grad_vol),
                                                loss.ctypes.data_as(C.c_void_p), ga.ctypes.data_as(C.c_void_p),
                                                gr.ctypes.data_as(C.c_void_p)), "volume_loss_grad")
        return float(loss[0]), ga, gr

    def refine_orient(self, V, angles, rot, A, m, n, p, l, steps, real_space=False, lr_volume=1e-3, lr_angle=1e-3,
                      lr_rot=1e-3):
        """Adam steps on the volume (real-space with real_space), the tilts and
        the in-plane rotations (rot None: not refined); returns the loss before
        each step."""
        import numpy as np
        loss = np.zeros(max(int(steps), 1), np.float64)
        _check(lib().cpra_b200_refine_orient(self._h, _addr(V), 1 if real_space else 0, _addr(angles), _addr(rot),
                                             _addr(A), int(m), int(n), int(p), int(l), int(steps), float(lr_volume),
                                             float(lr_angle), float(lr_rot), loss.ctypes.data_as(C.c_void_p)),
               "refine_orient")
        return loss[:int(steps)]

    def constraint3d(self, x, C, S, iters=1) -> bool:
        """iters x (Forward3D, complex DataConstraint with C, Backward3D,
        SpaceConstraint with S) on the context's volumes, fused."""
        return _check(lib().cpra_b200_constraint3d(self._h, _addr(x), _addr(C), _addr(S), int(iters)),
                      "constraint3d")

    def refine(self, V, angles, A, m, n, p, l, steps, lr_volume=1e-3, lr_angle=1e-3):
        """Adam steps on the volume and the angles against the amplitude loss
        (project-defined); V and angles are updated in place; returns the loss
        before each step (numpy float64)."""
        import numpy as np
        loss = np.zeros(max(int(steps), 1), np.float64)
        _check(lib().cpra_b200_refine(self._h, _addr(V), _addr(angles), _addr(A), int(m), int(n), int(p), int(l),
                                      int(steps), float(lr_volume), float(lr_angle), loss.ctypes.data_as(C.c_void_p)),
               "refine")
        return loss[:int(steps)]

    def best_start(self, x, A, P, batch, best_out=None):
        """(best start index, per-start scores) by the mean R-factor over the
        P angles (project-defined); best_out (device) receives its planes."""
        import numpy as np
        scores = np.zeros(int(batch), np.float64)
        best = np.zeros(1, np.uint64)
        _check(lib().cpra_b200_best_start(self._h, _addr(x), _addr(A), int(P), int(batch),
                                          scores.ctypes.data_as(C.c_void_p), best.ctypes.data_as(C.c_void_p),
                                          _addr(best_out)), "best_start")
        return int(best[0]), scores

    def rfactor(self, x, A, batch, a_stride=0):
        """R-factor per pattern, sum | |Forward2D(x_b)| - A_b | / sum A_b in
        double (project-defined metric); returns a numpy float64 array."""
        import numpy as np
        out = np.zeros(int(batch), np.float64)
        _check(lib().cpra_b200_rfactor(self._h, _addr(x), _addr(A), int(a_stride), int(batch),
                                       out.ctypes.data_as(C.c_void_p)), "rfactor")
        return out

    def kernel_timing(self):
        """(ms, launches, pattern_iterations) of the fused launches timed since
        the last call (needs set_option(OPT_KERNEL_TIMING, 1))."""
        ms, n, pi = C.c_double(), C.c_uint64(), C.c_uint64()
        _check(lib().cpra_b200_kernel_timing(self._h, C.byref(ms), C.byref(n), C.byref(pi)), "kernel_timing")
        return ms.value, n.value, pi.value

    def alloc(self, nbytes: int, managed: bool = True) -> int:
        p = C.c_void_p()
        _check(lib().cpra_b200_alloc(self._h, C.byref(p), int(nbytes), 1 if managed else 0), "alloc")
        return p.value or 0

    def free(self, ptr: int) -> bool:
        return _check(lib().cpra_b200_free(self._h, int(ptr)), "free")


def _host_addr(a) -> int:
    if isinstance(a, int):
        return a
    if hasattr(a, "ctypes"):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    raise TypeError("a host buffer (numpy array, CPU tensor or address) is required")


def NewCpraImpl(impl_type, m, n, l, batch_size, dtype: str = "float32") -> B200Impl:
    """Factory of include/Impl_Factory.hpp:14-30 with the B200 case; like the
    reference it throws for a type that is not compiled in."""
    if IMPL_TYPE(impl_type) != IMPL_TYPE.B200:
        raise ValueError("Wrong impl type! Only the B200 backend is built in this package.")
    return B200Impl(m, n, l, batch_size, dtype)
