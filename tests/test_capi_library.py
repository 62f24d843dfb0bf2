"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: these run without a GPU)."""
import ctypes
import re
from pathlib import Path

import pytest

from conftest import REPO

HEADERS = sorted((REPO / "include").glob("*.h"))


def declared_symbols():
    names = set()
    for h in HEADERS:
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(?:int|const char\*|void|uint64_t)\s+(cpra_b200_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    syms = declared_symbols()
    for required in ("cpra_b200_create", "cpra_b200_forward2d", "cpra_b200_backward2d", "cpra_b200_merge_add",
                     "cpra_b200_converge_error", "cpra_b200_dm_iterations", "cpra_b200_sync"):
        assert required in syms


def test_library_exports_every_declared_symbol():
    import cpra_b200
    path = cpra_b200.library_path()
    assert path.exists(), f"{path} not built"
    lib = ctypes.CDLL(str(path))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_bindings_cover_every_symbol():
    import cpra_b200
    bound = set(cpra_b200._SIGS) | {"cpra_b200_last_error", "cpra_b200_kernels_launched"}
    extra = [s for s in declared_symbols() if s not in bound]
    assert not extra, f"declared but not bound in Python: {extra}"


def test_bindings_cover_every_option():
    """Every CPRA_B200_OPT_* of the header has a Python constant of the same value."""
    import cpra_b200
    opts = {}
    for h in HEADERS:
        for m in re.finditer(r"#define\s+CPRA_B200_(OPT_\w+)\s+(\d+)", h.read_text()):
            opts[m.group(1)] = int(m.group(2))
    assert "OPT_LANES" in opts and "OPT_IO_CHUNK" in opts
    for name, value in opts.items():
        assert getattr(cpra_b200, name, None) == value, name


def test_no_cpu_fallback_in_package():
    """The product path has no CPU implementation: it never imports the oracle."""
    pkg = REPO / "carousel-phase-retrieval-algorithm_b200"
    for f in list(pkg.rglob("*.py")) + list(pkg.rglob("*.cu")) + list((REPO / "include").rglob("*")):
        if f.is_file():
            t = f.read_text(errors="replace")
            assert "cpra_oracle" not in t and "ref_lib" not in t, f


def test_factory_rejects_other_backends():
    import cpra_b200
    with pytest.raises(ValueError):
        cpra_b200.NewCpraImpl(cpra_b200.IMPL_TYPE.MKL, 4, 4, 1, 1)
