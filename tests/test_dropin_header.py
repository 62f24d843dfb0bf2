"""The C++ drop-in backend header compiles against the operator interface:
the project's restatement always, the reference's own include/CPRA_Impl.hpp
when the reference tree is present (compile-time only, no GPU)."""
import shutil
import subprocess
from pathlib import Path

import pytest

from conftest import REPO

from reference_dir import reference_dir

REF_INCLUDE = reference_dir() / "include"
TU = r'''
#include "cpra_b200/B200_Impl.hpp"
#include <memory>
int main() {
    // instantiating the class checks that every pure virtual is overridden
    std::unique_ptr<CPRA::CpraImpl<float>> f = CPRA::NewB200Impl<float>(8, 8, 1, 1);
    std::unique_ptr<CPRA::CpraImpl<double>> d = CPRA::NewB200Impl<double>(10, 10, 1, 1);
    return f && d ? 0 : 1;
}
'''


def _compile(tmp_path, extra):
    cxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else shutil.which("g++")
    src = tmp_path / "tu.cpp"
    src.write_text(TU)
    r = subprocess.run([cxx, "-std=c++17", "-fsyntax-only", "-Wall", "-Werror=overloaded-virtual",
                        "-I", str(REPO / "include"), *extra, str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_header_compiles_standalone(tmp_path):
    _compile(tmp_path, ["-DCPRA_B200_STANDALONE"])


@pytest.mark.skipif(not (REF_INCLUDE / "CPRA_Impl.hpp").exists(), reason="reference tree not present")
def test_header_compiles_against_reference_interface(tmp_path):
    _compile(tmp_path, ["-I", str(REF_INCLUDE)])
