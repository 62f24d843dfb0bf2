"""Location of the reference checkout for the build recipes: the environment
variable CPRA_REFERENCE_DIR, else the default of REFERENCE_DIR in
oracle/Makefile, so that the path is written in one place."""
from __future__ import annotations

import os
import re
from pathlib import Path

_MAKEFILE = Path(__file__).resolve().parent / "Makefile"


def reference_dir() -> Path:
    env = os.environ.get("CPRA_REFERENCE_DIR")
    if env:
        return Path(env)
    m = re.search(r"^REFERENCE_DIR\s*\?=\s*\$\(or \$\(CPRA_REFERENCE_DIR\),(.+)\)\s*$", _MAKEFILE.read_text(),
                  re.MULTILINE)
    if not m:
        raise RuntimeError("oracle/Makefile has no REFERENCE_DIR default")
    return Path(m.group(1).strip())
