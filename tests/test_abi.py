"""CPU-side checks of the C-ABI libraries: every function declared in
include/*.h is exported by each built library, and without a GPU the
library fails loudly instead of falling back to the CPU."""
import os
import re
import subprocess

import pytest

from conftest import ROOT, load_package

pkg = load_package()
from croma_fp_b200 import native, config  # noqa: E402

HEADERS = [os.path.join(ROOT, "include", h) for h in sorted(os.listdir(os.path.join(ROOT, "include")))
           if h.endswith(".h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(\w+)\s*\([^;{]*\)\s*;", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "return", "sizeof"):
                names.add(name)
    return sorted(names)


def built_libs():
    return [native.library_path(nb) for nb in (128, 256, 512) if os.path.exists(native.library_path(nb))]


def test_headers_declare_functions():
    assert len(declared_functions()) >= 15


@pytest.mark.parametrize("lib", built_libs() or [pytest.param(None, marks=pytest.mark.skip("library not built"))])
def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, f"{os.path.basename(lib)} lacks {missing}"


@pytest.mark.skipif(not built_libs(), reason="library not built")
def test_no_silent_cpu_fallback_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(native.CromaError, match="CUDA"):
        native.TracerFP(config.config0())
