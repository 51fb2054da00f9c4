"""The C-ABI library loads without a GPU and exports every declared symbol."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for fn in sorted(os.listdir(INC)):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(INC, fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        src = re.sub(r"#[^\n]*", "", src)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(([^;{}()]|\([^()]*\))*\)\s*;", src):
            name = m.group(1)
            if name in ("if", "while", "for", "return", "sizeof"):
                continue
            names.add(name)
    return names


def test_library_exports_all_declared_symbols():
    import hydrocode_astro1_b200 as hcb
    L = hcb.lib()   # loads without a GPU
    missing = [n for n in sorted(declared_functions()) if not hasattr(L, n)]
    assert not missing, f"declared in include/*.h but not exported: {missing}"


def test_python_mirror_covers_capi():
    import hydrocode_astro1_b200 as hcb
    src = open(os.path.join(INC, "hydrocode_b200.h")).read()
    hc_names = set(re.findall(r"\b(hc_[a-z_0-9]+)\s*\(", src))
    assert hc_names <= set(hcb.CAPI), sorted(hc_names - set(hcb.CAPI))


def test_no_gpu_error_is_loud():
    import hydrocode_astro1_b200 as hcb
    if hcb.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(hcb.HcError):
        hcb.HydroSolver3D((8, 8, 8))
