"""The C-ABI library loads and exports every entry declared in
include/ductgpu.h (no GPU needed; no compute calls)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(ductgpu_\w+|\w+_gpu_)\s*\(", src))
    return names


def test_header_declares_entries():
    assert {"ductgpu_create", "ductgpu_helm3d", "ductgpu_solve_fields_dev",
            "ductgpu_pseudomat"} <= declared()


def test_library_exports_every_declared_symbol():
    import duct_b200 as D
    L = D.lib()
    missing = [n for n in sorted(declared()) if not hasattr(L, n)]
    assert not missing, missing
    assert set(D.EXPORTS) <= declared()


def test_create_without_device_returns_status():
    import duct_b200 as D
    h = C.c_void_p()
    rc = D.lib().ductgpu_create(10_000, C.byref(h))
    assert rc != 0 and not h.value


def test_null_context_is_rejected():
    import duct_b200 as D
    L = D.lib()
    assert L.ductgpu_pseudomat(None, 33, 33) == D.EARG
    assert L.ductgpu_destroy(None) == D.EARG
    assert L.ductgpu_launch_count(None) == -1
    assert L.ductgpu_synchronize(None) == D.EARG
    assert L.ductgpu_selftest_wait_timeout(None, 16) == D.EARG


@pytest.mark.parametrize("lang", ["c", "c++"])
def test_header_compiles_for_c_and_cpp_hosts(tmp_path, lang):
    """include/ductgpu.h is plain C (a Fortran host binds it through
    ISO_C_BINDING; a C or C++ host includes it directly)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc" if lang == "c" else "g++")
    if cc is None:
        pytest.skip("no host compiler")
    src = tmp_path / "use.c"
    src.write_text('#include "ductgpu.h"\n'
                   'int main(void) { ductgpu_h5_header h; h.my = 1; (void)h; return DUCTGPU_OK; }\n')
    std = ["-std=c99", "-pedantic"] if lang == "c" else ["-std=c++11", "-x", "c++"]
    r = subprocess.run([cc, *std, "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-c", str(src), "-o",
                        str(tmp_path / "use.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_integration_interface_blocks_name_real_entries():
    """Every bind(C, name=...) of the Fortran interface blocks in
    INTEGRATION.md is declared in the header and exported by the library."""
    import duct_b200 as D
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    bound = set(re.findall(r'bind\(C,\s*name="(\w+)"\)', text))
    assert bound, "no interface blocks found"
    L = D.lib()
    assert bound <= declared(), sorted(bound - declared())
    assert all(hasattr(L, n) for n in bound)
