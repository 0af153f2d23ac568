"""Host-side checks that need no GPU: the library loads, exports the C ABI,
and the input validation / version logic behaves like the reference."""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

from gb200 import lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"\b(gb200_[A-Za-z0-9_]+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    L = lib.load()
    names = declared_symbols()
    assert "gb200_gw_sigma" in names and "gb200_hf_fock" in names
    for n in sorted(names):
        assert hasattr(L, n), f"missing export {n}"
    assert set(lib.EXPORTED) <= names


def test_version_check_matches_reference_rules():
    # CheckVersion (common_defs.h:191-212) against INPUT_VERSION 1.0.0
    assert lib.check_integral_version("1.0.0")
    assert lib.check_integral_version("1.1.0")
    assert lib.check_integral_version("1.0.0b10")
    with pytest.raises(lib.mbpt_outdated_input):
        lib.check_integral_version("0.3.0")
    with pytest.raises(ValueError):
        lib.check_integral_version("garbage")


def test_create_rejects_bad_dims_without_gpu():
    # argument validation happens before any CUDA call
    with pytest.raises(lib.mbpt_wrong_grid):
        lib.Context(4, 6, 1, 20, 21, 20, 21, 20.0)
    with pytest.raises(lib.mbpt_kernel_error):
        lib.Context(4, 6, 3, 20, 20, 20, 21, 20.0)
    with pytest.raises(lib.mbpt_kernel_error, match="nso must equal nao"):
        lib.Context(4, 6, 1, 20, 20, 20, 21, 20.0, nso=7)  # neither scalar nor two-component
    with pytest.raises(lib.mbpt_kernel_error, match="nso must equal nao"):
        lib.Context(4, 6, 2, 20, 20, 20, 21, 20.0, nso=12)  # two-component input has ns = 1
    with pytest.raises(lib.mbpt_kernel_error, match="nso > 64"):
        lib.Context(4, 40, 1, 20, 20, 20, 21, 20.0, nso=80)


def test_null_context_is_an_error():
    L = lib.load()
    assert L.gb200_gw_sigma(None, None, None) == lib.ERR_INVALID
    assert L.gb200_set_contraction_slices(None, None) == lib.ERR_INVALID
    assert L.gb200_set_memory_budget(None, 1e9) == lib.ERR_INVALID
    assert L.gb200_gw_sigma_vjp(None, None, None, None, None) == lib.ERR_INVALID
    t = (ctypes.c_float * 4)()
    assert L.gb200_last_timings(None, t) == lib.ERR_INVALID


@pytest.mark.parametrize("compiler,std,ext", [("gcc", "c99", "c"), ("g++", "c++17", "cpp")])
def test_header_is_plain_c_and_cpp(tmp_path, compiler, std, ext):
    """include/gb200.h compiles as ISO C99 and C++17 with warnings as errors, and declares every
    entry point (each one's address is taken)."""
    cc = shutil.which(compiler)
    if cc is None:
        pytest.skip(f"{compiler} not installed")
    names = sorted(declared_symbols())
    table = ",\n  ".join(f"(fn)&{n}" for n in names)
    src = tmp_path / f"t.{ext}"
    src.write_text('#include "gb200.h"\n'
                   "typedef void (*fn)(void);\n"
                   f"static const fn table[] = {{\n  {table}\n}};\n"
                   "int main(void) { return table[0] == 0; }\n")
    r = subprocess.run([cc, f"-std={std}", "-Wall", "-Wextra", "-Werror", "-pedantic", "-fsyntax-only",
                        "-I", os.path.join(ROOT, "include"), str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
