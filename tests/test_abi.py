"""The C ABI: libhydro_b200.so loads without a GPU and exports every function
include/hydro_b200.h declares; the structures in the header and in the
ctypes binding have the reference's layout (tests/golden/abi_layout.json,
generated from the reference's parametres.h)."""
import ctypes as C
import json
import os
import re
import subprocess

import pytest

from hydro_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hydro_b200.h")
GOLDEN = os.path.join(ROOT, "tests", "golden", "abi_layout.json")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"^\s*#.*$", "", src, flags=re.M)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", src)
    return sorted(set(n for n in names if n not in ("if", "while", "sizeof")))


def test_header_declares_reference_entry_points():
    names = declared_functions()
    for ref in ("hydro_godunov", "compute_deltat", "make_boundary", "compute_deltat_init_mem",
                "compute_deltat_clean_mem"):
        assert ref in names


def test_library_exports_every_declared_symbol(product_lib):
    missing = [n for n in declared_functions() if not hasattr(product_lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(declared_functions()) <= bound


def test_ctypes_layout_matches_reference():
    g = json.load(open(GOLDEN))
    H = _lib.HydroParam
    assert C.sizeof(H) == g["sizeof"]
    for name, off in g.items():
        if name.startswith("sizeof"):
            continue
        assert getattr(H, name).offset == off, name
    assert C.sizeof(_lib.HydroVar) == g["sizeof_hydrovar_t"]
    assert C.sizeof(_lib.HydroWork) == g["sizeof_hydrowork_t"]
    assert C.sizeof(_lib.HydroVarWork) == g["sizeof_hydrovarwork_t"]


def test_c_header_layout_matches_reference(tmp_path):
    g = json.load(open(GOLDEN))
    fields = [k for k in g if not k.startswith("sizeof")]
    prog = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void){",
            'printf("%zu\\n", sizeof(hydroparam_t));']
    prog += [f'printf("%zu\\n", offsetof(hydroparam_t, {f}));' for f in fields]
    prog += ['printf("%zu %zu %zu\\n", sizeof(hydrovar_t), sizeof(hydrowork_t), '
             'sizeof(hydrovarwork_t));', "return 0;}"]
    src = tmp_path / "lay.c"
    src.write_text("\n".join(prog))
    exe = tmp_path / "lay"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    vals = [int(x) for x in out]
    assert vals[0] == g["sizeof"]
    assert vals[1:1 + len(fields)] == [g[f] for f in fields]
    assert vals[-3:] == [g["sizeof_hydrovar_t"], g["sizeof_hydrowork_t"],
                         g["sizeof_hydrovarwork_t"]]


def test_library_has_no_oracle_dependency(product_lib):
    """The product never links the checkers."""
    out = subprocess.run(["nm", "-D", _lib.LIB_PATH], capture_output=True, text=True).stdout
    assert "orc_" not in out and "ref_create" not in out
    ldd = subprocess.run(["ldd", _lib.LIB_PATH], capture_output=True, text=True).stdout
    assert "oracle" not in ldd and "hydroref" not in ldd


def test_errors_are_reported_not_fatal(product_lib):
    """Invalid parameters record an error (the reference aborts instead)."""
    from hydro_b200 import make_params
    H = make_params(16, 16)
    H.nvar = 5
    d = product_lib.hydro_b200_domain_create(C.byref(H))
    assert not d
    assert product_lib.hydro_b200_last_error() == _lib.HB_ERR_ARG
    assert b"nvar" in product_lib.hydro_b200_last_error_message()
    product_lib.hydro_b200_clear_error()
    H = make_params(2, 16)
    assert not product_lib.hydro_b200_domain_create(C.byref(H))
    assert product_lib.hydro_b200_last_error() == _lib.HB_ERR_ARG
    product_lib.hydro_b200_clear_error()


def test_missing_library_fails_loudly(tmp_path):
    """Without the built library the package raises: it has no CPU path to
    fall back on.  Run in a child so this process keeps its loaded library."""
    code = (
        "from hydro_b200 import _lib, make_params, Domain\n"
        f"_lib.LIB_PATH = {str(tmp_path / 'libhydro_b200.so')!r}\n"
        "try:\n"
        "    Domain(make_params(32, 32))\n"
        "except _lib.HydroB200Error as e:\n"
        "    assert 'no CPU fallback' in str(e), e\n"
        "    print('raised')\n")
    r = subprocess.run(["python", "-c", code], capture_output=True, text=True, cwd=ROOT)
    assert r.returncode == 0 and r.stdout.strip() == "raised", (r.stdout, r.stderr)
