"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(kw_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ("kw_plan_create", "kw_run", "kw_plan_destroy", "kw_last_error", "kw_plan_outputs"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from kwave_b200 import _abi
    lib = _abi.load_library()
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    from kwave_b200 import _abi
    assert declared_symbols() <= set(_abi.SYMBOLS), declared_symbols() - set(_abi.SYMBOLS)


def test_abi_version_and_error_without_gpu():
    from kwave_b200 import _abi
    lib = _abi.load_library()
    assert lib.kw_abi_version() == _abi.KW_ABI_VERSION
    # a NULL problem is rejected on the host, before any CUDA call
    h = ctypes.c_void_p()
    st = lib.kw_plan_create(None, ctypes.byref(h))
    assert st == _abi.KW_ERR_INVALID
    assert b"NULL" in lib.kw_last_error()


def test_struct_layout_matches_header():
    """Compile a probe against the header and compare sizeof / offsetof."""
    import shutil
    import subprocess
    import tempfile
    from kwave_b200 import _abi
    cc = shutil.which("gcc")
    if cc is None:
        pytest.skip("gcc not available")
    fields = ["dim", "Nx", "dt", "c_ref", "c0", "rho0_sgz", "pml_z_alpha", "use_kspace", "BonA_scalar",
              "alpha_sign", "p_source", "u_source", "p0_source_input", "sensor_num", "record",
              "time_reversal_input", "inside_hi"]
    prog = ['#include <stdio.h>', '#include <stddef.h>', '#include "kwave_b200.h"', 'int main(void){',
            'printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(kw_problem), sizeof(kw_source), sizeof(kw_outputs), '
            'sizeof(kw_output_desc), sizeof(kw_server_config), sizeof(kw_server_stats));']
    for f in fields:
        prog.append('printf("%%zu\\n", offsetof(kw_problem, %s));' % f)
    prog.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "probe.c")
        open(c, "w").write("\n".join(prog))
        exe = os.path.join(d, "probe")
        subprocess.run([cc, "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    sizes = [int(v) for v in out[:6]]
    assert sizes == [ctypes.sizeof(_abi.kw_problem), ctypes.sizeof(_abi.kw_source),
                     ctypes.sizeof(_abi.kw_outputs), ctypes.sizeof(_abi.kw_output_desc),
                     ctypes.sizeof(_abi.kw_server_config), ctypes.sizeof(_abi.kw_server_stats)]
    offs = [int(v) for v in out[6:]]
    assert offs == [getattr(_abi.kw_problem, f).offset for f in fields]
