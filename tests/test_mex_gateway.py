"""The MATLAB MEX gateway (k-wave-ii_b200/mex/kwave_b200_mex.c) compiles
against the C ABI and links to the library.

MATLAB is not installed here, so the gateway is compiled against a stub
mex.h that declares the documented MEX / mx API subset it uses
(k-wave-ii_b200/mex/stub/mex.h); every C-ABI symbol it calls must be
declared in include/kwave_b200.h and exported by libkwave_b200.so.  No
compute call is made (this runs without a GPU)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MEX = os.path.join(ROOT, "k-wave-ii_b200", "mex")


def _undefined(obj):
    out = subprocess.run(["nm", "-u", obj], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_gateway_compiles_against_the_abi(tmp_path):
    obj = str(tmp_path / "kwave_b200_mex.o")
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-c",
                        "-I", os.path.join(MEX, "stub"), "-I", os.path.join(ROOT, "include"),
                        os.path.join(MEX, "kwave_b200_mex.c"), "-o", obj], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    und = _undefined(obj)
    assert "mexFunction" not in und
    kw_calls = {s for s in und if s.startswith("kw_")}
    assert {"kw_plan_create", "kw_plan_outputs", "kw_run", "kw_plan_destroy", "kw_last_error"} <= kw_calls
    from test_abi import declared_symbols
    from kwave_b200 import _abi
    lib = _abi.load_library()
    assert kw_calls <= declared_symbols()
    assert all(hasattr(lib, s) for s in kw_calls)
    # the link a `mex ... -lkwave_b200` build performs (MEX / mx symbols are
    # MATLAB's; only the library's must resolve here)
    so = str(tmp_path / "kwave_b200_mex.so")
    libdir = os.path.dirname(_abi.LIB_PATH)
    r = subprocess.run(["gcc", "-shared", "-o", so, obj, "-L", libdir, "-lkwave_b200",
                        "-Wl,--unresolved-symbols=ignore-all"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
