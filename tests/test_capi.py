"""The C-ABI library loads on a CPU host and exports every symbol the header
declares; the ctypes mirrors have the C layouts (checked against gcc)."""
import ctypes as C
import re
import subprocess
import sys

import pytest

from tests.conftest import ROOT

HEADER = ROOT / "include" / "hsc_c_api.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"HSC_EXPORT\s+[\w\s\*]+?\b(hsc_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from hsc_reimpl_b200 import build, _lib
    build.build()
    return _lib.load()


def test_header_declares_the_plugin_entry_points():
    syms = declared_symbols()
    for name in ("hsc_create", "hsc_destroy", "hsc_solve", "hsc_solve_batch", "hsc_spmv", "hsc_last_error",
                 "hsc_options_default", "hsc_options_reference"):
        assert name in syms


def test_library_exports_every_declared_symbol(lib):
    from hsc_reimpl_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (hsc_\w+)", out))
    assert set(declared_symbols()) <= exported
    assert set(_lib.EXPORTS) == set(declared_symbols())


def test_struct_layouts_match_c(tmp_path, lib):
    from hsc_reimpl_b200 import _lib
    src = tmp_path / "sz.c"
    src.write_text(f"""
#include <stdio.h>
#include <stddef.h>
#include "{HEADER}"
int main(void) {{
  printf("%zu %zu %zu %zu\\n", sizeof(hsc_options), sizeof(hsc_stats), sizeof(hsc_bcoo3), sizeof(hsc_dof_layout));
  printf("%zu %zu %zu %zu\\n", offsetof(hsc_options, poly_weights), offsetof(hsc_options, spin_limit),
         offsetof(hsc_stats, aca_relative_error), offsetof(hsc_stats, nnzb));
  return 0;
}}""")
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-std=c99", str(src), "-o", str(exe)], check=True)
    a, b = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")[:2]
    sizes = list(map(int, a.split()))
    offs = list(map(int, b.split()))
    assert sizes == [C.sizeof(_lib.Options), C.sizeof(_lib.Stats), C.sizeof(_lib.BCOO3), C.sizeof(_lib.Layout)]
    assert offs == [_lib.Options.poly_weights.offset, _lib.Options.spin_limit.offset,
                    _lib.Stats.aca_relative_error.offset, _lib.Stats.nnzb.offset]


def test_option_defaults_without_a_gpu(lib):
    from hsc_reimpl_b200 import _lib
    o = _lib.Options()
    assert lib.hsc_options_default(C.byref(o)) == 0
    assert o.neumann_order == 2 and o.abd_inverse == _lib.HSC_ABD_EXACT and o.precision == _lib.HSC_FP64
    r = _lib.Options()
    assert lib.hsc_options_reference(C.byref(r)) == 0
    # linear_hsc.cu:162-164 and integration.patch:33-54
    assert (r.max_rank, r.neumann_order, r.max_iter, r.omega, r.abd_inverse, r.abd_inverse_tol,
            r.full_residual_limit) == (128, 5, 2000, 0.7, _lib.HSC_ABD_ADAPTIVE, 1e-5, 0.1)
    assert lib.hsc_version() == 1
    assert lib.hsc_options_default(None) == _lib.HSC_ERR_INVALID


def test_plugin_selection_mirrors_do_build():
    from hsc_reimpl_b200.solver import LinearHSC, SimSystemException
    with pytest.raises(SimSystemException):
        LinearHSC().do_build({"linear_system/solver": "fused_pcg"})
    with pytest.raises(SimSystemException):
        LinearHSC().do_build({})                       # no solver key: not selected
    with pytest.raises(ValueError, match="Invalid HSC parameters"):
        LinearHSC().do_build({"linear_system/solver": "linear_hsc", "linear_system/hsc/omega": 1.5})
