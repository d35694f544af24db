"""The C-ABI library loads, exports every symbol declared in include/*.h, and
its struct layouts agree with the Python bindings (no GPU calls)."""
import ctypes
import glob
import os
import re
import subprocess

import pytest

import mgkmc_cpp_b200._lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        for m in re.finditer(r"MGK_API\s+[\w\s\*]+?\b(mgk_\w+)\s*\(", open(h).read()):
            syms.add(m.group(1))
    return syms


def test_library_exports_all_declared_symbols():
    lib = L.lib()
    syms = declared_symbols()
    assert len(syms) >= 14
    for s in sorted(syms):
        assert hasattr(lib, s), s
    assert set(L.EXPORTS) <= syms


def test_version_and_error_without_gpu_calls():
    lib = L.lib()
    assert lib.mgk_version() >= 100
    assert isinstance(lib.mgk_last_error(), bytes)


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text("""
#include <stdio.h>
#include <stddef.h>
#include "mgkmc_b200.h"
int main(void) {
    printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(mgk_kmc_params), offsetof(mgk_kmc_params, ls_max_iter),
           offsetof(mgk_kmc_params, bar_ratio), sizeof(mgk_run_params), offsetof(mgk_run_params, max_events),
           offsetof(mgk_run_params, vtk_elastic_only));
    return 0;
}
""")
    exe = tmp_path / "layout"
    r = subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], capture_output=True, text=True)
    if r.returncode != 0:
        pytest.skip("no C compiler: " + r.stderr[-200:])
    vals = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    P, R = L.KmcParamsC, L.RunParamsC
    assert vals == [ctypes.sizeof(P), P.ls_max_iter.offset, P.bar_ratio.offset, ctypes.sizeof(R), R.max_events.offset,
                    R.vtk_elastic_only.offset]


def test_python_api_fails_loudly_without_device():
    import mgkmc_cpp_b200 as G
    if L.lib().mgk_device_count() > 0:
        pytest.skip("a device is present")
    with pytest.raises(L.MgkError):
        G.LsSolver((4, 4), [1e9] * 16, [0.3] * 16)
