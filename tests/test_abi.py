"""CPU checks of the drop-in boundary: the C-ABI library loads without a GPU
and exports every entry point that include/*.h declares."""
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "cudakdtree_b200", "lib", "libcukd_b200.so")


def declared_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        syms |= set(re.findall(r"CUKD_API\s+[\w\s\*]*?\b(cukd_\w+)\s*\(", src))
    return syms


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("cukd_build_tree", "cukd_fcp", "cukd_knn", "cukd_compute_bounds"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        pytest.fail("libcukd_b200.so not built (run __graft_entry__.build())")
    out = subprocess.check_output(["nm", "-D", "--defined-only", LIB], text=True)
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = declared_symbols() - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"


def test_library_loads_without_gpu():
    import cudakdtree_b200 as ck
    L = ck.lib()
    assert L.cukd_status_string(2).decode().startswith("asked to build")
    p = ck.QueryParams()
    L.cukd_query_params_init(p)
    assert p.method == 0 and p.k == 8 and p.flags == ck.QUERY_MORTON


def test_invalid_layouts_are_rejected_before_any_device_work():
    import ctypes as C
    import cudakdtree_b200 as ck
    L = ck.lib()
    bad = [ck.layout_for("float32", 9), ck.layout_for("float32", 1), ck.layout_for("float32", 3, stride=10),
           ck.layout_for("float32", 3, stride=16, point_offset=8),
           ck.layout_for("float32", 3, stride=16, dim_offset=14),
           ck.layout_for("float32", 4, stride=20, dim_offset=16, dim_shift=31, dim_bits=1)]
    for lay in bad:
        assert L.cukd_build_tree(None, 10, C.byref(lay), None, 0, None, None) == 1
    # empty input is a no-op even without a device (builder_thrust.h:441)
    assert L.cukd_build_tree(None, 0, C.byref(ck.layout_for("float32", 3)), None, 0, None,
                             None) == 0
