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


def test_host_buffer_knn_refuses_bad_arguments_before_any_device_work():
    """The host-buffer kNN entry points check their arguments before they
    create a stream or touch memory: no queries, no answer buffer, k out of
    range, a bad layout or (asynchronous forms) no completion event give
    CUKD_ERR_INVALID_ARGUMENT; an empty batch is a no-op."""
    import ctypes as C
    import cudakdtree_b200 as ck
    L = ck.lib()
    lay = ck.layout_for("float32", 3)
    p = ck.QueryParams()
    L.cukd_query_params_init(p)
    p.k = 16
    fake = C.c_void_p(4096)  # never dereferenced: every call below fails first
    host = L.cukd_knn_host, L.cukd_knn_to_host
    for f in host:
        assert f(fake, 10, C.byref(lay), None, None, 5, C.byref(p), fake, fake, 0, None, None) == 1
        assert f(fake, 10, C.byref(lay), None, fake, 5, C.byref(p), None, fake, 0, None, None) == 1
        assert f(fake, 10, C.byref(ck.layout_for("float32", 9)), None, fake, 5, C.byref(p), fake,
                 fake, 0, None, None) == 1
        assert f(fake, 10, C.byref(lay), None, fake, 0, C.byref(p), fake, fake, 0, None, None) == 0
    for f in (L.cukd_knn_host_async, L.cukd_knn_to_host_async):
        assert f(fake, 10, C.byref(lay), None, fake, 5, C.byref(p), fake, fake, 0, None, None,
                 None) == 1  # no event
        assert f(fake, 10, C.byref(lay), None, None, 5, C.byref(p), fake, fake, 0, fake, None,
                 None) == 1  # no queries
    bad_k = ck.QueryParams()
    L.cukd_query_params_init(bad_k)
    for k in (0, 1025):
        bad_k.k = k
        for f in host:
            assert f(fake, 10, C.byref(lay), None, fake, 5, C.byref(bad_k), fake, fake, 0, None,
                     None) == 1
