"""CPU checks of the C ABI boundary: the library builds for sm_100a, loads without a GPU, and
exports every entry point that include/tf_b200.h declares (no compute call is made)."""
import ctypes
import os
import re

from tissueorigami_b200 import build, capi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "tf_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tf_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_bound_exports():
    assert sorted(capi.EXPORTS) == declared_functions()


def test_library_exports_every_declared_symbol():
    path = build.build()
    lib = ctypes.CDLL(path)
    missing = [f for f in declared_functions() if not hasattr(lib, f)]
    assert not missing, missing


def test_default_params_and_version_without_gpu():
    L = capi.load()
    p = capi.default_params()
    assert p.max_newton_iters == 20 and abs(p.newton_tol - 1e-8) < 1e-20
    assert b"sm_100a" in L.tf_version()


def test_create_rejects_bad_mesh_without_touching_the_gpu():
    L = capi.load()
    conn = (ctypes.c_int32 * 6)(0, 1, 2, 3, 4, 99)
    xref = (ctypes.c_double * 18)()
    desc = capi.MeshDesc(6, 1, ctypes.cast(conn, ctypes.POINTER(ctypes.c_int32)),
                         ctypes.cast(xref, ctypes.POINTER(ctypes.c_double)))
    h = ctypes.c_void_p()
    assert L.tf_create(ctypes.byref(desc), None, ctypes.byref(h)) == capi.TF_ERR_ARGUMENT
    assert not h.value
