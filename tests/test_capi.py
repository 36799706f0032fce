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


def _compiler(lang):
    import shutil

    import pytest

    cc = shutil.which("gcc" if lang == "c" else "g++")
    if cc is None:
        pytest.skip("no host compiler")
    return cc, ("-std=c99" if lang == "c" else "-std=c++17")


def _compile(tmp_path, src, lang, run):
    import subprocess

    cc, std = _compiler(lang)
    f = tmp_path / ("probe.c" if lang == "c" else "probe.cpp")
    f.write_text(src)
    flags = [cc, std, "-Wall", "-Wextra", "-Werror", "-I", os.path.dirname(HEADER), str(f)]
    if not run:  # a link would need the CUDA runtime: check the translation unit only
        subprocess.run(flags + ["-fsyntax-only"], check=True)
        return ""
    exe = tmp_path / "probe"
    subprocess.run(flags + ["-o", str(exe)], check=True)
    return subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout


def test_header_compiles_as_c_and_cpp(tmp_path):
    """A C or C++ host includes the header alone (no CUDA headers) and can take every entry
    point's address with the declared signature."""
    names = declared_functions()
    decls = "\n".join(f"    const void* f_{i} = (const void*)&{n};" for i, n in enumerate(names))
    uses = "\n".join(f'    printf("%d\\n", (int)(f_{i} != 0));' for i in range(len(names)))
    src = "#include <stdio.h>\n#include \"tf_b200.h\"\nint main(void) {\n" + decls + "\n" + uses + "\n    return 0;\n}\n"
    for lang in ("c", "cpp"):
        _compile(tmp_path, src, lang, run=False)


def test_ctypes_structs_match_the_c_layout(tmp_path):
    """The Python mirrors of tf_params, tf_step_stats and tf_mesh_desc have the C sizes and
    field offsets (the boundary passes them by pointer)."""
    structs = {"tf_params": capi.Params, "tf_step_stats": capi.StepStats, "tf_mesh_desc": capi.MeshDesc}
    lines = []
    for cname, py in structs.items():
        lines.append(f'    printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'    printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    src = ("#include <stddef.h>\n#include <stdio.h>\n#include \"tf_b200.h\"\nint main(void) {\n" + "\n".join(lines)
           + "\n    return 0;\n}\n")
    got = {}
    for line in _compile(tmp_path, src, "c", run=True).splitlines():
        cname, what, val = line.split()
        got[(cname, what)] = int(val)
    for cname, py in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)
