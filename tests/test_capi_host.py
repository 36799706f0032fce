"""A C++ host of the C ABI: tests/capi_host.cpp built with g++ and linked against libtf_b200.so,
as a C++ simulator would link it (no Python between the host and the library).

CPU: the host compiles and links with warnings as errors. GPU: it runs the small rectangle (342
prisms, 10 implicit steps of 60 s, Newton tolerance 1e-10) through tf_create / tf_set_* /
tf_time_step, and its positions and Newton iteration counts match the oracle's dense-LU run to
1e-9 of the tissue size.
"""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from tissueorigami_b200 import build, mesh

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _build_host(tmp_path):
    exe = str(tmp_path / "capi_host")
    lib_dir = os.path.dirname(build.build())
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(HERE, "capi_host.cpp"), "-L", lib_dir, "-ltf_b200", f"-Wl,-rpath,{lib_dir}", "-o", exe]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return exe


def test_host_compiles_and_links(tmp_path):
    exe = _build_host(tmp_path)
    assert os.path.exists(exe)


def _write_input(path, t, n_steps):
    with open(path, "wb") as f:
        np.array([t.n_nodes, t.n_elems, n_steps], np.int32).tofile(f)
        np.array([t.dt, t.newton_tol], np.float64).tofile(f)
        for a, dt in ((t.conn, np.int32), (t.xref, np.float64), (t.x, np.float64), (t.lam, np.float64),
                      (t.mu, np.float64), (t.eta, np.float64), (t.fixed, np.uint8), (t.ext_visc, np.float64),
                      (t.rates, np.float64), (t.angles, np.float64), (t.exposed, np.uint8), (t.peripodial, np.uint8)):
            np.ascontiguousarray(a, dtype=dt).tofile(f)


@pytest.mark.gpu
def test_host_steps_the_small_rectangle_like_the_oracle(tmp_path):
    exe = _build_host(tmp_path)
    t = mesh.small_rectangle()
    n_steps = 10
    _write_input(tmp_path / "in.bin", t, n_steps)
    res = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    out = np.fromfile(tmp_path / "out.bin", dtype=np.uint8)
    x = out[:8 * 3 * t.n_nodes].view(np.float64).reshape(-1, 3)
    iters = out[8 * 3 * t.n_nodes:].view(np.int32)
    x_ref, _, it_ref, _ = O.simulate_dense(t, n_steps=n_steps)
    assert list(iters) == list(it_ref)
    assert np.abs(x - x_ref).max() <= 1e-9 * t.size
