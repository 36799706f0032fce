"""Build tests/golden/run07007_grid_growth.npz from the reference's no-Pardiso regression run 07007.

That run (tests/sim_no_pardiso_reg/run07007 in the reference: smallRectangle.mesh, modelinput07007)
grows a three-layer rectangle with two grid-based growth functions (type 3, nearest-corner
interpolation, grids pinned on the initial mesh, z range 0.5-1): one in z from 120 s and one in x, y
from 60 s, both until 300 s, with explicit ECM and actin layers, for 11 steps of 60 s without
solving the mechanics. Its recorded growth tensors also carry column-wise volume conservation,
which this path does not compute, but its log (expected_out/tmp) prints the diagonal of every
grid-growth increment as it is made (ShapeBase::calculateFgFromGridCorners, ShapeBase.cpp:640-643):
per step, function by function in input order, element by element, the three values exp(rate dt)
to six significant digits. Those increments pin the grid-growth restatement.

The fixture keeps the mesh, the model input's tokens, the text of both grid files and, per step,
the logged increments.

Run from the repository root with the reference's checkout given:
    REFERENCE_ROOT=<path to the reference> python tests/golden/make_run07007_grid_growth.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from tissueorigami_b200 import mesh  # noqa: E402


def main():
    ref = os.environ.get("REFERENCE_ROOT")
    if not ref:
        raise SystemExit("set REFERENCE_ROOT to the reference checkout")
    run = os.path.join(ref, "tests", "sim_no_pardiso_reg", "run07007")
    x, place, ttype, circ, conn, xref = mesh.read_mesh(os.path.join(run, "smallRectangle.mesh"))
    text = open(os.path.join(run, "modelinput07007")).read()
    tokens = text.split()
    names = [tokens[i + 1] for i, t in enumerate(tokens) if t == "Filename(full-path):"]
    grids = {n: open(os.path.join(run, n)).read() for n in names if "ShapeChangeRate" in n}
    times, counts, values = [], [], []
    cur = None
    for line in open(os.path.join(run, "expected_out", "tmp")):
        if line.startswith("At time -- "):
            if cur is not None:
                times.append(cur[0])
                counts.append(len(cur[1]) // 3)
                values.extend(cur[1])
            cur = (float(line.split()[3]), [])
        elif line.startswith("Inside ShapeBase::calculateFgFromGridCorners") and cur is not None:
            axis, val = line.split("[Increment]:")[1].split()[:2]
            assert int(axis) == len(cur[1]) % 3
            cur[1].append(float(val))
    if cur is not None:
        times.append(cur[0])
        counts.append(len(cur[1]) // 3)
        values.extend(cur[1])
    out = os.path.join(HERE, "run07007_grid_growth.npz")
    np.savez_compressed(out, x=x, place=place, ttype=ttype, circ=circ, conn=conn, xref=xref,
                        modelinput_tokens=np.array(tokens), grid_names=np.array(list(grids)),
                        grid_texts=np.array([grids[n] for n in grids]), times=np.array(times),
                        counts=np.array(counts), increments=np.array(values).reshape(-1, 3))
    print(f"wrote {out}: {conn.shape[0]} elements, steps at {times}, {sum(counts)} logged increments")


if __name__ == "__main__":
    main()
