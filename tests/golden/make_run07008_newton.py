"""Build tests/golden/run07008_newton_step1.npz from the reference's Pardiso regression run 07008.

That run (tests/sim_pardiso_reg/run07008 in the reference; input files shared with
tests/sim_no_pardiso_reg/run07008) is the reference's own Newton-Raphson path with Pardiso on
a wing-disc mesh (144 nodes, 138 prisms in three layers: explicit basal ECM, columnar, apical
actin layer), uniform growth (0.2 / 0.1 per hour at 45 degrees, columnar layer), 3600 s steps,
y-symmetry and the circumference bound in x, y to the basal layer. Its expected_out records:

  Save_Frame        node positions after every step (10 significant digits)
  Save_PhysicalProp per element Young's modulus, internal viscosity, z remodelling; per node
                    the external viscosity (x, y, z)
  Save_NodeBinding  the slave -> master DoF pairs
  Save_SpecificElementAndNodeTypes   the actin and ECM element ids
  tmp               the log, with ||dU|| of every Newton iteration

The first step involves only what this library's path computes (growth prologue, element forces
and tangents, external drag, fixed DoFs, slave-master elimination, Newton loop): from the second
step on the run adds explicit-ECM remodelling, adhesion and node collapse, which are out of scope.
The fixture keeps the step-1 inputs and the recorded step-1 results:

  * the mesh; E per element, Poisson's ratio 0.29 (0 for ECM elements, Simulation.cpp:4030-4036);
    no internal viscosity; the external viscosity of every node;
  * fixed DoFs: y of every node with |y| < 0.1 (setupYsymmetricity, Simulation.cpp:9557-9567);
  * the binding pairs. Save_NodeBinding leaves out pairs whose master is node 0 (its writer keeps
    slaveTo[i] > 0, Simulation.cpp:8553), although the run binds node 0's column like every other
    circumference column (the recorded x of nodes 0, 36, 72, 108 coincide); those pairs - x of the
    nodes above node 0; their y is fixed like node 0's - are restored here;
  * exposed surfaces: basal face of the elements whose three basal nodes are basal, apical face
    of those whose three apical nodes are apical;
  * growth as in the no-Pardiso fixture (single-precision rates and angle, columnar elements);
  * the recorded positions after step 1 and the recorded ||dU|| trace of step 1;
  * the model input file's tokens (for the test of tissueorigami_b200.modelinput) and the first
    Save_Frame block verbatim (for the test of the Save_Frame writer).

Run from the repository root with the reference's checkout given in REFERENCE_ROOT:
    python tests/golden/make_run07008_newton.py
(after tests/golden/make_run07008_growth.py, whose fixture supplies the growth parameters).
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from tissueorigami_b200 import mesh  # noqa: E402

REF = os.environ.get("REFERENCE_ROOT", "")
INP = os.path.join(REF, "tests", "sim_no_pardiso_reg", "run07008")
OUT = os.path.join(REF, "tests", "sim_pardiso_reg", "run07008", "expected_out")


def _frames(path):
    lines = open(path).read().splitlines()
    out, i = [], 0
    while i < len(lines):
        if lines[i].startswith("=============== TIME:"):
            t = float(lines[i].split(":")[1].split("=")[0])
            n = int(lines[i + 1])
            pos = np.array([[float(v) for v in lines[i + 2 + k].split()[:3]] for k in range(n)])
            out.append((t, pos))
            i += 2 + n
        else:
            i += 1
    return out


def _du_traces(path):
    """||dU|| of every Newton iteration, one list per time step, from the run's log."""
    traces, cur = [], []
    for line in open(path, errors="replace"):
        m = re.search(r"not\s+yet converged via du: norm\s*([0-9.eE+-]+)", line)
        if m:
            cur.append(float(m.group(1)))
            continue
        m = re.search(r"converged with displacement: norm\s*([0-9.eE+-]+)", line)
        if m:
            cur.append(float(m.group(1)))
            traces.append(cur)
            cur = []
    return traces


def main():
    if not REF:
        raise SystemExit("set REFERENCE_ROOT to the reference checkout")
    x, place, ttype, circ, conn, xref = mesh.read_mesh(os.path.join(INP, "smallWingDisc.mesh"))
    N, E = x.shape[0], conn.shape[0]
    pp = np.fromfile(os.path.join(OUT, "Save_PhysicalProp"), dtype="<f8").reshape(-1, 3 * E + 3 * N)
    elem = pp[0, :3 * E].reshape(E, 3)
    ext_visc = pp[0, 3 * E:].reshape(N, 3)
    types = np.fromfile(os.path.join(OUT, "Save_SpecificElementAndNodeTypes"), dtype="<i4")
    n_actin = int(types[0])
    n_ecm = int(types[1 + n_actin])
    ecm = np.zeros(E, bool)
    ecm[types[2 + n_actin:2 + n_actin + n_ecm]] = True
    tok = open(os.path.join(OUT, "Save_NodeBinding")).read().split()
    nb = int(tok[0])
    pairs = [tuple(map(int, tok[1 + 2 * k:3 + 2 * k])) for k in range(nb)]
    fixed = np.zeros((N, 3), np.uint8)
    fixed[np.abs(x[:, 1]) < 0.1, 1] = 1
    # restore the bindings whose master is node 0 (left out of the file by its writer): x and y of
    # the nodes above node 0, except where the master is fixed - then the reference fixes the
    # slave instead of binding it (bindCircumferenceXY, Simulation.cpp:1382-1396)
    col0 = [k for k in range(N) if k != 0 and np.allclose(x[k, :2], x[0, :2])]
    for k in col0:
        for d in (0, 1):
            if fixed[0, d]:
                fixed[k, d] = 1
            else:
                pairs.append((3 * k + d, d))
    pairs = np.array(sorted(pairs), np.int32)
    exposed = np.zeros(E, np.uint8)
    for e in range(E):
        if (place[conn[e, :3]] == 0).all():
            exposed[e] |= 2
        if (place[conn[e, 3:]] == 1).all():
            exposed[e] |= 1
    g = np.load(os.path.join(HERE, "run07008_growth.npz"))
    frames = _frames(os.path.join(OUT, "Save_Frame"))
    assert frames[0][0] == 3600.0
    trace = _du_traces(os.path.join(OUT, "tmp"))[0]
    out = os.path.join(HERE, "run07008_newton_step1.npz")
    # the model input itself, as whitespace-separated tokens, for the model-input loader's test
    tokens = np.array(open(os.path.join(INP, "modelinput07008")).read().split())
    # the first Save_Frame block verbatim, to check that this library writes the same format
    lines = open(os.path.join(OUT, "Save_Frame")).read().splitlines(keepends=True)
    end = next(i for i, l in enumerate(lines) if l.startswith("=============== END OF TIME:"))
    frame_text = "".join(lines[:end + 1])
    np.savez_compressed(out, x=x, place=place, ttype=ttype, circ=circ, conn=conn, xref=xref, young=elem[:, 0], eta=elem[:, 1],
                        modelinput_tokens=tokens, frame_text=np.array(frame_text),
                        ecm=ecm, ext_visc=ext_visc, pairs=pairs, fixed=fixed, exposed=exposed, grown=g["grown"],
                        rates=g["rates"], angle=g["angle"], dt=g["dt"], x_step1=frames[0][1], du_trace=np.array(trace))
    print(f"wrote {out}: {N} nodes, {E} prisms, {len(pairs)} binding pairs ({len(col0)} restored), "
          f"{int(ecm.sum())} ECM prisms, step-1 trace {trace}")


if __name__ == "__main__":
    main()
