"""Build tests/golden/run07008_growth.npz from the reference's no-Pardiso regression run 07008.

That run (tests/sim_no_pardiso_reg/run07008 in the reference: smallWingDisc.mesh, modelinput07008)
grows a wing-disc mesh for 10 steps of 3600 s without solving the mechanics, so node positions
never move and every element's growth tensor is pure bookkeeping: Fg after step k is the uniform
growth increment R diag(exp(r dt)) R^T composed k times (steps with t < FinalTime). Its
expected_out/Save_Growth holds Fg (row-major, 9 doubles) of every element after every step.

The fixture keeps the mesh (node positions, connectivity, reference shapes), the growth
parameters exactly as the reference holds them (rates and angle are read into single-precision
floats and scaled in place), the elements that grow (those whose Fg leaves the identity in the
golden file) and the golden Fg of every element after every step.

Run from the repository root with the reference's checkout given:
    REFERENCE_ROOT=<path to the reference> python tests/golden/make_run07008_growth.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from tissueorigami_b200 import mesh  # noqa: E402

REF = os.environ.get("REFERENCE_ROOT", "")
RUN = os.path.join(REF, "tests", "sim_no_pardiso_reg", "run07008")


def _growth_block(path):
    tok = open(path).read().split()
    def after(key):
        return tok.index(key) + 1
    dt = float(tok[after("TimeStep(sec):")])
    length = float(tok[after("SimulationLength(sec):")])
    assert tok[after("GrowthFunctionType(int-seeDocumentation):")] == "1", "uniform growth expected"
    t0 = float(tok[after("InitialTime(sec):")])
    t1 = float(tok[after("FinalTime(sec):")])
    i = after("MaxValue(fractionPerHour-DV,AP,AB):")
    per_hour = [float(v) for v in tok[i:i + 3]]
    angle_deg = float(tok[after("Angle(degrees):")])
    # ModelInputObject reads these into float variables and scales them in place
    rates = [float(np.float32(np.float32(v) * (1.0 / 3600.0))) for v in per_hour]
    angle = float(np.float32(np.float32(angle_deg) * (np.pi / 180.0)))
    return dt, length, t0, t1, rates, angle


def main():
    if not REF:
        raise SystemExit("set REFERENCE_ROOT to the reference checkout")
    x, place, ttype, circ, conn, xref = mesh.read_mesh(os.path.join(RUN, "smallWingDisc.mesh"))
    dt, length, t0, t1, rates, angle = _growth_block(os.path.join(RUN, "modelinput07008"))
    E = conn.shape[0]
    fg = np.fromfile(os.path.join(RUN, "expected_out", "Save_Growth"), dtype="<f8")
    assert fg.size % (9 * E) == 0
    frames = fg.reshape(-1, E, 9)
    grown = np.any(np.abs(frames - np.eye(3).reshape(1, 1, 9)).max(axis=2) > 0, axis=0)
    out = os.path.join(HERE, "run07008_growth.npz")
    np.savez_compressed(out, x=x, place=place, circ=circ, conn=conn, xref=xref, dt=dt, t0=t0, t1=t1,
                        rates=np.array(rates), angle=angle, grown=grown, frames=frames)
    print(f"wrote {out}: {E} elements, {int(grown.sum())} growing, {frames.shape[0]} saved steps")


if __name__ == "__main__":
    main()
