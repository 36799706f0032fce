"""Load the reference's model inputs (``modelinput`` file + ``.mesh``) for the Newton step.

TissueFolding runs are configured by a ``modelinput`` text file (ModelInputObject.cpp) that
names a ``.mesh`` file and sets boundary conditions, material, drag and growth. This module
reads such a file and applies the reference's set-up rules for the options this path computes,
so the reference's own inputs run unchanged:

* node placement, tissue type and circumference flags from the mesh (Simulation.cpp:2286-2447);
  element placement from its nodes (ShapeBase::setTissuePlacement, ShapeBase.cpp:900-985);
* y-symmetry: nodes with |y| < 0.1 fixed in y and, unless at an x tip, no longer at the
  circumference (Simulation.cpp:3083-3125, 9557-9567);
* surface and circumference fixing (Simulation::checkForNodeFixing, Simulation.cpp:3667-3760),
  hard fixing only;
* explicit ECM (basal columnar elements, Simulation.cpp:8866-8900) with the ECM Young's modulus
  and Poisson's ratio 0; the non-ECM elements touching it take the basal modulus
  (Simulation.cpp:8931-8965); explicit actin (apical elements, Simulation.cpp:9010-9030), which
  do not grow (ShapeBase.cpp:482-489);
* Young's modulus by placement (Prism::setElasticProperties, Prism.cpp:464-510), Lame parameters
  lambda = E v / (1 + v) / (1 - 2 v), mu = E / 2 / (1 + v); internal viscosity by placement
  (ShapeBase::setViscosity, ShapeBase.cpp:1089-1101);
* external viscosity per node (Node::setExternalViscosity, Node.cpp:63-110), then the fixes the
  reference adds in a direction where no node has drag (checkForZeroExternalViscosity,
  Simulation.cpp:4126-4237, with the tips of assignTips, Simulation.cpp:8165-8182);
* circumference x, y binding to the basal node of each column, with a fixed master fixing its
  slaves instead (Simulation::bindCircumferenceXY, Simulation.cpp:1344-1436);
* exposed surfaces by element placement (Prism::assignExposedSurfaceAreaIndices,
  Prism.cpp:1650-1690);
* uniform growth functions (type 1): window [InitialTime, FinalTime), rates per second and the
  angle in radians as the reference holds them - read into single-precision floats
  (ModelInputObject.cpp:419-501) - on columnar elements (ECM only if asked, never actin).

Options outside this path raise ``NotImplementedError`` (other mesh modes, x / z symmetry,
peripodial membrane and linker zone, fixing by high external viscosity, notum fixing, ellipse
binding, noise on physical properties, non-uniform growth). Options that change the tissue
between steps without entering the Newton step's inputs - explicit-ECM remodelling, adhesion,
node collapse - are reported in ``ReferenceSetup.not_modelled``: runs that use them agree with
the reference for the first step only.
"""
from __future__ import annotations

import dataclasses
import os
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .mesh import Tissue, read_mesh

APICAL, BASAL, MID, LATERAL, APICAL_BULK = 1, 0, 2, 3, 4


def parse(text: str) -> List[Tuple[str, List[str]]]:
    """The file as (key, values) entries in order: a token ending in ':' starts a key, the
    tokens up to the next key are its values (section headers have none)."""
    out: List[Tuple[str, List[str]]] = []
    for tok in text.split():
        if tok.endswith(":"):
            out.append((tok[:-1], []))
        elif out:
            out[-1][1].append(tok)
    return out


class _Entries:
    def __init__(self, entries: Sequence[Tuple[str, List[str]]]):
        self.entries = list(entries)

    def get(self, key: str, default=None, index: int = 0):
        hits = [v for k, v in self.entries if k == key]
        if len(hits) <= index:
            return default
        return hits[index]

    def num(self, key: str, default=None, n: int = 1, index: int = 0):
        v = self.get(key, None, index)
        if v is None:
            return default
        vals = [float(t) for t in v[:n]]
        return vals[0] if n == 1 else vals

    def flag(self, key: str, default=False, index: int = 0) -> bool:
        v = self.get(key, None, index)
        return default if v is None else bool(int(float(v[0])))

    def flags3(self, key: str) -> Tuple[List[bool], bool]:
        """'Key(bool-x,y,z): a b c  <ExtVisc key>: e' -> ([a, b, c], e)."""
        v = self.get(key, None)
        if v is None:
            return [False] * 3, False
        return [bool(int(float(t))) for t in v[:3]], False


@dataclasses.dataclass
class UniformGrowth:
    t0: float
    t1: float
    rates: np.ndarray    # [E,3] 1/s (zero on elements it does not apply to)
    angles: np.ndarray   # [E] radians


@dataclasses.dataclass
class ReferenceSetup:
    tissue: Tissue
    growth: List[UniformGrowth]
    element_placement: np.ndarray
    ecm: np.ndarray
    actin: np.ndarray
    not_modelled: List[str]
    zero_viscosity_fixes: List[Tuple[int, int]] = dataclasses.field(default_factory=list)
    grid_growth: List[dict] = dataclasses.field(default_factory=list)
    grid_interpolation: int = 0
    grid_state: Optional[Tuple[np.ndarray, np.ndarray, np.ndarray]] = None  # rel_pos, rel_z, eflags

    def growth_at(self, t: float) -> Tuple[np.ndarray, np.ndarray]:
        """Per-element growth rates and angles applied by the step that starts at time t."""
        E = self.tissue.n_elems
        rates, angles = np.zeros((E, 3)), np.zeros(E)
        busy = np.zeros(E, bool)
        for g in self.growth:
            if g.t0 <= t < g.t1:
                on = np.any(g.rates != 0, axis=1)
                if np.any(busy & on):
                    raise NotImplementedError("two growth functions active on one element in the same step")
                rates[on], angles[on] = g.rates[on], g.angles[on]
                busy |= on
        return rates, angles

    def simulate(self, n_steps: Optional[int] = None, solver=None, **params):
        """Run n steps (default: the input's SimulationLength / TimeStep) through the library.
        Returns (positions after every step, per-step stats)."""
        from .newton import NewtonRaphsonSolver

        t = self.tissue
        own = solver is None
        s = solver or NewtonRaphsonSolver.from_tissue(t, **params)
        try:
            if self.grid_growth:
                s.set_grid_growth(self.grid_growth, self.grid_interpolation, *self.grid_state)
            s.set_time(0.0)
            x = np.array(t.x, dtype=np.float64, copy=True)
            xs, stats = [], []
            for k in range(n_steps if n_steps is not None else t.n_steps):
                rates, angles = self.growth_at(k * t.dt)
                fg, _ = s.get_growth()
                s.set_growth(fg, rates, angles, t.exposed, t.peripodial)
                x, rc, st = s.runOneStep(x, t.dt)
                st["rc"] = rc
                xs.append(x.copy())
                stats.append(st)
            return xs, stats
        finally:
            if own:
                s.close()


def _element_placement(conn, node_place):
    E = conn.shape[0]
    place = np.full(E, MID, np.int32)
    spans = np.zeros(E, bool)
    for e in range(E):
        p = node_place[conn[e]]
        if (p == LATERAL).any():
            place[e] = LATERAL
        elif (p == APICAL).any():
            if (p == BASAL).any():
                place[e], spans[e] = MID, True
            else:
                place[e] = APICAL
        elif (p == BASAL).any():
            place[e] = BASAL
        elif (p == APICAL_BULK).any():
            place[e] = APICAL_BULK
    return place, spans


def assign_tips(node_place, node_type, x) -> Tuple[int, int]:
    """Simulation::assignTips (Simulation.cpp:8165-8182): the dorsal / ventral tips are the basal
    columnar nodes of smallest / largest x (the first such node on ties); 0 and 1 when there are
    none (the Simulation constructor's values, Simulation.cpp:132-133). Returns (dorsal, ventral)."""
    dorsal, ventral = 0, 1
    lo, hi = 10000.0, -10000.0
    for i in np.nonzero((node_place == BASAL) & (node_type == 0))[0]:
        if x[i, 0] < lo:
            dorsal, lo = int(i), x[i, 0]
        if x[i, 0] > hi:
            ventral, hi = int(i), x[i, 0]
    return dorsal, ventral


def fix_zero_external_viscosity(fixed, ext_visc, node_place, node_type, x, fixes, symmetric_y: bool):
    """Simulation::checkForZeroExternalViscosity (Simulation.cpp:4126-4237), in place on fixed[N,3].

    A direction in which no node feels external drag leaves the tissue free to translate (and
    rotate) rigidly, so the Newton system is singular unless something else fixes it. Unless the
    apical, basal or linker-apical circumference fixing (CircumferentialNodeFix[0..2]; the
    whole-circumference option [4] is not consulted) or the apical / basal surface fixing already
    fixes that direction, the reference fixes the ventral tip in it, the dorsal tip in y and z,
    and a third node (node 1, else 2, else 3) in z; with y-symmetry the ventral tip in x (if
    needed) and y, both tips in z. Returns the (node, dim) fixes it applied."""
    zero = [not (ext_visc[:, d] > 0).any() for d in range(3)]
    applied = []
    if not any(zero):
        return applied
    circ = [fixes["ApicCircumFix(bool-x,y,z)"], fixes["BasalCircumFix(bool-x,y,z)"],
            fixes["LinkerApicCircumFix(bool-x,y,z)"]]
    apical, basal = fixes["ApicSurfaceFix(bool-x,y,z)"], fixes["BasalSurfaceFix(bool-x,y,z)"]
    sufficient = [(not zero[d]) or any(c[d] for c in circ) or basal[d] or apical[d] for d in range(3)]
    dorsal, ventral = assign_tips(node_place, node_type, x)

    def fix(n, d):
        fixed[n, d] = 1
        applied.append((int(n), d))

    if not symmetric_y:
        for d in range(3):
            if not sufficient[d]:
                fix(ventral, d)
        if not sufficient[1]:
            fix(dorsal, 1)
        if not sufficient[2]:
            fix(dorsal, 2)
            for third in (1, 2, 3):
                if dorsal != third and ventral != third:
                    fix(third, 2)
                    break
    else:
        if not sufficient[0]:
            fix(ventral, 0)
        fix(ventral, 1)
        if not sufficient[2]:
            fix(ventral, 2)
            fix(dorsal, 2)
    return applied


def growth_blocks(entries: Sequence[Tuple[str, List[str]]]) -> List[Tuple[int, List[Tuple[str, List[str]]]]]:
    """The growth functions of a model input in their order (ModelInputObject::readGrowthOptions):
    (type, entries up to the next function or section) for every GrowthFunctionType entry."""
    out: List[Tuple[int, List[Tuple[str, List[str]]]]] = []
    for k, v in entries:
        if k == "GrowthFunctionType(int-seeDocumentation)":
            out.append((int(float(v[0])), []))
        elif out and v:
            out[-1][1].append((k, v))
        elif out and not v:  # a section header ends the growth options
            break
    return out


def read_growth_grid(text: str):
    """A grid growth file as ModelInputObject::readGrowthType3 (ModelInputObject.cpp:782-833) reads
    it: nGridX nGridY, then the rates of every grid point (row j from nGridY-1 down to 0, i from 0,
    three axes) read into float, then the angles in degrees in the same order read into double;
    the rates are held per second (per-hour value x 1/3600). Returns (rates[nx, ny, 3], angles[nx, ny])."""
    tok = text.split()
    nx, ny = int(tok[0]), int(tok[1])
    pos = 2
    rates = np.zeros((nx, ny, 3))
    for j in range(ny - 1, -1, -1):
        for i in range(nx):
            for k in range(3):
                rates[i, j, k] = float(np.float32(tok[pos]))
                pos += 1
    angles = np.zeros((nx, ny))
    for j in range(ny - 1, -1, -1):
        for i in range(nx):
            angles[i, j] = float(tok[pos])
            pos += 1
    return rates * (1.0 / 3600.0), angles


def grid_element_state(x, conn, node_place, node_type, place, spans, ecm, actin):
    """Per-element inputs of the grid growth functions on the initial mesh:

    * rel_pos [E,2]: the element centre (mean of its six nodes, ShapeBase::getCentre) relative to the
      x, y bounding box of the nodes not owned by ECM elements only (calculateBoundingBox,
      Simulation.cpp:8388-8425; calculateRelativePosInBoundingBox, ShapeBase.cpp:2091-2095), with
      the apical element's value copied down its column as updateRelativePositionsToApicalPositioning
      does (Simulation.cpp:6147-6167: the column list runs basal to apical and the copy covers its
      first L-2 entries);
    * rel_z [E]: initialRelativePositionInZ = 1 - (centre z - minimum node z) / tissue height,
      clipped to [0, 1] (ShapeBase::setInitialZPosition, ShapeBase.cpp:813-828), the height summed
      along the first basal columnar node's column (calculateTissueHeight, Simulation.cpp:3275-3330);
    * eflags [E]: bit0 ECM-mimicking, bit1 actin-mimicking, bit2 basal placement; tissue type 0."""
    x = np.asarray(x, np.float64)
    conn = np.asarray(conn)
    E = conn.shape[0]
    cen = np.zeros((E, 3))
    for a in range(6):  # summed in node order, then divided, as getCentre does
        cen += x[conn[:, a]]
    cen /= 6
    owned = np.zeros(x.shape[0], bool)
    owned[conn[~ecm].ravel()] = True
    keep = owned if ecm.any() else np.ones(x.shape[0], bool)
    lo = x[keep, :2].min(axis=0)
    size = x[keep, :2].max(axis=0) - lo
    rel = np.zeros((E, 2))
    rel[:, 0] = (cen[:, 0] - lo[0]) / size[0]
    rel[:, 1] = (cen[:, 1] - lo[1]) / size[1]
    # columns: the element above e is the one whose basal nodes are e's apical nodes
    by_basal = {tuple(sorted(c[:3])): e for e, c in enumerate(conn)}
    height, layers = 0.0, 0
    first = next((n for n in range(x.shape[0]) if node_place[n] == BASAL and node_type[n] == 0), None)
    if first is not None:
        cur = first
        while node_place[cur] != APICAL:
            owner = next((e for e in range(E) if cur in conn[e, :3]), None)
            if owner is None:
                break
            height += float(np.linalg.norm(x[conn[owner, 0]] - x[conn[owner, 3]]))
            layers += 1
            cur = int(conn[owner, 3 + list(conn[owner, :3]).index(cur)])
    for e in range(E):
        if place[e] != APICAL:
            continue
        stack = [e]
        while True:  # walk down to the basal element of the column
            below = next((b for b, c in enumerate(conn) if tuple(sorted(c[3:])) == tuple(sorted(conn[stack[-1], :3]))), None)
            if below is None:
                break
            stack.append(below)
        stack = stack[::-1]  # basal first, as elementsIdsOnSameColumn
        for b in stack[:max(layers - 2, 0)]:
            rel[b] = rel[e]
    del by_basal
    zmin = x[:, 2].min()
    rel_z = np.clip(1.0 - (cen[:, 2] - zmin) / height, 0.0, 1.0) if height > 0 else np.zeros(E)
    eflags = ecm.astype(np.int32) | (actin.astype(np.int32) << 1) | ((np.asarray(place) == BASAL).astype(np.int32) << 2)
    return rel, rel_z, eflags


def setup(entries: Sequence[Tuple[str, List[str]]], mesh_arrays, grid_files=None) -> ReferenceSetup:
    """Apply the reference's set-up rules to parsed ``modelinput`` entries and ``read_mesh`` arrays.
    grid_files: the text of every grid growth file, keyed by its Filename entry."""
    m = _Entries(entries)
    x, node_place, node_type, circ, conn, xref = mesh_arrays
    x = np.asarray(x, np.float64)
    node_place = np.asarray(node_place, np.int32)
    circ = np.asarray(circ, np.int32).astype(bool).copy()
    conn = np.asarray(conn, np.int32)
    N, E = x.shape[0], conn.shape[0]
    unsupported = []

    mode = int(m.num("MeshInputMode(int-seeDocumentation)", 4))
    if mode != 4:
        unsupported.append(f"MeshInputMode {mode} (only 4, a .mesh file)")
    if m.flag("symmetricInX(bool)") or m.flag("symmetricInZ(bool)"):
        unsupported.append("x or z symmetry")
    if (np.asarray(node_type) != 0).any():
        unsupported.append("peripodial membrane / linker zone nodes")
    noise = [m.num("Noise(%-int)", 0, index=i) for i in range(3)]
    if any(v not in (None, 0, 0.0) for v in noise):
        unsupported.append("noise on physical properties")
    fix_keys = {"ApicSurfaceFix(bool-x,y,z)": "FixApicalExtVisc(bool)",
                "BasalSurfaceFix(bool-x,y,z)": "FixBasalExtVisc(bool)",
                "CircumferenceFix(bool-x,y,z)": "FixCircWithExtVisc(bool)",
                "ApicCircumFix(bool-x,y,z)": "FixApicCircWithExtVisc(bool)",
                "BasalCircumFix(bool-x,y,z)": "FixBasalCircWithExtVisc(bool)",
                "LinkerApicCircumFix(bool-x,y,z)": "FixLinkerApicCircWithExtVisc(bool)",
                "LinkerBasalCircumFix(bool-x,y,z)": "FixLinkerBasalCircWithExtVisc(bool)",
                "NotumFix(bool-x,y,z,double-xFracMin,xFracMax)": "FixNotumExtVisc(bool)"}
    fixes = {k: m.flags3(k)[0] for k in fix_keys}
    for k, visc_key in fix_keys.items():
        if any(fixes[k]) and m.flag(visc_key):
            unsupported.append(f"{k} by high external viscosity")
    for k in ("LinkerApicCircumFix(bool-x,y,z)", "LinkerBasalCircumFix(bool-x,y,z)",
              "NotumFix(bool-x,y,z,double-xFracMin,xFracMax)"):
        if any(fixes[k]):
            unsupported.append(k)
    ell = m.get("bindEllipses(bool,nFunctions)")
    if ell and int(float(ell[0])):
        unsupported.append("ellipse binding")
    blocks = growth_blocks(entries)
    types = [b[0] for b in blocks]
    if any(t not in (1, 3) for t in types):
        unsupported.append(f"growth function types {sorted(set(t for t in types if t not in (1, 3)))} "
                           "(only uniform, 1, and grid-based, 3)")
    if 3 in types:
        if not m.flag("GridGrowthsPinnedOnInitialMesh(bool)"):
            unsupported.append("grid growth read on the current mesh (GridGrowthsPinnedOnInitialMesh 0)")
        pins = m.get("PinningUpdateTimes(number-times(sec))", ["0"])
        if any(float(v) > 0 for v in pins[1:1 + int(float(pins[0]))]):
            unsupported.append("grid growth re-pinned during the run (PinningUpdateTimes after 0)")
        if 1 in types[types.index(3):]:
            unsupported.append("a uniform growth function listed after a grid-based one")
    if m.num("noTimeseriesInputs(size_t)", 0):
        unsupported.append("Young's modulus time series")
    if m.flag("AddLateralECM(bool)"):
        unsupported.append("lateral ECM")
    if unsupported:
        raise NotImplementedError("model input options outside this path: " + "; ".join(unsupported))

    # boundary: y-symmetry, then surface / circumference fixing
    fixed = np.zeros((N, 3), np.uint8)
    if m.flag("symmetricInY(bool)"):
        on_line = np.abs(x[:, 1]) < 0.1
        xmax, xmin = x[:, 0].max(), x[:, 0].min()
        tip = (np.abs(x[:, 0] - xmax) < 0.1) | (np.abs(x[:, 0] - xmin) < 0.1)
        circ &= ~(on_line & ~tip)
        fixed[on_line, 1] = 1
    circ_opts = [("ApicCircumFix(bool-x,y,z)", node_place == APICAL), ("BasalCircumFix(bool-x,y,z)", node_place == BASAL),
                 ("CircumferenceFix(bool-x,y,z)", np.ones(N, bool))]
    for key, sel in circ_opts:
        for d in range(3):
            if fixes[key][d]:
                fixed[circ & sel, d] = 1
    for key, sel in (("BasalSurfaceFix(bool-x,y,z)", node_place == BASAL), ("ApicSurfaceFix(bool-x,y,z)", node_place == APICAL)):
        for d in range(3):
            if fixes[key][d]:
                fixed[sel, d] = 1

    # elements: placement, explicit ECM / actin, material
    place, spans = _element_placement(conn, node_place)
    explicit_ecm = m.flag("ThereIsExplicitECM(bool)")
    explicit_actin = m.flag("ThereIsExplicitActin(bool)")
    ecm = np.zeros(E, bool)
    if explicit_ecm:
        ecm = (place == BASAL) | ((place == MID) & spans)
    actin = np.zeros(E, bool)
    if explicit_actin:
        actin = (place == APICAL) | (place == APICAL_BULK) | ((place == MID) & spans)
    border = np.zeros(E, bool)
    if explicit_ecm and ecm.any():
        ecm_nodes = np.zeros(N, bool)
        ecm_nodes[conn[ecm].ravel()] = True
        border = ~ecm & ecm_nodes[conn].any(axis=1)
    e_ap = m.num("YoungsModulusApical")
    e_ba = m.num("YoungsModulusBasal")
    e_mid = m.num("YoungsModulusMid")
    e_ecm = m.num("ECMColumnarYoungsModulus", 0.0) if explicit_ecm else 0.0
    young = np.full(E, e_mid)
    young[(place == APICAL) | (place == APICAL_BULK)] = e_ap
    young[(place == BASAL) | border] = e_ba  # checked before apical in the reference
    young[ecm] = e_ecm
    nu = np.full(E, min(max(m.num("PoissonsRatio"), 0.0), 0.5))
    nu[ecm] = 0.0
    lam = young * nu / (1 + nu) / (1 - 2.0 * nu)
    mu = young / 2.0 / (1 + nu)
    eta = np.full(E, m.num("MidLineViscosity", 0.0))
    eta[place == BASAL] = m.num("BasalViscosity", 0.0)
    eta[place == APICAL] = m.num("ApicalViscosity", 0.0)

    # external viscosity per node
    v_ap = m.num("DiscProperApicalExternalViscosity", 0.0)
    v_ba = m.num("DiscProperBasalExternalViscosity", 0.0)
    extend = m.flag("ExtendToWholeTissue")
    ev = np.zeros(N)
    ev[node_place == BASAL] = v_ba
    ev[node_place == APICAL] = v_ap
    rest = (node_place != BASAL) & (node_place != APICAL)
    ev[rest & circ] = min(v_ap, v_ba)
    if extend:
        ev[rest & ~circ & np.isin(node_place, [MID, LATERAL, APICAL_BULK])] = min(v_ap, v_ba)
    ext_visc = np.repeat(ev[:, None], 3, axis=1)
    zero_visc_fixes = fix_zero_external_viscosity(fixed, ext_visc, node_place, np.asarray(node_type), x, fixes,
                                                  m.flag("symmetricInY(bool)"))

    # circumference binding: x, y of every node above a basal circumference node to that node
    pairs = []
    if m.flag("bindCircumferenceXYToBasal(bool)"):
        above = {}
        for e in range(E):
            for a in range(3):
                above.setdefault(int(conn[e, a]), int(conn[e, a + 3]))
        for master in np.nonzero((node_place == BASAL) & circ)[0]:
            cur, hops = int(master), 0
            while hops < 10:
                hops += 1
                if cur not in above:
                    break
                slave = above[cur]
                for d in (0, 1):
                    if fixed[master, d]:
                        fixed[slave, d] = 1
                    if not fixed[slave, d]:
                        pairs.append((3 * slave + d, 3 * int(master) + d))
                cur = slave
                if node_place[cur] == APICAL:
                    break
    slave_master = np.array(sorted(pairs), np.int32).reshape(-1, 2)

    exposed = np.zeros(E, np.uint8)
    exposed[(place == APICAL) | ((place == MID) & spans)] |= 1
    exposed[(place == BASAL) | ((place == MID) & spans)] |= 2

    # growth: uniform functions, parameters held in single precision as the reference reads them
    # (resolved per element here); grid-based functions as the reference holds them, evaluated on
    # the device every step from the elements' pinned positions
    growth, grid = [], []
    for gtype, g in blocks:
        gm = _Entries(g)
        t0 = float(np.float32(gm.num("InitialTime(sec)")))
        t1 = float(np.float32(gm.num("FinalTime(sec)")))
        if gtype == 3:
            name = gm.get("Filename(full-path)")[0]
            if grid_files is None or name not in grid_files:
                raise ValueError(f"grid growth file {name} not given")
            rates_g, angles_g = read_growth_grid(grid_files[name])
            zr = gm.num("zRange", n=2)
            flags = (int(gm.flag("ApplyToColumnarLayer(bool)")) | int(gm.flag("ApplyToPeripodialMembrane(bool)")) << 1
                     | int(gm.flag("ApplyToBasalECM(bool)")) << 2 | int(gm.flag("ApplyToLateralECM(bool)")) << 3)
            grid.append({"t0": t0, "t1": t1, "rates": rates_g, "angles_deg": angles_g, "zmin": zr[0], "zmax": zr[1],
                         "flags": flags, "nx": rates_g.shape[0], "ny": rates_g.shape[1], "file": name})
            continue
        col = gm.flag("ApplyToColumnarLayer(bool)")
        basal_ecm = gm.flag("ApplyToBasalECM(bool)")
        per_hour = gm.num("MaxValue(fractionPerHour-DV,AP,AB)", n=3)
        rate = [float(np.float32(np.float32(v) * (1.0 / 3600.0))) for v in per_hour]
        angle = float(np.float32(np.float32(gm.num("Angle(degrees)")) * (np.pi / 180.0)))
        on = np.zeros(E, bool)
        if col:
            on |= ~ecm if explicit_ecm else np.ones(E, bool)
        if basal_ecm:
            on |= ecm & (place == BASAL)
        on &= ~actin
        rates = np.zeros((E, 3))
        rates[on] = rate
        growth.append(UniformGrowth(t0, t1, rates, np.full(E, angle)))
    grid_state = None
    if grid:
        grid_state = grid_element_state(x, conn, node_place, np.asarray(node_type), place, spans, ecm if explicit_ecm else
                                        np.zeros(E, bool), actin)

    dt = m.num("TimeStep(sec)")
    length = m.num("SimulationLength(sec)", dt)
    not_modelled = []
    if explicit_ecm:
        not_modelled.append("explicit-ECM remodelling")
    if m.flag("ThereIsAdhesion(bool)"):
        not_modelled.append("adhesion")
    if m.flag("ThereIsNodeCollapse(bool)"):
        not_modelled.append("node collapse")
    tissue = Tissue("modelinput", conn, np.asarray(xref, np.float64), x, lam, mu, eta, fixed, ext_visc, exposed,
                    np.zeros(E, np.uint8), np.zeros((E, 3)), np.zeros(E), node_place, circ.astype(np.int32),
                    slave_master=slave_master, dt=float(dt), n_steps=int(round(length / dt)), newton_tol=1e-8)
    interp = int(m.num("GridGrowthsInterpolationType(0=step,1=linear)", 0))
    return ReferenceSetup(tissue, growth, place, ecm, actin, not_modelled, zero_visc_fixes, grid, interp, grid_state)


def load(modelinput_path: str, mesh_path: Optional[str] = None) -> ReferenceSetup:
    """Read a ``modelinput`` file and its mesh (``MeshFile``, relative to the input file's folder
    unless ``mesh_path`` is given)."""
    text = open(modelinput_path).read()
    entries = parse(text)
    if mesh_path is None:
        name = _Entries(entries).get("MeshFile(full-path)", [None])[0]
        if name is None:
            raise ValueError("no MeshFile in the model input")
        mesh_path = name if os.path.isabs(name) else os.path.join(os.path.dirname(os.path.abspath(modelinput_path)), name)
    folder = os.path.dirname(os.path.abspath(modelinput_path))
    grid_files = {}
    for gtype, g in growth_blocks(entries):
        if gtype == 3:
            name = _Entries(g).get("Filename(full-path)")[0]
            with open(name if os.path.isabs(name) else os.path.join(folder, name)) as fh:
                grid_files[name] = fh.read()
    return setup(entries, read_mesh(mesh_path), grid_files)
