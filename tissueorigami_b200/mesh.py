"""Synthetic prism tissues and the reference's ``.mesh`` text format.

The reference builds its tissue from a ``.mesh`` file (``Simulation::initiateNodesFromMeshInput``
and ``initiatePrismFromMeshInput``, TissueFolding/SourceCode/Simulation.cpp:2286-2305, 2431-2447)
and then derives, per node and element, the placement flags, the external drag coefficients and
the fixed degrees of freedom during ``initiateSystem`` (Simulation.cpp:566-846). This module
produces the same per-node / per-element arrays directly, for the seeded synthetic workloads:

* ``small_rectangle``  - 20x10-node grid, 2 um spacing, one 10 um layer (342 prisms)
* ``wing_disc``        - Delaunay disc of radius 100 um, 2 um ECM layer under a 25 um columnar
                         layer (~80k prisms), radial Gaussian growth, rim clamped
* ``large_slab``       - 1000x500 nodes at 0.5 um, 3 layers (~3M prisms), log-normal stiffness,
                         anisotropic growth with a smooth random orientation field
* ``batch_tissues``    - many independent discs / rectangles of uneven size

All arrays are numpy, row-major, in the reference's ordering: node DoF ``3*node+dim``; prism nodes
0-2 basal triangle (counter-clockwise seen from the apical side, Prism.cpp:369-417), 3-5 apical.
Units follow the reference: micrometres, pascals, seconds.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

# Node::tissuePlacement values (Node.h; ShapeBase.cpp:900-984)
BASAL, APICAL, MIDLINE, LATERAL = 0, 1, 2, 3
# element exposure bits used by the viscosity-surface update (Prism.cpp:1650-1709)
EXPOSED_APICAL, EXPOSED_BASAL = 1, 2
# External viscosities of the reference's wing-disc runs (DiscProperApicalExternalViscosity 16000,
# DiscProperBasalExternalViscosity 10 in tests/sim_no_pardiso_reg/run07008/modelinput07008), used
# for the disc, slab and batch tissues whose drag the workload does not state.
WING_DISC_APICAL_VISC, WING_DISC_BASAL_VISC = 16000.0, 10.0


@dataclasses.dataclass
class Tissue:
    """Everything the Newton step reads, in the reference's ordering.

    conn[E,6] int32, xref[E,18] (ReferenceShape->Positions), x[N,3] (Node::Position),
    lam/mu/eta[E] (ShapeBase::lambda, mu, internalViscosity), fixed[N,3] uint8
    (Node::FixedPos), ext_visc[N,3] (Node::externalViscosity), exposed[E] uint8 (bits
    apical=1 / basal=2), peripodial[E] uint8, rates[E,3] growth rates in 1/s and
    angles[E] growth orientation in radians (UniformGrowthFunction semantics),
    slave_master[P,2] int32 DoF couples, fg[E,9] growth deformation gradient.
    """

    name: str
    conn: np.ndarray
    xref: np.ndarray
    x: np.ndarray
    lam: np.ndarray
    mu: np.ndarray
    eta: np.ndarray
    fixed: np.ndarray
    ext_visc: np.ndarray
    exposed: np.ndarray
    peripodial: np.ndarray
    rates: np.ndarray
    angles: np.ndarray
    node_placement: np.ndarray
    at_circumference: np.ndarray
    slave_master: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 2), np.int32))
    fg: Optional[np.ndarray] = None
    dt: float = 60.0
    n_steps: int = 10
    newton_tol: float = 1e-8
    seed: int = 0

    def __post_init__(self):
        if self.fg is None:
            self.fg = np.tile(np.eye(3).reshape(1, 9), (self.n_elems, 1))

    @property
    def n_nodes(self) -> int:
        return int(self.x.shape[0])

    @property
    def n_elems(self) -> int:
        return int(self.conn.shape[0])

    @property
    def size(self) -> float:
        """Tissue size used for position tolerances: the bounding-box diagonal."""
        span = self.x.max(axis=0) - self.x.min(axis=0)
        return float(np.linalg.norm(span))

    def copy(self) -> "Tissue":
        return dataclasses.replace(self, **{f.name: (np.array(getattr(self, f.name), copy=True)
                                                     if isinstance(getattr(self, f.name), np.ndarray)
                                                     else getattr(self, f.name))
                                            for f in dataclasses.fields(self)})


def lame(E: np.ndarray, nu: float):
    """Prism::setElasticProperties (Prism.cpp:464-517): nu clamped to [0, 0.5]."""
    nu = min(max(nu, 0.0), 0.5)
    lam = E * nu / (1 + nu) / (1 - 2.0 * nu)
    mu = E / 2.0 / (1 + nu)
    return lam, mu


def _orient(tri: np.ndarray, pts2: np.ndarray) -> np.ndarray:
    """Make every triangle counter-clockwise seen from +z (the check of Prism.cpp:369-417)."""
    p = pts2[tri]
    cross = (p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1]) - (p[:, 1, 1] - p[:, 0, 1]) * (p[:, 2, 0] - p[:, 0, 0])
    tri = tri.copy()
    neg = cross < 0
    tri[neg, 1], tri[neg, 2] = tri[neg, 2].copy(), tri[neg, 1].copy()
    return tri


def _extrude(pts2: np.ndarray, tri: np.ndarray, z_levels: List[float]):
    """Stack len(z_levels) node surfaces and connect consecutive ones with prisms.

    Nodes are numbered point-major (all surfaces of one in-plane point are consecutive) and
    prisms triangle-major (all layers of one triangle are consecutive), so that nodes and
    elements that touch sit close together in memory.
    """
    P = pts2.shape[0]
    S = len(z_levels)
    L = S - 1
    x = np.zeros((P * S, 3))
    for s, z in enumerate(z_levels):
        x[s::S, 0] = pts2[:, 0]
        x[s::S, 1] = pts2[:, 1]
        x[s::S, 2] = z
    T = tri.shape[0]
    conn = np.zeros((T * L, 6), np.int32)
    layer = np.zeros(T * L, np.int32)
    for l in range(L):
        conn[l::L, 0:3] = tri * S + l
        conn[l::L, 3:6] = tri * S + l + 1
        layer[l::L] = l
    xref = x[conn].reshape(-1, 18).copy()
    return x, conn, xref, layer


def _placement(n_points: int, n_surfaces: int):
    place = np.full(n_points * n_surfaces, MIDLINE, np.int32)
    place[0::n_surfaces] = BASAL
    place[n_surfaces - 1::n_surfaces] = APICAL
    return place


def _element_exposure(layer: np.ndarray, n_layers: int) -> np.ndarray:
    """ShapeBase::setTissuePlacement + Prism::assignExposedSurfaceAreaIndices for a columnar
    stack: a single layer spans the tissue (apical and basal exposed), otherwise the bottom layer
    is basal and the top layer apical."""
    exposed = np.zeros(layer.shape[0], np.uint8)
    exposed[layer == n_layers - 1] |= EXPOSED_APICAL
    exposed[layer == 0] |= EXPOSED_BASAL
    return exposed


def _ext_visc(place: np.ndarray, at_circ: np.ndarray, apical: float, basal: float) -> np.ndarray:
    """Node::setExternalViscosity (Node.cpp:63-110) without the inner-tissue extension."""
    ev = np.zeros((place.shape[0], 3))
    ev[place == BASAL] = basal
    ev[place == APICAL] = apical
    circ_mid = (place != BASAL) & (place != APICAL) & (at_circ != 0)
    ev[circ_mid] = min(apical, basal)
    return ev


def small_rectangle(seed: int = 1000, nx: int = 20, ny: int = 10, spacing: float = 2.0,
                    thickness: float = 10.0, E: float = 1000.0, nu: float = 0.3,
                    ext_visc: float = 10.0, growth: float = 1e-4, dt: float = 60.0,
                    n_steps: int = 10, newton_tol: float = 1e-10) -> Tissue:
    """Small rectangle, one prism layer: 20x10 nodes, 2 um, quads split on one diagonal,
    10 um thick (342 prisms); neo-Hookean E=1000 Pa, nu=0.3; nodal drag 10 Pa s on the apical
    and basal surfaces; uniform in-plane growth 1e-4 /s; basal nodes fixed in z; dt 60 s."""
    gx, gy = np.meshgrid(np.arange(nx) * spacing, np.arange(ny) * spacing, indexing="xy")
    pts2 = np.stack([gx.ravel(), gy.ravel()], axis=1)
    tris = []
    for j in range(ny - 1):
        for i in range(nx - 1):
            a, b, c, d = j * nx + i, j * nx + i + 1, (j + 1) * nx + i + 1, (j + 1) * nx + i
            tris.append((a, b, c))
            tris.append((a, c, d))
    tri = _orient(np.array(tris, np.int64), pts2)
    x, conn, xref, layer = _extrude(pts2, tri, [0.0, thickness])
    place = _placement(pts2.shape[0], 2)
    edge = (np.isclose(pts2[:, 0], 0) | np.isclose(pts2[:, 0], (nx - 1) * spacing)
            | np.isclose(pts2[:, 1], 0) | np.isclose(pts2[:, 1], (ny - 1) * spacing))
    at_circ = np.repeat(edge.astype(np.int32), 2)
    Ee = np.full(conn.shape[0], E)
    lam, mu = lame(Ee, nu)
    fixed = np.zeros((x.shape[0], 3), np.uint8)
    fixed[place == BASAL, 2] = 1
    rates = np.zeros((conn.shape[0], 3))
    rates[:, 0] = growth
    rates[:, 1] = growth
    return Tissue("small_rectangle", conn, xref, x, lam, mu, np.zeros(conn.shape[0]), fixed,
                  _ext_visc(place, at_circ, ext_visc, ext_visc), _element_exposure(layer, 1),
                  np.zeros(conn.shape[0], np.uint8), rates, np.zeros(conn.shape[0]), place,
                  at_circ, dt=dt, n_steps=n_steps, newton_tol=newton_tol, seed=seed)


def _disc_points(rng: np.random.Generator, radius: float, n_target: int, jitter: float = 0.15):
    """Seeded points in a disc: a jittered triangular lattice plus a ring on the rim.
    The lattice keeps the Delaunay triangles well shaped; the jitter is uniform random."""
    h = math.sqrt(2.0 * math.pi * radius * radius / (math.sqrt(3.0) * n_target))
    rows = int(2 * radius / (h * math.sqrt(3) / 2)) + 3
    cols = int(2 * radius / h) + 3
    jj, ii = np.meshgrid(np.arange(rows), np.arange(cols), indexing="ij")
    px = (ii - cols / 2) * h + (jj % 2) * h / 2
    py = (jj - rows / 2) * h * math.sqrt(3) / 2
    pts = np.stack([px.ravel(), py.ravel()], axis=1)
    pts += rng.uniform(-jitter * h, jitter * h, size=pts.shape)
    r = np.linalg.norm(pts, axis=1)
    pts = pts[r < radius - 0.6 * h]
    n_rim = max(12, int(round(2 * math.pi * radius / h)))
    th = np.arange(n_rim) * 2 * math.pi / n_rim
    rim = np.stack([radius * np.cos(th), radius * np.sin(th)], axis=1)
    allp = np.concatenate([pts, rim], axis=0)
    is_rim = np.zeros(allp.shape[0], bool)
    is_rim[pts.shape[0]:] = True
    return allp, is_rim


def _delaunay(pts2: np.ndarray) -> np.ndarray:
    from scipy.spatial import Delaunay

    tri = Delaunay(pts2).simplices.astype(np.int64)
    # spatial order of triangles: sort by a coarse Morton-like key of the centroid so that
    # consecutive prisms share nodes
    c = pts2[tri].mean(axis=1)
    span = np.maximum(c.max(axis=0) - c.min(axis=0), 1e-12)
    q = ((c - c.min(axis=0)) / span * 1023).astype(np.int64)
    key = _morton2(q[:, 0], q[:, 1])
    tri = tri[np.argsort(key, kind="stable")]
    return _orient(tri, pts2)


def _morton2(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    key = np.zeros_like(a)
    for bit in range(11):
        key |= ((a >> bit) & 1) << (2 * bit)
        key |= ((b >> bit) & 1) << (2 * bit + 1)
    return key


def _renumber_points(pts2: np.ndarray, tri: np.ndarray, flags: List[np.ndarray]):
    """Renumber in-plane points in the order triangles first touch them (locality)."""
    order = -np.ones(pts2.shape[0], np.int64)
    seen = np.zeros(pts2.shape[0], bool)
    nxt = 0
    for p in tri.ravel():
        if not seen[p]:
            seen[p] = True
            order[p] = nxt
            nxt += 1
    for p in range(pts2.shape[0]):
        if not seen[p]:
            order[p] = nxt
            nxt += 1
    inv = np.empty_like(order)
    inv[order] = np.arange(order.shape[0])
    return pts2[inv], order[tri], [f[inv] for f in flags]


def wing_disc(seed: int = 1001, radius: float = 100.0, n_surface_points: int = 20000,
              ecm: float = 2.0, columnar: float = 25.0, E_col: float = 1000.0,
              E_ecm: float = 4000.0, nu: float = 0.3, apical_visc: float = WING_DISC_APICAL_VISC,
              basal_visc: float = WING_DISC_BASAL_VISC,
              peak_growth: float = 2e-4, sigma: float = 40.0, noise: float = 0.1,
              dt: float = 60.0, n_steps: int = 50, newton_tol: float = 1e-8) -> Tissue:
    """Wing-disc-like disc: Delaunay-triangulated disc of radius 100 um from seeded points
    (~40k triangles), extruded into a 2 um ECM layer (E=4000 Pa) under a 25 um columnar layer
    (E=1000 Pa), ~80k prisms, nu=0.3; radial Gaussian in-plane growth, peak 2e-4 /s at the
    centre, sigma 40 um, times a uniform-random +-10 % per element; rim clamped; dt 60 s; apical /
    basal external viscosity of the reference's wing-disc runs (16000 / 10 Pa s)."""
    rng = np.random.default_rng(seed)
    pts2, is_rim = _disc_points(rng, radius, n_surface_points)
    tri = _delaunay(pts2)
    pts2, tri, (is_rim,) = _renumber_points(pts2, tri, [is_rim])
    x, conn, xref, layer = _extrude(pts2, tri, [0.0, ecm, ecm + columnar])
    place = _placement(pts2.shape[0], 3)
    at_circ = np.repeat(is_rim.astype(np.int32), 3)
    Ee = np.where(layer == 0, E_ecm, E_col)
    lam, mu = lame(Ee, nu)
    fixed = np.zeros((x.shape[0], 3), np.uint8)
    fixed[at_circ != 0, :] = 1
    cen = xref.reshape(-1, 6, 3).mean(axis=1)
    rho2 = cen[:, 0] ** 2 + cen[:, 1] ** 2
    r = peak_growth * np.exp(-rho2 / (2 * sigma * sigma)) * (1 + rng.uniform(-noise, noise, conn.shape[0]))
    rates = np.zeros((conn.shape[0], 3))
    rates[:, 0] = r
    rates[:, 1] = r
    return Tissue("wing_disc", conn, xref, x, lam, mu, np.zeros(conn.shape[0]), fixed,
                  _ext_visc(place, at_circ, apical_visc, basal_visc), _element_exposure(layer, 2),
                  np.zeros(conn.shape[0], np.uint8), rates, np.zeros(conn.shape[0]), place,
                  at_circ, dt=dt, n_steps=n_steps, newton_tol=newton_tol, seed=seed)


def _smooth_field(rng: np.random.Generator, xy: np.ndarray, length: float, n_feat: int = 64):
    """Seeded smooth random field with an RBF covariance of length scale ``length``, by random
    Fourier features (unit variance)."""
    w = rng.normal(0.0, 1.0 / length, size=(n_feat, 2))
    b = rng.uniform(0, 2 * math.pi, size=n_feat)
    a = rng.normal(0.0, 1.0, size=n_feat)
    return (np.cos(xy @ w.T + b) @ a) * math.sqrt(2.0 / n_feat)


def stacked_sheets(nx: int = 10, ny: int = 6, spacing: float = 2.0, thickness: float = 4.0, gap: float = 0.5,
                   E: float = 1000.0, n_steps: int = 3, **kw) -> Tissue:
    """Two one-layer rectangles (small_rectangle of nx x ny nodes) in one tissue, the second one
    mirrored through the plane between them so that the two apical surfaces face each other
    across `gap`: every apical node of the lower sheet lies `gap` below one of the upper sheet,
    which makes them packing pairs (the reference packs same-placement nodes that share no
    element and are closer than 0.4 x the local average side length). Each sheet's basal nodes
    are fixed in z. The upper sheet's prisms keep the reference's node order (0-2 basal, 3-5
    apical) with nodes 1 and 2 (4 and 5) swapped, so their orientation stays positive."""
    a = small_rectangle(nx=nx, ny=ny, spacing=spacing, thickness=thickness, E=E, n_steps=n_steps, **kw)
    n = a.n_nodes
    perm = [0, 2, 1, 3, 5, 4]
    top = 2.0 * thickness + gap
    xb = a.x.copy()
    xb[:, 2] = top - xb[:, 2]
    conn_b = a.conn[:, perm] + n
    xref_b = a.xref.reshape(-1, 6, 3)[:, perm, :].copy()
    xref_b[:, :, 2] = top - xref_b[:, :, 2]
    cat = lambda u, v: np.concatenate([u, v])
    t = Tissue("stacked_sheets", cat(a.conn, conn_b), cat(a.xref, xref_b.reshape(-1, 18)), cat(a.x, xb),
               cat(a.lam, a.lam), cat(a.mu, a.mu), cat(a.eta, a.eta), cat(a.fixed, a.fixed),
               cat(a.ext_visc, a.ext_visc), cat(a.exposed, a.exposed), cat(a.peripodial, a.peripodial),
               cat(a.rates, a.rates), cat(a.angles, a.angles), cat(a.node_placement, a.node_placement),
               cat(a.at_circumference, a.at_circumference), dt=a.dt, n_steps=n_steps,
               newton_tol=a.newton_tol, seed=a.seed)
    return t


def large_slab(seed: int = 1002, nx: int = 1000, ny: int = 500, spacing: float = 0.5,
               layer_thickness: float = 1.0, n_layers: int = 3, E_median: float = 1000.0,
               sigma_log: float = 0.3, nu: float = 0.3, apical_visc: float = WING_DISC_APICAL_VISC,
               basal_visc: float = WING_DISC_BASAL_VISC, r1: float = 2e-4, r2: float = 5e-5,
               angle_length: float = 20.0,
               dt: float = 60.0, n_steps: int = 20, newton_tol: float = 1e-8) -> Tissue:
    """Large slab: 1000x500-node rectangle at 0.5 um spacing, triangulated and extruded into
    3 layers (2,991,006 prisms); log-normal stiffness per element (median 1000 Pa,
    sigma_log 0.3); anisotropic growth (r1, r2, 0) rotated by a per-element angle from a smooth
    random field; basal nodes fixed in z, drag on apical and basal surfaces."""
    rng = np.random.default_rng(seed)
    gx, gy = np.meshgrid(np.arange(nx) * spacing, np.arange(ny) * spacing, indexing="xy")
    pts2 = np.stack([gx.ravel(), gy.ravel()], axis=1)
    j, i = np.meshgrid(np.arange(ny - 1), np.arange(nx - 1), indexing="ij")
    a = (j * nx + i).ravel()
    b = a + 1
    c = a + nx + 1
    d = a + nx
    tri = np.empty((2 * a.shape[0], 3), np.int64)
    tri[0::2] = np.stack([a, b, c], 1)
    tri[1::2] = np.stack([a, c, d], 1)
    z = [k * layer_thickness for k in range(n_layers + 1)]
    x, conn, xref, layer = _extrude(pts2, tri, z)
    place = _placement(pts2.shape[0], n_layers + 1)
    edge = ((gx == 0) | (gx == (nx - 1) * spacing) | (gy == 0) | (gy == (ny - 1) * spacing)).ravel()
    at_circ = np.repeat(edge.astype(np.int32), n_layers + 1)
    Ee = E_median * np.exp(rng.normal(0.0, sigma_log, conn.shape[0]))
    lam, mu = lame(Ee, nu)
    fixed = np.zeros((x.shape[0], 3), np.uint8)
    fixed[place == BASAL, 2] = 1
    cen = xref.reshape(-1, 6, 3).mean(axis=1)
    ang = math.pi * _smooth_field(rng, cen[:, :2], angle_length)
    rates = np.zeros((conn.shape[0], 3))
    rates[:, 0] = r1
    rates[:, 1] = r2
    return Tissue("large_slab", conn, xref, x, lam, mu, np.zeros(conn.shape[0]), fixed,
                  _ext_visc(place, at_circ, apical_visc, basal_visc),
                  _element_exposure(layer, n_layers), np.zeros(conn.shape[0], np.uint8), rates,
                  ang, place, at_circ, dt=dt, n_steps=n_steps, newton_tol=newton_tol, seed=seed)


def small_disc(seed: int, n_prisms: int, E: float, growth_length: float = 20.0,
               peak_growth: float = 2e-4, thickness: float = 10.0, nu: float = 0.3,
               apical_visc: float = WING_DISC_APICAL_VISC, basal_visc: float = WING_DISC_BASAL_VISC,
               dt: float = 60.0, n_steps: int = 30) -> Tissue:
    """One-layer disc with about n_prisms prisms (radius grows with the count), rim clamped,
    growth from a seeded smooth random field (RBF length scale growth_length)."""
    rng = np.random.default_rng(seed)
    n_pts = max(12, n_prisms // 2)
    radius = math.sqrt(n_pts * 2.0 * math.sqrt(3.0) / (2.0 * math.pi))  # ~2 um lattice
    pts2, is_rim = _disc_points(rng, radius, n_pts)
    tri = _delaunay(pts2)
    pts2, tri, (is_rim,) = _renumber_points(pts2, tri, [is_rim])
    x, conn, xref, layer = _extrude(pts2, tri, [0.0, thickness])
    place = _placement(pts2.shape[0], 2)
    at_circ = np.repeat(is_rim.astype(np.int32), 2)
    lam, mu = lame(np.full(conn.shape[0], E), nu)
    fixed = np.zeros((x.shape[0], 3), np.uint8)
    fixed[at_circ != 0, :] = 1
    cen = xref.reshape(-1, 6, 3).mean(axis=1)
    field = _smooth_field(rng, cen[:, :2], growth_length)
    r = peak_growth * (0.5 + 0.25 * np.tanh(field))
    rates = np.zeros((conn.shape[0], 3))
    rates[:, 0] = r
    rates[:, 1] = r
    return Tissue("small_disc", conn, xref, x, lam, mu, np.zeros(conn.shape[0]), fixed,
                  _ext_visc(place, at_circ, apical_visc, basal_visc), _element_exposure(layer, 1),
                  np.zeros(conn.shape[0], np.uint8), rates, np.zeros(conn.shape[0]), place,
                  at_circ, dt=dt, n_steps=n_steps, seed=seed)


def small_rect_sized(seed: int, n_prisms: int, E: float, growth_length: float = 20.0,
                     peak_growth: float = 2e-4, n_steps: int = 30) -> Tissue:
    """One-layer rectangle with about n_prisms prisms (aspect 2:1) and a smooth random growth
    field; rim clamped like the discs (a rectangle held in-plane by drag alone buckles under
    non-uniform growth and leaves the Newton step ill-posed)."""
    rng = np.random.default_rng(seed)
    ny = max(2, int(round(math.sqrt(n_prisms / 4.0))) + 1)
    nx = max(2, int(round(n_prisms / (2.0 * (ny - 1)))) + 1)
    t = small_rectangle(seed=seed, nx=nx, ny=ny, E=E, n_steps=n_steps, newton_tol=1e-8)
    t.fixed[t.at_circumference != 0, :] = 1
    t.ext_visc = _ext_visc(t.node_placement, t.at_circumference, WING_DISC_APICAL_VISC, WING_DISC_BASAL_VISC)
    cen = t.xref.reshape(-1, 6, 3).mean(axis=1)
    field = _smooth_field(rng, cen[:, :2], growth_length)
    r = peak_growth * (0.5 + 0.25 * np.tanh(field))
    t.rates[:, 0] = r
    t.rates[:, 1] = r
    t.name = "small_rect"
    return t


def batch_tissues(seed: int = 1003, n_tissues: int = 256, min_prisms: int = 500,
                  max_prisms: int = 20000, E_lo: float = 500.0, E_hi: float = 3000.0,
                  n_steps: int = 30) -> List[Tissue]:
    """Batched uneven tissues: discs and rectangles alternating, prism counts log-uniform in
    [500, 20000], growth from seeded smooth random fields (length scale 20 um), E uniform in
    [500, 3000] Pa."""
    rng = np.random.default_rng(seed)
    out = []
    for t in range(n_tissues):
        n = int(round(math.exp(rng.uniform(math.log(min_prisms), math.log(max_prisms)))))
        E = float(rng.uniform(E_lo, E_hi))
        s = int(rng.integers(0, 2**31 - 1))
        out.append(small_disc(s, n, E, n_steps=n_steps) if t % 2 == 0 else small_rect_sized(s, n, E, n_steps=n_steps))
    return out


def bilinear_growth_weights(t: Tissue, grid: int = 32):
    """Per-element bilinear weights of a grid x grid parameter field over the tissue's bounding
    box, as the grid growth function interpolates (ShapeBase.cpp:578-598). Returns
    (index[E,4] int64, weight[E,4]) such that rate_e = sum_k weight[e,k] * params[index[e,k]]."""
    cen = t.xref.reshape(-1, 6, 3).mean(axis=1)
    lo = t.x[:, :2].min(axis=0)
    hi = t.x[:, :2].max(axis=0)
    u = (cen[:, :2] - lo) / np.maximum(hi - lo, 1e-12) * (grid - 1)
    i0 = np.clip(np.floor(u).astype(np.int64), 0, grid - 2)
    f = u - i0
    ix, iy = i0[:, 0], i0[:, 1]
    fx, fy = f[:, 0], f[:, 1]
    idx = np.stack([iy * grid + ix, iy * grid + ix + 1, (iy + 1) * grid + ix, (iy + 1) * grid + ix + 1], 1)
    w = np.stack([(1 - fx) * (1 - fy), fx * (1 - fy), (1 - fx) * fy, fx * fy], 1)
    return idx, w


# ----------------------------------------------------------------------------------------
# .mesh text format (Simulation.cpp:2286-2322, 2431-2447)
# ----------------------------------------------------------------------------------------

def write_mesh(t: Tissue, path: str) -> None:
    """Write the reference's ``.mesh`` input: node count, then ``x y z placement type atCirc``
    per node; element count, then ``1 n0..n5`` and the 18 reference coordinates per prism;
    then the element-weights flag (0)."""
    with open(path, "w") as fh:
        fh.write(f"{t.n_nodes}\n")
        for i in range(t.n_nodes):
            fh.write(f"{t.x[i,0]:.10g} {t.x[i,1]:.10g} {t.x[i,2]:.10g} {int(t.node_placement[i])} 0 {int(t.at_circumference[i])}\n")
        fh.write(f"{t.n_elems}\n")
        for e in range(t.n_elems):
            c = " ".join(str(int(v)) for v in t.conn[e])
            r = " ".join(f"{v:.10g}" for v in t.xref[e])
            fh.write(f"1 {c} {r}\n")
        fh.write("0\n")


def read_mesh(path: str):
    """Read a ``.mesh`` file: returns (x[N,3], placement[N], tissue_type[N], at_circ[N],
    conn[E,6], xref[E,18])."""
    with open(path) as fh:
        tok = fh.read().split()
    p = 0
    n = int(tok[p]); p += 1
    x = np.zeros((n, 3)); place = np.zeros(n, np.int32); ttype = np.zeros(n, np.int32); circ = np.zeros(n, np.int32)
    for i in range(n):
        x[i] = [float(tok[p]), float(tok[p + 1]), float(tok[p + 2])]
        place[i] = int(tok[p + 3]); ttype[i] = int(tok[p + 4]); circ[i] = int(tok[p + 5])
        p += 6
    m = int(tok[p]); p += 1
    conn = np.zeros((m, 6), np.int32); xref = np.zeros((m, 18))
    for e in range(m):
        assert int(tok[p]) == 1, "only prisms (shape type 1) are supported"
        conn[e] = [int(v) for v in tok[p + 1:p + 7]]
        xref[e] = [float(v) for v in tok[p + 7:p + 25]]
        p += 25
    return x, place, ttype, circ, conn, xref


def _g(v: float, precision: int, width: int) -> str:
    """A value as a C++ ostream in its default float format prints it with the given precision
    and field width (the %g rules: shortest of fixed / scientific, no trailing zeros)."""
    return f"{float(v):>{width}.{precision}g}"


def save_frame_block(time_s: float, x, node_placement, tissue_type, at_circumference, conn, xref) -> str:
    """One time block of the reference's ``Save_Frame`` text format (Simulation::writeSaveFileStepHeader,
    writeNodes, writeElements, writeSaveFileStepFooter; Simulation.cpp:8445-8520): header with the
    time, the node count, each node's position (precision 10, width 20) with its placement,
    tissue type and circumference flag (width 4), the element count, each prism's shape type,
    ablation flag, node ids (width 9) and reference positions (precision 4, width 15), footer."""
    x = np.asarray(x, np.float64).reshape(-1, 3)
    conn = np.asarray(conn).reshape(-1, 6)
    xref = np.asarray(xref, np.float64).reshape(-1, 18)
    out = [f"=============== TIME: {_g(time_s, 6, 10)}===================================================\n",
           f"{x.shape[0]}\n"]
    for i in range(x.shape[0]):
        out.append("".join(_g(v, 10, 20) for v in x[i]) + f"{int(node_placement[i]):>4d}{int(tissue_type[i]):>4d}"
                   f"{int(at_circumference[i]):>4d}\n")
    out.append(f"{conn.shape[0]}\n")
    for e in range(conn.shape[0]):
        out.append(f"{1:>4d}{0:>4d}" + "".join(f"{int(v):>9d}" for v in conn[e]) + "".join(_g(v, 4, 15) for v in xref[e]) + "\n")
    out.append(f"=============== END OF TIME: {_g(time_s, 6, 10)}============================================\n")
    return "".join(out)


def write_save_frame(path: str, frames, t: "Tissue", tissue_type=None) -> None:
    """Write ``frames`` [(time in s, positions [N,3]), ...] as a reference ``Save_Frame`` file."""
    ttype = np.zeros(t.n_nodes, np.int32) if tissue_type is None else tissue_type
    with open(path, "w") as fh:
        for time_s, x in frames:
            fh.write(save_frame_block(time_s, x, t.node_placement, ttype, t.at_circumference, t.conn, t.xref))


def read_save_frame(path_or_text: str, is_text: bool = False):
    """Read a reference ``Save_Frame`` file: [(time in s, positions [N,3], node flags [N,3],
    conn [E,6]), ...] with the flags (placement, tissue type, circumference) of every frame."""
    text = path_or_text if is_text else open(path_or_text).read()
    lines = text.splitlines()
    frames, i = [], 0
    while i < len(lines):
        if lines[i].startswith("=============== TIME:"):
            time_s = float(lines[i].split(":", 1)[1].split("=")[0])
            n = int(lines[i + 1])
            rows = [lines[i + 2 + k].split() for k in range(n)]
            x = np.array([[float(v) for v in r[:3]] for r in rows])
            flags = np.array([[int(v) for v in r[3:6]] for r in rows], np.int32)
            m = int(lines[i + 2 + n])
            conn = np.array([[int(v) for v in lines[i + 3 + n + e].split()[2:8]] for e in range(m)], np.int32)
            frames.append((time_s, x, flags, conn))
            i += 3 + n + m
        else:
            i += 1
    return frames
