"""ctypes wrapper of the CPU oracle (``oracle/_build/libtf_oracle.so``).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of bench.py. The product never imports this module.
The oracle restates TissueOrigami's Newton-Raphson path in plain C++ (see tf_oracle.cpp for the
reference file:line of every function). It is pinned to the reference's recorded runs: the growth
prologue (tests/golden/run07008_growth.npz) and the first Newton step of the Pardiso run 07008
(tests/golden/run07008_newton_step1.npz).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libtf_oracle.so")
_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int32)
_U = ctypes.POINTER(ctypes.c_uint8)


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++ -O3 -fopenmp)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        c_int, c_double = ctypes.c_int, ctypes.c_double
        L.tfo_shape_derivatives.argtypes = [c_int, _D, _D, _D]
        L.tfo_element_forces_and_tangents.argtypes = [c_int, _I, _D, _D, _D, _D, _D, _D, _D, c_double, _U, _D, _D, _D, _D, _D, c_int]
        L.tfo_element_forces_and_tangents.restype = c_int
        L.tfo_assemble_dense.argtypes = [c_int, c_int, _I, _D, _D, _D, _D, _D, _D, _D, c_double, _U, _D, _D, _I, c_int, _D, _D, c_int]
        L.tfo_assemble_dense.restype = c_int
        L.tfo_solve_transposed.argtypes = [c_int, _D, _D, _I, c_int, c_int, _D]
        L.tfo_solve_transposed.restype = c_int
        L.tfo_newton_step_dense.argtypes = [c_int, c_int, _I, _D, _D, _D, _D, _D, _D, c_double, c_double, c_int, _U, _D, _D, _I, c_int, _D, _D, c_int]
        L.tfo_newton_step_dense.restype = c_int
        L.tfo_block_pattern.argtypes = [c_int, c_int, _I, _I, _I]
        L.tfo_block_pattern.restype = c_int
        L.tfo_assemble_bsr.argtypes = [c_int, c_int, _I, _D, _D, _D, _D, _D, _D, _D, c_double, _U, _D, _D, _I, _I, _D, _D, c_int]
        L.tfo_assemble_bsr.restype = c_int
        L.tfo_grow.argtypes = [c_int, _I, _D, _D, _D, _D, c_double, _D, _D, _D, _I, _D]
        L.tfo_grid_growth_increments.argtypes = [c_int, c_int, _I, _D, _D, _D, _D, _I, c_int, _D, _D, _I, c_double,
                                                 c_double, _D, _D]
        L.tfo_viscosity_surfaces.argtypes = [c_int, c_int, _I, _D, _U, _U, _D]
        L.tfo_detect_packing.argtypes = [c_int, c_int, _I, _D, _I, _U, _U, c_int, _I, _D]
        L.tfo_detect_packing.restype = c_int
        L.tfo_node_masses.argtypes = [c_int, c_int, _I, _D, _D, _D]
        L.tfo_node_masses.restype = None
        L.tfo_packing_terms.argtypes = [c_int, _I, _D, _D, c_double, _D, _D]
        L.tfo_packing_terms.restype = None
        L.tfo_lumen_volume.argtypes = [c_int, _I, _D]
        L.tfo_lumen_volume.restype = c_double
        L.tfo_lumen_terms.argtypes = [c_int, c_int, _I, _D, _U, c_double, c_double, _D, _D]
        L.tfo_lumen_terms.restype = None
        _lib = L
    return _lib


def _d(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def _i(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_I)


def _u(a):
    if a is None:
        return None
    assert a.dtype == np.uint8 and a.flags.c_contiguous
    return a.ctypes.data_as(_U)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def shape_derivatives(xref):
    xref = _c(xref, np.float64).reshape(-1, 18)
    E = xref.shape[0]
    inv = np.zeros((E, 6, 9))
    det = np.zeros((E, 6))
    lib().tfo_shape_derivatives(E, _d(xref), _d(inv), _d(det))
    return inv, det


def element_forces_and_tangents(t, x, v=None, dt=None, inv_fg=None, threads=0, strain=False):
    """Per-element (f_elastic[E,18], f_viscous[E,18], Ke[E,18,18], Kv[E,18,18]) at positions x
    and nodal velocity v = (uk-un)/dt, in the reference's storage."""
    E = t.n_elems
    conn = _c(t.conn, np.int32)
    xref = _c(t.xref, np.float64)
    inv_fg = _c(inv_fg if inv_fg is not None else np.linalg.inv(t.fg.reshape(-1, 3, 3)).reshape(-1, 9), np.float64)
    x = _c(x, np.float64)
    v = _c(v if v is not None else np.zeros_like(x), np.float64)
    fe = np.zeros((E, 18)); fv = np.zeros((E, 18))
    ke = np.zeros((E, 18, 18)); kv = np.zeros((E, 18, 18))
    st = np.zeros((E, 6, 6)) if strain else None
    bad = lib().tfo_element_forces_and_tangents(E, _i(conn), _d(xref), _d(inv_fg), _d(_c(t.lam, np.float64)),
                                                _d(_c(t.mu, np.float64)), _d(_c(t.eta, np.float64)), _d(x), _d(v),
                                                float(dt if dt is not None else t.dt), _u(_c(t.fixed, np.uint8)),
                                                _d(fe), _d(fv), _d(ke), _d(kv), _d(st), int(threads))
    return fe, fv, ke, kv, st, bad


def assemble_dense(t, uk, un, visc_surface, inv_fg, dt=None, threads=0):
    """Dense reference-storage K[3N,3N] and gSum[3N] after fixed-DoF and slave-master steps."""
    n = 3 * t.n_nodes
    K = np.zeros((n, n)); g = np.zeros(n)
    sm = _c(t.slave_master.reshape(-1), np.int32)
    lib().tfo_assemble_dense(t.n_nodes, t.n_elems, _i(_c(t.conn, np.int32)), _d(_c(t.xref, np.float64)),
                             _d(_c(inv_fg, np.float64)), _d(_c(t.lam, np.float64)), _d(_c(t.mu, np.float64)),
                             _d(_c(t.eta, np.float64)), _d(_c(uk, np.float64)), _d(_c(un, np.float64)),
                             float(dt if dt is not None else t.dt), _u(_c(t.fixed, np.uint8)),
                             _d(_c(visc_surface, np.float64)), _d(_c(t.ext_visc, np.float64)),
                             _i(sm) if sm.size else None, int(t.slave_master.shape[0]), _d(K), _d(g), int(threads))
    return K, g


def solve_transposed(K, g, slave_master=None, n_refine=1):
    n = g.shape[0]
    du = np.zeros(n)
    sm = _c(slave_master.reshape(-1), np.int32) if slave_master is not None and slave_master.size else None
    st = lib().tfo_solve_transposed(n, _d(_c(K, np.float64)), _d(_c(g, np.float64)), _i(sm),
                                    0 if sm is None else sm.size // 2, int(n_refine), _d(du))
    return du, st


def newton_step_dense(t, x_n, visc_surface, inv_fg, dt=None, tol=None, max_iter=20, threads=0):
    n = 3 * t.n_nodes
    x_out = np.zeros((t.n_nodes, 3))
    norms = np.zeros(max_iter + 2)
    sm = _c(t.slave_master.reshape(-1), np.int32)
    it = lib().tfo_newton_step_dense(t.n_nodes, t.n_elems, _i(_c(t.conn, np.int32)), _d(_c(t.xref, np.float64)),
                                     _d(_c(inv_fg, np.float64)), _d(_c(t.lam, np.float64)), _d(_c(t.mu, np.float64)),
                                     _d(_c(t.eta, np.float64)), _d(_c(x_n, np.float64)),
                                     float(dt if dt is not None else t.dt), float(tol if tol is not None else t.newton_tol),
                                     int(max_iter), _u(_c(t.fixed, np.uint8)), _d(_c(visc_surface, np.float64)),
                                     _d(_c(t.ext_visc, np.float64)), _i(sm) if sm.size else None,
                                     int(t.slave_master.shape[0]), _d(x_out), _d(norms), int(threads))
    del n
    return x_out, it, norms[:it]


def block_pattern(t):
    conn = _c(t.conn, np.int32)
    nnzb = lib().tfo_block_pattern(t.n_nodes, t.n_elems, _i(conn), None, None)
    rowptr = np.zeros(t.n_nodes + 1, np.int32)
    colidx = np.zeros(nnzb, np.int32)
    lib().tfo_block_pattern(t.n_nodes, t.n_elems, _i(conn), _i(rowptr), _i(colidx))
    return rowptr, colidx


def assemble_bsr(t, uk, un, visc_surface, inv_fg, rowptr, colidx, dt=None, threads=0):
    """True Jacobian J = K^T in BSR3 over (rowptr, colidx) and g, without slave-master pairs."""
    vals = np.zeros((colidx.shape[0], 3, 3))
    g = np.zeros(3 * t.n_nodes)
    lib().tfo_assemble_bsr(t.n_nodes, t.n_elems, _i(_c(t.conn, np.int32)), _d(_c(t.xref, np.float64)),
                           _d(_c(inv_fg, np.float64)), _d(_c(t.lam, np.float64)), _d(_c(t.mu, np.float64)),
                           _d(_c(t.eta, np.float64)), _d(_c(uk, np.float64)), _d(_c(un, np.float64)),
                           float(dt if dt is not None else t.dt), _u(_c(t.fixed, np.uint8)),
                           _d(_c(visc_surface, np.float64)), _d(_c(t.ext_visc, np.float64)),
                           _i(rowptr), _i(colidx), _d(vals), _d(g), int(threads))
    return vals, g


def grow(t, x, fg, dt=None, grid_inc=None):
    """One step of the growth prologue. grid_inc[E,9]: optional increments of grid-based growth
    functions (grid_growth_increments), applied after the uniform one.
    Returns (fg_new[E,9], inv_fg[E,9], det_fg[E], rotated[E])."""
    fg = np.array(fg, dtype=np.float64, copy=True).reshape(-1, 9)
    inv = np.zeros_like(fg)
    det = np.zeros(t.n_elems)
    rot = np.zeros(t.n_elems, np.int32)
    gi = None if grid_inc is None else _c(grid_inc, np.float64).reshape(-1, 9)
    lib().tfo_grow(t.n_elems, _i(_c(t.conn, np.int32)), _d(_c(t.xref, np.float64)), _d(_c(x, np.float64)),
                   _d(_c(t.rates, np.float64)), _d(_c(t.angles, np.float64)), float(dt if dt is not None else t.dt),
                   _d(fg), _d(inv), _d(det), _i(rot), _d(gi))
    return fg, inv, det, rot


def grid_growth_increments(funcs, rel_pos, rel_z, eflags, interpolation, t_now, dt, per_function=False):
    """Composed increments [E,9] of the grid-based growth functions active at t_now. funcs: list of
    dicts with nx, ny, rates[nx,ny,3] (1/s), angles_deg[nx,ny], t0, t1, zmin, zmax, flags.
    per_function: also return (applied[F,E] bool, increment[F,E,9]) of each function on its own."""
    E = rel_z.shape[0]
    dims = np.array([[f["nx"], f["ny"]] for f in funcs], np.int32).reshape(-1)
    rates = np.concatenate([np.asarray(f["rates"], np.float64).reshape(-1) for f in funcs])
    angs = np.concatenate([np.asarray(f["angles_deg"], np.float64).reshape(-1) for f in funcs])
    win = np.array([[f["t0"], f["t1"]] for f in funcs], np.float64).reshape(-1)
    zr = np.array([[f["zmin"], f["zmax"]] for f in funcs], np.float64).reshape(-1)
    fl = np.array([f["flags"] for f in funcs], np.int32)
    inc = np.zeros((E, 9))
    pf = np.zeros((len(funcs), E, 10)) if per_function else None
    lib().tfo_grid_growth_increments(E, len(funcs), _i(dims), _d(rates), _d(angs), _d(win), _d(zr), _i(fl),
                                     int(interpolation), _d(_c(rel_pos, np.float64)), _d(_c(rel_z, np.float64)),
                                     _i(_c(eflags, np.int32)), float(t_now), float(dt), _d(inc), _d(pf))
    if per_function:
        return inc, pf[:, :, 0] != 0, pf[:, :, 1:]
    return inc


def viscosity_surfaces(t, x):
    vs = np.zeros(t.n_nodes)
    lib().tfo_viscosity_surfaces(t.n_nodes, t.n_elems, _i(_c(t.conn, np.int32)), _d(_c(x, np.float64)),
                                 _u(_c(t.exposed, np.uint8)), _u(_c(t.peripodial, np.uint8)), _d(vs))
    return vs


def detect_packing(t, x):
    """Node-node packing candidates at positions x (Simulation::detectPacingNodes): returns
    (pairs[P,2] int32 in the reference's visiting order, packingThreshold)."""
    args = (t.n_nodes, t.n_elems, _i(_c(t.conn, np.int32)), _d(_c(x, np.float64)),
            _i(_c(t.node_placement, np.int32)), _u(_c(t.exposed, np.uint8)), _u(_c(t.peripodial, np.uint8)))
    thr = ctypes.c_double(0.0)
    n = lib().tfo_detect_packing(*args, 0, None, ctypes.byref(thr))
    pairs = np.zeros((max(n, 1), 2), np.int32)
    if n:
        lib().tfo_detect_packing(*args, n, _i(pairs), None)
    return pairs[:n], thr.value


def node_masses(t, fg):
    """Node masses after the step's growth (Simulation::updateNodeMasses): det(Fg) x reference
    volume / 6 from every element of the node."""
    mass = np.zeros(t.n_nodes)
    lib().tfo_node_masses(t.n_nodes, t.n_elems, _i(_c(t.conn, np.int32)), _d(_c(t.xref, np.float64)),
                          _d(_c(fg, np.float64)), _d(mass))
    return mass


def packing_terms(t, x, pairs, mass, threshold):
    """Packing forces [N,3] and the pairs' 3x3 derivative blocks dF_i/dx_i [P,3,3] at positions x
    (Simulation::calculatePackingForcesImplicit3D / calculatePackingJacobian3D)."""
    pairs = _c(np.asarray(pairs).reshape(-1, 2), np.int32)
    forces = np.zeros((t.n_nodes, 3))
    dfdx = np.zeros((max(pairs.shape[0], 1), 3, 3))
    if pairs.shape[0]:
        lib().tfo_packing_terms(pairs.shape[0], _i(pairs), _d(_c(x, np.float64)), _d(_c(mass, np.float64)),
                                float(threshold), _d(forces), _d(dfdx))
    return forces, dfdx[:pairs.shape[0]]


def add_packing(t, J, g, x, pairs, mass, threshold):
    """J + the packing Jacobian blocks (-D at (i, i) and (j, j), +D at (i, j) and (j, i)) and g +
    the packing forces, both with the fixed DoFs' rows and columns left out (calcutateFixedK runs
    after the packing terms, NewtonRaphsonSolver.cpp:195-219); D is symmetric, so J = K^T holds."""
    import scipy.sparse as sp

    forces, D = packing_terms(t, x, pairs, mass, threshold)
    free = (np.asarray(t.fixed).reshape(-1) == 0)
    g = g + np.where(free, forces.reshape(-1), 0.0)
    if len(pairs) == 0:
        return J, g
    rows, cols, vals = [], [], []
    for p, (i, j) in enumerate(np.asarray(pairs)):
        for (a, b, sgn) in ((i, i, -1.0), (i, j, 1.0), (j, j, -1.0), (j, i, 1.0)):
            for r in range(3):
                for c in range(3):
                    R, C = 3 * a + r, 3 * b + c
                    if free[R] and free[C]:
                        rows.append(R)
                        cols.append(C)
                        vals.append(sgn * D[p, r, c])
    n = 3 * t.n_nodes
    return (J + sp.csr_matrix((vals, (rows, cols)), shape=(n, n))).tocsr(), g


def lumen_triangles(t, elems):
    """The apical triangles (nodes 3, 4, 5) of the lumen elements (Lumen::Lumen, Lumen.cpp:11-68)."""
    return _c(np.asarray(t.conn)[np.asarray(elems)][:, 3:6], np.int32)


def lumen_volume(t, x, tri):
    tri = _c(np.asarray(tri).reshape(-1, 3), np.int32)
    return float(lib().tfo_lumen_volume(tri.shape[0], _i(tri), _d(_c(x, np.float64))))


def lumen_terms(t, x, tri, bulk, ideal):
    """Lumen pressure forces [N,3] and its Jacobian K[3N,3N] (the reference's storage, fixed rows
    and columns left out) at positions x (Lumen::calculateResiduals / calculateJacobian)."""
    tri = _c(np.asarray(tri).reshape(-1, 3), np.int32)
    n = 3 * t.n_nodes
    forces = np.zeros((t.n_nodes, 3))
    K = np.zeros((n, n))
    lib().tfo_lumen_terms(t.n_nodes, tri.shape[0], _i(tri), _d(_c(x, np.float64)), _u(_c(t.fixed, np.uint8)),
                          float(bulk), float(ideal), _d(forces), _d(K))
    return forces, K


def add_lumen(t, J, g, x, tri, bulk, ideal):
    """J + K_lumen^T (J = K^T) and g + the lumen forces."""
    import scipy.sparse as sp

    forces, K = lumen_terms(t, x, tri, bulk, ideal)
    return (J + sp.csr_matrix(K.T)).tocsr(), g + forces.reshape(-1)


def bsr_to_scipy(rowptr, colidx, vals, n_nodes):
    import scipy.sparse as sp

    return sp.bsr_matrix((np.asarray(vals).reshape(-1, 3, 3), colidx, rowptr), shape=(3 * n_nodes, 3 * n_nodes)).tocsr()


def simulate_dense(t, n_steps=None, max_iter=20, tol=None, threads=0):
    """Run n time steps of the reference path on the CPU with dense assembly and the LU
    stand-in for Pardiso: growth prologue, viscosity surfaces, Newton step.
    Returns (x, fg, per-step iteration counts, per-step norm traces)."""
    x = np.array(t.x, dtype=np.float64, copy=True)
    fg = np.array(t.fg, dtype=np.float64, copy=True)
    iters, traces = [], []
    for _ in range(n_steps if n_steps is not None else t.n_steps):
        fg, inv, _, _ = grow(t, x, fg)
        vs = viscosity_surfaces(t, x)
        x, it, norms = newton_step_dense(t, x, vs, inv, tol=tol, max_iter=max_iter, threads=threads)
        iters.append(it)
        traces.append(norms)
    return x, fg, iters, traces


def nested_dissection(t, rowptr, colidx, leaf=128):
    """Fill-reducing node order for the direct solve: recursive coordinate bisection of the
    reference positions (split at the median of the longer in-plane side), the nodes of the left
    half that couple to the right half forming the separator, ordered last. Returns the DoF
    permutation (3 DoFs of a node kept together)."""
    import scipy.sparse as sp

    N = t.n_nodes
    A = sp.csr_matrix((np.ones(colidx.shape[0]), colidx, rowptr), shape=(N, N))
    X = np.asarray(t.x)
    order = []

    def rec(nodes):
        if nodes.shape[0] <= leaf:
            order.append(nodes)
            return
        P = X[nodes, :2]
        ax = int(np.argmax(P.max(axis=0) - P.min(axis=0)))
        left = P[:, ax] < np.median(P[:, ax])
        if left.all() or not left.any():
            order.append(nodes)
            return
        L, R = nodes[left], nodes[~left]
        in_r = np.zeros(N, bool)
        in_r[R] = True
        sep = np.asarray(A[L].multiply(in_r[None, :]).sum(axis=1)).ravel() > 0
        rec(L[~sep])
        rec(R)
        order.append(L[sep])

    rec(np.arange(N))
    nodes = np.concatenate(order)
    return (3 * nodes[:, None] + np.arange(3)[None, :]).ravel()


def sparse_direct_solve(J, g, perm=None):
    """Direct solve of J du = g by SuperLU (the Pardiso stand-in of the sparse path); with a
    fill-reducing DoF permutation the factorisation keeps the natural order of the permuted
    matrix and prefers diagonal pivots (the matrix is structurally symmetric)."""
    import scipy.sparse.linalg as sla

    if perm is None:
        return sla.spsolve(J.tocsc(), g)
    Jp = J.tocsr()[perm][:, perm].tocsc()
    lu = sla.splu(Jp, permc_spec="NATURAL", options=dict(SymmetricMode=True))
    du = np.empty_like(g)
    du[perm] = lu.solve(g[perm])
    return du


def newton_step_sparse(t, x_n, visc_surface, inv_fg, dt=None, tol=None, max_iter=20, threads=0, perm=None,
                       packing=None, lumen=None):
    """Simulation::updateStepNR with sparse assembly of J = K^T and SuperLU (scipy) as the
    direct solve standing in for Pardiso. No slave-master pairs. Returns (x, iterations, norms).
    perm: optional fill-reducing DoF order for the factorisation (nested_dissection).
    packing: optional (pairs, masses, threshold) of the step; its forces and Jacobian are added
    at every iteration's positions. lumen: optional (triangles, bulk modulus, ideal volume)."""
    rowptr, colidx = block_pattern(t)
    un = np.array(x_n, dtype=np.float64, copy=True).reshape(-1, 3)
    uk = un.copy()
    norms = []
    it = 0
    converged = False
    tol = float(tol if tol is not None else t.newton_tol)
    while not converged:
        vals, g = assemble_bsr(t, uk, un, visc_surface, inv_fg, rowptr, colidx, dt=dt, threads=threads)
        J = bsr_to_scipy(rowptr, colidx, vals, t.n_nodes)
        if packing is not None:
            J, g = add_packing(t, J, g, uk, *packing)
        if lumen is not None:
            J, g = add_lumen(t, J, g, uk, *lumen)
        du = sparse_direct_solve(J, g, perm)
        d = float(np.sqrt(np.sum(du * du)))
        norms.append(d)
        converged = not (d > tol)
        uk = uk + du.reshape(-1, 3)
        it += 1
        if not converged and it > max_iter:
            converged = True
    return uk, it, np.array(norms)


def simulate_sparse(t, n_steps=None, max_iter=20, tol=None, threads=0, reorder=False, positions=None,
                    packing=False, pair_counts=None, lumen=None):
    """n time steps with the growth prologue and the sparse Newton step. reorder: factorise in
    nested-dissection order (large meshes). positions: optional list that receives the positions
    at the start of every step and after the last. packing: node masses and packing pairs
    detected after each step's growth (Simulation::runOneStep, Simulation.cpp:6065-6076), their
    forces and Jacobian in every Newton iteration; pair_counts: optional list of each step's
    number of pairs. lumen: optional (lumen elements, bulk modulus, growth fold per day): the
    ideal volume starts at the initial enclosed volume and grows as V0 exp(ln(fold) / 86400 t)
    to the end of each step (Lumen::growLumen, Lumen.cpp:331-334; Simulation.cpp:6019)."""
    x = np.array(t.x, dtype=np.float64, copy=True)
    fg = np.array(t.fg, dtype=np.float64, copy=True)
    iters, traces = [], []
    perm = nested_dissection(t, *block_pattern(t)) if reorder else None
    lm = None
    if lumen is not None:
        tri = lumen_triangles(t, lumen[0])
        v_init = lumen_volume(t, x, tri)
        rate = np.log(lumen[2]) / 3600.0 / 24.0 if lumen[2] > 0 else 0.0
    for step in range(n_steps if n_steps is not None else t.n_steps):
        if lumen is not None:
            lm = (tri, lumen[1], v_init * np.exp(rate * (step + 1) * t.dt))
        if positions is not None:
            positions.append(x.copy())
        fg, inv, _, _ = grow(t, x, fg)
        vs = viscosity_surfaces(t, x)
        pk = None
        if packing:
            pairs, thr = detect_packing(t, x)
            pk = (pairs, node_masses(t, fg), thr)
            if pair_counts is not None:
                pair_counts.append(len(pairs))
        x, it, norms = newton_step_sparse(t, x, vs, inv, tol=tol, max_iter=max_iter, threads=threads, perm=perm,
                                          packing=pk, lumen=lm)
        iters.append(it)
        traces.append(norms)
    if positions is not None:
        positions.append(x.copy())
    return x, fg, iters, traces
