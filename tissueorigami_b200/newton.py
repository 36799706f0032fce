"""Host-side mirror of TissueOrigami's NewtonRaphsonSolver over the B200 C ABI.

``NewtonRaphsonSolver`` keeps the reference's vocabulary (TissueFolding/SourceCode/
NewtonRaphsonSolver.h:51-91, Simulation.cpp:6605-6747): one object per tissue that owns the
device state, is fed the node and element data the reference keeps in ``Node`` / ``ShapeBase``
and performs ``updateStepNR`` or a whole ``runOneStep`` prologue + Newton step. All work runs
in the CUDA library; a missing library or GPU raises.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import capi
from .mesh import Tissue


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class NewtonRaphsonSolver:
    """One tissue on one GPU (``NewtonRaphsonSolver`` + the element and node state it reads)."""

    def __init__(self, conn, xref, n_nodes: int, params: Optional[capi.Params] = None, **overrides):
        L = capi.load()
        self._L = L
        self.n_nodes = int(n_nodes)
        self.conn = np.ascontiguousarray(conn, dtype=np.int32).reshape(-1, 6)
        self.xref = _f64(xref).reshape(-1, 18)
        self.n_elems = self.conn.shape[0]
        p = params if params is not None else capi.default_params()
        for k, v in overrides.items():
            setattr(p, k, v)
        self.params = p
        desc = capi.MeshDesc(self.n_nodes, self.n_elems, capi.iptr(self.conn), capi.dptr(self.xref))
        h = ctypes.c_void_p()
        capi.check(L.tf_create(ctypes.byref(desc), ctypes.byref(p), ctypes.byref(h)), "tf_create")
        self._h = h
        self.last_stats = None

    # -- construction from a synthetic / loaded tissue ---------------------------------------
    @classmethod
    def from_tissue(cls, t: Tissue, params: Optional[capi.Params] = None, packing: bool = False, **overrides):
        """packing: run the reference's node-node packing (detection after every step's growth,
        forces and Jacobian in every Newton iteration) with the tissue's node placements."""
        overrides.setdefault("newton_tol", t.newton_tol)
        s = cls(t.conn, t.xref, t.n_nodes, params, **overrides)
        s.set_material(t.lam, t.mu, t.eta)
        s.set_boundary(t.fixed, t.ext_visc, t.slave_master)
        s.set_growth(t.fg, t.rates, t.angles, t.exposed, t.peripodial)
        if packing:
            s.set_packing(t.node_placement)
        return s

    # -- lumen (Lumen.cpp) ------------------------------------------------------------------
    def set_lumen(self, elems=None, bulk_modulus: float = 0.0, growth_fold: float = 0.0, x=None):
        """Lumen on the apical triangles of `elems` (ideal volume: the volume at positions x), or
        none with elems None."""
        if elems is None or len(elems) == 0:
            capi.check(self._L.tf_set_lumen(self._h, 0, None, 0.0, 0.0, None), "tf_set_lumen", self._h)
            return
        e = np.ascontiguousarray(elems, dtype=np.int32)
        capi.check(self._L.tf_set_lumen(self._h, e.size, capi.iptr(e), float(bulk_modulus), float(growth_fold),
                                        capi.dptr(_f64(x).reshape(-1))), "tf_set_lumen", self._h)

    def lumen(self):
        """(enclosed volume at the last assembly, ideal volume, G [N,3])."""
        v, v0 = ctypes.c_double(), ctypes.c_double()
        G = np.zeros((self.n_nodes, 3))
        capi.check(self._L.tf_get_lumen(self._h, ctypes.byref(v), ctypes.byref(v0), capi.dptr(G)), "tf_get_lumen", self._h)
        return v.value, v0.value, G

    # -- packing (Simulation::detectPacingNodes, calculatePackingForcesImplicit3D / Jacobian3D) --
    def set_packing(self, node_placement=None):
        """Turn packing on with node_placement[N] (0 basal, 1 apical, 2 other), or off with None."""
        if node_placement is None:
            capi.check(self._L.tf_set_packing(self._h, 0, None), "tf_set_packing", self._h)
            return
        pl = np.ascontiguousarray(node_placement, dtype=np.int32)
        capi.check(self._L.tf_set_packing(self._h, 1, capi.iptr(pl)), "tf_set_packing", self._h)

    def detect_packing(self, x):
        """Detect the packing pairs at positions x with the current growth tensors; returns their count."""
        n = ctypes.c_int32()
        capi.check(self._L.tf_detect_packing(self._h, capi.dptr(_f64(x).reshape(-1)), ctypes.byref(n)),
                   "tf_detect_packing", self._h)
        return n.value

    def packing(self):
        """(pairs[P,2], packingThreshold, node masses[N], derivative blocks dF_i/dx_i [P,3,3] of the last assembly)."""
        n = ctypes.c_int32()
        capi.check(self._L.tf_get_packing(self._h, 0, ctypes.byref(n), None, None, None, None), "tf_get_packing", self._h)
        P = n.value
        pairs = np.zeros((max(P, 1), 2), np.int32)
        dfdx = np.zeros((max(P, 1), 3, 3))
        mass = np.zeros(self.n_nodes)
        thr = ctypes.c_double()
        capi.check(self._L.tf_get_packing(self._h, P, ctypes.byref(n), capi.iptr(pairs), ctypes.byref(thr),
                                          capi.dptr(mass), capi.dptr(dfdx)), "tf_get_packing", self._h)
        return pairs[:P], thr.value, mass, dfdx[:P]

    def close(self):
        if getattr(self, "_h", None):
            self._L.tf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state setters (Node / ShapeBase fields) ----------------------------------------------
    def set_material(self, lam, mu, eta=None):
        eta_a = _f64(eta) if eta is not None else None
        capi.check(self._L.tf_set_material(self._h, capi.dptr(_f64(lam)), capi.dptr(_f64(mu)), capi.dptr(eta_a)),
                   "tf_set_material", self._h)

    def set_inv_fg(self, inv_fg):
        capi.check(self._L.tf_set_inv_fg(self._h, capi.dptr(_f64(inv_fg).reshape(-1))), "tf_set_inv_fg", self._h)

    def set_boundary(self, fixed, ext_visc, slave_master=None):
        sm = np.ascontiguousarray(slave_master if slave_master is not None else np.zeros((0, 2)), dtype=np.int32).reshape(-1)
        fx = np.ascontiguousarray(fixed, dtype=np.uint8).reshape(-1)
        capi.check(self._L.tf_set_boundary(self._h, capi.uptr(fx), capi.dptr(_f64(ext_visc).reshape(-1)),
                                           capi.iptr(sm) if sm.size else None, sm.size // 2),
                   "tf_set_boundary", self._h)

    def set_viscosity_surface(self, visc_surface):
        capi.check(self._L.tf_set_viscosity_surface(self._h, capi.dptr(_f64(visc_surface))),
                   "tf_set_viscosity_surface", self._h)

    def set_growth(self, fg=None, rates=None, angles=None, exposed=None, peripodial=None):
        capi.check(self._L.tf_set_growth(
            self._h,
            capi.dptr(_f64(fg).reshape(-1)) if fg is not None else None,
            capi.dptr(_f64(rates).reshape(-1)) if rates is not None else None,
            capi.dptr(_f64(angles)) if angles is not None else None,
            capi.uptr(np.ascontiguousarray(exposed, dtype=np.uint8)) if exposed is not None else None,
            capi.uptr(np.ascontiguousarray(peripodial, dtype=np.uint8)) if peripodial is not None else None),
            "tf_set_growth", self._h)

    def set_grid_growth(self, funcs, interpolation: int, rel_pos, rel_z, elem_flags):
        """Grid-based growth functions (tf_set_grid_growth): funcs is a list of dicts with t0, t1,
        rates[nx,ny,3] (1/s), angles_deg[nx,ny], zmin, zmax, flags; per element the pinned relative
        position [E,2], initialRelativePositionInZ [E] and flags [E] (modelinput.grid_element_state)."""
        keep = []
        arr = (capi.GridGrowth * max(len(funcs), 1))()
        for i, f in enumerate(funcs):
            r = _f64(f["rates"]).reshape(-1)
            a = _f64(f["angles_deg"]).reshape(-1)
            nx, ny = int(f["rates"].shape[0]), int(f["rates"].shape[1])
            keep += [r, a]
            arr[i] = capi.GridGrowth(float(f["t0"]), float(f["t1"]), nx, ny, capi.dptr(r), capi.dptr(a),
                                     float(f["zmin"]), float(f["zmax"]), int(f["flags"]), 0)
        rp, rz = _f64(rel_pos).reshape(-1), _f64(rel_z)
        ef = np.ascontiguousarray(elem_flags, dtype=np.int32)
        capi.check(self._L.tf_set_grid_growth(self._h, len(funcs), arr, int(interpolation), capi.dptr(rp),
                                              capi.dptr(rz), capi.iptr(ef)), "tf_set_grid_growth", self._h)

    def set_time(self, t: float):
        """Simulation time at the start of the next step (Simulation::currSimTimeSec)."""
        capi.check(self._L.tf_set_time(self._h, float(t)), "tf_set_time", self._h)

    def time(self) -> float:
        v = ctypes.c_double()
        capi.check(self._L.tf_get_time(self._h, ctypes.byref(v)), "tf_get_time", self._h)
        return v.value

    def get_growth(self):
        fg = np.zeros((self.n_elems, 9))
        inv = np.zeros((self.n_elems, 9))
        capi.check(self._L.tf_get_growth(self._h, capi.dptr(fg), capi.dptr(inv)), "tf_get_growth", self._h)
        return fg, inv

    # -- the path -------------------------------------------------------------------------------
    def updateStepNR(self, x_n, dt: float):
        """Simulation::updateStepNR: returns (positions, status, stats dict)."""
        x = _f64(x_n).reshape(self.n_nodes, 3).copy()
        out = np.empty_like(x)
        st = capi.StepStats()
        rc = capi.check(self._L.tf_newton_step(self._h, capi.dptr(x), float(dt), capi.dptr(out), ctypes.byref(st)),
                        "tf_newton_step", self._h)
        self.last_stats = st.as_dict()
        return out, rc, self.last_stats

    def runOneStep(self, x_n, dt: float):
        """Growth prologue + viscosity surfaces + updateStepNR (Simulation::runOneStep subset)."""
        x = _f64(x_n).reshape(self.n_nodes, 3).copy()
        out = np.empty_like(x)
        st = capi.StepStats()
        rc = capi.check(self._L.tf_time_step(self._h, capi.dptr(x), float(dt), capi.dptr(out), ctypes.byref(st)),
                        "tf_time_step", self._h)
        self.last_stats = st.as_dict()
        return out, rc, self.last_stats

    def pattern(self):
        nnzb = ctypes.c_int32()
        self._L.tf_get_pattern(self._h, ctypes.byref(nnzb), None, None)
        rowptr = np.zeros(self.n_nodes + 1, np.int32)
        colidx = np.zeros(nnzb.value, np.int32)
        self._L.tf_get_pattern(self._h, None, capi.iptr(rowptr), capi.iptr(colidx))
        return rowptr, colidx

    def assemble(self, uk, un, dt: float, want_matrix: bool = True):
        """One Newton iteration's residual gSum and Jacobian J = K^T (BSR3 values)."""
        rowptr, colidx = self.pattern()
        g = np.zeros(3 * self.n_nodes)
        vals = np.zeros((colidx.shape[0], 3, 3)) if want_matrix else None
        rc = capi.check(self._L.tf_assemble(self._h, capi.dptr(_f64(uk).reshape(-1)), capi.dptr(_f64(un).reshape(-1)),
                                            float(dt), capi.dptr(g), capi.dptr(vals)), "tf_assemble", self._h)
        return g, vals, rowptr, colidx, rc

    def set_external_force(self, f=None):
        """NewtonRaphsonSolver::gExt: external nodal forces [N,3] added to the residual (None: none)."""
        capi.check(self._L.tf_set_external_force(self._h, capi.dptr(_f64(f).reshape(-1)) if f is not None else None),
                   "tf_set_external_force", self._h)

    def newton_iteration(self, uk, un, dt: float):
        """One Newton iteration's assembly and solve on the device (tf_newton_iteration):
        returns (deltaU [3N], status, BiCGStab iterations, relative residual)."""
        du = np.zeros(3 * self.n_nodes)
        it, rr = ctypes.c_int32(), ctypes.c_double()
        rc = capi.check(self._L.tf_newton_iteration(self._h, capi.dptr(_f64(uk).reshape(-1)), capi.dptr(_f64(un).reshape(-1)),
                                                    float(dt), capi.dptr(du), ctypes.byref(it), ctypes.byref(rr)),
                        "tf_newton_iteration", self._h)
        return du, rc, it.value, rr.value

    def solveForDeltaU(self, vals, g):
        """Solve J du = g on the context's pattern (NewtonRaphsonSolver::solveForDeltaU)."""
        du = np.zeros(3 * self.n_nodes)
        it = ctypes.c_int32()
        rr = ctypes.c_double()
        rc = capi.check(self._L.tf_solve(self._h, capi.dptr(_f64(vals).reshape(-1)), capi.dptr(_f64(g)), capi.dptr(du),
                                         ctypes.byref(it), ctypes.byref(rr)), "tf_solve", self._h)
        return du, rc, it.value, rr.value

    # -- discrete adjoint ------------------------------------------------------------------------
    def adjoint_forward(self, x0, n_steps: int, dt: float, checkpoint_every: int = 5):
        """Run n_steps time steps from x0 keeping checkpoints; returns (x_final, status, stats)."""
        x = _f64(x0).reshape(self.n_nodes, 3).copy()
        out = np.empty_like(x)
        st = capi.StepStats()
        rc = capi.check(self._L.tf_adjoint_forward(self._h, capi.dptr(x), int(n_steps), float(dt), int(checkpoint_every),
                                                   capi.dptr(out), ctypes.byref(st)), "tf_adjoint_forward", self._h)
        return out, rc, st.as_dict()

    def adjoint_backward(self, dL_dx_final, want_dx0: bool = False):
        """dL/d(growth rates) [E,3] (and dL/dx0 [N,3]) for dL/dx_final of the last forward run."""
        g = _f64(dL_dx_final).reshape(-1).copy()
        dr = np.zeros((self.n_elems, 3))
        dx0 = np.zeros((self.n_nodes, 3)) if want_dx0 else None
        st = capi.StepStats()
        rc = capi.check(self._L.tf_adjoint_backward(self._h, capi.dptr(g), capi.dptr(dr), capi.dptr(dx0), ctypes.byref(st)),
                        "tf_adjoint_backward", self._h)
        return dr, dx0, rc, st.as_dict()

    def solve_direct(self, vals, g):
        """cuSOLVER sparse Cholesky / QR solve of J du = g (timed beside the Krylov solve)."""
        du = np.zeros(3 * self.n_nodes)
        ms = ctypes.c_double()
        m = ctypes.c_int32()
        rc = capi.check(self._L.tf_solve_direct(self._h, capi.dptr(_f64(vals).reshape(-1)), capi.dptr(_f64(g)), capi.dptr(du),
                                                ctypes.byref(ms), ctypes.byref(m)), "tf_solve_direct", self._h)
        return du, rc, ms.value, m.value

    def schedule(self):
        nc, sc, t = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        self._L.tf_get_schedule(self._h, ctypes.byref(nc), ctypes.byref(sc), ctypes.byref(t))
        return {"n_colours": nc.value, "scatter": sc.value, "elems_per_block": t.value}

    def preconditioner(self):
        """(effective preconditioner, coarse unknowns, coarse refactorisations so far)."""
        pc, nc, rf = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        capi.check(self._L.tf_get_preconditioner(self._h, ctypes.byref(pc), ctypes.byref(nc), ctypes.byref(rf)),
                   "tf_get_preconditioner", self._h)
        return pc.value, nc.value, rf.value

    def krylov_method(self) -> int:
        """Krylov method of the last call's solves: 1 BiCGStab, 2 CG, 3 CG that fell back to BiCGStab."""
        m = ctypes.c_int32()
        capi.check(self._L.tf_get_krylov_method(self._h, ctypes.byref(m)), "tf_get_krylov_method", self._h)
        return m.value

    def smoother_block(self) -> int:
        """Nodes per block of the block-Jacobi smoother (1: 3x3 node blocks; 3: a prism column of
        three nodes, 9x9)."""
        g = ctypes.c_int32()
        capi.check(self._L.tf_get_smoother_block(self._h, ctypes.byref(g)), "tf_get_smoother_block", self._h)
        return g.value

    def coarse_unknowns(self) -> int:
        return self.preconditioner()[1]

    def autotune(self, x_n, dt: float):
        capi.check(self._L.tf_autotune(self._h, capi.dptr(_f64(x_n).reshape(-1)), float(dt)), "tf_autotune", self._h)
        return self.schedule()

    def time_kernels(self, reps: int = 20):
        me, ms = ctypes.c_double(), ctypes.c_double()
        capi.check(self._L.tf_time_kernels(self._h, int(reps), ctypes.byref(me), ctypes.byref(ms)), "tf_time_kernels", self._h)
        return me.value, ms.value


class BatchSolver(NewtonRaphsonSolver):
    """Many independent tissues in one context (tf_batch_create): one element launch over all
    prisms, one persistent solve with a CTA group per tissue, per-tissue Newton convergence.
    Per-node / per-element arrays are the tissues' arrays concatenated in order."""

    def __init__(self, tissues, params: Optional[capi.Params] = None, **overrides):
        L = capi.load()
        self._L = L
        self.tissues = list(tissues)
        self.node0 = np.cumsum([0] + [t.n_nodes for t in self.tissues])
        self.elem0 = np.cumsum([0] + [t.n_elems for t in self.tissues])
        self.n_nodes = int(self.node0[-1])
        self.n_elems = int(self.elem0[-1])
        self.n_tissues = len(self.tissues)
        p = params if params is not None else capi.default_params()
        overrides.setdefault("newton_tol", self.tissues[0].newton_tol)
        for k, v in overrides.items():
            setattr(p, k, v)
        self.params = p
        self._keep = []
        descs = (capi.MeshDesc * self.n_tissues)()
        for i, t in enumerate(self.tissues):
            conn = np.ascontiguousarray(t.conn, dtype=np.int32)
            xref = _f64(t.xref)
            self._keep += [conn, xref]
            descs[i] = capi.MeshDesc(t.n_nodes, t.n_elems, capi.iptr(conn), capi.dptr(xref))
        h = ctypes.c_void_p()
        capi.check(L.tf_batch_create(self.n_tissues, descs, ctypes.byref(p), ctypes.byref(h)), "tf_batch_create")
        self._h = h
        self.conn = np.concatenate([t.conn + self.node0[i] for i, t in enumerate(self.tissues)]).astype(np.int32)
        self.last_stats = None
        cat = np.concatenate
        sm = [t.slave_master + 3 * self.node0[i] for i, t in enumerate(self.tissues) if t.slave_master.size]
        self.set_material(cat([t.lam for t in self.tissues]), cat([t.mu for t in self.tissues]),
                          cat([t.eta for t in self.tissues]))
        self.set_boundary(cat([t.fixed for t in self.tissues]), cat([t.ext_visc for t in self.tissues]),
                          cat(sm) if sm else None)
        self.set_growth(cat([t.fg for t in self.tissues]), cat([t.rates for t in self.tissues]),
                        cat([t.angles for t in self.tissues]), cat([t.exposed for t in self.tissues]),
                        cat([t.peripodial for t in self.tissues]))

    def join(self, xs):
        return np.concatenate([np.asarray(x, dtype=np.float64).reshape(-1, 3) for x in xs])

    def split(self, x):
        x = np.asarray(x).reshape(-1, 3)
        return [x[self.node0[i]:self.node0[i + 1]] for i in range(self.n_tissues)]

    def tissue_stats(self):
        it = np.zeros(self.n_tissues, np.int32)
        st = np.zeros(self.n_tissues, np.int32)
        kr = np.zeros(self.n_tissues, np.int32)
        self._L.tf_get_tissue_stats(self._h, capi.iptr(it), capi.iptr(st), capi.iptr(kr))
        return {"newton_iters": it, "status": st, "krylov_iters": kr}


def simulate(t: Tissue, n_steps: Optional[int] = None, solver: Optional[NewtonRaphsonSolver] = None, **overrides):
    """Run n time steps of the path on the GPU; returns (positions, per-step stats)."""
    own = solver is None
    s = solver or NewtonRaphsonSolver.from_tissue(t, **overrides)
    try:
        x = np.array(t.x, dtype=np.float64, copy=True)
        stats = []
        for _ in range(n_steps if n_steps is not None else t.n_steps):
            x, rc, st = s.runOneStep(x, t.dt)
            st["rc"] = rc
            stats.append(st)
        return x, stats
    finally:
        if own:
            s.close()
