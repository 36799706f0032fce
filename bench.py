#!/usr/bin/env python
"""Benchmark of the implicit Newton-Raphson time step for growing prism tissue on B200.

Workload (default): the large slab - a 1000 x 500-node rectangle at 0.5 um spacing extruded into
3 layers (2,991,006 prisms, 2,000,000 nodes), log-normal stiffness per element, anisotropic growth
rotated by a smooth random angle field, 20 steps of dt = 60 s; the largest single-GPU workload.
`--workload wing_disc` runs the ~80k-prism disc, `small_rectangle` the 342-prism rectangle,
`batch` the 256 uneven tissues, `adjoint` the growth-map fit. One step = one full implicit time
step (growth prologue, viscosity surfaces, Newton iterations each with assembly + BiCGStab solve)
on synthetic seeded input.

Metric: prism assemblies/s = prisms x Newton assemblies / device time (FP64). Newton
iterations/s are reported beside it. `e2e` is the same metric through the public host-pointer
call tf_time_step, timed by the host clock around the call (host-to-device copy of the positions,
the step, device-to-host copy of the result).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload NAME]

Under torchrun (N > 1) every rank runs an independent replica of the tissue (the single-tissue
path does not shard); rank 0 prints one JSON line with the whole-job aggregate.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "prism assemblies/s (FP64 implicit Newton step)"
UNIT = "prisms*assemblies/s"


def make_tissue(name: str, slab_grid: str = "1000x500"):
    from tissueorigami_b200 import mesh

    if name == "wing_disc":
        return mesh.wing_disc()
    if name == "small_rectangle":
        return mesh.small_rectangle()
    if name == "large_slab":
        nx, ny = (int(v) for v in slab_grid.lower().split("x"))
        return mesh.large_slab(nx=nx, ny=ny)
    raise SystemExit(f"unknown workload {name}")


def workload_desc(t) -> dict:
    return {"workload": f"{t.name}: {t.n_elems} prisms, {t.n_nodes} nodes, dt={t.dt:g}s, "
                        f"Newton tol {t.newton_tol:g}", "prisms": t.n_elems, "nodes": t.n_nodes,
            "dt_s": t.dt, "seed": t.seed}


# ----------------------------------------------------------------------------------------
# CPU baseline: the oracle's line-by-line restatement of the reference element loop
# ----------------------------------------------------------------------------------------

def cpu_assembly_rate(t, seconds: float = 12.0):
    """Faithful element forces + tangents (the reference's naive D81 loop, OpenMP over
    elements with every host thread) on a bounded sample of the workload's prisms."""
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    sub = t.copy()
    n_cal = min(t.n_elems, 200 * threads)
    sub.conn = t.conn[:n_cal]
    sub.xref = t.xref[:n_cal]
    sub.lam, sub.mu, sub.eta = t.lam[:n_cal], t.mu[:n_cal], t.eta[:n_cal]
    t0 = time.perf_counter()
    O.element_forces_and_tangents(sub, t.x, threads=threads)
    rate0 = n_cal / (time.perf_counter() - t0)
    n = int(min(t.n_elems, max(n_cal, rate0 * seconds)))
    sub.conn, sub.xref = t.conn[:n], t.xref[:n]
    sub.lam, sub.mu, sub.eta = t.lam[:n], t.mu[:n], t.eta[:n]
    t0 = time.perf_counter()
    O.element_forces_and_tangents(sub, t.x, threads=threads)
    el = time.perf_counter() - t0
    return n / el, threads, n, el


def cpu_full_step_rate(t, threads=None):
    """One Newton iteration of the reference path on the CPU, assembly and direct solve together
    (the oracle's faithful element loop with CSR assembly and SuperLU in nested-dissection order
    standing in for Pardiso), at the first iteration of the workload's first step. Returns
    (prism assemblies/s, ms per Newton iteration, ms assembly, ms solve)."""
    from oracle import oracle as O

    threads = threads or os.cpu_count() or 1
    _, inv, _, _ = O.grow(t, t.x, t.fg)
    vs = O.viscosity_surfaces(t, t.x)
    rowptr, colidx = O.block_pattern(t)
    perm = O.nested_dissection(t, rowptr, colidx)
    t0 = time.perf_counter()
    vals, g = O.assemble_bsr(t, t.x, t.x, vs, inv, rowptr, colidx, threads=threads)
    t1 = time.perf_counter()
    O.sparse_direct_solve(O.bsr_to_scipy(rowptr, colidx, vals, t.n_nodes), g, perm)
    t2 = time.perf_counter()
    return t.n_elems / (t2 - t0), 1e3 * (t2 - t0), 1e3 * (t1 - t0), 1e3 * (t2 - t1)


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    t = make_tissue(args.workload, args.slab_grid)
    for _ in range(args.warmup):
        cpu_assembly_rate(t, seconds=1.0)
    rates, samples, secs = [], [], 0.0
    threads = os.cpu_count() or 1
    for _ in range(args.steps):
        r, threads, n, el = cpu_assembly_rate(t, seconds=args.ref_seconds)
        rates.append(r)
        samples.append(n)
        secs += el
    total_units = sum(samples)
    value = total_units / secs
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "config": workload_desc(t),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"faithful element forces + 18x18 tangents of the first {samples[0]} "
                                   f"of {t.n_elems} prisms per step (assembly only: the CPU path's "
                                   "direct solve is not included, which favours the CPU)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------------------
# clocks
# ----------------------------------------------------------------------------------------

class ClockSampler:
    QUERY = ("index,pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id=None):
        self.bus_id = bus_id
        self.proc = None
        self.lines = []

    def start(self):
        try:
            cmd = ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "200"]
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def _mine(self, bus: str) -> bool:
        """nvidia-smi lists every GPU of the host; keep the rows of the GPU this rank uses."""
        if not self.bus_id:
            return True
        a = bus.lower().split(":")
        b = self.bus_id.lower().split(":")
        return a[-2:] == b[-2:]

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in out.splitlines():
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 10 or not self._mine(f[1]):
                continue
            try:
                sm.append(float(f[2]))
                smax.append(float(f[3]))
            except ValueError:
                continue
            for nm, v in zip(names, f[6:10]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        mx = max(smax)
        loaded = [s for s in sm if s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------------------
# B200 arm
# ----------------------------------------------------------------------------------------

def run_b200(args) -> None:
    import ctypes

    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from tissueorigami_b200 import capi
    from tissueorigami_b200.newton import NewtonRaphsonSolver

    L = capi.load()
    t = make_tissue(args.workload, args.slab_grid)
    precond = {"block_jacobi": capi.TF_PRECOND_BLOCK_JACOBI, "ilu0": capi.TF_PRECOND_ILU0,
               "two_level": capi.TF_PRECOND_TWO_LEVEL, "multilevel": capi.TF_PRECOND_MULTILEVEL}[args.precond]
    s = NewtonRaphsonSolver.from_tissue(t, device=local, precond=precond, persistent=args.persistent,
                                        smoother_nodes=args.smoother_nodes, packing=bool(args.packing))
    sched = s.autotune(t.x, t.dt)
    sched["precond"] = args.precond
    sched["solve"] = {0: "graph-replayed iteration kernels", 1: "persistent cooperative kernel"}[args.persistent]
    n3 = 3 * t.n_nodes
    x_dev = torch.from_numpy(np.ascontiguousarray(t.x.reshape(-1))).to(f"cuda:{local}")
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")
    torch.cuda.synchronize()

    def dev_step():
        st = capi.StepStats()
        rc = L.tf_time_step_device(s._h, ctypes.c_void_p(x_dev.data_ptr()), float(t.dt),
                                   ctypes.c_void_p(x_dev.data_ptr()), ctypes.byref(st))
        capi.check(rc, "tf_time_step_device", s._h)
        return rc, st

    for _ in range(args.warmup):
        dev_step()

    bus = None
    try:
        p = torch.cuda.get_device_properties(local)
        bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
    except Exception:
        bus = None
    clocks = ClockSampler(bus)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    if args.profile_region:
        torch.cuda.cudart().cudaProfilerStart()
    ms, iters, kry, launches, worst = 0.0, 0, 0, 0, 0
    solve_ms, solve_launches, kry_cg, methods = 0.0, 0, 0, set()
    for _ in range(args.steps):
        flush.zero_()  # L2 flush between timed steps (outside the step's event window)
        torch.cuda.synchronize()
        rc, st = dev_step()
        ms += st.ms_total
        iters += st.newton_iters
        kry += st.krylov_iters_total
        launches += st.gpu_launches
        solve_ms += st.ms_solve_kernel
        solve_launches += st.solve_launches
        kry_cg += st.krylov_iters_cg
        methods.add(int(st.krylov_method))
        worst = max(worst, rc)
    torch.cuda.synchronize()
    if args.profile_region:
        torch.cuda.cudart().cudaProfilerStop()
    if dist:
        dist.barrier()
    clk = clocks.stop()

    # end to end through the public host-pointer call, pinned host buffers
    x_host = torch.from_numpy(x_dev.cpu().numpy().copy()).pin_memory()
    x_out = torch.empty_like(x_host).pin_memory()
    e2e_ms, e2e_iters = 0.0, 0
    p_in = ctypes.cast(x_host.data_ptr(), ctypes.POINTER(ctypes.c_double))
    p_out = ctypes.cast(x_out.data_ptr(), ctypes.POINTER(ctypes.c_double))
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        st = capi.StepStats()
        h0 = time.perf_counter()  # host clock around the public call: it returns with x_out filled
        rc = L.tf_time_step(s._h, p_in, float(t.dt), p_out, ctypes.byref(st))
        e2e_ms += 1e3 * (time.perf_counter() - h0)
        capi.check(rc, "tf_time_step", s._h)
        x_host.copy_(x_out)
        e2e_iters += st.newton_iters

    # the direct factorisation beside the Krylov solve, on the system at the current state
    nnz_scalar = 9 * int(s.pattern()[1].shape[0])
    if nnz_scalar <= 2e7:
        g_sys, vals_sys, _, _, _ = s.assemble(x_dev.cpu().numpy().reshape(-1, 3), x_dev.cpu().numpy().reshape(-1, 3),
                                              t.dt)
        try:
            _, rc_d, ms_direct, method = s.solve_direct(vals_sys, g_sys)
            direct = {"ms_factor_solve": ms_direct,
                      "method": {1: "cusolverSp Cholesky", 2: "cusolverSp QR"}.get(method), "status": rc_d,
                      "note": "cuDSS is unavailable on this box (not in the image); cuSOLVER sparse stands in"}
        except Exception as exc:  # reported, not fatal for the benchmark line
            direct = {"error": str(exc)[:200],
                      "note": "cuDSS is unavailable on this box (not in the image); cuSOLVER sparse stands in"}
    else:
        direct = {"skipped": f"{nnz_scalar} scalar non-zeros: beyond a single cusolverSp factorisation",
                  "note": "cuDSS is unavailable on this box (not in the image)"}
    direct["krylov_ms_per_solve"] = solve_ms / max(solve_launches, 1)

    # the preconditioner as built by the solves (two-level stands down to block-Jacobi when it cannot help)
    pc_eff, n_coarse, refreshes = s.preconditioner()
    sched["precond_effective"] = {0: "block_jacobi", 1: "ilu0", 2: "two_level", 3: "multilevel"}.get(pc_eff, pc_eff)
    sched["krylov_method"] = {1: "bicgstab", 2: "conjugate gradients",
                              3: "conjugate gradients, finished by bicgstab on indefinite solves",
                              4: "minres on steps with packing pairs"}.get(max(methods), "none")
    sched["krylov_iters_cg_share"] = kry_cg / max(kry, 1)
    # the reference detects node-node packing after every step's growth; the pairs it finds add
    # forces and Jacobian blocks to the Newton iterations
    sched["packing"] = ({"detection": "every step (device)", "pairs_last_step": int(len(s.packing()[0]))}
                        if args.packing else "off")
    sched["coarse_unknowns"] = n_coarse
    sched["coarse_refreshes"] = refreshes
    sched["smoother_block_nodes"] = s.smoother_block()

    # kernel timings for the roofline
    ms_el, ms_spmv = s.time_kernels(20)
    nnzb = int(s.pattern()[1].shape[0])
    E, N = t.n_elems, t.n_nodes
    bytes_asm = 408.0 * E + 97.0 * N + 72.0 * nnzb        # per assembly (element record, nodes, J written once)
    bytes_spmv = 76.0 * nnzb + 4.0 * (N + 1) + 48.0 * N    # per SpMV (J + colidx read once, x read, y written)
    share_el = ms_el * iters
    share_spmv = ms_spmv * 2 * kry
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    traffic = load_traffic()
    # the committed captures are of the default sizes: a reduced slab has no entry
    traffic_key = t.name if (t.name != "large_slab" or args.slab_grid == "1000x500") else None

    def roof(name, b, t_ms, iters=None):
        ach = b / (t_ms * 1e-3) / 1e9
        tr, tr_iters = traffic.get((name, traffic_key), (None, None))
        if tr is not None and tr_iters and iters:
            # a solve's DRAM traffic grows with its Krylov iterations: the capture's bytes per
            # launch scaled from its iteration count to this run's
            tr *= iters / tr_iters
        return {"kernel": name, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "peak_source": peak_src, "algorithmic_bytes": b, "ms_per_launch": t_ms, "traffic": tr}

    r_el = roof("element_assemble", bytes_asm, ms_el)
    r_sp = roof("bsr3_spmv", bytes_spmv, ms_spmv)
    # persistent solve: per BiCGStab iteration two SpMVs (each also reads one dot vector)
    # and three node-wise phases (p/phat: r,p,v,D -> p,phat; s/shat: r,v,D -> s,shat;
    # x/r: x,phat,shat,s,t,rhat -> x,r); plus one setup pass (diagonal inverses, r, rhat, p, v)
    # D^-1 is FP32, 36 G bytes per node with blocks of G nodes (a node's 3x3 inverse, or a prism
    # column's 3G x 3G inverse); with G > 1 it is set up by a separate kernel before the launch. Per conjugate-gradient iteration
    # one SpMV (plus the p re-read of its dot) and three node-wise phases (p = z + beta p:
    # z,p -> p; x += alpha p: x,p -> x; r -= alpha q, z = D^-1 r with (r,z), (r,r): r,q,D -> r,z
    # and the two dot vectors re-read).
    G = sched.get("smoother_block_nodes", 1)
    per_iter = 2.0 * (bytes_spmv + 24.0 * N) + N * (5 * 24 + 36 * G + 4 * 24 + 36 * G + 8 * 24)
    per_iter_cg = bytes_spmv + 24.0 * N + N * (3 * 24 + 3 * 24 + 4 * 24 + 36 * G + 2 * 24)
    per_setup = N * ((72.0 + 36 if G == 1 else 0.0) + 24 + 4 * 24)
    if sched.get("precond_effective") == "two_level" and sched.get("coarse_unknowns", 0) > 0:
        # two applications of the coarse correction per iteration, each reading the node modes
        # (d_i, mask) in the restriction and the prolongation and updating the preconditioned
        # vector once more; the coarse inverse is read once per solve into shared memory
        per_iter += 2.0 * N * (25 + 25 + 48)
        per_iter_cg += N * (25 + 25 + 48)
        per_setup += 8.0 * sched["coarse_unknowns"] ** 2
    if sched.get("precond_effective") == "multilevel":
        # per application: the node modes (d_i, mask) and the leaf node list in the restriction and
        # the prolongation, the preconditioned vector updated once more, the leaf inverses W_a
        # (288 bytes a leaf of ~64 nodes); the coarser levels and the top rows are below 1 %
        ml_app = N * (2 * (24 + 1 + 4) + 48 + 288.0 / 64)
        per_iter += 2.0 * ml_app
        per_iter_cg += ml_app
    kry_bi = kry - kry_cg
    if solve_launches > 0:
        bytes_solve = (kry_bi * per_iter + kry_cg * per_iter_cg + solve_launches * per_setup) / solve_launches
        r_solve = roof("bicgstab_persistent", bytes_solve, solve_ms / solve_launches, kry / solve_launches)
        r_solve["krylov_iterations_per_launch"] = kry / solve_launches
        r_solve["cg_iterations_per_launch"] = kry_cg / solve_launches
        # the element kernel's own bound is FP64, not HBM: the closed-form tangent costs ~15.2 k
        # flops per prism (counted from the kernel: ~640 per Gauss point for F, Fe, J, their
        # inverses and the spatial gradients, 648 for the nodal forces, ~85 per tangent block and
        # Gauss point for 21 blocks) against ~1.4 kB of algorithmic bytes
        flops_asm = 15200.0 * E
        fp64 = ctypes.c_double(0.0)
        if L.tf_measure_fp64(local, ctypes.byref(fp64)) == capi.TF_OK and fp64.value > 0:
            fp64_peak, fp64_src = fp64.value, "measured (FP64 FMA chains, tf_measure_fp64)"
        else:
            fp64_peak, fp64_src = 37.0, "nominal (measurement failed)"
        ach_fp64 = flops_asm / (ms_el * 1e-3) / 1e12
        r_el_fp64 = {"kernel": "element_assemble", "bound": "fp64", "achieved": ach_fp64, "peak": fp64_peak,
                     "unit": "TFLOP/s", "frac": ach_fp64 / fp64_peak, "peak_source": fp64_src,
                     "algorithmic_flops": flops_asm, "ms_per_launch": ms_el}
        dominant, other = r_solve, {"element_assemble": r_el, "element_assemble_fp64": r_el_fp64,
                                    "bsr3_spmv_standalone": r_sp}
    else:
        dominant, other = (r_sp, r_el) if share_spmv >= share_el else (r_el, r_sp)

    units = float(E) * iters
    t_dev = ms / 1000.0
    e2e_units = float(E) * e2e_iters
    t_e2e = e2e_ms / 1000.0
    if dist:
        buf = torch.tensor([units, e2e_units, float(iters), float(kry), float(launches)], dtype=torch.float64, device=f"cuda:{local}")
        tm = torch.tensor([t_dev, t_e2e], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(buf, op=dist.ReduceOp.SUM)
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        units, e2e_units, iters_all, kry_all, launches_all = buf.tolist()
        t_dev, t_e2e = tm.tolist()
    else:
        iters_all, kry_all, launches_all = iters, kry, launches

    cpu = None
    if rank == 0 and not args.no_cpu:
        r, threads, n, el = cpu_assembly_rate(t, seconds=args.cpu_seconds)
        cpu = {"value": r, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"faithful element forces + tangents of {n} of {t.n_elems} prisms "
                         f"({el:.1f} s on {threads} threads; assembly only)"}
        if t.n_nodes <= 100000:
            # a whole Newton iteration on the CPU: assembly + the direct solve standing in for Pardiso
            rf, ms_it, ms_a, ms_s = cpu_full_step_rate(t, threads)
            cpu["full_newton_iteration"] = {
                "value": rf, "unit": UNIT, "ms_per_newton_iteration": ms_it, "ms_assembly": ms_a,
                "ms_direct_solve": ms_s, "cores": threads,
                "sample": "one Newton iteration of the first step: faithful element loop + CSR assembly "
                          f"on {threads} threads, SuperLU (nested-dissection order, one thread)"}
        else:
            cpu["full_newton_iteration"] = {"skipped": "CPU per-assembly only: a sparse direct factorisation of "
                                                       f"{3 * t.n_nodes} unknowns does not fit the host"}
    if rank == 0:
        value = units / t_dev
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * t_dev / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded mesh and growth map)",
            "config": dict(workload_desc(t), l2="flushed (256 MB write) between timed steps",
                           parallelism=f"{world} independent replica(s), no collective on the data path",
                           schedule=sched),
            "newton_iters_per_s": iters_all / t_dev,
            "newton_iters_per_step": iters_all / (args.steps * world),
            "krylov_iters_per_newton": kry_all / max(iters_all, 1),
            "e2e": {"value": e2e_units / t_e2e, "unit": UNIT, "h2d_bytes_per_step": 8 * n3,
                    "d2h_bytes_per_step": 8 * n3},
            "gpu_launches": int(launches_all),
            "roofline": dominant, "roofline_other": other, "direct_solve_beside": direct,
            "cpu_baseline": cpu, "clocks": clk, "status_worst": worst,
        }
        print(json.dumps(line), flush=True)
    s.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_batch(args) -> None:
    """Batched uneven tissues: 256 discs / rectangles (500-20k prisms, log-uniform). One process
    per GPU: each rank runs its share of whole tissues (greedy bin packing on prisms x sqrt(nodes))
    as one batched context; no collective on the data path, time = max over ranks. At N = 1 the
    line also carries sequential single-tissue GPU runs of the same tissues."""
    import ctypes
    import datetime

    import torch

    from tissueorigami_b200 import capi, mesh
    from tissueorigami_b200.newton import BatchSolver, NewtonRaphsonSolver
    from tissueorigami_b200.sharding import ShardedBatch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    L = capi.load()
    ts = mesh.batch_tissues(n_tissues=args.n_tissues)
    E_all = float(sum(t.n_elems for t in ts))
    pc = {"block_jacobi": capi.TF_PRECOND_BLOCK_JACOBI, "ilu0": capi.TF_PRECOND_ILU0,
          "two_level": capi.TF_PRECOND_TWO_LEVEL}[args.precond]
    sb = ShardedBatch(ts, rank, world, lambda tl: BatchSolver(tl, device=local, precond=pc))
    b = sb.solver
    dev = f"cuda:{local}"
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    if b is not None:
        E_t = np.array([ts[i].n_elems for i in sb.mine], dtype=np.float64)
        x = torch.from_numpy(sb.initial_positions().reshape(-1).copy()).to(dev)
    torch.cuda.synchronize()

    def step():
        st = capi.StepStats()
        rc = L.tf_time_step_device(b._h, ctypes.c_void_p(x.data_ptr()), float(ts[0].dt), ctypes.c_void_p(x.data_ptr()),
                                   ctypes.byref(st))
        capi.check(rc, "tf_time_step_device", b._h)
        return rc, st

    if b is not None:
        for _ in range(args.warmup):
            step()
    clocks = ClockSampler(None)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms, units, launches, worst = 0.0, 0.0, 0, 0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        if b is None:
            continue
        rc, st = step()
        ts_stats = b.tissue_stats()
        units += float((E_t * ts_stats["newton_iters"]).sum())
        ms += st.ms_total
        launches += st.gpu_launches
        worst = max(worst, rc)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    pc_info = b.preconditioner() if b is not None else (pc, 0, 0)
    x_batch = b.split(x.cpu().numpy().reshape(-1, 3)) if b is not None else []
    sb.close()
    t_dev = ms / 1000.0
    if dist:
        tot = torch.tensor([units, float(launches), float(worst)], dtype=torch.float64, device=dev)
        tm = torch.tensor([t_dev], dtype=torch.float64, device=dev)
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        units, launches, worst = tot.tolist()
        t_dev = tm.item()
    seq = None
    if world == 1 and not args.no_sequential:
        # sequential baseline: the same tissues one after another, one context each, same steps
        # and the parity check of the batch against them: every tissue's positions after the same
        # steps, within 1e-9 of the tissue's size
        seq_ms, seq_units, worst_dev = 0.0, 0.0, 0.0
        for i, t in enumerate(ts):
            with NewtonRaphsonSolver.from_tissue(t, precond=pc) as s:
                xx = t.x.copy()
                for _ in range(args.warmup):
                    xx, _, _ = s.runOneStep(xx, t.dt)
                for _ in range(args.steps):
                    xx, _, st = s.runOneStep(xx, t.dt)
                    seq_ms += st["ms_total"]
                    seq_units += t.n_elems * st["newton_iters"]
            worst_dev = max(worst_dev, float(np.abs(x_batch[i] - xx).max()) / t.size)
        seq = {"value": seq_units / (seq_ms / 1000.0), "ms_per_step": seq_ms / args.steps,
               "tissue_steps_per_s": len(ts) * args.steps / (seq_ms / 1000.0),
               "max_position_difference_over_size": worst_dev, "positions_match_1e-9": worst_dev <= 1e-9}
    if rank == 0:
        line = {
            "metric": METRIC, "value": units / t_dev, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * t_dev / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded meshes and growth fields)",
            "config": {"workload": f"batch: {len(ts)} tissues, {int(E_all)} prisms, prism counts log-uniform 500-20000",
                       "l2": "flushed (256 MB write) between timed steps",
                       "parallelism": f"{world} rank(s), whole tissues per rank (greedy bin packing), "
                                      "no collective on the data path",
                       "tissues_per_rank": [len(s_) for s_ in sb.shards],
                       "precond": args.precond,
                       "precond_effective": {0: "block_jacobi", 1: "ilu0", 2: "two_level"}.get(pc_info[0], pc_info[0]),
                       "coarse_unknowns": pc_info[1], "coarse_refreshes": pc_info[2]},
            "tissue_steps_per_s": len(ts) * args.steps / t_dev,
            "gpu_launches": int(launches), "clocks": clk, "status_worst": int(worst),
        }
        if seq is not None:
            line["sequential"] = seq
            line["batch_speedup_vs_sequential"] = seq["ms_per_step"] / (1000.0 * t_dev / args.steps)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_adjoint(args) -> None:
    """Adjoint growth-map fit on the wing disc: per-element growth rates from a 32x32 bilinear
    grid (1024 parameters), loss = squared node-position misfit after 20 steps against the shape
    a seeded hidden grid produces, checkpoint every 5 steps. Reports the cost of one gradient
    (forward with checkpoints + adjoint backward) against one plain forward run."""
    from tissueorigami_b200 import capi, mesh
    from tissueorigami_b200.newton import NewtonRaphsonSolver

    t = mesh.wing_disc()
    n_steps, k, grid = 20, 5, 32
    idx, w = mesh.bilinear_growth_weights(t, grid)
    rng = np.random.default_rng(1004)
    gx, gy = np.meshgrid(np.linspace(t.x[:, 0].min(), t.x[:, 0].max(), grid),
                         np.linspace(t.x[:, 1].min(), t.x[:, 1].max(), grid), indexing="xy")
    rho2 = (gx ** 2 + gy ** 2).ravel()
    hidden = 2e-4 * np.exp(-rho2 / (2 * 40.0 ** 2)) * (1 + rng.uniform(-0.1, 0.1, grid * grid))
    theta = hidden * (1 + rng.uniform(-0.2, 0.2, grid * grid))

    def rates(p):
        r = (w * p[idx]).sum(axis=1)
        out = np.zeros((t.n_elems, 3))
        out[:, 0] = r
        out[:, 1] = r
        return out

    s = NewtonRaphsonSolver.from_tissue(t)
    s.set_growth(t.fg, rates(hidden), t.angles)
    target, rc, _ = s.adjoint_forward(t.x, n_steps, t.dt, k)
    fwd_ms, grad_ms, plain_ms, worst = [], [], [], rc
    for rep in range(args.warmup + args.steps):
        s.set_growth(t.fg, rates(theta), t.angles)
        x = t.x.copy()
        pm = 0.0
        for _ in range(n_steps):
            x, rc, st = s.runOneStep(x, t.dt)
            pm += st["ms_total"]
            worst = max(worst, rc)
        s.set_growth(t.fg, rates(theta), t.angles)
        xf, rc, stf = s.adjoint_forward(t.x, n_steps, t.dt, k)
        dr, _, rcb, stb = s.adjoint_backward(2 * (xf - target))
        worst = max(worst, rc, rcb)
        if rep >= args.warmup:
            plain_ms.append(pm)
            fwd_ms.append(stf["ms_total"])
            grad_ms.append(stf["ms_total"] + stb["ms_total"])
    s.close()
    dtheta = np.zeros(grid * grid)
    np.add.at(dtheta, idx.ravel(), (w * (dr[:, 0] + dr[:, 1])[:, None]).ravel())
    line = {
        "metric": "adjoint gradient cost / one forward run", "value": float(np.mean(grad_ms) / np.mean(plain_ms)),
        "unit": "x", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
        "dtype": "f64", "data": "synthetic (seeded disc, hidden and current 32x32 growth grids)",
        "config": {"workload": f"adjoint fit: wing_disc {t.n_elems} prisms, 1024 grid parameters, {n_steps} steps, "
                               f"checkpoint every {k}"},
        "ms_plain_forward": float(np.mean(plain_ms)), "ms_forward_with_checkpoints": float(np.mean(fwd_ms)),
        "ms_gradient": float(np.mean(grad_ms)), "grad_norm": float(np.linalg.norm(dtheta)),
        "status_worst": int(worst),
    }
    print(json.dumps(line), flush=True)


def load_traffic():
    """Per-launch DRAM bytes from committed ncu summaries (profiles/traffic.tsv:
    kernel<TAB>workload<TAB>bytes_per_launch[<TAB>Krylov iterations per launch of the capture]);
    missing entries read as null. Returns {(kernel, workload): (bytes, iterations or None)}."""
    out = {}
    p = os.path.join(ROOT, "profiles", "traffic.tsv")
    if os.path.exists(p):
        for ln in open(p):
            f = ln.strip().split("\t")
            if len(f) >= 3 and not ln.startswith("#"):
                try:
                    out[(f[0], f[1])] = (float(f[2]), float(f[3]) if len(f) >= 4 else None)
                except ValueError:
                    pass
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", default="large_slab",
                    choices=["large_slab", "wing_disc", "small_rectangle", "batch", "adjoint"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="CPU assembly sample of the cpu_baseline leg (seconds)")
    ap.add_argument("--ref-seconds", type=float, default=4.0,
                    help="CPU assembly sample per step of the reference arm (seconds)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--packing", type=int, choices=[0, 1], default=1,
                    help="node-node packing detection every step and its terms (the reference's default)")
    ap.add_argument("--slab-grid", default="1000x500",
                    help="in-plane points of the large_slab workload (a smaller slab for ncu captures)")
    ap.add_argument("--smoother-nodes", type=int, choices=[0, 1, 2, 3, 4], default=0,
                    help="block-Jacobi block of a single tissue: 0 = a prism column when the mesh "
                         "numbers it consecutively, 1 = one node")
    ap.add_argument("--no-sequential", action="store_true",
                    help="batch workload: skip the sequential single-tissue comparison (profiling runs)")
    ap.add_argument("--n-tissues", type=int, default=256, help="tissues of the batch workload")
    ap.add_argument("--precond", choices=["block_jacobi", "ilu0", "two_level", "multilevel"], default="two_level",
                    help="Krylov preconditioner of the single-tissue workloads")
    ap.add_argument("--persistent", type=int, choices=[0, 1], default=1,
                    help="solve path of the single-tissue workloads (tf_params.persistent)")
    ap.add_argument("--profile-region", action="store_true",
                    help="bracket the timed steps with cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "adjoint":
        run_adjoint(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
