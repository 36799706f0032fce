/*
 * tf_b200.h -- C ABI of the B200 implicit Newton-Raphson step for growing prism tissue.
 *
 * This is the drop-in boundary for TissueOrigami's Newton path
 * (TissueFolding/SourceCode: Simulation::updateStepNR -> NewtonRaphsonSolver ->
 * ShapeBase / Prism). Every entry point takes plain host pointers and sizes; no CUDA or
 * torch type appears in a signature. Each declaration names the reference interface it
 * replaces.
 *
 * Conventions
 *   - node DoF index is 3*node + dim, exactly the layout of NewtonRaphsonSolver::un / uk
 *     (NewtonRaphsonSolver.cpp:106-112).
 *   - prism node order is the reference's: 0-2 basal triangle, 3-5 apical triangle.
 *   - the Jacobian exposed by tf_assemble / tf_solve is the TRUE Newton Jacobian
 *     J = dR/du, which is the transpose of the reference's dense storage K: the reference
 *     writes the viscous tangent transposed (ShapeBase.cpp:3154-3160, 3193-3199) and asks
 *     Pardiso for a transposed solve (iparm[11] = 1, NewtonRaphsonSolver.cpp:716-723).
 *   - return value: 0 ok; > 0 numerical outcome the caller may continue from (the
 *     reference logs non-convergence and continues, Simulation.cpp:6724-6727); < 0 error.
 *     No entry point calls exit() or traps the GPU.
 *   - a context is used from one host thread at a time; its work runs on one CUDA stream.
 */
#ifndef TF_B200_H
#define TF_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------------------- */
#define TF_OK 0
#define TF_NEWTON_NOT_CONVERGED 1 /* hit the Newton cap; positions still updated          */
#define TF_KRYLOV_MAX_ITERS 2     /* a linear solve stopped at its iteration cap           */
#define TF_KRYLOV_BREAKDOWN 3     /* BiCGStab breakdown (rho or omega became zero)         */
#define TF_NONFINITE 4            /* NaN / Inf met in the residual or the update           */
#define TF_ELEMENT_INVERTED 5     /* det(Fe) <= 0 at some Gauss point                      */
#define TF_ERR_ARGUMENT (-1)
#define TF_ERR_CUDA (-2)
#define TF_ERR_OUT_OF_MEMORY (-3)
#define TF_ERR_STATE (-4)
#define TF_ERR_UNSUPPORTED (-5)
#define TF_ERR_TOO_LARGE (-6) /* system larger than tf_solve_bsr_noalloc's fixed scratch   */

/* Largest system (block rows) tf_solve_bsr_noalloc accepts. */
#define TF_NOALLOC_MAX_NODES 16384

/* ---- options ------------------------------------------------------------------------- */
#define TF_PRECOND_BLOCK_JACOBI 0 /* 3x3 node-block inverse of the diagonal               */
#define TF_PRECOND_ILU0 1         /* ILU(0) on the BSR3 pattern, multicolour ordered      */
#define TF_PRECOND_TWO_LEVEL 2    /* default: block-Jacobi + additive coarse correction on  */
                                  /* node-range aggregates with rigid-body modes, one coarse */
                                  /* operator per tissue; needs the persistent solve (a one- */
                                  /* tissue context with persistent = 0 uses block-Jacobi). */
                                  /* A tissue too large for one dense coarse operator (its   */
                                  /* aggregates would exceed 2048 nodes) takes the          */
                                  /* multilevel space below instead                         */
#define TF_PRECOND_MULTILEVEL 3   /* block-Jacobi + additive multilevel coarse correction:   */
                                  /* rigid-body modes of nested spatial sets (recursive      */
                                  /* bisection of the prism columns; leaves of ~16 columns,  */
                                  /* four sets per parent, a dense top of <= 160 sets), all  */
                                  /* rebuilt from every J; single tissue, persistent solve   */
                                  /* (a batch uses TF_PRECOND_TWO_LEVEL's space)             */

#define TF_KRYLOV_AUTO 0      /* conjugate gradients when J is symmetric (no internal     */
                              /* viscosity), else BiCGStab (persistent solve)             */
#define TF_KRYLOV_BICGSTAB 1  /* BiCGStab                                                 */
#define TF_KRYLOV_CG 2        /* preconditioned conjugate gradients; a tissue whose J turns */
                              /* out indefinite is solved again with BiCGStab              */

#define TF_SCATTER_AUTO 0     /* the autotuner's choice once tf_autotune ran, else ATOMIC */
#define TF_SCATTER_ATOMIC 1   /* FP64 atomics into the fixed BSR3 pattern                */
#define TF_SCATTER_COLOURED 2 /* greedy element colouring, plain read-modify-write       */
#define TF_SCATTER_STAGED 3   /* FP64 atomics from a shared-memory stage, one block's    */
                              /* entries on consecutive threads (fewer L2 sectors)       */

typedef struct tf_ctx tf_ctx;

/* Mesh handed over once per tissue: the reference's Nodes/Elements after
 * Simulation::initiateMesh (Simulation.cpp:2969-3014). */
typedef struct tf_mesh_desc {
    int32_t n_nodes;
    int32_t n_elems;
    const int32_t* conn; /* [n_elems*6]  ShapeBase::NodeIds                                  */
    const double* xref;  /* [n_elems*18] ReferenceShape->Positions (ReferenceShapeBase.h:21) */
} tf_mesh_desc;

typedef struct tf_params {
    int32_t max_newton_iters; /* Simulation.cpp:6615 maxIteration (20)                      */
    double newton_tol;        /* NewtonRaphsonSolver.cpp:22 threshold on ||du||_2 (1e-8)     */
    int32_t krylov_max_iters; /* BiCGStab iteration cap per linear solve                    */
    double krylov_rtol;       /* stop when ||r||_2 <= krylov_rtol * ||g||_2                 */
    int32_t precond;          /* TF_PRECOND_*                                               */
    int32_t scatter;          /* TF_SCATTER_*                                               */
    int32_t elems_per_block;  /* element-kernel teams per CTA: 0 = autotuned                */
    int32_t device;           /* CUDA device ordinal                                        */
    int32_t use_graphs;       /* capture the Krylov iteration in a CUDA graph (1) or not    */
    int32_t persistent;       /* whole solve in one cooperative persistent kernel (1) or    */
                              /* graph-replayed chunks of iteration kernels (0)             */
    int32_t smoother_nodes;   /* block-Jacobi block of the persistent solve: 0 = a prism    */
                              /* column of 2 or 3 nodes when the mesh numbers every column's */
                              /* nodes consecutively (in a batch: every tissue), else one   */
                              /* node; 1 = one node (3x3); 2-4 = that many consecutive nodes */
    int32_t krylov_refine;    /* tf_solve only: passes of iterative refinement after the      */
                              /* Krylov solve (FP64 residual g - J du, a second solve for the */
                              /* correction); 0 = none. The Newton loop needs none: each     */
                              /* Newton iteration corrects the previous one's solve error    */
    int32_t krylov_method;    /* TF_KRYLOV_*; the persistent solve only (the graph-replayed */
                              /* and allocation-free paths run BiCGStab)                    */
    int32_t krylov_warm_start; /* 1: in the Newton loop of a single tissue, conjugate       */
                              /* gradients start from the previous step's solution of the   */
                              /* same Newton iteration (x0, r0 = g - J x0; from zero if that */
                              /* residual is not below ||g||); 0: every solve from zero.    */
                              /* Same stopping rule either way; the adjoint runs cold       */
} tf_params;

typedef struct tf_step_stats {
    int32_t newton_iters;       /* iterations run (reference: iteratorK after the loop)     */
    int32_t krylov_iters_total; /* BiCGStab iterations summed over the step                 */
    int32_t krylov_iters_max;   /* largest single solve                                     */
    int32_t status;             /* worst status seen in the step                            */
    double du_norm[32];         /* ||du||_2 per Newton iteration (first 32)                 */
    double krylov_rel_res[32];  /* final relative residual of each linear solve             */
    double ms_assemble;         /* device time in assembly (element + node kernels)         */
    double ms_solve;            /* device time in the linear solves                         */
    double ms_total;            /* device time of the whole call, host copies included      */
    int64_t gpu_launches;       /* kernels this call launched (graph nodes counted)         */
    double ms_solve_kernel;     /* device time inside the persistent BiCGStab launches      */
    int32_t solve_launches;     /* number of those launches                                 */
    int32_t krylov_method;      /* 1 BiCGStab, 2 conjugate gradients, 3 CG fell back to     */
                                /* BiCGStab on some solve, 4 MINRES (a symmetric J with    */
                                /* packing pairs; block preconditioner |D|); the largest    */
                                /* over the call                                            */
    int32_t krylov_iters_cg;    /* the conjugate-gradient iterations in krylov_iters_total  */
                                /* (persistent solves; the rest are BiCGStab's)            */
} tf_step_stats;

/* Fill p with defaults: the reference's Newton cap (20) and threshold (1e-8), Krylov rtol
 * 1e-12 with cap 20000, the two-level preconditioner (TF_PRECOND_TWO_LEVEL), TF_SCATTER_AUTO,
 * device 0, graphs on, persistent solve on, smoother block chosen from the mesh, no refinement,
 * TF_KRYLOV_AUTO, warm starts on. */
void tf_default_params(tf_params* p);

/* Library version string. */
const char* tf_version(void);

/* Replaces NewtonRaphsonSolver::NewtonRaphsonSolver (NewtonRaphsonSolver.cpp:16-41) and the
 * per-element Prism::calculateElementShapeFunctionDerivatives (Prism.cpp:698-733): builds the
 * fixed BSR3 pattern, the element-to-block slot map and the element colouring on the host,
 * and allocates every device buffer of the tissue. */
int tf_create(const tf_mesh_desc* mesh, const tf_params* params, tf_ctx** out);

/* Batched mode (no single counterpart in the reference, which runs one tissue per process):
 * n_tissues independent tissues in one context. Tissue t's nodes and elements follow those of
 * tissue t-1 in every per-node / per-element array the other calls take (concatenated, node
 * ids of meshes[t].conn local to tissue t). Each tissue runs the reference's Newton loop on
 * its own - its own convergence test and cap - inside shared launches: one element-kernel
 * launch over all prisms, one persistent cooperative solve in which every tissue owns a group
 * of CTAs, per-tissue convergence flags that drop converged tissues from later iterations. */
int tf_batch_create(int32_t n_tissues, const tf_mesh_desc* meshes, const tf_params* params,
                    tf_ctx** out);

/* Per-tissue outcome of the last step of a batched (or single) context: Newton iterations,
 * status and BiCGStab iterations, each [n_tissues] (any may be NULL). */
int tf_get_tissue_stats(tf_ctx* ctx, int32_t* newton_iters, int32_t* status,
                        int32_t* krylov_iters);

/* Number of tissues of the context. */
int tf_get_n_tissues(tf_ctx* ctx);

/* Replaces NewtonRaphsonSolver::~NewtonRaphsonSolver (NewtonRaphsonSolver.cpp:43-71). */
void tf_destroy(tf_ctx* ctx);

/* Replaces Prism::setElasticProperties / updateElasticProperties (Prism.cpp:464-534) and
 * ShapeBase::internalViscosity: per-element lambda, mu, eta. */
int tf_set_material(tf_ctx* ctx, const double* lambda, const double* mu, const double* eta);

/* Replaces ShapeBase::InvFg as growShapeByFg leaves it (ShapeBase.cpp:1452-1506):
 * per-element inverse growth deformation gradient, [n_elems*9] row-major. */
int tf_set_inv_fg(tf_ctx* ctx, const double* inv_fg);

/* Replaces Node::FixedPos (Node.h), Node::externalViscosity (Node.cpp:63-110) and
 * NewtonRaphsonSolver::slaveMasterList (NewtonRaphsonSolver.h:49). fixed [n_nodes*3];
 * ext_visc [n_nodes*3]; slave_master [n_pairs*2] (slave DoF, master DoF). A master must not
 * itself be a slave (the reference enforces this in checkMasterUpdate). */
int tf_set_boundary(tf_ctx* ctx, const uint8_t* fixed, const double* ext_visc,
                    const int32_t* slave_master, int32_t n_pairs);

/* Replaces Node::viscositySurface as Simulation::updateNodeViscositySurfaces leaves it
 * (Simulation.cpp:7598-7620): per-node exposed area, [n_nodes]. */
int tf_set_viscosity_surface(tf_ctx* ctx, const double* visc_surface);

/* Replaces the external-force vector NewtonRaphsonSolver::gExt (NewtonRaphsonSolver.h:39) that
 * addExernalForces adds to the residual (NewtonRaphsonSolver.cpp:449-457): packing, pipette or
 * random forces the host computes, [n_nodes*3]; added on free DoFs, routed through slave-master
 * pairs like every force. Kept until replaced; NULL removes it. */
int tf_set_external_force(tf_ctx* ctx, const double* f);

/* One Newton iteration at the method level of NewtonRaphsonSolver: the sequence
 * calculateDisplacementMatrix ... calculateBoundKWithSlavesMasterDoF, solveForDeltaU
 * (NewtonRaphsonSolver.cpp:95-488; Simulation.cpp:6651-6716) on the device, from host positions
 * uk (iteration k) and un (end of the previous step), [n_nodes*3] each; du [n_nodes*3] receives
 * deltaU (slaves equal to their masters). The Jacobian never leaves the device. For hosts that keep
 * the reference's Newton loop (checkConvergenceViaDeltaU, updateUkInIteration) on the host.
 * iters / rel_res (may be NULL): BiCGStab iterations and final relative residual. */
int tf_newton_iteration(tf_ctx* ctx, const double* uk, const double* un, double dt, double* du, int32_t* iters,
                        double* rel_res);

/* Replaces Simulation::updateStepNR (Simulation.cpp:6605-6747) with the surface-based
 * external viscosity of NewtonRaphsonSolver (externalViscosityVolumeBased = false) and no
 * packing or lumen terms: x_n [n_nodes*3] host positions at the end of the previous step,
 * x_out [n_nodes*3] host positions after the step (may alias x_n). stats may be NULL. */
int tf_newton_step(tf_ctx* ctx, const double* x_n, double dt, double* x_out,
                   tf_step_stats* stats);

/* tf_newton_step on device-resident buffers (cudaMalloc'd by the caller, same layout), for
 * callers that keep positions on the GPU between steps. Stream-ordered on the context's
 * stream; returns after the step completed. */
int tf_newton_step_device(tf_ctx* ctx, const double* d_x_n, double dt, double* d_x_out,
                          tf_step_stats* stats);

/* Number of 3x3 blocks of the Jacobian pattern, and the pattern itself (rowptr [n_nodes+1],
 * colidx [nnzb], each may be NULL to query only). */
int tf_get_pattern(tf_ctx* ctx, int32_t* nnzb, int32_t* rowptr, int32_t* colidx);

/* Parity hook for one Newton iteration's system. Replaces the sequence
 * calculateDisplacementMatrix, calculateForcesAndJacobianMatrixNR,
 * writeForcesTogeAndgvInternal, writeImplicitElementalKToJacobian,
 * calculateExternalViscousForcesForNR, addImplicitKViscousExternalToJacobian,
 * calculateSumOfInternalForces, calcutateFixedK, calculateBoundKWithSlavesMasterDoF
 * (NewtonRaphsonSolver.cpp:95-457). uk, un [n_nodes*3]; g_out [n_nodes*3] is gSum;
 * bsr_vals_out [nnzb*9] (may be NULL) holds J = K^T block-row-major. */
int tf_assemble(tf_ctx* ctx, const double* uk, const double* un, double dt, double* g_out,
                double* bsr_vals_out);

/* Replaces NewtonRaphsonSolver::solveForDeltaU / solveWithPardiso
 * (NewtonRaphsonSolver.cpp:461-763) including equateSlaveDisplacementsToMasters: solves
 * J du = g with preconditioned BiCGStab on the context's pattern, followed by
 * params.krylov_refine passes of iterative refinement (Pardiso refines once, iparm[7] = 1).
 * bsr_vals [nnzb*9], g and du [n_nodes*3]. iters (BiCGStab iterations of every pass) and
 * rel_res (||g - J du|| / ||g|| of the result; with refinement the true residual) may be NULL. */
int tf_solve(tf_ctx* ctx, const double* bsr_vals, const double* g, double* du, int32_t* iters,
             double* rel_res);

/* Direct alternative to tf_solve, timed beside it: the same J du = g factorised and solved on
 * the GPU by cuSOLVER's sparse Cholesky (QR when Cholesky meets a non-positive pivot and the
 * system has at most 30,000 unknowns), the way the reference refactorises every system with
 * Pardiso (NewtonRaphsonSolver.cpp:498-763). ms_factor_solve receives the device time of
 * factorisation + solve, method 1 (Cholesky) or 2 (QR); either may be NULL. Returns
 * TF_KRYLOV_BREAKDOWN when the matrix is singular and TF_ERR_UNSUPPORTED when it is not positive
 * definite and larger than the QR limit. */
int tf_solve_direct(tf_ctx* ctx, const double* bsr_vals, const double* g, double* du,
                    double* ms_factor_solve, int32_t* method);

/* Growth state for the per-step prologue on the device: fg [n_elems*9] (ShapeBase::Fg),
 * rates [n_elems*3] growth rates in 1/s and angles [n_elems] in radians with the uniform
 * growth function's semantics (GrowthFunctionTypes.h:14-99, ShapeBase.cpp:471-505),
 * exposed [n_elems] bit0 apical / bit1 basal exposed surface and peripodial [n_elems]
 * (Prism.cpp:1650-1709). Any pointer may be NULL to keep the current value. */
int tf_set_growth(tf_ctx* ctx, const double* fg, const double* rates, const double* angles,
                  const uint8_t* exposed, const uint8_t* peripodial);

/* Read back the device growth state: fg and inv_fg [n_elems*9] (either may be NULL). */
int tf_get_growth(tf_ctx* ctx, double* fg, double* inv_fg);

/* One grid-based growth function (growth type 3, GridBasedGrowthFunction,
 * GrowthFunctionTypes.h:269-548), with the values the reference holds after reading its input
 * (ModelInputObject::readGrowthType3, ModelInputObject.cpp:684-866). */
typedef struct tf_grid_growth {
    double t0, t1;        /* active in steps that start at t with t0 <= t < t1 (InitialTime,    */
                          /* FinalTime; read into float by the reference)                       */
    int32_t nx, ny;       /* grid points (nGridX, nGridY), each >= 2                             */
    const double* rates;  /* [nx*ny*3] growth rate in 1/s of grid point (i, j), axis k at       */
                          /* (i*ny + j)*3 + k (GrowthMatrix: the file's per-hour values / 3600) */
    const double* angles; /* [nx*ny] orientation of grid point (i, j) in degrees, at i*ny + j    */
    double z_min, z_max;  /* zRange: applies where initialRelativePositionInZ is in the range    */
    int32_t flags;        /* bit0 ApplyToColumnarLayer, bit1 ApplyToPeripodialMembrane,          */
                          /* bit2 ApplyToBasalECM, bit3 ApplyToLateralECM                       */
    int32_t reserved;
} tf_grid_growth;

/* Replaces the grid-based branch of Simulation::calculateGrowth (calculateGrowthGridBased,
 * Simulation.cpp:9038-9085, with ShapeBase::calculateFgFromGridCorners, ShapeBase.cpp:513-658, and
 * convertRelativePosToGridIndex, :834-860) for grids pinned on the initial mesh
 * (GridGrowthsPinnedOnInitialMesh). In every time step the functions active at the context's
 * simulation time (tf_set_time; each tf_time_step advances it by dt) give each element an
 * increment - nearest grid corner (interpolation 0) or bilinear rates and orientation
 * (interpolation 1) - composed in list order after the uniform increment of tf_set_growth.
 * Per element: rel_pos [n_elems*2] the pinned position relative to the tissue's bounding box
 * (ShapeBase::initialRelativePosInBoundingBox), rel_z [n_elems] initialRelativePositionInZ
 * (0 apical, 1 basal), elem_flags [n_elems] bit0 ECM-mimicking, bit1 actin-mimicking (no growth
 * in height), bit2 basal placement, bit3 ECM at the circumference, bits 4-5 tissue type
 * (0 columnar, 1 peripodial). n_funcs = 0 removes the grid functions. At most 8 may be active
 * in one step (TF_ERR_UNSUPPORTED). */
int tf_set_grid_growth(tf_ctx* ctx, int32_t n_funcs, const tf_grid_growth* funcs, int32_t interpolation,
                       const double* rel_pos, const double* rel_z, const int32_t* elem_flags);

/* Simulation::currSimTimeSec: the time at the start of the next step (starts at 0); it selects the
 * grid growth functions of a step. tf_time_step and tf_time_step_device add dt to it. */
int tf_set_time(tf_ctx* ctx, double t);
int tf_get_time(tf_ctx* ctx, double* t);

/* One full time step of the path, replacing the part of Simulation::runOneStep that feeds
 * and runs the Newton step (Simulation.cpp:6008-6112): CalculateGrowthRotationByF,
 * calculateGrowth (uniform-type rates), growShapeByFg, updateNodeViscositySurfaces, then
 * updateStepNR. Host positions in and out. */
int tf_time_step(tf_ctx* ctx, const double* x_n, double dt, double* x_out,
                 tf_step_stats* stats);

/* tf_time_step on device-resident positions. */
int tf_time_step_device(tf_ctx* ctx, const double* d_x_n, double dt, double* d_x_out,
                        tf_step_stats* stats);

/* Number of element colours and the chosen scatter / teams-per-CTA after autotuning. */
int tf_get_schedule(tf_ctx* ctx, int32_t* n_colours, int32_t* scatter, int32_t* elems_per_block);

/* The preconditioner the context actually uses (TF_PRECOND_TWO_LEVEL stands down to
 * TF_PRECOND_BLOCK_JACOBI on the non-persistent path and reports TF_PRECOND_MULTILEVEL where it
 * took the multilevel space), the number of coarse unknowns of the
 * two-level space summed over the tissues (0 until the first solve, and 0 when a single tissue's
 * aggregates would be too large to help), and how many times the coarse operators have been
 * refactorised. */
int tf_get_preconditioner(tf_ctx* ctx, int32_t* precond, int32_t* n_coarse, int32_t* coarse_refreshes);

/* The Krylov method of the last call's linear solves (no counterpart in the reference, whose
 * Pardiso solve is direct): 1 BiCGStab, 2 conjugate gradients, 3 conjugate gradients that met a
 * non-positive curvature on some tissue, solved again by BiCGStab; 0 before any solve. */
int tf_get_krylov_method(tf_ctx* ctx, int32_t* method);

/* Nodes per block of the block-Jacobi smoother the context uses (1: 3x3 node blocks; G > 1:
 * the 3G x 3G diagonal sub-block of G consecutive nodes, a prism column). No counterpart in the
 * reference, whose Pardiso solve needs no smoother. */
int tf_get_smoother_block(tf_ctx* ctx, int32_t* nodes);

/* Time the assembly variants on the context's current state and keep the fastest
 * (scatter mode x teams per CTA). Returns the chosen pair through tf_get_schedule. */
int tf_autotune(tf_ctx* ctx, const double* x_n, double dt);

/* Benchmark hook (no reference counterpart): mean device time in ms over `reps` launches of
 * the element-assembly kernels of the current schedule, on the positions of the last call, and
 * of one BSR3 SpMV, each bracketed by CUDA events on the context's stream. Overwrites the
 * context's Jacobian buffers. */
int tf_time_kernels(tf_ctx* ctx, int32_t reps, double* ms_element, double* ms_spmv);

/* Discrete adjoint of the time loop (no reference counterpart; the reference has no gradients).
 * tf_adjoint_forward runs n_steps full time steps (tf_time_step) from host positions x0 and the
 * context's growth state, stores the positions and Fg every checkpoint_every steps on the device
 * and writes the final positions to x_final [n_nodes*3]. tf_adjoint_backward then takes
 * dL/dx_final [n_nodes*3] of a loss of the final positions and returns dL/d(growth rates)
 * [n_elems*3] (the rates of tf_set_growth, constant over the steps) and, if dL_dx0 is not
 * NULL, dL/dx0 [n_nodes*3] of the free degrees of freedom. Each segment between checkpoints
 * is recomputed forward; each step then costs one assembly at its converged state, one solve
 * with J^T (= J here) and hand-written element / node VJP kernels. Single tissue, no internal
 * viscosity, no slave-master pairs; the growth rotation is held at its forward value. The
 * growth state after tf_adjoint_backward is unspecified: set it again before the next run. */
int tf_adjoint_forward(tf_ctx* ctx, const double* x0, int32_t n_steps, double dt,
                       int32_t checkpoint_every, double* x_final, tf_step_stats* stats);
int tf_adjoint_backward(tf_ctx* ctx, const double* dL_dx_final, double* dL_drates, double* dL_dx0,
                        tf_step_stats* stats);

/* Measurement hook (no reference counterpart): FP64 FMA throughput of `device` in TFLOP/s (an FMA
 * counted as two flops), from one CUDA-event-timed launch of independent FMA chains that fill
 * every SM. The element kernel's own ceiling: its closed-form tangent is compute-bound. */
int tf_measure_fp64(int32_t device, double* tflops);

/* Lumen (Lumen.cpp, added to the Newton system at NewtonRaphsonSolver.cpp:242-249): the pressure
 * of the volume V = sum (1/6) (x3 x x1) . x2 enclosed by the apical triangles (element nodes 3,
 * 4, 5) of the n_elems listed elements (the reference's lumen elements: apical, or single-layer
 * elements spanning the tissue). The ideal volume V0 is V at positions x [N*3] (the constructor,
 * Lumen.cpp:11-68) and grows by exp(ln(growth_fold) / 86400 s x t) to the end of every step
 * (Lumen::growLumen; growth_fold <= 0: no growth). Every Newton iteration adds the forces
 * -bulk_modulus (V - V0) / V0 / (6 V0) x 6 dV/dx and the Jacobian of Lumen::calculateJacobian:
 * its triangle-local blocks in J, its rank-one part bulk / (36 V0^2) G G^T by a second Krylov
 * solve (Sherman-Morrison), so a step with a lumen costs two solves per Newton iteration.
 * n_elems = 0 removes the lumen. Single tissue, no slave-master pairs, persistent solve. */
int tf_set_lumen(tf_ctx* ctx, int32_t n_elems, const int32_t* elems, double bulk_modulus, double growth_fold,
                 const double* x);
/* The enclosed volume at the last assembly, the step's ideal volume, and G [N*3] (the nodal sums
 * of 6 dV/dx with fixed components zeroed; may be NULL). */
int tf_get_lumen(tf_ctx* ctx, double* volume, double* ideal_volume, double* G);

/* Packing (node-node contact): Simulation::detectPacingNodes (Simulation.cpp:7997-8153) after
 * every time step's growth, with the node masses of Simulation::updateNodeMasses (:7587-7596),
 * and in every Newton iteration the forces and Jacobian blocks of
 * Simulation::calculatePackingForcesImplicit3D / calculatePackingJacobian3D (:7307-7575):
 * pairs of apical (or basal) nodes that share no element and lie closer than 0.4 x the local
 * average element side, force 5000 m S(d) along the pair (m the pair's average mass, S a sigmoid
 * centred at 0.6 x packingThreshold). enabled != 0 turns it on with node_placement[N] (0 basal,
 * 1 apical, 2 other: never packs); tf_time_step / tf_time_step_device then detect the pairs of
 * each step on the device. Single tissue without slave-master pairs (TF_ERR_UNSUPPORTED
 * otherwise); while a step has pairs, tf_solve_direct returns TF_ERR_UNSUPPORTED; the adjoint
 * does not support packing. The two-level and multilevel coarse operators leave the pairs' blocks
 * outside the element pattern out (a preconditioner only); the solves include them. */
int tf_set_packing(tf_ctx* ctx, int32_t enabled, const int32_t* node_placement);
/* Detect the pairs at host positions x [N*3] with the current growth tensors (masses from them),
 * as the step prologue does; for hosts that run their own step loop (and for tests). */
int tf_detect_packing(tf_ctx* ctx, const double* x, int32_t* n_pairs);
/* The pairs of the last detection: their number, up to max_pairs pairs (i < j, the reference's
 * visiting order) in pairs[2*max_pairs], Simulation::packingThreshold, the node masses [N] and the
 * derivative blocks dF_i/dx_i [P][9] (row-major; the reference adds -D at (i, i), (j, j) and +D at
 * (i, j), (j, i)) of the last assembly. Any output may be NULL. */
int tf_get_packing(tf_ctx* ctx, int32_t max_pairs, int32_t* n_pairs, int32_t* pairs, double* threshold, double* mass,
                   double* dfdx);

/* Dense inverse utility (no reference counterpart): inverts `count` column-major n x n matrices
 * `a` of host memory in place on `device` with the Gauss-Jordan kernels that invert the two-level
 * preconditioner's coarse operators (partial pivoting; one CTA per matrix, or each matrix over a
 * cooperative grid when `cooperative` != 0). info[t] = 0, or k + 1 when step k of matrix t met a
 * zero or non-finite pivot (that matrix is then left partly eliminated). */
int tf_invert_dense(int32_t device, int32_t n, int32_t count, int32_t cooperative, double* a, int32_t* info);

/* Text of the last error recorded on the context (no reference counterpart); with ctx = NULL,
 * the reason the calling thread's last tf_create / tf_batch_create failed. */
const char* tf_last_error(tf_ctx* ctx);

/* No counterpart in the reference. The linear solve of tf_solve (block-Jacobi BiCGStab on
 * J du = g) for callers that cannot allocate GPU memory: hosts that give all device memory to
 * their own allocator or to a pool fixed at start-up, and therefore cannot let a library call
 * cudaMalloc / cudaFree. Every pointer is a DEVICE pointer the caller owns: the BSR3 pattern
 * (rowptr [n_nodes+1], colidx [nnzb] with the column indices of each row sorted ascending and
 * every row holding its diagonal block), the values vals [nnzb*9], the right-hand side g and
 * the solution du [n_nodes*3]. The work vectors live in one fixed __device__ array inside the
 * library (about 4.5 MB, held by every GPU where the library's kernels are loaded until the
 * process exits), so n_nodes may not exceed TF_NOALLOC_MAX_NODES; larger systems return
 * TF_ERR_TOO_LARGE before any GPU work. Every call looks up that array's address on the
 * current device with cudaGetSymbolAddress, which allocates nothing. Under CUDA's default lazy
 * module loading the array is reserved when the library's kernels first load on a device,
 * inside the first call there: a host whose pool takes all device memory makes one call of
 * this library on each device before the pool claims it (a reservation that fails returns
 * TF_ERR_OUT_OF_MEMORY). The call synchronises its stream every 32 iterations to poll
 * convergence, so it cannot be called while that stream is captured into a CUDA graph. Calls
 * share the array: ones that overlap on the GPU race, so serialise them. stream is a
 * cudaStream_t passed as a pointer (NULL: the legacy default stream); the call returns after
 * the solve has finished. The call makes no cudaMalloc, cudaFree or other allocating call.
 * Returns the status codes of tf_solve (TF_ERR_ARGUMENT when a row has no diagonal block);
 * iters / rel_res may be NULL. */
int tf_solve_bsr_noalloc(int32_t n_nodes, const int32_t* d_rowptr, const int32_t* d_colidx,
                         const double* d_vals, const double* d_g, double* d_du, double rtol,
                         int32_t max_iters, void* stream, int32_t* iters, double* rel_res);

#ifdef __cplusplus
}
#endif
#endif
