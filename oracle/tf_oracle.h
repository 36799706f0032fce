/*
 * tf_oracle.h -- CPU restatement of TissueOrigami's implicit Newton-Raphson step
 * for 6-node prism tissue.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the parity checker for the CUDA path
 * in tissueorigami_b200 and the timed CPU baseline of bench.py. Nothing in the
 * product links or calls it. It restates, in plain C++ without GSL, the reference
 * algorithm (TissueFolding/SourceCode, cited per function in tf_oracle.cpp):
 *   - Prism shape-function derivatives and Gauss points  (Prism.cpp:97-130, 597-733)
 *   - element forces, neo-Hookean stress, B matrices     (Prism.cpp:766-888, ShapeBase.cpp:2356-2845)
 *   - elastic tangent as the literal 10-deep D81 loop      (ShapeBase.cpp:2846-2866, 3010-3095)
 *   - viscous tangent, written transposed                  (ShapeBase.cpp:2868-2933, 3097-3209)
 *   - dense scatter, external drag, fixed DoF, slave-master elimination
 *                                                          (NewtonRaphsonSolver.cpp:95-457)
 *   - dense->CSR scan with the 1e-13 drop and the transposed solve that Pardiso does
 *                                                          (NewtonRaphsonSolver.cpp:461-804)
 *   - the Newton loop of Simulation::updateStepNR          (Simulation.cpp:6605-6747)
 *   - the per-step growth prologue                         (ShapeBase.cpp:471-505, 764-787, 1452-1506, 1914-2041)
 *   - exposed-surface drag areas                           (Prism.cpp:1485-1556, ShapeBase.cpp:3749-3776)
 *
 * Array conventions (all row-major, 0-based):
 *   x[N*3]            node positions, DoF index 3*node+dim (the reference's un/uk layout)
 *   conn[E*6]         prism node ids; 0-2 basal triangle, 3-5 apical triangle
 *   xref[E*18]        ReferenceShape->Positions per element, [node][dim]
 *   fixed[N*3]        Node::FixedPos
 *   K[(3N)*(3N)]      the reference's dense Jacobian storage (NewtonRaphsonSolver::K)
 */
#ifndef TF_ORACLE_H
#define TF_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Gauss-point shape data from the reference shape: InvdXdes[6][3][3] and detdXdes[6]
 * per element (Prism::calculateElementShapeFunctionDerivatives, Prism.cpp:698-733). */
void tfo_shape_derivatives(int n_elems, const double* xref, double* inv_dxde, double* det_dxde);

/* Per-element forces and 18x18 tangents (ShapeBase::calculateForces3D,
 * calculateImplicitKElastic, calculateImplicitKViscous). Outputs, per element:
 *   f_elastic[18]  ElementalElasticSystemForces (already negated, fixed DoFs left 0)
 *   f_viscous[18]  ElementalInternalViscousSystemForces
 *   ke[324], kv[324] TriPointKe / TriPointKv in the reference's storage
 *   strain[36]     Green strain per Gauss point in Voigt order (may be NULL)
 * Returns the number of elements whose detFe <= 0 (the reference prints a NaN warning). */
int tfo_element_forces_and_tangents(int n_elems, const int32_t* conn, const double* xref,
                                    const double* inv_fg, const double* lam, const double* mu,
                                    const double* eta, const double* x, const double* disp_per_dt,
                                    double dt, const uint8_t* fixed, double* f_elastic,
                                    double* f_viscous, double* ke, double* kv, double* strain,
                                    int n_threads);

/* One Newton iteration's dense system in reference storage: zero, element loop, scatter
 * (viscous then elastic), external drag, sum, fixed DoF, slave-master binding
 * (NewtonRaphsonSolver.cpp:95-457, Simulation.cpp:6651-6712). slave_master holds n_pairs
 * (slave DoF, master DoF) couples. K is (3N)^2 doubles, g is 3N. */
int tfo_assemble_dense(int n_nodes, int n_elems, const int32_t* conn, const double* xref,
                       const double* inv_fg, const double* lam, const double* mu,
                       const double* eta, const double* uk, const double* un, double dt,
                       const uint8_t* fixed, const double* visc_surface, const double* ext_visc,
                       const int32_t* slave_master, int n_pairs, double* K, double* g,
                       int n_threads);

/* Pardiso stand-in: drop |K_ij| <= 1e-13 (constructiaForPardiso), solve K^T du = g by
 * LU with partial pivoting plus n_refine steps of iterative refinement (iparm[7]=1),
 * then copy master displacements to slaves (equateSlaveDisplacementsToMasters).
 * Returns 0, or 1 if a zero pivot was met. */
int tfo_solve_transposed(int n, const double* K, const double* g, const int32_t* slave_master,
                         int n_pairs, int n_refine, double* du);

/* Simulation::updateStepNR with the dense path above. Positions x_n -> x_out.
 * Iteration cap semantics follow the reference: the loop stops once
 * ||du||_2 <= tol, or when more than max_iter iterations ran without convergence.
 * norms[] receives ||du||_2 per iteration (capacity max_iter+2). Returns iterations run. */
int tfo_newton_step_dense(int n_nodes, int n_elems, const int32_t* conn, const double* xref,
                          const double* inv_fg, const double* lam, const double* mu,
                          const double* eta, const double* x_n, double dt, double tol,
                          int max_iter, const uint8_t* fixed, const double* visc_surface,
                          const double* ext_visc, const int32_t* slave_master, int n_pairs,
                          double* x_out, double* norms, int n_threads);

/* Block (3x3) sparsity pattern of the Jacobian: block (A,B) present when nodes A and B
 * share an element, plus every node's diagonal block. rowptr[N+1]; colidx sorted per row.
 * Call once with colidx == NULL to get nnzb (return value), then again to fill. */
int tfo_block_pattern(int n_nodes, int n_elems, const int32_t* conn, int32_t* rowptr,
                      int32_t* colidx);

/* Sparse assembly of the TRUE Jacobian J = K^T (the matrix Pardiso's transposed solve
 * uses) into BSR3 values over the pattern from tfo_block_pattern, with g, drag, fixed DoF
 * (row/column identity) but no slave-master pairs. Same element math as the dense path,
 * serial scatter after an OpenMP element loop, as NewtonRaphsonSolver.cpp:221-360 does.
 * vals has nnzb*9 doubles, block-row-major. */
int tfo_assemble_bsr(int n_nodes, int n_elems, const int32_t* conn, const double* xref,
                     const double* inv_fg, const double* lam, const double* mu, const double* eta,
                     const double* uk, const double* un, double dt, const uint8_t* fixed,
                     const double* visc_surface, const double* ext_visc, const int32_t* rowptr,
                     const int32_t* colidx, double* vals, double* g, int n_threads);

/* Growth prologue for one time step (Simulation::runOneStep 6008-6058):
 * CalculateGrowthRotationByF from current positions (ShapeBase.cpp:1914-2041),
 * uniform-type growth increment R(angle) diag(exp(r*dt)) R(angle)^T
 * (ShapeBase.cpp:471-505, GrowthFunctionTypes.h:22-40), updateGrowthIncrement
 * (ShapeBase.cpp:764-787) and growShapeByFg (ShapeBase.cpp:1452-1506).
 * fg[E*9] is updated in place; inv_fg[E*9] and grown_volume factor det(Fg) are written.
 * rotated[E] (may be NULL) receives the rotatedGrowth flag. */
void tfo_grow(int n_elems, const int32_t* conn, const double* xref, const double* x,
              const double* rates, const double* angles, double dt, double* fg, double* inv_fg,
              double* det_fg, int32_t* rotated, const double* grid_inc);

/* Growth increments of the grid-based growth functions (type 3) active at time t
 * (Simulation::calculateGrowthGridBased, Simulation.cpp:9038-9085; GridBasedGrowthFunction,
 * GrowthFunctionTypes.h:269-548; ShapeBase::calculateFgFromGridCorners, ShapeBase.cpp:513-658;
 * convertRelativePosToGridIndex :834-860; updateGrowthIncrement :764-787), composed in function
 * order into inc[E*9] (identity where none applies). Per function f: dims[2f..] = (nGridX, nGridY),
 * rates (1/s) and angles_deg (degrees, as read from the grid file) at grid point (i, j) at
 * offset i*nGridY + j of the function's block (blocks concatenated), windows[2f..] = [t0, t1),
 * zrange[2f..] = (zMin, zMax), fflags[f] bit0 columnar, bit1 peripodial, bit2 basal ECM, bit3
 * lateral ECM. interpolation 0 = nearest corner, 1 = bilinear. Per element: rel_pos[E*2] the
 * (pinned) relative position in the bounding box, rel_z[E] initialRelativePositionInZ,
 * eflags[E] bit0 ECM-mimicking, bit1 actin-mimicking, bit2 basal placement, bit3 ECM at the
 * circumference, bits 4-5 tissue type (0 columnar, 1 peripodial). tfo_grow applies inc after
 * the uniform increment. per_func[F*E*10] (may be NULL) receives, per function and element,
 * 1 when calculateFgFromGridCorners passed its applicability test (the reference then prints the
 * increment's diagonal) and that function's own increment (9 doubles). */
void tfo_grid_growth_increments(int n_elems, int n_funcs, const int32_t* dims, const double* rates,
                                const double* angles_deg, const double* windows, const double* zrange,
                                const int32_t* fflags, int interpolation, const double* rel_pos,
                                const double* rel_z, const int32_t* eflags, double t, double dt, double* inc,
                                double* per_func);

/* Node viscosity surfaces (Simulation::updateNodeViscositySurfaces, Sim.cpp:7598-7620):
 * exposed[E] bit0 = exposed apical surface, bit1 = exposed basal surface,
 * peripodial[E] = 1 swaps apical/basal node triples (Prism.cpp:1485-1556). */
void tfo_viscosity_surfaces(int n_nodes, int n_elems, const int32_t* conn, const double* x,
                            const uint8_t* exposed, const uint8_t* peripodial,
                            double* visc_surface);

/* Node-node packing candidates of one time step (Simulation::detectPacingNodes,
 * Simulation.cpp:7997-8153, with getAverageSideLength :3197-3262 and
 * Node::checkIfNodeHasPacking, Node.cpp:128-146): apical/basal nodes of the same placement that
 * share no element and lie closer than 0.4 x the average side length of the threshold grid
 * cell of the first node. node_placement[N] (0 basal, 1 apical, 2 midline), exposed[E] as in
 * tfo_viscosity_surfaces. Returns the number of pairs and writes up to max_pairs of them,
 * (i, j) with i < j in the reference's visiting order, to pairs[2*max_pairs] (may be NULL);
 * packing_threshold (may be NULL) receives Simulation::packingThreshold = 0.4 x the columnar
 * average side length. */
int tfo_detect_packing(int n_nodes, int n_elems, const int32_t* conn, const double* x,
                       const int32_t* node_placement, const uint8_t* exposed, const uint8_t* peripodial,
                       int max_pairs, int32_t* pairs, double* packing_threshold);

/* Node masses of one step (Simulation::updateNodeMasses, Simulation.cpp:7587-7596): every node
 * collects det(Fg) x the element's reference volume / 6 from each of its elements. */
void tfo_node_masses(int n_nodes, int n_elems, const int32_t* conn, const double* xref, const double* fg,
                     double* mass);

/* Packing forces (added to forces[3N], may be NULL) and the 3 x 3 derivative blocks dfdx[P][9] of
 * the pairs of one step at positions x (Simulation::calculatePackingForcesImplicit3D and
 * calculatePackingJacobian3D, Simulation.cpp:7307-7575); thr = Simulation::packingThreshold. */
void tfo_packing_terms(int n_pairs, const int32_t* pairs, const double* x, const double* mass, double thr,
                       double* forces, double* dfdx);

/* Lumen (Lumen.cpp): the enclosed volume of the triangles tri[3t..3t+2] (apical nodes of the
 * lumen elements), and at positions x with ideal volume `ideal` the pressure forces (added to
 * forces[3N], free DoFs) and the Jacobian (added to the dense reference-storage K[3N][3N]). */
double tfo_lumen_volume(int n_tri, const int32_t* tri, const double* x);
void tfo_lumen_terms(int n_nodes, int n_tri, const int32_t* tri, const double* x, const uint8_t* fixed,
                     double bulk, double ideal, double* forces, double* K);

#ifdef __cplusplus
}
#endif
#endif
