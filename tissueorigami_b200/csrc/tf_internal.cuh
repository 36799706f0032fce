// tf_internal.cuh -- device data model and kernel entry points of the B200 Newton step.
//
// Layout in HBM (one tissue):
//   nodes     : positions uk / un / x_out as [N][3] doubles (DoF 3*node+dim, gathered by
//               elements), fixed mask [N] (bit d = FixedPos[d]), drag coefficient inputs.
//   elements  : one 416-byte record per prism (ElemRecord) in the mesh's own order, so a team
//               of threads reads a whole record with a few coalesced loads whether it is
//               reached directly (atomic scatter) or through the colour permutation.
//   Jacobian  : BSR3 - rowptr [N+1], colidx [nnzb], vals [nnzb][3][3] row-major blocks.
//   Krylov    : eight [N][3] work vectors + the 3x3 inverse diagonal [N][9].
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tfb {

// One prism, 416 bytes (13 x 32-byte sectors). slots[a*6+b] is the BSR block index of
// block (conn[a], conn[b]) in block row conn[a]; -1 for elements that touch a slave DoF
// (those take the routed slow path).
struct __align__(16) ElemRecord {
    int32_t conn[6];
    int32_t slots[36];
    int32_t flags;   // bit0: element touches a slave DoF (slave-master routing needed)
    int32_t tissue;  // tissue of a batched context (0 for a single tissue)
    double xref[18];
    double inv_fg[9];
    double lam, mu, eta;
};
static_assert(sizeof(ElemRecord) == 416, "element record must stay 416 bytes");

constexpr int kElemWords = sizeof(ElemRecord) / 8;  // 52 doubles

// Device scalars of one BiCGStab solve. All updates happen on the device; the host only
// polls `status` between chunks of iterations.
struct KrylovScalars {
    double rho_prev, rho, alpha, omega;
    double bb, rr, tol2, du2;
    int32_t iter, max_iter, status, method;  // method: the Krylov method that produced the result (KM_*)
    uint32_t ticket[6];
    int32_t pad[2];
};

enum KrylovMethod : int32_t {
    KM_BICGSTAB = 1,     // BiCGStab
    KM_CG = 2,           // preconditioned conjugate gradients (symmetric J)
    KM_CG_FALLBACK = 3,  // CG met a non-positive curvature; BiCGStab solved the system
    KM_MINRES = 4,       // MINRES with the |D| block preconditioner (symmetric J with packing pairs)
};

enum KrylovStatus : int32_t {
    KS_RUNNING = 0,
    KS_CONVERGED = 1,
    KS_MAXIT = 2,
    KS_BREAKDOWN = 3,
    KS_NONFINITE = 4,
    KS_INDEFINITE = 5,  // conjugate gradients met (p, J p) <= 0 or (r, M^-1 r) <= 0
};

// Device-side error / outcome bits written by kernels.
enum DeviceFlags : int32_t {
    DF_INVERTED = 1,      // det(Fe) <= 0 somewhere
    DF_NONFINITE = 2,     // non-finite value produced
    DF_PATTERN_MISS = 4,  // routed entry had no block in the pattern (never expected)
    DF_SINGULAR_DIAG = 8,   // a diagonal 3x3 block was singular
    DF_BARRIER_TIMEOUT = 16 // a persistent kernel's grid barrier gave up waiting
};

// Generation-counting grid barrier state of a cooperative launch (zero-initialised).
struct GridBarrier {
    uint32_t count;
    uint32_t gen;
};

struct AssembleArgs {
    const ElemRecord* elems;
    const int32_t* elem_list;  // NULL: element i of the launch is elems[e_begin+i]
    int32_t e_begin, e_count;
    const double* uk;          // [N][3]
    const double* un;          // [N][3]
    double inv_dt;
    const uint8_t* fixmask;    // [N]
    const int32_t* dofmap;     // [3N] routed DoF (identity when no binding)
    const int32_t* rowptr;
    const int32_t* colidx;
    double* vals;              // [nnzb][9]
    double* g;                 // [3N]
    int32_t* dflags;
    const int32_t* tissue_active;  // [T] 0 = converged tissue, skip (NULL: all active)
};

struct NodeArgs {
    int32_t n_nodes;
    const double* uk;
    const double* un;
    double dt;
    const uint8_t* fixmask;
    const double* ext_visc;      // [3N]
    const double* visc_surface;  // [N]
    const double* ext_force;     // [3N] external forces added to g (gExt of the reference), or NULL
    const int32_t* dofmap;
    const int32_t* diag;         // [N] slot of the diagonal block
    const int32_t* rowptr;
    const int32_t* colidx;
    double* vals;
    double* g;
    int32_t* dflags;
    const int32_t* node_tissue;    // [N] tissue of each node
    const int32_t* tissue_active;  // [T] (NULL: all active)
};

constexpr int kMlMaxLevels = 10;  // levels of the multilevel coarse space (leaves .. top)

// CTA plan of the batched persistent solve: tissue t owns CTAs [cta0[t], cta0[t]+ncta[t]) and
// node rows [row0[t], row0[t+1]); each tissue has its own barrier, scalars and partials
// (4 doubles per CTA of the tissue, starting at 4*cta0[t]).
struct BatchPlan {
    int32_t n_tissues;
    int32_t n_cta;
    const int32_t* cta_list_ptr; // [n_cta+1] tissues of each CTA in cta_list: one for a CTA of a
    const int32_t* cta_list;     //   multi-CTA group, several small tissues for a packing CTA
    const int32_t* cta0;         // [T]
    const int32_t* ncta;         // [T]
    const int32_t* row0;         // [T+1]
    const int32_t* active;       // [T]
    // smoother block of the persistent solve: G consecutive nodes (a prism column when the mesh
    // numbers a column's nodes consecutively; a batch's tissues share G, and their aggregates'
    // node lists hold whole groups). G = 1: the node's 3x3 inverse in dinv [N][9]; G > 1: the
    // inverse of the 3G x 3G diagonal sub-block of group g in FP32, column-major at
    // (float*)dinv + g (3G)^2, computed before the launch and applied one DoF per lane; row
    // ranges and aggregates hold whole groups.
    int32_t group;
    // conjugate gradients instead of BiCGStab (every tissue's J symmetric: no internal viscosity);
    // a tissue whose CG ends with KS_INDEFINITE is solved again by a BiCGStab launch
    int32_t cg;
    // BiCGStab starts from the iterate x and residual r already in the work vectors (those that
    // conjugate gradients left when it met a non-positive curvature) instead of x = 0, r = b
    int32_t warm;
    // MINRES instead (symmetric J that packing pairs make indefinite; block preconditioner only)
    int32_t minres;
    // tissues solved by one CTA each (the packing CTAs' tissues), heaviest first: once its group
    // tissue (if any) is solved, every CTA takes the next one (atomic ticket in queue_head, zeroed
    // before each launch), so these tissues are spread over the CTAs as they become free
    const int32_t* queue;        // [n_queue]
    int32_t n_queue;
    int32_t* queue_head;
    GridBarrier* barriers;       // [T]
    KrylovScalars* scalars;      // [T]
    double* du2;                 // [T] ||du||^2 of the last Newton update
    // two-level preconditioner of a single tissue (agg_per_cta = 0: block-Jacobi only). Each
    // CTA's rows [r0, r1) split into agg_per_cta aggregates [r0 + L k / m, r0 + L (k+1) / m);
    // aggregate a (CTA lc, local k: a = lc m + k) owns coarse unknowns 6a .. 6a+5.
    // The modes of node i in aggregate a are P_i = mask_i o (B_i M_a), B_i = [I | (d_i x)]
    // (translations, rotations about the aggregate centroid, d_i = X_i - centroid), mask_i the
    // node's free DoFs (bit d), M_a a 6x6 orthonormalising transform (dropped modes: zero columns).
    int32_t agg_per_cta;
    int32_t n_coarse;            // 6 x aggregates
    const double* node_d;        // [N][3] d_i
    const uint8_t* node_mask;    // [N]
    const double* agg_m;         // [aggregates][6][6] M_a, row-major
    const double* coarse_inv;    // [n_coarse][n_coarse] row-major inverse of P^T J P (read once per solve)
    double* coarse_r;            // [n_coarse] restricted vector
    // two-level preconditioner of a batch (batch_coarse = 1; agg_per_cta = 0): every tissue has
    // fixed aggregates, spatial node sets (recursive coordinate bisection) listed in agg_nodes
    // [agg_ptr[a], agg_ptr[a+1]); CTA lc of tissue t's group of nct CTAs applies the
    // preconditioner on the aggregates [a0 + na lc / nct, a0 + na (lc + 1) / nct) of the tissue's
    // na (its SpMV and vector rows stay the contiguous row range). Aggregate a (global numbering)
    // owns coarse unknowns 6a .. 6a+5 of coarse_r; tissue t's coarse inverse is row-major with
    // leading dimension coarse_ld at coarse_inv + coarse_base[t].
    int32_t batch_coarse;
    int32_t coarse_ld;
    const int32_t* tissue_agg0;  // [T+1]
    const int32_t* agg_ptr;      // [aggregates+1]
    const int32_t* agg_nodes;    // [N] node ids, aggregate after aggregate
    const int64_t* coarse_base;  // [T]
    // multilevel coarse space of a single tissue (ml = 1; agg_per_cta = batch_coarse = 0): the
    // tissue's prism columns split by recursive coordinate bisection into ml_n_leaf leaves (node
    // lists in agg_ptr / agg_nodes, node_d relative to the leaf centroid); a set of level l
    // (l = 1: the leaves) is ml_span[l-1] consecutive leaves, the top level L = ml_levels is
    // inverted densely. Every set has the six rigid modes about its centroid (fixed / slave DoFs
    // zeroed), and
    //   M^-1 r = D^-1 r + sum_{l < L} sum_S Q_S W_S Q_S^T r + Q_L A_L^-1 Q_L^T r,
    // W_S the pseudo-inverse of the set's diagonal block Q_S^T J Q_S (an additive multilevel
    // Schwarz preconditioner, symmetric positive semi-definite for an SPD J). CTA lc of the
    // tissue's nct applies it on the leaves [n_leaf lc / nct, n_leaf (lc + 1) / nct).
    int32_t ml;
    int32_t ml_levels;
    int32_t ml_n_leaf;
    int32_t ml_span[kMlMaxLevels];  // leaves per set of each level (4^(l-1))
    int32_t ml_count[kMlMaxLevels]; // sets of each level
    int32_t ml_set0[kMlMaxLevels];  // first index of each level's sets in the per-set arrays
    const double* ml_cen;        // [sets][3] centroids, level after level
    const double* ml_w;          // [sets below the top][36] W_S row-major (index: set0[l-1] + S)
    const double* ml_top_inv;    // [6 ml_count[L-1]]^2 row-major inverse of the top operator
    double* ml_leaf_m;           // [n_leaf][6] raw moments Q_a^T r of the leaves (scratch)
    double* ml_part;             // [partials][6] per-CTA partial moments of the sets of levels >= 2
    const int32_t* ml_pstart;    // [sets+1] first partial of each set (levels >= 2)
    const int32_t* ml_first_cta; // [sets] first CTA of the group whose leaves overlap the set
    const int32_t* ml_pos_leaf;  // [N] the leaf of each position of the leaf node list (agg_nodes)
};

constexpr int kMaxAggPerCta = 4;
constexpr int kMaxCoarse = 2048;  // coarse unknowns the persistent solve stages in shared memory
// Each CTA keeps its 6m rows of the coarse inverse in dynamic shared memory for the whole solve,
// rounded to FP32 (6m x n_coarse floats; the correction is accumulated in FP64 and the solve's
// convergence test is on the FP64 residual, so this only changes the fixed preconditioner).
// The block stays small enough that the SM keeps most of its L1 for the SpMV's matrix reuse.
// The two-level solve runs one 768-thread CTA per SM.
constexpr int kCoarseSmemBytes = 96 * 1024;

// --- element assembly (tf_element.cu) ---------------------------------------------------
// mode: 0 = atomic scatter, 1 = plain read-modify-write (caller guarantees a colour class),
// 2 = atomics from a shared-memory stage, a block's entries on consecutive threads
cudaError_t launch_element_assemble(const AssembleArgs& a, int teams, bool visc, int mode,
                                    cudaStream_t s);
cudaError_t launch_node_terms(const NodeArgs& a, cudaStream_t s);

// --- growth prologue (tf_element.cu) ------------------------------------------------------
// grid_inc [E][9] (may be NULL): the increments of the step's grid-based growth functions, applied
// after the uniform increment (the reference composes its growth functions in list order)
cudaError_t launch_grow(ElemRecord* elems, int32_t n_elems, const double* x, double* fg,
                        const double* rates, const double* angles, double dt, int32_t* rotated,
                        const double* grid_inc, cudaStream_t s);

// One cell of a grid-based growth function (GridBasedGrowthFunction, GrowthFunctionTypes.h:269-548):
// the growth rates (1/s) and orientation angles (radians) of its four corners (0: (i, j), 1: (i+1, j),
// 2: (i, j+1), 3: (i+1, j+1)) after the reference's compatible-averaging pass, which brings the
// angles within 45 degrees of the first corner with an aspect ratio over 1.1 and swaps x / y
// growth where it turned an angle by 90 degrees; elim bit q: corner q's angle left out of the
// average.
struct GridCell {
    double g[4][3];
    double a[4];
    int32_t elim;
    int32_t pad;
};

constexpr int kMaxGridFuncs = 8;  // grid-based growth functions active in one step
struct GridFunc {
    const GridCell* cells;  // [(nx-1)*(ny-1)], cell (i, j) at i*(ny-1) + j
    int32_t nx, ny;
    double zmin, zmax;      // range of initialRelativePositionInZ the function applies to
    int32_t flags;          // bit0 columnar, bit1 peripodial, bit2 basal ECM, bit3 lateral ECM
    int32_t pad;
};
struct GridStep {
    int32_t n;              // active functions, in the reference's list order
    int32_t interpolation;  // 0 nearest corner, 1 bilinear
    double dt;
    GridFunc f[kMaxGridFuncs];
};
// inc [E][9] = the product of the active functions' increments (ShapeBase::calculateFgFromGridCorners,
// updateGrowthIncrement); rel_pos [E][2] pinned relative positions, rel_z [E], eflags [E] as in
// tf_set_grid_growth.
cudaError_t launch_grid_increment(int32_t n_elems, const GridStep& gs, const double* rel_pos, const double* rel_z,
                                  const int32_t* eflags, double* inc, cudaStream_t s);
cudaError_t launch_viscosity_surface(const ElemRecord* elems, int32_t n_elems, int32_t n_nodes,
                                     const double* x, const uint8_t* exposed,
                                     const uint8_t* peripodial, double* visc_surface,
                                     cudaStream_t s);

// --- adjoint (tf_adjoint.cu) ------------------------------------------------------------------
cudaError_t launch_growth_vjp(const ElemRecord* elems, int32_t n_elems, const double* lam, const uint8_t* fixmask,
                              const double* x1, const double* fg_n, const double* rates, const double* angles, double dt,
                              double* mubar, double* dLdr, cudaStream_t s);
cudaError_t launch_position_vjp(const ElemRecord* elems, int32_t n_elems, int32_t n_nodes, const double* lam,
                                const uint8_t* fixmask, const double* x0, const double* x1, const double* visc_surface,
                                const double* ext_visc, const uint8_t* exposed, const uint8_t* peripodial, double dt,
                                double* q, double* abar, cudaStream_t s);
cudaError_t launch_set_inv_fg(ElemRecord* elems, int32_t n_elems, const double* fg, cudaStream_t s);
cudaError_t launch_mask_fixed(int32_t n_nodes, const uint8_t* fixmask, double* v, cudaStream_t s);

// --- direct solve (tf_direct.cu) -----------------------------------------------------------
// 0 ok, 3 singular, 4 not positive definite and too large for the QR fallback, < 0 CUDA / cuSOLVER
// failure; ms = factorise + solve time; method 1 = Cholesky, 2 = QR.
int direct_solve_bsr3(int32_t n_nodes, int64_t nnzb, const int32_t* rowptr, const int32_t* colidx, const double* vals,
                      const double* b, double* x, cudaStream_t s, float* ms, int* method);

// --- Krylov (tf_krylov.cu) ----------------------------------------------------------------
struct KrylovWork {
    int32_t n_nodes;
    const int32_t* rowptr;
    const int32_t* colidx;
    const int32_t* diag;
    const double* vals;
    double *x, *b;                      // solution du, right-hand side g
    double *r, *rhat, *p, *v, *s, *t, *phat, *shat;
    double* dinv;                       // [N][9]
    double* partials;                   // reduction scratch
    int32_t n_partials;                 // capacity in doubles
    KrylovScalars* sc;
    int32_t* dflags;
    // packing blocks outside the element pattern (NULL when the step has no packing pair): row
    // n's extra blocks are pk_vals[pk_blk[k]] at column pk_col[k], k in [pk_ptr[n], pk_ptr[n+1])
    const int32_t* pk_ptr;
    const int32_t* pk_col;
    const int32_t* pk_blk;
    const double* pk_vals;
};

cudaError_t launch_find_diag(const int32_t* rowptr, const int32_t* colidx, int32_t n, int32_t* diag,
                             int32_t* dflags, cudaStream_t s);
// Multicolour block ILU(0) on the BSR3 pattern. Nodes of one colour never couple, so every
// colour class is factorised / solved in parallel once the earlier classes are done.
struct IluPlan {
    int32_t n_colours;
    const int32_t* colour_ptr;    // host: offsets into nodes by colour [n_colours+1]
    const int32_t* cnodes;        // device: nodes sorted by colour
    const int32_t* lo_ptr;        // device [N+1]: lower blocks of each row, sorted by colour
    const int32_t* lo_idx;
    const int32_t* up_ptr;        // device [N+1]: upper blocks of each row
    const int32_t* up_idx;
    double* lu;                   // device [nnzb][9]: L (unit diagonal implied) and U blocks
    double* uinv;                 // device [N][9]: inverse of the U diagonal blocks
    double* y;                    // device [N][3]: forward-solve scratch
};
cudaError_t launch_ilu_factor(const KrylovWork& w, const IluPlan& ilu, cudaStream_t s);
cudaError_t launch_bicgstab_iteration_ilu(const KrylovWork& w, const IluPlan& ilu, cudaStream_t s);
cudaError_t launch_block_jacobi_setup(const KrylovWork& w, cudaStream_t s);
cudaError_t launch_krylov_init(const KrylovWork& w, double rtol, int max_iter, cudaStream_t s);
cudaError_t launch_bicgstab_iteration(const KrylovWork& w, cudaStream_t s);
cudaError_t launch_spmv(const KrylovWork& w, const double* xin, double* yout, cudaStream_t s);
// rout = b - J x and ||rout||^2 into w.sc->du2 (w.partials holds spmv_grid(N) doubles)
cudaError_t launch_residual(const KrylovWork& w, const double* xin, const double* b, double* rout, cudaStream_t s);
cudaError_t launch_axpy(int n, double a, const double* x, double* y, cudaStream_t s);  // y += a x
cudaError_t launch_newton_update(const KrylovWork& w, double* uk, const int32_t* slaves,
                                 const int32_t* masters, int32_t n_pairs, cudaStream_t s);
int spmv_grid(int n_nodes);
// Persistent cooperative BiCGStab over a batch of tissues (one tissue: a plan with T = 1).
// w.partials must hold 4 * plan.n_cta doubles.
// threads: CTA width, 256 (three CTAs per SM, for batches of many tissues) or 768 (one per SM).
int persistent_max_grid(int device, int threads);
// Coarse operator of the two-level preconditioner, row-major dense n_coarse^2: entry
// (6a+r, 6b+c) = sum over the Jacobian blocks k in rows of aggregate a and columns of
// aggregate b of P_row(k)[:, r]^T J_k P_col(k)[:, c]. Blocks are listed per (aggregate, slot)
// with slot_agg[slot] = b, summed in list order (deterministic). Coarse unknowns whose mode is
// empty get a unit diagonal.
struct CoarseAssembly {
    int32_t n_agg, n_coarse;
    // batch: tissue t's matrix is written transposed (row-major for its inverse) into
    // a_cm + tissue_base[t] with leading dimension ld, indices local to the tissue; the unit
    // diagonal entries (modes without support, padding) are the offsets in `empty`
    const int32_t* agg_tissue;     // [n_agg] or null (single tissue)
    const int32_t* tissue_agg0;    // [T+1]
    const int64_t* tissue_base;    // [T]
    int32_t ld;
    const int64_t* empty_offsets;  // [n_empty] batch unit-diagonal offsets
    const int32_t* agg_slot_ptr;   // [n_agg+1] slots of each aggregate
    const int32_t* slot_agg;       // [slots] neighbour aggregate of each slot
    const int32_t* slot_ptr;       // [slots+1] offsets into blk / blk_row
    const int32_t* blk;            // Jacobian block ids
    const int32_t* blk_row;        // their block rows
    const int32_t* empty;          // [n_empty] coarse unknowns without a mode
    int32_t n_empty;
};
cudaError_t launch_coarse_assemble(const KrylovWork& w, const CoarseAssembly& ca, const double* pmode, double* a_cm,
                                   size_t a_cm_doubles, cudaStream_t s);

// --- multilevel coarse space (tf_multilevel.cu) -----------------------------------------------
// Set-up of the multilevel preconditioner from the current J, every solve:
//  pairs:  C_s = sum over the blocks k of leaf pair s (row leaf slot_a[s], column leaf
//          slot_agg[s], blocks listed in slot_ptr / blk / blk_row) of P_i^T J_k P_j, P_i the
//          masked rigid modes of node i about its leaf centroid (node_d, node_mask); one warp per
//          pair, 36 sums in fixed order.
//  blocks: output o (out_ptr / out_slots) = sum over its pairs of T_a^T C_s T_b, T the transport
//          of a rigid motion from the output's row / column set centroid to the leaf centroids;
//          output o < n_diag is set out_set[o]'s diagonal block (to W after pinv6), the others
//          are blocks (out_set[o], out_col[o]) of the dense top operator (6 n_top, row-major).
//  pinv6:  W = V diag(1 / lambda) V^T over the eigenpairs of the symmetric 6 x 6 block with
//          lambda > 1e-12 lambda_max (cyclic Jacobi rotations), in place.
struct MlSetup {
    int32_t n_slots, n_out, n_diag, n_top;
    const int32_t* slot_a;
    const int32_t* slot_agg;
    const int32_t* slot_ptr;
    const int32_t* blk;
    const int32_t* blk_row;
    const double* node_d;
    const uint8_t* node_mask;
    const double* leaf_cen;   // [n_leaf][3]
    const double* set_cen;    // [sets][3] (indexed by out_set / out_col)
    const int32_t* out_ptr;   // [n_out+1]
    const int32_t* out_slots;
    const int32_t* out_set;   // [n_out] global set index of the row set
    const int32_t* out_col;   // [n_out] global set index of the column set
    const int32_t* out_dst;   // [n_out] destination: block index in w_blocks (diag) or top block (S * n_top + T)
    double* pairs;            // [n_slots][36]
    double* w_blocks;         // [n_diag][36]
    double* top;              // [6 n_top]^2
    int32_t* dflags;
};
// top = false: the diagonal blocks and their pseudo-inverses only (m.n_out = m.n_diag), the top
// operator left as it is
cudaError_t launch_ml_setup(const KrylovWork& w, const MlSetup& m, bool top, cudaStream_t s);

// --- packing (tf_packing.cu) ------------------------------------------------------------------
// Node-node contact of a single tissue (Simulation::detectPacingNodes, Simulation.cpp:7997-8153;
// calculatePackingForcesImplicit3D / calculatePackingJacobian3D, :7307-7575).
struct PackParams {
    double bb0[2], bbs[2];  // bounding box minimum and size in x, y (Simulation::calculateBoundingBox)
    double grid_sum[50];    // 10 x 5 grid of summed element side averages ([i * 5 + j]), then the
    double grid_cnt[50];    //   squared detection thresholds (0.4 x the cell average)^2 in grid_sum
    double col_sum, col_cnt;
    double threshold;       // Simulation::packingThreshold = 0.4 x the columnar average side length
    double cell;            // cell size of the candidate search: the largest detection threshold
};
struct PackArgs {
    int32_t n_nodes, n_elems;
    const ElemRecord* elems;
    const double* x;             // [N][3] positions of the detection (the step's start)
    const double* fg;            // [E][9]
    const double* v0;            // [E] reference volumes
    const uint8_t* exposed;      // [E] bit 0 apical, bit 1 basal exposed
    const uint8_t* peripodial;   // [E]
    const int8_t* placement;     // [N] 0 basal, 1 apical, other: never packs
    const int32_t* rowptr;       // element pattern: nodes sharing an element with a node
    const int32_t* colidx;
    double* mass;                // [N]
    PackParams* prm;
    int32_t hash_bits;
    int32_t* bucket_cnt;         // [2^hash_bits + 1]
    int32_t* bucket_start;       // [2^hash_bits + 1]
    int32_t* bucket_nodes;       // [N]
    int32_t* node_cnt;           // [N + 1]
    int32_t* node_start;         // [N + 1]
    int32_t* scan_tmp;           // scan scratch
    int32_t* pairs;              // [capacity][2]
    int32_t capacity;
};
// masses, bounding box, thresholds, bucket fill and the per-node pair counts (node_start holds
// their exclusive scan, node_start[N] the total)
cudaError_t launch_packing_detect(const PackArgs& a, cudaStream_t s);
// the pairs (i, j), i < j, in the reference's visiting order, into pairs[0 .. total) (total <= capacity)
cudaError_t launch_packing_pairs(const PackArgs& a, cudaStream_t s);
// Per Newton iteration: forces into g (free DoFs), -D into the diagonal blocks of i and j and +D
// into the extra blocks (i, j) = pk_vals[2p], (j, i) = pk_vals[2p+1] (rows / columns of fixed DoFs
// left out), D into dfdx[p] (the derivative block of pair p)
struct PackTerms {
    int32_t n_pairs;
    const int32_t* pairs;
    const double* x;             // [N][3] Newton iterate
    const double* mass;
    const PackParams* prm;
    const uint8_t* fixmask;
    const int32_t* diag;
    double* vals;
    double* g;
    double* pk_vals;             // [2 P][9]
    double* dfdx;                // [P][9]
};
cudaError_t launch_packing_terms(const PackTerms& a, cudaStream_t s);
// Exclusive scan of n int32 counts into out[0 .. n] (out[n] = total); tmp holds scan_tmp_ints(n)
int scan_tmp_ints(int n);
cudaError_t launch_scan_i32(const int32_t* in, int32_t* out, int n, int32_t* tmp, cudaStream_t s);

// --- lumen (tf_lumen.cu) ----------------------------------------------------------------------
struct LumenState {
    double volume;  // enclosed volume at the last assembly
    double ideal;   // the step's ideal volume
};
struct LumenArgs {
    int32_t n_nodes, n_tri;
    const ElemRecord* elems;
    const int32_t* tri_elem;  // [n_tri] the lumen elements (apical triangle: nodes 3, 4, 5)
    const double* x;          // [N][3] Newton iterate
    const uint8_t* fixmask;
    double bulk;
    LumenState* state;
    double* part;             // lumen_partials(n_tri) doubles
    double* g;                // residual: += the pressure forces
    double* G;                // [3N] nodal sums of 6 dV/dx (fixed components zeroed)
    double* vals;             // J: += the triangle-local blocks
};
int lumen_partials(int n_tri);
cudaError_t launch_lumen_terms(const LumenArgs& a, cudaStream_t s);
cudaError_t launch_lumen_set_ideal(LumenState* state, double ideal, cudaStream_t s);
// out[0] = (a, b1), out[1] = (a, b2) over n doubles; part holds dot2_partials() doubles
int dot2_partials();
cudaError_t launch_dot2(int n, const double* a, const double* b1, const double* b2, double* part, double* out,
                        cudaStream_t s);

// --- dense inverses of the coarse operators (tf_dense.cu) -------------------------------------
// In-place Gauss-Jordan inverse with partial pivoting of column-major matrices (a row-major
// matrix in, its row-major inverse out). Batched: matrix t of order order[t] at a + base[t], leading
// dimension ld, one CTA each; info[t] = 0, or k + 1 when step k met a zero pivot.
cudaError_t launch_invert_batched(double* a, const int64_t* base, const int32_t* order, int ld, int count,
                                  int32_t* info, cudaStream_t s);
// One n x n matrix over a cooperative grid; scratch holds invert_coop_scratch_bytes(n); *status = 0,
// k + 1 for a zero pivot at step k, -1 when a grid barrier timed out.
size_t invert_coop_scratch_bytes(int n);
cudaError_t launch_invert_coop(double* a, int n, void* scratch, int32_t* status, int device, cudaStream_t s);
// m = (m + m^T) / 2 for count matrices of order n, leading dimension ld, stride doubles apart
cudaError_t launch_symmetrize(double* m, int n, int ld, long long stride, int count, cudaStream_t s);
// Rows [r0, r1) of part k of n of the rows [b0, b1), cut at multiples of G from b0 (G = 1: the
// proportional split b0 + L k / n). The persistent solve's CTA row ranges and a single tissue's
// two-level aggregates are cut this way, so a smoother group never straddles two of them.
__host__ __device__ inline void group_split(int b0, int b1, int k, int n, int G, int& r0, int& r1) {
    const long long ng = (b1 - b0 + G - 1) / G;
    r0 = b0 + (int)(G * (ng * k / n));
    const int e = b0 + (int)(G * (ng * (k + 1) / n));
    r1 = e < b1 ? e : b1;
}
// Inverses of the 3G x 3G diagonal sub-blocks of J (G > 1 layout of BatchPlan::group).
cudaError_t launch_group_jacobi_setup(const KrylovWork& w, int G, cudaStream_t s);
cudaError_t launch_bicgstab_batched(const KrylovWork& w, const BatchPlan& plan, double rtol, int max_iter,
                                    int threads, cudaStream_t s);  // dynamic smem: the plan's coarse row block
// uk += du on active tissues, du[slave] = du[master], per-tissue ||du||^2 into plan.du2
cudaError_t launch_newton_update_batched(const KrylovWork& w, const BatchPlan& plan, double* uk,
                                         const int32_t* slaves, const int32_t* masters, int32_t n_pairs,
                                         cudaStream_t s);
int vec_grid(int n_nodes);

}  // namespace tfb
