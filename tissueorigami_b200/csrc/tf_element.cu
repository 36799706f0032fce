// tf_element.cu -- prism element kernels of the B200 Newton step (FP64).
//
// k_element_assemble: one team of 6 threads per prism (5 teams per warp).
//   phase 0  the team copies the prism's 416-byte record and gathers its 6 nodes;
//   phase 1  thread g evaluates Gauss point g: dX/dxi from the reference shape, F, Fe = F InvFg,
//            J_e, ln J_e, the neo-Hookean Cauchy stress, spatial shape gradients and the
//            scalars of the closed-form tangent (TissueFolding/SourceCode/Prism.cpp:766-888,
//            ShapeBase.cpp:2389-2845);
//   phase 2  the six threads split the 21 symmetric 3x3 blocks (36 when internal viscosity
//            is on) and the 6 nodal forces, sum the Gauss points and scatter straight into
//            the BSR3 Jacobian and the residual - no 18x18 element matrix ever reaches HBM.
//   phase 3  (staged scatter only) the blocks wait in shared memory and the whole CTA adds
//            them to J with consecutive threads on consecutive entries of one block, so a
//            warp's FP64 reductions reach L2 as ~12 sectors instead of 32.
//
// Closed-form tangent. For the neo-Hookean law of Prism.cpp:793-794 the reference's D81
// contraction (ShapeBase.cpp:3010-3062) pushes forward to
//     c_ijkl = lambda d_ij d_kl + (mu - lambda ln J_e)(d_ik d_jl + d_il d_jk)
// because Fe C^-1 Fe^T = I, so with a = grad N_a, b = grad N_b (current configuration) and
// dv = det F det(dX/dxi) w_g:
//     K_ab,ik = dv/J_e [lambda a_i b_k + (mu - lambda ln J_e)(d_ik a.b + a_k b_i)]
//             + d_ik (a^T sigma b) dv                       (Integral2, ShapeBase.cpp:3064-3095)
// The reference's Jacobian storage holds the viscous part transposed; this kernel writes the
// true Jacobian J = K^T, whose viscous blocks are (ShapeBase.cpp:3123-3209, untransposed):
//     Jv_ab = 0.5 eta dv [(a.b) P + b (P^T a)^T] + (sv a) b^T - (sv b) a^T,  P = I/dt - grad v.
#include <math.h>

#include "tf_internal.cuh"

namespace tfb {
namespace {

// Shape-function derivatives of the 6-point prism rule, uploaded once from the host
// (Prism.cpp:97-130, 597-652). c_dN[g][k][n] = dN_n / dxi_k at Gauss point g.
__constant__ double c_dN[6][3][6];
constexpr double kGaussWeight = 1.0 / 6.0;

__device__ __forceinline__ double det3(const double m[3][3]) {
    double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]);
    det -= m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]);
    det += m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    return det;
}

__device__ __forceinline__ void inv3(const double m[3][3], double det, double o[3][3]) {
    const double id = 1.0 / det;
    o[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]) * id;
    o[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * id;
    o[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * id;
    o[1][0] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) * id;
    o[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * id;
    o[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * id;
    o[2][0] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) * id;
    o[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * id;
    o[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * id;
}

__device__ __forceinline__ void mm3(const double a[3][3], const double b[3][3], double c[3][3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) c[i][j] = a[i][0] * b[0][j] + a[i][1] * b[1][j] + a[i][2] * b[2][j];
}

// (dN * pos)^T at Gauss point g: out[r][k] = sum_n dN[g][k][n] pos[n][r]
__device__ __forceinline__ void grad_xi(const double* pos18, int g, double out[3][3]) {
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double s = 0.0;
#pragma unroll
            for (int n = 0; n < 6; ++n) s += c_dN[g][k][n] * pos18[n * 3 + r];
            out[r][k] = s;
        }
}

// Symmetric-pair order for the 21 unique blocks: 15 off-diagonal pairs, then 6 diagonal.
__constant__ int8_t c_pairA[36] = {0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 3, 3, 4, 0, 1, 2, 3, 4, 5,
                                   1, 2, 3, 4, 5, 2, 3, 4, 5, 3, 4, 5, 4, 5, 5};
__constant__ int8_t c_pairB[36] = {1, 2, 3, 4, 5, 2, 3, 4, 5, 3, 4, 5, 4, 5, 5, 0, 1, 2, 3, 4, 5,
                                   0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 3, 3, 4};

// Scatter modes of k_element_assemble: each lane adds its own blocks with FP64 atomics (0), adds
// them with plain read-modify-writes inside one element colour (1), or stages them in shared
// memory for a CTA-wide pass of atomics laid out entry by entry (2).
constexpr int kScatterAtomic = 0, kScatterColoured = 1, kScatterStaged = 2;

template <int MODE>
__device__ __forceinline__ void add_entry(double* p, double v) {
    if (MODE == kScatterColoured)
        *p += v;
    else
        atomicAdd(p, v);
}

// Position in the pair order above of the off-diagonal pair (a, b), a < b.
__device__ __forceinline__ int upper_pair(int a, int b) { return a * 5 - (a * (a - 1)) / 2 + (b - a - 1); }

__device__ int find_block(const int32_t* rowptr, const int32_t* colidx, int row, int col) {
    int lo = rowptr[row], hi = rowptr[row + 1] - 1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        const int c = colidx[mid];
        if (c == col) return mid;
        if (c < col)
            lo = mid + 1;
        else
            hi = mid - 1;
    }
    return -1;
}

// Routed add of one Jacobian entry (row DoF rd, column DoF cd before routing).
__device__ __forceinline__ void routed_add(const AssembleArgs& A, int rd, int cd, double v) {
    const int r = A.dofmap[rd], c = A.dofmap[cd];
    const int slot = find_block(A.rowptr, A.colidx, r / 3, c / 3);
    if (slot < 0) {
        atomicOr(A.dflags, DF_PATTERN_MISS);
        return;
    }
    atomicAdd(A.vals + (size_t)slot * 9 + (r % 3) * 3 + (c % 3), v);
}

template <int TEAMS, bool VISC, int MODE>
__global__ void __launch_bounds__(TEAMS * 6) k_element_assemble(AssembleArgs A) {
    constexpr int GPW = VISC ? 42 : 26;  // doubles per Gauss point kept for phase 2
    extern __shared__ __align__(16) double smem_dyn[];
    double(*s_rec)[kElemWords] = reinterpret_cast<double(*)[kElemWords]>(smem_dyn);
    double(*s_x)[18] = reinterpret_cast<double(*)[18]>(smem_dyn + TEAMS * kElemWords);
    double(*s_v)[18] = reinterpret_cast<double(*)[18]>(smem_dyn + TEAMS * (kElemWords + 18));
    double(*s_gp)[6][GPW] = reinterpret_cast<double(*)[6][GPW]>(smem_dyn + TEAMS * (kElemWords + (VISC ? 36 : 18)));
    constexpr int NB = VISC ? 36 : 21;  // blocks a team computes (21 symmetric pairs without viscosity)
    double(*s_K)[NB][9] = reinterpret_cast<double(*)[NB][9]>(smem_dyn + TEAMS * (kElemWords + (VISC ? 36 : 18) + 6 * GPW));
    int(*s_fix)[6] = reinterpret_cast<int(*)[6]>(smem_dyn + TEAMS * (kElemWords + (VISC ? 36 : 18) + 6 * GPW +
                                                                   (MODE == kScatterStaged ? NB * 9 : 0)));
    int* s_go = reinterpret_cast<int*>(s_fix + TEAMS);  // staged scatter: team active and not routed

    const int team = threadIdx.x / 6;
    const int lane = threadIdx.x - team * 6;
    const int idx = blockIdx.x * TEAMS + team;
    bool active = idx < A.e_count;
    int e = 0;
    if (active) e = A.elem_list ? A.elem_list[A.e_begin + idx] : A.e_begin + idx;

    // ---- phase 0: element record and node gather ------------------------------------------
    if (active) {
        const double* src = reinterpret_cast<const double*>(A.elems + e);
        for (int k = lane; k < kElemWords; k += 6) s_rec[team][k] = __ldg(src + k);
    }
    __syncthreads();
    const ElemRecord& R = *reinterpret_cast<const ElemRecord*>(&s_rec[team][0]);
    if (active && A.tissue_active && !A.tissue_active[R.tissue]) active = false;  // converged tissue
    if (active) {
        const int nd = R.conn[lane];
        s_fix[team][lane] = A.fixmask[nd];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double xk = A.uk[(size_t)nd * 3 + k];
            s_x[team][lane * 3 + k] = xk;
            if (VISC) s_v[team][lane * 3 + k] = (xk - A.un[(size_t)nd * 3 + k]) * A.inv_dt;
        }
    }
    __syncthreads();

    // ---- phase 1: Gauss point g = lane -----------------------------------------------------
    if (active) {
        const int g = lane;
        double dX[3][3], invdX[3][3], J[3][3], invJ[3][3], F[3][3], Fe[3][3], Fg[3][3];
        grad_xi(R.xref, g, dX);
        const double detdX = det3(dX);
        inv3(dX, detdX, invdX);
        grad_xi(&s_x[team][0], g, J);
        inv3(J, det3(J), invJ);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) Fg[i][j] = R.inv_fg[i * 3 + j];
        mm3(J, invdX, F);
        mm3(F, Fg, Fe);
        const double detF = det3(F);
        const double Je = det3(Fe);
        if (isnan(Je))
            atomicOr(A.dflags, DF_NONFINITE);
        else if (!(Je > 0.0))
            atomicOr(A.dflags, DF_INVERTED);
        const double lnJ = log(Je);
        const double dv = detF * detdX * kGaussWeight;
        const double iJe = 1.0 / Je;
        double* G = &s_gp[team][g][0];
        // spatial gradients: dNx[m][n] = sum_k invJ[k][m] dN[g][k][n]
#pragma unroll
        for (int m = 0; m < 3; ++m)
#pragma unroll
            for (int n = 0; n < 6; ++n)
                G[m * 6 + n] = invJ[0][m] * c_dN[g][0][n] + invJ[1][m] * c_dN[g][1][n] + invJ[2][m] * c_dN[g][2][n];
        // sigma dv = (mu (Fe Fe^T - I) + lambda lnJ I) dv / Je
        double bmat[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                bmat[i][j] = Fe[i][0] * Fe[j][0] + Fe[i][1] * Fe[j][1] + Fe[i][2] * Fe[j][2];
        const double lam = R.lam, mu = R.mu;
        const double sdv = dv * iJe;
        G[18] = lam * sdv;                  // c1
        G[19] = (mu - lam * lnJ) * sdv;     // c2
        G[20] = (mu * (bmat[0][0] - 1.0) + lam * lnJ) * sdv;  // S xx
        G[21] = (mu * (bmat[1][1] - 1.0) + lam * lnJ) * sdv;  // S yy
        G[22] = (mu * (bmat[2][2] - 1.0) + lam * lnJ) * sdv;  // S zz
        G[23] = mu * bmat[0][1] * sdv;                        // S xy
        G[24] = mu * bmat[1][2] * sdv;                        // S yz
        G[25] = mu * bmat[0][2] * sdv;                        // S xz
        if (VISC) {
            // velocity gradient L = sum_c v_c (x) grad N_c (ShapeBase.cpp:3097-3121)
            double L[3][3];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    double s = 0.0;
#pragma unroll
                    for (int c = 0; c < 6; ++c) s += s_v[team][c * 3 + i] * G[j * 6 + c];
                    L[i][j] = s;
                }
            const double eta = R.eta, inv_dt = A.inv_dt;
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) G[26 + i * 3 + j] = (i == j ? inv_dt : 0.0) - L[i][j];
            G[35] = 0.5 * eta * dv;
            const double ed = eta * dv;
            G[36] = ed * L[0][0];
            G[37] = ed * L[1][1];
            G[38] = ed * L[2][2];
            G[39] = ed * 0.5 * (L[0][1] + L[1][0]);
            G[40] = ed * 0.5 * (L[1][2] + L[2][1]);
            G[41] = ed * 0.5 * (L[0][2] + L[2][0]);
        }
    }
    __syncthreads();
    if (MODE != kScatterStaged && !active) return;

    const bool routed = active && (R.flags & 1) != 0;
    if (MODE == kScatterStaged && lane == 0) s_go[team] = active && !routed;

    // ---- phase 2a: nodal forces, node a = lane ---------------------------------------------
    if (active) {
        const int a = lane;
        double f0 = 0.0, f1 = 0.0, f2 = 0.0;
#pragma unroll
        for (int g = 0; g < 6; ++g) {
            const double* G = &s_gp[team][g][0];
            const double ax = G[a], ay = G[6 + a], az = G[12 + a];
            double sxx = G[20], syy = G[21], szz = G[22], sxy = G[23], syz = G[24], sxz = G[25];
            if (VISC) {
                sxx += G[36]; syy += G[37]; szz += G[38]; sxy += G[39]; syz += G[40]; sxz += G[41];
            }
            f0 -= sxx * ax + sxy * ay + sxz * az;
            f1 -= sxy * ax + syy * ay + syz * az;
            f2 -= sxz * ax + syz * ay + szz * az;
        }
        const int nd = R.conn[a];
        const int fm = s_fix[team][a];
        const double f[3] = {f0, f1, f2};
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            if ((fm >> i) & 1) continue;
            if (routed)
                atomicAdd(A.g + A.dofmap[nd * 3 + i], f[i]);
            else
                add_entry<MODE>(A.g + (size_t)nd * 3 + i, f[i]);
        }
    }

    // ---- phase 2b: tangent blocks ----------------------------------------------------------
    for (int pb = lane; active && pb < NB; pb += 6) {
        const int a = c_pairA[pb], b = c_pairB[pb];
        double K[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
        for (int g = 0; g < 6; ++g) {
            const double* G = &s_gp[team][g][0];
            const double av[3] = {G[a], G[6 + a], G[12 + a]};
            const double bv[3] = {G[b], G[6 + b], G[12 + b]};
            const double c1 = G[18], c2 = G[19];
            const double sxx = G[20], syy = G[21], szz = G[22], sxy = G[23], syz = G[24], sxz = G[25];
            const double ab = av[0] * bv[0] + av[1] * bv[1] + av[2] * bv[2];
            const double Sb0 = sxx * bv[0] + sxy * bv[1] + sxz * bv[2];
            const double Sb1 = sxy * bv[0] + syy * bv[1] + syz * bv[2];
            const double Sb2 = sxz * bv[0] + syz * bv[1] + szz * bv[2];
            const double dg = c2 * ab + av[0] * Sb0 + av[1] * Sb1 + av[2] * Sb2;
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int k = 0; k < 3; ++k) K[i][k] += c1 * av[i] * bv[k] + c2 * av[k] * bv[i];
            K[0][0] += dg;
            K[1][1] += dg;
            K[2][2] += dg;
            if (VISC) {
                const double* P = G + 26;
                const double cv = G[35];
                const double vxx = G[36], vyy = G[37], vzz = G[38], vxy = G[39], vyz = G[40], vxz = G[41];
                const double Pta[3] = {P[0] * av[0] + P[3] * av[1] + P[6] * av[2],
                                       P[1] * av[0] + P[4] * av[1] + P[7] * av[2],
                                       P[2] * av[0] + P[5] * av[1] + P[8] * av[2]};
                const double Sva[3] = {vxx * av[0] + vxy * av[1] + vxz * av[2],
                                       vxy * av[0] + vyy * av[1] + vyz * av[2],
                                       vxz * av[0] + vyz * av[1] + vzz * av[2]};
                const double Svb[3] = {vxx * bv[0] + vxy * bv[1] + vxz * bv[2],
                                       vxy * bv[0] + vyy * bv[1] + vyz * bv[2],
                                       vxz * bv[0] + vyz * bv[1] + vzz * bv[2]};
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j)
                        K[i][j] += cv * (ab * P[i * 3 + j] + bv[i] * Pta[j]) + Sva[i] * bv[j] - Svb[i] * av[j];
            }
        }
        if (MODE == kScatterStaged && !routed) {
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int k = 0; k < 3; ++k) s_K[team][pb][i * 3 + k] = K[i][k];
            continue;
        }
        const int fa = s_fix[team][a], fb = s_fix[team][b];
        if (routed) {
            const int na = R.conn[a], nb = R.conn[b];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    if (((fa >> i) & 1) || ((fb >> k) & 1)) continue;
                    routed_add(A, na * 3 + i, nb * 3 + k, K[i][k]);
                    if (!VISC && a != b) routed_add(A, nb * 3 + k, na * 3 + i, K[i][k]);
                }
            continue;
        }
        double* blk = A.vals + (size_t)R.slots[a * 6 + b] * 9;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int k = 0; k < 3; ++k)
                if (!((fa >> i) & 1) && !((fb >> k) & 1)) add_entry<MODE>(blk + i * 3 + k, K[i][k]);
        if (!VISC && a != b) {
            double* blkT = A.vals + (size_t)R.slots[b * 6 + a] * 9;
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    if (!((fa >> i) & 1) && !((fb >> k) & 1)) add_entry<MODE>(blkT + k * 3 + i, K[i][k]);
        }
    }

    // ---- phase 3 (staged scatter): the CTA's 36 destination blocks per prism, one entry per
    // thread, entries of a block on consecutive threads. The (block, entry) a thread adds is the
    // same for every prism of the CTA, so it is decoded once: bits 0-8 source offset in the
    // team's stage (< 36 * 9), 9-14 destination block p*6+q, 15-18 entry r*3+c, 19-21 p,
    // 22-23 r, 24-26 q, 27-28 c.
    if (MODE == kScatterStaged) {
        constexpr int NT = TEAMS * 6, NJ = (324 + NT - 1) / NT;
        int desc[NJ];
#pragma unroll
        for (int j = 0; j < NJ; ++j) {
            const int rem = threadIdx.x + j * NT;
            const int d = rem / 9, en = rem - d * 9;
            const int p = d / 6, q = d - p * 6, r = en / 3, c = en - r * 3;
            int src;
            if (p == q)
                src = (15 + p) * 9 + en;
            else if (p < q)
                src = upper_pair(p, q) * 9 + en;
            else if (VISC)
                src = (21 + upper_pair(q, p)) * 9 + en;
            else
                src = upper_pair(q, p) * 9 + c * 3 + r;
            desc[j] = rem < 324 ? src | d << 9 | en << 15 | p << 19 | r << 22 | q << 24 | c << 27 : -1;
        }
        __syncthreads();
        for (int tm = 0; tm < TEAMS; ++tm) {
            if (!s_go[tm]) continue;
            const ElemRecord& Rt = *reinterpret_cast<const ElemRecord*>(&s_rec[tm][0]);
            const double* stage = &s_K[tm][0][0];
#pragma unroll
            for (int j = 0; j < NJ; ++j) {
                const int dj = desc[j];
                if (dj < 0) continue;
                if (((s_fix[tm][(dj >> 19) & 7] >> ((dj >> 22) & 3)) & 1) ||
                    ((s_fix[tm][(dj >> 24) & 7] >> ((dj >> 27) & 3)) & 1))
                    continue;
                atomicAdd(A.vals + (size_t)Rt.slots[(dj >> 9) & 63] * 9 + ((dj >> 15) & 15), stage[dj & 511]);
            }
        }
    }
}

// Drag, fixed-DoF identity and slave identity on the diagonal, plus the external drag force
// (NewtonRaphsonSolver.cpp:362-423, 195-219, 128-183).
__global__ void k_node_terms(NodeArgs a) {
    const int A = blockIdx.x * blockDim.x + threadIdx.x;
    if (A >= a.n_nodes) return;
    if (a.tissue_active && !a.tissue_active[a.node_tissue[A]]) return;  // converged tissue
    const int fm = a.fixmask[A];
    const double vs = a.visc_surface[A];
    const double inv_dt = 1.0 / a.dt;
    const double surfacePerDt = vs / a.dt;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int d = A * 3 + i;
        const int md = a.dofmap[d];
        const int row = md / 3, ci = md % 3;
        double* dg = a.vals + (size_t)a.diag[row] * 9 + ci * 4;
        if ((fm >> i) & 1) {
            atomicAdd(dg, 1.0);
        } else {
            const double ev = a.ext_visc[d];
            const double v = (a.uk[d] - a.un[d]) * inv_dt;
            atomicAdd(dg, surfacePerDt * ev);
            atomicAdd(a.g + md, -((vs * ev) * v));
            // addExernalForces (NewtonRaphsonSolver.cpp:449-457): gSum += gExt on free DoFs (the
            // fixed ones are zeroed afterwards by calcutateFixedK), routed like every force
            if (a.ext_force) atomicAdd(a.g + md, a.ext_force[d]);
        }
        if (md != d) a.vals[(size_t)a.diag[A] * 9 + i * 4] = 1.0;
    }
}

// ---- growth prologue -----------------------------------------------------------------------

// Per-element growth step (ShapeBase.cpp:1914-2041 rotation extraction, 471-505 increment,
// 1452-1506 growShapeByFg) from the positions at the start of the step.
__global__ void k_grow(ElemRecord* elems, int32_t n_elems, const double* x, double* fg,
                       const double* rates, const double* angles, double dt, int32_t* rotated,
                       const double* grid_inc) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_elems) return;
    ElemRecord& R = elems[e];
    double pos[18];
#pragma unroll
    for (int n = 0; n < 6; ++n)
#pragma unroll
        for (int k = 0; k < 3; ++k) pos[n * 3 + k] = x[(size_t)R.conn[n] * 3 + k];
    double TF[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int g = 0; g < 6; ++g) {
        double dX[3][3], invdX[3][3], J[3][3], F[3][3];
        grad_xi(R.xref, g, dX);
        inv3(dX, det3(dX), invdX);
        grad_xi(pos, g, J);
        mm3(J, invdX, F);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) TF[i][j] += F[i][j] * kGaussWeight;
    }
    // orthogonal polar factor U V^T of the SVD by the Newton polar iteration
    double Rm[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Rm[i][j] = TF[i][j];
    for (int it = 0; it < 100; ++it) {
        double inv[3][3], diff = 0.0;
        inv3(Rm, det3(Rm), inv);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const double nx = 0.5 * (Rm[i][j] + inv[j][i]);
                diff = fmax(diff, fabs(nx - Rm[i][j]));
                Rm[i][j] = nx;
            }
        if (diff < 1e-15) break;
    }
    bool rot = false;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            if (i != j && (Rm[i][j] > 0.017 || Rm[i][j] < -0.017)) rot = true;
    double Gm[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    if (rot) {
        const double tz = atan2(Rm[0][1], Rm[0][0]);
        if (tz > 0.017 || tz < -0.017) {
            const double c = cos(tz), s = sin(tz);
            // GrowthStrainsRotMat = Rz(tz)^T
            Gm[0][0] = c; Gm[0][1] = s; Gm[1][0] = -1.0 * s; Gm[1][1] = c;
        } else {
            rot = false;
        }
    }
    if (rotated) rotated[e] = rot ? 1 : 0;
    const double ang = angles ? angles[e] : 0.0;
    const double c = cos(ang), s = sin(ang);
    const double Ra[3][3] = {{c, -1.0 * s, 0.0}, {s, c, 0.0}, {0.0, 0.0, 1.0}};
    double inc[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    inc[0][0] = exp(rates[(size_t)e * 3 + 0] * 1.0 * dt);
    inc[1][1] = exp(rates[(size_t)e * 3 + 1] * 1.0 * dt);
    inc[2][2] = exp(rates[(size_t)e * 3 + 2] * 1.0 * dt);
    double tmp[3][3], gi[3][3];
    mm3(Ra, inc, tmp);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) gi[i][j] = tmp[i][0] * Ra[j][0] + tmp[i][1] * Ra[j][1] + tmp[i][2] * Ra[j][2];
    if (grid_inc) {  // updateGrowthIncrement of the step's grid functions: growthInc = G growthInc
        double G[3][3], prod[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) G[i][j] = grid_inc[(size_t)e * 9 + i * 3 + j];
        mm3(G, gi, prod);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) gi[i][j] = prod[i][j];
    }
    if (rot) {
        double GtI[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) GtI[i][j] = Gm[0][i] * gi[0][j] + Gm[1][i] * gi[1][j] + Gm[2][i] * gi[2][j];
        mm3(GtI, Gm, gi);
    }
    double Fg[3][3], Fn[3][3], inv[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Fg[i][j] = fg[(size_t)e * 9 + i * 3 + j];
    mm3(gi, Fg, Fn);
    inv3(Fn, det3(Fn), inv);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            fg[(size_t)e * 9 + i * 3 + j] = Fn[i][j];
            R.inv_fg[i * 3 + j] = inv[i][j];
        }
}

// Growth increments of the step's grid-based functions, one element per thread
// (Simulation::calculateGrowthGridBased, Simulation.cpp:9038-9085; ShapeBase::calculateFgFromGridCorners,
// ShapeBase.cpp:513-658; convertRelativePosToGridIndex :834-860; isGrowthRateApplicable :297-334;
// updateGrowthIncrement :764-787). eflags: bit0 ECM-mimicking, bit1 actin-mimicking, bit2 basal
// placement, bit3 ECM at the circumference, bits 4-5 tissue type (0 columnar, 1 peripodial).
__global__ void k_grid_increment(int32_t n_elems, GridStep gs, const double* __restrict__ rel_pos,
                                 const double* __restrict__ rel_z, const int32_t* __restrict__ eflags,
                                 double* __restrict__ inc) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_elems) return;
    const int ef = eflags[e];
    const bool ecm = ef & 1, actin = ef & 2, basal = ef & 4, ecm_circ = ef & 8;
    const int ttype = (ef >> 4) & 3;
    const double rx = rel_pos[2 * e], ry = rel_pos[2 * e + 1], rz = rel_z[e];
    double acc[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int f = 0; f < gs.n; ++f) {
        const GridFunc& F = gs.f[f];
        const double px = rx * (double)(float)(F.nx - 1), py = ry * (double)(float)(F.ny - 1);
        int ix = (int)floor(px), iy = (int)floor(py);
        double fx = px - ix, fy = py - iy;
        if (ix >= F.nx - 1) {
            ix = F.nx - 2;
            fx = 1.0;
        } else if (ix < 0) {
            ix = 0;
            fx = 0.0;
        }
        if (iy >= F.ny - 1) {
            iy = F.ny - 2;
            fy = 1.0;
        } else if (iy < 0) {
            iy = 0;
            fy = 0.0;
        }
        const GridCell& c = F.cells[(size_t)ix * (F.ny - 1) + iy];
        // which increment the element takes from this function: the columnar one (also through
        // the ECM options) or the peripodial one; -1: neither (identity)
        int source = -1;
        if (((F.flags & 4) && ecm && basal) || ((F.flags & 8) && ecm_circ && !basal)) source = 0;
        if (!ecm) {
            if ((F.flags & 1) && ttype == 0) source = 0;
            if ((F.flags & 2) && ttype == 1) source = 1;
        }
        if (source < 0 || (source == 0 && ttype != 0) || (source == 1 && ttype != 1)) continue;
        if (rz < F.zmin || rz > F.zmax) continue;  // outside the function's z range: identity
        double g[3] = {0.0, 0.0, 0.0}, angle = 0.0;
        if (gs.interpolation == 0) {
            const int q = fx > 0.5 ? (fy > 0.5 ? 3 : 1) : (fy > 0.5 ? 2 : 0);
#pragma unroll
            for (int k = 0; k < 3; ++k) g[k] = c.g[q][k];
        } else {
            const double w[4] = {(1.0 - fx) * (1.0 - fy), fx * (1.0 - fy), (1.0 - fx) * fy, fx * fy};
            double elim = 0.0;
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if ((c.elim >> q) & 1) elim += w[q];
            angle = c.a[0] * w[0] + c.a[1] * w[1] + c.a[2] * w[2] + c.a[3] * w[3];
            if (elim > 0) angle = elim >= 0.9999999 ? 0.0 : angle / (1.0 - elim);
#pragma unroll
            for (int k = 0; k < 3; ++k) g[k] = c.g[0][k] * w[0] + c.g[1][k] * w[1] + c.g[2][k] * w[2] + c.g[3][k] * w[3];
        }
        if (actin) g[2] = 0.0;  // actin-mimicking elements do not grow in height
        double D[3][3] = {{exp(g[0] * gs.dt), 0, 0}, {0, exp(g[1] * gs.dt), 0}, {0, 0, exp(g[2] * gs.dt)}};
        if (angle != 0.0) {
            const double cs = cos(angle), sn = sin(angle);
            const double R[3][3] = {{cs, -1.0 * sn, 0.0}, {sn, cs, 0.0}, {0.0, 0.0, 1.0}};
            double T[3][3];
            mm3(R, D, T);
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) D[i][j] = T[i][0] * R[j][0] + T[i][1] * R[j][1] + T[i][2] * R[j][2];
        }
        double P[3][3];
        mm3(D, acc, P);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) acc[i][j] = P[i][j];
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) inc[(size_t)e * 9 + i * 3 + j] = acc[i][j];
}

// Exposed-triangle area (Prism::calculateApicalArea / calculateBasalArea, Prism.cpp:1485-1556)
__device__ double tri_area(const double* x, int n0, int n1, int n2) {
    const double Threshold = 1E-5;
    double s1[3], s2[3], costet = 0.0, Side1 = 0.0, Side2 = 0.0, Area = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        s1[i] = x[(size_t)n1 * 3 + i] - x[(size_t)n0 * 3 + i];
        s2[i] = x[(size_t)n2 * 3 + i] - x[(size_t)n0 * 3 + i];
        costet += s1[i] * s2[i];
        Side1 += s1[i] * s1[i];
        Side2 += s2[i] * s2[i];
    }
    if (Side1 > Threshold && Side2 > Threshold) {
        Side1 = sqrt(Side1);
        Side2 = sqrt(Side2);
        costet /= (Side1 * Side2);
        const double sinTetSq = 1 - costet * costet;
        double sintet = 0;
        if (sinTetSq > Threshold) sintet = sqrt(sinTetSq);
        Area = Side1 * Side2 * sintet / 2.0;
    }
    return Area;
}

__global__ void k_viscosity_surface(const ElemRecord* elems, int32_t n_elems, const double* x,
                                    const uint8_t* exposed, const uint8_t* peripodial,
                                    double* visc_surface) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_elems) return;
    const int ex = exposed[e];
    if (!ex) return;
    const int32_t* c = elems[e].conn;
    const bool per = peripodial && peripodial[e];
    if (ex & 1) {
        const int i0 = per ? 0 : 3;
        const double A = tri_area(x, c[i0], c[i0 + 1], c[i0 + 2]) / 3;
        for (int i = 0; i < 3; ++i) atomicAdd(visc_surface + c[i0 + i], A);
    }
    if (ex & 2) {
        const int i0 = per ? 3 : 0;
        const double A = tri_area(x, c[i0], c[i0 + 1], c[i0 + 2]) / 3;
        for (int i = 0; i < 3; ++i) atomicAdd(visc_surface + c[i0 + i], A);
    }
}

template <int TEAMS, bool VISC, int MODE>
constexpr size_t element_smem_bytes() {
    return sizeof(double) * TEAMS *
               (kElemWords + (VISC ? 36 : 18) + 6 * (VISC ? 42 : 26) + (MODE == kScatterStaged ? (VISC ? 36 : 21) * 9 : 0)) +
           sizeof(int) * TEAMS * 7;
}

template <int TEAMS, bool VISC, int MODE>
cudaError_t launch_t(const AssembleArgs& a, cudaStream_t s) {
    // the shared-memory opt-in is a per-device attribute of the kernel: set once per device
    constexpr int kDevices = 64;
    static bool attr_set[kDevices] = {};
    constexpr size_t smem = element_smem_bytes<TEAMS, VISC, MODE>();
    int dev = 0;
    cudaError_t derr = cudaGetDevice(&dev);
    if (derr != cudaSuccess) return derr;
    if (dev < 0 || dev >= kDevices || !attr_set[dev]) {
        cudaError_t err = cudaFuncSetAttribute(k_element_assemble<TEAMS, VISC, MODE>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err != cudaSuccess) return err;
        if (dev >= 0 && dev < kDevices) attr_set[dev] = true;
    }
    if (a.e_count <= 0) return cudaSuccess;
    const int grid = (a.e_count + TEAMS - 1) / TEAMS;
    k_element_assemble<TEAMS, VISC, MODE><<<grid, TEAMS * 6, smem, s>>>(a);
    return cudaGetLastError();
}

template <int TEAMS, bool VISC>
cudaError_t launch_modes(const AssembleArgs& a, int mode, cudaStream_t s) {
    switch (mode) {
        case kScatterColoured: return launch_t<TEAMS, VISC, kScatterColoured>(a, s);
        case kScatterStaged: return launch_t<TEAMS, VISC, kScatterStaged>(a, s);
        default: return launch_t<TEAMS, VISC, kScatterAtomic>(a, s);
    }
}

template <int TEAMS>
cudaError_t launch_teams(const AssembleArgs& a, bool visc, int mode, cudaStream_t s) {
    return visc ? launch_modes<TEAMS, true>(a, mode, s) : launch_modes<TEAMS, false>(a, mode, s);
}

bool g_table_ready = false;

cudaError_t upload_gauss_table() {
    if (g_table_ready) return cudaSuccess;
    // Prism.cpp:105-130 (6-point rule) and 597-652 (derivatives)
    const double s = 1.0 / pow(3.0, 0.5);
    const double pts[3][2] = {{1.0 / 6.0, 1.0 / 6.0}, {2.0 / 3.0, 1.0 / 6.0}, {1.0 / 6.0, 2.0 / 3.0}};
    double dN[6][3][6];
    for (int g = 0; g < 6; ++g) {
        const double eta = pts[g % 3][0], nu = pts[g % 3][1], zeta = g < 3 ? s : -s;
        const double alpha = (1 - zeta) / 2, beta = (1 + zeta) / 2, lambda = 1 - eta - nu;
        const double r0[6] = {-alpha, alpha, 0, -beta, beta, 0};
        const double r1[6] = {-alpha, 0, alpha, -beta, 0, beta};
        const double r2[6] = {-lambda / 2, -eta / 2, -nu / 2, lambda / 2, eta / 2, nu / 2};
        for (int n = 0; n < 6; ++n) {
            dN[g][0][n] = r0[n];
            dN[g][1][n] = r1[n];
            dN[g][2][n] = r2[n];
        }
    }
    cudaError_t err = cudaMemcpyToSymbol(c_dN, dN, sizeof(dN));
    if (err == cudaSuccess) g_table_ready = true;
    return err;
}

}  // namespace

cudaError_t launch_element_assemble(const AssembleArgs& a, int teams, bool visc, int mode,
                                    cudaStream_t s) {
    cudaError_t err = upload_gauss_table();
    if (err != cudaSuccess) return err;
    switch (teams) {
        case 8: return launch_teams<8>(a, visc, mode, s);
        case 16: return launch_teams<16>(a, visc, mode, s);
        default: return launch_teams<32>(a, visc, mode, s);
    }
}

cudaError_t launch_node_terms(const NodeArgs& a, cudaStream_t s) {
    if (a.n_nodes <= 0) return cudaSuccess;
    k_node_terms<<<(a.n_nodes + 255) / 256, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_grow(ElemRecord* elems, int32_t n_elems, const double* x, double* fg,
                        const double* rates, const double* angles, double dt, int32_t* rotated,
                        const double* grid_inc, cudaStream_t s) {
    cudaError_t err = upload_gauss_table();
    if (err != cudaSuccess) return err;
    if (n_elems <= 0) return cudaSuccess;
    k_grow<<<(n_elems + 127) / 128, 128, 0, s>>>(elems, n_elems, x, fg, rates, angles, dt, rotated, grid_inc);
    return cudaGetLastError();
}

cudaError_t launch_grid_increment(int32_t n_elems, const GridStep& gs, const double* rel_pos, const double* rel_z,
                                  const int32_t* eflags, double* inc, cudaStream_t s) {
    if (n_elems <= 0) return cudaSuccess;
    if (gs.n < 0 || gs.n > kMaxGridFuncs) return cudaErrorInvalidValue;
    k_grid_increment<<<(n_elems + 127) / 128, 128, 0, s>>>(n_elems, gs, rel_pos, rel_z, eflags, inc);
    return cudaGetLastError();
}

cudaError_t launch_viscosity_surface(const ElemRecord* elems, int32_t n_elems, int32_t n_nodes,
                                     const double* x, const uint8_t* exposed,
                                     const uint8_t* peripodial, double* visc_surface,
                                     cudaStream_t s) {
    cudaError_t err = cudaMemsetAsync(visc_surface, 0, sizeof(double) * (size_t)n_nodes, s);
    if (err != cudaSuccess || n_elems <= 0) return err;
    k_viscosity_surface<<<(n_elems + 255) / 256, 256, 0, s>>>(elems, n_elems, x, exposed, peripodial,
                                                              visc_surface);
    return cudaGetLastError();
}

}  // namespace tfb
