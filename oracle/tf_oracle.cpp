/*
 * tf_oracle.cpp -- CPU restatement of the TissueOrigami implicit Newton-Raphson path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for tissueorigami_b200's CUDA path and the timed
 * CPU baseline in bench.py. It is never linked into the product.
 *
 * Each function names the reference lines (TissueFolding/SourceCode/...) it follows.
 * The restatement keeps the reference's algorithm literally where it matters for parity:
 * LU-with-partial-pivoting 3x3 inverses (ShapeBase::InvertMatrix, ShapeBase.cpp:3546-3561),
 * the cofactor determinant (ShapeBase.cpp:2264-2271), the naive D81 contraction of the
 * elastic tangent (ShapeBase.cpp:3010-3062), the transposed viscous scatter
 * (ShapeBase.cpp:3154-3160, 3193-3199), the dense Jacobian and its 1e-13 drop
 * (NewtonRaphsonSolver.cpp:766-787) and the transposed solve (iparm[11]=1, :716-723).
 * GSL is replaced by plain loops; the sums run in the same index order as GSL's dgemm.
 *
 * Pinning: against the reference's own recorded regression runs. The growth prologue
 * (tfo_grow) reproduces the growth tensors of the no-Pardiso run 07008 bit for bit
 * (tests/test_golden_growth.py); the Newton step (element forces and tangents, drag, fixed and
 * bound DoFs, Newton loop) reproduces the first step of the Pardiso run 07008 - positions to the
 * recording's 10 digits, the ||dU|| trace to its printed digits (tests/test_golden_newton.py).
 * The viscous (eta != 0) terms, which those runs do not exercise, are checked by finite
 * differences.
 */
#include "tf_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef double M3[3][3];

/* Gauss points and weights of the 6-point prism rule (Prism.cpp:105-130). The reference
 * stores (xi, eta, zeta) per point and calls setShapeFunctionDerivatives(.., eta=gp[0],
 * zeta=gp[2], nu=gp[1]) (Prism.cpp:717-721). */
struct GaussRule {
    double gp[6][3];
    double w[6];
    double dN[6][3][6];  // ShapeFuncDerivatives[g]: rows d/dxi, d/deta, d/dzeta; cols nodes
    GaussRule() {
        const double s = 1.0 / std::pow(3.0, 0.5);
        const double pts[3][2] = {{1.0 / 6.0, 1.0 / 6.0}, {2.0 / 3.0, 1.0 / 6.0}, {1.0 / 6.0, 2.0 / 3.0}};
        for (int g = 0; g < 6; ++g) {
            gp[g][0] = pts[g % 3][0];
            gp[g][1] = pts[g % 3][1];
            gp[g][2] = g < 3 ? s : -s;
            w[g] = 1.0 / 6.0;
        }
        for (int g = 0; g < 6; ++g) {
            // Prism::setShapeFunctionDerivatives (Prism.cpp:597-652)
            const double eta = gp[g][0], nu = gp[g][1], zeta = gp[g][2];
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
    }
};
const GaussRule& rule() {
    static GaussRule r;
    return r;
}

/* ShapeBase::determinant3by3Matrix (ShapeBase.cpp:2264-2271). */
double det3(const M3 m) {
    double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]);
    det -= m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]);
    det += m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    return det;
}

/* ShapeBase::InvertMatrix (ShapeBase.cpp:3546-3561): LU decomposition with partial
 * (row) pivoting as gsl_linalg_LU_decomp does, then column-by-column solves. */
void lu_inverse3(const M3 in, M3 out) {
    double a[3][3];
    int perm[3] = {0, 1, 2};
    std::memcpy(a, in, sizeof(a));
    for (int j = 0; j < 2; ++j) {
        double amax = std::fabs(a[j][j]);
        int ipiv = j;
        for (int i = j + 1; i < 3; ++i) {
            if (std::fabs(a[i][j]) > amax) {
                amax = std::fabs(a[i][j]);
                ipiv = i;
            }
        }
        if (ipiv != j) {
            for (int k = 0; k < 3; ++k) std::swap(a[j][k], a[ipiv][k]);
            std::swap(perm[j], perm[ipiv]);
        }
        const double ajj = a[j][j];
        if (ajj != 0.0) {
            for (int i = j + 1; i < 3; ++i) {
                const double aij = a[i][j] / ajj;
                a[i][j] = aij;
                for (int k = j + 1; k < 3; ++k) a[i][k] -= aij * a[j][k];
            }
        }
    }
    for (int col = 0; col < 3; ++col) {
        double b[3];
        for (int i = 0; i < 3; ++i) b[i] = (perm[i] == col) ? 1.0 : 0.0;
        for (int i = 1; i < 3; ++i)
            for (int k = 0; k < i; ++k) b[i] -= a[i][k] * b[k];
        for (int i = 2; i >= 0; --i) {
            for (int k = i + 1; k < 3; ++k) b[i] -= a[i][k] * b[k];
            b[i] /= a[i][i];
        }
        for (int i = 0; i < 3; ++i) out[i][col] = b[i];
    }
}

void matmul3(const M3 a, const M3 b, M3 c) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += a[i][k] * b[k][j];
            c[i][j] = s;
        }
}
void matmul3_tn(const M3 a, const M3 b, M3 c) {  // a^T b
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += a[k][i] * b[k][j];
            c[i][j] = s;
        }
}
void matmul3_nt(const M3 a, const M3 b, M3 c) {  // a b^T
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += a[i][k] * b[j][k];
            c[i][j] = s;
        }
}

/* dX/dxi at Gauss point g, its determinant and inverse (Prism.cpp:698-733):
 * dXde = (ShapeFuncDer * CurrRelaxedShape)^T. */
void shape_at_gp(const double* xref18, int g, M3 inv, double* det) {
    const GaussRule& R = rule();
    M3 d;
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) {
            double s = 0.0;
            for (int n = 0; n < 6; ++n) s += R.dN[g][k][n] * xref18[n * 3 + r];
            d[r][k] = s;
        }
    *det = det3(d);
    lu_inverse3(d, inv);
}

/* Current deformation gradient at Gauss point g: Jacobian = (dN * x)^T, F = J * InvdXde
 * (Prism.cpp:776-785). */
void jacobian_at_gp(const double* x18, int g, M3 J) {
    const GaussRule& R = rule();
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) {
            double s = 0.0;
            for (int n = 0; n < 6; ++n) s += R.dN[g][k][n] * x18[n * 3 + r];
            J[r][k] = s;
        }
}

/* One element: ShapeBase::calculateForces3D + Prism::calculateCurrNodalForces for the
 * forces, then calculateImplicitKElastic / calculateImplicitKViscous for the tangents. */
int element_kernel(const double* x18, const double* v18, const double* xref18,
                   const double* invfg9, double lam, double mu, double eta, double dt,
                   const uint8_t* fixed18, double* fe_out, double* fv_out, double* ke_out,
                   double* kv_out, double* strain_out) {
    const GaussRule& R = rule();
    M3 InvFg;
    std::memcpy(InvFg, invfg9, sizeof(InvFg));
    double TriPointge[18] = {0}, TriPointgv[18] = {0};
    std::vector<double> TriPointKe(324, 0.0), TriPointKv(324, 0.0), currK(324);
    int bad = 0;

    // Per-GP state kept between the force pass and the tangent passes, as the reference
    // stores FeMatrices, detFs, invJShapeFuncDerStack, elasticStress, viscousStress, D81.
    M3 FeG[6], StressG[6], ViscG[6];
    double detFG[6], detdXdeG[6], dNxG[6][3][6], BG[6][6][18];
    static thread_local double D81[6][3][3][3][3];

    for (int g = 0; g < 6; ++g) {
        M3 invdXde, J, F, Fe, C, invC, S, tmp, Stress, invJ;
        double detdXde;
        shape_at_gp(xref18, g, invdXde, &detdXde);
        jacobian_at_gp(x18, g, J);
        matmul3(J, invdXde, F);
        matmul3(F, InvFg, Fe);
        matmul3_tn(Fe, Fe, C);  // calculateCauchyGreenDeformationTensor (ShapeBase.cpp:2448-2457)
        const double detFe = det3(Fe);
        const double lnJ = std::log(detFe);
        if (!(detFe > 0.0)) ++bad;
        lu_inverse3(C, invC);
        // calculateSForNodalForcesNeoHookean (ShapeBase.cpp:2507-2525)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const double Iij = (i == j ? 1.0 : 0.0);
                S[i][j] = invC[i][j] * (lam * lnJ) + (Iij - invC[i][j]) * mu;
            }
        // updateLagrangianElasticityTensorNeoHookean (ShapeBase.cpp:2527-2545)
        const double multiplier = 2 * (mu - lam * lnJ);
        for (int I = 0; I < 3; ++I)
            for (int Jx = 0; Jx < 3; ++Jx)
                for (int K = 0; K < 3; ++K)
                    for (int L = 0; L < 3; ++L) {
                        const double Iijkl = 0.5 * (invC[I][K] * invC[Jx][L] + invC[I][L] * invC[Jx][K]);
                        D81[g][I][Jx][K][L] = lam * invC[I][Jx] * invC[K][L] + multiplier * Iijkl;
                    }
        if (strain_out) {  // Green strain record (Prism.cpp:829-837)
            double E[3][3];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) E[i][j] = (C[i][j] - (i == j ? 1.0 : 0.0)) * 0.5;
            double* s = strain_out + g * 6;
            s[0] = E[0][0]; s[1] = E[1][1]; s[2] = E[2][2];
            s[3] = 2.0 * E[0][1]; s[4] = 2.0 * E[2][1]; s[5] = 2.0 * E[0][2];
        }
        // calculateCompactStressForNodalForces (ShapeBase.cpp:2547-2568)
        matmul3(Fe, S, tmp);
        matmul3_nt(tmp, Fe, Stress);
        const double invDetFe = 1.0 / detFe;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) Stress[i][j] *= invDetFe;
        const double cs[6] = {Stress[0][0], Stress[1][1], Stress[2][2], Stress[0][1], Stress[2][1], Stress[0][2]};
        // calculateInverseJacobianStackForNodalForces + calculateBTforNodalForces
        // (ShapeBase.cpp:2605-2638): spatial gradients dNx[m][n] = sum_k InvJ[k][m] dN[k][n].
        lu_inverse3(J, invJ);
        const double detF = det3(F);
        double(&dNx)[3][6] = dNxG[g];
        for (int m = 0; m < 3; ++m)
            for (int n = 0; n < 6; ++n) {
                double s = 0.0;
                for (int k = 0; k < 3; ++k) s += invJ[k][m] * R.dN[g][k][n];
                dNx[m][n] = s;
            }
        double(&B)[6][18] = BG[g];
        std::memset(B, 0, sizeof(B));
        for (int n = 0; n < 6; ++n) {  // CoeffMat (Prism.cpp:323-367) applied to the stack
            B[0][n * 3 + 0] = dNx[0][n];
            B[1][n * 3 + 1] = dNx[1][n];
            B[2][n * 3 + 2] = dNx[2][n];
            B[3][n * 3 + 0] = dNx[1][n];
            B[3][n * 3 + 1] = dNx[0][n];
            B[4][n * 3 + 1] = dNx[2][n];
            B[4][n * 3 + 2] = dNx[1][n];
            B[5][n * 3 + 0] = dNx[2][n];
            B[5][n * 3 + 2] = dNx[0][n];
        }
        // ge = B^T * detF * detdXde * compactStress (Prism.cpp:858-860)
        double BTs[18][6];
        for (int p = 0; p < 18; ++p)
            for (int v = 0; v < 6; ++v) BTs[p][v] = (B[v][p] * detF) * detdXde;
        double ge[18], gv[18] = {0};
        for (int p = 0; p < 18; ++p) {
            double s = 0.0;
            for (int v = 0; v < 6; ++v) s += BTs[p][v] * cs[v];
            ge[p] = s;
        }
        M3 visc = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        if (eta != 0.0) {
            // calculateVelocityGradientTensor / RateOfDeformation / ViscousStress / ViscousForces
            // (ShapeBase.cpp:2640-2845)
            double l[6];
            for (int v = 0; v < 6; ++v) {
                double s = 0.0;
                for (int p = 0; p < 18; ++p) s += B[v][p] * v18[p];
                l[v] = s;
            }
            M3 d = {{l[0], 0.5 * l[3], 0.5 * l[5]}, {0.5 * l[3], l[1], 0.5 * l[4]}, {0.5 * l[5], 0.5 * l[4], l[2]}};
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) visc[i][j] = d[i][j] * eta;
            const double csv[6] = {visc[0][0], visc[1][1], visc[2][2], visc[0][1], visc[2][1], visc[0][2]};
            for (int p = 0; p < 18; ++p) {
                double s = 0.0;
                for (int v = 0; v < 6; ++v) s += BTs[p][v] * csv[v];
                gv[p] = s;
            }
        }
        for (int p = 0; p < 18; ++p) {
            TriPointge[p] += ge[p] * R.w[g];
            TriPointgv[p] += gv[p] * R.w[g];
        }
        std::memcpy(FeG[g], Fe, sizeof(M3));
        std::memcpy(StressG[g], Stress, sizeof(M3));
        std::memcpy(ViscG[g], visc, sizeof(M3));
        detFG[g] = detF;
        detdXdeG[g] = detdXde;
    }

    // calculateImplicitKElastic (ShapeBase.cpp:2846-2866): integrals 1 and 2 per GP.
    for (int g = 0; g < 6; ++g) {
        std::fill(currK.begin(), currK.end(), 0.0);
        const M3& Fe = FeG[g];
        const double detF = detFG[g], detdXde = detdXdeG[g], detFe = det3(Fe);
        const double(&dNx)[3][6] = dNxG[g];
        // calculateElasticKIntegral1 (ShapeBase.cpp:3010-3062): the literal loop.
        for (int a = 0; a < 6; ++a)
            for (int b = 0; b < 6; ++b) {
                double Keab[3][3] = {{0}};
                const double DNa[3] = {dNx[0][a], dNx[1][a], dNx[2][a]};
                const double DNb[3] = {dNx[0][b], dNx[1][b], dNx[2][b]};
                for (int i = 0; i < 3; ++i)
                    for (int k = 0; k < 3; ++k) {
                        double value = 0;
                        for (int j = 0; j < 3; ++j)
                            for (int l = 0; l < 3; ++l)
                                for (int I = 0; I < 3; ++I)
                                    for (int Jx = 0; Jx < 3; ++Jx)
                                        for (int K = 0; K < 3; ++K)
                                            for (int L = 0; L < 3; ++L)
                                                value += (Fe[i][I] * Fe[j][Jx] * Fe[k][K] * Fe[l][L] *
                                                          D81[g][I][Jx][K][L] * DNb[l] * DNa[j]);
                        value *= detF * detdXde;
                        value /= detFe;
                        value += Keab[i][k];
                        Keab[i][k] = value;
                    }
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) currK[(a * 3 + i) * 18 + b * 3 + j] += Keab[i][j];
            }
        // calculateElasticKIntegral2 (ShapeBase.cpp:3064-3095)
        for (int a = 0; a < 6; ++a)
            for (int b = 0; b < 6; ++b) {
                double tmp1[3];
                for (int j = 0; j < 3; ++j) {
                    double s = 0.0;
                    for (int i = 0; i < 3; ++i) s += dNx[i][a] * StressG[g][i][j];
                    tmp1[j] = s;
                }
                double q = 0.0;
                for (int j = 0; j < 3; ++j) q += tmp1[j] * dNx[j][b];
                const double value = q * detF * detdXde;
                for (int i = 0; i < 3; ++i) currK[(a * 3 + i) * 18 + b * 3 + i] += value;
            }
        for (int p = 0; p < 324; ++p) TriPointKe[p] += currK[p] * R.w[g];
    }

    // calculateImplicitKViscous (ShapeBase.cpp:2868-2933), skipped when eta == 0.
    if (eta != 0.0) {
        for (int g = 0; g < 6; ++g) {
            std::fill(currK.begin(), currK.end(), 0.0);
            const double(&dNx)[3][6] = dNxG[g];
            const double(&B)[6][18] = BG[g];
            // calculateVelocityGradient (ShapeBase.cpp:3097-3121): L = sum_c v_c (x) dN_c
            M3 Lv = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            for (int c = 0; c < 6; ++c)
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) Lv[i][j] += v18[c * 3 + i] * dNx[j][c];
            M3 P;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) P[i][j] = (i == j ? 1.0 * (1.0 / dt) : 0.0) - Lv[i][j];
            // calculateViscousKIntegral1 (ShapeBase.cpp:3123-3168), transposed write
            for (int a = 0; a < 6; ++a)
                for (int b = 0; b < 6; ++b) {
                    double BaT[3][6], Bb[6][3];
                    for (int i = 0; i < 6; ++i)
                        for (int j = 0; j < 3; ++j) {
                            BaT[j][i] = B[i][a * 3 + j];
                            Bb[i][j] = B[i][b * 3 + j];
                        }
                    for (int i = 3; i < 6; ++i)
                        for (int j = 0; j < 3; ++j) Bb[i][j] = 0.5 * Bb[i][j];
                    M3 BaTBb, K1;
                    for (int i = 0; i < 3; ++i)
                        for (int j = 0; j < 3; ++j) {
                            double s = 0.0;
                            for (int k = 0; k < 6; ++k) s += BaT[i][k] * Bb[k][j];
                            BaTBb[i][j] = s;
                        }
                    matmul3(BaTBb, P, K1);
                    for (int i = 0; i < 3; ++i)
                        for (int j = 0; j < 3; ++j) {
                            const double val = ((K1[i][j] * detFG[g]) * detdXdeG[g]) * eta;
                            currK[(b * 3 + j) * 18 + a * 3 + i] += val;
                        }
                }
            // calculateViscousKIntegral2 (ShapeBase.cpp:3170-3209), transposed write
            for (int a = 0; a < 6; ++a)
                for (int b = 0; b < 6; ++b) {
                    M3 par, K2;
                    for (int i = 0; i < 3; ++i)
                        for (int j = 0; j < 3; ++j) par[i][j] = dNx[i][a] * dNx[j][b] - dNx[i][b] * dNx[j][a];
                    matmul3(ViscG[g], par, K2);
                    for (int i = 0; i < 3; ++i)
                        for (int j = 0; j < 3; ++j) {
                            const double val = (K2[i][j] * detFG[g]) * detdXdeG[g];
                            currK[(b * 3 + j) * 18 + a * 3 + i] += val;
                        }
                }
            for (int p = 0; p < 324; ++p) TriPointKv[p] += currK[p] * R.w[g];
        }
    }

    // calculateForces3D tail (ShapeBase.cpp:2418-2438): negate, skip fixed DoFs.
    for (int p = 0; p < 18; ++p) {
        const bool fx = fixed18 && fixed18[p];
        fe_out[p] = fx ? 0.0 : -TriPointge[p];
        fv_out[p] = fx ? 0.0 : -TriPointgv[p];
    }
    std::memcpy(ke_out, TriPointKe.data(), 324 * sizeof(double));
    std::memcpy(kv_out, TriPointKv.data(), 324 * sizeof(double));
    return bad;
}

void gather18(const int32_t* conn6, const double* x, double* out) {
    for (int n = 0; n < 6; ++n)
        for (int d = 0; d < 3; ++d) out[n * 3 + d] = x[(size_t)conn6[n] * 3 + d];
}

void set_threads(int n_threads) {
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#else
    (void)n_threads;
#endif
}

}  // namespace

extern "C" {

void tfo_shape_derivatives(int n_elems, const double* xref, double* inv_dxde, double* det_dxde) {
    for (int e = 0; e < n_elems; ++e)
        for (int g = 0; g < 6; ++g) {
            M3 inv;
            shape_at_gp(xref + (size_t)e * 18, g, inv, det_dxde + (size_t)e * 6 + g);
            std::memcpy(inv_dxde + ((size_t)e * 6 + g) * 9, inv, sizeof(inv));
        }
}

int tfo_element_forces_and_tangents(int n_elems, const int32_t* conn, const double* xref,
                                    const double* inv_fg, const double* lam, const double* mu,
                                    const double* eta, const double* x, const double* disp_per_dt,
                                    double dt, const uint8_t* fixed, double* f_elastic,
                                    double* f_viscous, double* ke, double* kv, double* strain,
                                    int n_threads) {
    set_threads(n_threads);
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : bad)
    for (int e = 0; e < n_elems; ++e) {
        double x18[18], v18[18];
        uint8_t fx18[18];
        const int32_t* c = conn + (size_t)e * 6;
        gather18(c, x, x18);
        if (disp_per_dt)
            gather18(c, disp_per_dt, v18);
        else
            std::memset(v18, 0, sizeof(v18));
        for (int n = 0; n < 6; ++n)
            for (int d = 0; d < 3; ++d) fx18[n * 3 + d] = fixed ? fixed[(size_t)c[n] * 3 + d] : 0;
        bad += element_kernel(x18, v18, xref + (size_t)e * 18, inv_fg + (size_t)e * 9, lam[e], mu[e],
                              eta ? eta[e] : 0.0, dt, fx18, f_elastic + (size_t)e * 18,
                              f_viscous + (size_t)e * 18, ke + (size_t)e * 324, kv + (size_t)e * 324,
                              strain ? strain + (size_t)e * 36 : nullptr);
    }
    return bad;
}

int tfo_assemble_dense(int n_nodes, int n_elems, const int32_t* conn, const double* xref,
                       const double* inv_fg, const double* lam, const double* mu,
                       const double* eta, const double* uk, const double* un, double dt,
                       const uint8_t* fixed, const double* visc_surface, const double* ext_visc,
                       const int32_t* slave_master, int n_pairs, double* K, double* g,
                       int n_threads) {
    const size_t n = (size_t)n_nodes * 3;
    // setMatricesToZeroInsideIteration (NewtonRaphsonSolver.cpp:95-104)
    std::memset(K, 0, n * n * sizeof(double));
    std::vector<double> ge(n, 0.0), gvInt(n, 0.0), gvExt(n, 0.0), v(n);
    // calculateDisplacementMatrix (NewtonRaphsonSolver.cpp:119-126)
    for (size_t i = 0; i < n; ++i) v[i] = (uk[i] - un[i]) * (1.0 / dt);
    std::vector<double> fe((size_t)n_elems * 18), fv((size_t)n_elems * 18);
    std::vector<double> ke((size_t)n_elems * 324), kv((size_t)n_elems * 324);
    int bad = tfo_element_forces_and_tangents(n_elems, conn, xref, inv_fg, lam, mu, eta, uk,
                                              v.data(), dt, fixed, fe.data(), fv.data(),
                                              ke.data(), kv.data(), nullptr, n_threads);
    // writeForcesTogeAndgvInternal (NewtonRaphsonSolver.cpp:342-348; ShapeBase.cpp:2362-2387)
    for (int e = 0; e < n_elems; ++e)
        for (int a = 0; a < 6; ++a)
            for (int j = 0; j < 3; ++j) {
                const size_t idx = (size_t)conn[e * 6 + a] * 3 + j;
                ge[idx] += fe[(size_t)e * 18 + a * 3 + j];
                gvInt[idx] += fv[(size_t)e * 18 + a * 3 + j];
            }
    // writeImplicitElementalKToJacobian: viscous for all elements, then elastic
    // (NewtonRaphsonSolver.cpp:350-360; ShapeBase.cpp:2935-2983)
    for (int pass = 0; pass < 2; ++pass)
        for (int e = 0; e < n_elems; ++e) {
            if (pass == 0 && !(eta && eta[e] != 0.0)) continue;
            const double* Ke = (pass == 0 ? kv.data() : ke.data()) + (size_t)e * 324;
            for (int a = 0; a < 6; ++a)
                for (int b = 0; b < 6; ++b) {
                    const size_t r0 = (size_t)conn[e * 6 + a] * 3, c0 = (size_t)conn[e * 6 + b] * 3;
                    for (int i = 0; i < 3; ++i)
                        for (int j = 0; j < 3; ++j) K[(r0 + i) * n + c0 + j] += Ke[(a * 3 + i) * 18 + b * 3 + j];
                }
        }
    // calculateExternalViscousForcesForNR / addImplicitKViscousExternalToJacobian
    // (NewtonRaphsonSolver.cpp:362-423), surface based.
    for (int i = 0; i < n_nodes; ++i)
        for (int j = 0; j < 3; ++j) {
            const double sv = visc_surface[i] * ext_visc[i * 3 + j];
            gvExt[(size_t)i * 3 + j] = -(sv * v[(size_t)i * 3 + j]);
        }
    for (int i = 0; i < n_nodes; ++i) {
        const double surfaceAreaPerDt = visc_surface[i] / dt;
        for (int j = 0; j < 3; ++j) {
            const size_t d = (size_t)i * 3 + j;
            K[d * n + d] = surfaceAreaPerDt * ext_visc[d] + K[d * n + d];
        }
    }
    // calculateSumOfInternalForces, addExernalForces (NewtonRaphsonSolver.cpp:441-457)
    for (size_t i = 0; i < n; ++i) g[i] = ge[i] + gvInt[i] + gvExt[i];
    // calcutateFixedK (NewtonRaphsonSolver.cpp:195-219)
    if (fixed)
        for (size_t d = 0; d < n; ++d) {
            if (!fixed[d]) continue;
            g[d] = 0.0;
            for (size_t k = 0; k < n; ++k) {
                const double value = (k == d) ? 1.0 : 0.0;
                K[d * n + k] = value;
                K[k * n + d] = value;
            }
        }
    // calculateBoundKWithSlavesMasterDoF (NewtonRaphsonSolver.cpp:128-183)
    for (int p = 0; p < n_pairs; ++p) {
        const size_t s = (size_t)slave_master[2 * p], m = (size_t)slave_master[2 * p + 1];
        g[m] += g[s];
        g[s] = 0.0;
        for (size_t k = 0; k < n; ++k) {
            K[m * n + k] += K[s * n + k];
            K[s * n + k] = 0.0;
        }
        for (size_t k = 0; k < n; ++k) {
            K[k * n + m] += K[k * n + s];
            K[k * n + s] = 0.0;
        }
        K[s * n + s] = 1.0;
    }
    return bad;
}

int tfo_solve_transposed(int n_int, const double* K, const double* g, const int32_t* slave_master,
                         int n_pairs, int n_refine, double* du) {
    const size_t n = (size_t)n_int;
    // A = K^T with the constructiaForPardiso drop (NewtonRaphsonSolver.cpp:766-787)
    std::vector<double> A(n * n), LU(n * n);
    for (size_t i = 0; i < n; ++i)
        for (size_t j = 0; j < n; ++j) {
            const double kv = K[i * n + j];
            A[j * n + i] = (kv > 1e-13 || kv < -1e-13) ? kv : 0.0;
        }
    LU = A;
    std::vector<size_t> perm(n);
    for (size_t i = 0; i < n; ++i) perm[i] = i;
    int status = 0;
    for (size_t j = 0; j < n; ++j) {
        size_t piv = j;
        double amax = std::fabs(LU[j * n + j]);
        for (size_t i = j + 1; i < n; ++i)
            if (std::fabs(LU[i * n + j]) > amax) {
                amax = std::fabs(LU[i * n + j]);
                piv = i;
            }
        if (amax == 0.0) {
            status = 1;
            continue;
        }
        if (piv != j) {
            for (size_t k = 0; k < n; ++k) std::swap(LU[j * n + k], LU[piv * n + k]);
            std::swap(perm[j], perm[piv]);
        }
        const double inv = 1.0 / LU[j * n + j];
        double* rowj = &LU[j * n];
        for (size_t i = j + 1; i < n; ++i) {
            double* rowi = &LU[i * n];
            const double f = rowi[j] * inv;
            if (f == 0.0) continue;
            rowi[j] = f;
            for (size_t k = j + 1; k < n; ++k) rowi[k] -= f * rowj[k];
        }
    }
    auto lu_solve = [&](const std::vector<double>& b, std::vector<double>& x) {
        x.resize(n);
        for (size_t i = 0; i < n; ++i) x[i] = b[perm[i]];
        for (size_t i = 0; i < n; ++i) {
            double s = x[i];
            for (size_t k = 0; k < i; ++k) s -= LU[i * n + k] * x[k];
            x[i] = s;
        }
        for (size_t ii = n; ii-- > 0;) {
            double s = x[ii];
            for (size_t k = ii + 1; k < n; ++k) s -= LU[ii * n + k] * x[k];
            x[ii] = s / LU[ii * n + ii];
        }
    };
    std::vector<double> b(g, g + n), x, r(n), dx;
    lu_solve(b, x);
    for (int it = 0; it < n_refine; ++it) {
        for (size_t i = 0; i < n; ++i) {
            double s = b[i];
            for (size_t k = 0; k < n; ++k) s -= A[i * n + k] * x[k];
            r[i] = s;
        }
        lu_solve(r, dx);
        for (size_t i = 0; i < n; ++i) x[i] += dx[i];
    }
    for (size_t i = 0; i < n; ++i) du[i] = x[i];
    // equateSlaveDisplacementsToMasters (NewtonRaphsonSolver.cpp:185-193)
    for (int p = 0; p < n_pairs; ++p) du[slave_master[2 * p]] = du[slave_master[2 * p + 1]];
    return status;
}

int tfo_newton_step_dense(int n_nodes, int n_elems, const int32_t* conn, const double* xref,
                          const double* inv_fg, const double* lam, const double* mu,
                          const double* eta, const double* x_n, double dt, double tol,
                          int max_iter, const uint8_t* fixed, const double* visc_surface,
                          const double* ext_visc, const int32_t* slave_master, int n_pairs,
                          double* x_out, double* norms, int n_threads) {
    const size_t n = (size_t)n_nodes * 3;
    std::vector<double> un(x_n, x_n + n), uk(un), K(n * n), g(n), du(n);
    int iteratorK = 0;
    bool converged = false;
    while (!converged) {
        tfo_assemble_dense(n_nodes, n_elems, conn, xref, inv_fg, lam, mu, eta, uk.data(), un.data(),
                           dt, fixed, visc_surface, ext_visc, slave_master, n_pairs, K.data(),
                           g.data(), n_threads);
        tfo_solve_transposed((int)n, K.data(), g.data(), slave_master, n_pairs, 1, du.data());
        // checkConvergenceViaDeltaU (NewtonRaphsonSolver.cpp:807-825)
        double ss = 0.0;
        for (size_t i = 0; i < n; ++i) ss += du[i] * du[i];
        const double d = std::sqrt(ss);
        if (norms) norms[iteratorK] = d;
        converged = !(d > tol);
        // updateUkInIteration (NewtonRaphsonSolver.cpp:844-854)
        for (size_t i = 0; i < n; ++i) uk[i] = uk[i] + du[i];
        iteratorK++;
        if (!converged && iteratorK > max_iter) converged = true;  // Simulation.cpp:6724-6727
    }
    std::memcpy(x_out, uk.data(), n * sizeof(double));
    return iteratorK;
}

int tfo_block_pattern(int n_nodes, int n_elems, const int32_t* conn, int32_t* rowptr,
                      int32_t* colidx) {
    std::vector<std::vector<int32_t>> rows((size_t)n_nodes);
    for (int i = 0; i < n_nodes; ++i) rows[i].push_back(i);
    for (int e = 0; e < n_elems; ++e)
        for (int a = 0; a < 6; ++a)
            for (int b = 0; b < 6; ++b) rows[conn[e * 6 + a]].push_back(conn[e * 6 + b]);
    int32_t nnzb = 0;
    for (int i = 0; i < n_nodes; ++i) {
        std::sort(rows[i].begin(), rows[i].end());
        rows[i].erase(std::unique(rows[i].begin(), rows[i].end()), rows[i].end());
        if (rowptr) rowptr[i] = nnzb;
        if (colidx) std::copy(rows[i].begin(), rows[i].end(), colidx + nnzb);
        nnzb += (int32_t)rows[i].size();
    }
    if (rowptr) rowptr[n_nodes] = nnzb;
    return nnzb;
}

int tfo_assemble_bsr(int n_nodes, int n_elems, const int32_t* conn, const double* xref,
                     const double* inv_fg, const double* lam, const double* mu, const double* eta,
                     const double* uk, const double* un, double dt, const uint8_t* fixed,
                     const double* visc_surface, const double* ext_visc, const int32_t* rowptr,
                     const int32_t* colidx, double* vals, double* g, int n_threads) {
    const size_t n = (size_t)n_nodes * 3;
    const size_t nnzb = (size_t)rowptr[n_nodes];
    std::memset(vals, 0, nnzb * 9 * sizeof(double));
    std::vector<double> v(n);
    for (size_t i = 0; i < n; ++i) v[i] = (uk[i] - un[i]) * (1.0 / dt);
    std::vector<double> fe((size_t)n_elems * 18), fv((size_t)n_elems * 18);
    std::vector<double> ke((size_t)n_elems * 324), kv((size_t)n_elems * 324);
    int bad = tfo_element_forces_and_tangents(n_elems, conn, xref, inv_fg, lam, mu, eta, uk,
                                              v.data(), dt, fixed, fe.data(), fv.data(),
                                              ke.data(), kv.data(), nullptr, n_threads);
    auto slot = [&](int A, int B) -> size_t {
        const int32_t* b0 = colidx + rowptr[A];
        const int32_t* b1 = colidx + rowptr[A + 1];
        return (size_t)(std::lower_bound(b0, b1, B) - colidx);
    };
    std::fill(g, g + n, 0.0);
    for (int e = 0; e < n_elems; ++e) {
        const bool visc = eta && eta[e] != 0.0;
        for (int a = 0; a < 6; ++a) {
            const int A = conn[e * 6 + a];
            for (int j = 0; j < 3; ++j) g[(size_t)A * 3 + j] += fe[(size_t)e * 18 + a * 3 + j] + fv[(size_t)e * 18 + a * 3 + j];
            for (int b = 0; b < 6; ++b) {
                // J block (A,B) entry (i,j) = stored K[(B,j),(A,i)] = TriPointK[b*3+j][a*3+i]
                const int B = conn[e * 6 + b];
                double* blk = vals + slot(A, B) * 9;
                const double* Ke = ke.data() + (size_t)e * 324;
                const double* Kv = kv.data() + (size_t)e * 324;
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        double val = Ke[(b * 3 + j) * 18 + a * 3 + i];
                        if (visc) val += Kv[(b * 3 + j) * 18 + a * 3 + i];
                        blk[i * 3 + j] += val;
                    }
            }
        }
    }
    for (int i = 0; i < n_nodes; ++i) {
        double* blk = vals + slot(i, i) * 9;
        for (int j = 0; j < 3; ++j) {
            const size_t d = (size_t)i * 3 + j;
            blk[j * 3 + j] += visc_surface[i] / dt * ext_visc[d];
            g[d] += -(visc_surface[i] * ext_visc[d] * v[d]);
        }
    }
    if (fixed) {
        for (int A = 0; A < n_nodes; ++A)
            for (int k = rowptr[A]; k < rowptr[A + 1]; ++k) {
                const int B = colidx[k];
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j)
                        if (fixed[(size_t)A * 3 + i] || fixed[(size_t)B * 3 + j])
                            vals[(size_t)k * 9 + i * 3 + j] = (A == B && i == j) ? 1.0 : 0.0;
            }
        for (size_t d = 0; d < n; ++d)
            if (fixed[d]) g[d] = 0.0;
    }
    return bad;
}

void tfo_grow(int n_elems, const int32_t* conn, const double* xref, const double* x,
              const double* rates, const double* angles, double dt, double* fg, double* inv_fg,
              double* det_fg, int32_t* rotated, const double* grid_inc) {
    const GaussRule& R = rule();
    for (int e = 0; e < n_elems; ++e) {
        double x18[18];
        gather18(conn + (size_t)e * 6, x, x18);
        // calculateTriPointFForRatation (ShapeBase.cpp:1935-1948)
        M3 TriPointF = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int g = 0; g < 6; ++g) {
            M3 invdXde, J, F;
            double det;
            shape_at_gp(xref + (size_t)e * 18, g, invdXde, &det);
            jacobian_at_gp(x18, g, J);
            matmul3(J, invdXde, F);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) TriPointF[i][j] += F[i][j] * R.w[g];
        }
        // calculate3DRotMatFromF (ShapeBase.cpp:1999-2041): rotation U V^T of the SVD, i.e.
        // the orthogonal polar factor, computed here by the Newton polar iteration.
        M3 Rm;
        std::memcpy(Rm, TriPointF, sizeof(M3));
        for (int it = 0; it < 100; ++it) {
            M3 inv, next;
            lu_inverse3(Rm, inv);
            double diff = 0.0;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    next[i][j] = 0.5 * (Rm[i][j] + inv[j][i]);
                    diff = std::max(diff, std::fabs(next[i][j] - Rm[i][j]));
                }
            std::memcpy(Rm, next, sizeof(M3));
            if (diff < 1e-15) break;
        }
        bool rot = false;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                if (i != j && (Rm[i][j] > 0.017 || Rm[i][j] < -0.017)) rot = true;
        M3 GrowthStrainsRotMat = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        if (rot) {
            // disassembleRotationMatrixForZ (ShapeBase.cpp:1950-1990)
            const double tz = std::atan2(Rm[0][1], Rm[0][0]);
            if (tz > 0.017 || tz < -0.017) {
                const double c = std::cos(tz), s = std::sin(tz);
                const M3 Rz = {{c, -1.0 * s, 0.0}, {s, c, 0.0}, {0.0, 0.0, 1.0}};
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) GrowthStrainsRotMat[i][j] = Rz[j][i];
            } else {
                rot = false;
            }
        }
        if (rotated) rotated[e] = rot ? 1 : 0;
        // calculateFgFromRates with the uniform function's ShearAngleRotationMatrix
        // (ShapeBase.cpp:471-505; GrowthFunctionTypes.h:22-40)
        const double ang = angles ? angles[e] : 0.0;
        const double c = std::cos(ang), s = std::sin(ang);
        const M3 Ra = {{c, -1.0 * s, 0.0}, {s, c, 0.0}, {0.0, 0.0, 1.0}};
        M3 inc = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, tmp, growthInc, t1, t2, t3;
        inc[0][0] = std::exp(rates[e * 3 + 0] * 1.0 * dt);
        inc[1][1] = std::exp(rates[e * 3 + 1] * 1.0 * dt);
        inc[2][2] = std::exp(rates[e * 3 + 2] * 1.0 * dt);
        matmul3(Ra, inc, tmp);
        matmul3_nt(tmp, Ra, inc);
        // updateGrowthIncrement on a fresh identity (cleanUpGrowthRates, Sim.cpp:8678-8683)
        const M3 I3 = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        matmul3(inc, I3, growthInc);
        if (grid_inc) {  // the grid-based functions of the step, applied after the uniform one
            M3 gi;
            std::memcpy(gi, grid_inc + (size_t)e * 9, sizeof(M3));
            matmul3(gi, growthInc, tmp);
            std::memcpy(growthInc, tmp, sizeof(M3));
        }
        // growShapeByFg (ShapeBase.cpp:1452-1506)
        if (rot) {
            matmul3_tn(GrowthStrainsRotMat, growthInc, tmp);
            matmul3(tmp, GrowthStrainsRotMat, growthInc);
        }
        M3 Fg;
        std::memcpy(Fg, fg + (size_t)e * 9, sizeof(M3));
        matmul3(I3, growthInc, t1);  // plasticDeformationIncrement = I
        matmul3(I3, t1, t2);         // shapeChangeIncrement = I
        matmul3(t2, Fg, t3);
        std::memcpy(fg + (size_t)e * 9, t3, sizeof(M3));
        M3 inv;
        lu_inverse3(t3, inv);
        std::memcpy(inv_fg + (size_t)e * 9, inv, sizeof(M3));
        if (det_fg) det_fg[e] = det3(t3);
    }
}

void tfo_viscosity_surfaces(int n_nodes, int n_elems, const int32_t* conn, const double* x,
                            const uint8_t* exposed, const uint8_t* peripodial,
                            double* visc_surface) {
    std::fill(visc_surface, visc_surface + n_nodes, 0.0);
    // Prism::calculateApicalArea / calculateBasalArea (Prism.cpp:1485-1556)
    auto area = [&](const int32_t* c, int id0, int id1, int id2) {
        const double Threshold = 1E-5;
        double s1[3], s2[3], costet = 0.0, Side1 = 0.0, Side2 = 0.0, Area = 0.0;
        for (int i = 0; i < 3; ++i) {
            s1[i] = x[(size_t)c[id1] * 3 + i] - x[(size_t)c[id0] * 3 + i];
            s2[i] = x[(size_t)c[id2] * 3 + i] - x[(size_t)c[id0] * 3 + i];
            costet += s1[i] * s2[i];
            Side1 += s1[i] * s1[i];
            Side2 += s2[i] * s2[i];
        }
        if (Side1 > Threshold && Side2 > Threshold) {
            Side1 = std::sqrt(Side1);
            Side2 = std::sqrt(Side2);
            costet /= (Side1 * Side2);
            const double sinTetSq = 1 - costet * costet;
            double sintet = 0;
            if (sinTetSq > Threshold) sintet = std::sqrt(sinTetSq);
            Area = Side1 * Side2 * sintet / 2.0;
        }
        return Area;
    };
    // assignViscositySurfaceAreaToNodes (ShapeBase.cpp:3764-3775)
    for (int e = 0; e < n_elems; ++e) {
        const int32_t* c = conn + (size_t)e * 6;
        const bool per = peripodial && peripodial[e];
        const int ap[3] = {per ? 0 : 3, per ? 1 : 4, per ? 2 : 5};
        const int ba[3] = {per ? 3 : 0, per ? 4 : 1, per ? 5 : 2};
        if (exposed[e] & 1) {
            const double A = area(c, ap[0], ap[1], ap[2]);
            for (int i = 0; i < 3; ++i) visc_surface[c[ap[i]]] += A / 3;
        }
        if (exposed[e] & 2) {
            const double A = area(c, ba[0], ba[1], ba[2]);
            for (int i = 0; i < 3; ++i) visc_surface[c[ba[i]]] += A / 3;
        }
    }
}

void tfo_grid_growth_increments(int n_elems, int n_funcs, const int32_t* dims, const double* rates,
                                const double* angles_deg, const double* windows, const double* zrange,
                                const int32_t* fflags, int interpolation, const double* rel_pos,
                                const double* rel_z, const int32_t* eflags, double t, double dt, double* inc,
                                double* per_func) {
    // GridBasedGrowthFunction (GrowthFunctionTypes.h:269-548): per function, the corner tables of
    // every grid cell with the angles brought next to each other (preCalculateAnglesForCompatibleAveraging)
    struct Cell {
        double g[4][3], a[4];
        bool elim[4];
    };
    std::vector<std::vector<Cell>> cells(n_funcs);
    size_t off = 0;
    for (int f = 0; f < n_funcs; ++f) {
        const int nx = dims[2 * f], ny = dims[2 * f + 1];
        const double* G = rates + 3 * off;
        const double* A = angles_deg + off;
        off += (size_t)nx * ny;
        auto gm = [&](int i, int j, int k) { return G[((size_t)i * ny + j) * 3 + k]; };
        auto ang = [&](int i, int j) { return A[(size_t)i * ny + j] * M_PI / 180.0; };
        auto ar_over = [&](int i, int j) {  // aspect ratio x / y against the 1.1 threshold
            double AR = gm(i, j, 0) / gm(i, j, 1);
            if (AR < 0) AR *= -1.0;
            if (AR < 1.0) AR = 1 / AR;
            return !(AR < 1.1);
        };
        cells[f].assign((size_t)(nx - 1) * (ny - 1), Cell());
        for (int IX = 0; IX < nx - 1; ++IX)
            for (int IY = 0; IY < ny - 1; ++IY) {
                Cell& c = cells[f][(size_t)IX * (ny - 1) + IY];
                const int ci[4][2] = {{IX, IY}, {IX + 1, IY}, {IX, IY + 1}, {IX + 1, IY + 1}};
                double angles[4] = {0, 0, 0, 0};
                bool elim[4] = {false, false, false, false};
                for (int q = 0; q < 4; ++q) {
                    for (int k = 0; k < 3; ++k) c.g[q][k] = gm(ci[q][0], ci[q][1], k);
                    if (ar_over(ci[q][0], ci[q][1]))
                        angles[q] = ang(ci[q][0], ci[q][1]);
                    else
                        elim[q] = true;
                }
                for (int q = 0; q < 4; ++q) {
                    while (angles[q] < 0) angles[q] += M_PI;
                    while (angles[q] > M_PI) angles[q] -= M_PI;
                }
                // the base angle: the first corner that was not eliminated; adjustment starts there
                bool selected = false;
                int sel = 3;
                double tet = 0;
                for (int q = 0; q < 4; ++q) {
                    if (!elim[q] && !selected) {
                        tet = angles[q];
                        selected = true;
                    }
                    if (selected) {
                        sel = q;
                        break;
                    }
                }
                bool flip[4] = {false, false, false, false};
                for (int q = sel; q < 4; ++q) {
                    const double d = angles[q] - tet;
                    if (d > 0) {
                        if (d >= M_PI / 4.0 && d < 3.0 * M_PI / 4.0) {
                            angles[q] -= M_PI / 2.0;
                            flip[q] = true;
                        } else if (d >= 3.0 * M_PI / 4.0 && d < 5.0 * M_PI / 4.0) {
                            angles[q] -= M_PI;
                        } else if (d >= 5.0 * M_PI / 4.0 && d < 7.0 * M_PI / 4.0) {
                            angles[q] -= 6.0 * M_PI / 4.0;
                            flip[q] = true;
                        } else if (d >= 7.0 * M_PI / 4.0) {
                            angles[q] -= 2.0 * M_PI;
                        }
                    } else if (d < 0) {
                        if (d <= -M_PI / 4.0 && d > -3.0 * M_PI / 4.0) {
                            angles[q] += M_PI / 2.0;
                            flip[q] = true;
                        } else if (d <= -3.0 * M_PI / 4.0 && d > -5.0 * M_PI / 4.0) {
                            angles[q] += M_PI;
                        } else if (d <= -5.0 * M_PI / 4.0 && d > -7.0 * M_PI / 4.0) {
                            angles[q] += 6.0 * M_PI / 4.0;
                            flip[q] = true;
                        } else if (d <= -7.0 * M_PI / 4.0) {
                            angles[q] += 2.0 * M_PI;
                        }
                    }
                }
                for (int q = 0; q < 4; ++q) {
                    if (flip[q]) std::swap(c.g[q][0], c.g[q][1]);
                    c.a[q] = angles[q];
                    c.elim[q] = elim[q];
                }
            }
    }
    const M3 I3 = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int e = 0; e < n_elems; ++e) {
        M3 growthInc;
        std::memcpy(growthInc, I3, sizeof(M3));
        const int ef = eflags[e];
        const bool ecm = ef & 1, actin = ef & 2, basal = ef & 4, ecm_circ = ef & 8;
        const int ttype = (ef >> 4) & 3;
        for (int f = 0; f < n_funcs; ++f) {
            // Simulation::calculateGrowthGridBased (Simulation.cpp:9038-9085): active on [t0, t1)
            if (!(t >= windows[2 * f] && t < windows[2 * f + 1])) continue;
            const int nx = dims[2 * f], ny = dims[2 * f + 1];
            // ShapeBase::convertRelativePosToGridIndex (ShapeBase.cpp:834-860)
            double rp0 = rel_pos[2 * e] * (float)(nx - 1), rp1 = rel_pos[2 * e + 1] * (float)(ny - 1);
            int IX = (int)std::floor(rp0), IY = (int)std::floor(rp1);
            double FX = rp0 - IX, FY = rp1 - IY;
            if (IX >= nx - 1) {
                IX = nx - 2;
                FX = 1.0;
            } else if (IX < 0) {
                IX = 0;
                FX = 0.0;
            }
            if (IY >= ny - 1) {
                IY = ny - 2;
                FY = 1.0;
            } else if (IY < 0) {
                IY = 0;
                FY = 0.0;
            }
            const Cell& c = cells[f][(size_t)IX * (ny - 1) + IY];
            // ShapeBase::calculateFgFromGridCorners (ShapeBase.cpp:513-658) into a fresh identity
            bool applied = false;
            auto corner_increment = [&](int source, M3 out) {
                std::memcpy(out, I3, sizeof(M3));
                // isGrowthRateApplicable (ShapeBase.cpp:297-334); columnar and peripodial elements
                // only (linker elements, with their transition weights, are not built here)
                if (rel_z[e] < zrange[2 * f] || rel_z[e] > zrange[2 * f + 1]) return;
                const double weight = 1.0;
                if (!((source == 0 && ttype == 0) || (source == 1 && ttype == 1))) return;
                applied = true;
                double growth[3] = {0.0, 0.0, 0.0};
                double angle = 0;
                if (interpolation == 0) {
                    const int q = FX > 0.5 ? (FY > 0.5 ? 3 : 1) : (FY > 0.5 ? 2 : 0);
                    for (int k = 0; k < 3; ++k) growth[k] = c.g[q][k];
                } else {
                    double elimFrac = 0.0;
                    if (c.elim[0]) elimFrac += (1.0 - FX) * (1.0 - FY);
                    if (c.elim[1]) elimFrac += FX * (1.0 - FY);
                    if (c.elim[2]) elimFrac += (1.0 - FX) * FY;
                    if (c.elim[3]) elimFrac += FX * FY;
                    angle = c.a[0] * (1.0 - FX) * (1.0 - FY) + c.a[1] * FX * (1.0 - FY) + c.a[2] * (1.0 - FX) * FY +
                            c.a[3] * FX * FY;
                    if (elimFrac > 0) {
                        if (elimFrac >= 0.9999999)
                            angle = 0.0;
                        else
                            angle /= (1.0 - elimFrac);
                    }
                    for (int k = 0; k < 3; ++k) {
                        growth[k] = c.g[0][k] * (1.0 - FX) * (1.0 - FY) + c.g[1][k] * FX * (1.0 - FY) +
                                    c.g[2][k] * (1.0 - FX) * FY + c.g[3][k] * FX * FY;
                        growth[k] *= weight;
                    }
                }
                if (actin) growth[2] = 0;  // actin-mimicking elements do not grow in height
                for (int k = 0; k < 3; ++k) out[k][k] = std::exp(growth[k] * dt);
                if (angle != 0.0) {
                    const double cs = std::cos(angle), sn = std::sin(angle);
                    const M3 R = {{cs, -1.0 * sn, 0.0}, {sn, cs, 0.0}, {0.0, 0.0, 1.0}};
                    M3 tmp;
                    matmul3(R, out, tmp);
                    matmul3_nt(tmp, R, out);
                }
            };
            const int fl = fflags[f];
            M3 col, per, tmp;
            std::memcpy(col, I3, sizeof(M3));
            std::memcpy(per, I3, sizeof(M3));
            if (fl & 12) {  // apply to basal / lateral ECM
                if ((fl & 4) && ecm && basal) corner_increment(0, col);
                if ((fl & 8) && ecm_circ && !basal) corner_increment(0, col);
            }
            if (!ecm) {
                if (fl & 1) corner_increment(0, col);
                if (fl & 2) corner_increment(1, per);
            }
            if (per_func) {  // this function's own increment (1 + 9 doubles: applied flag, matrix)
                double* o = per_func + ((size_t)f * n_elems + e) * 10;
                o[0] = applied ? 1.0 : 0.0;
                std::memcpy(o + 1, ttype == 1 ? per : col, sizeof(M3));
            }
            // ShapeBase::updateGrowthIncrement (ShapeBase.cpp:764-787)
            if (ttype == 0) {
                matmul3(col, growthInc, tmp);
                std::memcpy(growthInc, tmp, sizeof(M3));
            } else if (ttype == 1) {
                matmul3(per, growthInc, tmp);
                std::memcpy(growthInc, tmp, sizeof(M3));
            }
        }
        std::memcpy(inc + (size_t)e * 9, growthInc, sizeof(M3));
    }
}

int tfo_detect_packing(int n_nodes, int n_elems, const int32_t* conn, const double* x,
                       const int32_t* node_placement, const uint8_t* exposed, const uint8_t* peripodial,
                       int max_pairs, int32_t* pairs, double* packing_threshold) {
    // Simulation::calculateBoundingBox (Simulation.cpp:8388-8425): extent of every node (no node
    // of these tissues belongs only to explicit-ECM elements; no y-symmetry extension)
    double bb0[2] = {100000.0, 100000.0}, bb1[2] = {-100000.0, -100000.0};
    for (int n = 0; n < n_nodes; ++n)
        for (int d = 0; d < 2; ++d) {
            const double p = x[(size_t)n * 3 + d];
            if (p < bb0[d])
                bb0[d] = p;
            else if (p > bb1[d])
                bb1[d] = p;
        }
    const double bbs[2] = {bb1[0] - bb0[0], bb1[1] - bb0[1]};
    // Simulation::getAverageSideLength (Simulation.cpp:3197-3262) with Prism::getApicalSideLengthAverage /
    // getBasalSideLengthAverage (Prism.cpp:1329-1395): columnar elements only; the 10 x 5 grid
    // takes, per element, the apical average, or the basal one for basal / whole-tissue elements
    auto side_avg = [&](const int32_t* c, int o) {
        const int pr[3][2] = {{o, o + 1}, {o, o + 2}, {o + 1, o + 2}};
        double dsum = 0.0;
        int counter = 0;
        for (int i = 0; i < 3; ++i) {
            double d2 = 0.0;
            for (int k = 0; k < 3; ++k) {
                const double dd = x[(size_t)c[pr[i][0]] * 3 + k] - x[(size_t)c[pr[i][1]] * 3 + k];
                d2 += dd * dd;
            }
            if (d2 > 0) {
                dsum += std::pow(d2, 0.5);
                counter++;
            }
        }
        return counter > 0 ? dsum / counter : 0.0;
    };
    double grid[10][5] = {{0}}, gcount[10][5] = {{0}};
    double dsum_col = 0.0;
    int col_counter = 0;
    for (int e = 0; e < n_elems; ++e) {
        if (peripodial && peripodial[e]) continue;  // tissueType 1: the peripodial average is unused here
        const int32_t* c = conn + (size_t)e * 6;
        // element tissuePlacement from its exposed surfaces (ShapeBase::setTissuePlacement):
        // basal (0) when only the basal face is exposed, whole tissue when both are
        const bool basal_like = (exposed[e] & 2) != 0;
        double cur = side_avg(c, 3);
        if (cur > 0) {
            dsum_col += cur;
            col_counter++;
        }
        if (basal_like) {
            cur = side_avg(c, 0);
            if (cur > 0) {
                dsum_col += cur;
                col_counter++;
            }
        }
        // ShapeBase::calculateRelativePosInBoundingBox (ShapeBase.cpp:2091-2095): centre relative to the box
        double cx = 0.0, cy = 0.0;
        for (int a = 0; a < 6; ++a) {
            cx += x[(size_t)c[a] * 3 + 0];
            cy += x[(size_t)c[a] * 3 + 1];
        }
        cx /= 6.0;
        cy /= 6.0;
        int relX = (int)std::floor((cx - bb0[0]) / bbs[0]);
        int relY = (int)std::floor(((cy - bb0[1]) / bbs[1]) / 2.0);
        relX = std::min(9, std::max(0, relX));
        relY = std::min(4, std::max(0, relY));
        grid[relX][relY] += cur;
        gcount[relX][relY]++;
    }
    double gridSq[10][5];
    for (int i = 0; i < 10; ++i)
        for (int j = 0; j < 5; ++j) {
            if (gcount[i][j] > 0) grid[i][j] /= gcount[i][j];
            grid[i][j] *= 0.4;  // Simulation.cpp:8009-8014
            gridSq[i][j] = grid[i][j] * grid[i][j];
        }
    const double col_avg = col_counter > 0 ? dsum_col / col_counter : 0.0;
    if (packing_threshold) *packing_threshold = 0.4 * col_avg;  // Simulation.cpp:8015

    // Node::checkIfNodeHasPacking (Node.cpp:128-146): apical or basal nodes (none is ablated or
    // owned by a lateral element here); Node::immediateNeigs = the nodes sharing an element
    // (ShapeBase::fillNodeNeighbourhood, ShapeBase.cpp:3259-3277)
    // node -> element lists; two nodes are neighbours when one element holds both (checked only
    // for the few pairs that are close enough)
    std::vector<int64_t> eptr((size_t)n_nodes + 1, 0);
    for (size_t k = 0; k < (size_t)n_elems * 6; ++k) eptr[conn[k] + 1]++;
    for (int n = 0; n < n_nodes; ++n) eptr[n + 1] += eptr[n];
    std::vector<int32_t> elist(eptr[n_nodes]);
    {
        std::vector<int64_t> fill(eptr.begin(), eptr.end() - 1);
        for (int e = 0; e < n_elems; ++e)
            for (int a = 0; a < 6; ++a) elist[fill[conn[(size_t)e * 6 + a]]++] = e;
    }
    auto neighbours = [&](int i, int j) {
        for (int64_t k = eptr[i]; k < eptr[i + 1]; ++k) {
            const int32_t* c = conn + (size_t)elist[k] * 6;
            for (int a = 0; a < 6; ++a)
                if (c[a] == j) return true;
        }
        return false;
    };
    auto eligible = [&](int n) { return node_placement[n] == 0 || node_placement[n] == 1; };
    // detectPacingNodes (Simulation.cpp:8036-8070) visits every node pair i < j; the pairs it
    // keeps are those of one placement, not neighbours, closer than the threshold of the master's
    // grid cell floor((pos - box min) / box size). The same pairs are found here through a cell
    // list of the largest threshold, then sorted into the reference's (i, j) visiting order.
    double tmax = 0.0;
    for (int i = 0; i < 10; ++i)
        for (int j = 0; j < 5; ++j) tmax = std::max(tmax, grid[i][j]);
    std::vector<std::pair<int32_t, int32_t>> found;
    if (tmax > 0.0) {
        double lo[3] = {1e300, 1e300, 1e300};
        for (int n = 0; n < n_nodes; ++n)
            for (int d = 0; d < 3; ++d) lo[d] = std::min(lo[d], x[(size_t)n * 3 + d]);
        auto cell = [&](int n, int d) { return (int64_t)std::floor((x[(size_t)n * 3 + d] - lo[d]) / tmax); };
        auto key = [](int64_t a, int64_t b, int64_t c) { return (a * 73856093) ^ (b * 19349663) ^ (c * 83492791); };
        std::vector<std::pair<int64_t, int32_t>> cells;
        for (int n = 0; n < n_nodes; ++n)
            if (eligible(n)) cells.push_back({key(cell(n, 0), cell(n, 1), cell(n, 2)), n});
        std::sort(cells.begin(), cells.end());
        for (int i = 0; i < n_nodes; ++i) {
            if (!eligible(i)) continue;
            int gx = (int)std::floor((x[(size_t)i * 3 + 0] - bb0[0]) / bbs[0]);
            int gy = (int)std::floor((x[(size_t)i * 3 + 1] - bb0[1]) / bbs[1]);
            if (gx < 0 || gx > 9 || gy < 0 || gy > 4) continue;  // outside the reference's grid: never met here
            const double t2 = gridSq[gx][gy];
            const int64_t c0 = cell(i, 0), c1 = cell(i, 1), c2 = cell(i, 2);
            for (int64_t a = c0 - 1; a <= c0 + 1; ++a)
                for (int64_t b = c1 - 1; b <= c1 + 1; ++b)
                    for (int64_t c = c2 - 1; c <= c2 + 1; ++c) {
                        const int64_t k = key(a, b, c);
                        auto it = std::lower_bound(cells.begin(), cells.end(), std::make_pair(k, (int32_t)-1));
                        for (; it != cells.end() && it->first == k; ++it) {
                            const int j = it->second;
                            if (j <= i || node_placement[j] != node_placement[i]) continue;
                            if (cell(j, 0) != a || cell(j, 1) != b || cell(j, 2) != c) continue;  // hash clash
                            double d2 = 0.0;
                            for (int d = 0; d < 3; ++d) {
                                const double dd = x[(size_t)i * 3 + d] - x[(size_t)j * 3 + d];
                                d2 += dd * dd;
                            }
                            if (d2 < t2 && !neighbours(i, j)) found.push_back({i, j});
                        }
                    }
        }
        std::sort(found.begin(), found.end());
    }
    const int np = (int)found.size();
    if (pairs)
        for (int p = 0; p < np && p < max_pairs; ++p) {
            pairs[2 * p] = found[p].first;
            pairs[2 * p + 1] = found[p].second;
        }
    return np;
}


// Simulation::updateNodeMasses (Simulation.cpp:7587-7596) with ShapeBase::assignVolumesToNodes
// (ShapeBase.cpp:3749-3753): every node collects GrownVolume / 6 of each of its elements,
// GrownVolume = det(Fg) x the reference volume (ShapeBase.cpp:1498). The reference volume is
// Prism::calculateReferenceVolume (Prism.cpp:890-923) through
// ShapeBase::calculateVolumeForInputShapeStructure (ShapeBase.cpp:3364-3400): the prism's eight
// triangular faces, each the base of a tetrahedron with the element's centre as apex, |height| x
// area / 3 summed.
void tfo_node_masses(int n_nodes, int n_elems, const int32_t* conn, const double* xref, const double* fg,
                     double* mass) {
    static const int faces[8][3] = {{0, 1, 2}, {3, 4, 5}, {0, 1, 3}, {1, 3, 4}, {1, 2, 4}, {2, 4, 5}, {0, 2, 3}, {2, 3, 5}};
    for (int n = 0; n < n_nodes; ++n) mass[n] = 0.0;
    for (int e = 0; e < n_elems; ++e) {
        const double* X = xref + (size_t)e * 18;
        double c[3] = {0.0, 0.0, 0.0};
        for (int a = 0; a < 6; ++a)
            for (int d = 0; d < 3; ++d) c[d] += X[a * 3 + d];
        for (int d = 0; d < 3; ++d) c[d] /= 6.0;
        double vol = 0.0;
        for (int f = 0; f < 8; ++f) {
            const double* p0 = X + faces[f][0] * 3;
            const double* p1 = X + faces[f][1] * 3;
            const double* p2 = X + faces[f][2] * 3;
            double v1[3], v2[3], vm[3];
            for (int d = 0; d < 3; ++d) {
                v1[d] = p1[d] - p0[d];
                v2[d] = p2[d] - p0[d];
                vm[d] = c[d] - p0[d];
            }
            const double b[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2], v1[0] * v2[1] - v1[1] * v2[0]};
            const double nb = std::sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
            const double area = nb / 2.0;
            double h = (vm[0] * b[0] + vm[1] * b[1] + vm[2] * b[2]) / nb;
            if (h < 0) h = -h;
            vol += 1.0 / 3.0 * (h * area);
        }
        const double* F = fg + (size_t)e * 9;
        const double det = F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) +
                           F[2] * (F[3] * F[7] - F[4] * F[6]);
        const double per_node = det * vol / 6.0;
        for (int a = 0; a < 6; ++a) mass[conn[(size_t)e * 6 + a]] += per_node;
    }
}

// Simulation::calculatePackingForcesImplicit3D (Simulation.cpp:7307-7424) and
// calculatePackingJacobian3D (:7426-7575) for the pairs of one step at positions x: with
// e = (x_i - x_j) / d (d = |x_i - x_j|; e = (1, 0, 0) and d = 1e-3 when d <= 1e-3),
// S = 1 / (1 + exp(5 / thr * 2 * (d - 0.6 thr))) and m the pair's average mass, F_i = 5000 m S e
// is added to forces[i] and subtracted from forces[j]; dfdx[p] = 5000 m [S / d (I - e e^T) +
// dS/dd e e^T], dS/dd = -2 * 5 / thr * S (1 - S), is the 3 x 3 block the reference adds to K as
// -dfdx at (i, i) and (j, j) and +dfdx at (i, j) and (j, i). Row-major blocks; forces may be NULL.
void tfo_packing_terms(int n_pairs, const int32_t* pairs, const double* x, const double* mass, double thr,
                       double* forces, double* dfdx) {
    const double zero_threshold = 1e-3, multiplier = 5000.0, saturation = 5.0;
    for (int p = 0; p < n_pairs; ++p) {
        const int i = pairs[2 * p], j = pairs[2 * p + 1];
        const double dx = x[(size_t)i * 3] - x[(size_t)j * 3], dy = x[(size_t)i * 3 + 1] - x[(size_t)j * 3 + 1],
                     dz = x[(size_t)i * 3 + 2] - x[(size_t)j * 3 + 2];
        double d = std::pow(dx * dx + dy * dy + dz * dz, 0.5);
        const double m = 0.5 * (mass[i] + mass[j]);
        double e[3] = {1.0, 0.0, 0.0};
        if (d > zero_threshold) {
            e[0] = dx / d;
            e[1] = dy / d;
            e[2] = dz / d;
        } else {
            d = zero_threshold;
        }
        const double shifted = d - 0.6 * thr;
        const double S = 1 / (1 + std::exp(saturation / thr * 2.0 * shifted));
        const double fmag = multiplier * m * S;
        if (forces)
            for (int k = 0; k < 3; ++k) {
                forces[(size_t)i * 3 + k] += fmag * e[k];
                forces[(size_t)j * 3 + k] -= fmag * e[k];
            }
        const double dS = (-saturation / thr * 2.0) * S * (1 - S);
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                const double ee = e[r] * e[c];
                const double v = ((r == c ? 1.0 : 0.0) - ee) * (S / d) + ee * dS;
                dfdx[(size_t)p * 9 + r * 3 + c] = v * (multiplier * m);
            }
    }
}


// Lumen (Lumen.cpp) over triangles tri[3t .. 3t+2] (the apical nodes 3, 4, 5 of each lumen
// element, Lumen::Lumen, Lumen.cpp:11-68): Lumen::calculateCurrentVolume (:120-148) sums
// (1/6) (x3 x x1) . x2 per triangle (xCap_k x = x_k x x, Lumen::updateMatrices :92-118).
double tfo_lumen_volume(int n_tri, const int32_t* tri, const double* x) {
    double vol = 0.0;
    for (int t = 0; t < n_tri; ++t) {
        const double* a = x + (size_t)tri[3 * t] * 3;
        const double* b = x + (size_t)tri[3 * t + 1] * 3;
        const double* c = x + (size_t)tri[3 * t + 2] * 3;
        const double cx[3] = {c[1] * a[2] - c[2] * a[1], c[2] * a[0] - c[0] * a[2], c[0] * a[1] - c[1] * a[0]};
        vol += 1.0 / 6.0 * (cx[0] * b[0] + cx[1] * b[1] + cx[2] * b[2]);
    }
    return vol;
}

// Lumen::calculateResiduals (Lumen.cpp:150-192), calculateJacobian (:218-301) and
// writeLumenJacobianToSystemJacobian (:303-329) at positions x with ideal volume V0:
// rV = (V - V0) / V0; per triangle g1 = x2 x x3, g2 = x3 x x1, g3 = x1 x x2 (fixed components
// zeroed); forces[3 node + j] += -bulk rV / (6 V0) g_k[j] on free DoFs; K (3N x 3N, the
// reference's storage) += bulk / (36 V0^2) G G^T with G the nodal sum of the g_k, and per
// triangle and corner pair i != j the block (node_i, node_j)[m][k] -= s[k][m] of
// s = -/+ bulk rV / (6 V0) xCap (the reference's table: (0,1) -xCap3, (0,2) +xCap2, (1,0) +xCap3,
// (1,2) -xCap1, (2,0) -xCap2, (2,1) +xCap1); rows and columns of fixed DoFs are left out.
void tfo_lumen_terms(int n_nodes, int n_tri, const int32_t* tri, const double* x, const uint8_t* fixed,
                     double bulk, double ideal, double* forces, double* K) {
    const size_t n = (size_t)n_nodes * 3;
    const double vol = tfo_lumen_volume(n_tri, tri, x);
    const double rV = (vol - ideal) / ideal;
    const double rv6 = rV / 6.0 / ideal;
    std::vector<double> G(n, 0.0);
    auto cross = [](const double* u, const double* v, double* o) {
        o[0] = u[1] * v[2] - u[2] * v[1];
        o[1] = u[2] * v[0] - u[0] * v[2];
        o[2] = u[0] * v[1] - u[1] * v[0];
    };
    for (int t = 0; t < n_tri; ++t) {
        const double* xs[3] = {x + (size_t)tri[3 * t] * 3, x + (size_t)tri[3 * t + 1] * 3, x + (size_t)tri[3 * t + 2] * 3};
        double g[3][3];
        cross(xs[1], xs[2], g[0]);
        cross(xs[2], xs[0], g[1]);
        cross(xs[0], xs[1], g[2]);
        for (int i = 0; i < 3; ++i) {
            const int node = tri[3 * t + i];
            for (int j = 0; j < 3; ++j) {
                if (!fixed[(size_t)node * 3 + j]) {
                    forces[(size_t)node * 3 + j] += -1.0 * bulk * rv6 * g[i][j];
                } else {
                    g[i][j] = 0.0;
                }
                G[(size_t)node * 3 + j] += g[i][j];
            }
        }
    }
    const double c1 = bulk / ideal / ideal / 36.0, c2 = bulk * rV / 6.0 / ideal;
    for (size_t r = 0; r < n; ++r) {
        if (fixed[r] || G[r] == 0.0) continue;
        for (size_t c = 0; c < n; ++c)
            if (!fixed[c]) K[r * n + c] += c1 * G[r] * G[c];
    }
    for (int t = 0; t < n_tri; ++t) {
        double cap[3][9];
        for (int k = 0; k < 3; ++k) {
            const double* p = x + (size_t)tri[3 * t + k] * 3;
            const double m[9] = {0.0, -p[2], p[1], p[2], 0.0, -p[0], -p[1], p[0], 0.0};
            std::memcpy(cap[k], m, sizeof(m));
        }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                if (i == j) continue;
                int which = 0;
                double sgn = 0.0;
                if (i == 0 && j == 1) { which = 2; sgn = -1.0; }
                if (i == 0 && j == 2) { which = 1; sgn = 1.0; }
                if (i == 1 && j == 0) { which = 2; sgn = 1.0; }
                if (i == 1 && j == 2) { which = 0; sgn = -1.0; }
                if (i == 2 && j == 0) { which = 1; sgn = -1.0; }
                if (i == 2 && j == 1) { which = 0; sgn = 1.0; }
                const int ni = tri[3 * t + i], nj = tri[3 * t + j];
                for (int k = 0; k < 3; ++k)
                    for (int m = 0; m < 3; ++m) {
                        const size_t R = (size_t)ni * 3 + m, C = (size_t)nj * 3 + k;
                        if (fixed[R] || fixed[C]) continue;
                        K[R * n + C] -= sgn * c2 * cap[which][k * 3 + m];
                    }
            }
    }
}

}  // extern "C"
