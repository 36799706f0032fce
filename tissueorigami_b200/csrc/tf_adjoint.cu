// tf_adjoint.cu -- hand-written adjoint (vector-Jacobian) kernels of the implicit growth step.
//
// One time step maps (x_n, Fg_n) to (x_{n+1}, Fg_{n+1}):
//   Fg_{n+1} = inc_n Fg_n,  inc_n = Ra diag(exp(r dt)) Ra^T          (ShapeBase.cpp:471-505, 1452-1506)
//   g(x_{n+1}; x_n, Fg_{n+1}) = 0                                      (the Newton step)
// with g = element forces - A(x_n) eta (x_{n+1} - x_n)/dt (surface drag, NewtonRaphsonSolver.cpp:362-397)
// and J = -dg/dx_{n+1}. For a loss L(x_N) the discrete adjoint of the step is
//   J^T lambda = dL/dx_{n+1}
//   dL/dFg_{n+1} += lambda^T dg/dFg_{n+1}      (k_growth_vjp, through InvFg = Fg^-1)
//   dL/dr        += dL/dFg_{n+1} : d(inc_n Fg_n)/dr,   dL/dFg_n = inc_n^T dL/dFg_{n+1}
//   dL/dx_n       = lambda^T dg/dx_n            (k_drag_vjp + k_area_vjp: drag and exposed areas)
// Fixed degrees of freedom never move, so their adjoints are left at zero. Internal viscosity is
// zero on this path and the growth rotation of ShapeBase::CalculateGrowthRotationByF is held at
// the forward value (it only switches at its 1 degree threshold).
//
// Element-residual VJP: with a = grad N_a (current configuration), dv = det F det(dX/dxi) w_g,
// S = sigma dv and H = sym(sum_a lambda_a a^T), lambda^T f = -sum_g S : H, and
//   d(S:H)/dFe = dv/Je [2 mu H Fe + (lambda tr H - mu (b:H - tr H) - lambda ln Je tr H) Fe^-T],
//   d/dInvFg   = F^T d/dFe   (Fe = F InvFg),   d/dFg = -InvFg^T (d/dInvFg) InvFg^T.
#include <math.h>

#include "tf_internal.cuh"

namespace tfb {
namespace {

constexpr double kW = 1.0 / 6.0;

__device__ __forceinline__ double det3(const double m[3][3]) {
    double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]);
    det -= m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]);
    det += m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    return det;
}

__device__ __forceinline__ void inv3(const double m[3][3], double o[3][3]) {
    const double id = 1.0 / det3(m);
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

__device__ __forceinline__ void mm(const double a[3][3], const double b[3][3], double c[3][3]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) c[i][j] = a[i][0] * b[0][j] + a[i][1] * b[1][j] + a[i][2] * b[2][j];
}

// dN/dxi of the 6-point prism rule (Prism.cpp:105-130, 597-652), computed in place.
__device__ void dN_at(int g, double dN[3][6]) {
    const double s = 0.57735026918962573;  // 1/sqrt(3), the rule's zeta
    const double pts[3][2] = {{1.0 / 6.0, 1.0 / 6.0}, {2.0 / 3.0, 1.0 / 6.0}, {1.0 / 6.0, 2.0 / 3.0}};
    const double eta = pts[g % 3][0], nu = pts[g % 3][1], zeta = g < 3 ? s : -s;
    const double alpha = (1 - zeta) / 2, beta = (1 + zeta) / 2, lambda = 1 - eta - nu;
    const double r[3][6] = {{-alpha, alpha, 0, -beta, beta, 0},
                            {-alpha, 0, alpha, -beta, 0, beta},
                            {-lambda / 2, -eta / 2, -nu / 2, lambda / 2, eta / 2, nu / 2}};
    for (int k = 0; k < 3; ++k)
        for (int n = 0; n < 6; ++n) dN[k][n] = r[k][n];
}

__device__ void grad_xi(const double dN[3][6], const double* pos18, double out[3][3]) {
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) {
            double acc = 0.0;
            for (int n = 0; n < 6; ++n) acc += dN[k][n] * pos18[n * 3 + r];
            out[r][k] = acc;
        }
}

__global__ void k_growth_vjp(const ElemRecord* elems, int32_t n_elems, const double* lam, const uint8_t* fixmask,
                             const double* x1, const double* fg_n, const double* rates, const double* angles,
                             double dt, double* mubar, double* dLdr) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_elems) return;
    const ElemRecord& R = elems[e];
    // increment of the step and Fg_{n+1}
    const double ang = angles ? angles[e] : 0.0;
    const double c = cos(ang), s = sin(ang);
    const double Ra[3][3] = {{c, -1.0 * s, 0.0}, {s, c, 0.0}, {0.0, 0.0, 1.0}};
    double Dg[3];
    for (int i = 0; i < 3; ++i) Dg[i] = exp(rates[(size_t)e * 3 + i] * 1.0 * dt);
    double inc[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) inc[i][j] = Ra[i][0] * Dg[0] * Ra[j][0] + Ra[i][1] * Dg[1] * Ra[j][1] + Ra[i][2] * Dg[2] * Ra[j][2];
    double Fgn[3][3], Fg1[3][3], iFg[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Fgn[i][j] = fg_n[(size_t)e * 9 + i * 3 + j];
    mm(inc, Fgn, Fg1);
    inv3(Fg1, iFg);
    double pos[18], lv[18];
    for (int n = 0; n < 6; ++n) {
        const int nd = R.conn[n];
        const int fm = fixmask[nd];
        for (int k = 0; k < 3; ++k) {
            pos[n * 3 + k] = x1[(size_t)nd * 3 + k];
            lv[n * 3 + k] = ((fm >> k) & 1) ? 0.0 : lam[(size_t)nd * 3 + k];
        }
    }
    double gInv[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int g = 0; g < 6; ++g) {
        double dN[3][6], dX[3][3], invdX[3][3], J[3][3], invJ[3][3], F[3][3], Fe[3][3], iFe[3][3];
        dN_at(g, dN);
        grad_xi(dN, R.xref, dX);
        inv3(dX, invdX);
        grad_xi(dN, pos, J);
        inv3(J, invJ);
        mm(J, invdX, F);
        mm(F, iFg, Fe);
        const double Je = det3(Fe);
        const double lnJ = log(Je);
        const double dv = det3(F) * det3(dX) * kW;
        inv3(Fe, iFe);
        // H = sym(sum_a lambda_a (x) grad N_a)
        double G[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int a = 0; a < 6; ++a) {
            double gr[3];
            for (int m = 0; m < 3; ++m) gr[m] = invJ[0][m] * dN[0][a] + invJ[1][m] * dN[1][a] + invJ[2][m] * dN[2][a];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) G[i][j] += lv[a * 3 + i] * gr[j];
        }
        double H[3][3], b[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                H[i][j] = 0.5 * (G[i][j] + G[j][i]);
                b[i][j] = Fe[i][0] * Fe[j][0] + Fe[i][1] * Fe[j][1] + Fe[i][2] * Fe[j][2];
            }
        const double trH = H[0][0] + H[1][1] + H[2][2];
        double bH = 0.0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) bH += b[i][j] * H[i][j];
        const double cH = R.lam * trH - R.mu * (bH - trH) - R.lam * lnJ * trH;
        double HFe[3][3];
        mm(H, Fe, HFe);
        double M[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) M[i][j] = dv / Je * (2.0 * R.mu * HFe[i][j] + cH * iFe[j][i]);
        // lambda^T f = -sum_g S:H  ->  d/dInvFg = -F^T M
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) gInv[i][j] -= F[0][i] * M[0][j] + F[1][i] * M[1][j] + F[2][i] * M[2][j];
    }
    // dL/dFg_{n+1}: -InvFg^T gInv InvFg^T, plus what later steps left in mubar
    double t1[3][3], mb[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t1[i][j] = iFg[0][i] * gInv[0][j] + iFg[1][i] * gInv[1][j] + iFg[2][i] * gInv[2][j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            mb[i][j] = mubar[(size_t)e * 9 + i * 3 + j] - (t1[i][0] * iFg[j][0] + t1[i][1] * iFg[j][1] + t1[i][2] * iFg[j][2]);
    // through Fg_{n+1} = inc Fg_n: dL/dinc = mb Fg_n^T; dL/dD = Ra^T dL/dinc Ra; dL/dFg_n = inc^T mb
    double dinc[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) dinc[i][j] = mb[i][0] * Fgn[j][0] + mb[i][1] * Fgn[j][1] + mb[i][2] * Fgn[j][2];
    for (int k = 0; k < 3; ++k) {
        double dD = 0.0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) dD += Ra[i][k] * dinc[i][j] * Ra[j][k];
        dLdr[(size_t)e * 3 + k] += dD * dt * Dg[k];
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            mubar[(size_t)e * 9 + i * 3 + j] = inc[0][i] * mb[0][j] + inc[1][i] * mb[1][j] + inc[2][i] * mb[2][j];
}

// Drag part of lambda^T dg/dx_n at the nodes: abar_n = lambda A eta / dt (free DoFs) and the
// area weight q_i = -sum_d lambda_d eta_d v_d with v = (x_{n+1} - x_n)/dt.
__global__ void k_drag_vjp(int32_t n_nodes, const double* lam, const uint8_t* fixmask, const double* x0,
                           const double* x1, const double* visc_surface, const double* ext_visc, double dt,
                           double* abar, double* q) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    const int fm = fixmask[i];
    double qi = 0.0;
    for (int d = 0; d < 3; ++d) {
        const size_t k = (size_t)i * 3 + d;
        if ((fm >> d) & 1) {
            abar[k] = 0.0;
            continue;
        }
        const double v = (x1[k] - x0[k]) * (1.0 / dt);
        abar[k] = lam[k] * visc_surface[i] * ext_visc[k] / dt;
        qi -= lam[k] * ext_visc[k] * v;
    }
    q[i] = qi;
}

// Exposed-triangle area gradient (areas of Prism.cpp:1485-1556, each shared /3 by its nodes).
__device__ void area_vjp(const double* x, int n0, int n1, int n2, double w, const uint8_t* fixmask, double* abar) {
    double e1[3], e2[3], nn[3];
    for (int i = 0; i < 3; ++i) {
        e1[i] = x[(size_t)n1 * 3 + i] - x[(size_t)n0 * 3 + i];
        e2[i] = x[(size_t)n2 * 3 + i] - x[(size_t)n0 * 3 + i];
    }
    const double l1 = e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2];
    const double l2 = e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2];
    nn[0] = e1[1] * e2[2] - e1[2] * e2[1];
    nn[1] = e1[2] * e2[0] - e1[0] * e2[2];
    nn[2] = e1[0] * e2[1] - e1[1] * e2[0];
    const double len = sqrt(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]);
    if (!(l1 > 1e-5 && l2 > 1e-5) || len == 0.0) return;
    const double sin2 = len * len / (l1 * l2);
    if (!(sin2 > 1e-5)) return;
    double u[3] = {nn[0] / len, nn[1] / len, nn[2] / len};
    // d(area)/dp1 = 0.5 e2 x u, d(area)/dp2 = 0.5 u x e1, d(area)/dp0 = -(both)
    double g1[3], g2[3];
    g1[0] = 0.5 * (e2[1] * u[2] - e2[2] * u[1]);
    g1[1] = 0.5 * (e2[2] * u[0] - e2[0] * u[2]);
    g1[2] = 0.5 * (e2[0] * u[1] - e2[1] * u[0]);
    g2[0] = 0.5 * (u[1] * e1[2] - u[2] * e1[1]);
    g2[1] = 0.5 * (u[2] * e1[0] - u[0] * e1[2]);
    g2[2] = 0.5 * (u[0] * e1[1] - u[1] * e1[0]);
    const int nodes[3] = {n0, n1, n2};
    for (int k = 0; k < 3; ++k) {
        const int nd = nodes[k];
        const int fm = fixmask[nd];
        for (int d = 0; d < 3; ++d) {
            if ((fm >> d) & 1) continue;
            const double gv = k == 0 ? -(g1[d] + g2[d]) : (k == 1 ? g1[d] : g2[d]);
            atomicAdd(abar + (size_t)nd * 3 + d, w * gv);
        }
    }
}

__global__ void k_area_vjp(const ElemRecord* elems, int32_t n_elems, const double* x0, const uint8_t* exposed,
                           const uint8_t* peripodial, const double* q, const uint8_t* fixmask, double* abar) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_elems) return;
    const int ex = exposed[e];
    if (!ex) return;
    const int32_t* c = elems[e].conn;
    const bool per = peripodial && peripodial[e];
    if (ex & 1) {
        const int i0 = per ? 0 : 3;
        const double w = (q[c[i0]] + q[c[i0 + 1]] + q[c[i0 + 2]]) / 3.0;
        area_vjp(x0, c[i0], c[i0 + 1], c[i0 + 2], w, fixmask, abar);
    }
    if (ex & 2) {
        const int i0 = per ? 3 : 0;
        const double w = (q[c[i0]] + q[c[i0 + 1]] + q[c[i0 + 2]]) / 3.0;
        area_vjp(x0, c[i0], c[i0 + 1], c[i0 + 2], w, fixmask, abar);
    }
}

// InvFg of every record from an Fg array (the growth state of a recomputed step).
__global__ void k_set_inv_fg(ElemRecord* elems, int32_t n_elems, const double* fg) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_elems) return;
    double m[3][3], o[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) m[i][j] = fg[(size_t)e * 9 + i * 3 + j];
    inv3(m, o);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) elems[e].inv_fg[i * 3 + j] = o[i][j];
}

__global__ void k_mask_fixed(int32_t n_nodes, const uint8_t* fixmask, double* v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    const int fm = fixmask[i];
    for (int d = 0; d < 3; ++d)
        if ((fm >> d) & 1) v[(size_t)i * 3 + d] = 0.0;
}

}  // namespace

cudaError_t launch_growth_vjp(const ElemRecord* elems, int32_t n_elems, const double* lam, const uint8_t* fixmask,
                              const double* x1, const double* fg_n, const double* rates, const double* angles, double dt,
                              double* mubar, double* dLdr, cudaStream_t s) {
    k_growth_vjp<<<(n_elems + 127) / 128, 128, 0, s>>>(elems, n_elems, lam, fixmask, x1, fg_n, rates, angles, dt, mubar, dLdr);
    return cudaGetLastError();
}

cudaError_t launch_position_vjp(const ElemRecord* elems, int32_t n_elems, int32_t n_nodes, const double* lam,
                                const uint8_t* fixmask, const double* x0, const double* x1, const double* visc_surface,
                                const double* ext_visc, const uint8_t* exposed, const uint8_t* peripodial, double dt,
                                double* q, double* abar, cudaStream_t s) {
    k_drag_vjp<<<(n_nodes + 255) / 256, 256, 0, s>>>(n_nodes, lam, fixmask, x0, x1, visc_surface, ext_visc, dt, abar, q);
    k_area_vjp<<<(n_elems + 255) / 256, 256, 0, s>>>(elems, n_elems, x0, exposed, peripodial, q, fixmask, abar);
    return cudaGetLastError();
}

cudaError_t launch_set_inv_fg(ElemRecord* elems, int32_t n_elems, const double* fg, cudaStream_t s) {
    k_set_inv_fg<<<(n_elems + 255) / 256, 256, 0, s>>>(elems, n_elems, fg);
    return cudaGetLastError();
}

cudaError_t launch_mask_fixed(int32_t n_nodes, const uint8_t* fixmask, double* v, cudaStream_t s) {
    k_mask_fixed<<<(n_nodes + 255) / 256, 256, 0, s>>>(n_nodes, fixmask, v);
    return cudaGetLastError();
}

}  // namespace tfb
