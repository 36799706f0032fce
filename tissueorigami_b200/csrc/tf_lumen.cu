// tf_lumen.cu -- the lumen pressure term of a single tissue (Lumen.cpp; added to the Newton system
// at NewtonRaphsonSolver.cpp:242-249) on the device.
//
// The lumen is bounded by the apical triangles (element nodes 3, 4, 5) of the listed elements. Per
// Newton iteration, at the iterate x:
//   V   = sum over triangles of (1/6) (x3 x x1) . x2           (Lumen::calculateCurrentVolume)
//   rV  = (V - V0) / V0, V0 the ideal volume of the step
//   g_k = x2 x x3, x3 x x1, x1 x x2 for the corners (6 dV/dx_k), fixed components zeroed
//   force on corner k: -bulk rV / (6 V0) g_k on free DoFs         (Lumen::calculateResiduals)
//   Jacobian: bulk / (36 V0^2) G G^T (G = the nodal sums of the g_k) plus, per triangle and corner
//   pair, bulk rV / (6 V0) times the cross-product matrix of the third corner (Lumen::calculateJacobian,
//   written into K by writeLumenJacobianToSystemJacobian, fixed rows and columns left out).
// The triangle-local blocks join nodes of one element, so they go into the element pattern
// through the element's slot map (J = K^T: the reference's block (n_i, n_j) transposed lands in
// block (n_j, n_i)). The rank-one term couples every lumen node; it stays out of J and the host
// applies it with a second solve (Sherman-Morrison).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "tf_internal.cuh"

namespace tfb {
namespace {

constexpr int kLmThreads = 256;

__device__ __forceinline__ void cross3(const double* u, const double* v, double* o) {
    o[0] = u[1] * v[2] - u[2] * v[1];
    o[1] = u[2] * v[0] - u[0] * v[2];
    o[2] = u[0] * v[1] - u[1] * v[0];
}

// per-CTA sums of the triangles' volumes, in a fixed order
__global__ void __launch_bounds__(kLmThreads) k_lm_volume(LumenArgs a) {
    __shared__ double red[kLmThreads];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (t < a.n_tri) {
        const int32_t* c = a.elems[a.tri_elem[t]].conn;
        const double* x1 = a.x + (size_t)c[3] * 3;
        const double* x2 = a.x + (size_t)c[4] * 3;
        const double* x3 = a.x + (size_t)c[5] * 3;
        double cx[3];
        cross3(x3, x1, cx);
        v = 1.0 / 6.0 * (cx[0] * x2[0] + cx[1] * x2[1] + cx[2] * x2[2]);
    }
    red[threadIdx.x] = v;
    __syncthreads();
    for (int off = kLmThreads / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) red[threadIdx.x] += red[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) a.part[blockIdx.x] = red[0];
}

__global__ void k_lm_volume_final(LumenArgs a, int nb) {
    if (threadIdx.x != 0) return;
    double v = 0.0;
    for (int b = 0; b < nb; ++b) v += a.part[b];
    a.state->volume = v;
}

__global__ void __launch_bounds__(kLmThreads) k_lm_terms(LumenArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n_tri) return;
    const ElemRecord& er = a.elems[a.tri_elem[t]];
    const double V0 = a.state->ideal;
    const double rV = (a.state->volume - V0) / V0;
    const double rv6 = rV / 6.0 / V0;
    const double c2 = a.bulk * rV / 6.0 / V0;
    int node[3];
    const double* xs[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        node[k] = er.conn[3 + k];
        xs[k] = a.x + (size_t)node[k] * 3;
    }
    double g[3][3];
    cross3(xs[1], xs[2], g[0]);
    cross3(xs[2], xs[0], g[1]);
    cross3(xs[0], xs[1], g[2]);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int fm = a.fixmask[node[i]];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            if (!((fm >> j) & 1)) {
                atomicAdd(a.g + (size_t)node[i] * 3 + j, -a.bulk * rv6 * g[i][j]);
                atomicAdd(a.G + (size_t)node[i] * 3 + j, g[i][j]);
            }
        }
    }
    // corner pairs: the reference's K block (n_i, n_j)[m][k] -= s[k][m], s = sgn c2 xCap_w; in J
    // (= K^T) that is block (n_j, n_i)[k][m] -= sgn c2 xCap_w[k][m]
    const int which[3][3] = {{-1, 2, 1}, {2, -1, 0}, {1, 0, -1}};
    const double sgn[3][3] = {{0.0, -1.0, 1.0}, {1.0, 0.0, -1.0}, {-1.0, 1.0, 0.0}};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            if (i == j) continue;
            const double* p = xs[which[i][j]];
            const double cap[9] = {0.0, -p[2], p[1], p[2], 0.0, -p[0], -p[1], p[0], 0.0};
            const int slot = er.slots[(3 + j) * 6 + (3 + i)];
            if (slot < 0) continue;  // slave-routed element: refused on the host
            double* B = a.vals + (size_t)slot * 9;
            const int fi = a.fixmask[node[i]], fj = a.fixmask[node[j]];
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int m = 0; m < 3; ++m)
                    if (!((fj >> k) & 1) && !((fi >> m) & 1)) atomicAdd(B + k * 3 + m, -sgn[i][j] * c2 * cap[k * 3 + m]);
        }
}

__global__ void k_lm_set_ideal(LumenState* s, double ideal) {
    if (threadIdx.x == 0) s->ideal = ideal;
}

// out[0] = (a, b1), out[1] = (a, b2): per-CTA sums in fixed order, then one CTA over them
__global__ void __launch_bounds__(kLmThreads) k_dot2(int n, const double* a, const double* b1, const double* b2,
                                                     double* part) {
    __shared__ double r1[kLmThreads], r2[kLmThreads];
    double s1 = 0.0, s2 = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        s1 += a[i] * b1[i];
        s2 += a[i] * b2[i];
    }
    r1[threadIdx.x] = s1;
    r2[threadIdx.x] = s2;
    __syncthreads();
    for (int off = kLmThreads / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            r1[threadIdx.x] += r1[threadIdx.x + off];
            r2[threadIdx.x] += r2[threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = r1[0];
        part[2 * blockIdx.x + 1] = r2[0];
    }
}

__global__ void k_dot2_final(const double* part, int nb, double* out) {
    if (threadIdx.x != 0) return;
    double s1 = 0.0, s2 = 0.0;
    for (int b = 0; b < nb; ++b) {
        s1 += part[2 * b];
        s2 += part[2 * b + 1];
    }
    out[0] = s1;
    out[1] = s2;
}

}  // namespace

int lumen_partials(int n_tri) { return (n_tri + kLmThreads - 1) / kLmThreads + 1; }

cudaError_t launch_lumen_terms(const LumenArgs& a, cudaStream_t s) {
    const int nb = (a.n_tri + kLmThreads - 1) / kLmThreads;
    cudaError_t e = cudaMemsetAsync(a.G, 0, sizeof(double) * 3 * (size_t)a.n_nodes, s);
    if (e != cudaSuccess) return e;
    if (nb > 0) k_lm_volume<<<nb, kLmThreads, 0, s>>>(a);
    k_lm_volume_final<<<1, 32, 0, s>>>(a, nb);
    if (nb > 0) k_lm_terms<<<nb, kLmThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_lumen_set_ideal(LumenState* state, double ideal, cudaStream_t s) {
    k_lm_set_ideal<<<1, 32, 0, s>>>(state, ideal);
    return cudaGetLastError();
}

int dot2_partials() { return 2 * 148 * 2 + 2; }

cudaError_t launch_dot2(int n, const double* a, const double* b1, const double* b2, double* part, double* out,
                        cudaStream_t s) {
    int nb = (n + kLmThreads - 1) / kLmThreads;
    if (nb > 148 * 2) nb = 148 * 2;
    if (nb < 1) nb = 1;
    k_dot2<<<nb, kLmThreads, 0, s>>>(n, a, b1, b2, part);
    k_dot2_final<<<1, 32, 0, s>>>(part, nb, out);
    return cudaGetLastError();
}

}  // namespace tfb
