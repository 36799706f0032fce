// tf_krylov.cu -- BSR3 sparse kernels and block-Jacobi preconditioned BiCGStab (FP64).
//
// Stands in for the Pardiso transposed solve of NewtonRaphsonSolver::solveWithPardiso
// (TissueFolding/SourceCode/NewtonRaphsonSolver.cpp:498-763): the matrix handed over is
// already the true Jacobian J = K^T, so this solves J du = g directly.
//
// One BiCGStab iteration is five stream-ordered kernels:
//   k_bicg_p   p = r + beta (p - omega v);  phat = D^-1 p             (node-wise)
//   k_spmv     v = J phat;                   alpha = rho / (rhat, v)   (SpMV + 1 dot)
//   k_bicg_s   s = r - alpha v;              shat = D^-1 s             (node-wise)
//   k_spmv     t = J shat;                   omega = (t,s) / (t,t)     (SpMV + 2 dots)
//   k_bicg_xr  x += alpha phat + omega shat; r = s - omega t; rho, ||r||^2 (node-wise + 2 dots)
// Every scalar lives in device memory (KrylovScalars) and is finalised by the last CTA of
// the kernel that reduces it (threadfence + ticket), summing the per-CTA partials in a fixed
// order so results are deterministic. Kernels return at once when the solve has stopped, so
// the host can queue (or graph-replay) chunks of iterations and poll the status rarely.
#include <math.h>

#include "tf_internal.cuh"

namespace tfb {
namespace {

constexpr int kVecThreads = 256;
constexpr int kSpmvThreads = 256;
constexpr int kGroup = 8;  // lanes per block row in the SpMV

__device__ __forceinline__ bool running(const KrylovScalars* sc) {
    return *reinterpret_cast<const volatile int32_t*>(&sc->status) == KS_RUNNING;
}

// Block-wide sum of NDOT values; thread 0 gets the totals.
template <int NDOT>
__device__ __forceinline__ void block_sum(double (&v)[NDOT], double* smem /*[32*NDOT]*/) {
#pragma unroll
    for (int k = 0; k < NDOT; ++k)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], off);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NDOT; ++k) smem[warp * NDOT + k] = v[k];
    __syncthreads();
    const int nw = blockDim.x >> 5;
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NDOT; ++k) {
            double t = lane < nw ? smem[lane * NDOT + k] : 0.0;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
            v[k] = t;
        }
    }
}

// Write this CTA's partials; returns true in every thread of the last CTA to arrive, which
// then holds the grid totals in `tot` (thread 0 only).
template <int NDOT>
__device__ bool grid_sum(double (&v)[NDOT], double* partials, uint32_t* ticket, double (&tot)[NDOT]) {
    __shared__ double smem[32 * NDOT];
    __shared__ bool am_last;
    block_sum<NDOT>(v, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NDOT; ++k) partials[blockIdx.x * NDOT + k] = v[k];
        __threadfence();
        const uint32_t t = atomicAdd(ticket, 1u);
        am_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    double acc[NDOT];
#pragma unroll
    for (int k = 0; k < NDOT; ++k) acc[k] = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x)
#pragma unroll
        for (int k = 0; k < NDOT; ++k) acc[k] += __ldcg(partials + i * NDOT + k);
    __syncthreads();
    block_sum<NDOT>(acc, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NDOT; ++k) tot[k] = acc[k];
        *ticket = 0u;
    }
    return true;
}

__device__ __forceinline__ void apply_dinv(const double* dinv, int n, const double* in, double* out) {
    const double* D = dinv + (size_t)n * 9;
    const double a = in[n * 3], b = in[n * 3 + 1], c = in[n * 3 + 2];
    out[n * 3 + 0] = D[0] * a + D[1] * b + D[2] * c;
    out[n * 3 + 1] = D[3] * a + D[4] * b + D[5] * c;
    out[n * 3 + 2] = D[6] * a + D[7] * b + D[8] * c;
}

__global__ void k_block_jacobi(KrylovWork w) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= w.n_nodes) return;
    const double* B = w.vals + (size_t)w.diag[n] * 9;
    double m[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) m[k] = B[k];
    double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) + m[2] * (m[3] * m[7] - m[4] * m[6]);
    double* D = w.dinv + (size_t)n * 9;
    if (det == 0.0 || !isfinite(det)) {
        atomicOr(w.dflags, DF_SINGULAR_DIAG);
        for (int k = 0; k < 9; ++k) D[k] = (k % 4 == 0) ? 1.0 : 0.0;
        return;
    }
    const double id = 1.0 / det;
    D[0] = (m[4] * m[8] - m[5] * m[7]) * id;
    D[1] = (m[2] * m[7] - m[1] * m[8]) * id;
    D[2] = (m[1] * m[5] - m[2] * m[4]) * id;
    D[3] = (m[5] * m[6] - m[3] * m[8]) * id;
    D[4] = (m[0] * m[8] - m[2] * m[6]) * id;
    D[5] = (m[2] * m[3] - m[0] * m[5]) * id;
    D[6] = (m[3] * m[7] - m[4] * m[6]) * id;
    D[7] = (m[1] * m[6] - m[0] * m[7]) * id;
    D[8] = (m[0] * m[4] - m[1] * m[3]) * id;
}

__global__ void k_krylov_init(KrylovWork w, double rtol, int max_iter) {
    double v[1] = {0.0}, tot[1];
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < w.n_nodes; n += gridDim.x * blockDim.x) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int d = n * 3 + i;
            const double b = w.b[d];
            w.x[d] = 0.0;
            w.r[d] = b;
            w.rhat[d] = b;
            w.p[d] = 0.0;
            w.v[d] = 0.0;
            v[0] += b * b;
        }
    }
    if (grid_sum<1>(v, w.partials, &w.sc->ticket[0], tot) && threadIdx.x == 0) {
        KrylovScalars* sc = w.sc;
        sc->bb = tot[0];
        sc->rr = tot[0];
        sc->rho = tot[0];
        sc->rho_prev = 1.0;
        sc->alpha = 1.0;
        sc->omega = 1.0;
        sc->tol2 = rtol * rtol * tot[0];
        sc->iter = 0;
        sc->max_iter = max_iter;
        sc->finish = 0;
        sc->status = !isfinite(tot[0]) ? KS_NONFINITE : (tot[0] == 0.0 ? KS_CONVERGED : KS_RUNNING);
    }
}

__global__ void k_bicg_p(KrylovWork w) {
    if (!running(w.sc)) return;
    const double beta = (w.sc->rho / w.sc->rho_prev) * (w.sc->alpha / w.sc->omega);
    const double omega = w.sc->omega;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < w.n_nodes; n += gridDim.x * blockDim.x) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int d = n * 3 + i;
            w.p[d] = w.r[d] + beta * (w.p[d] - omega * w.v[d]);
        }
        apply_dinv(w.dinv, n, w.p, w.phat);
    }
}

__global__ void k_bicg_s(KrylovWork w) {
    if (!running(w.sc)) return;
    const double alpha = w.sc->alpha;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < w.n_nodes; n += gridDim.x * blockDim.x) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int d = n * 3 + i;
            w.s[d] = w.r[d] - alpha * w.v[d];
        }
        apply_dinv(w.dinv, n, w.s, w.shat);
    }
}

__global__ void k_bicg_xr(KrylovWork w) {
    if (!running(w.sc)) return;
    const double alpha = w.sc->alpha, omega = w.sc->omega;
    double v[2] = {0.0, 0.0}, tot[2];
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < w.n_nodes; n += gridDim.x * blockDim.x) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int d = n * 3 + i;
            w.x[d] += alpha * w.phat[d] + omega * w.shat[d];
            const double r = w.s[d] - omega * w.t[d];
            w.r[d] = r;
            v[0] += w.rhat[d] * r;
            v[1] += r * r;
        }
    }
    if (grid_sum<2>(v, w.partials, &w.sc->ticket[3], tot) && threadIdx.x == 0) {
        KrylovScalars* sc = w.sc;
        sc->rho_prev = sc->rho;
        sc->rho = tot[0];
        sc->rr = tot[1];
        sc->iter += 1;
        int st = KS_RUNNING;
        if (!isfinite(tot[0]) || !isfinite(tot[1]))
            st = KS_NONFINITE;
        else if (tot[1] <= sc->tol2)
            st = KS_CONVERGED;
        else if (sc->iter >= sc->max_iter)
            st = KS_MAXIT;
        else if (tot[0] == 0.0 || sc->omega == 0.0)
            st = KS_BREAKDOWN;
        sc->status = st;
    }
}

// y = J x for G lanes per block row; NDOT = 0, 1 (kind 1: (rhat, y) -> alpha) or
// 2 (kind 2: (y, s), (y, y) -> omega).
template <int NDOT>
__global__ void __launch_bounds__(kSpmvThreads) k_spmv(KrylovWork w, const double* __restrict__ xin,
                                                       double* __restrict__ yout, int check_status) {
    if (check_status && !running(w.sc)) return;
    const int gl = threadIdx.x & (kGroup - 1);
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) / kGroup;
    double y0 = 0.0, y1 = 0.0, y2 = 0.0;
    if (row < w.n_nodes) {
        const int k1 = __ldg(w.rowptr + row + 1);
        for (int k = __ldg(w.rowptr + row) + gl; k < k1; k += kGroup) {
            const int c = __ldg(w.colidx + k);
            const double* B = w.vals + (size_t)k * 9;
            const double x0 = __ldg(xin + c * 3), x1 = __ldg(xin + c * 3 + 1), x2 = __ldg(xin + c * 3 + 2);
            y0 += __ldg(B + 0) * x0 + __ldg(B + 1) * x1 + __ldg(B + 2) * x2;
            y1 += __ldg(B + 3) * x0 + __ldg(B + 4) * x1 + __ldg(B + 5) * x2;
            y2 += __ldg(B + 6) * x0 + __ldg(B + 7) * x1 + __ldg(B + 8) * x2;
        }
    }
#pragma unroll
    for (int off = kGroup / 2; off > 0; off >>= 1) {
        y0 += __shfl_xor_sync(0xffffffffu, y0, off);
        y1 += __shfl_xor_sync(0xffffffffu, y1, off);
        y2 += __shfl_xor_sync(0xffffffffu, y2, off);
    }
    double v[NDOT > 0 ? NDOT : 1];
    v[0] = 0.0;
    if (NDOT == 2) v[NDOT - 1] = 0.0;
    if (row < w.n_nodes && gl == 0) {
        yout[row * 3 + 0] = y0;
        yout[row * 3 + 1] = y1;
        yout[row * 3 + 2] = y2;
        if (NDOT == 1) {
            v[0] = w.rhat[row * 3] * y0 + w.rhat[row * 3 + 1] * y1 + w.rhat[row * 3 + 2] * y2;
        } else if (NDOT == 2) {
            v[0] = w.s[row * 3] * y0 + w.s[row * 3 + 1] * y1 + w.s[row * 3 + 2] * y2;
            v[NDOT - 1] = y0 * y0 + y1 * y1 + y2 * y2;
        }
    }
    if (NDOT == 0) return;
    double tot[NDOT > 0 ? NDOT : 1];
    const bool last = grid_sum<(NDOT > 0 ? NDOT : 1)>(v, w.partials, &w.sc->ticket[NDOT], tot);
    if (!last || threadIdx.x != 0) return;
    KrylovScalars* sc = w.sc;
    if (NDOT == 1) {
        if (!isfinite(tot[0]))
            sc->status = KS_NONFINITE;
        else if (tot[0] == 0.0)
            sc->status = KS_BREAKDOWN;
        else
            sc->alpha = sc->rho / tot[0];
    } else {
        const double ts = tot[0], tt = tot[NDOT - 1];
        if (!isfinite(ts) || !isfinite(tt))
            sc->status = KS_NONFINITE;
        else
            sc->omega = tt == 0.0 ? 0.0 : ts / tt;
    }
}

// Slot of the diagonal block of every block row (binary search of the sorted column list).
__global__ void k_find_diag(const int32_t* rowptr, const int32_t* colidx, int32_t n, int32_t* diag,
                            int32_t* dflags) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    int lo = rowptr[r], hi = rowptr[r + 1] - 1, found = -1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        const int c = colidx[mid];
        if (c == r) {
            found = mid;
            break;
        }
        if (c < r)
            lo = mid + 1;
        else
            hi = mid - 1;
    }
    if (found < 0) {
        atomicOr(dflags, DF_PATTERN_MISS);
        found = rowptr[r];  // keep the index in range; the flag reports the missing diagonal
    }
    diag[r] = found;
}

// du[slave] = du[master] (equateSlaveDisplacementsToMasters), then uk += du and ||du||^2.
__global__ void k_equate_slaves(double* du, const int32_t* slaves, const int32_t* masters, int32_t n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) du[slaves[i]] = du[masters[i]];
}

__global__ void k_newton_update(KrylovWork w, double* uk) {
    double v[1] = {0.0}, tot[1];
    const int n3 = w.n_nodes * 3;
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < n3; d += gridDim.x * blockDim.x) {
        const double du = w.x[d];
        v[0] += du * du;
        uk[d] = uk[d] + du;
    }
    if (grid_sum<1>(v, w.partials, &w.sc->ticket[5], tot) && threadIdx.x == 0) w.sc->du2 = tot[0];
}

}  // namespace

int vec_grid(int n_nodes) {
    int g = (n_nodes + kVecThreads - 1) / kVecThreads;
    return g < 1 ? 1 : (g > 148 * 8 ? 148 * 8 : g);
}

int spmv_grid(int n_nodes) {
    const int rows_per_cta = kSpmvThreads / kGroup;
    const int g = (n_nodes + rows_per_cta - 1) / rows_per_cta;
    return g < 1 ? 1 : g;
}

cudaError_t launch_find_diag(const int32_t* rowptr, const int32_t* colidx, int32_t n, int32_t* diag,
                             int32_t* dflags, cudaStream_t s) {
    k_find_diag<<<(n + 255) / 256, 256, 0, s>>>(rowptr, colidx, n, diag, dflags);
    return cudaGetLastError();
}

cudaError_t launch_block_jacobi_setup(const KrylovWork& w, cudaStream_t s) {
    k_block_jacobi<<<(w.n_nodes + 255) / 256, 256, 0, s>>>(w);
    return cudaGetLastError();
}

cudaError_t launch_krylov_init(const KrylovWork& w, double rtol, int max_iter, cudaStream_t s) {
    k_krylov_init<<<vec_grid(w.n_nodes), kVecThreads, 0, s>>>(w, rtol, max_iter);
    return cudaGetLastError();
}

cudaError_t launch_bicgstab_iteration(const KrylovWork& w, cudaStream_t s) {
    const int vg = vec_grid(w.n_nodes), sg = spmv_grid(w.n_nodes);
    k_bicg_p<<<vg, kVecThreads, 0, s>>>(w);
    k_spmv<1><<<sg, kSpmvThreads, 0, s>>>(w, w.phat, w.v, 1);
    k_bicg_s<<<vg, kVecThreads, 0, s>>>(w);
    k_spmv<2><<<sg, kSpmvThreads, 0, s>>>(w, w.shat, w.t, 1);
    k_bicg_xr<<<vg, kVecThreads, 0, s>>>(w);
    return cudaGetLastError();
}

cudaError_t launch_spmv(const KrylovWork& w, const double* xin, double* yout, cudaStream_t s) {
    k_spmv<0><<<spmv_grid(w.n_nodes), kSpmvThreads, 0, s>>>(w, xin, yout, 0);
    return cudaGetLastError();
}

cudaError_t launch_newton_update(const KrylovWork& w, double* uk, const int32_t* slaves,
                                 const int32_t* masters, int32_t n_pairs, cudaStream_t s) {
    if (n_pairs > 0) k_equate_slaves<<<(n_pairs + 255) / 256, 256, 0, s>>>(w.x, slaves, masters, n_pairs);
    k_newton_update<<<vec_grid(w.n_nodes), kVecThreads, 0, s>>>(w, uk);
    return cudaGetLastError();
}

}  // namespace tfb
