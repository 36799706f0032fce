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

// Partial row product of one lane: blocks k0, k0+G, ... of the row. x is read with ordinary
// L1-cached loads (ld.ca; consecutive rows share most of their columns): inside a persistent
// kernel it was written by other CTAs before the group barrier, whose fence makes those writes
// visible to these loads. Never the read-only path (ld.global.nc), which assumes data that does
// not change during the kernel.
template <int G>
__device__ __forceinline__ void row_dot(const KrylovWork& w, int k0, int k1, const double* __restrict__ xin,
                                        double& y0, double& y1, double& y2) {
    // the next block's column index is loaded one iteration ahead, so that the x gathers of a
    // block do not wait for its column index
    int c = k0 < k1 ? __ldg(w.colidx + k0) : 0;
    for (int k = k0; k < k1; k += G) {
        const int cn = k + G < k1 ? __ldg(w.colidx + k + G) : 0;
        const double* B = w.vals + (size_t)k * 9;
        const double x0 = __ldca(xin + c * 3), x1 = __ldca(xin + c * 3 + 1), x2 = __ldca(xin + c * 3 + 2);
        y0 += __ldg(B + 0) * x0 + __ldg(B + 1) * x1 + __ldg(B + 2) * x2;
        y1 += __ldg(B + 3) * x0 + __ldg(B + 4) * x1 + __ldg(B + 5) * x2;
        y2 += __ldg(B + 6) * x0 + __ldg(B + 7) * x1 + __ldg(B + 8) * x2;
        c = cn;
    }
}

// y += the row's packing blocks outside the element pattern (none when w.pk_ptr is NULL); lane gl
// of the row's G takes every G-th of them.
template <int G>
__device__ __forceinline__ void row_aux(const KrylovWork& w, int row, int gl, const double* __restrict__ xin,
                                        double& y0, double& y1, double& y2) {
    if (!w.pk_ptr) return;
    for (int k = w.pk_ptr[row] + gl; k < w.pk_ptr[row + 1]; k += G) {
        const int c = w.pk_col[k];
        const double* B = w.pk_vals + (size_t)w.pk_blk[k] * 9;
        const double x0 = __ldca(xin + c * 3), x1 = __ldca(xin + c * 3 + 1), x2 = __ldca(xin + c * 3 + 2);
        y0 += B[0] * x0 + B[1] * x1 + B[2] * x2;
        y1 += B[3] * x0 + B[4] * x1 + B[5] * x2;
        y2 += B[6] * x0 + B[7] * x1 + B[8] * x2;
    }
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
        sc->method = KM_BICGSTAB;
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
        row_dot<kGroup>(w, __ldg(w.rowptr + row) + gl, __ldg(w.rowptr + row + 1), xin, y0, y1, y2);
        row_aux<kGroup>(w, row, gl, xin, y0, y1, y2);
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

// True residual r = b - J x with ||r||^2 summed in fixed order into sc->du2 (the iterative
// refinement of tf_solve reads it; the Newton loop does not use this kernel).
__global__ void __launch_bounds__(kSpmvThreads) k_residual(KrylovWork w, const double* __restrict__ xin,
                                                           const double* __restrict__ b, double* __restrict__ rout) {
    const int gl = threadIdx.x & (kGroup - 1);
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) / kGroup;
    double y0 = 0.0, y1 = 0.0, y2 = 0.0;
    if (row < w.n_nodes) {
        row_dot<kGroup>(w, __ldg(w.rowptr + row) + gl, __ldg(w.rowptr + row + 1), xin, y0, y1, y2);
        row_aux<kGroup>(w, row, gl, xin, y0, y1, y2);
    }
#pragma unroll
    for (int off = kGroup / 2; off > 0; off >>= 1) {
        y0 += __shfl_xor_sync(0xffffffffu, y0, off);
        y1 += __shfl_xor_sync(0xffffffffu, y1, off);
        y2 += __shfl_xor_sync(0xffffffffu, y2, off);
    }
    double v[1] = {0.0}, tot[1];
    if (row < w.n_nodes && gl == 0) {
        const double r0 = b[row * 3] - y0, r1 = b[row * 3 + 1] - y1, r2 = b[row * 3 + 2] - y2;
        rout[row * 3] = r0;
        rout[row * 3 + 1] = r1;
        rout[row * 3 + 2] = r2;
        v[0] = r0 * r0 + r1 * r1 + r2 * r2;
    }
    if (grid_sum<1>(v, w.partials, &w.sc->ticket[4], tot) && threadIdx.x == 0) w.sc->du2 = tot[0];
}

__global__ void k_axpy(int n, double a, const double* __restrict__ x, double* __restrict__ y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] += a * x[i];
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

// ---- persistent cooperative solve over a batch of tissues -------------------------------
//
// k_bicgstab_batched runs block-Jacobi BiCGStab for every active tissue of a batch in one
// cooperative launch. Tissue t owns a group of CTAs (BatchPlan) and each CTA of the group a
// contiguous range of the tissue's block rows. The five phases of an iteration are separated
// by the group's barrier; each of the three reductions is summed by every CTA of the group
// from the same per-CTA partials in the same order, so the group holds bit-identical scalars
// and takes one convergence decision. Partials alternate between two buffers so a CTA can
// write the next reduction while a slower one still reads the previous. Groups are
// independent: a tissue that converges frees its CTAs while the others iterate on. The
// barrier wait is bounded: a CTA that waits longer than kBarrierTimeoutCycles sets
// DF_BARRIER_TIMEOUT and returns; the cooperative launch guarantees co-residency, so this
// never fires in a correct launch.

// Barrier wait bound in SM clock cycles (~2 s at the B200 boost clock).
constexpr long long kBarrierTimeoutCycles = 4000000000ll;

__device__ bool group_barrier(GridBarrier* bar, int n_group, int32_t* dflags) {
    __shared__ int ok;
    if (n_group == 1) {
        __syncthreads();
        return true;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        volatile uint32_t* vgen = &bar->gen;
        const uint32_t g = *vgen;
        __threadfence();
        const uint32_t arrived = atomicAdd(&bar->count, 1u);
        if (arrived == (uint32_t)n_group - 1) {
            bar->count = 0u;
            __threadfence();
            atomicAdd(&bar->gen, 1u);
        } else {
            const long long t0 = clock64();
            unsigned polls = 0;
            while (*vgen == g) {
                if ((++polls & 255u) == 0u && clock64() - t0 > kBarrierTimeoutCycles) {
                    atomicOr(dflags, DF_BARRIER_TIMEOUT);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        if (*reinterpret_cast<volatile int32_t*>(dflags) & DF_BARRIER_TIMEOUT) ok = 0;
    }
    __syncthreads();
    return ok != 0;
}

// Sum NDOT per-CTA partials of the n_group CTAs (same order in every CTA); all threads get the totals.
template <int NDOT>
__device__ void sum_partials(const double* buf, int n_group, double (&tot)[NDOT], double* smem, double* sbcast) {
    double acc[NDOT];
#pragma unroll
    for (int k = 0; k < NDOT; ++k) acc[k] = 0.0;
    for (int i = threadIdx.x; i < n_group; i += blockDim.x)
#pragma unroll
        for (int k = 0; k < NDOT; ++k) acc[k] += __ldcg(buf + i * NDOT + k);
    block_sum<NDOT>(acc, smem);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NDOT; ++k) sbcast[k] = acc[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NDOT; ++k) tot[k] = sbcast[k];
    __syncthreads();
}

template <int NDOT>
__device__ void write_partials(double (&v)[NDOT], double* buf, int local, double* smem) {
    block_sum<NDOT>(v, smem);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NDOT; ++k) buf[local * NDOT + k] = v[k];
}

// y = J x for rows [r0, r1) with kGroup lanes per row; returns this thread's share of the
// dots (rhat,y) [KIND 1], (s,y), (y,y) [KIND 2] or (p,y) [KIND 3].
template <int KIND>
__device__ __forceinline__ void spmv_rows(const KrylovWork& w, int r0, int r1, const double* __restrict__ xin,
                                          double* __restrict__ yout, double& d0, double& d1) {
    const int gl = threadIdx.x & (kGroup - 1);
    const int groups = blockDim.x / kGroup;
    // the block range of the thread's next row is loaded one row ahead
    int row_n = r0 + threadIdx.x / kGroup;
    int ka = row_n < r1 ? __ldg(w.rowptr + row_n) : 0, kz = row_n < r1 ? __ldg(w.rowptr + row_n + 1) : 0;
    for (int rb = r0; rb < r1; rb += groups) {
        const int row = rb + threadIdx.x / kGroup;
        row_n = row + groups;
        const int ka_n = row_n < r1 ? __ldg(w.rowptr + row_n) : 0, kz_n = row_n < r1 ? __ldg(w.rowptr + row_n + 1) : 0;
        double y0 = 0.0, y1 = 0.0, y2 = 0.0;
        // the row's entries of the dot products' other vectors, loaded by the reducing lane ahead
        // of the row product so that their latency overlaps it
        double a[3] = {0.0, 0.0, 0.0}, b[3] = {0.0, 0.0, 0.0};
        if (row < r1 && gl == 0) {
            const double* av = KIND == 1 ? w.rhat : (KIND == 3 || KIND == 4 ? w.p : w.s);
#pragma unroll
            for (int i = 0; i < 3; ++i) a[i] = av[row * 3 + i];
            if (KIND == 4)
#pragma unroll
                for (int i = 0; i < 3; ++i) b[i] = w.r[row * 3 + i];
        }
        if (row < r1) {
            row_dot<kGroup>(w, ka + gl, kz, xin, y0, y1, y2);
            row_aux<kGroup>(w, row, gl, xin, y0, y1, y2);
        }
        ka = ka_n;
        kz = kz_n;
#pragma unroll
        for (int off = kGroup / 2; off > 0; off >>= 1) {
            y0 += __shfl_xor_sync(0xffffffffu, y0, off);
            y1 += __shfl_xor_sync(0xffffffffu, y1, off);
            y2 += __shfl_xor_sync(0xffffffffu, y2, off);
        }
        if (row < r1 && gl == 0) {
            yout[row * 3 + 0] = y0;
            yout[row * 3 + 1] = y1;
            yout[row * 3 + 2] = y2;
            // KIND 1: (rhat, y); 3: (p, y); 4 (MINRES): (v, A v) and (v, r1), v in p, r1 in r;
            // 2: (s, y) and (y, y)
            d0 += a[0] * y0 + a[1] * y1 + a[2] * y2;
            if (KIND == 4)
                d1 += a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
            else if (KIND == 2)
                d1 += y0 * y0 + y1 * y1 + y2 * y2;
        }
    }
}

// The persistent solve keeps a node block's 3x3 inverse in FP32 at dinv32(w) + 9 n (it only
// preconditions: the residual and the stopping test stay FP64); products are formed in FP64.
__device__ __forceinline__ float* dinv32(const KrylovWork& w) { return reinterpret_cast<float*>(w.dinv); }

__device__ __forceinline__ void apply_dinv32(const KrylovWork& w, int n, const double* in, double* out) {
    const float* D = dinv32(w) + (size_t)n * 9;
    const double a = in[n * 3], b = in[n * 3 + 1], c = in[n * 3 + 2];
    out[n * 3 + 0] = (double)D[0] * a + (double)D[1] * b + (double)D[2] * c;
    out[n * 3 + 1] = (double)D[3] * a + (double)D[4] * b + (double)D[5] * c;
    out[n * 3 + 2] = (double)D[6] * a + (double)D[7] * b + (double)D[8] * c;
}

// |D_n|^-1 = V |Lambda|^-1 V^T of the symmetric part of node n's diagonal block (cyclic Jacobi
// rotations): a symmetric positive definite block preconditioner for an indefinite symmetric J
// (MINRES). An eigenvalue below 1e-300 in magnitude is taken as 1.
__device__ __forceinline__ void block_abs_inverse_row(const KrylovWork& w, int n) {
    const double* B = w.vals + (size_t)w.diag[n] * 9;
    double A[9], V[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) A[r * 3 + c] = 0.5 * (B[r * 3 + c] + B[c * 3 + r]);
    for (int sweep = 0; sweep < 12; ++sweep) {
        const double off = A[1] * A[1] + A[2] * A[2] + A[5] * A[5];
        const double dia = A[0] * A[0] + A[4] * A[4] + A[8] * A[8];
        if (!(off > 1e-32 * dia)) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                const double apq = A[p * 3 + q];
                if (apq == 0.0) continue;
                const double tau = (A[q * 3 + q] - A[p * 3 + p]) / (2.0 * apq);
                const double tt = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                const double c = 1.0 / sqrt(1.0 + tt * tt), s = tt * c;
                for (int k = 0; k < 3; ++k) {
                    const double akp = A[k * 3 + p], akq = A[k * 3 + q];
                    A[k * 3 + p] = c * akp - s * akq;
                    A[k * 3 + q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {
                    const double apk = A[p * 3 + k], aqk = A[q * 3 + k];
                    A[p * 3 + k] = c * apk - s * aqk;
                    A[q * 3 + k] = s * apk + c * aqk;
                }
                A[p * 3 + q] = A[q * 3 + p] = 0.0;
                for (int k = 0; k < 3; ++k) {
                    const double vkp = V[k * 3 + p], vkq = V[k * 3 + q];
                    V[k * 3 + p] = c * vkp - s * vkq;
                    V[k * 3 + q] = s * vkp + c * vkq;
                }
            }
    }
    double inv[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double l = fabs(A[k * 4]);
        inv[k] = (l > 1e-300 && isfinite(l)) ? 1.0 / l : 1.0;
    }
    float* D = dinv32(w) + (size_t)n * 9;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            D[r * 3 + c] = (float)(V[r * 3] * V[c * 3] * inv[0] + V[r * 3 + 1] * V[c * 3 + 1] * inv[1] +
                                   V[r * 3 + 2] * V[c * 3 + 2] * inv[2]);
}

__device__ __forceinline__ void block_jacobi_row(const KrylovWork& w, int n) {
    const double* B = w.vals + (size_t)w.diag[n] * 9;
    double m[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) m[k] = B[k];
    const double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) + m[2] * (m[3] * m[7] - m[4] * m[6]);
    float* D = dinv32(w) + (size_t)n * 9;
    if (det == 0.0 || !isfinite(det)) {
        atomicOr(w.dflags, DF_SINGULAR_DIAG);
        for (int k = 0; k < 9; ++k) D[k] = (k % 4 == 0) ? 1.0f : 0.0f;
        return;
    }
    const double id = 1.0 / det;
    D[0] = (float)((m[4] * m[8] - m[5] * m[7]) * id);
    D[1] = (float)((m[2] * m[7] - m[1] * m[8]) * id);
    D[2] = (float)((m[1] * m[5] - m[2] * m[4]) * id);
    D[3] = (float)((m[5] * m[6] - m[3] * m[8]) * id);
    D[4] = (float)((m[0] * m[8] - m[2] * m[6]) * id);
    D[5] = (float)((m[2] * m[3] - m[0] * m[5]) * id);
    D[6] = (float)((m[3] * m[7] - m[4] * m[6]) * id);
    D[7] = (float)((m[1] * m[6] - m[0] * m[7]) * id);
    D[8] = (float)((m[0] * m[4] - m[1] * m[3]) * id);
}

// The vector a phase updates and the one its preconditioner writes: BiCGStab's p / phat (PH 0)
// and s / shat (PH 1); conjugate gradients' r / z (PH 2: r -= alpha q with q in w.v, z in w.phat).
template <int PH>
__device__ __forceinline__ double* phase_in(const KrylovWork& w) {
    return PH == 0 ? w.p : (PH == 1 ? w.s : w.r);
}
template <int PH>
__device__ __forceinline__ double* phase_out(const KrylovWork& w) {
    return PH == 0 ? w.phat : (PH == 1 ? w.shat : w.phat);
}

// Smoother groups of G > 1 nodes are handled one DoF per lane: a warp takes 32 / 3G groups at a
// time (lanes gl * 3G + r, r < 3G; the remaining lanes idle), every lane updates its DoF (phase A:
// u = p = r + beta (p - omega v); phase C: u = s = r - alpha v, written to vin) and forms its row of
// out = D_g^-1 u, the group's other entries of u arriving by warp shuffles. D_g^-1 is stored
// column-major per group in FP32 (k_group_jacobi_setup), so a warp's loads of one column are
// contiguous; the products are summed in FP64.
// Called by all 32 lanes of the warp; valid = this lane has a DoF. Returns u (0 when not valid).
template <int PH>
__device__ __forceinline__ double group_dof_update_apply(const KrylovWork& w, int g, int r, int n3, bool valid,
                                                         double alpha, double beta, double omega, double* vin,
                                                         double* out) {
    const int d = g * n3 + r;
    double u = 0.0;
    if (valid) {
        u = PH == 0 ? w.r[d] + beta * (w.p[d] - omega * w.v[d]) : w.r[d] - alpha * w.v[d];
        vin[d] = u;
    }
    const int base = ((threadIdx.x & 31) / n3) * n3;
    const float* D = reinterpret_cast<const float*>(w.dinv) + (size_t)g * n3 * n3 + r;
    double o = 0.0;
    for (int c = 0; c < n3; ++c) {
        const double uc = __shfl_sync(0xffffffffu, u, min(base + c, 31));
        if (valid) o += (double)D[c * n3] * uc;
    }
    if (valid) out[d] = o;
    return u;
}

// Phase A (PH 0: p = r + beta (p - omega v), phat = M^-1 p) or C (PH 1: s = r - alpha v,
// shat = M^-1 s) of an iteration on the CTA's rows [r0, r1), with the two-level
// preconditioner M^-1 = D^-1 + P (P^T J P)^-1 P^T (plan.agg_per_cta = m > 0). The CTA's warps
// split evenly over its m aggregates and keep one row mapping throughout, so the vector
// update, D^-1, the restriction (mask o u, d x (mask o u)) and later the prolongation touch
// each row from the same thread. The restriction is summed in fixed order (warp sums, then over
// the aggregate's warps), multiplied by M_a^T and written to coarse_r; after a group barrier
// every CTA stages the whole restricted vector, multiplies its 6m rows of the coarse inverse
// (held in shared memory) with it, forms z_a = M_a y_a and adds t + omega x d to its rows.
// Returns false when the group barrier timed out.
template <int PH>
__device__ bool precond_phase(const KrylovWork& w, const BatchPlan& plan, int lc, int r0, int r1, double alpha,
                              double beta, double omega, GridBarrier* bar, int nct, double* red, double* ys,
                              double* cs, const float* cinv, const double* Ms) {
    double* vin = phase_in<PH>(w);
    double* out = phase_out<PH>(w);
    const int m = plan.agg_per_cta, G = plan.group;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int wpa = nw / m;
    const int k = warp / wpa, wi = warp - k * wpa;
    int a0, a1;
    group_split(r0, r1, k, m, G, a0, a1);
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (k < m && G > 1) {
        const int n3 = 3 * G, gpw = 32 / n3, gl = lane / n3, rr = lane - gl * n3;
        const int g1 = a1 / G;
        for (int gc = a0 / G + wi * gpw; gc < g1; gc += wpa * gpw) {
            const int g = gc + gl;
            const bool valid = gl < gpw && g < g1;
            const double u = group_dof_update_apply<PH>(w, valid ? g : gc, rr, n3, valid, alpha, beta, omega, vin, out);
            if (valid) {
                // restriction of this DoF: translation i, and the rotations d x (mask o u)
                const int n = g * G + rr / 3, i = rr % 3;
                const double ui = ((plan.node_mask[n] >> i) & 1) ? u : 0.0;
                const double dx = plan.node_d[n * 3], dy = plan.node_d[n * 3 + 1], dz = plan.node_d[n * 3 + 2];
                acc[i] += ui;
                if (i == 0) {
                    acc[4] += dz * ui;
                    acc[5] -= dy * ui;
                } else if (i == 1) {
                    acc[3] -= dz * ui;
                    acc[5] += dx * ui;
                } else {
                    acc[3] += dy * ui;
                    acc[4] -= dx * ui;
                }
            }
        }
    } else if (k < m) {
        for (int n = a0 + wi * 32 + lane; n < a1; n += wpa * 32) {
            double u[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int d = n * 3 + i;
                u[i] = PH == 0 ? w.r[d] + beta * (w.p[d] - omega * w.v[d]) : w.r[d] - alpha * w.v[d];
                vin[d] = u[i];
            }
            const float* D = dinv32(w) + (size_t)n * 9;
            out[n * 3 + 0] = (double)D[0] * u[0] + (double)D[1] * u[1] + (double)D[2] * u[2];
            out[n * 3 + 1] = (double)D[3] * u[0] + (double)D[4] * u[1] + (double)D[5] * u[2];
            out[n * 3 + 2] = (double)D[6] * u[0] + (double)D[7] * u[1] + (double)D[8] * u[2];
            const int mk = plan.node_mask[n];
            const double u0 = (mk & 1) ? u[0] : 0.0, u1 = (mk & 2) ? u[1] : 0.0, u2 = (mk & 4) ? u[2] : 0.0;
            const double dx = plan.node_d[n * 3], dy = plan.node_d[n * 3 + 1], dz = plan.node_d[n * 3 + 2];
            acc[0] += u0;
            acc[1] += u1;
            acc[2] += u2;
            acc[3] += dy * u2 - dz * u1;
            acc[4] += dz * u0 - dx * u2;
            acc[5] += dx * u1 - dy * u0;
        }
    }
#pragma unroll
    for (int q = 0; q < 6; ++q)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], off);
    if (lane == 0 && k < m)
#pragma unroll
        for (int q = 0; q < 6; ++q) red[warp * 6 + q] = acc[q];
    __syncthreads();
    if (threadIdx.x < 6 * m) {
        const int kk = threadIdx.x / 6, q = threadIdx.x - 6 * kk;
        const double* M = Ms + kk * 36;
        double sum = 0.0;
        for (int p = 0; p < 6; ++p) {
            double t = 0.0;
            for (int j = 0; j < wpa; ++j) t += red[(kk * wpa + j) * 6 + p];
            sum += M[p * 6 + q] * t;
        }
        plan.coarse_r[6 * lc * m + threadIdx.x] = sum;
    }
    if (!group_barrier(bar, nct, w.dflags)) return false;
    const int nc = plan.n_coarse;
    for (int c = threadIdx.x; c < nc; c += blockDim.x) cs[c] = __ldcg(plan.coarse_r + c);
    __syncthreads();
    for (int kk = 0; kk < m; ++kk) {
        const float* rb = cinv + (size_t)(6 * kk) * nc;
        double sacc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int c = threadIdx.x; c < nc; c += blockDim.x) {
            const double x = cs[c];
#pragma unroll
            for (int q = 0; q < 6; ++q) sacc[q] += (double)rb[(size_t)q * nc + c] * x;
        }
#pragma unroll
        for (int q = 0; q < 6; ++q)
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) sacc[q] += __shfl_xor_sync(0xffffffffu, sacc[q], off);
        if (lane == 0)
#pragma unroll
            for (int q = 0; q < 6; ++q) red[warp * 6 + q] = sacc[q];
        __syncthreads();
        if (threadIdx.x < 6) {
            double t = 0.0;
            for (int j = 0; j < nw; ++j) t += red[j * 6 + threadIdx.x];
            ys[6 * kk + threadIdx.x] = t;
        }
        __syncthreads();
    }
    if (threadIdx.x < 6 * m) {
        const int kk = threadIdx.x / 6, q = threadIdx.x - 6 * kk;
        const double* M = Ms + kk * 36;
        double z = 0.0;
        for (int p = 0; p < 6; ++p) z += M[q * 6 + p] * ys[6 * kk + p];
        red[threadIdx.x] = z;
    }
    __syncthreads();
    if (k < m) {
        const double* z = red + 6 * k;
        for (int n = a0 + wi * 32 + lane; n < a1; n += wpa * 32) {
            const int mk = plan.node_mask[n];
            const double dx = plan.node_d[n * 3], dy = plan.node_d[n * 3 + 1], dz = plan.node_d[n * 3 + 2];
            // t + omega x d
            if (mk & 1) out[n * 3] += z[0] + z[4] * dz - z[5] * dy;
            if (mk & 2) out[n * 3 + 1] += z[1] + z[5] * dx - z[3] * dz;
            if (mk & 4) out[n * 3 + 2] += z[2] + z[3] * dy - z[4] * dx;
        }
    }
    return true;
}

// Phase A (PH 0) or C (PH 1) of a batch tissue with the two-level preconditioner: the CTA owns
// the tissue's aggregates [a0, a1), one warp per aggregate. A warp updates its aggregate's nodes,
// applies D^-1, restricts ((mask o u, d x (mask o u)) summed in fixed order, M_a^T applied by
// lanes 0-5) into coarse_r; after the group barrier the CTA stages the tissue's restricted vector,
// and the same warp forms its aggregate's six rows of the tissue's coarse inverse times it,
// z_a = M_a y_a, and adds t + omega x d to the same rows. Returns false when the barrier timed out.
template <int PH>
__device__ bool precond_batch(const KrylovWork& w, const BatchPlan& plan, int t, int a0, int a1, double alpha,
                              double beta, double omega, GridBarrier* bar, int nct, double* cs) {
    double* vin = phase_in<PH>(w);
    double* out = phase_out<PH>(w);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int G = plan.group;
    for (int a = a0 + warp; a < a1; a += nw) {
        const int k0 = plan.agg_ptr[a], k1 = plan.agg_ptr[a + 1];
        double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (G > 1) {
            // the aggregate's list holds whole smoother groups, each group's nodes consecutive:
            // one DoF per lane, as in the single-tissue phase
            const int n3 = 3 * G, gpw = 32 / n3, gl = lane / n3, rr = lane - gl * n3;
            const int ng = (k1 - k0) / G;
            for (int q = 0; q < ng; q += gpw) {
                const bool valid = gl < gpw && q + gl < ng;
                const int g = plan.agg_nodes[k0 + (valid ? q + gl : q) * G] / G;
                const double u = group_dof_update_apply<PH>(w, g, rr, n3, valid, alpha, beta, omega, vin, out);
                if (valid) {
                    const int n = g * G + rr / 3, i = rr % 3;
                    const double ui = ((plan.node_mask[n] >> i) & 1) ? u : 0.0;
                    const double dx = plan.node_d[n * 3], dy = plan.node_d[n * 3 + 1], dz = plan.node_d[n * 3 + 2];
                    acc[i] += ui;
                    if (i == 0) {
                        acc[4] += dz * ui;
                        acc[5] -= dy * ui;
                    } else if (i == 1) {
                        acc[3] -= dz * ui;
                        acc[5] += dx * ui;
                    } else {
                        acc[3] += dy * ui;
                        acc[4] -= dx * ui;
                    }
                }
            }
        }
        for (int k = k0 + lane; G == 1 && k < k1; k += 32) {
            const int n = plan.agg_nodes[k];
            double u[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int d = n * 3 + i;
                u[i] = PH == 0 ? w.r[d] + beta * (w.p[d] - omega * w.v[d]) : w.r[d] - alpha * w.v[d];
                vin[d] = u[i];
            }
            const float* D = dinv32(w) + (size_t)n * 9;
            out[n * 3 + 0] = (double)D[0] * u[0] + (double)D[1] * u[1] + (double)D[2] * u[2];
            out[n * 3 + 1] = (double)D[3] * u[0] + (double)D[4] * u[1] + (double)D[5] * u[2];
            out[n * 3 + 2] = (double)D[6] * u[0] + (double)D[7] * u[1] + (double)D[8] * u[2];
            const int mk = plan.node_mask[n];
            const double u0 = (mk & 1) ? u[0] : 0.0, u1 = (mk & 2) ? u[1] : 0.0, u2 = (mk & 4) ? u[2] : 0.0;
            const double dx = plan.node_d[n * 3], dy = plan.node_d[n * 3 + 1], dz = plan.node_d[n * 3 + 2];
            acc[0] += u0;
            acc[1] += u1;
            acc[2] += u2;
            acc[3] += dy * u2 - dz * u1;
            acc[4] += dz * u0 - dx * u2;
            acc[5] += dx * u1 - dy * u0;
        }
#pragma unroll
        for (int q = 0; q < 6; ++q)
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], off);
        if (lane < 6) {
            const double* M = plan.agg_m + (size_t)a * 36;
            double c = 0.0;
#pragma unroll
            for (int p = 0; p < 6; ++p) c += M[p * 6 + lane] * acc[p];
            plan.coarse_r[6 * (size_t)a + lane] = c;
        }
    }
    if (!group_barrier(bar, nct, w.dflags)) return false;
    const int g0 = plan.tissue_agg0[t];
    const int nc = 6 * (plan.tissue_agg0[t + 1] - g0);
    for (int c = threadIdx.x; c < nc; c += blockDim.x) cs[c] = __ldcg(plan.coarse_r + 6 * (size_t)g0 + c);
    __syncthreads();
    const double* inv = plan.coarse_inv + plan.coarse_base[t];
    const int ld = plan.coarse_ld;
    for (int a = a0 + warp; a < a1; a += nw) {
        const double* rows = inv + (size_t)(6 * (a - g0)) * ld;
        double y[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int c = lane; c < nc; c += 32) {
            const double x = cs[c];
#pragma unroll
            for (int q = 0; q < 6; ++q) y[q] += __ldcg(rows + (size_t)q * ld + c) * x;
        }
#pragma unroll
        for (int q = 0; q < 6; ++q)
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) y[q] += __shfl_xor_sync(0xffffffffu, y[q], off);
        const double* M = plan.agg_m + (size_t)a * 36;
        double z[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            double v = 0.0;
#pragma unroll
            for (int p = 0; p < 6; ++p) v += M[q * 6 + p] * y[p];
            z[q] = v;
        }
        const int k0 = plan.agg_ptr[a], k1 = plan.agg_ptr[a + 1];
        for (int k = k0 + lane; k < k1; k += 32) {
            const int n = plan.agg_nodes[k];
            const int mk = plan.node_mask[n];
            const double dx = plan.node_d[n * 3], dy = plan.node_d[n * 3 + 1], dz = plan.node_d[n * 3 + 2];
            if (mk & 1) out[n * 3] += z[0] + z[4] * dz - z[5] * dy;
            if (mk & 2) out[n * 3 + 1] += z[1] + z[5] * dx - z[3] * dz;
            if (mk & 4) out[n * 3 + 2] += z[2] + z[3] * dy - z[4] * dx;
        }
    }
    return true;
}

// The vector update of a phase and the preconditioner applied to it, on the rows this CTA
// preconditions (its contiguous range [r0, r1), or the node lists of its aggregates [ba0, ba1)
// for a batch tissue with the two-level preconditioner): PH 0 p = r + beta (p - omega v),
// phat = M^-1 p; PH 1 s = r - alpha v, shat = M^-1 s (BiCGStab); PH 2 r = r - alpha q (q in v),
// z = M^-1 r (z in phat; conjugate gradients). Returns false when a group barrier timed out.
// The phase's vector update and block-Jacobi smoother on the contiguous rows [r0, r1) (node
// blocks one node per thread; column blocks one DoF per lane).
template <int PH>
__device__ __forceinline__ void smooth_rows(const KrylovWork& w, const BatchPlan& plan, int r0, int r1, double alpha,
                                            double beta, double omega) {
    double* vin = phase_in<PH>(w);
    double* out = phase_out<PH>(w);
    if (plan.group > 1) {
        const int n3 = 3 * plan.group, gpw = 32 / n3, lane = threadIdx.x & 31, gl = lane / n3;
        const int g1 = r1 / plan.group;
        for (int gc = r0 / plan.group + (threadIdx.x >> 5) * gpw; gc < g1; gc += (blockDim.x >> 5) * gpw) {
            const bool valid = gl < gpw && gc + gl < g1;
            group_dof_update_apply<PH>(w, valid ? gc + gl : gc, lane - gl * n3, n3, valid, alpha, beta, omega, vin, out);
        }
        return;
    }
    for (int n = r0 + threadIdx.x; n < r1; n += blockDim.x) {
        // every load of the node before its first store (the vectors may alias as far as the
        // compiler knows): one round trip to memory per node
        double u[3], D[9];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int d = n * 3 + i;
            const double rv = w.r[d], vv = w.v[d];
            u[i] = PH == 0 ? rv + beta * (w.p[d] - omega * vv) : rv - alpha * vv;
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) D[k] = (double)__ldg(dinv32(w) + (size_t)n * 9 + k);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int d = n * 3 + i;
            vin[d] = u[i];
            out[d] = D[3 * i] * u[0] + D[3 * i + 1] * u[1] + D[3 * i + 2] * u[2];
        }
    }
}

// The aggregates of tissue t a CTA of its group preconditions (batch two-level space), or its
// leaves (multilevel space of a single tissue).
__device__ __forceinline__ void ml_or_batch_range(const BatchPlan& plan, int t, int lc, int nct, int& b0, int& b1) {
    b0 = b1 = 0;
    if (plan.batch_coarse) {
        const int g0 = plan.tissue_agg0[t], na = plan.tissue_agg0[t + 1] - g0;
        b0 = g0 + (int)((long long)na * lc / nct);
        b1 = g0 + (int)((long long)na * (lc + 1) / nct);
    } else if (plan.ml) {
        b0 = (int)((long long)plan.ml_n_leaf * lc / nct);
        b1 = (int)((long long)plan.ml_n_leaf * (lc + 1) / nct);
    }
}

// Multilevel additive coarse correction (plan.ml) applied by CTA lc of nct on its leaves [l0, l1):
//  A  the smoother on the leaves' nodes (vin updated, out = D^-1 u) and the raw leaf moments
//     m_a = sum_i P_i^T u_i (force, torque about the leaf centroid) into ml_leaf_m;
//  B  the CTA's partial moment of every set of levels 2..L that overlaps its leaves (its leaves'
//     moments moved to the set centroid: torque += (c_a - c_S) x force) at the CTA's slot;
//  -- group barrier --
//  C  every top set's moment (its partials summed in CTA order) into cs[0, 6 n_top); after it in
//     cs the motion of each overlapping set: W_S m_S below the top, the set's rows of the top
//     inverse times the top moments at the top;
//  D  each leaf's motion W_a m_a plus every ancestor's motion moved to the leaf centroid
//     (u += w x (c_a - c_S)), prolonged to the leaf's nodes: out_i += mask_i o (u + w x d_i).
// Jobs (level, set) are numbered in level order and dealt to the warps round-robin, the same
// numbering in C and D. Every sum has a fixed order.
template <int PH>
__device__ bool precond_ml(const KrylovWork& w, const BatchPlan& plan, int lc, int r0, int r1, int l0, int l1,
                           double alpha, double beta, double omega, GridBarrier* bar, int nct, double* cs,
                           double* red, double* dots) {
    double* vin = phase_in<PH>(w);
    double* out = phase_out<PH>(w);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int L = plan.ml_levels;
    const int kb = plan.agg_ptr[l0], ke = l1 > l0 ? plan.agg_ptr[l1] : kb;  // the CTA's span of the leaf node list
    // A1: the smoother on the CTA's contiguous rows (coalesced); the leaves' nodes lie in other
    // CTAs' rows as well, hence the group barrier before their moments
    smooth_rows<PH>(w, plan, r0, r1, alpha, beta, omega);
    if (!group_barrier(bar, nct, w.dflags)) return false;
    // A2: the leaf moments from the updated vector, one warp per leaf; a lane takes two list
    // positions at a time with every load issued first, and the next leaf's range is loaded one
    // leaf ahead
    int ka = l0 + warp < l1 ? plan.agg_ptr[l0 + warp] : 0, kz = l0 + warp < l1 ? plan.agg_ptr[l0 + warp + 1] : 0;
    for (int a = l0 + warp; a < l1; a += nw) {
        const int k0 = ka, k1 = kz;
        ka = a + nw < l1 ? plan.agg_ptr[a + nw] : 0;
        kz = a + nw < l1 ? plan.agg_ptr[a + nw + 1] : 0;
        double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int k = k0 + lane; k < k1; k += 64) {
            const bool two = k + 32 < k1;
            int n[2];
            n[0] = plan.agg_nodes[k];
            n[1] = two ? plan.agg_nodes[k + 32] : n[0];
            double u[2][3], d[2][3];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int mk = (h == 0 || two) ? plan.node_mask[n[h]] : 0;
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    u[h][i] = ((mk >> i) & 1) ? vin[n[h] * 3 + i] : 0.0;
                    d[h][i] = plan.node_d[n[h] * 3 + i];
                }
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                acc[0] += u[h][0];
                acc[1] += u[h][1];
                acc[2] += u[h][2];
                acc[3] += d[h][1] * u[h][2] - d[h][2] * u[h][1];
                acc[4] += d[h][2] * u[h][0] - d[h][0] * u[h][2];
                acc[5] += d[h][0] * u[h][1] - d[h][1] * u[h][0];
            }
        }
#pragma unroll
        for (int q = 0; q < 6; ++q)
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], off);
#pragma unroll
        for (int q = 0; q < 6; ++q)
            if (lane == q) plan.ml_leaf_m[6 * (size_t)a + q] = acc[q];
    }
    __syncthreads();
    // B: this CTA's partial moment of every set of levels >= 2 its leaves overlap, level after
    // level, one thread per set, each from its children's partials one level down (the leaves for
    // level 2) moved to the set's centroid; children in index order
    int job = 0;
    for (int lev = 2; lev <= L; ++lev) {
        const int span = plan.ml_span[lev - 1], cspan = plan.ml_span[lev - 2], fan = span / cspan;
        const int s0 = l0 / span, s1 = l1 > l0 ? (l1 - 1) / span : s0 - 1;    // none for an empty range
        const int c0 = l0 / cspan, c1 = l1 > l0 ? (l1 - 1) / cspan : c0 - 1;  // the children's range
        for (int S = s0 + (int)threadIdx.x; S <= s1; S += blockDim.x) {
            const int gS = plan.ml_set0[lev - 1] + S;
            const double* cS = plan.ml_cen + 3 * (size_t)gS;
            double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            const int k0 = max(c0, S * fan), k1 = min(c1, S * fan + fan - 1);
#pragma unroll 4
            for (int Sc = k0; Sc <= k1; ++Sc) {
                const int gC = plan.ml_set0[lev - 2] + Sc;
                const double* m = lev == 2 ? plan.ml_leaf_m + 6 * (size_t)Sc
                                           : plan.ml_part + 6 * (size_t)(plan.ml_pstart[gC] + lc - plan.ml_first_cta[gC]);
                const double* ca = plan.ml_cen + 3 * (size_t)gC;
                const double dx = ca[0] - cS[0], dy = ca[1] - cS[1], dz = ca[2] - cS[2];
                const double f0 = m[0], f1 = m[1], f2 = m[2];
                acc[0] += f0;
                acc[1] += f1;
                acc[2] += f2;
                acc[3] += m[3] + dy * f2 - dz * f1;
                acc[4] += m[4] + dz * f0 - dx * f2;
                acc[5] += m[5] + dx * f1 - dy * f0;
            }
            double* dst = plan.ml_part + 6 * (size_t)(plan.ml_pstart[gS] + lc - plan.ml_first_cta[gS]);
#pragma unroll
            for (int q = 0; q < 6; ++q) dst[q] = acc[q];
        }
        __syncthreads();  // the next level reads these partials
    }
    if (!group_barrier(bar, nct, w.dflags)) return false;
    // C
    const int nt = plan.ml_count[L - 1], gt0 = plan.ml_set0[L - 1], n6 = 6 * nt;
    for (int e = threadIdx.x; e < n6; e += blockDim.x) {
        const int gS = gt0 + e / 6, q = e % 6;
        double v = 0.0;
        for (int k = plan.ml_pstart[gS]; k < plan.ml_pstart[gS + 1]; ++k) v += __ldcg(plan.ml_part + 6 * (size_t)k + q);
        cs[e] = v;
    }
    __syncthreads();
    double* ys = cs + n6;
    // the levels below the top: one thread per (set, component), jobs numbered level by level;
    // each thread sums its set's partial moments in CTA order and applies its row of W_S
    job = 0;
    for (int lev = 2; lev < L; ++lev) {
        const int span = plan.ml_span[lev - 1];
        job += l1 > l0 ? (l1 - 1) / span - l0 / span + 1 : 0;
    }
    for (int e = threadIdx.x; e < 6 * job; e += blockDim.x) {
        const int jg = e / 6, q = e - 6 * jg;
        int jl = jg, lev = 2, S = 0;
        for (; lev < L; ++lev) {  // the job's level and set (l1 > l0 here)
            const int span = plan.ml_span[lev - 1];
            const int s0 = l0 / span, ns = (l1 - 1) / span - s0 + 1;
            if (jl < ns) {
                S = s0 + jl;
                break;
            }
            jl -= ns;
        }
        const int gS = plan.ml_set0[lev - 1] + S;
        double m[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int k = plan.ml_pstart[gS]; k < plan.ml_pstart[gS + 1]; ++k)
#pragma unroll
            for (int p = 0; p < 6; ++p) m[p] += __ldcg(plan.ml_part + 6 * (size_t)k + p);
        const double* W = plan.ml_w + 36 * (size_t)gS + 6 * q;
        double v = 0.0;
#pragma unroll
        for (int p = 0; p < 6; ++p) v += W[p] * m[p];
        ys[6 * jg + q] = v;
    }
    // the top sets the CTA's leaves overlap (jobs job, job + 1, ...): their rows of the dense top
    // inverse times the top moments, every set's columns cut into kTopChunks chunks that the
    // warps share (chunk sums in red, then added in chunk order)
    {
        constexpr int kTopChunks = 8, kTopSets = 4;  // red holds kTopSets x kTopChunks x 6 sums
        const int span = plan.ml_span[L - 1];
        const int s0 = l0 / span, ntop = l1 > l0 ? (l1 - 1) / span - s0 + 1 : 0;
        for (int base = 0; base < ntop; base += kTopSets) {
            const int nb = min(kTopSets, ntop - base);
            for (int item = warp; item < nb * kTopChunks; item += nw) {
                const int jt = item / kTopChunks, ch = item % kTopChunks;
                const double* rows = plan.ml_top_inv + (size_t)(6 * (s0 + base + jt)) * n6;
                const int c0 = n6 * ch / kTopChunks, c1 = n6 * (ch + 1) / kTopChunks;
                double y[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                for (int c = c0 + lane; c < c1; c += 32) {
                    const double x = cs[c];
#pragma unroll
                    for (int q = 0; q < 6; ++q) y[q] += __ldg(rows + (size_t)q * n6 + c) * x;
                }
#pragma unroll
                for (int q = 0; q < 6; ++q)
#pragma unroll
                    for (int off = 16; off > 0; off >>= 1) y[q] += __shfl_xor_sync(0xffffffffu, y[q], off);
#pragma unroll
                for (int q = 0; q < 6; ++q)
                    if (lane == q) red[(jt * kTopChunks + ch) * 6 + q] = y[q];
            }
            __syncthreads();
            for (int e = threadIdx.x; e < nb * 6; e += blockDim.x) {
                const int jt = e / 6, q = e % 6;
                double v = 0.0;
                for (int ch = 0; ch < kTopChunks; ++ch) v += red[(jt * kTopChunks + ch) * 6 + q];
                ys[6 * (job + base + jt) + q] = v;
            }
            __syncthreads();  // red is written again by the next sets
        }
    }
    __syncthreads();
    // D1: each leaf's motion, one thread per leaf, over the leaf's moment in ml_leaf_m
    for (int a = l0 + (int)threadIdx.x; a < l1; a += blockDim.x) {
        double* ma = plan.ml_leaf_m + 6 * (size_t)a;
        const double* Wa = plan.ml_w + 36 * (size_t)a;
        double m[6], y[6];
#pragma unroll
        for (int p = 0; p < 6; ++p) m[p] = ma[p];
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            double v = 0.0;
#pragma unroll
            for (int p = 0; p < 6; ++p) v += __ldg(Wa + q * 6 + p) * m[p];
            y[q] = v;
        }
        const double* ca = plan.ml_cen + 3 * (size_t)a;
        int jb = 0;
        for (int lev = 2; lev <= L; ++lev) {
            const int span = plan.ml_span[lev - 1];
            const int s0 = l0 / span, s1 = (l1 - 1) / span, S = a / span;  // l1 > l0 here
            const double* yS = ys + 6 * (jb + S - s0);
            const double* cS = plan.ml_cen + 3 * (size_t)(plan.ml_set0[lev - 1] + S);
            const double dx = ca[0] - cS[0], dy = ca[1] - cS[1], dz = ca[2] - cS[2];
            y[0] += yS[0] + yS[4] * dz - yS[5] * dy;
            y[1] += yS[1] + yS[5] * dx - yS[3] * dz;
            y[2] += yS[2] + yS[3] * dy - yS[4] * dx;
            y[3] += yS[3];
            y[4] += yS[4];
            y[5] += yS[5];
            jb += s1 - s0 + 1;
        }
#pragma unroll
        for (int q = 0; q < 6; ++q) ma[q] = y[q];  // the moment is not needed again: the motion replaces it
    }
    __syncthreads();
    // D2: the prolongation, one node per thread (the leaf of each list position in ml_pos_leaf);
    // conjugate gradients' (r, z) and (r, r) over the same nodes on the way
    double rz = 0.0, rr = 0.0;
    // the next position's node and leaf are loaded one iteration ahead
    int n_nx = kb + (int)threadIdx.x < ke ? plan.agg_nodes[kb + threadIdx.x] : 0;
    int lf_nx = kb + (int)threadIdx.x < ke ? plan.ml_pos_leaf[kb + threadIdx.x] : 0;
    for (int k = kb + threadIdx.x; k < ke; k += blockDim.x) {
        const int n = n_nx;
        const double* y = plan.ml_leaf_m + 6 * (size_t)lf_nx;
        n_nx = k + (int)blockDim.x < ke ? plan.agg_nodes[k + blockDim.x] : 0;
        lf_nx = k + (int)blockDim.x < ke ? plan.ml_pos_leaf[k + blockDim.x] : 0;
        const int mk = plan.node_mask[n];
        const double dx = plan.node_d[n * 3], dy = plan.node_d[n * 3 + 1], dz = plan.node_d[n * 3 + 2];
        double z0 = out[n * 3], z1 = out[n * 3 + 1], z2 = out[n * 3 + 2];
        double q0 = 0.0, q1 = 0.0, q2 = 0.0;
        if (PH == 2) {  // loaded before the stores below, in the same round trip
            q0 = w.r[n * 3];
            q1 = w.r[n * 3 + 1];
            q2 = w.r[n * 3 + 2];
        }
        if (mk & 1) z0 += y[0] + y[4] * dz - y[5] * dy;
        if (mk & 2) z1 += y[1] + y[5] * dx - y[3] * dz;
        if (mk & 4) z2 += y[2] + y[3] * dy - y[4] * dx;
        out[n * 3] = z0;
        out[n * 3 + 1] = z1;
        out[n * 3 + 2] = z2;
        if (PH == 2) {
            rz += q0 * z0 + q1 * z1 + q2 * z2;
            rr += q0 * q0 + q1 * q1 + q2 * q2;
        }
    }
    if (dots) {
        dots[0] = rz;
        dots[1] = rr;
    }
    return true;
}

template <int PH>
// dots (multilevel space, PH 2 only): this CTA's partial (r, z) and (r, r) over its leaves' nodes,
// formed on the way (the caller then skips precond_rows_dots)
__device__ bool update_precondition(const KrylovWork& w, const BatchPlan& plan, int t, int lc, int r0, int r1, int ba0,
                                    int ba1, double alpha, double beta, double omega, GridBarrier* bar, int nct,
                                    double* red, double* ys, double* cs, const float* cinv_s, const double* Ms,
                                    double* dots = nullptr) {
    if (plan.agg_per_cta > 0)
        return precond_phase<PH>(w, plan, lc, r0, r1, alpha, beta, omega, bar, nct, red, ys, cs, cinv_s, Ms);
    if (plan.batch_coarse) return precond_batch<PH>(w, plan, t, ba0, ba1, alpha, beta, omega, bar, nct, cs);
    if (plan.ml) return precond_ml<PH>(w, plan, lc, r0, r1, ba0, ba1, alpha, beta, omega, bar, nct, cs, red, dots);
    smooth_rows<PH>(w, plan, r0, r1, alpha, beta, omega);
    return true;
}

// (r, z) and (r, r) over the rows this CTA preconditions (z in phat), after update_precondition<2>.
__device__ __forceinline__ void precond_rows_dots(const KrylovWork& w, const BatchPlan& plan, int r0, int r1, int ba0,
                                                  int ba1, double& rz, double& rr) {
    __syncthreads();  // z of these rows may have been written by another warp of the CTA
    if (plan.batch_coarse || plan.ml) {
        const int k0 = plan.agg_ptr[ba0], k1 = plan.agg_ptr[ba1];
        for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
            const int n = plan.agg_nodes[k];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const double r = w.r[n * 3 + i];
                rz += r * w.phat[n * 3 + i];
                rr += r * r;
            }
        }
        return;
    }
    for (int n = r0 + threadIdx.x; n < r1; n += blockDim.x)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double r = w.r[n * 3 + i];
            rz += r * w.phat[n * 3 + i];
            rr += r * r;
        }
}

// BiCGStab restart after a breakdown: rhat = r, p = v = 0, rho = (r, r); at most kMaxRestarts
// per solve. Returns false when the restarts are used up (the caller reports a breakdown).
constexpr int kMaxRestarts = 8;

__device__ bool restart(const KrylovWork& w, int r0, int r1, double& rho, double& rho_prev, double& alpha,
                        double& omega, int& restarts, double* buf, int lc, int nct, GridBarrier* bar, double* smem,
                        double* sb) {
    if (++restarts > kMaxRestarts) return false;
    double v[1] = {0.0}, tot[1];
    for (int n = r0 + threadIdx.x; n < r1; n += blockDim.x)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int d = n * 3 + i;
            const double r = w.r[d];
            w.rhat[d] = r;
            w.p[d] = 0.0;
            w.v[d] = 0.0;
            v[0] += r * r;
        }
    write_partials<1>(v, buf, lc, smem);
    if (!group_barrier(bar, nct, w.dflags)) return false;
    sum_partials<1>(buf, nct, tot, smem, sb);
    rho = tot[0];
    rho_prev = 1.0;
    alpha = 1.0;
    omega = 1.0;
    return rho > 0.0 && isfinite(rho);
}

// The whole block-Jacobi (or two-level) BiCGStab solve of tissue t by this CTA, which is CTA lc of
// the tissue's group (nct = 1: a tissue solved by this CTA alone, with CTA-level barriers only).
// The group's per-CTA partial sums live at partials[4 pbase ..) (4 nct doubles). Returns false
// when a group barrier timed out.
__device__ bool solve_tissue(const KrylovWork& w, const BatchPlan& plan, int t, int lc, int pbase, double rtol,
                             int max_iter, double* smem, double* sb, double* red, double* ys, double* Ms, double* cs,
                             float* cinv_s) {
    if (!plan.active[t]) return true;
    const int nct = plan.ncta[t];
    const int tr0 = plan.row0[t], tr1 = plan.row0[t + 1];
    int r0, r1;
    group_split(tr0, tr1, lc, nct, plan.group, r0, r1);
    int ba0 = 0, ba1 = 0;  // this CTA's aggregates of a batch tissue / leaves of the multilevel space
    ml_or_batch_range(plan, t, lc, nct, ba0, ba1);
    GridBarrier* bar = plan.barriers + t;
    double* part[2] = {w.partials + 4 * pbase, w.partials + 4 * pbase + 2 * nct};
    int pb = 0;
    if (plan.agg_per_cta > 0) {
        const size_t cnt = (size_t)6 * plan.agg_per_cta * plan.n_coarse;
        const double* src = plan.coarse_inv + (size_t)6 * lc * plan.agg_per_cta * plan.n_coarse;
        for (size_t i = threadIdx.x; i < cnt; i += blockDim.x) cinv_s[i] = (float)src[i];
        for (int i = threadIdx.x; i < 36 * plan.agg_per_cta; i += blockDim.x)
            Ms[i] = plan.agg_m[(size_t)lc * plan.agg_per_cta * 36 + i];
    }
    // phase 0: block-Jacobi inverses, x = 0, r = rhat = b, p = v = 0, ||b||^2; warm start (the
    // iterate x and residual r that conjugate gradients left): x, r kept, rhat = r, ||r||^2
    double v0[2] = {0.0, 0.0};
    for (int n = r0 + threadIdx.x; n < r1; n += blockDim.x) {
        if (plan.group == 1) block_jacobi_row(w, n);  // G > 1: inverses set up before the launch
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int d = n * 3 + i;
            const double b = w.b[d];
            double r = b;
            if (plan.warm)
                r = w.r[d];
            else
                w.x[d] = 0.0;
            w.r[d] = r;
            w.rhat[d] = r;
            w.p[d] = 0.0;
            w.v[d] = 0.0;
            v0[0] += b * b;
            v0[1] += r * r;
        }
    }
    write_partials<2>(v0, part[pb], lc, smem);
    if (!group_barrier(bar, nct, w.dflags)) return false;
    double v1[1], t1[1], t2[2];
    sum_partials<2>(part[pb], nct, t2, smem, sb);
    pb ^= 1;
    const double bb = t2[0];
    double rr = t2[1];
    double rho = rr, rho_prev = 1.0, alpha = 1.0, omega = 1.0;
    const double tol2 = rtol * rtol * bb;
    int it = 0, restarts = 0;
    int status = !isfinite(bb) || !isfinite(rr) ? KS_NONFINITE : (rr <= tol2 ? KS_CONVERGED : KS_RUNNING);
    while (status == KS_RUNNING) {
        // A: p = r + beta (p - omega v); phat = M^-1 p
        const double beta = (rho / rho_prev) * (alpha / omega);
        if (!update_precondition<0>(w, plan, t, lc, r0, r1, ba0, ba1, alpha, beta, omega, bar, nct, red, ys, cs, cinv_s,
                                    Ms))
            return false;
        if (!group_barrier(bar, nct, w.dflags)) return false;
        // B: v = J phat; (rhat, v)
        double d0 = 0.0, d1 = 0.0;
        spmv_rows<1>(w, r0, r1, w.phat, w.v, d0, d1);
        v1[0] = d0;
        write_partials<1>(v1, part[pb], lc, smem);
        if (!group_barrier(bar, nct, w.dflags)) return false;
        sum_partials<1>(part[pb], nct, t1, smem, sb);
        pb ^= 1;
        if (!isfinite(t1[0])) { status = KS_NONFINITE; break; }
        if (t1[0] == 0.0) {  // (rhat, v) vanished: restart with rhat = r
            if (!restart(w, r0, r1, rho, rho_prev, alpha, omega, restarts, part[pb], lc, nct, bar, smem, sb)) {
                status = KS_BREAKDOWN;
                break;
            }
            pb ^= 1;
            continue;
        }
        alpha = rho / t1[0];
        // C: s = r - alpha v; shat = M^-1 s
        if (!update_precondition<1>(w, plan, t, lc, r0, r1, ba0, ba1, alpha, 0.0, 0.0, bar, nct, red, ys, cs, cinv_s, Ms))
            return false;
        if (!group_barrier(bar, nct, w.dflags)) return false;
        // D: t = J shat; (t, s), (t, t)
        d0 = 0.0;
        d1 = 0.0;
        spmv_rows<2>(w, r0, r1, w.shat, w.t, d0, d1);
        double v2[2] = {d0, d1};
        write_partials<2>(v2, part[pb], lc, smem);
        if (!group_barrier(bar, nct, w.dflags)) return false;
        sum_partials<2>(part[pb], nct, t2, smem, sb);
        pb ^= 1;
        if (!isfinite(t2[0]) || !isfinite(t2[1])) { status = KS_NONFINITE; break; }
        omega = t2[1] == 0.0 ? 0.0 : t2[0] / t2[1];
        // E: x += alpha phat + omega shat; r = s - omega t; (rhat, r), (r, r)
        double e0 = 0.0, e1 = 0.0;
        for (int n = r0 + threadIdx.x; n < r1; n += blockDim.x) {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int d = n * 3 + i;
                w.x[d] += alpha * w.phat[d] + omega * w.shat[d];
                const double r = w.s[d] - omega * w.t[d];
                w.r[d] = r;
                e0 += w.rhat[d] * r;
                e1 += r * r;
            }
        }
        double v3[2] = {e0, e1};
        write_partials<2>(v3, part[pb], lc, smem);
        if (!group_barrier(bar, nct, w.dflags)) return false;
        sum_partials<2>(part[pb], nct, t2, smem, sb);
        pb ^= 1;
        rho_prev = rho;
        rho = t2[0];
        rr = t2[1];
        ++it;
        if (!isfinite(rho) || !isfinite(rr))
            status = KS_NONFINITE;
        else if (rr <= tol2)
            status = KS_CONVERGED;
        else if (it >= max_iter)
            status = KS_MAXIT;
        else if (rho == 0.0 || omega == 0.0) {  // breakdown: restart with rhat = r
            if (!restart(w, r0, r1, rho, rho_prev, alpha, omega, restarts, part[pb], lc, nct, bar, smem, sb))
                status = KS_BREAKDOWN;
            pb ^= 1;
        }
    }
    if (lc == 0 && threadIdx.x == 0) {
        KrylovScalars* sc = plan.scalars + t;
        sc->bb = bb;
        sc->rr = rr;
        sc->rho = rho;
        sc->rho_prev = rho_prev;
        sc->alpha = alpha;
        sc->omega = omega;
        sc->tol2 = tol2;
        sc->iter = it;
        sc->max_iter = max_iter;
        sc->status = status;
        sc->method = KM_BICGSTAB;
    }
    return true;
}

// Preconditioned conjugate gradients on tissue t by this CTA (CTA lc of the tissue's group), for a
// symmetric J - no internal viscosity: the elastic tangent, the diagonal drag and the fixed /
// slave-master elimination are all symmetric - with the symmetric preconditioner of solve_tissue
// (block-Jacobi inverses, the column smoother's inverses stored symmetrised, the coarse inverse
// symmetrised). One SpMV per iteration and three group barriers (four with the two-level coarse
// correction):  p = z + beta p  |  q = J p, (p, q)  |  x += alpha p, r -= alpha q, z = M^-1 r,
// (r, z), (r, r). Same stopping rule as BiCGStab (||r||^2 <= rtol^2 ||b||^2). When (p, J p) <= 0
// or (r, z) <= 0 before convergence (J or M not positive definite) the tissue's status is
// KS_INDEFINITE and the host finishes it with BiCGStab from the iterate reached. Returns false when a group barrier
// timed out.
__device__ bool solve_tissue_cg(const KrylovWork& w, const BatchPlan& plan, int t, int lc, int pbase, double rtol,
                                int max_iter, double* smem, double* sb, double* red, double* ys, double* Ms, double* cs,
                                float* cinv_s, bool& indefinite) {
    indefinite = false;
    if (!plan.active[t]) return true;
    const int nct = plan.ncta[t];
    const int tr0 = plan.row0[t], tr1 = plan.row0[t + 1];
    int r0, r1;
    group_split(tr0, tr1, lc, nct, plan.group, r0, r1);
    int ba0 = 0, ba1 = 0;
    ml_or_batch_range(plan, t, lc, nct, ba0, ba1);
    GridBarrier* bar = plan.barriers + t;
    double* part[2] = {w.partials + 4 * pbase, w.partials + 4 * pbase + 2 * nct};
    int pb = 0;
    if (plan.agg_per_cta > 0) {
        const size_t cnt = (size_t)6 * plan.agg_per_cta * plan.n_coarse;
        const double* src = plan.coarse_inv + (size_t)6 * lc * plan.agg_per_cta * plan.n_coarse;
        for (size_t i = threadIdx.x; i < cnt; i += blockDim.x) cinv_s[i] = (float)src[i];
        for (int i = threadIdx.x; i < 36 * plan.agg_per_cta; i += blockDim.x)
            Ms[i] = plan.agg_m[(size_t)lc * plan.agg_per_cta * 36 + i];
    }
    // set-up: block-Jacobi inverses, x = 0, r = b, p = q = 0, ||b||^2; warm start (plan.warm):
    // x0 and r0 = b - J x0 given by the host, ||r0||^2 beside ||b||^2
    double v1[1] = {0.0}, t1[1], t2[2];
    {
        double v0[2] = {0.0, 0.0};
        for (int n = r0 + threadIdx.x; n < r1; n += blockDim.x) {
            if (plan.group == 1) block_jacobi_row(w, n);
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int d = n * 3 + i;
                const double b = w.b[d];
                double r = b;
                if (plan.warm)
                    r = w.r[d];
                else
                    w.x[d] = 0.0;
                w.r[d] = r;
                w.p[d] = 0.0;
                w.v[d] = 0.0;
                v0[0] += b * b;
                v0[1] += r * r;
            }
        }
        write_partials<2>(v0, part[pb], lc, smem);
    }
    if (!group_barrier(bar, nct, w.dflags)) return false;
    sum_partials<2>(part[pb], nct, t2, smem, sb);
    pb ^= 1;
    const double bb = t2[0];
    double rr = t2[1];
    if (plan.warm && !(rr < bb)) {
        // the guess is no better than zero (or not finite): every CTA of the group sees the same
        // sums and takes this branch; start from x = 0 and wait until every row is reset
        for (int n = r0 + threadIdx.x; n < r1; n += blockDim.x)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int d = n * 3 + i;
                w.x[d] = 0.0;
                w.r[d] = w.b[d];
            }
        rr = bb;
        if (!group_barrier(bar, nct, w.dflags)) return false;
    }
    const double tol2 = rtol * rtol * bb;
    double rz = 0.0, alpha = 0.0, beta = 0.0;
    int it = 0;
    int status = !isfinite(bb) ? KS_NONFINITE : (rr <= tol2 ? KS_CONVERGED : KS_RUNNING);
    if (status == KS_RUNNING) {  // z = M^-1 r, (r, z)
        double dd[2] = {0.0, 0.0};
        if (!update_precondition<2>(w, plan, t, lc, r0, r1, ba0, ba1, 0.0, 0.0, 0.0, bar, nct, red, ys, cs, cinv_s, Ms, dd))
            return false;
        double d0 = dd[0], d1 = dd[1];
        if (!plan.ml) precond_rows_dots(w, plan, r0, r1, ba0, ba1, d0, d1);
        double v2[2] = {d0, d1};
        write_partials<2>(v2, part[pb], lc, smem);
        if (!group_barrier(bar, nct, w.dflags)) return false;
        sum_partials<2>(part[pb], nct, t2, smem, sb);
        pb ^= 1;
        rz = t2[0];
        if (!isfinite(rz)) status = KS_NONFINITE;
        else if (!(rz > 0.0)) indefinite = true;
    }
    while (status == KS_RUNNING && !indefinite) {
        // p = z + beta p on the contiguous rows (z of every row is final after the last barrier)
        for (int n = r0 + threadIdx.x; n < r1; n += blockDim.x)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int d = n * 3 + i;
                w.p[d] = w.phat[d] + beta * w.p[d];
            }
        if (!group_barrier(bar, nct, w.dflags)) return false;
        // q = J p, (p, q)
        double d0 = 0.0, d1 = 0.0;
        spmv_rows<3>(w, r0, r1, w.p, w.v, d0, d1);
        v1[0] = d0;
        write_partials<1>(v1, part[pb], lc, smem);
        if (!group_barrier(bar, nct, w.dflags)) return false;
        sum_partials<1>(part[pb], nct, t1, smem, sb);
        pb ^= 1;
        const double pq = t1[0];
        if (!isfinite(pq)) { status = KS_NONFINITE; break; }
        if (!(pq > 0.0)) { indefinite = true; break; }
        alpha = rz / pq;
        // x += alpha p (p is still in L2 from the SpMV's gathers; a separate pass: folded into
        // the smoother's, its live registers spill); r -= alpha q; z = M^-1 r; (r, z), (r, r)
        for (int n = r0 + threadIdx.x; n < r1; n += blockDim.x)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int d = n * 3 + i;
                w.x[d] += alpha * w.p[d];
            }
        double dd2[2] = {0.0, 0.0};
        if (!update_precondition<2>(w, plan, t, lc, r0, r1, ba0, ba1, alpha, 0.0, 0.0, bar, nct, red, ys, cs, cinv_s, Ms,
                                    dd2))
            return false;
        d0 = dd2[0];
        d1 = dd2[1];
        if (!plan.ml) precond_rows_dots(w, plan, r0, r1, ba0, ba1, d0, d1);
        double v2[2] = {d0, d1};
        write_partials<2>(v2, part[pb], lc, smem);
        if (!group_barrier(bar, nct, w.dflags)) return false;
        sum_partials<2>(part[pb], nct, t2, smem, sb);
        pb ^= 1;
        const double rz_new = t2[0];
        rr = t2[1];
        ++it;
        if (!isfinite(rz_new) || !isfinite(rr))
            status = KS_NONFINITE;
        else if (rr <= tol2)
            status = KS_CONVERGED;
        else if (it >= max_iter)
            status = KS_MAXIT;
        else if (!(rz_new > 0.0))
            indefinite = true;
        beta = rz_new / rz;
        rz = rz_new;
    }
    if (indefinite) status = KS_INDEFINITE;  // the host solves the tissue again with BiCGStab
    if (lc == 0 && threadIdx.x == 0) {
        KrylovScalars* sc = plan.scalars + t;
        sc->bb = bb;
        sc->rr = rr;
        sc->rho = rz;
        sc->rho_prev = 0.0;
        sc->alpha = alpha;
        sc->omega = beta;
        sc->tol2 = tol2;
        sc->iter = it;
        sc->max_iter = max_iter;
        sc->status = status;
        sc->method = KM_CG;
    }
    return true;
}

// Preconditioned MINRES (Paige and Saunders' recurrences, as in the reference implementation
// that SciPy's minres follows) on tissue t for a symmetric but indefinite J - the Jacobian of a
// step with packing pairs, whose repulsion has a negative stiffness across each pair - with the
// symmetric positive definite block preconditioner |D|^-1 (block_abs_inverse_row). Vectors: x, v
// in p, A v in v, r1 in r, r2 in rhat, z = M^-1 r2 in phat, the direction w in s and its
// predecessor in shat. Three group barriers per iteration: after v (the SpMV gathers it), after
// the SpMV with (v, A v) and (v, r1), after r2 / z with (r2, z). Stops when the preconditioned
// residual estimate phibar <= rtol phibar_0 (the host reports phibar / phibar_0 as the relative
// residual). Returns false when a group barrier timed out.
__device__ bool solve_tissue_minres(const KrylovWork& w, const BatchPlan& plan, int t, int lc, int pbase, double rtol,
                                    int max_iter, double* smem, double* sb) {
    if (!plan.active[t]) return true;
    const int nct = plan.ncta[t];
    int r0, r1;
    group_split(plan.row0[t], plan.row0[t + 1], lc, nct, plan.group, r0, r1);
    GridBarrier* bar = plan.barriers + t;
    double* part[2] = {w.partials + 4 * pbase, w.partials + 4 * pbase + 2 * nct};
    int pb = 0;
    double v2[2] = {0.0, 0.0};
    for (int n = r0 + threadIdx.x; n < r1; n += blockDim.x) {
        block_abs_inverse_row(w, n);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int d = n * 3 + i;
            const double b = w.b[d];
            w.x[d] = 0.0;
            w.r[d] = b;
            w.rhat[d] = b;
            w.s[d] = 0.0;
            w.shat[d] = 0.0;
            v2[0] += b * b;
        }
        apply_dinv32(w, n, w.rhat, w.phat);
#pragma unroll
        for (int i = 0; i < 3; ++i) v2[1] += w.rhat[n * 3 + i] * w.phat[n * 3 + i];
    }
    write_partials<2>(v2, part[pb], lc, smem);
    if (!group_barrier(bar, nct, w.dflags)) return false;
    double t1[1], t2[2];
    sum_partials<2>(part[pb], nct, t2, smem, sb);
    pb ^= 1;
    const double bb = t2[0];
    double beta = t2[1] > 0.0 ? sqrt(t2[1]) : 0.0;
    const double beta1 = beta;
    double oldb = 0.0, dbar = 0.0, epsln = 0.0, phibar = beta1, cs = -1.0, sn = 0.0;
    int it = 0;
    int status = (!isfinite(bb) || !isfinite(t2[1])) ? KS_NONFINITE
                 : (bb == 0.0 || beta1 == 0.0)       ? (bb == 0.0 ? KS_CONVERGED : KS_BREAKDOWN)
                                                     : KS_RUNNING;
    if (status == KS_RUNNING) {
        for (int n = r0 + threadIdx.x; n < r1; n += blockDim.x)
#pragma unroll
            for (int i = 0; i < 3; ++i) w.p[n * 3 + i] = w.phat[n * 3 + i] / beta;
        if (!group_barrier(bar, nct, w.dflags)) return false;
    }
    while (status == KS_RUNNING) {
        double d0 = 0.0, d1 = 0.0;
        spmv_rows<4>(w, r0, r1, w.p, w.v, d0, d1);
        double v3[2] = {d0, d1};
        write_partials<2>(v3, part[pb], lc, smem);
        if (!group_barrier(bar, nct, w.dflags)) return false;
        sum_partials<2>(part[pb], nct, t2, smem, sb);
        pb ^= 1;
        const double c1 = it >= 1 ? beta / oldb : 0.0;
        const double alfa = t2[0] - c1 * t2[1];
        const double c2 = alfa / beta;
        double e1[1] = {0.0};
        for (int n = r0 + threadIdx.x; n < r1; n += blockDim.x) {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int d = n * 3 + i;
                const double y = w.v[d] - c1 * w.r[d] - c2 * w.rhat[d];
                w.r[d] = w.rhat[d];
                w.rhat[d] = y;
            }
            apply_dinv32(w, n, w.rhat, w.phat);
#pragma unroll
            for (int i = 0; i < 3; ++i) e1[0] += w.rhat[n * 3 + i] * w.phat[n * 3 + i];
        }
        write_partials<1>(e1, part[pb], lc, smem);
        if (!group_barrier(bar, nct, w.dflags)) return false;
        sum_partials<1>(part[pb], nct, t1, smem, sb);
        pb ^= 1;
        oldb = beta;
        if (!isfinite(t1[0]) || !isfinite(alfa)) {
            status = KS_NONFINITE;
            break;
        }
        beta = t1[0] > 0.0 ? sqrt(t1[0]) : 0.0;
        const double oldeps = epsln;
        const double delta = cs * dbar + sn * alfa;
        const double gbar = sn * dbar - cs * alfa;
        epsln = sn * beta;
        dbar = -cs * beta;
        const double gamma = sqrt(gbar * gbar + beta * beta);
        if (!(gamma > 0.0)) {
            status = KS_BREAKDOWN;
            break;
        }
        cs = gbar / gamma;
        sn = beta / gamma;
        const double phi = cs * phibar;
        phibar = sn * phibar;
        // w2 <- w, w <- (v - oldeps w2_old - delta w) / gamma, x += phi w, next v = z / beta
        for (int n = r0 + threadIdx.x; n < r1; n += blockDim.x)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int d = n * 3 + i;
                const double wo = w.s[d], w2o = w.shat[d];
                const double wn = (w.p[d] - oldeps * w2o - delta * wo) / gamma;
                w.shat[d] = wo;
                w.s[d] = wn;
                w.x[d] += phi * wn;
                w.p[d] = beta > 0.0 ? w.phat[d] / beta : 0.0;
            }
        ++it;
        if (!isfinite(phibar))
            status = KS_NONFINITE;
        else if (phibar <= rtol * beta1 || beta == 0.0)
            status = KS_CONVERGED;
        else if (it >= max_iter)
            status = KS_MAXIT;
        else if (!group_barrier(bar, nct, w.dflags))
            return false;
    }
    if (lc == 0 && threadIdx.x == 0) {
        KrylovScalars* sc = plan.scalars + t;
        const double rel = beta1 > 0.0 ? phibar / beta1 : 0.0;
        sc->bb = bb;
        sc->rr = rel * rel * bb;  // the relative residual the host reports is phibar / phibar_0
        sc->rho = beta;
        sc->rho_prev = oldb;
        sc->alpha = cs;
        sc->omega = sn;
        sc->tol2 = rtol * rtol * bb;
        sc->iter = it;
        sc->max_iter = max_iter;
        sc->status = status;
        sc->method = KM_MINRES;
    }
    return true;
}

// Two builds of the persistent solve: one 768-thread CTA per SM (single tissues with the
// two-level preconditioner, large tissues; up to 80 registers) and four 256-thread CTAs per SM
// (batches, small block-Jacobi tissues; registers capped at 64 so that 32 warps per SM hide the
// latency of the memory-bound batched solve).
// METHOD: 0 BiCGStab, 1 conjugate gradients, 2 MINRES (each its own build, so none pays the
// others' registers).
template <int THREADS, int MIN_BLOCKS, int METHOD>
__device__ __forceinline__ bool solve_by(const KrylovWork& w, const BatchPlan& plan, int t, int lc, int pbase,
                                         double rtol, int max_iter, double* smem, double* sb, double* red, double* ys,
                                         double* Ms, double* cs, float* cinv_s) {
    if (METHOD == 1) {
        bool indefinite = false;
        return solve_tissue_cg(w, plan, t, lc, pbase, rtol, max_iter, smem, sb, red, ys, Ms, cs, cinv_s, indefinite);
    }
    if (METHOD == 2) return solve_tissue_minres(w, plan, t, lc, pbase, rtol, max_iter, smem, sb);
    return solve_tissue(w, plan, t, lc, pbase, rtol, max_iter, smem, sb, red, ys, Ms, cs, cinv_s);
}

template <int THREADS, int MIN_BLOCKS, int METHOD>
__global__ void __launch_bounds__(THREADS, MIN_BLOCKS) k_bicgstab_batched(KrylovWork w, BatchPlan plan, double rtol,
                                                                        int max_iter) {

    __shared__ double smem[32 * 2];
    __shared__ double sb[2];
    __shared__ double red[32 * 6];  // per-warp partial sums of the coarse steps
    __shared__ double ys[kMaxAggPerCta * 6];
    __shared__ double Ms[kMaxAggPerCta * 36];  // M_a of the CTA's aggregates
    __shared__ double cs[kMaxCoarse];
    extern __shared__ float cinv_s[];  // this CTA's 6m rows of the coarse inverse (FP32)
    __shared__ int ticket;
    // a CTA of a multi-CTA group solves its tissue first (partials at its group's slots)
    const int j0 = plan.cta_list_ptr[blockIdx.x];
    if (j0 < plan.cta_list_ptr[blockIdx.x + 1]) {
        const int t = plan.cta_list[j0];
        if (plan.ncta[t] > 1 &&
            !solve_by<THREADS, MIN_BLOCKS, METHOD>(w, plan, t, blockIdx.x - plan.cta0[t], plan.cta0[t], rtol, max_iter, smem,
                                               sb, red, ys, Ms, cs, cinv_s))
            return;
    }
    // then every CTA takes single-CTA tissues from the queue until it is empty; their partials use
    // this CTA's own slots past the groups' (a group partner may still be reading the group's)
    for (;;) {
        if (threadIdx.x == 0) ticket = atomicAdd(plan.queue_head, 1);
        __syncthreads();
        const int q = ticket;
        __syncthreads();
        if (q >= plan.n_queue) break;
        if (!solve_by<THREADS, MIN_BLOCKS, METHOD>(w, plan, plan.queue[q], 0, plan.n_cta + blockIdx.x, rtol, max_iter, smem, sb,
                                               red, ys, Ms, cs, cinv_s))
            return;
    }
}

// Newton update of a batch: du[slave] = du[master] first (separate kernel), then per CTA of
// the plan uk += du over its rows (active tissues only) and ||du||^2 partials; the last CTA of
// each tissue (ticket in its barrier counter, which is idle between solves) sums the tissue's
// partials in order.
__global__ void k_newton_update_batched(KrylovWork w, BatchPlan plan, double* uk) {
    __shared__ double smem[32];
    __shared__ bool last;
    for (int j = plan.cta_list_ptr[blockIdx.x]; j < plan.cta_list_ptr[blockIdx.x + 1]; ++j) {
        const int t = plan.cta_list[j];
        if (!plan.active[t]) continue;
        const int c0 = plan.cta0[t], nct = plan.ncta[t];
        const int lc = blockIdx.x - c0;
        const int tr0 = plan.row0[t], tr1 = plan.row0[t + 1];
        const int r0 = tr0 + (int)((long long)(tr1 - tr0) * lc / nct);
        const int r1 = tr0 + (int)((long long)(tr1 - tr0) * (lc + 1) / nct);
        double v[1] = {0.0};
        for (int d = r0 * 3 + threadIdx.x; d < r1 * 3; d += blockDim.x) {
            const double du = w.x[d];
            v[0] += du * du;
            uk[d] = uk[d] + du;
        }
        block_sum<1>(v, smem);
        double* part = w.partials + 4 * c0;
        if (threadIdx.x == 0) {
            part[lc] = v[0];
            __threadfence();
            const uint32_t k = atomicAdd(&plan.barriers[t].count, 1u);
            last = (k == (uint32_t)nct - 1);
        }
        __syncthreads();
        if (last && threadIdx.x == 0) {
            __threadfence();
            double sum = 0.0;
            for (int i = 0; i < nct; ++i) sum += __ldcg(part + i);
            plan.du2[t] = sum;
            plan.barriers[t].count = 0u;
        }
        __syncthreads();
    }
}

// ---- multicolour block ILU(0) ---------------------------------------------------------------

__device__ __forceinline__ void mat3_mul(const double* a, const double* b, double* c) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) c[i * 3 + j] = a[i * 3] * b[j] + a[i * 3 + 1] * b[3 + j] + a[i * 3 + 2] * b[6 + j];
}

__device__ __forceinline__ void mat3_inv(const double* m, double* o, int32_t* dflags) {
    const double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) + m[2] * (m[3] * m[7] - m[4] * m[6]);
    if (det == 0.0 || !isfinite(det)) {
        atomicOr(dflags, DF_SINGULAR_DIAG);
        for (int k = 0; k < 9; ++k) o[k] = (k % 4 == 0) ? 1.0 : 0.0;
        return;
    }
    const double id = 1.0 / det;
    o[0] = (m[4] * m[8] - m[5] * m[7]) * id;
    o[1] = (m[2] * m[7] - m[1] * m[8]) * id;
    o[2] = (m[1] * m[5] - m[2] * m[4]) * id;
    o[3] = (m[5] * m[6] - m[3] * m[8]) * id;
    o[4] = (m[0] * m[8] - m[2] * m[6]) * id;
    o[5] = (m[2] * m[3] - m[0] * m[5]) * id;
    o[6] = (m[3] * m[7] - m[4] * m[6]) * id;
    o[7] = (m[1] * m[6] - m[0] * m[7]) * id;
    o[8] = (m[0] * m[4] - m[1] * m[3]) * id;
}

__device__ int find_col(const int32_t* colidx, int k0, int k1, int col) {
    int lo = k0, hi = k1 - 1;
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

// Factorise the rows of one colour class: for each lower block (i,K) in colour order,
// L_iK = A_iK U_KK^-1, then A_iJ -= L_iK U_KJ over row K's upper blocks that exist in row i
// (the ILU(0) rule: no fill outside the pattern); finally invert the U diagonal block of row i.
__global__ void k_ilu_factor_colour(KrylovWork w, IluPlan ilu, int c0, int c1) {
    const int q = c0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= c1) return;
    const int i = ilu.cnodes[q];
    const int r0 = w.rowptr[i], r1 = w.rowptr[i + 1];
    for (int t = ilu.lo_ptr[i]; t < ilu.lo_ptr[i + 1]; ++t) {
        const int k = ilu.lo_idx[t];
        const int K = w.colidx[k];
        double L[9];
        mat3_mul(ilu.lu + (size_t)k * 9, ilu.uinv + (size_t)K * 9, L);
#pragma unroll
        for (int m = 0; m < 9; ++m) ilu.lu[(size_t)k * 9 + m] = L[m];
        for (int u = ilu.up_ptr[K]; u < ilu.up_ptr[K + 1]; ++u) {
            const int j = ilu.up_idx[u];
            const int pos = find_col(w.colidx, r0, r1, w.colidx[j]);
            if (pos < 0) continue;
            double P[9];
            mat3_mul(L, ilu.lu + (size_t)j * 9, P);
#pragma unroll
            for (int m = 0; m < 9; ++m) ilu.lu[(size_t)pos * 9 + m] -= P[m];
        }
    }
    mat3_inv(ilu.lu + (size_t)w.diag[i] * 9, ilu.uinv + (size_t)i * 9, w.dflags);
}

// Forward solve of one colour class: y_i = r_i - sum_{lower k} L_ik y_K.
__global__ void k_ilu_fwd_colour(KrylovWork w, IluPlan ilu, int c0, int c1, const double* rin) {
    if (!running(w.sc)) return;
    const int q = c0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= c1) return;
    const int i = ilu.cnodes[q];
    double y0 = rin[i * 3], y1 = rin[i * 3 + 1], y2 = rin[i * 3 + 2];
    for (int t = ilu.lo_ptr[i]; t < ilu.lo_ptr[i + 1]; ++t) {
        const int k = ilu.lo_idx[t];
        const int K = w.colidx[k];
        const double* Lb = ilu.lu + (size_t)k * 9;
        const double a = ilu.y[K * 3], b = ilu.y[K * 3 + 1], c = ilu.y[K * 3 + 2];
        y0 -= Lb[0] * a + Lb[1] * b + Lb[2] * c;
        y1 -= Lb[3] * a + Lb[4] * b + Lb[5] * c;
        y2 -= Lb[6] * a + Lb[7] * b + Lb[8] * c;
    }
    ilu.y[i * 3] = y0;
    ilu.y[i * 3 + 1] = y1;
    ilu.y[i * 3 + 2] = y2;
}

// Backward solve of one colour class: z_i = U_ii^-1 (y_i - sum_{upper j} U_ij z_J).
__global__ void k_ilu_bwd_colour(KrylovWork w, IluPlan ilu, int c0, int c1, double* zout) {
    if (!running(w.sc)) return;
    const int q = c0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= c1) return;
    const int i = ilu.cnodes[q];
    double y0 = ilu.y[i * 3], y1 = ilu.y[i * 3 + 1], y2 = ilu.y[i * 3 + 2];
    for (int u = ilu.up_ptr[i]; u < ilu.up_ptr[i + 1]; ++u) {
        const int j = ilu.up_idx[u];
        const int J = w.colidx[j];
        const double* Ub = ilu.lu + (size_t)j * 9;
        const double a = zout[J * 3], b = zout[J * 3 + 1], c = zout[J * 3 + 2];
        y0 -= Ub[0] * a + Ub[1] * b + Ub[2] * c;
        y1 -= Ub[3] * a + Ub[4] * b + Ub[5] * c;
        y2 -= Ub[6] * a + Ub[7] * b + Ub[8] * c;
    }
    const double* D = ilu.uinv + (size_t)i * 9;
    zout[i * 3] = D[0] * y0 + D[1] * y1 + D[2] * y2;
    zout[i * 3 + 1] = D[3] * y0 + D[4] * y1 + D[5] * y2;
    zout[i * 3 + 2] = D[6] * y0 + D[7] * y1 + D[8] * y2;
}

__global__ void k_bicg_p_only(KrylovWork w) {
    if (!running(w.sc)) return;
    const double beta = (w.sc->rho / w.sc->rho_prev) * (w.sc->alpha / w.sc->omega);
    const double omega = w.sc->omega;
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < w.n_nodes * 3; d += gridDim.x * blockDim.x)
        w.p[d] = w.r[d] + beta * (w.p[d] - omega * w.v[d]);
}

__global__ void k_bicg_s_only(KrylovWork w) {
    if (!running(w.sc)) return;
    const double alpha = w.sc->alpha;
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < w.n_nodes * 3; d += gridDim.x * blockDim.x)
        w.s[d] = w.r[d] - alpha * w.v[d];
}

void ilu_apply(const KrylovWork& w, const IluPlan& ilu, const double* rin, double* zout, cudaStream_t s) {
    for (int c = 0; c < ilu.n_colours; ++c) {
        const int c0 = ilu.colour_ptr[c], c1 = ilu.colour_ptr[c + 1];
        if (c1 > c0) k_ilu_fwd_colour<<<(c1 - c0 + 127) / 128, 128, 0, s>>>(w, ilu, c0, c1, rin);
    }
    for (int c = ilu.n_colours - 1; c >= 0; --c) {
        const int c0 = ilu.colour_ptr[c], c1 = ilu.colour_ptr[c + 1];
        if (c1 > c0) k_ilu_bwd_colour<<<(c1 - c0 + 127) / 128, 128, 0, s>>>(w, ilu, c0, c1, zout);
    }
}

}  // namespace

cudaError_t launch_ilu_factor(const KrylovWork& w, const IluPlan& ilu, cudaStream_t s) {
    for (int c = 0; c < ilu.n_colours; ++c) {
        const int c0 = ilu.colour_ptr[c], c1 = ilu.colour_ptr[c + 1];
        if (c1 > c0) k_ilu_factor_colour<<<(c1 - c0 + 127) / 128, 128, 0, s>>>(w, ilu, c0, c1);
    }
    return cudaGetLastError();
}

cudaError_t launch_bicgstab_iteration_ilu(const KrylovWork& w, const IluPlan& ilu, cudaStream_t s) {
    const int vg = vec_grid(w.n_nodes), sg = spmv_grid(w.n_nodes);
    k_bicg_p_only<<<vg, kVecThreads, 0, s>>>(w);
    ilu_apply(w, ilu, w.p, w.phat, s);
    k_spmv<1><<<sg, kSpmvThreads, 0, s>>>(w, w.phat, w.v, 1);
    k_bicg_s_only<<<vg, kVecThreads, 0, s>>>(w);
    ilu_apply(w, ilu, w.s, w.shat, s);
    k_spmv<2><<<sg, kSpmvThreads, 0, s>>>(w, w.shat, w.t, 1);
    k_bicg_xr<<<vg, kVecThreads, 0, s>>>(w);
    return cudaGetLastError();
}

namespace {

// One thread per smoother group g of G nodes: gathers the 3G x 3G diagonal sub-block of J from
// the BSR3 rows (the group's diagonal blocks and the blocks that couple its nodes), inverts it by
// Gauss-Jordan elimination with partial pivoting (FP64) and writes the inverse column-major,
// rounded to FP32: it only preconditions (the solve tests convergence on the FP64 residual), and
// half the bytes keep the apply's loads near those of the 3x3 node blocks. A singular sub-block (zero or non-finite pivot) sets DF_SINGULAR_DIAG and leaves the
// identity, as the 3x3 block-Jacobi does.
__global__ void __launch_bounds__(128) k_group_jacobi_setup(KrylovWork w, int G) {
    const int NG = w.n_nodes / G;
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= NG) return;
    const int n3 = 3 * G, gs = g * G;
    double A[12][12], B[12][12];
    for (int r = 0; r < n3; ++r)
        for (int c = 0; c < n3; ++c) {
            A[r][c] = 0.0;
            B[r][c] = r == c ? 1.0 : 0.0;
        }
    for (int i = 0; i < G; ++i) {
        const int n = gs + i;
        for (int k = w.rowptr[n]; k < w.rowptr[n + 1]; ++k) {
            const int c = w.colidx[k];
            if (c < gs || c >= gs + G) continue;
            const double* blk = w.vals + (size_t)k * 9;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) A[3 * i + a][3 * (c - gs) + b] = blk[a * 3 + b];
        }
    }
    bool ok = true;
    for (int col = 0; col < n3 && ok; ++col) {
        int piv = col;
        double best = fabs(A[col][col]);
        for (int r = col + 1; r < n3; ++r)
            if (fabs(A[r][col]) > best) {
                best = fabs(A[r][col]);
                piv = r;
            }
        if (!(best > 0.0) || !isfinite(best)) {
            ok = false;
            break;
        }
        if (piv != col)
            for (int c = 0; c < n3; ++c) {
                const double ta = A[col][c], tb = B[col][c];
                A[col][c] = A[piv][c];
                B[col][c] = B[piv][c];
                A[piv][c] = ta;
                B[piv][c] = tb;
            }
        const double inv = 1.0 / A[col][col];
        for (int c = 0; c < n3; ++c) {
            A[col][c] *= inv;
            B[col][c] *= inv;
        }
        for (int r = 0; r < n3; ++r) {
            if (r == col) continue;
            const double f = A[r][col];
            if (f == 0.0) continue;
            for (int c = 0; c < n3; ++c) {
                A[r][c] -= f * A[col][c];
                B[r][c] -= f * B[col][c];
            }
        }
    }
    if (!ok) atomicOr(w.dflags, DF_SINGULAR_DIAG);
    for (int r = 0; r < n3; ++r)
        for (int c = 0; c < n3; ++c)
            reinterpret_cast<float*>(w.dinv)[(size_t)g * n3 * n3 + c * n3 + r] =
                (float)(ok ? 0.5 * (B[r][c] + B[c][r]) : (r == c ? 1.0 : 0.0));
}

// One CTA per aggregate a; thread t of a slot s computes entry e = (r, c) of the 6x6 coarse
// block (a, slot_agg[s]) by summing its Jacobian blocks in list order.
__global__ void k_coarse_assemble(KrylovWork w, CoarseAssembly ca, const double* __restrict__ pmode,
                                  double* __restrict__ a_cm) {
    const int a = blockIdx.x;
    if (a >= ca.n_agg) return;
    const int s0 = ca.agg_slot_ptr[a], ns = ca.agg_slot_ptr[a + 1] - s0;
    for (int t = threadIdx.x; t < ns * 36; t += blockDim.x) {
        const int s = s0 + t / 36, e = t % 36, r = e / 6, c = e % 6;
        double sum = 0.0;
        for (int q = ca.slot_ptr[s]; q < ca.slot_ptr[s + 1]; ++q) {
            const int k = ca.blk[q];
            const int i = ca.blk_row[q], j = __ldg(w.colidx + k);
            const double* J = w.vals + (size_t)k * 9;
            const double* Pi = pmode + (size_t)i * 18;
            const double* Pj = pmode + (size_t)j * 18;
            const double u0 = Pj[c], u1 = Pj[6 + c], u2 = Pj[12 + c];
#pragma unroll
            for (int d = 0; d < 3; ++d)
                sum += Pi[d * 6 + r] * (__ldg(J + d * 3) * u0 + __ldg(J + d * 3 + 1) * u1 + __ldg(J + d * 3 + 2) * u2);
        }
        if (ca.agg_tissue) {
            const int tt = ca.agg_tissue[a], g0 = ca.tissue_agg0[tt];
            const int R = 6 * (a - g0) + r, C = 6 * (ca.slot_agg[s] - g0) + c;
            a_cm[ca.tissue_base[tt] + (size_t)C + (size_t)R * ca.ld] = sum;
        } else {
            const int R = 6 * a + r, C = 6 * ca.slot_agg[s] + c;
            a_cm[(size_t)C + (size_t)R * ca.n_coarse] = sum;  // row-major
        }
    }
}

__global__ void k_coarse_empty(double* a_cm, int n, const int32_t* empty, int n_empty) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_empty) a_cm[(size_t)empty[i] * (n + 1)] = 1.0;
}

__global__ void k_coarse_unit(double* a_cm, const int64_t* offsets, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a_cm[offsets[i]] = 1.0;
}

// m = (m + m^T) / 2 for count matrices of order n, leading dimension ld, stride apart: the inverse
// of the symmetric coarse operator, made exactly symmetric so conjugate gradients see a symmetric
// preconditioner (the factorisation leaves rounding-level asymmetry).
__global__ void k_symmetrize(double* m, int n, int ld, long long stride, int count) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long per = (long long)n * n;
    if (i >= per * count) return;
    const int mat = (int)(i / per);
    const int r = (int)((i % per) / n), c = (int)(i % n);
    if (c <= r) return;
    double* a = m + mat * stride;
    const double v = 0.5 * (a[(size_t)r * ld + c] + a[(size_t)c * ld + r]);
    a[(size_t)r * ld + c] = v;
    a[(size_t)c * ld + r] = v;
}

}  // namespace

cudaError_t launch_coarse_assemble(const KrylovWork& w, const CoarseAssembly& ca, const double* pmode, double* a_cm,
                                   size_t a_cm_doubles, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(a_cm, 0, sizeof(double) * a_cm_doubles, s);
    if (e != cudaSuccess) return e;
    if (ca.n_agg > 0) k_coarse_assemble<<<ca.n_agg, 256, 0, s>>>(w, ca, pmode, a_cm);
    if (ca.n_empty > 0) {
        if (ca.agg_tissue)
            k_coarse_unit<<<(ca.n_empty + 255) / 256, 256, 0, s>>>(a_cm, ca.empty_offsets, ca.n_empty);
        else
            k_coarse_empty<<<(ca.n_empty + 255) / 256, 256, 0, s>>>(a_cm, ca.n_coarse, ca.empty, ca.n_empty);
    }
    return cudaGetLastError();
}

cudaError_t launch_group_jacobi_setup(const KrylovWork& w, int G, cudaStream_t s) {
    if (G < 2 || G > 4 || w.n_nodes % G != 0) return cudaErrorInvalidValue;
    const int NG = w.n_nodes / G;
    if (NG > 0) k_group_jacobi_setup<<<(NG + 127) / 128, 128, 0, s>>>(w, G);
    return cudaGetLastError();
}

cudaError_t launch_symmetrize(double* m, int n, int ld, long long stride, int count, cudaStream_t s) {
    const long long total = (long long)n * n * count;
    if (total > 0) k_symmetrize<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(m, n, ld, stride, count);
    return cudaGetLastError();
}

namespace {
void (*persist_kernel(int threads, int method))(KrylovWork, BatchPlan, double, int) {
    if (method == 2) return threads == 768 ? k_bicgstab_batched<768, 1, 2> : k_bicgstab_batched<256, 4, 2>;
    if (method == 1) return threads == 768 ? k_bicgstab_batched<768, 1, 1> : k_bicgstab_batched<256, 4, 1>;
    return threads == 768 ? k_bicgstab_batched<768, 1, 0> : k_bicgstab_batched<256, 4, 0>;
}
}  // namespace

int persistent_max_grid(int device, int threads) {
    int sms = 0, occ = 0;
    if (threads != 256 && threads != 768) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    occ = 1 << 30;
    for (int method = 0; method < 3; ++method) {  // every method's build must fit the same plan
        const auto kern = persist_kernel(threads, method);
        int o = 0;
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kCoarseSmemBytes) != cudaSuccess)
            return 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, threads, 0) != cudaSuccess) return 0;
        occ = o < occ ? o : occ;
        if (threads == 768) {  // the two-level solve adds its coarse row block: still one CTA per SM
            int occ_c = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_c, kern, threads, kCoarseSmemBytes) != cudaSuccess ||
                occ_c < 1)
                return 0;
        }
    }
    const int want = threads == 768 ? 1 : 4;  // the CTAs per SM each build is compiled for
    return sms * (occ < want ? occ : want);
}

cudaError_t launch_bicgstab_batched(const KrylovWork& w, const BatchPlan& plan, double rtol, int max_iter,
                                    int threads, cudaStream_t s) {
    KrylovWork wc = w;
    BatchPlan pc = plan;
    void* args[] = {&wc, &pc, &rtol, &max_iter};
    const size_t smem = plan.agg_per_cta > 0 ? sizeof(float) * 6 * plan.agg_per_cta * (size_t)plan.n_coarse : 0;
    if (smem > (size_t)kCoarseSmemBytes) return cudaErrorInvalidValue;
    if (threads != 256 && threads != 768) return cudaErrorInvalidValue;
    const int method = plan.minres ? 2 : (plan.cg ? 1 : 0);
    return cudaLaunchCooperativeKernel(reinterpret_cast<void*>(persist_kernel(threads, method)), dim3(plan.n_cta),
                                       dim3(threads), args, smem, s);
}

cudaError_t launch_newton_update_batched(const KrylovWork& w, const BatchPlan& plan, double* uk,
                                         const int32_t* slaves, const int32_t* masters, int32_t n_pairs,
                                         cudaStream_t s) {
    if (n_pairs > 0) k_equate_slaves<<<(n_pairs + 255) / 256, 256, 0, s>>>(w.x, slaves, masters, n_pairs);
    k_newton_update_batched<<<plan.n_cta, 256, 0, s>>>(w, plan, uk);
    return cudaGetLastError();
}

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

cudaError_t launch_residual(const KrylovWork& w, const double* xin, const double* b, double* rout, cudaStream_t s) {
    k_residual<<<spmv_grid(w.n_nodes), kSpmvThreads, 0, s>>>(w, xin, b, rout);
    return cudaGetLastError();
}

cudaError_t launch_axpy(int n, double a, const double* x, double* y, cudaStream_t s) {
    k_axpy<<<vec_grid(n / 3 + 1), kVecThreads, 0, s>>>(n, a, x, y);
    return cudaGetLastError();
}

cudaError_t launch_newton_update(const KrylovWork& w, double* uk, const int32_t* slaves,
                                 const int32_t* masters, int32_t n_pairs, cudaStream_t s) {
    if (n_pairs > 0) k_equate_slaves<<<(n_pairs + 255) / 256, 256, 0, s>>>(w.x, slaves, masters, n_pairs);
    k_newton_update<<<vec_grid(w.n_nodes), kVecThreads, 0, s>>>(w, uk);
    return cudaGetLastError();
}

}  // namespace tfb
