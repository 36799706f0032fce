// tf_dense.cu -- dense FP64 inverses of the two-level preconditioner's coarse operators.
//
// The coarse operator P^T J P of the two-level preconditioner is a dense matrix of a few hundred
// (a batch tissue) to two thousand (one tissue) unknowns, refreshed every few dozen solves. Its
// inverse is applied as a dense product inside the persistent solve. Both kernels here invert in
// place by Gauss-Jordan elimination with partial pivoting (the pivot of column k is the entry of
// largest magnitude in rows k..n-1, the first one on ties), column-major storage:
//
//   step k:  swap rows k and p;  piv = A[k][k]
//            column k:       A[i][k] <- -A[i][k] / piv (i != k),  A[k][k] <- 1 / piv
//            other columns:  A[k][j] <- A[k][j] / piv,  A[i][j] <- A[i][j] - A[i][k] A[k][j] (i != k)
//
// after which the columns are swapped back in reverse order of the row swaps. A zero or
// non-finite pivot stops the elimination and reports the step (info = k + 1), as LAPACK's getrf.
//
// k_gj_batched: one CTA per matrix (a batch's per-tissue operators, each with its own order in a
//   common leading dimension); a step is CTA-local: threads over rows, the pivot column and row
//   staged in shared memory.
// k_gj_coop: one matrix over a cooperative grid (a single tissue's operator); every CTA owns a
//   contiguous block of columns, rows over its threads. The column k every CTA needs is staged by
//   its owner in a double buffer at the end of step k-1, so a step needs one grid barrier; every
//   CTA finds the same pivot from the same staged column (same data, same order). The barrier's
//   wait is bounded (about 2 s of SM clock) and reports a timeout instead of hanging.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <vector>

#include "../../include/tf_b200.h"
#include "tf_internal.cuh"

namespace tfb {
namespace {

constexpr int kGjThreads = 512;
constexpr int kGjCoopThreads = 256;
constexpr long long kGjBarrierCycles = 4000000000ll;

// Pivot of the staged column f[0..n) among rows k..n-1: largest |f|, the smallest row on ties.
// Every thread of the CTA returns the same row.
__device__ int pivot_row(const double* f, int k, int n, double* sval, int* sidx) {
    double best = -1.0;
    int bi = n;
    for (int i = k + threadIdx.x; i < n; i += blockDim.x) {
        const double a = fabs(f[i]);
        if (a > best || (a == best && i < bi)) {
            best = a;
            bi = i;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, off);
        const int oi = __shfl_down_sync(0xffffffffu, bi, off);
        if (ob > best || (ob == best && oi < bi)) {
            best = ob;
            bi = oi;
        }
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (lane == 0) {
        sval[warp] = best;
        sidx[warp] = bi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < nw; ++w)
            if (sval[w] > sval[0] || (sval[w] == sval[0] && sidx[w] < sidx[0])) {
                sval[0] = sval[w];
                sidx[0] = sidx[w];
            }
    }
    __syncthreads();
    const int p = sidx[0];
    __syncthreads();
    return p;
}

// one CTA inverts matrix t: order n[t], column-major with leading dimension ld at a + base[t]
__global__ void __launch_bounds__(kGjThreads) k_gj_batched(double* a_all, const int64_t* base, const int32_t* order,
                                                           int ld, int32_t* info) {
    extern __shared__ double sm[];
    double* f = sm;          // [ld] pivot column
    double* rowk = sm + ld;  // [ld] pivot row
    int* ipiv = reinterpret_cast<int*>(sm + 2 * ld);
    __shared__ double sval[32];
    __shared__ int sidx[32];
    const int t = blockIdx.x;
    double* A = a_all + base[t];
    const int n = order[t];
    int bad = 0;
    for (int k = 0; k < n; ++k) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) f[i] = A[i + (size_t)k * ld];
        __syncthreads();
        const int p = pivot_row(f, k, n, sval, sidx);  // n when every candidate is NaN
        const double piv = p < n ? f[p] : 0.0;
        if (!(fabs(piv) > 0.0) || !isfinite(piv)) {
            bad = k + 1;
            break;
        }
        // swap rows k and p; stage row k (after the swap) and the column
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const double ak = A[k + (size_t)j * ld], ap = A[p + (size_t)j * ld];
            A[k + (size_t)j * ld] = ap;
            A[p + (size_t)j * ld] = ak;
            rowk[j] = ap;
        }
        if (threadIdx.x == 0) ipiv[k] = p;
        __syncthreads();
        if (threadIdx.x == 0 && p != k) {
            const double tmp = f[k];
            f[k] = f[p];
            f[p] = tmp;
        }
        __syncthreads();
        const double inv = 1.0 / piv;
        // one thread per entry (rows fastest: coalesced), each reading only its own entry
        for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
            const int i = idx % n, j = idx / n;
            double* a = A + i + (size_t)j * ld;
            if (i == k)
                *a = j == k ? inv : rowk[j] * inv;
            else
                *a = j == k ? -f[i] * inv : *a - f[i] * (rowk[j] * inv);
        }
        __syncthreads();
    }
    if (bad) {
        if (threadIdx.x == 0) info[t] = bad;
        return;
    }
    // undo the row swaps as column swaps, last first; each thread owns its rows
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        for (int k = n - 1; k >= 0; --k) {
            const int p = ipiv[k];
            if (p == k) continue;
            const double a = A[i + (size_t)k * ld];
            A[i + (size_t)k * ld] = A[i + (size_t)p * ld];
            A[i + (size_t)p * ld] = a;
        }
    if (threadIdx.x == 0) info[t] = 0;
}

// Bounded generation barrier over the whole cooperative grid (bar[0] arrivals, bar[1] generation).
__device__ bool coop_barrier(unsigned* bar, int32_t* status) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        volatile unsigned* vgen = bar + 1;
        const unsigned g = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(bar, 1u);
        if (arrived == gridDim.x - 1) {
            bar[0] = 0u;
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            const long long t0 = clock64();
            unsigned polls = 0;
            while (*vgen == g) {
                if ((++polls & 255u) == 0u && clock64() - t0 > kGjBarrierCycles) {
                    atomicExch(status, -1);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        if (*reinterpret_cast<volatile int32_t*>(status) < 0) ok = 0;
    }
    __syncthreads();
    return ok != 0;
}

// The cooperative inverse of one n x n column-major matrix (leading dimension n). colbuf [2][n]
// stages the pivot columns, ipiv [n] the pivot rows, bar [2] the barrier (zeroed), status: 0 ok,
// k + 1 for a zero pivot at step k, -1 barrier timeout.
__global__ void __launch_bounds__(kGjCoopThreads) k_gj_coop(double* A, int n, double* colbuf, int32_t* ipiv,
                                                            unsigned* bar, int32_t* status) {
    extern __shared__ double sm[];
    double* f = sm;          // [n]
    double* rowk = sm + n;   // [columns of this CTA]
    __shared__ double sval[32];
    __shared__ int sidx[32];
    const int c0 = (int)((long long)n * blockIdx.x / gridDim.x);
    const int c1 = (int)((long long)n * (blockIdx.x + 1) / gridDim.x);
    if (c0 <= 0 && 0 < c1)
        for (int i = threadIdx.x; i < n; i += blockDim.x) colbuf[i] = A[i];  // column 0, staged
    if (!coop_barrier(bar, status)) return;
    for (int k = 0; k < n; ++k) {
        const double* col = colbuf + (size_t)(k & 1) * n;
        for (int i = threadIdx.x; i < n; i += blockDim.x) f[i] = __ldcg(col + i);
        __syncthreads();
        const int p = pivot_row(f, k, n, sval, sidx);  // n when every candidate is NaN
        const double piv = p < n ? f[p] : 0.0;
        if (!(fabs(piv) > 0.0) || !isfinite(piv)) {  // every CTA sees the same pivot and stops
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(status, 0, k + 1);
            return;
        }
        if (threadIdx.x == 0 && p != k) {
            const double tmp = f[k];
            f[k] = f[p];
            f[p] = tmp;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) ipiv[k] = p;
        for (int j = c0 + threadIdx.x; j < c1; j += blockDim.x) {
            const double ak = A[k + (size_t)j * n], ap = A[p + (size_t)j * n];
            A[k + (size_t)j * n] = ap;
            A[p + (size_t)j * n] = ak;
            rowk[j - c0] = ap;
        }
        __syncthreads();
        const double inv = 1.0 / piv;
        for (int j = c0; j < c1; ++j) {
            double* a = A + (size_t)j * n;
            if (j == k) {
                for (int i = threadIdx.x; i < n; i += blockDim.x) a[i] = i == k ? inv : -f[i] * inv;
            } else {
                const double r = rowk[j - c0] * inv;
                for (int i = threadIdx.x; i < n; i += blockDim.x) a[i] = i == k ? r : a[i] - f[i] * r;
            }
        }
        __syncthreads();
        if (k + 1 < n && c0 <= k + 1 && k + 1 < c1) {  // stage the next pivot column
            double* nxt = colbuf + (size_t)((k + 1) & 1) * n;
            for (int i = threadIdx.x; i < n; i += blockDim.x) nxt[i] = A[i + (size_t)(k + 1) * n];
        }
        if (!coop_barrier(bar, status)) return;
    }
}

// Undo the row swaps of k_gj_coop as column swaps, last first; one thread per row.
__global__ void k_gj_unswap(double* A, int n, const int32_t* ipiv, const int32_t* status) {
    if (*status != 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = n - 1; k >= 0; --k) {
        const int p = ipiv[k];
        if (p == k) continue;
        const double a = A[i + (size_t)k * n];
        A[i + (size_t)k * n] = A[i + (size_t)p * n];
        A[i + (size_t)p * n] = a;
    }
}

}  // namespace

cudaError_t launch_invert_batched(double* a, const int64_t* base, const int32_t* order, int ld, int count,
                                  int32_t* info, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    const size_t smem = sizeof(double) * 2 * (size_t)ld + sizeof(int) * (size_t)ld;
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k_gj_batched, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_gj_batched<<<count, kGjThreads, smem, s>>>(a, base, order, ld, info);
    return cudaGetLastError();
}

size_t invert_coop_scratch_bytes(int n) {
    return sizeof(double) * 2 * (size_t)n + sizeof(int32_t) * ((size_t)n + 4);
}

cudaError_t launch_invert_coop(double* a, int n, void* scratch, int32_t* status, int device, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    double* colbuf = static_cast<double*>(scratch);
    int32_t* ipiv = reinterpret_cast<int32_t*>(colbuf + 2 * (size_t)n);
    unsigned* bar = reinterpret_cast<unsigned*>(ipiv + n);
    int sms = 0, occ = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    int grid = sms < n ? sms : n;
    const size_t smem = sizeof(double) * ((size_t)n + (size_t)(n + grid - 1) / grid + 1);
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    if ((e = cudaFuncSetAttribute(k_gj_coop, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
        return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_gj_coop, kGjCoopThreads, smem)) != cudaSuccess)
        return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    if ((e = cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(status, 0, sizeof(int32_t), s)) != cudaSuccess) return e;
    void* args[] = {&a, &n, &colbuf, &ipiv, &bar, &status};
    if ((e = cudaLaunchCooperativeKernel(reinterpret_cast<void*>(k_gj_coop), dim3(grid), dim3(kGjCoopThreads), args, smem,
                                         s)) != cudaSuccess)
        return e;
    k_gj_unswap<<<(n + 255) / 256, 256, 0, s>>>(a, n, ipiv, status);
    return cudaGetLastError();
}

}  // namespace tfb

// Inverts `count` dense n x n matrices of host memory in place with the kernels above (one CTA per
// matrix when cooperative = 0, else each over a cooperative grid). info[t] = 0, or k + 1 for a zero
// pivot at step k (that matrix is then left partly eliminated). Host copies on a private stream.
extern "C" int tf_invert_dense(int32_t device, int32_t n, int32_t count, int32_t cooperative, double* a,
                               int32_t* info) {
    if (n <= 0 || count <= 0 || !a || !info) return TF_ERR_ARGUMENT;
    if (cudaSetDevice(device) != cudaSuccess) return TF_ERR_CUDA;
    const size_t nn = (size_t)n * n;
    double* d_a = nullptr;
    int64_t* d_base = nullptr;
    int32_t *d_order = nullptr, *d_info = nullptr;
    void* scratch = nullptr;
    cudaStream_t s = nullptr;
    int rc = TF_OK;
    if (cudaMalloc(&d_a, sizeof(double) * nn * count) != cudaSuccess || cudaMalloc(&d_base, sizeof(int64_t) * count) != cudaSuccess ||
        cudaMalloc(&d_order, sizeof(int32_t) * count) != cudaSuccess || cudaMalloc(&d_info, sizeof(int32_t) * count) != cudaSuccess ||
        cudaMalloc(&scratch, tfb::invert_coop_scratch_bytes(n)) != cudaSuccess)
        rc = TF_ERR_OUT_OF_MEMORY;
    if (rc == TF_OK && cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) rc = TF_ERR_CUDA;
    if (rc == TF_OK) {
        std::vector<int64_t> base(count);
        std::vector<int32_t> order(count, n);
        for (int t = 0; t < count; ++t) base[t] = (int64_t)t * (int64_t)nn;
        bool ok = cudaMemcpyAsync(d_a, a, sizeof(double) * nn * count, cudaMemcpyHostToDevice, s) == cudaSuccess &&
                  cudaMemcpyAsync(d_base, base.data(), sizeof(int64_t) * count, cudaMemcpyHostToDevice, s) == cudaSuccess &&
                  cudaMemcpyAsync(d_order, order.data(), sizeof(int32_t) * count, cudaMemcpyHostToDevice, s) == cudaSuccess;
        if (ok && !cooperative) ok = tfb::launch_invert_batched(d_a, d_base, d_order, n, count, d_info, s) == cudaSuccess;
        for (int t = 0; ok && cooperative && t < count; ++t)
            ok = tfb::launch_invert_coop(d_a + (size_t)t * nn, n, scratch, d_info + t, device, s) == cudaSuccess;
        ok = ok && cudaMemcpyAsync(a, d_a, sizeof(double) * nn * count, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
             cudaMemcpyAsync(info, d_info, sizeof(int32_t) * count, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
             cudaStreamSynchronize(s) == cudaSuccess;
        if (!ok) rc = TF_ERR_CUDA;
    }
    if (s) cudaStreamDestroy(s);
    cudaFree(d_a);
    cudaFree(d_base);
    cudaFree(d_order);
    cudaFree(d_info);
    cudaFree(scratch);
    return rc;
}
