// tf_direct.cu -- sparse direct solve of J du = g with cuSOLVER, timed beside the Krylov solve.
//
// The reference factorises every Newton system from scratch with Pardiso (phases 11/22/33,
// NewtonRaphsonSolver.cpp:498-763). The library's own solve is BiCGStab; this file offers the
// direct alternative on the GPU for comparison and cross-checks: the BSR3 matrix is expanded to
// scalar CSR by a kernel and handed to cuSOLVER's sparse Cholesky (J is symmetric on the
// elastic path). J is positive definite at rest, but growth against clamped boundaries puts
// elements in compression, whose geometric stiffness can make J indefinite; Cholesky then meets
// a non-positive pivot. Sparse QR handles that case but costs ~20x more (80 s on the 180k-unknown
// wing-disc system), so it runs only up to kQrMaxRows unknowns; larger indefinite systems report
// "not positive definite".
#include <cuda_runtime.h>
#include <cusolverSp.h>
#include <cusparse.h>

#include "tf_internal.cuh"

namespace tfb {
namespace {

constexpr int kQrMaxRows = 30000;  // largest system the QR fallback takes

// Scalar CSR of a BSR3 matrix: row 3A+i holds, for every block k of block row A (sorted), the
// columns 3*colidx[k] + j, j = 0..2.
__global__ void k_bsr3_to_csr(int32_t n_nodes, const int32_t* rowptr, const int32_t* colidx, const double* vals,
                              int32_t* crow, int32_t* ccol, double* cval) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= 3 * n_nodes) return;
    const int A = r / 3, i = r - 3 * A;
    const int k0 = rowptr[A], k1 = rowptr[A + 1];
    const int nb = k1 - k0;
    const int start = 9 * k0 + 3 * i * nb;
    crow[r] = start;
    if (r == 3 * n_nodes - 1) crow[r + 1] = 9 * rowptr[n_nodes];
    for (int k = k0; k < k1; ++k)
        for (int j = 0; j < 3; ++j) {
            const int pos = start + 3 * (k - k0) + j;
            ccol[pos] = 3 * colidx[k] + j;
            cval[pos] = vals[(size_t)k * 9 + i * 3 + j];
        }
}

}  // namespace

int direct_solve_bsr3(int32_t n_nodes, int64_t nnzb, const int32_t* rowptr, const int32_t* colidx, const double* vals,
                      const double* b, double* x, cudaStream_t s, float* ms, int* method) {
    const int n = 3 * n_nodes;
    const int64_t nnz = 9 * nnzb;
    if (nnz > INT32_MAX) return -1;
    int32_t *crow = nullptr, *ccol = nullptr;
    double* cval = nullptr;
    int rc = 0;
    cusolverSpHandle_t h = nullptr;
    cusparseMatDescr_t d = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaMalloc(&crow, sizeof(int32_t) * (n + 1)) != cudaSuccess || cudaMalloc(&ccol, sizeof(int32_t) * nnz) != cudaSuccess ||
        cudaMalloc(&cval, sizeof(double) * nnz) != cudaSuccess) {
        rc = -3;
    }
    if (rc == 0) {
        k_bsr3_to_csr<<<(n + 255) / 256, 256, 0, s>>>(n_nodes, rowptr, colidx, vals, crow, ccol, cval);
        if (cudaGetLastError() != cudaSuccess) rc = -2;
    }
    if (rc == 0 && (cusolverSpCreate(&h) != CUSOLVER_STATUS_SUCCESS || cusolverSpSetStream(h, s) != CUSOLVER_STATUS_SUCCESS ||
                    cusparseCreateMatDescr(&d) != CUSPARSE_STATUS_SUCCESS))
        rc = -2;
    if (rc == 0) {
        cusparseSetMatType(d, CUSPARSE_MATRIX_TYPE_GENERAL);
        cusparseSetMatIndexBase(d, CUSPARSE_INDEX_BASE_ZERO);
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, s);
        int singular = -1;
        const int reorder = 3;  // METIS nested dissection
        cusolverStatus_t st = cusolverSpDcsrlsvchol(h, n, (int)nnz, d, cval, crow, ccol, b, 0.0, reorder, x, &singular);
        *method = 1;
        bool not_spd = false;
        if (st != CUSOLVER_STATUS_SUCCESS || singular >= 0) {
            if (n <= kQrMaxRows) {
                st = cusolverSpDcsrlsvqr(h, n, (int)nnz, d, cval, crow, ccol, b, 0.0, reorder, x, &singular);
                *method = 2;
            } else {
                not_spd = true;
            }
        }
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(ms, e0, e1);
        if (not_spd) rc = 4;
        else if (st != CUSOLVER_STATUS_SUCCESS) rc = -2;
        else if (singular >= 0) rc = 3;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (d) cusparseDestroyMatDescr(d);
    if (h) cusolverSpDestroy(h);
    cudaFree(crow);
    cudaFree(ccol);
    cudaFree(cval);
    return rc;
}

}  // namespace tfb
