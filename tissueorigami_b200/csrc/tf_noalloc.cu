// tf_noalloc.cu -- tf_solve_bsr_noalloc: the block-Jacobi BiCGStab solve of tf_solve for callers
// that cannot allocate GPU memory.
//
// Who needs it: host applications that hand all device memory to their own allocator or to
// a fixed pool reserved at start-up (a framework's caching allocator, a simulation driver that
// forbids allocation once it runs), and so cannot let a library call cudaMalloc / cudaFree
// per solve. Such a caller already holds the matrix, the right-hand side and the output on the
// device; what the solve still needs is scratch: the eight BiCGStab work vectors, the 3x3
// block-Jacobi inverses, the diagonal slots, the reduction partials and the device scalars.
// Here that scratch is one file-scope __device__ array of fixed size, reserved when the
// library is loaded and kept by every GPU that loads it until the process exits.
//
// Limits and rules:
//   - at most kNoAllocMaxNodes block rows (3 * kNoAllocMaxNodes unknowns); larger systems are
//     rejected with TF_ERR_TOO_LARGE before any GPU work;
//   - every call looks up the array's device address on the current device with
//     cudaGetSymbolAddress (which allocates nothing), so a device reset or a new primary context
//     never leaves a stale address behind. Under CUDA's lazy module loading the array is reserved
//     when the library's kernels first load on a device, which is inside the first call there:
//     a host whose pool takes all device memory must make one call (or any other call of this
//     library) before its pool claims the memory; a failed reservation returns
//     TF_ERR_OUT_OF_MEMORY;
//   - the column indices of each block row must be sorted ascending (the diagonal block is
//     found by binary search);
//   - the call synchronises its stream after every 32 iterations to poll convergence, so it
//     cannot be called while that stream is being captured into a CUDA graph;
//   - every call on a device shares the one array, which keeps the previous call's contents:
//     the call clears the parts that must start at zero (scalars, tickets, flags) itself, and
//     calls that overlap on the GPU (two streams, two host threads) race on it.
// The call makes no cudaMalloc, cudaFree, cudaMallocHost or graph instantiation; it only
// launches kernels and copies the 128-byte scalar block into a host stack variable to poll
// convergence.
#include <cuda_runtime.h>

#include <cstring>

#include "../../include/tf_b200.h"
#include "tf_internal.cuh"

using namespace tfb;

namespace {

constexpr int32_t kNoAllocMaxNodes = TF_NOALLOC_MAX_NODES;
constexpr size_t kVec = 3 * (size_t)kNoAllocMaxNodes;       // doubles in one [N][3] vector
constexpr size_t kDinv = 9 * (size_t)kNoAllocMaxNodes;      // block-Jacobi inverses
constexpr size_t kDiag = (size_t)kNoAllocMaxNodes / 2 + 1;  // int32 diagonal slots, as doubles
constexpr size_t kPartials = 4096;                         // >= 2 x the largest reduction grid
constexpr size_t kScalars = (sizeof(KrylovScalars) + 7) / 8 + 2;  // scalars + device flags
constexpr size_t kScratchDoubles = 8 * kVec + kDinv + kDiag + kPartials + kScalars;

static_assert(sizeof(KrylovScalars) % 8 == 0, "scalar block must be a whole number of doubles");

// The scratch: 8 work vectors | Dinv | diag slots | partials | scalars + flags.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Device address of the scratch array in the current device's context. Looked up on every call:
// the lookup allocates nothing, and an address cached across calls would go stale once the
// context is destroyed and made again (cudaDeviceReset), when the module reloads elsewhere.
cudaError_t scratch_address(double** out) {
    void* p = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (err != cudaSuccess) return err;
    *out = static_cast<double*>(p);
    return cudaSuccess;
}

int status_of(int ks) {
    switch (ks) {
        case KS_CONVERGED: return TF_OK;
        case KS_BREAKDOWN: return TF_KRYLOV_BREAKDOWN;
        case KS_NONFINITE: return TF_NONFINITE;
        default: return TF_KRYLOV_MAX_ITERS;
    }
}

}  // namespace

extern "C" int tf_solve_bsr_noalloc(int32_t n_nodes, const int32_t* d_rowptr, const int32_t* d_colidx,
                                    const double* d_vals, const double* d_g, double* d_du, double rtol,
                                    int32_t max_iters, void* stream, int32_t* iters, double* rel_res) {
    if (n_nodes > kNoAllocMaxNodes) return TF_ERR_TOO_LARGE;
    if (n_nodes <= 0 || !d_rowptr || !d_colidx || !d_vals || !d_g || !d_du || max_iters <= 0 || !(rtol >= 0))
        return TF_ERR_ARGUMENT;
    double* base = nullptr;
    const cudaError_t serr = scratch_address(&base);
    if (serr != cudaSuccess) {
        cudaGetLastError();
        return serr == cudaErrorMemoryAllocation ? TF_ERR_OUT_OF_MEMORY : TF_ERR_CUDA;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    KrylovWork w;
    w.n_nodes = n_nodes;
    w.rowptr = d_rowptr;
    w.colidx = d_colidx;
    w.vals = d_vals;
    w.x = d_du;
    w.b = const_cast<double*>(d_g);  // read only by the kernels
    double* v = base;
    w.r = v + 0 * kVec;
    w.rhat = v + 1 * kVec;
    w.p = v + 2 * kVec;
    w.v = v + 3 * kVec;
    w.s = v + 4 * kVec;
    w.t = v + 5 * kVec;
    w.phat = v + 6 * kVec;
    w.shat = v + 7 * kVec;
    w.dinv = v + 8 * kVec;
    int32_t* diag = reinterpret_cast<int32_t*>(w.dinv + kDinv);
    w.diag = diag;
    w.partials = w.dinv + kDinv + kDiag;
    w.n_partials = (int32_t)kPartials;
    w.sc = reinterpret_cast<KrylovScalars*>(w.partials + kPartials);
    w.dflags = reinterpret_cast<int32_t*>(reinterpret_cast<double*>(w.sc) + (sizeof(KrylovScalars) + 7) / 8);
    w.pk_ptr = w.pk_col = w.pk_blk = nullptr;  // the caller's matrix is all there is
    w.pk_vals = nullptr;

    // scalars, tickets and flags must start at zero; everything else is overwritten
    if (cudaMemsetAsync(w.sc, 0, sizeof(double) * kScalars, s) != cudaSuccess) return TF_ERR_CUDA;
    if (launch_find_diag(d_rowptr, d_colidx, n_nodes, diag, w.dflags, s) != cudaSuccess) return TF_ERR_CUDA;
    if (launch_block_jacobi_setup(w, s) != cudaSuccess) return TF_ERR_CUDA;
    if (launch_krylov_init(w, rtol, max_iters, s) != cudaSuccess) return TF_ERR_CUDA;
    KrylovScalars h;
    std::memset(&h, 0, sizeof(h));
    const int chunk = 32;
    const int max_chunks = max_iters / chunk + 2;
    for (int c = 0; c < max_chunks; ++c) {
        for (int i = 0; i < chunk; ++i)
            if (launch_bicgstab_iteration(w, s) != cudaSuccess) return TF_ERR_CUDA;
        if (cudaMemcpyAsync(&h, w.sc, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess) return TF_ERR_CUDA;
        if (cudaStreamSynchronize(s) != cudaSuccess) return TF_ERR_CUDA;
        if (h.status != KS_RUNNING) break;
    }
    int32_t flags = 0;
    if (cudaMemcpyAsync(&flags, w.dflags, sizeof(flags), cudaMemcpyDeviceToHost, s) != cudaSuccess) return TF_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return TF_ERR_CUDA;
    if (flags & DF_PATTERN_MISS) return TF_ERR_ARGUMENT;  // a block row without its diagonal block
    if (iters) *iters = h.iter;
    if (rel_res) *rel_res = h.bb > 0 ? sqrt(h.rr / h.bb) : 0.0;
    return status_of(h.status);
}
