// tf_packing.cu -- node-node packing (contact) of a single tissue on the device.
//
// Once per time step, after the growth (Simulation::runOneStep, Simulation.cpp:6065-6076):
//  * node masses (Simulation::updateNodeMasses, :7587-7596): every node collects det(Fg) x the
//    element's reference volume / 6 from each of its elements;
//  * the detection thresholds (Simulation::detectPacingNodes, :7997-8016, with
//    getAverageSideLength, :3197-3262): the x-y bounding box of the nodes, the average triangle
//    side of every columnar element's apical face (and basal face where it is basal-exposed)
//    summed into a 10 x 5 grid by the element centre's relative position in the box, the cell
//    averages times 0.4 as the detection distances, 0.4 x the overall average as
//    Simulation::packingThreshold;
//  * the pairs (:8036-8080): apical or basal nodes (mass > 0) of the same placement that share no
//    element (no block of the element pattern joins them) and lie closer than the detection
//    distance of the first node's grid cell, i < j. Instead of the reference's all-pairs loop, the
//    eligible nodes are hashed into cells of the largest detection distance and each node visits
//    the 27 cells around its own; the pairs are then counted per node, scanned, written and each
//    node's partners sorted, which gives the reference's (i, j) visiting order.
// Every Newton iteration (calculatePackingForcesImplicit3D / calculatePackingJacobian3D,
// :7307-7575): one thread per pair adds the force to g and the derivative blocks to J.
//
// The box and grid sums use atomics, so their last bits depend on the order of the additions;
// the reference's box loop also leaves node 0 out of the maximum (its first comparison updates
// only the minimum), which is kept; its further quirk - a node that is a new running minimum
// is not compared with the maximum - only matters for coordinates that decrease along the whole
// node order and is not reproduced.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "tf_internal.cuh"

namespace tfb {
namespace {

constexpr int kPkThreads = 256;
constexpr int kScanBlock = 1024;

__device__ __forceinline__ double atomic_min_d(double* a, double v) {
    unsigned long long* p = reinterpret_cast<unsigned long long*>(a);
    unsigned long long old = *p, assumed;
    while (v < __longlong_as_double((long long)old)) {
        assumed = old;
        old = atomicCAS(p, assumed, (unsigned long long)__double_as_longlong(v));
        if (old == assumed) break;
    }
    return __longlong_as_double((long long)old);
}

__device__ __forceinline__ double atomic_max_d(double* a, double v) {
    unsigned long long* p = reinterpret_cast<unsigned long long*>(a);
    unsigned long long old = *p, assumed;
    while (v > __longlong_as_double((long long)old)) {
        assumed = old;
        old = atomicCAS(p, assumed, (unsigned long long)__double_as_longlong(v));
        if (old == assumed) break;
    }
    return __longlong_as_double((long long)old);
}

__global__ void k_pk_init(PackParams* prm) {
    if (threadIdx.x == 0) {
        prm->bb0[0] = prm->bb0[1] = 1e300;
        prm->bbs[0] = prm->bbs[1] = -1e300;  // the maximum until k_pk_grid_final
        prm->col_sum = prm->col_cnt = 0.0;
        prm->threshold = prm->cell = 0.0;
    }
    if (threadIdx.x < 50) {
        prm->grid_sum[threadIdx.x] = 0.0;
        prm->grid_cnt[threadIdx.x] = 0.0;
    }
}

// node masses (mass zeroed before) and the bounding box
__global__ void __launch_bounds__(kPkThreads) k_pk_mass(PackArgs a) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.n_elems) return;
    const double* F = a.fg + (size_t)e * 9;
    const double det = F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) +
                       F[2] * (F[3] * F[7] - F[4] * F[6]);
    const double per_node = det * a.v0[e] / 6.0;
    const int32_t* c = a.elems[e].conn;
#pragma unroll
    for (int k = 0; k < 6; ++k) atomicAdd(a.mass + c[k], per_node);
}

__global__ void __launch_bounds__(kPkThreads) k_pk_bbox(PackArgs a) {
    __shared__ double red[4][kPkThreads / 32];
    double lo0 = 1e300, lo1 = 1e300, hi0 = -1e300, hi1 = -1e300;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < a.n_nodes; n += gridDim.x * blockDim.x) {
        const double x0 = a.x[(size_t)n * 3], x1 = a.x[(size_t)n * 3 + 1];
        lo0 = fmin(lo0, x0);
        lo1 = fmin(lo1, x1);
        if (n > 0) {  // the reference's first node only ever lowers the minimum
            hi0 = fmax(hi0, x0);
            hi1 = fmax(hi1, x1);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        lo0 = fmin(lo0, __shfl_xor_sync(0xffffffffu, lo0, off));
        lo1 = fmin(lo1, __shfl_xor_sync(0xffffffffu, lo1, off));
        hi0 = fmax(hi0, __shfl_xor_sync(0xffffffffu, hi0, off));
        hi1 = fmax(hi1, __shfl_xor_sync(0xffffffffu, hi1, off));
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[0][w] = lo0;
        red[1][w] = lo1;
        red[2][w] = hi0;
        red[3][w] = hi1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < kPkThreads / 32; ++k) {
            red[0][0] = fmin(red[0][0], red[0][k]);
            red[1][0] = fmin(red[1][0], red[1][k]);
            red[2][0] = fmax(red[2][0], red[2][k]);
            red[3][0] = fmax(red[3][0], red[3][k]);
        }
        atomic_min_d(&a.prm->bb0[0], red[0][0]);
        atomic_min_d(&a.prm->bb0[1], red[1][0]);
        atomic_max_d(&a.prm->bbs[0], red[2][0]);
        atomic_max_d(&a.prm->bbs[1], red[3][0]);
    }
}

__global__ void k_pk_bbox_final(PackParams* prm) {
    if (threadIdx.x == 0) {
        prm->bbs[0] -= prm->bb0[0];
        prm->bbs[1] -= prm->bb0[1];
    }
}

// average length of the nonzero sides of the triangle of element nodes o, o+1, o+2 (Prism.cpp:1329-1395)
__device__ double side_average(const PackArgs& a, const int32_t* c, int o) {
    const int pr[3][2] = {{o, o + 1}, {o, o + 2}, {o + 1, o + 2}};
    double sum = 0.0;
    int cnt = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        double d2 = 0.0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double dd = a.x[(size_t)c[pr[i][0]] * 3 + k] - a.x[(size_t)c[pr[i][1]] * 3 + k];
            d2 += dd * dd;
        }
        if (d2 > 0) {
            sum += sqrt(d2);
            cnt++;
        }
    }
    return cnt > 0 ? sum / cnt : 0.0;
}

// the side-length grid (Simulation::getAverageSideLength): per-CTA sums in shared memory, then
// one atomic per cell and CTA
__global__ void __launch_bounds__(kPkThreads) k_pk_grid(PackArgs a) {
    __shared__ double gs[50], gc[50], cs[2];
    for (int k = threadIdx.x; k < 50; k += blockDim.x) gs[k] = gc[k] = 0.0;
    if (threadIdx.x < 2) cs[threadIdx.x] = 0.0;
    __syncthreads();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < a.n_elems && !(a.peripodial && a.peripodial[e])) {
        const int32_t* c = a.elems[e].conn;
        double cur = side_average(a, c, 3);
        if (cur > 0) {
            atomicAdd(&cs[0], cur);
            atomicAdd(&cs[1], 1.0);
        }
        if (a.exposed[e] & 2) {  // basal or whole-tissue element: its basal face as well
            cur = side_average(a, c, 0);
            if (cur > 0) {
                atomicAdd(&cs[0], cur);
                atomicAdd(&cs[1], 1.0);
            }
        }
        double cx = 0.0, cy = 0.0;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            cx += a.x[(size_t)c[k] * 3];
            cy += a.x[(size_t)c[k] * 3 + 1];
        }
        cx /= 6.0;
        cy /= 6.0;
        const PackParams* p = a.prm;
        int rx = (int)floor((cx - p->bb0[0]) / p->bbs[0]);
        int ry = (int)floor(((cy - p->bb0[1]) / p->bbs[1]) / 2.0);
        rx = min(9, max(0, rx));
        ry = min(4, max(0, ry));
        atomicAdd(&gs[rx * 5 + ry], cur);
        atomicAdd(&gc[rx * 5 + ry], 1.0);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < 50; k += blockDim.x)
        if (gc[k] != 0.0) {
            atomicAdd(&a.prm->grid_sum[k], gs[k]);
            atomicAdd(&a.prm->grid_cnt[k], gc[k]);
        }
    if (threadIdx.x < 2 && cs[threadIdx.x] != 0.0) atomicAdd(threadIdx.x == 0 ? &a.prm->col_sum : &a.prm->col_cnt, cs[threadIdx.x]);
}

// squared detection distances into grid_sum, the packing threshold and the search cell
__global__ void k_pk_grid_final(PackParams* prm) {
    __shared__ double mx[64];
    const int k = threadIdx.x;
    double t = 0.0;
    if (k < 50) {
        const double avg = prm->grid_cnt[k] > 0 ? prm->grid_sum[k] / prm->grid_cnt[k] : prm->grid_sum[k];
        t = 0.4 * avg;
        prm->grid_sum[k] = t * t;
    }
    mx[k] = t;
    __syncthreads();
    if (k == 0) {
        double m = 0.0;
        for (int q = 0; q < 50; ++q) m = fmax(m, mx[q]);
        prm->cell = m;
        prm->threshold = 0.4 * (prm->col_cnt > 0 ? prm->col_sum / prm->col_cnt : 0.0);
    }
}

__device__ __forceinline__ bool eligible(const PackArgs& a, int n) {
    const int pl = a.placement[n];
    return (pl == 0 || pl == 1) && a.mass[n] != 0.0;
}

__device__ __forceinline__ void cell_of(const PackArgs& a, int n, long long c[3]) {
    const double h = a.prm->cell;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double v = floor(a.x[(size_t)n * 3 + d] / h);  // clamped: no overflow in the cell loops
        c[d] = (long long)fmin(fmax(v, -1e15), 1e15);
    }
}

__device__ __forceinline__ unsigned cell_hash(long long cx, long long cy, long long cz, int bits) {
    const unsigned long long h = ((unsigned long long)cx * 73856093ull) ^ ((unsigned long long)cy * 19349663ull) ^
                                 ((unsigned long long)cz * 83492791ull);
    return (unsigned)(h ^ (h >> 29)) & ((1u << bits) - 1u);
}

__global__ void __launch_bounds__(kPkThreads) k_pk_hash_count(PackArgs a) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.n_nodes || !(a.prm->cell > 0.0) || !eligible(a, n)) return;
    long long c[3];
    cell_of(a, n, c);
    atomicAdd(a.bucket_cnt + cell_hash(c[0], c[1], c[2], a.hash_bits), 1);
}

__global__ void __launch_bounds__(kPkThreads) k_pk_hash_fill(PackArgs a) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.n_nodes || !(a.prm->cell > 0.0) || !eligible(a, n)) return;
    long long c[3];
    cell_of(a, n, c);
    const unsigned h = cell_hash(c[0], c[1], c[2], a.hash_bits);
    a.bucket_nodes[a.bucket_start[h] + atomicAdd(a.bucket_cnt + h, 1)] = n;
}

__device__ bool shares_element(const PackArgs& a, int i, int j) {
    int lo = a.rowptr[i], hi = a.rowptr[i + 1] - 1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        const int c = a.colidx[mid];
        if (c == j) return true;
        if (c < j)
            lo = mid + 1;
        else
            hi = mid - 1;
    }
    return false;
}

// EMIT = false: node_cnt[i] = pairs (i, j > i); EMIT = true: the pairs at node_start[i], sorted by j
template <bool EMIT>
__global__ void __launch_bounds__(kPkThreads) k_pk_pairs(PackArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_nodes) return;
    int count = 0;
    const PackParams* p = a.prm;
    if (p->cell > 0.0 && eligible(a, i)) {
        const double xi = a.x[(size_t)i * 3], yi = a.x[(size_t)i * 3 + 1], zi = a.x[(size_t)i * 3 + 2];
        const int gx = (int)floor((xi - p->bb0[0]) / p->bbs[0]);
        const int gy = (int)floor((yi - p->bb0[1]) / p->bbs[1]);
        const double t2 = (gx >= 0 && gx <= 9 && gy >= 0 && gy <= 4) ? p->grid_sum[gx * 5 + gy] : 0.0;
        if (t2 > 0.0) {
            long long c[3];
            cell_of(a, i, c);
            const int base = EMIT ? a.node_start[i] : 0;
            for (long long ax = c[0] - 1; ax <= c[0] + 1; ++ax)
                for (long long ay = c[1] - 1; ay <= c[1] + 1; ++ay)
                    for (long long az = c[2] - 1; az <= c[2] + 1; ++az) {
                        const unsigned h = cell_hash(ax, ay, az, a.hash_bits);
                        for (int k = a.bucket_start[h]; k < a.bucket_start[h + 1]; ++k) {
                            const int j = a.bucket_nodes[k];
                            if (j <= i || a.placement[j] != a.placement[i]) continue;
                            long long cj[3];
                            cell_of(a, j, cj);
                            if (cj[0] != ax || cj[1] != ay || cj[2] != az) continue;  // another cell in the bucket
                            const double dx = xi - a.x[(size_t)j * 3], dy = yi - a.x[(size_t)j * 3 + 1],
                                         dz = zi - a.x[(size_t)j * 3 + 2];
                            if (!(dx * dx + dy * dy + dz * dz < t2) || shares_element(a, i, j)) continue;
                            if (EMIT) {
                                const int q = base + count;
                                if (q < a.capacity) {
                                    // insertion by j: the node's partners end up ascending
                                    int r = q;
                                    while (r > base && a.pairs[2 * (r - 1) + 1] > j) {
                                        a.pairs[2 * r] = i;
                                        a.pairs[2 * r + 1] = a.pairs[2 * (r - 1) + 1];
                                        --r;
                                    }
                                    a.pairs[2 * r] = i;
                                    a.pairs[2 * r + 1] = j;
                                }
                            }
                            ++count;
                        }
                    }
        }
    }
    if (!EMIT) a.node_cnt[i] = count;
}

// --- exclusive scan of int32 counts -------------------------------------------------------------
__global__ void __launch_bounds__(kScanBlock) k_scan_block(const int32_t* in, int32_t* out, int n, int32_t* sums) {
    __shared__ int32_t warp_tot[kScanBlock / 32];
    const int i = blockIdx.x * kScanBlock + threadIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int32_t v = i < n ? in[i] : 0;
    int32_t inc = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int32_t u = __shfl_up_sync(0xffffffffu, inc, off);
        if (lane >= off) inc += u;
    }
    if (lane == 31) warp_tot[w] = inc;
    __syncthreads();
    if (w == 0) {
        int32_t t = warp_tot[lane];
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int32_t u = __shfl_up_sync(0xffffffffu, t, off);
            if (lane >= off) t += u;
        }
        warp_tot[lane] = t;  // inclusive over warps
    }
    __syncthreads();
    const int32_t before = w > 0 ? warp_tot[w - 1] : 0;
    if (i < n) out[i] = before + inc - v;
    if (threadIdx.x == kScanBlock - 1) sums[blockIdx.x] = warp_tot[31];
}

// exclusive scan of the nb block sums by one CTA (each thread a contiguous chunk), total at sums[nb]
__global__ void __launch_bounds__(kScanBlock) k_scan_sums(int32_t* sums, int nb) {
    __shared__ int32_t part[kScanBlock];
    const int per = (nb + kScanBlock - 1) / kScanBlock;
    const int b0 = threadIdx.x * per, b1 = min(nb, b0 + per);
    int32_t t = 0;
    for (int b = b0; b < b1; ++b) t += sums[b];
    part[threadIdx.x] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        int32_t run = 0;
        for (int k = 0; k < kScanBlock; ++k) {
            const int32_t v = part[k];
            part[k] = run;
            run += v;
        }
        sums[nb] = run;
    }
    __syncthreads();
    int32_t run = part[threadIdx.x];
    for (int b = b0; b < b1; ++b) {
        const int32_t v = sums[b];
        sums[b] = run;
        run += v;
    }
}

__global__ void k_scan_add(int32_t* out, int n, const int32_t* sums, int nb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += sums[i / kScanBlock];
    if (i == 0) out[n] = sums[nb];
}

// --- per Newton iteration -----------------------------------------------------------------------
__global__ void __launch_bounds__(kPkThreads) k_pk_terms(PackTerms a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n_pairs) return;
    const int i = a.pairs[2 * p], j = a.pairs[2 * p + 1];
    const double thr = a.prm->threshold;
    const double dx = a.x[(size_t)i * 3] - a.x[(size_t)j * 3], dy = a.x[(size_t)i * 3 + 1] - a.x[(size_t)j * 3 + 1],
                 dz = a.x[(size_t)i * 3 + 2] - a.x[(size_t)j * 3 + 2];
    double d = sqrt(dx * dx + dy * dy + dz * dz);
    const double m = 0.5 * (a.mass[i] + a.mass[j]);
    double e[3] = {1.0, 0.0, 0.0};
    if (d > 1e-3) {
        e[0] = dx / d;
        e[1] = dy / d;
        e[2] = dz / d;
    } else {
        d = 1e-3;
    }
    const double S = 1.0 / (1.0 + exp(5.0 / thr * 2.0 * (d - 0.6 * thr)));
    const double fmag = 5000.0 * m * S;
    const double dS = (-5.0 / thr * 2.0) * S * (1.0 - S);
    const int fi = a.fixmask[i], fj = a.fixmask[j];
    double D[9];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        if (!((fi >> r) & 1)) atomicAdd(a.g + (size_t)i * 3 + r, fmag * e[r]);
        if (!((fj >> r) & 1)) atomicAdd(a.g + (size_t)j * 3 + r, -fmag * e[r]);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double ee = e[r] * e[c];
            D[r * 3 + c] = (((r == c) ? 1.0 : 0.0) - ee) * (S / d) + ee * dS;
            D[r * 3 + c] *= 5000.0 * m;
        }
    }
    double* Bii = a.vals + (size_t)a.diag[i] * 9;
    double* Bjj = a.vals + (size_t)a.diag[j] * 9;
    double* Pij = a.pk_vals + (size_t)(2 * p) * 9;
    double* Pji = Pij + 9;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double v = D[r * 3 + c];
            const bool ri = !((fi >> r) & 1), ci = !((fi >> c) & 1), rj = !((fj >> r) & 1), cj = !((fj >> c) & 1);
            if (ri && ci) atomicAdd(Bii + r * 3 + c, -v);
            if (rj && cj) atomicAdd(Bjj + r * 3 + c, -v);
            Pij[r * 3 + c] = (ri && cj) ? v : 0.0;
            Pji[r * 3 + c] = (rj && ci) ? v : 0.0;
            a.dfdx[(size_t)p * 9 + r * 3 + c] = v;
        }
}

}  // namespace

int scan_tmp_ints(int n) { return (n + kScanBlock - 1) / kScanBlock + 1; }

cudaError_t launch_scan_i32(const int32_t* in, int32_t* out, int n, int32_t* tmp, cudaStream_t s) {
    const int nb = (n + kScanBlock - 1) / kScanBlock;
    if (nb > 0) {
        k_scan_block<<<nb, kScanBlock, 0, s>>>(in, out, n, tmp);
        k_scan_sums<<<1, kScanBlock, 0, s>>>(tmp, nb);
    } else {
        cudaError_t e = cudaMemsetAsync(tmp, 0, sizeof(int32_t), s);
        if (e != cudaSuccess) return e;
    }
    k_scan_add<<<(n + 255) / 256 + 1, 256, 0, s>>>(out, n, tmp, nb);
    return cudaGetLastError();
}

cudaError_t launch_packing_detect(const PackArgs& a, cudaStream_t s) {
    cudaError_t e;
    const int H = 1 << a.hash_bits;
    if ((e = cudaMemsetAsync(a.mass, 0, sizeof(double) * (size_t)a.n_nodes, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(a.bucket_cnt, 0, sizeof(int32_t) * ((size_t)H + 1), s)) != cudaSuccess) return e;
    k_pk_init<<<1, 64, 0, s>>>(a.prm);
    const int eb = (a.n_elems + kPkThreads - 1) / kPkThreads, nb = (a.n_nodes + kPkThreads - 1) / kPkThreads;
    k_pk_mass<<<eb, kPkThreads, 0, s>>>(a);
    k_pk_bbox<<<min(nb, 148 * 4), kPkThreads, 0, s>>>(a);
    k_pk_bbox_final<<<1, 32, 0, s>>>(a.prm);
    k_pk_grid<<<eb, kPkThreads, 0, s>>>(a);
    k_pk_grid_final<<<1, 64, 0, s>>>(a.prm);
    k_pk_hash_count<<<nb, kPkThreads, 0, s>>>(a);
    if ((e = launch_scan_i32(a.bucket_cnt, a.bucket_start, H, a.scan_tmp, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(a.bucket_cnt, 0, sizeof(int32_t) * (size_t)H, s)) != cudaSuccess) return e;
    k_pk_hash_fill<<<nb, kPkThreads, 0, s>>>(a);
    k_pk_pairs<false><<<nb, kPkThreads, 0, s>>>(a);
    if ((e = launch_scan_i32(a.node_cnt, a.node_start, a.n_nodes, a.scan_tmp, s)) != cudaSuccess) return e;
    return cudaGetLastError();
}

cudaError_t launch_packing_pairs(const PackArgs& a, cudaStream_t s) {
    k_pk_pairs<true><<<(a.n_nodes + kPkThreads - 1) / kPkThreads, kPkThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_packing_terms(const PackTerms& a, cudaStream_t s) {
    if (a.n_pairs > 0) k_pk_terms<<<(a.n_pairs + kPkThreads - 1) / kPkThreads, kPkThreads, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace tfb
