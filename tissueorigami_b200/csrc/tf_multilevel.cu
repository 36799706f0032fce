// tf_multilevel.cu -- set-up of the multilevel coarse space of a single tissue, from the current J.
//
// The preconditioner is an additive multilevel Schwarz method over nested spatial sets: the
// tissue's prism columns are split into leaves by recursive coordinate bisection, and a set of
// level l is 4^(l-1) consecutive leaves (a subtree of the bisection), up to a top level small
// enough to invert densely. Each set contributes the six rigid modes about its centroid (three
// translations, three rotations, fixed DoFs zeroed). With B_i = [I | R_i], R_i w = w x d_i
// (d_i = node position - centroid) and T the transport of a rigid motion (u, w) about a parent
// centroid to a child centroid at offset D (u' = u + w x D, w' = w), every set's modes are its
// leaves' modes composed with T, so every coarse block follows from the leaf-pair blocks
//
//     C_ab = sum_{i in a, j in b} P_i^T J_ij P_j    (P_i = mask_i o B_i, 6 x 6)
//
// as  A_ST = sum_{a in S, b in T} T_a^T C_ab T_b.  The set-up kernels below compute C for every
// pair of leaves that J couples (one warp per pair), then each output block (the diagonal block
// of every set below the top, and every block of the top operator) as a fixed-order sum over its
// pairs, and finally the pseudo-inverse of every diagonal block by cyclic Jacobi rotations. The
// top operator is inverted by the Gauss-Jordan kernels of tf_dense.cu.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "tf_internal.cuh"

namespace tfb {
namespace {

constexpr int kMlThreads = 256;

// R such that R w = w x d (the rotation columns of a node's rigid modes about the origin of d).
__device__ __forceinline__ void cross_matrix(const double d[3], double R[9]) {
    R[0] = 0.0;
    R[1] = d[2];
    R[2] = -d[1];
    R[3] = -d[2];
    R[4] = 0.0;
    R[5] = d[0];
    R[6] = d[1];
    R[7] = -d[0];
    R[8] = 0.0;
}

// Sum of 36 values over the warp, every lane ending with the totals; entry e is written by
// lane e % 32 (fixed reduction order: deterministic).
__device__ __forceinline__ void warp_sum36(double c[36]) {
#pragma unroll
    for (int e = 0; e < 36; ++e)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) c[e] += __shfl_xor_sync(0xffffffffu, c[e], off);
}

__device__ __forceinline__ void store36(const double c[36], double* dst, int lane) {
#pragma unroll
    for (int e = 0; e < 36; ++e)
        if ((e & 31) == lane) dst[e] = c[e];
}

// C_s for leaf pair s: one warp, the lanes over the pair's Jacobian blocks.
__global__ void __launch_bounds__(kMlThreads) k_ml_pairs(KrylovWork w, MlSetup m) {
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (s >= m.n_slots) return;
    double c[36];
#pragma unroll
    for (int e = 0; e < 36; ++e) c[e] = 0.0;
    for (int q = m.slot_ptr[s] + lane; q < m.slot_ptr[s + 1]; q += 32) {
        const int k = m.blk[q], i = m.blk_row[q], j = __ldg(w.colidx + k);
        const double* B = w.vals + (size_t)k * 9;
        const int mi = m.node_mask[i], mj = m.node_mask[j];
        double Jm[9];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) Jm[r * 3 + cc] = ((mi >> r) & 1) && ((mj >> cc) & 1) ? __ldg(B + r * 3 + cc) : 0.0;
        double di[3], dj[3], Ri[9], Rj[9];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            di[d] = m.node_d[(size_t)i * 3 + d];
            dj[d] = m.node_d[(size_t)j * 3 + d];
        }
        cross_matrix(di, Ri);
        cross_matrix(dj, Rj);
        double JR[9];  // Jm R_j
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int cc = 0; cc < 3; ++cc)
                JR[r * 3 + cc] = Jm[r * 3] * Rj[cc] + Jm[r * 3 + 1] * Rj[3 + cc] + Jm[r * 3 + 2] * Rj[6 + cc];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                c[r * 6 + cc] += Jm[r * 3 + cc];
                c[r * 6 + 3 + cc] += JR[r * 3 + cc];
                // R_i^T Jm and R_i^T JR: (R_i^T X)[r][cc] = sum_k R_i[k][r] X[k][cc]
                c[(3 + r) * 6 + cc] += Ri[r] * Jm[cc] + Ri[3 + r] * Jm[3 + cc] + Ri[6 + r] * Jm[6 + cc];
                c[(3 + r) * 6 + 3 + cc] += Ri[r] * JR[cc] + Ri[3 + r] * JR[3 + cc] + Ri[6 + r] * JR[6 + cc];
            }
    }
    warp_sum36(c);
    store36(c, m.pairs + (size_t)s * 36, lane);
}

// Output block o = sum over its pairs of T_a^T C_s T_b: one warp, the lanes over the pairs.
__global__ void __launch_bounds__(kMlThreads) k_ml_blocks(MlSetup m) {
    const int o = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (o >= m.n_out) return;
    const double* cS = m.set_cen + (size_t)m.out_set[o] * 3;
    const double* cT = m.set_cen + (size_t)m.out_col[o] * 3;
    double acc[36];
#pragma unroll
    for (int e = 0; e < 36; ++e) acc[e] = 0.0;
    for (int q = m.out_ptr[o] + lane; q < m.out_ptr[o + 1]; q += 32) {
        const int s = m.out_slots[q], a = m.slot_a[s], b = m.slot_agg[s];
        double Da[3], Db[3], Xa[9], Xb[9];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            Da[d] = m.leaf_cen[(size_t)a * 3 + d] - cS[d];
            Db[d] = m.leaf_cen[(size_t)b * 3 + d] - cT[d];
        }
        cross_matrix(Da, Xa);  // T_a = [[I, Xa], [0, I]]
        cross_matrix(Db, Xb);
        const double* C = m.pairs + (size_t)s * 36;
        double ct[36];  // C T_b: columns 3..5 gain C[:, 0..2] Xb
#pragma unroll
        for (int r = 0; r < 6; ++r)
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                const double c0 = C[r * 6], c1 = C[r * 6 + 1], c2 = C[r * 6 + 2];
                ct[r * 6 + cc] = C[r * 6 + cc];
                ct[r * 6 + 3 + cc] = C[r * 6 + 3 + cc] + c0 * Xb[cc] + c1 * Xb[3 + cc] + c2 * Xb[6 + cc];
            }
        // T_a^T (C T_b): rows 3..5 gain Xa^T rows 0..2
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int cc = 0; cc < 6; ++cc) {
                acc[r * 6 + cc] += ct[r * 6 + cc];
                acc[(3 + r) * 6 + cc] +=
                    ct[(3 + r) * 6 + cc] + Xa[r] * ct[cc] + Xa[3 + r] * ct[6 + cc] + Xa[6 + r] * ct[12 + cc];
            }
    }
    warp_sum36(acc);
    if (o < m.n_diag) {
        store36(acc, m.w_blocks + (size_t)m.out_dst[o] * 36, lane);
    } else {
        const int S = m.out_dst[o] / m.n_top, T = m.out_dst[o] % m.n_top;
        const size_t ld = (size_t)6 * m.n_top;
#pragma unroll
        for (int e = 0; e < 36; ++e)
            if ((e & 31) == lane) m.top[(size_t)(6 * S + e / 6) * ld + 6 * T + e % 6] = acc[e];
    }
}

// In place: the symmetric pseudo-inverse of each 6 x 6 diagonal block (eigenvalues at or below
// 1e-12 of the largest, negative ones included, are dropped: W stays positive semi-definite).
__global__ void k_ml_pinv6(double* blocks, int n, int32_t* dflags) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double* blk = blocks + (size_t)t * 36;
    double A[36], V[36];
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c) {
            A[r * 6 + c] = 0.5 * (blk[r * 6 + c] + blk[c * 6 + r]);
            V[r * 6 + c] = r == c ? 1.0 : 0.0;
        }
    double scale = 0.0;
    for (int e = 0; e < 36; ++e) scale += A[e] * A[e];
    if (!isfinite(scale)) {
        atomicOr(dflags, DF_NONFINITE);
        for (int e = 0; e < 36; ++e) blk[e] = 0.0;
        return;
    }
    for (int sweep = 0; sweep < 20; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < 6; ++p)
            for (int q = p + 1; q < 6; ++q) off += A[p * 6 + q] * A[p * 6 + q];
        if (off <= 1e-32 * scale) break;
        for (int p = 0; p < 5; ++p)
            for (int q = p + 1; q < 6; ++q) {
                const double apq = A[p * 6 + q];
                if (apq == 0.0) continue;
                const double tau = (A[q * 6 + q] - A[p * 6 + p]) / (2.0 * apq);
                const double tt = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                const double c = 1.0 / sqrt(1.0 + tt * tt), s = tt * c;
                for (int k = 0; k < 6; ++k) {  // columns p, q
                    const double akp = A[k * 6 + p], akq = A[k * 6 + q];
                    A[k * 6 + p] = c * akp - s * akq;
                    A[k * 6 + q] = s * akp + c * akq;
                }
                for (int k = 0; k < 6; ++k) {  // rows p, q
                    const double apk = A[p * 6 + k], aqk = A[q * 6 + k];
                    A[p * 6 + k] = c * apk - s * aqk;
                    A[q * 6 + k] = s * apk + c * aqk;
                }
                A[p * 6 + q] = A[q * 6 + p] = 0.0;
                for (int k = 0; k < 6; ++k) {
                    const double vkp = V[k * 6 + p], vkq = V[k * 6 + q];
                    V[k * 6 + p] = c * vkp - s * vkq;
                    V[k * 6 + q] = s * vkp + c * vkq;
                }
            }
    }
    double lmax = 0.0;
    for (int k = 0; k < 6; ++k) lmax = fmax(lmax, A[k * 6 + k]);
    double inv[6];
    for (int k = 0; k < 6; ++k) inv[k] = (lmax > 0.0 && A[k * 6 + k] > 1e-12 * lmax) ? 1.0 / A[k * 6 + k] : 0.0;
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c) {
            double sum = 0.0;
            for (int k = 0; k < 6; ++k) sum += V[r * 6 + k] * V[c * 6 + k] * inv[k];
            blk[r * 6 + c] = sum;
        }
}

// Unit diagonal for every top mode without support (an exactly zero diagonal entry: all its
// DoFs fixed); its restricted residual is zero, so the unit only keeps the matrix invertible.
__global__ void k_ml_top_fix(double* top, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && top[(size_t)i * n + i] == 0.0) top[(size_t)i * n + i] = 1.0;
}

}  // namespace

cudaError_t launch_ml_setup(const KrylovWork& w, const MlSetup& m, bool top, cudaStream_t s) {
    const int n6 = 6 * m.n_top;
    if (top) {
        cudaError_t e = cudaMemsetAsync(m.top, 0, sizeof(double) * (size_t)n6 * n6, s);
        if (e != cudaSuccess) return e;
    }
    const int wpb = kMlThreads / 32;
    if (m.n_slots > 0) k_ml_pairs<<<(m.n_slots + wpb - 1) / wpb, kMlThreads, 0, s>>>(w, m);
    if (m.n_out > 0) k_ml_blocks<<<(m.n_out + wpb - 1) / wpb, kMlThreads, 0, s>>>(m);
    if (m.n_diag > 0) k_ml_pinv6<<<(m.n_diag + 127) / 128, 128, 0, s>>>(m.w_blocks, m.n_diag, m.dflags);
    if (top && n6 > 0) k_ml_top_fix<<<(n6 + 255) / 256, 256, 0, s>>>(m.top, n6);
    return cudaGetLastError();
}

}  // namespace tfb
