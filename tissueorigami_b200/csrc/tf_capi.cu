// tf_capi.cu -- host runtime and C ABI of the B200 Newton step (see include/tf_b200.h).
//
// The host side owns what the reference keeps in NewtonRaphsonSolver and the element objects:
// it builds, once per mesh, the BSR3 pattern of the Jacobian, the element-to-block slot map,
// a greedy element colouring and the slave-master routing, packs each prism into a 416-byte
// record, and drives the Newton loop of Simulation::updateStepNR
// (TissueFolding/SourceCode/Simulation.cpp:6605-6747) with one host synchronisation per
// Newton iteration. The linear solve runs as graph-replayed chunks of BiCGStab iterations
// whose scalars never leave the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <thread>
#include <vector>

#include "../../include/tf_b200.h"
#include "tf_internal.cuh"

using namespace tfb;

namespace {

constexpr int kChunk = 32;  // BiCGStab iterations per graph replay / status poll
constexpr int kCoarseMaxAge = 64;  // solves between refreshes of the two-level coarse operator
constexpr int kMaxAggNodes = 2048;  // largest useful two-level aggregate (nodes)
constexpr int kBatchAggNodes = 256;  // aggregate size of a batch tissue's two-level space
constexpr int kMlLeafCols = 16;      // prism columns per leaf of the multilevel space
constexpr int kMlTopMax = 160;       // sets of the multilevel space's densely inverted top level
constexpr int kMlAutoNodes = 100000; // single tissues from this size take the multilevel space
constexpr int kMlTopMaxAge = 8;      // solves between refreshes of the multilevel top inverse
constexpr int kWarmSlots = 8;        // Newton iterations whose solutions are kept for warm starts

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

template <class T>
T* dptr(DevBuf& b) {
    return static_cast<T*>(b.p);
}

}  // namespace

struct tf_ctx {
    tf_params params{};
    // Warm starts of the Newton loop's solves (single tissue, conjugate gradients): the solution
    // of Newton iteration k of the last step that reached it, and the iteration the current
    // solve belongs to (-1 outside the Newton loop).
    std::vector<DevBuf> warm_hist;
    std::vector<char> warm_valid;
    int warm_k = -1;
    bool warm_call = false;  // the current call is a time step of the public API (not the adjoint's)
    int device = 0;
    cudaStream_t stream = nullptr;
    int32_t N = 0, E = 0;
    int64_t nnzb = 0;

    // host mirrors
    std::vector<int32_t> conn;  // [E*6]
    std::vector<double> xref;   // [E*18]
    std::vector<int32_t> dofmap;
    std::vector<int32_t> slave, master;
    std::vector<int32_t> rowptr, colidx, diag;
    std::vector<int32_t> colour_offsets;  // colour c: elements colour_list[off[c]..off[c+1])
    std::vector<int32_t> colour_list;     // colour-sorted element ids, routed ones at the end
    int32_t n_routed = 0;
    int smooth_G = 1;  // smoother block: G consecutive nodes (single tissue, persistent solve)
    int n_colours = 0;
    bool has_visc = false;

    // device buffers
    DevBuf elems, fixmask, ext_visc, visc_surface, dofmap_d, slaves_d, masters_d;
    DevBuf rowptr_d, colidx_d, diag_d, vals, colour_list_d;
    DevBuf uk, un, g, du, r, rhat, p, v, s, t, phat, shat, dinv, partials, sc, dflags;
    DevBuf fg, rates, angles, exposed, peripodial, rotated, xio, barrier;
    DevBuf refine_acc, refine_g;  // tf_solve's iterative refinement: accumulated du, saved g
    DevBuf ext_force;             // gExt [3N] (tf_set_external_force); used when has_ext_force
    bool has_ext_force = false;

    // grid-based growth functions (tf_set_grid_growth) and the simulation clock that selects the
    // ones active in a step (currSimTimeSec of the reference)
    struct GridFuncHost {
        double t0, t1, zmin, zmax;
        int32_t nx, ny, flags;
        DevBuf cells;
    };
    std::vector<GridFuncHost> grid_funcs;
    int32_t grid_interp = 0;
    DevBuf grid_rel_pos, grid_rel_z, grid_eflags, grid_inc;
    double sim_time = 0.0;
    int persistent_grid_max = 0;  // 0: cooperative launch unavailable
    int persist_threads = 256;    // CTA width of the persistent solve

    // batch partition: tissue t owns nodes [tissue_node0[t], tissue_node0[t+1]) and elements
    // [tissue_elem0[t], tissue_elem0[t+1]); a single tissue is T = 1.
    int32_t T = 1;
    std::vector<int32_t> tissue_node0, tissue_elem0;
    std::vector<int32_t> plan_list_ptr, plan_list, plan_cta0, plan_ncta;
    DevBuf plan_queue_d, queue_head_d;
    std::vector<int32_t> plan_queue;
    DevBuf node_tissue_d, plan_list_ptr_d, plan_list_d, plan_cta0_d, plan_ncta_d, plan_row0_d, active_d, tbarriers, tscalars,
        tdu2;
    int32_t* h_active = nullptr;     // pinned [T]
    double* h_du2 = nullptr;         // pinned [T]
    KrylovScalars* h_tsc = nullptr;  // pinned [T]
    std::vector<int32_t> t_iters, t_status, t_krylov;
    std::vector<int32_t> last_krylov;  // first-round BiCGStab iterations of each tissue, last step

    // two-level preconditioner (precond == TF_PRECOND_TWO_LEVEL, persistent solve; the fields
    // below serve a single tissue, the bc_* ones further down a batch)
    std::vector<uint8_t> h_fixmask;
    bool coarse_dirty = true;
    int coarse_m = 0, n_coarse = 0, n_agg = 0, n_coarse_empty = 0;
    bool coarse_ok = false;  // the last coarse factorisation succeeded
    DevBuf pmode_d, coarse_inv, coarse_r, coarse_info, coarse_work;
    DevBuf node_d, node_mask, agg_m;
    int coarse_age = 0, coarse_base_iters = 0;  // solves since the last coarse refresh; iterations of the first
    int last_solve_iters = 0;
    int32_t coarse_refreshes = 0;
    DevBuf ca_agg_slot_ptr, ca_slot_agg, ca_slot_ptr, ca_blk, ca_blk_row, ca_empty;
    int32_t* h_coarse_info = nullptr;  // pinned
    // two-level preconditioner of a batch: fixed aggregates per tissue, padded per-tissue coarse
    // matrices (leading dimension bc_ld) inverted together by batched LU
    bool bc_active = false;
    int bc_ld = 0;
    int64_t bc_n_unit = 0;
    std::vector<int32_t> bc_tissue_agg0;
    DevBuf bc_tissue_agg0_d, bc_agg_ptr_d, bc_agg_nodes_d, bc_agg_tissue_d, bc_base_d, bc_unit_d, bc_order_d, bc_info_d;
    // lumen (tf_set_lumen): triangles, ideal volume, the rank-one term's vector and solve scratch
    bool lm_on = false, reuse_precond = false;
    int lm_n_tri = 0;
    double lm_bulk = 0.0, lm_v_init = 0.0, lm_rate = 0.0, lm_ideal = 0.0;
    DevBuf lm_tri_d, lm_state_d, lm_part_d, lm_G_d, lm_y_d, lm_z_d, lm_gsave_d, lm_dot_part_d, lm_dots_d;
    double* h_lm_dots = nullptr;  // pinned [2]
    // packing (tf_set_packing): detection per step, pairs and their blocks outside the pattern
    bool pk_on = false;
    int pk_hash_bits = 10, pk_capacity = 0, pk_pairs_n = 0;
    std::vector<int32_t> h_pk_pairs;
    DevBuf pk_place_d, pk_v0_d, pk_mass_d, pk_prm_d, pk_bucket_cnt_d, pk_bucket_start_d, pk_bucket_nodes_d,
        pk_node_cnt_d, pk_node_start_d, pk_scan_d, pk_pairs_d, pk_ptr_d, pk_col_d, pk_blk_d, pk_vals_d, pk_dfdx_d, pk_x_d;
    // multilevel coarse space of a single tissue (build_ml): leaves, levels, set-up lists
    bool ml_active = false;
    bool ml_top_ok = false, ml_top_fresh = false;  // the top inverse exists / was refreshed for this solve
    int ml_top_age = 0;                            // solves since the top inverse was refreshed
    int32_t last_solve_method = 0;                 // KM_* of the last persistent solve (largest over tissues)
    int col_G = 1;  // nodes per prism column when the mesh numbers columns consecutively, else 1
    int ml_levels = 0, ml_n_leaf = 0, ml_n_slots = 0, ml_n_out = 0, ml_n_diag = 0, ml_n_top = 0, ml_nct = 0;
    int32_t ml_span[kMlMaxLevels] = {0}, ml_count[kMlMaxLevels] = {0}, ml_set0[kMlMaxLevels] = {0};
    std::vector<int32_t> h_slot_agg, h_agg_slot_ptr;  // host copies of the last coarse_space_upload's slots
    DevBuf ml_leaf_ptr_d, ml_leaf_nodes_d, ml_cen_d, ml_w_d, ml_top_d, ml_top_work, ml_info_d, ml_leaf_m_d, ml_part_d,
        ml_pstart_d, ml_first_cta_d, ml_slot_a_d, ml_out_ptr_d, ml_out_slots_d, ml_out_set_d, ml_out_col_d, ml_out_dst_d,
        ml_pairs_d, ml_pos_leaf_d;

    // multicolour block ILU(0) (precond == TF_PRECOND_ILU0)
    std::vector<int32_t> ilu_colour_ptr;
    int32_t ilu_colours = 0;
    DevBuf ilu_cnodes, ilu_lo_ptr, ilu_lo_idx, ilu_up_ptr, ilu_up_idx, ilu_lu, ilu_uinv, ilu_y;
    cudaGraphExec_t ilu_graph = nullptr;

    // adjoint: forward checkpoints every adj_k steps, segment recompute buffers, adjoint state
    int32_t adj_steps = 0, adj_k = 0;
    double adj_dt = 0.0;
    std::vector<DevBuf> cp_x, cp_fg, seg_x, seg_fg;
    DevBuf abar, abar2, mubar, dLdr, qbuf;
    KrylovScalars* h_sc = nullptr;  // pinned
    int32_t* h_flags = nullptr;     // pinned

    int32_t last_method = 0;  // Krylov method of the current call's solves (KM_*; the largest seen)
    int64_t cg_iters = 0;     // conjugate-gradient iterations of the current call's solves
    int scatter = TF_SCATTER_ATOMIC;
    int teams = 32;
    bool tuned = false;

    cudaGraphExec_t krylov_graph = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t ev_call[2] = {nullptr, nullptr};  // brackets a whole public call
    cudaEvent_t ev_solve[2] = {nullptr, nullptr}; // brackets one persistent solve launch
    double solve_kernel_ms = 0.0;                 // accumulated over the current call
    int32_t solve_kernel_launches = 0;
    int64_t launches = 0;                         // kernels launched by the current call
    char last_error[256] = {0};
};

namespace {

// The message of the last failed tf_create / tf_batch_create on this thread (the context itself
// is gone by then); tf_last_error(NULL) returns it.
thread_local char g_create_error[256] = {0};

int set_error(tf_ctx* c, int code, const char* msg) {
    if (c) std::snprintf(c->last_error, sizeof(c->last_error), "%s", msg);
    return code;
}

int set_error(tf_ctx* c, int code, const char* msg, const char* where) {
    if (c) std::snprintf(c->last_error, sizeof(c->last_error), "%s (%s)", msg, where);
    return code;
}

#define TF_CK(call)                                                                   \
    do {                                                                              \
        cudaError_t err__ = (call);                                                   \
        if (err__ != cudaSuccess) {                                                   \
            cudaGetLastError();                                                       \
            return set_error(ctx, err__ == cudaErrorMemoryAllocation ? TF_ERR_OUT_OF_MEMORY : TF_ERR_CUDA, \
                             cudaGetErrorString(err__), #call);                       \
        }                                                                             \
    } while (0)

cudaError_t dalloc(DevBuf& b, size_t bytes) {
    if (b.p && b.bytes >= bytes) return cudaSuccess;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    if (bytes == 0) bytes = 16;
    cudaError_t err = cudaMalloc(&b.p, bytes);
    if (err == cudaSuccess) b.bytes = bytes;
    return err;
}

void dfree(DevBuf& b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
}

template <class F>
void parallel_for(int64_t n, F f) {
    unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (n < 200000) nt = 1;
    if (nt == 1) {
        f(0, n);
        return;
    }
    std::vector<std::thread> th;
    const int64_t chunk = (n + nt - 1) / nt;
    for (unsigned t = 0; t < nt; ++t) {
        const int64_t b = t * chunk, e = std::min<int64_t>(n, b + chunk);
        if (b < e) th.emplace_back([=] { f(b, e); });
    }
    for (auto& x : th) x.join();
}

// Block pattern under slave-master routing: block (r, c) exists when some element holds
// nodes A, B whose DoFs route to nodes r and c; every node keeps its diagonal block.
void build_pattern(tf_ctx* c) {
    const int N = c->N, E = c->E;
    std::vector<int32_t> ecount(N + 1, 0), eoff(N + 1, 0), elist((size_t)E * 6);
    for (int e = 0; e < E; ++e)
        for (int a = 0; a < 6; ++a) ecount[c->conn[(size_t)e * 6 + a]]++;
    for (int i = 0; i < N; ++i) eoff[i + 1] = eoff[i] + ecount[i];
    std::vector<int32_t> fill(eoff.begin(), eoff.end() - 1);
    for (int e = 0; e < E; ++e)
        for (int a = 0; a < 6; ++a) elist[fill[c->conn[(size_t)e * 6 + a]]++] = e;

    // routed rows of each node and, inversely, the source nodes of each routed row
    auto routes = [&](int A, int32_t out[3]) {
        int n = 0;
        for (int i = 0; i < 3; ++i) {
            const int r = c->dofmap[(size_t)A * 3 + i] / 3;
            bool dup = false;
            for (int k = 0; k < n; ++k) dup |= out[k] == r;
            if (!dup) out[n++] = r;
        }
        return n;
    };
    std::vector<std::vector<int32_t>> extra_src;  // only for rows that receive routed DoFs
    std::vector<int32_t> extra_idx(N, -1);
    if (!c->slave.empty()) {
        for (int A = 0; A < N; ++A) {
            int32_t rr[3];
            const int n = routes(A, rr);
            for (int k = 0; k < n; ++k)
                if (rr[k] != A) {
                    if (extra_idx[rr[k]] < 0) {
                        extra_idx[rr[k]] = (int32_t)extra_src.size();
                        extra_src.emplace_back();
                    }
                    extra_src[extra_idx[rr[k]]].push_back(A);
                }
        }
    }
    std::vector<std::vector<int32_t>> rows(N);
    parallel_for(N, [&](int64_t b0, int64_t b1) {
        std::vector<int32_t> mark(N, -1);
        std::vector<int32_t> tmp;
        for (int64_t r = b0; r < b1; ++r) {
            tmp.clear();
            auto add_src = [&](int A) {
                for (int k = eoff[A]; k < eoff[A + 1]; ++k) {
                    const int e = elist[k];
                    for (int bn = 0; bn < 6; ++bn) {
                        int32_t cc[3];
                        const int nc = c->slave.empty() ? (cc[0] = c->conn[(size_t)e * 6 + bn], 1)
                                                        : routes(c->conn[(size_t)e * 6 + bn], cc);
                        for (int q = 0; q < nc; ++q)
                            if (mark[cc[q]] != r) {
                                mark[cc[q]] = (int32_t)r;
                                tmp.push_back(cc[q]);
                            }
                    }
                }
            };
            if (mark[r] != r) {
                mark[r] = (int32_t)r;
                tmp.push_back((int32_t)r);
            }
            // node r itself contributes to row r unless all its DoFs are routed elsewhere
            bool self = true;
            if (!c->slave.empty()) {
                self = false;
                for (int i = 0; i < 3; ++i) self |= c->dofmap[r * 3 + i] / 3 == r;
            }
            if (self) add_src((int)r);
            if (!c->slave.empty() && extra_idx[r] >= 0)
                for (int A : extra_src[extra_idx[r]]) add_src(A);
            std::sort(tmp.begin(), tmp.end());
            rows[r] = tmp;
        }
    });
    c->rowptr.assign(N + 1, 0);
    for (int i = 0; i < N; ++i) c->rowptr[i + 1] = c->rowptr[i] + (int32_t)rows[i].size();
    c->nnzb = c->rowptr[N];
    c->colidx.resize(c->nnzb);
    c->diag.resize(N);
    for (int i = 0; i < N; ++i) {
        std::copy(rows[i].begin(), rows[i].end(), c->colidx.begin() + c->rowptr[i]);
        c->diag[i] = c->rowptr[i] + (int32_t)(std::lower_bound(rows[i].begin(), rows[i].end(), i) - rows[i].begin());
    }
}

// Greedy colouring over elements in mesh order: no two prisms of one colour share a node.
// Elements that touch a slave DoF are kept out of the colours and listed last.
void build_colouring(tf_ctx* c, const std::vector<int32_t>& routed) {
    const int E = c->E;
    std::vector<uint64_t> used(c->N, 0);
    std::vector<int8_t> col(E, -1);
    int ncol = 0;
    bool ok = true;
    for (int e = 0; e < E && ok; ++e) {
        if (routed[e]) continue;
        uint64_t forb = 0;
        for (int a = 0; a < 6; ++a) forb |= used[c->conn[(size_t)e * 6 + a]];
        if (~forb == 0) {
            ok = false;
            break;
        }
        const int k = __builtin_ctzll(~forb);
        col[e] = (int8_t)k;
        ncol = std::max(ncol, k + 1);
        for (int a = 0; a < 6; ++a) used[c->conn[(size_t)e * 6 + a]] |= (1ull << k);
    }
    c->colour_list.clear();
    c->colour_offsets.clear();
    c->n_routed = 0;
    if (!ok) {
        c->n_colours = 0;
        return;
    }
    std::vector<int32_t> cnt(ncol + 1, 0);
    for (int e = 0; e < E; ++e)
        if (col[e] >= 0) cnt[col[e] + 1]++;
    for (int k = 0; k < ncol; ++k) cnt[k + 1] += cnt[k];
    c->colour_offsets = cnt;
    c->colour_list.resize(E);
    std::vector<int32_t> pos(cnt.begin(), cnt.end() - 1);
    int32_t tail = cnt[ncol];
    for (int e = 0; e < E; ++e) {
        if (col[e] >= 0)
            c->colour_list[pos[col[e]]++] = e;
        else
            c->colour_list[tail++] = e;
    }
    c->n_routed = E - cnt[ncol];
    c->n_colours = ncol;
}

int build_ilu(tf_ctx* ctx);

int upload_structure(tf_ctx* ctx) {
    const int N = ctx->N, E = ctx->E;
    build_pattern(ctx);
    // element flags and slot map
    std::vector<int32_t> routed(E, 0);
    std::vector<uint8_t> node_bound(N, 0);
    for (int A = 0; A < N; ++A)
        for (int i = 0; i < 3; ++i)
            if (ctx->dofmap[(size_t)A * 3 + i] != A * 3 + i) node_bound[A] = 1;
    std::vector<ElemRecord> rec(E);
    // keep the previous material / growth values if the records already exist on the device
    const bool keep = ctx->elems.p != nullptr && ctx->elems.bytes >= sizeof(ElemRecord) * (size_t)E;
    if (keep) TF_CK(cudaMemcpy(rec.data(), ctx->elems.p, sizeof(ElemRecord) * (size_t)E, cudaMemcpyDeviceToHost));
    std::vector<int32_t> elem_tissue(E, 0);
    for (int t = 0; t < ctx->T; ++t)
        for (int e = ctx->tissue_elem0[t]; e < ctx->tissue_elem0[t + 1]; ++e) elem_tissue[e] = t;
    parallel_for(E, [&](int64_t b0, int64_t b1) {
        for (int64_t e = b0; e < b1; ++e) {
            ElemRecord& R = rec[e];
            if (!keep) {
                std::memset(&R, 0, sizeof(R));
                for (int k = 0; k < 9; ++k) R.inv_fg[k] = (k % 4 == 0) ? 1.0 : 0.0;
            }
            R.tissue = elem_tissue[e];
            const int32_t* cn = &ctx->conn[(size_t)e * 6];
            bool rt = false;
            for (int a = 0; a < 6; ++a) {
                R.conn[a] = cn[a];
                rt |= node_bound[cn[a]] != 0;
            }
            for (int k = 0; k < 18; ++k) R.xref[k] = ctx->xref[(size_t)e * 18 + k];
            routed[e] = rt;
            R.flags = rt ? 1 : 0;
            for (int a = 0; a < 6; ++a)
                for (int b = 0; b < 6; ++b) {
                    int32_t slot = -1;
                    if (!rt) {
                        const int32_t* r0 = ctx->colidx.data() + ctx->rowptr[cn[a]];
                        const int32_t* r1 = ctx->colidx.data() + ctx->rowptr[cn[a] + 1];
                        slot = (int32_t)(std::lower_bound(r0, r1, cn[b]) - ctx->colidx.data());
                    }
                    R.slots[a * 6 + b] = slot;
                }
        }
    });
    build_colouring(ctx, routed);
    TF_CK(dalloc(ctx->elems, sizeof(ElemRecord) * (size_t)E));
    TF_CK(cudaMemcpy(ctx->elems.p, rec.data(), sizeof(ElemRecord) * (size_t)E, cudaMemcpyHostToDevice));
    TF_CK(dalloc(ctx->rowptr_d, sizeof(int32_t) * (N + 1)));
    TF_CK(dalloc(ctx->colidx_d, sizeof(int32_t) * (size_t)ctx->nnzb));
    TF_CK(dalloc(ctx->diag_d, sizeof(int32_t) * N));
    TF_CK(dalloc(ctx->vals, sizeof(double) * 9 * (size_t)ctx->nnzb));
    TF_CK(cudaMemcpy(ctx->rowptr_d.p, ctx->rowptr.data(), sizeof(int32_t) * (N + 1), cudaMemcpyHostToDevice));
    TF_CK(cudaMemcpy(ctx->colidx_d.p, ctx->colidx.data(), sizeof(int32_t) * (size_t)ctx->nnzb, cudaMemcpyHostToDevice));
    TF_CK(cudaMemcpy(ctx->diag_d.p, ctx->diag.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice));
    TF_CK(dalloc(ctx->colour_list_d, sizeof(int32_t) * std::max<size_t>(1, ctx->colour_list.size())));
    if (!ctx->colour_list.empty())
        TF_CK(cudaMemcpy(ctx->colour_list_d.p, ctx->colour_list.data(), sizeof(int32_t) * ctx->colour_list.size(),
                         cudaMemcpyHostToDevice));
    TF_CK(dalloc(ctx->dofmap_d, sizeof(int32_t) * 3 * (size_t)N));
    TF_CK(cudaMemcpy(ctx->dofmap_d.p, ctx->dofmap.data(), sizeof(int32_t) * 3 * (size_t)N, cudaMemcpyHostToDevice));
    const size_t np = std::max<size_t>(1, ctx->slave.size());
    TF_CK(dalloc(ctx->slaves_d, sizeof(int32_t) * np));
    TF_CK(dalloc(ctx->masters_d, sizeof(int32_t) * np));
    if (!ctx->slave.empty()) {
        TF_CK(cudaMemcpy(ctx->slaves_d.p, ctx->slave.data(), sizeof(int32_t) * ctx->slave.size(), cudaMemcpyHostToDevice));
        TF_CK(cudaMemcpy(ctx->masters_d.p, ctx->master.data(), sizeof(int32_t) * ctx->master.size(), cudaMemcpyHostToDevice));
    }
    if (ctx->params.precond == TF_PRECOND_ILU0) {
        const int irc = build_ilu(ctx);
        if (irc != TF_OK) return irc;
    }
    ctx->coarse_dirty = true;
    const size_t np2 = std::max((size_t)std::max(spmv_grid(N), vec_grid(N)) * 2,
                                (size_t)ctx->persistent_grid_max * 8) + 64;
    TF_CK(dalloc(ctx->partials, sizeof(double) * np2));
    if (ctx->krylov_graph) {
        cudaGraphExecDestroy(ctx->krylov_graph);
        ctx->krylov_graph = nullptr;
    }
    return TF_OK;
}

// Multicolour structure of ILU(0): greedy colouring of the block-row graph (two rows share a
// colour only if the pattern has no block between them), nodes sorted by colour, and for every
// row its lower blocks (earlier colour, sorted by colour) and upper blocks (later colour).
int build_ilu(tf_ctx* ctx) {
    const int N = ctx->N;
    std::vector<int32_t> col(N, -1);
    int ncol = 0;
    std::vector<char> used;
    for (int i = 0; i < N; ++i) {
        used.assign(ncol + 1, 0);
        for (int k = ctx->rowptr[i]; k < ctx->rowptr[i + 1]; ++k) {
            const int c = col[ctx->colidx[k]];
            if (c >= 0) used[c] = 1;
        }
        int c = 0;
        while (c < ncol && used[c]) ++c;
        col[i] = c;
        ncol = std::max(ncol, c + 1);
    }
    std::vector<int32_t> cptr(ncol + 1, 0), cnodes(N);
    for (int i = 0; i < N; ++i) cptr[col[i] + 1]++;
    for (int c = 0; c < ncol; ++c) cptr[c + 1] += cptr[c];
    std::vector<int32_t> pos(cptr.begin(), cptr.end() - 1);
    for (int i = 0; i < N; ++i) cnodes[pos[col[i]]++] = i;
    std::vector<int32_t> lo_ptr(N + 1, 0), up_ptr(N + 1, 0), lo_idx, up_idx;
    for (int i = 0; i < N; ++i) {
        std::vector<std::pair<int, int>> lo;
        for (int k = ctx->rowptr[i]; k < ctx->rowptr[i + 1]; ++k) {
            const int c = col[ctx->colidx[k]];
            if (ctx->colidx[k] == i) continue;
            if (c < col[i]) lo.emplace_back(c, k);
            else up_idx.push_back(k);
        }
        std::sort(lo.begin(), lo.end());
        for (auto& q : lo) lo_idx.push_back(q.second);
        lo_ptr[i + 1] = (int32_t)lo_idx.size();
        up_ptr[i + 1] = (int32_t)up_idx.size();
    }
    ctx->ilu_colour_ptr = cptr;
    ctx->ilu_colours = ncol;
    auto up = [&](DevBuf& b, const std::vector<int32_t>& v) -> cudaError_t {
        cudaError_t e = dalloc(b, sizeof(int32_t) * std::max<size_t>(1, v.size()));
        if (e == cudaSuccess && !v.empty()) e = cudaMemcpy(b.p, v.data(), sizeof(int32_t) * v.size(), cudaMemcpyHostToDevice);
        return e;
    };
    TF_CK(up(ctx->ilu_cnodes, cnodes));
    TF_CK(up(ctx->ilu_lo_ptr, lo_ptr));
    TF_CK(up(ctx->ilu_lo_idx, lo_idx));
    TF_CK(up(ctx->ilu_up_ptr, up_ptr));
    TF_CK(up(ctx->ilu_up_idx, up_idx));
    TF_CK(dalloc(ctx->ilu_lu, sizeof(double) * 9 * (size_t)ctx->nnzb));
    TF_CK(dalloc(ctx->ilu_uinv, sizeof(double) * 9 * (size_t)N));
    TF_CK(dalloc(ctx->ilu_y, sizeof(double) * 3 * (size_t)N));
    if (ctx->ilu_graph) {
        cudaGraphExecDestroy(ctx->ilu_graph);
        ctx->ilu_graph = nullptr;
    }
    return TF_OK;
}

IluPlan make_ilu(tf_ctx* c) {
    IluPlan p;
    p.n_colours = c->ilu_colours;
    p.colour_ptr = c->ilu_colour_ptr.data();
    p.cnodes = dptr<int32_t>(c->ilu_cnodes);
    p.lo_ptr = dptr<int32_t>(c->ilu_lo_ptr);
    p.lo_idx = dptr<int32_t>(c->ilu_lo_idx);
    p.up_ptr = dptr<int32_t>(c->ilu_up_ptr);
    p.up_idx = dptr<int32_t>(c->ilu_up_idx);
    p.lu = dptr<double>(c->ilu_lu);
    p.uinv = dptr<double>(c->ilu_uinv);
    p.y = dptr<double>(c->ilu_y);
    return p;
}

// Conjugate gradients for the persistent solve: asked for, or left to the library (TF_KRYLOV_AUTO)
// and every tissue's Jacobian symmetric (no element has internal viscosity).
bool use_cg(const tf_ctx* c) {
    return c->params.krylov_method == TF_KRYLOV_CG || (c->params.krylov_method == TF_KRYLOV_AUTO && !c->has_visc);
}

KrylovWork make_work(tf_ctx* c) {
    KrylovWork w;
    w.n_nodes = c->N;
    w.rowptr = dptr<int32_t>(c->rowptr_d);
    w.colidx = dptr<int32_t>(c->colidx_d);
    w.diag = dptr<int32_t>(c->diag_d);
    w.vals = dptr<double>(c->vals);
    w.x = dptr<double>(c->du);
    w.b = dptr<double>(c->g);
    w.r = dptr<double>(c->r);
    w.rhat = dptr<double>(c->rhat);
    w.p = dptr<double>(c->p);
    w.v = dptr<double>(c->v);
    w.s = dptr<double>(c->s);
    w.t = dptr<double>(c->t);
    w.phat = dptr<double>(c->phat);
    w.shat = dptr<double>(c->shat);
    w.dinv = dptr<double>(c->dinv);
    w.partials = dptr<double>(c->partials);
    w.n_partials = (int32_t)(c->partials.bytes / sizeof(double));
    w.sc = dptr<KrylovScalars>(c->sc);
    w.dflags = dptr<int32_t>(c->dflags);
    const bool pk = c->pk_on && c->pk_pairs_n > 0;
    w.pk_ptr = pk ? dptr<int32_t>(c->pk_ptr_d) : nullptr;
    w.pk_col = pk ? dptr<int32_t>(c->pk_col_d) : nullptr;
    w.pk_blk = pk ? dptr<int32_t>(c->pk_blk_d) : nullptr;
    w.pk_vals = pk ? dptr<double>(c->pk_vals_d) : nullptr;
    return w;
}

AssembleArgs make_assemble(tf_ctx* c, double dt) {
    AssembleArgs a;
    a.elems = dptr<ElemRecord>(c->elems);
    a.elem_list = nullptr;
    a.e_begin = 0;
    a.e_count = c->E;
    a.uk = dptr<double>(c->uk);
    a.un = dptr<double>(c->un);
    a.inv_dt = 1.0 / dt;
    a.fixmask = dptr<uint8_t>(c->fixmask);
    a.dofmap = dptr<int32_t>(c->dofmap_d);
    a.rowptr = dptr<int32_t>(c->rowptr_d);
    a.colidx = dptr<int32_t>(c->colidx_d);
    a.vals = dptr<double>(c->vals);
    a.g = dptr<double>(c->g);
    a.dflags = dptr<int32_t>(c->dflags);
    a.tissue_active = dptr<int32_t>(c->active_d);
    return a;
}

// CTA plan of the persistent solve. A tissue's expected work is weight[t] (rows x BiCGStab
// iterations). The plan minimises the largest per-CTA load Q over the C co-resident CTAs: every
// tissue heavier than Q gets a group of ceil(weight / Q) CTAs (at least 64 rows each; with a
// batch coarse space at most one CTA per aggregate) and runs with group barriers; the lighter
// tissues are packed first-fit-decreasing into bins of capacity Q, and each bin's CTA solves its
// tissues one after another (CTA-level barriers only). Q is the smallest value (by bisection)
// whose groups and bins fit in C. Inactive tissues get none. The plan is rebuilt every Newton
// round of a batch with the last Krylov iteration counts as weights.
int build_plan(tf_ctx* ctx, const std::vector<double>& weight, const int32_t* active) {
    const int T = ctx->T;
    const int cmax = std::max(ctx->persistent_grid_max, 1);
    std::vector<int64_t> rows(T);
    double wsum = 0.0;
    int n_act = 0;
    for (int t = 0; t < T; ++t) {
        rows[t] = ctx->tissue_node0[t + 1] - ctx->tissue_node0[t];
        if (active[t]) {
            wsum += weight[t];
            ++n_act;
        }
    }
    std::vector<int32_t> n(T, 0);                 // CTAs of a group tissue (0: packed or inactive)
    std::vector<std::vector<int32_t>> lists;      // tissues of every CTA
    if (ctx->persistent_grid_max > 0 && n_act > 0) {
        std::vector<int64_t> cap(T, 1);  // most CTAs a tissue's group may have
        std::vector<int> order;          // active tissues, heaviest first
        for (int t = 0; t < T; ++t) {
            if (!active[t]) continue;
            cap[t] = std::max<int64_t>(1, (rows[t] + 63) / 64);
            if (ctx->bc_active && (int)ctx->bc_tissue_agg0.size() == T + 1)  // every CTA owns whole aggregates
                cap[t] = std::min<int64_t>(cap[t], ctx->bc_tissue_agg0[t + 1] - ctx->bc_tissue_agg0[t]);
            order.push_back(t);
        }
        std::sort(order.begin(), order.end(),
                  [&](int a, int b) { return weight[a] > weight[b] || (weight[a] == weight[b] && a < b); });
        // CTAs needed when no CTA should carry more than Q: a group of ceil(w / Q) CTAs for every
        // tissue heavier than Q, first-fit-decreasing bins of capacity Q for the others
        std::vector<double> load;
        std::vector<std::vector<int32_t>> bins;
        auto need = [&](double Q, bool keep) -> int64_t {
            int64_t groups = 0;
            load.clear();
            bins.clear();
            for (int t : order) {
                const double w = std::max(weight[t], 0.0);
                if (w > Q && cap[t] > 1) {
                    const int64_t k = std::min<int64_t>(cap[t], std::max<int64_t>(2, (int64_t)std::ceil(w / Q)));
                    if (keep) n[t] = (int32_t)k;
                    groups += k;
                    continue;
                }
                size_t b = 0;
                while (b < load.size() && load[b] + w > Q) ++b;
                if (b == load.size()) {
                    load.push_back(0.0);
                    bins.emplace_back();
                }
                load[b] += w;
                bins[b].push_back(t);
            }
            return groups + (int64_t)load.size();
        };
        // the smallest per-CTA load that fits the co-resident CTAs (bisection; Q = W always fits)
        double lo = wsum / cmax, hi = std::max(wsum, 1e-300);
        if (need(lo, false) <= cmax) hi = lo;
        for (int it = 0; it < 60 && hi > lo * (1.0 + 1e-9); ++it) {
            const double mid = 0.5 * (lo + hi);
            if (need(mid, false) <= cmax)
                hi = mid;
            else
                lo = mid;
        }
        need(hi, true);
        ctx->plan_cta0.resize(T);
        for (int t : order)
            if (n[t] > 0) {
                ctx->plan_cta0[t] = (int32_t)lists.size();
                for (int k = 0; k < n[t]; ++k) lists.push_back({t});
            }
        for (auto& bin : bins) {
            for (int32_t t : bin) {
                ctx->plan_cta0[t] = (int32_t)lists.size();
                n[t] = 1;
            }
            lists.push_back(bin);
        }
        // the solve takes the bins' tissues from a queue, heaviest first, on every CTA as it
        // becomes free (the bins remain the static assignment of the Newton update); the grid is
        // filled up to the co-resident CTAs
        ctx->plan_queue.clear();
        for (int t : order)
            if (n[t] == 1) ctx->plan_queue.push_back(t);
        while ((int)lists.size() < cmax && !ctx->plan_queue.empty()) lists.emplace_back();
    } else {
        ctx->plan_queue.clear();
        for (int t = 0; t < T; ++t)
            if (active[t]) {
                n[t] = 1;
                lists.push_back({t});
                ctx->plan_queue.push_back(t);
            }
    }
    ctx->plan_cta0.resize(T, 0);
    if (ctx->persistent_grid_max == 0)
        for (int t = 0, k = 0; t < T; ++t)
            if (active[t]) ctx->plan_cta0[t] = k++;
    ctx->plan_ncta = n;
    ctx->plan_list_ptr.assign(1, 0);
    ctx->plan_list.clear();
    for (auto& l : lists) {
        for (int32_t t : l) ctx->plan_list.push_back(t);
        ctx->plan_list_ptr.push_back((int32_t)ctx->plan_list.size());
    }
    if (lists.empty()) {  // keeps a valid launch shape: one CTA with nothing to do
        ctx->plan_list_ptr.push_back(0);
    }
    const size_t C = ctx->plan_list_ptr.size() - 1;
    TF_CK(dalloc(ctx->plan_list_ptr_d, sizeof(int32_t) * ((size_t)cmax + 2)));
    // every CTA of a group lists its tissue once; a packed tissue appears once in its bin
    TF_CK(dalloc(ctx->plan_list_d, sizeof(int32_t) * ((size_t)cmax + T + 1)));
    TF_CK(dalloc(ctx->plan_cta0_d, sizeof(int32_t) * T));
    TF_CK(dalloc(ctx->plan_queue_d, sizeof(int32_t) * (T + 1)));
    TF_CK(dalloc(ctx->queue_head_d, sizeof(int32_t) * 4));
    if (!ctx->plan_queue.empty())
        TF_CK(cudaMemcpyAsync(ctx->plan_queue_d.p, ctx->plan_queue.data(), sizeof(int32_t) * ctx->plan_queue.size(),
                              cudaMemcpyHostToDevice, ctx->stream));
    TF_CK(dalloc(ctx->plan_ncta_d, sizeof(int32_t) * T));
    TF_CK(dalloc(ctx->plan_row0_d, sizeof(int32_t) * (T + 1)));
    TF_CK(cudaMemcpyAsync(ctx->plan_list_ptr_d.p, ctx->plan_list_ptr.data(), sizeof(int32_t) * (C + 1),
                          cudaMemcpyHostToDevice, ctx->stream));
    if (!ctx->plan_list.empty())
        TF_CK(cudaMemcpyAsync(ctx->plan_list_d.p, ctx->plan_list.data(), sizeof(int32_t) * ctx->plan_list.size(),
                              cudaMemcpyHostToDevice, ctx->stream));
    TF_CK(cudaMemcpyAsync(ctx->plan_cta0_d.p, ctx->plan_cta0.data(), sizeof(int32_t) * T, cudaMemcpyHostToDevice, ctx->stream));
    TF_CK(cudaMemcpyAsync(ctx->plan_ncta_d.p, ctx->plan_ncta.data(), sizeof(int32_t) * T, cudaMemcpyHostToDevice, ctx->stream));
    TF_CK(cudaMemcpyAsync(ctx->plan_row0_d.p, ctx->tissue_node0.data(), sizeof(int32_t) * (T + 1), cudaMemcpyHostToDevice,
                          ctx->stream));
    TF_CK(cudaStreamSynchronize(ctx->stream));  // the host vectors may change before the next round
    const size_t need = 8 * (size_t)cmax + 64;  // groups' slots, then every CTA's own queue slots
    if (ctx->partials.bytes < sizeof(double) * need) TF_CK(dalloc(ctx->partials, sizeof(double) * need));
    return TF_OK;
}

// Initial work estimate of a tissue: rows x sqrt(rows) (BiCGStab iterations grow with the
// mesh's linear size).
std::vector<double> rows_weight(tf_ctx* ctx) {
    std::vector<double> w(ctx->T);
    for (int t = 0; t < ctx->T; ++t) {
        const double r = ctx->tissue_node0[t + 1] - ctx->tissue_node0[t];
        w[t] = r * std::sqrt(r);
    }
    return w;
}

int build_plan_all(tf_ctx* ctx) {
    std::vector<int32_t> all(ctx->T, 1);
    return build_plan(ctx, rows_weight(ctx), all.data());
}

BatchPlan make_plan(tf_ctx* c) {
    BatchPlan p{};
    p.cg = use_cg(c) ? 1 : 0;
    p.warm = 0;
    // a symmetric J with packing pairs is indefinite across every pair: MINRES
    p.minres = (p.cg && c->pk_on && c->pk_pairs_n > 0) ? 1 : 0;
    p.agg_per_cta = (c->coarse_m > 0 && c->coarse_ok) ? c->coarse_m : 0;
    p.n_coarse = c->n_coarse;
    p.node_d = dptr<double>(c->node_d);
    p.node_mask = dptr<uint8_t>(c->node_mask);
    p.agg_m = dptr<double>(c->agg_m);
    p.coarse_inv = dptr<double>(c->coarse_inv);
    p.coarse_r = dptr<double>(c->coarse_r);
    p.batch_coarse = (c->bc_active && c->coarse_ok) ? 1 : 0;
    p.coarse_ld = c->bc_ld;
    p.tissue_agg0 = dptr<int32_t>(c->bc_tissue_agg0_d);
    p.agg_ptr = dptr<int32_t>(c->bc_agg_ptr_d);
    p.agg_nodes = dptr<int32_t>(c->bc_agg_nodes_d);
    p.coarse_base = dptr<int64_t>(c->bc_base_d);
    // the partial-moment slots were laid out for ml_nct CTAs
    p.ml = (c->ml_active && c->coarse_ok && !c->plan_ncta.empty() && c->plan_ncta[0] == c->ml_nct) ? 1 : 0;
    if (p.ml) {
        p.agg_ptr = dptr<int32_t>(c->ml_leaf_ptr_d);
        p.agg_nodes = dptr<int32_t>(c->ml_leaf_nodes_d);
    }
    p.ml_levels = c->ml_levels;
    p.ml_n_leaf = c->ml_n_leaf;
    for (int l = 0; l < kMlMaxLevels; ++l) {
        p.ml_span[l] = c->ml_span[l];
        p.ml_count[l] = c->ml_count[l];
        p.ml_set0[l] = c->ml_set0[l];
    }
    p.ml_cen = dptr<double>(c->ml_cen_d);
    p.ml_w = dptr<double>(c->ml_w_d);
    p.ml_top_inv = dptr<double>(c->ml_top_d);
    p.ml_leaf_m = dptr<double>(c->ml_leaf_m_d);
    p.ml_part = dptr<double>(c->ml_part_d);
    p.ml_pstart = dptr<int32_t>(c->ml_pstart_d);
    p.ml_first_cta = dptr<int32_t>(c->ml_first_cta_d);
    p.ml_pos_leaf = dptr<int32_t>(c->ml_pos_leaf_d);
    p.n_tissues = c->T;
    p.n_cta = (int32_t)c->plan_list_ptr.size() - 1;
    p.cta_list_ptr = dptr<int32_t>(c->plan_list_ptr_d);
    p.cta_list = dptr<int32_t>(c->plan_list_d);
    p.cta0 = dptr<int32_t>(c->plan_cta0_d);
    p.ncta = dptr<int32_t>(c->plan_ncta_d);
    p.row0 = dptr<int32_t>(c->plan_row0_d);
    p.active = dptr<int32_t>(c->active_d);
    p.group = c->smooth_G;
    p.queue = dptr<int32_t>(c->plan_queue_d);
    p.n_queue = (int32_t)c->plan_queue.size();
    p.queue_head = dptr<int32_t>(c->queue_head_d);
    p.barriers = dptr<GridBarrier>(c->tbarriers);
    p.scalars = dptr<KrylovScalars>(c->tscalars);
    p.du2 = dptr<double>(c->tdu2);
    return p;
}

// Element kernels for the current schedule (no memset, no node terms).
cudaError_t launch_elements(tf_ctx* c, double dt, int scatter, int teams) {
    AssembleArgs a = make_assemble(c, dt);
    if (scatter == TF_SCATTER_COLOURED && c->n_colours > 0) {
        c->launches += c->n_colours + (c->n_routed > 0 ? 1 : 0);
        a.elem_list = dptr<int32_t>(c->colour_list_d);
        for (int k = 0; k < c->n_colours; ++k) {
            a.e_begin = c->colour_offsets[k];
            a.e_count = c->colour_offsets[k + 1] - c->colour_offsets[k];
            cudaError_t err = launch_element_assemble(a, teams, c->has_visc, 1, c->stream);
            if (err != cudaSuccess) return err;
        }
        if (c->n_routed > 0) {
            a.e_begin = c->E - c->n_routed;
            a.e_count = c->n_routed;
            return launch_element_assemble(a, teams, c->has_visc, 0, c->stream);
        }
        return cudaSuccess;
    }
    c->launches += 1;
    return launch_element_assemble(a, teams, c->has_visc, scatter == TF_SCATTER_STAGED ? 2 : 0, c->stream);
}

// One Newton iteration's system: J (BSR3) and g in the context's buffers.
int assemble_system(tf_ctx* ctx, double dt) {
    TF_CK(cudaMemsetAsync(ctx->vals.p, 0, sizeof(double) * 9 * (size_t)ctx->nnzb, ctx->stream));
    TF_CK(cudaMemsetAsync(ctx->g.p, 0, sizeof(double) * 3 * (size_t)ctx->N, ctx->stream));
    TF_CK(launch_elements(ctx, dt, ctx->scatter, ctx->teams));
    NodeArgs na;
    na.n_nodes = ctx->N;
    na.uk = dptr<double>(ctx->uk);
    na.un = dptr<double>(ctx->un);
    na.dt = dt;
    na.fixmask = dptr<uint8_t>(ctx->fixmask);
    na.ext_visc = dptr<double>(ctx->ext_visc);
    na.visc_surface = dptr<double>(ctx->visc_surface);
    na.ext_force = ctx->has_ext_force ? dptr<double>(ctx->ext_force) : nullptr;
    na.dofmap = dptr<int32_t>(ctx->dofmap_d);
    na.diag = dptr<int32_t>(ctx->diag_d);
    na.rowptr = dptr<int32_t>(ctx->rowptr_d);
    na.colidx = dptr<int32_t>(ctx->colidx_d);
    na.vals = dptr<double>(ctx->vals);
    na.g = dptr<double>(ctx->g);
    na.dflags = dptr<int32_t>(ctx->dflags);
    na.node_tissue = dptr<int32_t>(ctx->node_tissue_d);
    na.tissue_active = dptr<int32_t>(ctx->active_d);
    TF_CK(launch_node_terms(na, ctx->stream));
    ctx->launches += 1;
    if (ctx->pk_on && ctx->pk_pairs_n > 0) {
        PackTerms pt;
        pt.n_pairs = ctx->pk_pairs_n;
        pt.pairs = dptr<int32_t>(ctx->pk_pairs_d);
        pt.x = dptr<double>(ctx->uk);
        pt.mass = dptr<double>(ctx->pk_mass_d);
        pt.prm = dptr<PackParams>(ctx->pk_prm_d);
        pt.fixmask = dptr<uint8_t>(ctx->fixmask);
        pt.diag = dptr<int32_t>(ctx->diag_d);
        pt.vals = dptr<double>(ctx->vals);
        pt.g = dptr<double>(ctx->g);
        pt.pk_vals = dptr<double>(ctx->pk_vals_d);
        pt.dfdx = dptr<double>(ctx->pk_dfdx_d);
        TF_CK(launch_packing_terms(pt, ctx->stream));
        ctx->launches += 1;
    }
    if (ctx->lm_on) {
        LumenArgs la;
        la.n_nodes = ctx->N;
        la.n_tri = ctx->lm_n_tri;
        la.elems = dptr<ElemRecord>(ctx->elems);
        la.tri_elem = dptr<int32_t>(ctx->lm_tri_d);
        la.x = dptr<double>(ctx->uk);
        la.fixmask = dptr<uint8_t>(ctx->fixmask);
        la.bulk = ctx->lm_bulk;
        la.state = dptr<LumenState>(ctx->lm_state_d);
        la.part = dptr<double>(ctx->lm_part_d);
        la.g = dptr<double>(ctx->g);
        la.G = dptr<double>(ctx->lm_G_d);
        la.vals = dptr<double>(ctx->vals);
        TF_CK(launch_lumen_terms(la, ctx->stream));
        ctx->launches += 3;
    }
    return TF_OK;
}

// The step's packing pairs at positions x (device [N][3]) with the current Fg: node masses,
// thresholds and pairs on the device; the pair list comes back to the host, which lays out the
// rows of the extra blocks (i, j) and (j, i) for the SpMVs.
int packing_detect(tf_ctx* ctx, const double* x) {
    const int N = ctx->N;
    const int before = ctx->pk_pairs_n;
    // the captured Krylov graphs hold the packing rows' pointers (make_work): drop them whenever
    // the step has pairs or had some, so the next chunked solve captures the current ones
    struct DropGraphs {
        tf_ctx* c;
        int before;
        ~DropGraphs() {
            if (before == 0 && c->pk_pairs_n == 0) return;
            if (c->krylov_graph) {
                cudaGraphExecDestroy(c->krylov_graph);
                c->krylov_graph = nullptr;
            }
            if (c->ilu_graph) {
                cudaGraphExecDestroy(c->ilu_graph);
                c->ilu_graph = nullptr;
            }
        }
    } drop{ctx, before};
    PackArgs a;
    a.n_nodes = N;
    a.n_elems = ctx->E;
    a.elems = dptr<ElemRecord>(ctx->elems);
    a.x = x;
    a.fg = dptr<double>(ctx->fg);
    a.v0 = dptr<double>(ctx->pk_v0_d);
    a.exposed = dptr<uint8_t>(ctx->exposed);
    a.peripodial = dptr<uint8_t>(ctx->peripodial);
    a.placement = dptr<int8_t>(ctx->pk_place_d);
    a.rowptr = dptr<int32_t>(ctx->rowptr_d);
    a.colidx = dptr<int32_t>(ctx->colidx_d);
    a.mass = dptr<double>(ctx->pk_mass_d);
    a.prm = dptr<PackParams>(ctx->pk_prm_d);
    a.hash_bits = ctx->pk_hash_bits;
    a.bucket_cnt = dptr<int32_t>(ctx->pk_bucket_cnt_d);
    a.bucket_start = dptr<int32_t>(ctx->pk_bucket_start_d);
    a.bucket_nodes = dptr<int32_t>(ctx->pk_bucket_nodes_d);
    a.node_cnt = dptr<int32_t>(ctx->pk_node_cnt_d);
    a.node_start = dptr<int32_t>(ctx->pk_node_start_d);
    a.scan_tmp = dptr<int32_t>(ctx->pk_scan_d);
    a.pairs = dptr<int32_t>(ctx->pk_pairs_d);
    a.capacity = ctx->pk_capacity;
    TF_CK(launch_packing_detect(a, ctx->stream));
    ctx->launches += 14;
    int32_t total = 0;
    TF_CK(cudaMemcpyAsync(&total, a.node_start + N, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    TF_CK(cudaStreamSynchronize(ctx->stream));
    ctx->pk_pairs_n = 0;
    ctx->h_pk_pairs.clear();
    if (total <= 0) return TF_OK;
    if (total > ctx->pk_capacity) {
        ctx->pk_capacity = total + total / 2;
        TF_CK(dalloc(ctx->pk_pairs_d, sizeof(int32_t) * 2 * (size_t)ctx->pk_capacity));
        TF_CK(dalloc(ctx->pk_vals_d, sizeof(double) * 18 * (size_t)ctx->pk_capacity));
        TF_CK(dalloc(ctx->pk_dfdx_d, sizeof(double) * 9 * (size_t)ctx->pk_capacity));
        TF_CK(dalloc(ctx->pk_col_d, sizeof(int32_t) * 2 * (size_t)ctx->pk_capacity));
        TF_CK(dalloc(ctx->pk_blk_d, sizeof(int32_t) * 2 * (size_t)ctx->pk_capacity));
        a.pairs = dptr<int32_t>(ctx->pk_pairs_d);
        a.capacity = ctx->pk_capacity;
    }
    TF_CK(launch_packing_pairs(a, ctx->stream));
    ctx->launches += 1;
    ctx->h_pk_pairs.resize((size_t)2 * total);
    TF_CK(cudaMemcpyAsync(ctx->h_pk_pairs.data(), a.pairs, sizeof(int32_t) * 2 * (size_t)total, cudaMemcpyDeviceToHost,
                          ctx->stream));
    TF_CK(cudaStreamSynchronize(ctx->stream));
    // extra blocks by row: row i holds (i, j) = block 2p, row j holds (j, i) = block 2p + 1
    std::vector<int32_t> ptr((size_t)N + 1, 0), col((size_t)2 * total), blk((size_t)2 * total);
    for (int p = 0; p < total; ++p) {
        ptr[ctx->h_pk_pairs[2 * p] + 1]++;
        ptr[ctx->h_pk_pairs[2 * p + 1] + 1]++;
    }
    for (int n = 0; n < N; ++n) ptr[n + 1] += ptr[n];
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    for (int p = 0; p < total; ++p) {
        const int i = ctx->h_pk_pairs[2 * p], j = ctx->h_pk_pairs[2 * p + 1];
        col[fill[i]] = j;
        blk[fill[i]++] = 2 * p;
        col[fill[j]] = i;
        blk[fill[j]++] = 2 * p + 1;
    }
    TF_CK(dalloc(ctx->pk_ptr_d, sizeof(int32_t) * ptr.size()));
    TF_CK(cudaMemcpyAsync(ctx->pk_ptr_d.p, ptr.data(), sizeof(int32_t) * ptr.size(), cudaMemcpyHostToDevice, ctx->stream));
    TF_CK(cudaMemcpyAsync(ctx->pk_col_d.p, col.data(), sizeof(int32_t) * col.size(), cudaMemcpyHostToDevice, ctx->stream));
    TF_CK(cudaMemcpyAsync(ctx->pk_blk_d.p, blk.data(), sizeof(int32_t) * blk.size(), cudaMemcpyHostToDevice, ctx->stream));
    TF_CK(cudaStreamSynchronize(ctx->stream));  // the host vectors go out of scope
    ctx->pk_pairs_n = total;
    return TF_OK;
}

int krylov_status_to_tf(int ks) {
    switch (ks) {
        case KS_CONVERGED: return TF_OK;
        case KS_MAXIT: return TF_KRYLOV_MAX_ITERS;
        case KS_BREAKDOWN: return TF_KRYLOV_BREAKDOWN;
        case KS_NONFINITE: return TF_NONFINITE;
        default: return TF_KRYLOV_MAX_ITERS;
    }
}

// ---- two-level preconditioner ----------------------------------------------------------
//
// Coarse space of one tissue for the persistent solve: the plan's CTA row ranges, each split
// into m contiguous aggregates (the kernel's formula), so restriction and prolongation stay
// inside a CTA. Meshes numbered point-major along a space-filling curve make contiguous node
// ranges compact patches. Each aggregate gets six modes - three translations and three
// rotations about its centroid in reference coordinates - with fixed and slave DoFs zeroed
// (the solve never moves them), orthonormalised by modified Gram-Schmidt; a mode that
// vanishes there (below 1e-10 of its initial norm) is dropped and its coarse unknown gets a
// unit diagonal. The coarse operator P^T J P is assembled on the device every solve and
// inverted explicitly (LU, cuSOLVER), so an application is a dense row-block product.
// Modes (translations, rotations about the centroid in reference coordinates; fixed and slave
// DoFs zeroed; two-pass modified Gram-Schmidt with the coefficient transform tracked; a mode
// below 1e-6 of its initial norm dropped and listed in `empty`) of the aggregates with node
// boundaries agg0, the per-aggregate block lists of the coarse assembly, all uploaded.
int coarse_space_upload(tf_ctx* ctx, const std::vector<int32_t>& agg_ptr, const std::vector<int32_t>& agg_nodes,
                        std::vector<int32_t>& empty, bool raw = false) {
    const int N = ctx->N, n_agg = (int)agg_ptr.size() - 1;
    std::vector<double> X((size_t)N * 3, 0.0);
    for (int e = 0; e < ctx->E; ++e)
        for (int a = 0; a < 6; ++a)
            for (int d = 0; d < 3; ++d) X[(size_t)ctx->conn[(size_t)e * 6 + a] * 3 + d] = ctx->xref[(size_t)e * 18 + a * 3 + d];
    std::vector<double> pm(raw ? 0 : (size_t)N * 18, 0.0), nd((size_t)N * 3, 0.0), am(raw ? 0 : (size_t)n_agg * 36, 0.0);
    std::vector<uint8_t> nmask(N, 0);
    empty.clear();
    for (int i = 0; i < N; ++i)
        for (int d = 0; d < 3; ++d) {
            const size_t dof = (size_t)i * 3 + d;
            const bool fixed = (ctx->h_fixmask.size() == (size_t)N) && (ctx->h_fixmask[i] >> d & 1);
            if (!fixed && ctx->dofmap[dof] == (int32_t)dof) nmask[i] |= (uint8_t)(1u << d);
        }
    for (int a = 0; a < n_agg; ++a) {
        const int32_t* nodes = agg_nodes.data() + agg_ptr[a];
        const int n = agg_ptr[a + 1] - agg_ptr[a];
        double c[3] = {0, 0, 0};
        for (int i = 0; i < n; ++i)
            for (int d = 0; d < 3; ++d) c[d] += X[(size_t)nodes[i] * 3 + d] / n;
        // the masked modes B_i = [I | (d_i x)] as explicit columns over the aggregate's DoFs
        const size_t len = (size_t)3 * n;
        std::vector<double> B(6 * len, 0.0);
        for (int i = 0; i < n; ++i) {
            const int node = nodes[i];
            double dd[3];
            for (int d = 0; d < 3; ++d) dd[d] = nd[(size_t)node * 3 + d] = X[(size_t)node * 3 + d] - c[d];
            const double Bi[3][6] = {{1, 0, 0, 0, dd[2], -dd[1]}, {0, 1, 0, -dd[2], 0, dd[0]}, {0, 0, 1, dd[1], -dd[0], 0}};
            for (int d = 0; d < 3; ++d)
                if (nmask[node] >> d & 1)
                    for (int q = 0; q < 6; ++q) B[q * len + 3 * i + d] = Bi[d][q];
        }
        if (raw) continue;  // raw rigid modes (multilevel space): node_d and the mask are all it needs
        // modified Gram-Schmidt (two passes) on the explicit columns, the same operations applied
        // to coefficient vectors, so that the orthonormal columns are B m_q; a mode whose norm
        // falls below 1e-6 of its initial norm is dropped
        double M[36] = {0};
        bool kept[6] = {false, false, false, false, false, false};
        double cols[6][6] = {{0}};
        for (int q = 0; q < 6; ++q) {
            double* bq = &B[q * len];
            double v[6] = {0, 0, 0, 0, 0, 0};
            v[q] = 1.0;
            double n0 = 0.0;
            for (size_t r = 0; r < len; ++r) n0 += bq[r] * bq[r];
            n0 = std::sqrt(n0);
            for (int pass = 0; pass < 2; ++pass)
                for (int p = 0; p < q; ++p) {
                    if (!kept[p]) continue;
                    const double* bp = &B[p * len];
                    double dot = 0.0;
                    for (size_t r = 0; r < len; ++r) dot += bp[r] * bq[r];
                    for (size_t r = 0; r < len; ++r) bq[r] -= dot * bp[r];
                    for (int r = 0; r < 6; ++r) v[r] -= dot * cols[p][r];
                }
            double nq = 0.0;
            for (size_t r = 0; r < len; ++r) nq += bq[r] * bq[r];
            nq = std::sqrt(nq);
            if (n == 0 || n0 == 0.0 || nq <= 1e-6 * n0) {
                for (size_t r = 0; r < len; ++r) bq[r] = 0.0;
                empty.push_back(6 * a + q);
                continue;
            }
            kept[q] = true;
            for (size_t r = 0; r < len; ++r) bq[r] /= nq;
            for (int r = 0; r < 6; ++r) cols[q][r] = v[r] / nq;
        }
        for (int p = 0; p < 6; ++p)
            for (int q = 0; q < 6; ++q) M[p * 6 + q] = kept[q] ? cols[q][p] : 0.0;  // M[p][q] = (m_q)_p
        for (int k = 0; k < 36; ++k) am[(size_t)a * 36 + k] = M[k];
        // explicit modes for the coarse-operator assembly: P_i = mask_i o (B_i M)
        for (int i = 0; i < n; ++i)
            for (int d = 0; d < 3; ++d)
                for (int q = 0; q < 6; ++q) pm[(size_t)nodes[i] * 18 + d * 6 + q] = B[q * len + 3 * i + d];
    }
    // Jacobian blocks grouped by (row aggregate, column aggregate)
    std::vector<int32_t> aggof(N);
    for (int a = 0; a < n_agg; ++a)
        for (int k = agg_ptr[a]; k < agg_ptr[a + 1]; ++k) aggof[agg_nodes[k]] = a;
    std::vector<int32_t> agg_slot_ptr(n_agg + 1, 0), slot_agg, slot_ptr(1, 0), blk, blk_row;
    blk.reserve(ctx->nnzb);
    blk_row.reserve(ctx->nnzb);
    std::vector<std::array<int32_t, 3>> items;
    for (int a = 0; a < n_agg; ++a) {
        items.clear();
        for (int q = agg_ptr[a]; q < agg_ptr[a + 1]; ++q) {
            const int i = agg_nodes[q];
            for (int k = ctx->rowptr[i]; k < ctx->rowptr[i + 1]; ++k) items.push_back({aggof[ctx->colidx[k]], k, i});
        }
        std::sort(items.begin(), items.end());
        for (size_t q = 0; q < items.size(); ++q) {
            if (q == 0 || items[q][0] != items[q - 1][0]) {
                if (q > 0) slot_ptr.push_back((int32_t)blk.size());
                slot_agg.push_back(items[q][0]);
            }
            blk.push_back(items[q][1]);
            blk_row.push_back(items[q][2]);
        }
        if (!items.empty()) slot_ptr.push_back((int32_t)blk.size());
        agg_slot_ptr[a + 1] = (int32_t)slot_agg.size();
    }
    auto up = [&](DevBuf& b, const void* h, size_t bytes) -> cudaError_t {
        cudaError_t e = dalloc(b, std::max<size_t>(bytes, 16));
        if (e == cudaSuccess && bytes) e = cudaMemcpy(b.p, h, bytes, cudaMemcpyHostToDevice);
        return e;
    };
    TF_CK(up(ctx->pmode_d, pm.data(), raw ? 0 : sizeof(double) * pm.size()));
    TF_CK(up(ctx->node_d, nd.data(), sizeof(double) * nd.size()));
    TF_CK(up(ctx->node_mask, nmask.data(), nmask.size()));
    TF_CK(up(ctx->agg_m, am.data(), raw ? 0 : sizeof(double) * am.size()));
    ctx->h_slot_agg = slot_agg;
    ctx->h_agg_slot_ptr = agg_slot_ptr;
    TF_CK(up(ctx->ca_agg_slot_ptr, agg_slot_ptr.data(), sizeof(int32_t) * agg_slot_ptr.size()));
    TF_CK(up(ctx->ca_slot_agg, slot_agg.data(), sizeof(int32_t) * slot_agg.size()));
    TF_CK(up(ctx->ca_slot_ptr, slot_ptr.data(), sizeof(int32_t) * slot_ptr.size()));
    TF_CK(up(ctx->ca_blk, blk.data(), sizeof(int32_t) * blk.size()));
    TF_CK(up(ctx->ca_blk_row, blk_row.data(), sizeof(int32_t) * blk_row.size()));
    TF_CK(up(ctx->ca_empty, empty.data(), sizeof(int32_t) * empty.size()));
    ctx->n_coarse_empty = (int)empty.size();
    return TF_OK;
}

int build_batch_coarse(tf_ctx* ctx);
int build_ml(tf_ctx* ctx);
int newton_solve(tf_ctx* ctx);

int build_coarse(tf_ctx* ctx) {
    ctx->coarse_dirty = false;
    ctx->coarse_m = 0;
    ctx->bc_active = false;
    if (ctx->params.precond != TF_PRECOND_TWO_LEVEL && ctx->params.precond != TF_PRECOND_MULTILEVEL) return TF_OK;
    ctx->ml_active = false;
    if (ctx->T > 1) return build_batch_coarse(ctx);
    if (ctx->plan_ncta.empty()) return TF_OK;
    const int N = ctx->N, nct = ctx->plan_ncta[0];
    if (nct <= 0) return TF_OK;
    // the multilevel space when asked for, and for large tissues: the one-level space's
    // per-CTA aggregates grow with the tissue (measured: a 180,000-node slab 364 CG iterations per
    // solve with them against ~127 with the multilevel space; the 60,441-node wing disc 243
    // against 226, but its solves are short enough that the multilevel set-up made the step slower)
    if (ctx->params.precond == TF_PRECOND_MULTILEVEL || N >= kMlAutoNodes) return build_ml(ctx);
    int m = std::max(1, std::min(kMaxAggPerCta, 2048 / (6 * nct)));
    while (m > 1 && N / (nct * m) < 8) --m;
    // each CTA's 6m rows of the n_coarse = 6 nct m inverse must fit its shared-memory block
    while (m > 1 && (size_t)36 * nct * m * m * sizeof(float) > (size_t)kCoarseSmemBytes) --m;
    if ((size_t)36 * nct * m * m * sizeof(float) > (size_t)kCoarseSmemBytes) return TF_OK;
    // aggregates much larger than this no longer cut the iteration count (measured on the 2 M-node
    // slab: 6,800-node aggregates left it unchanged); such tissues take the multilevel space
    if (N / (nct * m) > kMaxAggNodes) return build_ml(ctx);
    const int nw = ctx->persist_threads / 32;
    while (m > 1 && nw / m < 1) --m;
    const int n_agg = nct * m, nc = 6 * n_agg;
    if (nc > kMaxCoarse) return TF_OK;  // plan too large for a staged coarse vector: block-Jacobi only
    std::vector<int32_t> agg0(n_agg + 1);
    for (int lc = 0; lc < nct; ++lc) {  // the persistent solve's CTA row ranges and aggregates
        int r0, r1, a0, a1;
        group_split(0, N, lc, nct, ctx->smooth_G, r0, r1);
        for (int k = 0; k < m; ++k) {
            group_split(r0, r1, k, m, ctx->smooth_G, a0, a1);
            agg0[lc * m + k] = a0;
        }
    }
    agg0[n_agg] = N;
    std::vector<int32_t> empty;
    {
        std::vector<int32_t> iota(N);
        for (int k = 0; k < N; ++k) iota[k] = k;
        const int rc = coarse_space_upload(ctx, agg0, iota, empty);
        if (rc != TF_OK) return rc;
    }
    TF_CK(dalloc(ctx->coarse_inv, sizeof(double) * (size_t)nc * nc));
    TF_CK(dalloc(ctx->coarse_r, sizeof(double) * (size_t)nc));
    TF_CK(dalloc(ctx->coarse_info, sizeof(int32_t)));
    TF_CK(dalloc(ctx->coarse_work, invert_coop_scratch_bytes(nc)));
    if (!ctx->h_coarse_info) TF_CK(cudaMallocHost(&ctx->h_coarse_info, sizeof(int32_t)));
    ctx->n_agg = n_agg;
    ctx->n_coarse = nc;
    ctx->n_coarse_empty = (int)empty.size();
    ctx->coarse_m = m;
    ctx->coarse_age = 0;
    ctx->coarse_ok = false;
    return TF_OK;
}

// Recursive coordinate bisection of the n nodes in `nodes` into `parts` spatial sets of nearly
// equal size: each range is split across the longest side of its bounding box, in proportion to
// the parts on either side; nodes at the same coordinate stay on one side where the split allows
// (a prism column's nodes share x and y). On return nodes[cuts[k] .. cuts[k+1]) is part k.
void bisect_nodes(const std::vector<double>& X, int32_t* nodes, int n, int parts, std::vector<int32_t>& cuts) {
    cuts.assign(1, 0);
    struct Range { int b, e, parts; };
    std::vector<Range> stack{{0, n, parts}};
    std::vector<std::pair<int, int>> done;  // (begin, end) of finished parts, in order of completion
    while (!stack.empty()) {
        const Range r = stack.back();
        stack.pop_back();
        if (r.parts <= 1 || r.e - r.b <= 1) {
            done.push_back({r.b, r.e});
            continue;
        }
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int i = r.b; i < r.e; ++i)
            for (int d = 0; d < 3; ++d) {
                lo[d] = std::min(lo[d], X[(size_t)nodes[i] * 3 + d]);
                hi[d] = std::max(hi[d], X[(size_t)nodes[i] * 3 + d]);
            }
        int ax = 0;
        for (int d = 1; d < 3; ++d)
            if (hi[d] - lo[d] > hi[ax] - lo[ax]) ax = d;
        std::sort(nodes + r.b, nodes + r.e, [&](int32_t u, int32_t v) {
            const double cu = X[(size_t)u * 3 + ax], cv = X[(size_t)v * 3 + ax];
            return cu < cv || (cu == cv && u < v);
        });
        const int p1 = r.parts / 2;
        int k = r.b + (int)((long long)(r.e - r.b) * p1 / r.parts);
        auto coord = [&](int i) { return X[(size_t)nodes[i] * 3 + ax]; };
        int kf = k;
        while (kf < r.e && kf > r.b && coord(kf) == coord(kf - 1)) ++kf;
        if (kf < r.e && kf - k <= 8) {
            k = kf;
        } else {
            int kb = k;
            while (kb > r.b && coord(kb) == coord(kb - 1)) --kb;
            if (kb > r.b && k - kb <= 8) k = kb;
        }
        k = std::min(std::max(k, r.b + 1), r.e - 1);
        stack.push_back({k, r.e, r.parts - p1});  // popped after the left half: parts stay in order
        stack.push_back({r.b, k, p1});
    }
    std::sort(done.begin(), done.end());
    for (auto& d : done) cuts.push_back(d.second);
    while ((int)cuts.size() < parts + 1) cuts.push_back(n);  // fewer nodes than parts: empty tails
}

// Coarse space of a batch: every tissue's nodes split into spatial aggregates of about
// kBatchAggNodes nodes (at least one, at most kMaxCoarse / 6) by coordinate bisection, so that
// the aggregates are compact whatever the mesh's node numbering. Tissue t's coarse matrix
// (6 na_t unknowns) sits at t ld^2 in a batch of ld x ld matrices, written transposed so that the
// batched LU inverse comes out row-major; dropped modes and the padding rows get unit diagonals.
int build_batch_coarse(tf_ctx* ctx) {
    const int T = ctx->T;
    std::vector<double> X((size_t)ctx->N * 3, 0.0);  // reference positions of the nodes
    for (int e = 0; e < ctx->E; ++e)
        for (int a = 0; a < 6; ++a)
            for (int d = 0; d < 3; ++d) X[(size_t)ctx->conn[(size_t)e * 6 + a] * 3 + d] = ctx->xref[(size_t)e * 18 + a * 3 + d];
    std::vector<int32_t> agg_ptr(1, 0), agg_nodes(ctx->N), tagg0(T + 1, 0), agg_tissue;
    int ld = 6;
    for (int t = 0; t < T; ++t) {
        const int n0 = ctx->tissue_node0[t], nt = ctx->tissue_node0[t + 1] - n0;
        int na = std::max(1, (int)std::lround((double)nt / kBatchAggNodes));
        na = std::min(na, std::max(1, nt / 8));
        na = std::min(na, kMaxCoarse / 6);
        // bisect the tissue's smoother groups (whole prism columns with G > 1, so that a column
        // stays in one aggregate, consecutive in its sorted node list), each by its first node
        const int G = ctx->smooth_G, ng = nt / G;
        na = std::min(na, ng);
        std::vector<int32_t> reps(ng), cuts;
        for (int k = 0; k < ng; ++k) reps[k] = n0 + k * G;
        bisect_nodes(X, reps.data(), ng, na, cuts);
        for (int k = 0; k < na; ++k) {
            std::sort(reps.begin() + cuts[k], reps.begin() + cuts[k + 1]);
            for (int q = cuts[k]; q < cuts[k + 1]; ++q)
                for (int j = 0; j < G; ++j) agg_nodes[n0 + q * G + j] = reps[q] + j;
            agg_ptr.push_back(n0 + cuts[k + 1] * G);
            agg_tissue.push_back(t);
        }
        tagg0[t + 1] = tagg0[t] + na;
        ld = std::max(ld, 6 * na);
    }
    std::vector<int32_t> empty;
    {
        const int rc = coarse_space_upload(ctx, agg_ptr, agg_nodes, empty);
        if (rc != TF_OK) return rc;
    }
    const size_t ld2 = (size_t)ld * ld;
    std::vector<int64_t> base(T), unit;
    for (int t = 0; t < T; ++t) base[t] = (int64_t)t * (int64_t)ld2;
    for (int32_t q : empty) {
        const int a = q / 6;
        const int t = agg_tissue[a];
        const int local = q - 6 * tagg0[t];
        unit.push_back(base[t] + (int64_t)local * (ld + 1));
    }
    for (int t = 0; t < T; ++t)
        for (int local = 6 * (tagg0[t + 1] - tagg0[t]); local < ld; ++local) unit.push_back(base[t] + (int64_t)local * (ld + 1));
    auto up = [&](DevBuf& b, const void* h, size_t bytes) -> cudaError_t {
        cudaError_t e = dalloc(b, std::max<size_t>(bytes, 16));
        if (e == cudaSuccess && bytes) e = cudaMemcpy(b.p, h, bytes, cudaMemcpyHostToDevice);
        return e;
    };
    TF_CK(dalloc(ctx->coarse_inv, sizeof(double) * ld2 * T));
    TF_CK(dalloc(ctx->coarse_r, sizeof(double) * 6 * (size_t)tagg0[T]));
    TF_CK(dalloc(ctx->bc_info_d, sizeof(int32_t) * (size_t)T));
    std::vector<int32_t> order(T);  // each tissue's coarse order; the padding beyond it is the identity
    for (int t = 0; t < T; ++t) order[t] = 6 * (tagg0[t + 1] - tagg0[t]);
    TF_CK(up(ctx->bc_order_d, order.data(), sizeof(int32_t) * T));
    TF_CK(up(ctx->bc_tissue_agg0_d, tagg0.data(), sizeof(int32_t) * tagg0.size()));
    TF_CK(up(ctx->bc_agg_ptr_d, agg_ptr.data(), sizeof(int32_t) * agg_ptr.size()));
    TF_CK(up(ctx->bc_agg_nodes_d, agg_nodes.data(), sizeof(int32_t) * agg_nodes.size()));
    TF_CK(up(ctx->bc_agg_tissue_d, agg_tissue.data(), sizeof(int32_t) * agg_tissue.size()));
    TF_CK(up(ctx->bc_base_d, base.data(), sizeof(int64_t) * base.size()));
    TF_CK(up(ctx->bc_unit_d, unit.data(), sizeof(int64_t) * unit.size()));
    if (!ctx->h_coarse_info) TF_CK(cudaMallocHost(&ctx->h_coarse_info, sizeof(int32_t)));
    ctx->bc_tissue_agg0 = tagg0;
    ctx->bc_ld = ld;
    ctx->bc_n_unit = (int64_t)unit.size();
    ctx->n_agg = tagg0[T];
    ctx->n_coarse = 6 * tagg0[T];
    ctx->bc_active = true;
    ctx->coarse_age = 0;
    ctx->coarse_ok = false;
    return TF_OK;
}

// ---- multilevel coarse space of a single tissue -------------------------------------------
//
// The tissue's prism columns (col_G consecutive nodes, or single nodes) are split by recursive
// coordinate bisection into a power of two of leaves of about kMlLeafCols columns, in the
// bisection's order, so that 4^k consecutive leaves form a subtree: a compact patch. Level l
// groups 4^(l-1) consecutive leaves; levels are added until one has at most kMlTopMax sets (at
// least two levels), whose operator is inverted densely. Every set's six rigid modes are taken
// about its node centroid. The persistent solve's CTA lc owns the leaves
// [n_leaf lc / nct, n_leaf (lc + 1) / nct); a set of level >= 2 gets one partial-moment slot for
// every CTA whose leaves overlap it (pstart / first_cta), so the restriction needs one group
// barrier and no atomics. The set-up lists name, for every diagonal block below the top and every
// nonzero block of the top operator, the leaf pairs whose blocks sum into it.
int build_ml(tf_ctx* ctx) {
    const int N = ctx->N, nct = ctx->plan_ncta.empty() ? 0 : ctx->plan_ncta[0];
    if (nct <= 0) return TF_OK;
    std::vector<double> X((size_t)N * 3, 0.0);
    for (int e = 0; e < ctx->E; ++e)
        for (int a = 0; a < 6; ++a)
            for (int d = 0; d < 3; ++d) X[(size_t)ctx->conn[(size_t)e * 6 + a] * 3 + d] = ctx->xref[(size_t)e * 18 + a * 3 + d];
    // leaves hold whole smoother groups (the solve's G > 1 path walks them), else whole columns
    const int cg = ctx->smooth_G > 1 ? ctx->smooth_G : ((ctx->col_G > 1 && N % ctx->col_G == 0) ? ctx->col_G : 1);
    const int ncol = N / cg;
    const double want = std::max(1.0, (double)ncol / kMlLeafCols);
    int n_leaf = 1 << (int)std::lround(std::log2(want));
    while (n_leaf > ncol) n_leaf >>= 1;
    if (n_leaf < 2) return TF_OK;  // too small for a coarse space: block-Jacobi alone
    std::vector<int32_t> reps(ncol), cuts;
    for (int k = 0; k < ncol; ++k) reps[k] = k * cg;
    bisect_nodes(X, reps.data(), ncol, n_leaf, cuts);
    std::vector<int32_t> leaf_ptr(1, 0), leaf_nodes;
    leaf_nodes.reserve(N);
    for (int k = 0; k < n_leaf; ++k) {
        std::sort(reps.begin() + cuts[k], reps.begin() + cuts[k + 1]);
        for (int q = cuts[k]; q < cuts[k + 1]; ++q)
            for (int j = 0; j < cg; ++j) leaf_nodes.push_back(reps[q] + j);
        leaf_ptr.push_back((int32_t)leaf_nodes.size());
    }
    if ((int)leaf_nodes.size() != N) return set_error(ctx, TF_ERR_STATE, "multilevel leaves do not cover the nodes");
    // levels
    int L = 1;
    int32_t span[kMlMaxLevels] = {0}, count[kMlMaxLevels] = {0}, set0[kMlMaxLevels] = {0};
    span[0] = 1;
    count[0] = n_leaf;
    do {
        if (L == kMlMaxLevels) return TF_OK;
        span[L] = span[L - 1] * 4;
        count[L] = (n_leaf + span[L] - 1) / span[L];
        ++L;
    } while (count[L - 1] > kMlTopMax);
    for (int l = 1; l < L; ++l) set0[l] = set0[l - 1] + count[l - 1];
    const int n_sets = set0[L - 1] + count[L - 1], n_top = count[L - 1], n_below = set0[L - 1];
    // centroids: leaves from their nodes, higher sets node-weighted from their leaves
    std::vector<double> cen((size_t)n_sets * 3, 0.0);
    std::vector<double> wsum(n_sets, 0.0);
    for (int a = 0; a < n_leaf; ++a) {
        const int n = leaf_ptr[a + 1] - leaf_ptr[a];
        for (int k = leaf_ptr[a]; k < leaf_ptr[a + 1]; ++k)
            for (int d = 0; d < 3; ++d) cen[(size_t)a * 3 + d] += X[(size_t)leaf_nodes[k] * 3 + d] / n;
        for (int l = 1; l < L; ++l) {
            const int g = set0[l] + a / span[l];
            for (int d = 0; d < 3; ++d) cen[(size_t)g * 3 + d] += cen[(size_t)a * 3 + d] * n;
            wsum[g] += n;
        }
    }
    for (int g = count[0]; g < n_sets; ++g)
        for (int d = 0; d < 3; ++d) cen[(size_t)g * 3 + d] /= std::max(wsum[g], 1.0);
    // leaf modes and the leaf-pair block lists
    {
        std::vector<int32_t> empty;
        const int rc = coarse_space_upload(ctx, leaf_ptr, leaf_nodes, empty, true);
        if (rc != TF_OK) return rc;
    }
    const std::vector<int32_t>& sptr = ctx->h_agg_slot_ptr;
    const std::vector<int32_t>& sagg = ctx->h_slot_agg;
    const int n_slots = (int)sagg.size();
    std::vector<int32_t> slot_a(n_slots);
    for (int a = 0; a < n_leaf; ++a)
        for (int q = sptr[a]; q < sptr[a + 1]; ++q) slot_a[q] = a;
    // set-up outputs: the diagonal block of every set below the top, then the top's blocks
    std::vector<int32_t> out_ptr(1, 0), out_slots, out_set, out_col, out_dst;
    for (int l = 0; l + 1 < L; ++l)
        for (int S = 0; S < count[l]; ++S) {
            const int a0 = S * span[l], a1 = std::min(n_leaf, (S + 1) * span[l]);
            for (int a = a0; a < a1; ++a)
                for (int q = sptr[a]; q < sptr[a + 1]; ++q)
                    if (sagg[q] >= a0 && sagg[q] < a1) out_slots.push_back(q);
            out_ptr.push_back((int32_t)out_slots.size());
            out_set.push_back(set0[l] + S);
            out_col.push_back(set0[l] + S);
            out_dst.push_back(set0[l] + S);
        }
    const int n_diag = (int)out_set.size();
    {
        const int sp = span[L - 1];
        std::vector<std::pair<int32_t, int32_t>> items;  // (column top set, slot)
        for (int S = 0; S < n_top; ++S) {
            items.clear();
            for (int a = S * sp; a < std::min(n_leaf, (S + 1) * sp); ++a)
                for (int q = sptr[a]; q < sptr[a + 1]; ++q) items.push_back({sagg[q] / sp, q});
            std::sort(items.begin(), items.end());
            for (size_t k = 0; k < items.size(); ++k) {
                out_slots.push_back(items[k].second);
                if (k + 1 == items.size() || items[k + 1].first != items[k].first) {
                    const int T = items[k].first;
                    out_ptr.push_back((int32_t)out_slots.size());
                    out_set.push_back(set0[L - 1] + S);
                    out_col.push_back(set0[L - 1] + T);
                    out_dst.push_back(S * n_top + T);
                }
            }
        }
    }
    // partial-moment slots of the sets of levels >= 2 for this plan's CTA split
    std::vector<int32_t> cta_of(n_leaf, 0);
    for (int c = 0; c < nct; ++c)
        for (int a = (int)((long long)n_leaf * c / nct); a < (int)((long long)n_leaf * (c + 1) / nct); ++a) cta_of[a] = c;
    std::vector<int32_t> pstart(n_sets + 1, 0), first_cta(n_sets, 0);
    for (int l = 0; l < L; ++l)
        for (int S = 0; S < count[l]; ++S) {
            const int g = set0[l] + S;
            int np = 0;
            if (l > 0) {
                const int a0 = S * span[l], a1 = std::min(n_leaf, (S + 1) * span[l]);
                first_cta[g] = cta_of[a0];
                np = cta_of[a1 - 1] - cta_of[a0] + 1;
            }
            pstart[g + 1] = pstart[g] + np;
        }
    // every CTA stages the top moments and one motion per overlapping set in the solve's
    // shared coarse vector
    for (int c = 0; c < nct; ++c) {
        const int l0 = (int)((long long)n_leaf * c / nct), l1 = (int)((long long)n_leaf * (c + 1) / nct);
        int jobs = 0;
        for (int l = 1; l < L && l1 > l0; ++l) jobs += (l1 - 1) / span[l] - l0 / span[l] + 1;
        if (6 * (n_top + jobs) > kMaxCoarse) return TF_OK;  // too many levels for the staging: block-Jacobi
    }
    auto up = [&](DevBuf& b, const void* h, size_t bytes) -> cudaError_t {
        cudaError_t e = dalloc(b, std::max<size_t>(bytes, 16));
        if (e == cudaSuccess && bytes) e = cudaMemcpy(b.p, h, bytes, cudaMemcpyHostToDevice);
        return e;
    };
    const int n6 = 6 * n_top;
    std::vector<int32_t> pos_leaf(N);
    for (int a = 0; a < n_leaf; ++a)
        for (int k = leaf_ptr[a]; k < leaf_ptr[a + 1]; ++k) pos_leaf[k] = a;
    TF_CK(up(ctx->ml_pos_leaf_d, pos_leaf.data(), sizeof(int32_t) * pos_leaf.size()));
    TF_CK(up(ctx->ml_leaf_ptr_d, leaf_ptr.data(), sizeof(int32_t) * leaf_ptr.size()));
    TF_CK(up(ctx->ml_leaf_nodes_d, leaf_nodes.data(), sizeof(int32_t) * leaf_nodes.size()));
    TF_CK(up(ctx->ml_cen_d, cen.data(), sizeof(double) * cen.size()));
    TF_CK(up(ctx->ml_pstart_d, pstart.data(), sizeof(int32_t) * pstart.size()));
    TF_CK(up(ctx->ml_first_cta_d, first_cta.data(), sizeof(int32_t) * first_cta.size()));
    TF_CK(up(ctx->ml_slot_a_d, slot_a.data(), sizeof(int32_t) * slot_a.size()));
    TF_CK(up(ctx->ml_out_ptr_d, out_ptr.data(), sizeof(int32_t) * out_ptr.size()));
    TF_CK(up(ctx->ml_out_slots_d, out_slots.data(), sizeof(int32_t) * out_slots.size()));
    TF_CK(up(ctx->ml_out_set_d, out_set.data(), sizeof(int32_t) * out_set.size()));
    TF_CK(up(ctx->ml_out_col_d, out_col.data(), sizeof(int32_t) * out_col.size()));
    TF_CK(up(ctx->ml_out_dst_d, out_dst.data(), sizeof(int32_t) * out_dst.size()));
    TF_CK(dalloc(ctx->ml_w_d, sizeof(double) * 36 * (size_t)std::max(n_below, 1)));
    TF_CK(dalloc(ctx->ml_top_d, sizeof(double) * (size_t)n6 * n6));
    TF_CK(dalloc(ctx->ml_top_work, invert_coop_scratch_bytes(n6)));
    TF_CK(dalloc(ctx->ml_info_d, sizeof(int32_t)));
    TF_CK(dalloc(ctx->ml_leaf_m_d, sizeof(double) * 6 * (size_t)n_leaf));
    TF_CK(dalloc(ctx->ml_part_d, sizeof(double) * 6 * (size_t)std::max(pstart[n_sets], 1)));
    // zero once: a CTA without leaves (more CTAs than leaves) never writes its slots
    TF_CK(cudaMemset(ctx->ml_part_d.p, 0, sizeof(double) * 6 * (size_t)std::max(pstart[n_sets], 1)));
    TF_CK(dalloc(ctx->ml_pairs_d, sizeof(double) * 36 * (size_t)std::max(n_slots, 1)));
    if (!ctx->h_coarse_info) TF_CK(cudaMallocHost(&ctx->h_coarse_info, sizeof(int32_t)));
    for (int l = 0; l < kMlMaxLevels; ++l) {
        ctx->ml_span[l] = span[l];
        ctx->ml_count[l] = count[l];
        ctx->ml_set0[l] = set0[l];
    }
    ctx->ml_levels = L;
    ctx->ml_n_leaf = n_leaf;
    ctx->ml_n_slots = n_slots;
    ctx->ml_n_out = (int)out_set.size();
    ctx->ml_n_diag = n_diag;
    ctx->ml_n_top = n_top;
    ctx->ml_nct = nct;
    ctx->n_coarse = 6 * n_sets;
    ctx->ml_active = true;
    ctx->ml_top_ok = false;
    ctx->coarse_age = 0;
    ctx->coarse_ok = false;
    return TF_OK;
}

// The multilevel operators from the current J: leaf-pair blocks, every set's diagonal block and
// its pseudo-inverse, the top operator and its Gauss-Jordan inverse (symmetrised for conjugate
// gradients). A singular top operator leaves the solve with block-Jacobi alone (coarse_ok false).
int ml_setup(tf_ctx* ctx, bool refresh_top) {
    ctx->coarse_ok = false;
    MlSetup m;
    m.n_slots = ctx->ml_n_slots;
    m.n_out = refresh_top ? ctx->ml_n_out : ctx->ml_n_diag;  // the diagonal blocks come first
    m.n_diag = ctx->ml_n_diag;
    m.n_top = ctx->ml_n_top;
    m.slot_a = dptr<int32_t>(ctx->ml_slot_a_d);
    m.slot_agg = dptr<int32_t>(ctx->ca_slot_agg);
    m.slot_ptr = dptr<int32_t>(ctx->ca_slot_ptr);
    m.blk = dptr<int32_t>(ctx->ca_blk);
    m.blk_row = dptr<int32_t>(ctx->ca_blk_row);
    m.node_d = dptr<double>(ctx->node_d);
    m.node_mask = dptr<uint8_t>(ctx->node_mask);
    m.leaf_cen = dptr<double>(ctx->ml_cen_d);
    m.set_cen = dptr<double>(ctx->ml_cen_d);
    m.out_ptr = dptr<int32_t>(ctx->ml_out_ptr_d);
    m.out_slots = dptr<int32_t>(ctx->ml_out_slots_d);
    m.out_set = dptr<int32_t>(ctx->ml_out_set_d);
    m.out_col = dptr<int32_t>(ctx->ml_out_col_d);
    m.out_dst = dptr<int32_t>(ctx->ml_out_dst_d);
    m.pairs = dptr<double>(ctx->ml_pairs_d);
    m.w_blocks = dptr<double>(ctx->ml_w_d);
    m.top = dptr<double>(ctx->ml_top_d);
    m.dflags = dptr<int32_t>(ctx->dflags);
    TF_CK(launch_ml_setup(make_work(ctx), m, refresh_top, ctx->stream));
    ctx->launches += 3;  // pairs, blocks, pinv6
    if (refresh_top) {
        ctx->ml_top_ok = false;
        const int n6 = 6 * ctx->ml_n_top;
        int32_t* info = dptr<int32_t>(ctx->ml_info_d);
        TF_CK(launch_invert_coop(m.top, n6, ctx->ml_top_work.p, info, ctx->device, ctx->stream));
        ctx->launches += 3;  // top fix, Gauss-Jordan, unswap
        TF_CK(cudaMemcpyAsync(ctx->h_coarse_info, info, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
        TF_CK(cudaStreamSynchronize(ctx->stream));
        if (*ctx->h_coarse_info < 0) return set_error(ctx, TF_ERR_STATE, "multilevel top inverse: grid barrier timed out");
        if (*ctx->h_coarse_info != 0) return TF_OK;  // singular top operator: block-Jacobi only
        if (use_cg(ctx)) {
            TF_CK(launch_symmetrize(m.top, n6, n6, 0, 1, ctx->stream));
            ctx->launches += 1;
        }
        ctx->ml_top_ok = true;
        ctx->ml_top_age = 0;
    }
    if (!ctx->ml_top_ok) return TF_OK;
    ctx->coarse_ok = true;
    return TF_OK;
}


int batch_coarse_setup(tf_ctx* ctx) {
    const int T = ctx->T, ld = ctx->bc_ld;
    CoarseAssembly ca;
    ca.n_agg = ctx->n_agg;
    ca.n_coarse = ctx->n_coarse;
    ca.agg_slot_ptr = dptr<int32_t>(ctx->ca_agg_slot_ptr);
    ca.slot_agg = dptr<int32_t>(ctx->ca_slot_agg);
    ca.slot_ptr = dptr<int32_t>(ctx->ca_slot_ptr);
    ca.blk = dptr<int32_t>(ctx->ca_blk);
    ca.blk_row = dptr<int32_t>(ctx->ca_blk_row);
    ca.empty = nullptr;
    ca.n_empty = (int32_t)ctx->bc_n_unit;
    ca.agg_tissue = dptr<int32_t>(ctx->bc_agg_tissue_d);
    ca.tissue_agg0 = dptr<int32_t>(ctx->bc_tissue_agg0_d);
    ca.tissue_base = dptr<int64_t>(ctx->bc_base_d);
    ca.ld = ld;
    ca.empty_offsets = dptr<int64_t>(ctx->bc_unit_d);
    // each tissue's operator is written row-major (transposed, in column-major terms), so the
    // in-place column-major inverse is the row-major inverse the solve reads
    TF_CK(launch_coarse_assemble(make_work(ctx), ca, dptr<double>(ctx->pmode_d), dptr<double>(ctx->coarse_inv),
                                 (size_t)ld * ld * T, ctx->stream));
    int32_t* info = dptr<int32_t>(ctx->bc_info_d);
    TF_CK(launch_invert_batched(dptr<double>(ctx->coarse_inv), dptr<int64_t>(ctx->bc_base_d), dptr<int32_t>(ctx->bc_order_d),
                                ld, T, info, ctx->stream));
    ctx->launches += 2 + (ca.n_empty > 0 ? 1 : 0);
    if (use_cg(ctx)) {  // symmetric J: a symmetric coarse inverse for conjugate gradients
        TF_CK(launch_symmetrize(dptr<double>(ctx->coarse_inv), ld, ld, (long long)ld * ld, T, ctx->stream));
        ctx->launches += 1;
    }
    std::vector<int32_t> h_info(T);
    TF_CK(cudaMemcpyAsync(h_info.data(), info, sizeof(int32_t) * T, cudaMemcpyDeviceToHost, ctx->stream));
    TF_CK(cudaStreamSynchronize(ctx->stream));
    for (int32_t v : h_info)
        if (v != 0) return TF_OK;  // a singular coarse operator: block-Jacobi only
    ctx->coarse_ok = true;
    return TF_OK;
}

// Assemble P^T J P for the current J and invert it; on a singular coarse operator the solve
// runs with block-Jacobi alone (coarse_ok = false).
int coarse_setup(tf_ctx* ctx) {
    ctx->coarse_ok = false;
    if (ctx->bc_active) return batch_coarse_setup(ctx);
    if (ctx->coarse_m == 0) return TF_OK;
    const int nc = ctx->n_coarse;
    CoarseAssembly ca;
    ca.n_agg = ctx->n_agg;
    ca.n_coarse = nc;
    ca.agg_slot_ptr = dptr<int32_t>(ctx->ca_agg_slot_ptr);
    ca.slot_agg = dptr<int32_t>(ctx->ca_slot_agg);
    ca.slot_ptr = dptr<int32_t>(ctx->ca_slot_ptr);
    ca.blk = dptr<int32_t>(ctx->ca_blk);
    ca.blk_row = dptr<int32_t>(ctx->ca_blk_row);
    ca.empty = dptr<int32_t>(ctx->ca_empty);
    ca.n_empty = ctx->n_coarse_empty;
    ca.agg_tissue = nullptr;
    ca.tissue_agg0 = nullptr;
    ca.tissue_base = nullptr;
    ca.ld = nc;
    ca.empty_offsets = nullptr;
    double* inv = dptr<double>(ctx->coarse_inv);
    int32_t* info = dptr<int32_t>(ctx->coarse_info);
    // P^T J P written row-major, inverted in place (column-major terms): the row-major inverse
    TF_CK(launch_coarse_assemble(make_work(ctx), ca, dptr<double>(ctx->pmode_d), inv, (size_t)nc * nc, ctx->stream));
    TF_CK(launch_invert_coop(inv, nc, ctx->coarse_work.p, info, ctx->device, ctx->stream));
    ctx->launches += 3 + (ca.n_empty > 0 ? 1 : 0);
    TF_CK(cudaMemcpyAsync(ctx->h_coarse_info, info, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    TF_CK(cudaStreamSynchronize(ctx->stream));
    if (*ctx->h_coarse_info < 0) return set_error(ctx, TF_ERR_STATE, "coarse inverse: grid barrier timed out");
    if (*ctx->h_coarse_info != 0) return TF_OK;  // singular: block-Jacobi only
    if (use_cg(ctx)) {  // symmetric J: a symmetric coarse inverse for conjugate gradients
        TF_CK(launch_symmetrize(inv, nc, nc, 0, 1, ctx->stream));
        ctx->launches += 1;
    }
    ctx->coarse_ok = true;
    return TF_OK;
}

bool use_persistent(tf_ctx* ctx) {
    return (ctx->params.precond == TF_PRECOND_BLOCK_JACOBI || ctx->params.precond == TF_PRECOND_TWO_LEVEL ||
            ctx->params.precond == TF_PRECOND_MULTILEVEL) &&
           ctx->persistent_grid_max > 0 && (ctx->params.persistent || ctx->T > 1);
}

// Solve J du = g (buffers in the context) for every active tissue. Leaves the scalars in
// ctx->h_tsc[T] (persistent) or ctx->h_sc (chunked, single tissue).
int krylov_solve(tf_ctx* ctx) {
    KrylovWork w = make_work(ctx);
    if (use_persistent(ctx)) {
        if (ctx->params.precond == TF_PRECOND_TWO_LEVEL || ctx->params.precond == TF_PRECOND_MULTILEVEL) {
            if (ctx->ml_active && (ctx->plan_ncta.empty() || ctx->plan_ncta[0] != ctx->ml_nct))
                ctx->coarse_dirty = true;  // the CTA split changed: lay the partial slots out again
        }
        if ((ctx->params.precond == TF_PRECOND_TWO_LEVEL || ctx->params.precond == TF_PRECOND_MULTILEVEL) &&
            !ctx->reuse_precond) {
            if (ctx->coarse_dirty) {
                const int crc = build_coarse(ctx);
                if (crc != TF_OK) return crc;
            }
            // The coarse operator is refreshed from the current J when it is missing, after
            // kCoarseMaxAge solves, or when the last solve needed 1.3x the iterations of the
            // first solve after the refresh; in between the previous inverse preconditions (any
            // fixed operator is a valid preconditioner: convergence is tested on the residual).
            const bool stale = !ctx->coarse_ok || ctx->coarse_age >= kCoarseMaxAge ||
                               (ctx->coarse_age > 1 && ctx->last_solve_iters * 10 > ctx->coarse_base_iters * 13);
            if ((ctx->coarse_m > 0 || ctx->bc_active) && stale) {
                const int crc = coarse_setup(ctx);
                if (crc != TF_OK) return crc;
                ctx->coarse_age = 0;
                ++ctx->coarse_refreshes;
            }
            // the multilevel operators are rebuilt from every J (a few set-up kernels, about one
            // SpMV of traffic): an operator kept from an indefinite first Newton iterate would
            // leave conjugate gradients an indefinite preconditioner for the positive definite rest
            // (The dense top inverse, a Gauss-Jordan elimination with one grid barrier per step,
            // is the expensive part: it is refreshed on the first solve, after kMlTopMaxAge solves,
            // after a solve needed 1.3x the iterations of the first one since the refresh, and
            // after conjugate gradients met an indefinite system, since a top inverse taken from
            // an indefinite J would stay indefinite for the positive definite ones that follow.)
            if (ctx->ml_active) {
                const bool top = !ctx->ml_top_ok || ctx->ml_top_age >= kMlTopMaxAge || ctx->last_solve_method == KM_CG_FALLBACK ||
                                 (ctx->ml_top_age > 1 && ctx->last_solve_iters * 10 > ctx->coarse_base_iters * 13);
                const int crc = ml_setup(ctx, top);
                if (crc != TF_OK) return crc;
                ++ctx->coarse_refreshes;
                if (top) ctx->ml_top_fresh = true;
            }
        }
        BatchPlan plan = make_plan(ctx);
        // Warm start (tf_params.krylov_warm_start): inside the Newton loop of a single tissue,
        // conjugate gradients start from the solution of the same Newton iteration of the last
        // step that reached it, with its true residual r0 = g - J x0 (the kernel falls back to
        // x0 = 0 when ||r0|| is not below ||g||). Consecutive steps grow the tissue by similar
        // increments, so ||r0|| is 0.06-0.5 of ||g|| on the first three Newton iterations of a
        // slab. Not for the lumen's second solve (another right-hand side) or MINRES.
        const size_t bytes3 = sizeof(double) * 3 * (size_t)ctx->N;
        const int wk = ctx->warm_k;
        const bool warm_slot = ctx->params.krylov_warm_start && ctx->T == 1 && plan.cg && !plan.minres &&
                               !ctx->reuse_precond && wk >= 0 && wk < kWarmSlots;
        if (warm_slot && wk < (int)ctx->warm_valid.size() && ctx->warm_valid[wk]) {
            TF_CK(cudaMemcpyAsync(ctx->du.p, ctx->warm_hist[wk].p, bytes3, cudaMemcpyDeviceToDevice, ctx->stream));
            TF_CK(launch_residual(w, dptr<double>(ctx->du), dptr<double>(ctx->g), dptr<double>(ctx->r), ctx->stream));
            ctx->launches += 1;
            plan.warm = 1;
        }
        if (plan.group > 1) {
            TF_CK(launch_group_jacobi_setup(w, plan.group, ctx->stream));
            ctx->launches += 1;
        }
        TF_CK(cudaMemsetAsync(ctx->queue_head_d.p, 0, sizeof(int32_t), ctx->stream));
        TF_CK(cudaEventRecord(ctx->ev_solve[0], ctx->stream));
        TF_CK(launch_bicgstab_batched(w, plan, ctx->params.krylov_rtol, ctx->params.krylov_max_iters,
                                      ctx->persist_threads, ctx->stream));
        TF_CK(cudaEventRecord(ctx->ev_solve[1], ctx->stream));
        ctx->launches += 1;
        TF_CK(cudaMemcpyAsync(ctx->h_tsc, ctx->tscalars.p, sizeof(KrylovScalars) * ctx->T, cudaMemcpyDeviceToHost,
                              ctx->stream));
        TF_CK(cudaMemcpyAsync(ctx->h_flags, ctx->dflags.p, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
        TF_CK(cudaStreamSynchronize(ctx->stream));
        {
            float kms = 0.0f;
            TF_CK(cudaEventElapsedTime(&kms, ctx->ev_solve[0], ctx->ev_solve[1]));
            ctx->solve_kernel_ms += kms;
            ctx->solve_kernel_launches += 1;
        }
        if (*ctx->h_flags & DF_BARRIER_TIMEOUT) {
            TF_CK(cudaMemsetAsync(ctx->tbarriers.p, 0, sizeof(GridBarrier) * ctx->T, ctx->stream));
            TF_CK(cudaMemsetAsync(ctx->dflags.p, 0, sizeof(int32_t), ctx->stream));
            return set_error(ctx, TF_ERR_STATE, "persistent solve: grid barrier timed out");
        }
        if (plan.cg) {
            // Tissues whose conjugate gradients met a non-positive curvature (J indefinite: e.g.
            // the growth's compressive prestress outweighing the drag on a rigid in-plane rotation)
            // are finished by BiCGStab in a second launch with only them active, starting from the
            // iterate and residual CG reached; the others keep their CG result.
            std::vector<int32_t> redo(ctx->T, 0), cg_iters(ctx->T, 0);
            bool any = false;
            for (int t = 0; t < ctx->T; ++t)
                if ((ctx->T == 1 || ctx->h_active[t]) && ctx->h_tsc[t].status == KS_INDEFINITE) {
                    redo[t] = any = 1;
                    cg_iters[t] = ctx->h_tsc[t].iter;
                }
            if (any) {
                BatchPlan p2 = plan;
                p2.cg = 0;
                p2.warm = 1;
                TF_CK(cudaMemcpyAsync(ctx->active_d.p, redo.data(), sizeof(int32_t) * ctx->T, cudaMemcpyHostToDevice,
                                      ctx->stream));
                TF_CK(cudaMemsetAsync(ctx->queue_head_d.p, 0, sizeof(int32_t), ctx->stream));
                TF_CK(cudaEventRecord(ctx->ev_solve[0], ctx->stream));
                TF_CK(launch_bicgstab_batched(w, p2, ctx->params.krylov_rtol, ctx->params.krylov_max_iters,
                                              ctx->persist_threads, ctx->stream));
                TF_CK(cudaEventRecord(ctx->ev_solve[1], ctx->stream));
                ctx->launches += 1;
                TF_CK(cudaMemcpyAsync(ctx->active_d.p, ctx->h_active, sizeof(int32_t) * ctx->T, cudaMemcpyHostToDevice,
                                      ctx->stream));  // the Newton loop's active tissues again
                TF_CK(cudaMemcpyAsync(ctx->h_tsc, ctx->tscalars.p, sizeof(KrylovScalars) * ctx->T, cudaMemcpyDeviceToHost,
                                      ctx->stream));
                TF_CK(cudaMemcpyAsync(ctx->h_flags, ctx->dflags.p, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
                TF_CK(cudaStreamSynchronize(ctx->stream));
                float kms = 0.0f;
                TF_CK(cudaEventElapsedTime(&kms, ctx->ev_solve[0], ctx->ev_solve[1]));
                ctx->solve_kernel_ms += kms;
                ctx->solve_kernel_launches += 1;
                if (*ctx->h_flags & DF_BARRIER_TIMEOUT) {
                    TF_CK(cudaMemsetAsync(ctx->tbarriers.p, 0, sizeof(GridBarrier) * ctx->T, ctx->stream));
                    TF_CK(cudaMemsetAsync(ctx->dflags.p, 0, sizeof(int32_t), ctx->stream));
                    return set_error(ctx, TF_ERR_STATE, "persistent solve: grid barrier timed out");
                }
                for (int t = 0; t < ctx->T; ++t)
                    if (redo[t]) {
                        ctx->h_tsc[t].method = KM_CG_FALLBACK;
                        ctx->h_tsc[t].iter += cg_iters[t];  // iterations of both methods
                        ctx->cg_iters += cg_iters[t];
                    }
            }
        }
        *ctx->h_sc = ctx->h_tsc[0];
        if (warm_slot && ctx->h_tsc[0].status == KS_CONVERGED) {
            if ((int)ctx->warm_hist.size() <= wk) {
                ctx->warm_hist.resize(wk + 1);
                ctx->warm_valid.resize(wk + 1, 0);
            }
            if (dalloc(ctx->warm_hist[wk], bytes3) == cudaSuccess) {
                TF_CK(cudaMemcpyAsync(ctx->warm_hist[wk].p, ctx->du.p, bytes3, cudaMemcpyDeviceToDevice, ctx->stream));
                ctx->warm_valid[wk] = 1;
            } else {
                (void)cudaGetLastError();  // no room for the history: this iteration keeps starting from zero
            }
        }
        for (int t = 0; t < ctx->T; ++t)
            if (ctx->T == 1 || ctx->h_active[t]) {
                ctx->last_method = std::max(ctx->last_method, ctx->h_tsc[t].method);
                if (ctx->h_tsc[t].method == KM_CG) ctx->cg_iters += ctx->h_tsc[t].iter;
            }
        ctx->last_solve_iters = 0;
        for (int t = 0; t < ctx->T; ++t)
            if (ctx->T == 1 || ctx->h_active[t]) ctx->last_solve_iters = std::max(ctx->last_solve_iters, ctx->h_tsc[t].iter);
        if ((ctx->coarse_m > 0 || ctx->bc_active) && ctx->coarse_ok) {
            if (ctx->coarse_age == 0) ctx->coarse_base_iters = ctx->last_solve_iters;
            ++ctx->coarse_age;
        }
        ctx->last_solve_method = 0;
        for (int t = 0; t < ctx->T; ++t)
            if (ctx->T == 1 || ctx->h_active[t]) ctx->last_solve_method = std::max(ctx->last_solve_method, ctx->h_tsc[t].method);
        if (ctx->ml_active && ctx->coarse_ok) {
            if (ctx->ml_top_fresh) ctx->coarse_base_iters = ctx->last_solve_iters;
            ctx->ml_top_fresh = false;
            ++ctx->ml_top_age;
        }
        return TF_OK;
    }
    ctx->last_method = std::max<int32_t>(ctx->last_method, KM_BICGSTAB);  // graph-replayed iterations: BiCGStab
    const bool ilu = ctx->params.precond == TF_PRECOND_ILU0;
    if (ilu) {
        TF_CK(cudaMemcpyAsync(ctx->ilu_lu.p, ctx->vals.p, sizeof(double) * 9 * (size_t)ctx->nnzb, cudaMemcpyDeviceToDevice,
                              ctx->stream));
        TF_CK(launch_ilu_factor(w, make_ilu(ctx), ctx->stream));
        ctx->launches += ctx->ilu_colours;
    } else {
        TF_CK(launch_block_jacobi_setup(w, ctx->stream));
        ctx->launches += 1;
    }
    TF_CK(launch_krylov_init(w, ctx->params.krylov_rtol, ctx->params.krylov_max_iters, ctx->stream));
    ctx->launches += 1;
    if (ilu) {
        const IluPlan ip = make_ilu(ctx);
        if (ctx->params.use_graphs && !ctx->ilu_graph) {
            cudaGraph_t graph;
            TF_CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            for (int i = 0; i < kChunk; ++i) launch_bicgstab_iteration_ilu(w, ip, ctx->stream);
            cudaError_t cerr = cudaStreamEndCapture(ctx->stream, &graph);
            TF_CK(cerr);
            cerr = cudaGraphInstantiate(&ctx->ilu_graph, graph, 0);
            cudaGraphDestroy(graph);
            TF_CK(cerr);
        }
        const int max_chunks = ctx->params.krylov_max_iters / kChunk + 2;
        for (int ch = 0; ch < max_chunks; ++ch) {
            if (ctx->params.use_graphs)
                TF_CK(cudaGraphLaunch(ctx->ilu_graph, ctx->stream));
            else
                for (int i = 0; i < kChunk; ++i) TF_CK(launch_bicgstab_iteration_ilu(w, ip, ctx->stream));
            ctx->launches += (int64_t)kChunk * (5 + 4 * ctx->ilu_colours);
            TF_CK(cudaMemcpyAsync(ctx->h_sc, ctx->sc.p, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, ctx->stream));
            TF_CK(cudaStreamSynchronize(ctx->stream));
            if (ctx->h_sc->status != KS_RUNNING) break;
        }
        return TF_OK;
    }
    if (ctx->params.use_graphs && !ctx->krylov_graph) {
        cudaGraph_t graph;
        TF_CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < kChunk; ++i) launch_bicgstab_iteration(w, ctx->stream);
        cudaError_t cerr = cudaStreamEndCapture(ctx->stream, &graph);
        TF_CK(cerr);
        cerr = cudaGraphInstantiate(&ctx->krylov_graph, graph, 0);
        cudaGraphDestroy(graph);
        TF_CK(cerr);
    }
    const int max_chunks = ctx->params.krylov_max_iters / kChunk + 2;
    for (int ch = 0; ch < max_chunks; ++ch) {
        if (ctx->params.use_graphs) {
            TF_CK(cudaGraphLaunch(ctx->krylov_graph, ctx->stream));
        } else {
            for (int i = 0; i < kChunk; ++i) TF_CK(launch_bicgstab_iteration(w, ctx->stream));
        }
        ctx->launches += 5 * kChunk;
        TF_CK(cudaMemcpyAsync(ctx->h_sc, ctx->sc.p, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, ctx->stream));
        TF_CK(cudaStreamSynchronize(ctx->stream));
        if (ctx->h_sc->status != KS_RUNNING) break;
    }
    return TF_OK;
}

int read_flags(tf_ctx* ctx) {
    TF_CK(cudaMemcpyAsync(ctx->h_flags, ctx->dflags.p, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    TF_CK(cudaStreamSynchronize(ctx->stream));
    return TF_OK;
}

// Most severe of two outcomes: errors first, then non-finite values, then the rest by code.
int worse(int a, int b) {
    if (a < 0 || b < 0) return std::min(a, b);
    if (a == TF_NONFINITE || b == TF_NONFINITE) return TF_NONFINITE;
    return std::max(a, b);
}

// Newton loop on device buffers: un holds x_n; result left in uk.
// Newton loop on device buffers: un holds x_n; result left in uk. Every tissue of a batch
// follows Simulation::updateStepNR on its own: it stops once its ||du||_2 <= tol
// (checkConvergenceViaDeltaU, NewtonRaphsonSolver.cpp:807-825) or after more than
// max_newton_iters iterations (Simulation.cpp:6724-6727), the last update applied either way;
// tissues that stopped are skipped by the assembly, the solve and the update.
int newton_core(tf_ctx* ctx, double dt, tf_step_stats* st) {
    const int T = ctx->T;
    TF_CK(cudaMemcpyAsync(ctx->uk.p, ctx->un.p, sizeof(double) * 3 * (size_t)ctx->N, cudaMemcpyDeviceToDevice, ctx->stream));
    TF_CK(cudaMemsetAsync(ctx->dflags.p, 0, sizeof(int32_t), ctx->stream));
    ctx->t_iters.assign(T, 0);
    ctx->t_status.assign(T, TF_OK);
    ctx->t_krylov.assign(T, 0);
    for (int t = 0; t < T; ++t) ctx->h_active[t] = 1;
    const bool persistent = use_persistent(ctx);
    int n_active = T;
    int round = 0;
    float ms;
    std::vector<double> weight = rows_weight(ctx);
    if (T > 1 && ctx->last_krylov.size() == (size_t)T)
        for (int t = 0; t < T; ++t)
            weight[t] = (ctx->tissue_node0[t + 1] - ctx->tissue_node0[t]) * std::max(8.0, (double)ctx->last_krylov[t]);
    ctx->last_krylov.assign(T, 0);
    if (T > 1 && persistent && ctx->params.precond == TF_PRECOND_TWO_LEVEL && ctx->coarse_dirty) {
        const int crc = build_coarse(ctx);  // the batch plan gives every CTA whole aggregates
        if (crc != TF_OK) return crc;
    }
    while (n_active > 0) {
        if (T > 1 && persistent) {
            int rc = build_plan(ctx, weight, ctx->h_active);
            if (rc != TF_OK) return rc;
        }
        TF_CK(cudaMemcpyAsync(ctx->active_d.p, ctx->h_active, sizeof(int32_t) * T, cudaMemcpyHostToDevice, ctx->stream));
        TF_CK(cudaEventRecord(ctx->ev[1], ctx->stream));
        int rc = assemble_system(ctx, dt);
        if (rc != TF_OK) return rc;
        TF_CK(cudaEventRecord(ctx->ev[2], ctx->stream));
        ctx->warm_k = ctx->warm_call && T == 1 ? ctx->t_iters[0] : -1;
        rc = newton_solve(ctx);
        ctx->warm_k = -1;
        if (rc != TF_OK) return rc;
        KrylovWork w = make_work(ctx);
        if (persistent) {
            TF_CK(launch_newton_update_batched(w, make_plan(ctx), dptr<double>(ctx->uk), dptr<int32_t>(ctx->slaves_d),
                                               dptr<int32_t>(ctx->masters_d), (int32_t)ctx->slave.size(), ctx->stream));
            TF_CK(cudaMemcpyAsync(ctx->h_du2, ctx->tdu2.p, sizeof(double) * T, cudaMemcpyDeviceToHost, ctx->stream));
        } else {
            *ctx->h_tsc = *ctx->h_sc;
            TF_CK(launch_newton_update(w, dptr<double>(ctx->uk), dptr<int32_t>(ctx->slaves_d), dptr<int32_t>(ctx->masters_d),
                                       (int32_t)ctx->slave.size(), ctx->stream));
            TF_CK(cudaMemcpyAsync(ctx->h_sc, ctx->sc.p, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, ctx->stream));
        }
        ctx->launches += ctx->slave.empty() ? 1 : 2;
        TF_CK(cudaEventRecord(ctx->ev[3], ctx->stream));
        rc = read_flags(ctx);
        if (rc != TF_OK) return rc;
        if (!persistent) ctx->h_du2[0] = ctx->h_sc->du2;
        TF_CK(cudaEventElapsedTime(&ms, ctx->ev[1], ctx->ev[2]));
        st->ms_assemble += ms;
        TF_CK(cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]));
        st->ms_solve += ms;
        if (*ctx->h_flags & DF_PATTERN_MISS) return set_error(ctx, TF_ERR_STATE, "routed entry outside the pattern");
        int flag_status = TF_OK;
        if (*ctx->h_flags & DF_NONFINITE)
            flag_status = TF_NONFINITE;
        else if (*ctx->h_flags & DF_INVERTED)
            flag_status = TF_ELEMENT_INVERTED;
        double dmax = 0.0, relmax = 0.0;
        int kit_max = 0;
        for (int t = 0; t < T; ++t) {
            if (!ctx->h_active[t]) continue;
            const KrylovScalars& sc = ctx->h_tsc[t];
            const int ks = krylov_status_to_tf(sc.status);
            if (ks != TF_OK) ctx->t_status[t] = worse(ctx->t_status[t], ks);
            if (flag_status != TF_OK) ctx->t_status[t] = worse(ctx->t_status[t], flag_status);
            ctx->t_krylov[t] += sc.iter;
            st->krylov_iters_total += sc.iter;
            weight[t] = (ctx->tissue_node0[t + 1] - ctx->tissue_node0[t]) * std::max(8.0, (double)sc.iter);
            if (round == 0) ctx->last_krylov[t] = sc.iter;
            kit_max = std::max(kit_max, sc.iter);
            const double d = std::sqrt(ctx->h_du2[t]);
            dmax = std::max(dmax, std::isfinite(d) ? d : INFINITY);
            relmax = std::max(relmax, sc.bb > 0 ? std::sqrt(sc.rr / sc.bb) : 0.0);
            ctx->t_iters[t]++;
            bool done;
            if (!std::isfinite(d)) {
                ctx->t_status[t] = worse(ctx->t_status[t], TF_NONFINITE);
                done = true;
            } else {
                done = !(d > ctx->params.newton_tol);
                if (!done && ctx->t_iters[t] > ctx->params.max_newton_iters) {
                    ctx->t_status[t] = worse(ctx->t_status[t], TF_NEWTON_NOT_CONVERGED);
                    done = true;
                }
            }
            if (done) {
                ctx->h_active[t] = 0;
                --n_active;
            }
        }
        st->krylov_iters_max = std::max(st->krylov_iters_max, kit_max);
        if (round < 32) {
            st->du_norm[round] = dmax;
            st->krylov_rel_res[round] = relmax;
        }
        ++round;
    }
    int status = TF_OK;
    for (int t = 0; t < T; ++t) status = worse(status, ctx->t_status[t]);
    st->newton_iters = round;
    st->status = status;
    return status;
}

// Bracket a public call: reset the stats and the launch counter, record the start event.
int call_begin(tf_ctx* ctx, tf_step_stats* st) {
    std::memset(st, 0, sizeof(*st));
    ctx->launches = 0;
    ctx->last_method = 0;
    ctx->cg_iters = 0;
    ctx->solve_kernel_ms = 0.0;
    ctx->solve_kernel_launches = 0;
    TF_CK(cudaEventRecord(ctx->ev_call[0], ctx->stream));
    return TF_OK;
}

int call_end(tf_ctx* ctx, tf_step_stats* st) {
    TF_CK(cudaEventRecord(ctx->ev_call[1], ctx->stream));
    TF_CK(cudaEventSynchronize(ctx->ev_call[1]));
    float ms = 0.0f;
    TF_CK(cudaEventElapsedTime(&ms, ctx->ev_call[0], ctx->ev_call[1]));
    st->ms_total = ms;
    st->gpu_launches = ctx->launches;
    st->ms_solve_kernel = ctx->solve_kernel_ms;
    st->solve_launches = ctx->solve_kernel_launches;
    st->krylov_method = ctx->last_method;
    st->krylov_iters_cg = (int32_t)std::min<int64_t>(ctx->cg_iters, INT32_MAX);
    return TF_OK;
}

// The growth prologue of a step at the context's simulation time: the grid-based functions active
// then (InitialTime <= t < FinalTime, Simulation.cpp:9041) give a per-element increment, applied
// after the uniform one; then the growth update and the exposed areas.
// The Newton system's solve: J du = g, and with a lumen (J + a G G^T) du = g by Sherman-Morrison
// from two solves with the sparse J: y = J^-1 g, z = J^-1 G, du = y - a (G.y) / (1 + a G.z) z,
// a = bulk / (36 V0^2) (the rank-one term of Lumen::calculateJacobian couples every lumen node,
// so it stays out of the sparse J). The second solve reuses the first one's preconditioner; the
// scalars left for the Newton loop carry both solves' iterations and the worse status.
int newton_solve(tf_ctx* ctx) {
    int rc = krylov_solve(ctx);
    if (rc != TF_OK || !ctx->lm_on) return rc;
    const size_t bytes = sizeof(double) * 3 * (size_t)ctx->N;
    const KrylovScalars first = ctx->h_tsc[0];
    TF_CK(cudaMemcpyAsync(ctx->lm_y_d.p, ctx->du.p, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    TF_CK(cudaMemcpyAsync(ctx->lm_gsave_d.p, ctx->g.p, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    TF_CK(cudaMemcpyAsync(ctx->g.p, ctx->lm_G_d.p, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    ctx->reuse_precond = true;
    rc = krylov_solve(ctx);
    ctx->reuse_precond = false;
    if (rc != TF_OK) return rc;
    TF_CK(cudaMemcpyAsync(ctx->lm_z_d.p, ctx->du.p, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    TF_CK(launch_dot2(3 * ctx->N, dptr<double>(ctx->lm_G_d), dptr<double>(ctx->lm_y_d), dptr<double>(ctx->lm_z_d),
                      dptr<double>(ctx->lm_dot_part_d), dptr<double>(ctx->lm_dots_d), ctx->stream));
    ctx->launches += 2;
    TF_CK(cudaMemcpyAsync(ctx->h_lm_dots, ctx->lm_dots_d.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    TF_CK(cudaStreamSynchronize(ctx->stream));
    const double a = ctx->lm_bulk / (36.0 * ctx->lm_ideal * ctx->lm_ideal);
    const double coef = a * ctx->h_lm_dots[0] / (1.0 + a * ctx->h_lm_dots[1]);
    TF_CK(cudaMemcpyAsync(ctx->du.p, ctx->lm_y_d.p, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    TF_CK(launch_axpy(3 * ctx->N, -coef, dptr<double>(ctx->lm_z_d), dptr<double>(ctx->du), ctx->stream));
    TF_CK(cudaMemcpyAsync(ctx->g.p, ctx->lm_gsave_d.p, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    ctx->launches += 1;
    KrylovScalars& sc = ctx->h_tsc[0];
    const KrylovScalars second = sc;
    sc = first;
    sc.iter = first.iter + second.iter;
    if (second.status != KS_CONVERGED) sc.status = second.status;
    *ctx->h_sc = sc;
    if (!std::isfinite(coef)) return set_error(ctx, TF_ERR_STATE, "lumen: 1 + a G.z vanished");
    return TF_OK;
}

int prologue(tf_ctx* ctx, double dt) {
    const double* grid_inc = nullptr;
    GridStep gs;
    std::memset(&gs, 0, sizeof(gs));
    gs.interpolation = ctx->grid_interp;
    gs.dt = dt;
    for (const auto& gf : ctx->grid_funcs) {
        if (!(ctx->sim_time >= gf.t0 && ctx->sim_time < gf.t1)) continue;
        if (gs.n >= kMaxGridFuncs) return set_error(ctx, TF_ERR_UNSUPPORTED, "more than 8 grid growth functions in a step");
        GridFunc& f = gs.f[gs.n++];
        f.cells = static_cast<const GridCell*>(gf.cells.p);
        f.nx = gf.nx;
        f.ny = gf.ny;
        f.zmin = gf.zmin;
        f.zmax = gf.zmax;
        f.flags = gf.flags;
    }
    if (gs.n > 0) {
        TF_CK(launch_grid_increment(ctx->E, gs, dptr<double>(ctx->grid_rel_pos), dptr<double>(ctx->grid_rel_z),
                                    dptr<int32_t>(ctx->grid_eflags), dptr<double>(ctx->grid_inc), ctx->stream));
        grid_inc = dptr<double>(ctx->grid_inc);
        ctx->launches += 1;
    }
    TF_CK(launch_grow(dptr<ElemRecord>(ctx->elems), ctx->E, dptr<double>(ctx->un), dptr<double>(ctx->fg),
                      dptr<double>(ctx->rates), dptr<double>(ctx->angles), dt, dptr<int32_t>(ctx->rotated), grid_inc,
                      ctx->stream));
    TF_CK(launch_viscosity_surface(dptr<ElemRecord>(ctx->elems), ctx->E, ctx->N, dptr<double>(ctx->un),
                                   dptr<uint8_t>(ctx->exposed), dptr<uint8_t>(ctx->peripodial),
                                   dptr<double>(ctx->visc_surface), ctx->stream));
    ctx->launches += 2;
    if (ctx->lm_on) {  // Lumen::growLumen(currSimTimeSec + dt) (Simulation.cpp:6019, Lumen.cpp:331-334)
        ctx->lm_ideal = ctx->lm_v_init * std::exp(ctx->lm_rate * (ctx->sim_time + dt));
        TF_CK(launch_lumen_set_ideal(dptr<LumenState>(ctx->lm_state_d), ctx->lm_ideal, ctx->stream));
        ctx->launches += 1;
    }
    if (ctx->pk_on) return packing_detect(ctx, dptr<double>(ctx->un));  // after the growth (Simulation.cpp:6065-6076)
    return TF_OK;
}

// Mark every tissue active on the device (the parity hooks and timers act on all tissues).
int activate_all(tf_ctx* ctx) {
    for (int t = 0; t < ctx->T; ++t) ctx->h_active[t] = 1;
    TF_CK(cudaMemcpyAsync(ctx->active_d.p, ctx->h_active, sizeof(int32_t) * ctx->T, cudaMemcpyHostToDevice, ctx->stream));
    return ctx->T > 1 ? build_plan_all(ctx) : TF_OK;
}

int check_ctx(tf_ctx* ctx) {
    if (!ctx) return TF_ERR_ARGUMENT;
    cudaError_t err = cudaSetDevice(ctx->device);
    if (err != cudaSuccess) return set_error(ctx, TF_ERR_CUDA, cudaGetErrorString(err));
    return TF_OK;
}

// Per-element field setter: writes `ncomp` doubles at byte offset `off` of every record.
int set_record_field(tf_ctx* ctx, size_t off, int ncomp, const double* src) {
    std::vector<ElemRecord> rec(ctx->E);
    TF_CK(cudaMemcpy(rec.data(), ctx->elems.p, sizeof(ElemRecord) * (size_t)ctx->E, cudaMemcpyDeviceToHost));
    for (int e = 0; e < ctx->E; ++e)
        std::memcpy(reinterpret_cast<char*>(&rec[e]) + off, src + (size_t)e * ncomp, sizeof(double) * ncomp);
    TF_CK(cudaMemcpy(ctx->elems.p, rec.data(), sizeof(ElemRecord) * (size_t)ctx->E, cudaMemcpyHostToDevice));
    return TF_OK;
}

}  // namespace

extern "C" {

void tf_default_params(tf_params* p) {
    if (!p) return;
    p->max_newton_iters = 20;
    p->newton_tol = 1e-8;
    p->krylov_max_iters = 20000;
    p->krylov_rtol = 1e-12;
    p->precond = TF_PRECOND_TWO_LEVEL;
    p->scatter = TF_SCATTER_AUTO;
    p->elems_per_block = 0;
    p->device = 0;
    p->use_graphs = 1;
    p->persistent = 1;
    p->smoother_nodes = 0;
    p->krylov_refine = 0;
    p->krylov_method = TF_KRYLOV_AUTO;
    p->krylov_warm_start = 1;
}

const char* tf_version(void) { return "tissueorigami_b200 0.1 (sm_100a, FP64)"; }

struct CtxDeleter {
    void operator()(tf_ctx* c) const { tf_destroy(c); }
};

// Create a context over one mesh whose nodes and elements are split into T consecutive
// tissues (node0 / elem0 hold T+1 offsets); T = 1 is the single-tissue context.
// Nodes per prism column when the mesh numbers every column's nodes consecutively (all G nodes
// of each group 0..G-1, G..2G-1, ... at the same reference x, y), trying G = 4, 3, 2; else 1.
int column_size(tf_ctx* ctx) {
    const int N = ctx->N;
    std::vector<double> X((size_t)N * 3, 0.0);
    for (int e = 0; e < ctx->E; ++e)
        for (int a = 0; a < 6; ++a)
            for (int d = 0; d < 3; ++d) X[(size_t)ctx->conn[(size_t)e * 6 + a] * 3 + d] = ctx->xref[(size_t)e * 18 + a * 3 + d];
    double scale = 0.0;
    for (double v : X) scale = std::max(scale, std::fabs(v));
    const double tol = 1e-9 * std::max(scale, 1.0);
    for (int G = 4; G >= 2; --G) {
        if (N % G != 0) continue;
        bool ok = true;
        for (int g = 0; g < N / G && ok; ++g)
            for (int j = 1; j < G && ok; ++j) {
                const size_t a = (size_t)g * G, b = a + j;
                ok = std::fabs(X[a * 3] - X[b * 3]) <= tol && std::fabs(X[a * 3 + 1] - X[b * 3 + 1]) <= tol;
            }
        if (ok) return G;
    }
    return 1;
}

static int create_ctx(const tf_mesh_desc* mesh, const tf_params* params, int32_t T, const int32_t* node0,
                      const int32_t* elem0, tf_ctx** out) {
    if (!out) return TF_ERR_ARGUMENT;
    *out = nullptr;
    if (!mesh || mesh->n_nodes <= 0 || mesh->n_elems <= 0 || !mesh->conn || !mesh->xref || T <= 0) return TF_ERR_ARGUMENT;
    for (int t = 0; t < T; ++t)
        for (int e = elem0[t]; e < elem0[t + 1]; ++e)
            for (int a = 0; a < 6; ++a) {
                const int32_t v = mesh->conn[(int64_t)e * 6 + a];
                if (v < node0[t] || v >= node0[t + 1]) return TF_ERR_ARGUMENT;
            }
    std::unique_ptr<tf_ctx, CtxDeleter> holder(new (std::nothrow) tf_ctx());
    // on failure, keep the context's last message for tf_last_error(NULL) before it is destroyed
    struct KeepMessage {
        std::unique_ptr<tf_ctx, CtxDeleter>& h;
        ~KeepMessage() {
            if (h) std::snprintf(g_create_error, sizeof(g_create_error), "%s", h->last_error);
        }
    } keep{holder};
    g_create_error[0] = 0;
    tf_ctx* ctx = holder.get();
    if (!ctx) return TF_ERR_OUT_OF_MEMORY;
    ctx->T = T;
    ctx->tissue_node0.assign(node0, node0 + T + 1);
    ctx->tissue_elem0.assign(elem0, elem0 + T + 1);
    if (params)
        ctx->params = *params;
    else
        tf_default_params(&ctx->params);
    // the two-level preconditioner runs in the persistent solve (which a batch always uses); a
    // single tissue solved in chunks stands down to block-Jacobi
    // a batch takes the multilevel choice as two-level (its own per-tissue coarse space)
    if (ctx->params.precond == TF_PRECOND_MULTILEVEL && T > 1) ctx->params.precond = TF_PRECOND_TWO_LEVEL;
    if ((ctx->params.precond == TF_PRECOND_TWO_LEVEL || ctx->params.precond == TF_PRECOND_MULTILEVEL) && T == 1 &&
        !ctx->params.persistent)
        ctx->params.precond = TF_PRECOND_BLOCK_JACOBI;
    if (ctx->params.precond != TF_PRECOND_BLOCK_JACOBI && !(ctx->params.precond == TF_PRECOND_ILU0 && T == 1) &&
        ctx->params.precond != TF_PRECOND_TWO_LEVEL && ctx->params.precond != TF_PRECOND_MULTILEVEL)
        return TF_ERR_UNSUPPORTED;
    if (ctx->params.krylov_max_iters <= 0 || ctx->params.max_newton_iters < 0) return TF_ERR_ARGUMENT;
    ctx->device = ctx->params.device;
    TF_CK(cudaSetDevice(ctx->device));
    TF_CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    for (auto& e : ctx->ev) TF_CK(cudaEventCreate(&e));
    for (auto& e : ctx->ev_call) TF_CK(cudaEventCreate(&e));
    for (auto& e : ctx->ev_solve) TF_CK(cudaEventCreate(&e));
    ctx->N = mesh->n_nodes;
    ctx->E = mesh->n_elems;
    ctx->conn.assign(mesh->conn, mesh->conn + (size_t)ctx->E * 6);
    ctx->xref.assign(mesh->xref, mesh->xref + (size_t)ctx->E * 18);
    ctx->dofmap.resize((size_t)ctx->N * 3);
    for (size_t i = 0; i < ctx->dofmap.size(); ++i) ctx->dofmap[i] = (int32_t)i;
    const size_t n3 = (size_t)ctx->N * 3, N = ctx->N, E = ctx->E;
    DevBuf* vecs[] = {&ctx->uk, &ctx->un, &ctx->g, &ctx->du, &ctx->r, &ctx->rhat, &ctx->p, &ctx->v,
                      &ctx->s, &ctx->t, &ctx->phat, &ctx->shat, &ctx->xio};
    for (DevBuf* b : vecs) TF_CK(dalloc(*b, sizeof(double) * n3));
    TF_CK(dalloc(ctx->dinv, sizeof(double) * 9 * N));
    TF_CK(dalloc(ctx->fixmask, N));
    TF_CK(dalloc(ctx->ext_visc, sizeof(double) * n3));
    TF_CK(dalloc(ctx->visc_surface, sizeof(double) * N));
    TF_CK(dalloc(ctx->sc, sizeof(KrylovScalars)));
    TF_CK(dalloc(ctx->dflags, sizeof(int32_t)));
    TF_CK(dalloc(ctx->fg, sizeof(double) * 9 * E));
    TF_CK(dalloc(ctx->rates, sizeof(double) * 3 * E));
    TF_CK(dalloc(ctx->angles, sizeof(double) * E));
    TF_CK(dalloc(ctx->exposed, E));
    TF_CK(dalloc(ctx->peripodial, E));
    TF_CK(dalloc(ctx->rotated, sizeof(int32_t) * E));
    TF_CK(dalloc(ctx->barrier, sizeof(GridBarrier)));
    TF_CK(cudaMemset(ctx->barrier.p, 0, sizeof(GridBarrier)));
    {
        const size_t T = ctx->T;
        TF_CK(dalloc(ctx->active_d, sizeof(int32_t) * T));
        TF_CK(dalloc(ctx->tbarriers, sizeof(GridBarrier) * T));
        TF_CK(dalloc(ctx->tscalars, sizeof(KrylovScalars) * T));
        TF_CK(dalloc(ctx->tdu2, sizeof(double) * T));
        TF_CK(cudaMemset(ctx->tbarriers.p, 0, sizeof(GridBarrier) * T));
        TF_CK(cudaMemset(ctx->tscalars.p, 0, sizeof(KrylovScalars) * T));
        std::vector<int32_t> ones(T, 1);
        TF_CK(cudaMemcpy(ctx->active_d.p, ones.data(), sizeof(int32_t) * T, cudaMemcpyHostToDevice));
        TF_CK(cudaMallocHost(&ctx->h_active, sizeof(int32_t) * T));
        TF_CK(cudaMallocHost(&ctx->h_du2, sizeof(double) * T));
        TF_CK(cudaMallocHost(&ctx->h_tsc, sizeof(KrylovScalars) * T));
        std::vector<int32_t> nt(ctx->N);
        for (int t = 0; t < ctx->T; ++t)
            for (int i = ctx->tissue_node0[t]; i < ctx->tissue_node0[t + 1]; ++i) nt[i] = t;
        TF_CK(dalloc(ctx->node_tissue_d, sizeof(int32_t) * N));
        TF_CK(cudaMemcpy(ctx->node_tissue_d.p, nt.data(), sizeof(int32_t) * N, cudaMemcpyHostToDevice));
    }
    {
        int coop = 0;
        TF_CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, ctx->device));
        // a large single tissue: one 768-thread CTA per SM (fewest grid-barrier participants);
        // small tissues and batches: three 256-thread CTAs per SM (more, smaller row ranges, and
        // in a batch many tissues each with their own CTAs)
        int sms = 0;
        TF_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
        ctx->persist_threads = (T == 1 && ((int64_t)ctx->N >= (int64_t)sms * 256 ||
                                           ctx->params.precond == TF_PRECOND_TWO_LEVEL ||
                                           ctx->params.precond == TF_PRECOND_MULTILEVEL))
                                   ? 768
                                   : 256;
        ctx->persistent_grid_max = coop ? persistent_max_grid(ctx->device, ctx->persist_threads) : 0;
    }
    TF_CK(cudaMemset(ctx->sc.p, 0, sizeof(KrylovScalars)));
    TF_CK(cudaMemset(ctx->fixmask.p, 0, N));
    TF_CK(cudaMemset(ctx->ext_visc.p, 0, sizeof(double) * n3));
    TF_CK(cudaMemset(ctx->visc_surface.p, 0, sizeof(double) * N));
    TF_CK(cudaMemset(ctx->rates.p, 0, sizeof(double) * 3 * E));
    TF_CK(cudaMemset(ctx->angles.p, 0, sizeof(double) * E));
    TF_CK(cudaMemset(ctx->exposed.p, 0, E));
    TF_CK(cudaMemset(ctx->peripodial.p, 0, E));
    {
        std::vector<double> eye((size_t)9 * E);
        for (size_t e = 0; e < E; ++e)
            for (int k = 0; k < 9; ++k) eye[e * 9 + k] = (k % 4 == 0) ? 1.0 : 0.0;
        TF_CK(cudaMemcpy(ctx->fg.p, eye.data(), sizeof(double) * 9 * E, cudaMemcpyHostToDevice));
    }
    TF_CK(cudaMallocHost(&ctx->h_sc, sizeof(KrylovScalars)));
    TF_CK(cudaMallocHost(&ctx->h_flags, sizeof(int32_t)));
    int rc = upload_structure(ctx);
    if (rc != TF_OK) return rc;
    rc = build_plan_all(ctx);
    if (rc != TF_OK) return rc;
    if (ctx->T > 1 && ctx->persistent_grid_max == 0) return TF_ERR_UNSUPPORTED;
    if ((ctx->params.precond == TF_PRECOND_TWO_LEVEL || ctx->params.precond == TF_PRECOND_MULTILEVEL) &&
        ctx->persistent_grid_max == 0)
        ctx->params.precond = TF_PRECOND_BLOCK_JACOBI;
    ctx->h_fixmask.assign(N, 0);
    if (ctx->params.scatter < TF_SCATTER_AUTO || ctx->params.scatter > TF_SCATTER_STAGED) return TF_ERR_ARGUMENT;
    if (ctx->params.scatter == TF_SCATTER_COLOURED && ctx->n_colours == 0) return TF_ERR_UNSUPPORTED;
    ctx->scatter = ctx->params.scatter == TF_SCATTER_AUTO ? TF_SCATTER_ATOMIC : ctx->params.scatter;
    ctx->teams = ctx->params.elems_per_block > 0 ? ctx->params.elems_per_block : 16;
    if (ctx->teams != 8 && ctx->teams != 16 && ctx->teams != 32) return TF_ERR_ARGUMENT;
    {
        const int sn = ctx->params.smoother_nodes;
        if (sn < 0 || sn > 4) return TF_ERR_ARGUMENT;
        if (sn >= 2 && N % sn != 0) return TF_ERR_ARGUMENT;
        ctx->smooth_G = 1;
        bool even = true;  // every tissue holds whole groups (a batch's tissues share G)
        for (int t = 0; t < ctx->T && sn >= 2; ++t)
            even = even && (ctx->tissue_node0[t + 1] - ctx->tissue_node0[t]) % sn == 0;
        if (!even) return TF_ERR_ARGUMENT;
        if (use_persistent(ctx)) {
            // auto: columns of two or three nodes (the wing disc's three-node columns cut the
            // iterations by 16 %; the large slab's four-node columns cut none and cost 16 % more
            // time per step, so they keep node blocks unless asked for)
            ctx->col_G = column_size(ctx);
            int cs = sn == 0 ? ctx->col_G : 1;
            for (int t = 0; t < ctx->T; ++t)
                if ((ctx->tissue_node0[t + 1] - ctx->tissue_node0[t]) % cs != 0) cs = 1;
            ctx->smooth_G = sn >= 2 ? sn : (cs <= 3 ? cs : 1);
        }
        if (ctx->smooth_G > 1) TF_CK(dalloc(ctx->dinv, sizeof(double) * 9 * (size_t)ctx->smooth_G * N));
    }
    *out = holder.release();
    return TF_OK;
}

int tf_create(const tf_mesh_desc* mesh, const tf_params* params, tf_ctx** out) {
    if (!mesh) return TF_ERR_ARGUMENT;
    const int32_t node0[2] = {0, mesh->n_nodes}, elem0[2] = {0, mesh->n_elems};
    return create_ctx(mesh, params, 1, node0, elem0, out);
}

int tf_batch_create(int32_t n_tissues, const tf_mesh_desc* meshes, const tf_params* params, tf_ctx** out) {
    if (!out) return TF_ERR_ARGUMENT;
    *out = nullptr;
    if (n_tissues <= 0 || !meshes) return TF_ERR_ARGUMENT;
    std::vector<int32_t> node0(n_tissues + 1, 0), elem0(n_tissues + 1, 0);
    for (int t = 0; t < n_tissues; ++t) {
        const tf_mesh_desc& m = meshes[t];
        if (m.n_nodes <= 0 || m.n_elems <= 0 || !m.conn || !m.xref) return TF_ERR_ARGUMENT;
        if ((int64_t)node0[t] + m.n_nodes > INT32_MAX || (int64_t)elem0[t] + m.n_elems > INT32_MAX) return TF_ERR_ARGUMENT;
        node0[t + 1] = node0[t] + m.n_nodes;
        elem0[t + 1] = elem0[t] + m.n_elems;
    }
    std::vector<int32_t> conn((size_t)elem0[n_tissues] * 6);
    std::vector<double> xref((size_t)elem0[n_tissues] * 18);
    for (int t = 0; t < n_tissues; ++t) {
        const tf_mesh_desc& m = meshes[t];
        for (int64_t k = 0; k < (int64_t)m.n_elems * 6; ++k) {
            if (m.conn[k] < 0 || m.conn[k] >= m.n_nodes) return TF_ERR_ARGUMENT;
            conn[(size_t)elem0[t] * 6 + k] = m.conn[k] + node0[t];
        }
        std::memcpy(&xref[(size_t)elem0[t] * 18], m.xref, sizeof(double) * 18 * m.n_elems);
    }
    const tf_mesh_desc all{node0[n_tissues], elem0[n_tissues], conn.data(), xref.data()};
    return create_ctx(&all, params, n_tissues, node0.data(), elem0.data(), out);
}

int tf_get_tissue_stats(tf_ctx* ctx, int32_t* newton_iters, int32_t* status, int32_t* krylov_iters) {
    if (!ctx) return TF_ERR_ARGUMENT;
    for (int t = 0; t < ctx->T; ++t) {
        const bool have = (size_t)t < ctx->t_iters.size();
        if (newton_iters) newton_iters[t] = have ? ctx->t_iters[t] : 0;
        if (status) status[t] = have ? ctx->t_status[t] : TF_OK;
        if (krylov_iters) krylov_iters[t] = have ? ctx->t_krylov[t] : 0;
    }
    return TF_OK;
}

int tf_get_n_tissues(tf_ctx* ctx) { return ctx ? ctx->T : TF_ERR_ARGUMENT; }

void tf_destroy(tf_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->krylov_graph) cudaGraphExecDestroy(ctx->krylov_graph);
    DevBuf* all[] = {&ctx->elems, &ctx->fixmask, &ctx->ext_visc, &ctx->visc_surface, &ctx->dofmap_d,
                     &ctx->slaves_d, &ctx->masters_d, &ctx->rowptr_d, &ctx->colidx_d, &ctx->diag_d,
                     &ctx->vals, &ctx->colour_list_d, &ctx->uk, &ctx->un, &ctx->g, &ctx->du, &ctx->r,
                     &ctx->rhat, &ctx->p, &ctx->v, &ctx->s, &ctx->t, &ctx->phat, &ctx->shat, &ctx->dinv,
                     &ctx->partials, &ctx->sc, &ctx->dflags, &ctx->fg, &ctx->rates, &ctx->angles,
                     &ctx->exposed, &ctx->peripodial, &ctx->rotated, &ctx->xio, &ctx->barrier,
                     &ctx->refine_acc, &ctx->refine_g, &ctx->ext_force, &ctx->grid_rel_pos, &ctx->grid_rel_z,
                     &ctx->grid_eflags, &ctx->grid_inc};
    for (DevBuf* b : all) dfree(*b);
    for (auto& gf : ctx->grid_funcs) dfree(gf.cells);
    DevBuf* batch[] = {&ctx->plan_queue_d, &ctx->queue_head_d, &ctx->node_tissue_d, &ctx->plan_list_ptr_d,
                       &ctx->plan_list_d, &ctx->plan_cta0_d, &ctx->plan_ncta_d, &ctx->plan_row0_d, &ctx->active_d, &ctx->tbarriers, &ctx->tscalars, &ctx->tdu2};
    for (DevBuf* b : batch) dfree(*b);
    for (auto* v : {&ctx->cp_x, &ctx->cp_fg, &ctx->seg_x, &ctx->seg_fg, &ctx->warm_hist})
        for (DevBuf& b : *v) dfree(b);
    DevBuf* adj[] = {&ctx->abar, &ctx->abar2, &ctx->mubar, &ctx->dLdr, &ctx->qbuf, &ctx->ilu_cnodes, &ctx->ilu_lo_ptr,
                     &ctx->ilu_lo_idx, &ctx->ilu_up_ptr, &ctx->ilu_up_idx, &ctx->ilu_lu, &ctx->ilu_uinv, &ctx->ilu_y};
    for (DevBuf* b : adj) dfree(*b);
    if (ctx->ilu_graph) cudaGraphExecDestroy(ctx->ilu_graph);
    DevBuf* coarse[] = {&ctx->node_d, &ctx->node_mask, &ctx->agg_m, &ctx->pmode_d, &ctx->coarse_inv, &ctx->coarse_r,
                        &ctx->coarse_info, &ctx->coarse_work, &ctx->ca_agg_slot_ptr, &ctx->ca_slot_agg,
                        &ctx->ca_slot_ptr, &ctx->ca_blk, &ctx->ca_blk_row, &ctx->ca_empty};
    for (DevBuf* b : coarse) dfree(*b);
    DevBuf* bcb[] = {&ctx->bc_tissue_agg0_d, &ctx->bc_agg_ptr_d, &ctx->bc_agg_nodes_d, &ctx->bc_agg_tissue_d, &ctx->bc_base_d, &ctx->bc_unit_d,
                     &ctx->bc_order_d, &ctx->bc_info_d};
    for (DevBuf* b : bcb) dfree(*b);
    DevBuf* lmb[] = {&ctx->lm_tri_d, &ctx->lm_state_d, &ctx->lm_part_d, &ctx->lm_G_d, &ctx->lm_y_d, &ctx->lm_z_d,
                     &ctx->lm_gsave_d, &ctx->lm_dot_part_d, &ctx->lm_dots_d};
    for (DevBuf* b : lmb) dfree(*b);
    if (ctx->h_lm_dots) cudaFreeHost(ctx->h_lm_dots);
    DevBuf* pkb[] = {&ctx->pk_place_d, &ctx->pk_v0_d, &ctx->pk_mass_d, &ctx->pk_prm_d, &ctx->pk_bucket_cnt_d,
                     &ctx->pk_bucket_start_d, &ctx->pk_bucket_nodes_d, &ctx->pk_node_cnt_d, &ctx->pk_node_start_d,
                     &ctx->pk_scan_d, &ctx->pk_pairs_d, &ctx->pk_ptr_d, &ctx->pk_col_d, &ctx->pk_blk_d, &ctx->pk_vals_d,
                     &ctx->pk_dfdx_d, &ctx->pk_x_d};
    for (DevBuf* b : pkb) dfree(*b);
    DevBuf* mlb[] = {&ctx->ml_leaf_ptr_d, &ctx->ml_leaf_nodes_d, &ctx->ml_cen_d, &ctx->ml_w_d, &ctx->ml_top_d,
                     &ctx->ml_top_work, &ctx->ml_info_d, &ctx->ml_leaf_m_d, &ctx->ml_part_d, &ctx->ml_pstart_d,
                     &ctx->ml_first_cta_d, &ctx->ml_slot_a_d, &ctx->ml_out_ptr_d, &ctx->ml_out_slots_d,
                     &ctx->ml_out_set_d, &ctx->ml_out_col_d, &ctx->ml_out_dst_d, &ctx->ml_pairs_d, &ctx->ml_pos_leaf_d};
    for (DevBuf* b : mlb) dfree(*b);
    if (ctx->h_coarse_info) cudaFreeHost(ctx->h_coarse_info);
    if (ctx->h_active) cudaFreeHost(ctx->h_active);
    if (ctx->h_du2) cudaFreeHost(ctx->h_du2);
    if (ctx->h_tsc) cudaFreeHost(ctx->h_tsc);
    if (ctx->h_sc) cudaFreeHost(ctx->h_sc);
    if (ctx->h_flags) cudaFreeHost(ctx->h_flags);
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : ctx->ev_call)
        if (e) cudaEventDestroy(e);
    for (auto& e : ctx->ev_solve)
        if (e) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int tf_set_material(tf_ctx* ctx, const double* lambda, const double* mu, const double* eta) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    if (!lambda || !mu) return TF_ERR_ARGUMENT;
    std::vector<double> lme((size_t)ctx->E * 3);
    bool visc = false;
    for (int e = 0; e < ctx->E; ++e) {
        lme[(size_t)e * 3 + 0] = lambda[e];
        lme[(size_t)e * 3 + 1] = mu[e];
        lme[(size_t)e * 3 + 2] = eta ? eta[e] : 0.0;
        visc |= eta && eta[e] != 0.0;
    }
    ctx->has_visc = visc;
    return set_record_field(ctx, offsetof(ElemRecord, lam), 3, lme.data());
}

int tf_set_inv_fg(tf_ctx* ctx, const double* inv_fg) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    if (!inv_fg) return TF_ERR_ARGUMENT;
    return set_record_field(ctx, offsetof(ElemRecord, inv_fg), 9, inv_fg);
}

int tf_set_boundary(tf_ctx* ctx, const uint8_t* fixed, const double* ext_visc,
                    const int32_t* slave_master, int32_t n_pairs) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    const int N = ctx->N;
    if (n_pairs < 0 || (n_pairs > 0 && !slave_master)) return TF_ERR_ARGUMENT;
    std::vector<uint8_t> fm(N, 0);
    if (fixed)
        for (int i = 0; i < N; ++i)
            fm[i] = (uint8_t)((fixed[i * 3] ? 1 : 0) | (fixed[i * 3 + 1] ? 2 : 0) | (fixed[i * 3 + 2] ? 4 : 0));
    TF_CK(cudaMemcpy(ctx->fixmask.p, fm.data(), N, cudaMemcpyHostToDevice));
    ctx->h_fixmask = fm;
    ctx->coarse_dirty = true;
    if (ext_visc) TF_CK(cudaMemcpy(ctx->ext_visc.p, ext_visc, sizeof(double) * 3 * N, cudaMemcpyHostToDevice));
    std::vector<int32_t> dm((size_t)N * 3);
    for (size_t i = 0; i < dm.size(); ++i) dm[i] = (int32_t)i;
    std::vector<int32_t> sl, ms;
    for (int p = 0; p < n_pairs; ++p) {
        const int32_t s = slave_master[2 * p], m = slave_master[2 * p + 1];
        if (s < 0 || m < 0 || s >= 3 * N || m >= 3 * N || s == m) return TF_ERR_ARGUMENT;
        dm[s] = m;
        sl.push_back(s);
        ms.push_back(m);
    }
    for (int32_t m : ms)
        if (dm[m] != m) return set_error(ctx, TF_ERR_ARGUMENT, "a master DoF is itself a slave");
    if (n_pairs > 0 && ctx->pk_on) return set_error(ctx, TF_ERR_UNSUPPORTED, "slave-master pairs with packing");
    if (n_pairs > 0 && ctx->lm_on) return set_error(ctx, TF_ERR_UNSUPPORTED, "slave-master pairs with a lumen");
    const bool changed = dm != ctx->dofmap;
    ctx->dofmap = dm;
    ctx->slave = sl;
    ctx->master = ms;
    if (changed) return upload_structure(ctx);
    TF_CK(cudaMemcpy(ctx->dofmap_d.p, dm.data(), sizeof(int32_t) * dm.size(), cudaMemcpyHostToDevice));
    return TF_OK;
}

int tf_set_external_force(tf_ctx* ctx, const double* f) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    if (!f) {
        ctx->has_ext_force = false;
        return TF_OK;
    }
    TF_CK(dalloc(ctx->ext_force, sizeof(double) * 3 * (size_t)ctx->N));
    TF_CK(cudaMemcpy(ctx->ext_force.p, f, sizeof(double) * 3 * (size_t)ctx->N, cudaMemcpyHostToDevice));
    ctx->has_ext_force = true;
    return TF_OK;
}

int tf_set_lumen(tf_ctx* ctx, int32_t n_elems, const int32_t* elems, double bulk_modulus, double growth_fold,
                 const double* x) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    if (n_elems <= 0) {
        ctx->lm_on = false;
        return TF_OK;
    }
    if (!elems || !x || !(bulk_modulus >= 0.0)) return TF_ERR_ARGUMENT;
    if (ctx->T != 1 || !ctx->slave.empty() || !use_persistent(ctx))
        return set_error(ctx, TF_ERR_UNSUPPORTED, "lumen: single tissue, no slave-master pairs, persistent solve");
    // Lumen::calculateCurrentVolume at the given positions: the ideal volume of the constructor
    double vol = 0.0;
    for (int k = 0; k < n_elems; ++k) {
        const int e = elems[k];
        if (e < 0 || e >= ctx->E) return TF_ERR_ARGUMENT;
        const int32_t* c = ctx->conn.data() + (size_t)e * 6;
        const double* x1 = x + (size_t)c[3] * 3;
        const double* x2 = x + (size_t)c[4] * 3;
        const double* x3 = x + (size_t)c[5] * 3;
        const double cx[3] = {x3[1] * x1[2] - x3[2] * x1[1], x3[2] * x1[0] - x3[0] * x1[2], x3[0] * x1[1] - x3[1] * x1[0]};
        vol += 1.0 / 6.0 * (cx[0] * x2[0] + cx[1] * x2[1] + cx[2] * x2[2]);
    }
    if (!(std::fabs(vol) > 0.0)) return set_error(ctx, TF_ERR_ARGUMENT, "lumen: the triangles enclose no volume");
    const size_t bytes = sizeof(double) * 3 * (size_t)ctx->N;
    TF_CK(dalloc(ctx->lm_tri_d, sizeof(int32_t) * (size_t)n_elems));
    TF_CK(cudaMemcpy(ctx->lm_tri_d.p, elems, sizeof(int32_t) * (size_t)n_elems, cudaMemcpyHostToDevice));
    TF_CK(dalloc(ctx->lm_state_d, sizeof(LumenState)));
    TF_CK(dalloc(ctx->lm_part_d, sizeof(double) * (size_t)lumen_partials(n_elems)));
    TF_CK(dalloc(ctx->lm_G_d, bytes));
    TF_CK(dalloc(ctx->lm_y_d, bytes));
    TF_CK(dalloc(ctx->lm_z_d, bytes));
    TF_CK(dalloc(ctx->lm_gsave_d, bytes));
    TF_CK(dalloc(ctx->lm_dot_part_d, sizeof(double) * (size_t)dot2_partials()));
    TF_CK(dalloc(ctx->lm_dots_d, 2 * sizeof(double)));
    if (!ctx->h_lm_dots) TF_CK(cudaMallocHost(&ctx->h_lm_dots, 2 * sizeof(double)));
    ctx->lm_n_tri = n_elems;
    ctx->lm_bulk = bulk_modulus;
    ctx->lm_v_init = vol;
    ctx->lm_rate = growth_fold > 0.0 ? std::log(growth_fold) / 3600.0 / 24.0 : 0.0;  // Lumen.cpp:19-22
    ctx->lm_ideal = vol;
    LumenState st{vol, vol};
    TF_CK(cudaMemcpy(ctx->lm_state_d.p, &st, sizeof(st), cudaMemcpyHostToDevice));
    ctx->lm_on = true;
    return TF_OK;
}

int tf_get_lumen(tf_ctx* ctx, double* volume, double* ideal_volume, double* G) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    if (!ctx->lm_on) return set_error(ctx, TF_ERR_STATE, "no lumen (tf_set_lumen)");
    LumenState st;
    TF_CK(cudaMemcpy(&st, ctx->lm_state_d.p, sizeof(st), cudaMemcpyDeviceToHost));
    if (volume) *volume = st.volume;
    if (ideal_volume) *ideal_volume = st.ideal;
    if (G) TF_CK(cudaMemcpy(G, ctx->lm_G_d.p, sizeof(double) * 3 * (size_t)ctx->N, cudaMemcpyDeviceToHost));
    return TF_OK;
}

int tf_set_packing(tf_ctx* ctx, int32_t enabled, const int32_t* node_placement) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    if (!enabled) {
        if (ctx->pk_pairs_n > 0) {  // graphs captured with packing rows
            if (ctx->krylov_graph) cudaGraphExecDestroy(ctx->krylov_graph);
            if (ctx->ilu_graph) cudaGraphExecDestroy(ctx->ilu_graph);
            ctx->krylov_graph = nullptr;
            ctx->ilu_graph = nullptr;
        }
        ctx->pk_on = false;
        ctx->pk_pairs_n = 0;
        return TF_OK;
    }
    if (!node_placement) return TF_ERR_ARGUMENT;
    if (ctx->T != 1 || !ctx->slave.empty())
        return set_error(ctx, TF_ERR_UNSUPPORTED, "packing: single tissue without slave-master pairs");
    const int N = ctx->N, E = ctx->E;
    std::vector<int8_t> pl(N);
    int eligible = 0;
    for (int n = 0; n < N; ++n) {
        pl[n] = (int8_t)((node_placement[n] == 0 || node_placement[n] == 1) ? node_placement[n] : 2);
        eligible += pl[n] != 2;
    }
    // reference volumes (Prism::calculateReferenceVolume, Prism.cpp:890-923, with
    // ShapeBase::calculateVolumeForInputShapeStructure, ShapeBase.cpp:3364-3400): eight triangular
    // faces, each the base of a tetrahedron with the element centre, |height| x area / 3 summed
    static const int faces[8][3] = {{0, 1, 2}, {3, 4, 5}, {0, 1, 3}, {1, 3, 4}, {1, 2, 4}, {2, 4, 5}, {0, 2, 3}, {2, 3, 5}};
    std::vector<double> v0(E);
    for (int e = 0; e < E; ++e) {
        const double* X = ctx->xref.data() + (size_t)e * 18;
        double c[3] = {0, 0, 0};
        for (int k = 0; k < 6; ++k)
            for (int d = 0; d < 3; ++d) c[d] += X[k * 3 + d] / 6.0;
        double vol = 0.0;
        for (const auto& f : faces) {
            double v1[3], v2[3], vm[3];
            for (int d = 0; d < 3; ++d) {
                v1[d] = X[f[1] * 3 + d] - X[f[0] * 3 + d];
                v2[d] = X[f[2] * 3 + d] - X[f[0] * 3 + d];
                vm[d] = c[d] - X[f[0] * 3 + d];
            }
            const double b[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2], v1[0] * v2[1] - v1[1] * v2[0]};
            const double nb = std::sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
            vol += std::fabs((vm[0] * b[0] + vm[1] * b[1] + vm[2] * b[2]) / nb) * (nb / 2.0) / 3.0;
        }
        v0[e] = vol;
    }
    int bits = 10;
    while (bits < 24 && (1 << bits) < 2 * eligible) ++bits;
    const int H = 1 << bits;
    TF_CK(dalloc(ctx->pk_place_d, (size_t)N));
    TF_CK(cudaMemcpy(ctx->pk_place_d.p, pl.data(), (size_t)N, cudaMemcpyHostToDevice));
    TF_CK(dalloc(ctx->pk_v0_d, sizeof(double) * (size_t)E));
    TF_CK(cudaMemcpy(ctx->pk_v0_d.p, v0.data(), sizeof(double) * (size_t)E, cudaMemcpyHostToDevice));
    TF_CK(dalloc(ctx->pk_mass_d, sizeof(double) * (size_t)N));
    TF_CK(dalloc(ctx->pk_prm_d, sizeof(PackParams)));
    TF_CK(dalloc(ctx->pk_bucket_cnt_d, sizeof(int32_t) * ((size_t)H + 1)));
    TF_CK(dalloc(ctx->pk_bucket_start_d, sizeof(int32_t) * ((size_t)H + 1)));
    TF_CK(dalloc(ctx->pk_bucket_nodes_d, sizeof(int32_t) * (size_t)std::max(eligible, 1)));
    TF_CK(dalloc(ctx->pk_node_cnt_d, sizeof(int32_t) * ((size_t)N + 1)));
    TF_CK(dalloc(ctx->pk_node_start_d, sizeof(int32_t) * ((size_t)N + 1)));
    TF_CK(dalloc(ctx->pk_scan_d, sizeof(int32_t) * (size_t)std::max(scan_tmp_ints(H), scan_tmp_ints(N))));
    TF_CK(dalloc(ctx->pk_x_d, sizeof(double) * 3 * (size_t)N));
    ctx->pk_capacity = std::max(ctx->pk_capacity, 1024);
    TF_CK(dalloc(ctx->pk_pairs_d, sizeof(int32_t) * 2 * (size_t)ctx->pk_capacity));
    TF_CK(dalloc(ctx->pk_vals_d, sizeof(double) * 18 * (size_t)ctx->pk_capacity));
    TF_CK(dalloc(ctx->pk_dfdx_d, sizeof(double) * 9 * (size_t)ctx->pk_capacity));
    TF_CK(dalloc(ctx->pk_col_d, sizeof(int32_t) * 2 * (size_t)ctx->pk_capacity));
    TF_CK(dalloc(ctx->pk_blk_d, sizeof(int32_t) * 2 * (size_t)ctx->pk_capacity));
    ctx->pk_hash_bits = bits;
    ctx->pk_pairs_n = 0;
    ctx->pk_on = true;
    return TF_OK;
}

int tf_detect_packing(tf_ctx* ctx, const double* x, int32_t* n_pairs) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    if (!x) return TF_ERR_ARGUMENT;
    if (!ctx->pk_on) return set_error(ctx, TF_ERR_STATE, "packing is not enabled (tf_set_packing)");
    TF_CK(cudaMemcpyAsync(ctx->pk_x_d.p, x, sizeof(double) * 3 * (size_t)ctx->N, cudaMemcpyHostToDevice, ctx->stream));
    rc = packing_detect(ctx, dptr<double>(ctx->pk_x_d));
    if (rc != TF_OK) return rc;
    if (n_pairs) *n_pairs = ctx->pk_pairs_n;
    return TF_OK;
}

int tf_get_packing(tf_ctx* ctx, int32_t max_pairs, int32_t* n_pairs, int32_t* pairs, double* threshold, double* mass,
                   double* dfdx) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    if (max_pairs < 0) return TF_ERR_ARGUMENT;
    if (n_pairs) *n_pairs = ctx->pk_on ? ctx->pk_pairs_n : 0;
    if (!ctx->pk_on) return TF_OK;
    const int np = std::min(max_pairs, ctx->pk_pairs_n);
    if (pairs && np > 0) std::memcpy(pairs, ctx->h_pk_pairs.data(), sizeof(int32_t) * 2 * (size_t)np);
    if (threshold) {
        PackParams prm;
        TF_CK(cudaMemcpy(&prm, ctx->pk_prm_d.p, sizeof(PackParams), cudaMemcpyDeviceToHost));
        *threshold = prm.threshold;
    }
    if (mass) TF_CK(cudaMemcpy(mass, ctx->pk_mass_d.p, sizeof(double) * (size_t)ctx->N, cudaMemcpyDeviceToHost));
    if (dfdx && np > 0) TF_CK(cudaMemcpy(dfdx, ctx->pk_dfdx_d.p, sizeof(double) * 9 * (size_t)np, cudaMemcpyDeviceToHost));
    return TF_OK;
}

int tf_newton_iteration(tf_ctx* ctx, const double* uk, const double* un, double dt, double* du, int32_t* iters,
                        double* rel_res) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    rc = activate_all(ctx);
    if (rc != TF_OK) return rc;
    if (!uk || !un || !du || !(dt > 0)) return TF_ERR_ARGUMENT;
    const size_t bytes = sizeof(double) * 3 * (size_t)ctx->N;
    TF_CK(cudaMemcpyAsync(ctx->uk.p, uk, bytes, cudaMemcpyHostToDevice, ctx->stream));
    TF_CK(cudaMemcpyAsync(ctx->un.p, un, bytes, cudaMemcpyHostToDevice, ctx->stream));
    TF_CK(cudaMemsetAsync(ctx->dflags.p, 0, sizeof(int32_t), ctx->stream));
    ctx->last_method = 0;
    ctx->cg_iters = 0;
    rc = assemble_system(ctx, dt);
    if (rc != TF_OK) return rc;
    rc = newton_solve(ctx);
    if (rc != TF_OK) return rc;
    const KrylovScalars sc = *ctx->h_sc;
    if (!ctx->slave.empty()) {
        KrylovWork w = make_work(ctx);
        TF_CK(cudaMemsetAsync(ctx->xio.p, 0, bytes, ctx->stream));  // equate slaves only: scratch positions
        TF_CK(launch_newton_update(w, dptr<double>(ctx->xio), dptr<int32_t>(ctx->slaves_d), dptr<int32_t>(ctx->masters_d),
                                   (int32_t)ctx->slave.size(), ctx->stream));
    }
    TF_CK(cudaMemcpyAsync(du, ctx->du.p, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    rc = read_flags(ctx);
    if (rc != TF_OK) return rc;
    if (iters) *iters = sc.iter;
    if (rel_res) *rel_res = sc.bb > 0 ? std::sqrt(sc.rr / sc.bb) : 0.0;
    if (*ctx->h_flags & DF_PATTERN_MISS) return set_error(ctx, TF_ERR_STATE, "routed entry outside the pattern");
    if (*ctx->h_flags & DF_NONFINITE) return TF_NONFINITE;
    if (*ctx->h_flags & DF_INVERTED) return TF_ELEMENT_INVERTED;
    return krylov_status_to_tf(sc.status);
}

int tf_set_viscosity_surface(tf_ctx* ctx, const double* visc_surface) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    if (!visc_surface) return TF_ERR_ARGUMENT;
    TF_CK(cudaMemcpy(ctx->visc_surface.p, visc_surface, sizeof(double) * ctx->N, cudaMemcpyHostToDevice));
    return TF_OK;
}

// Shared body of the four step entry points. `host` selects host (H2D/D2H) or device
// pointers; `grow` adds the per-step prologue.
static int step_entry(tf_ctx* ctx, const double* x_n, double dt, double* x_out, tf_step_stats* stats,
                      bool host, bool grow) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    if (!x_n || !x_out || !(dt > 0)) return TF_ERR_ARGUMENT;
    tf_step_stats local;
    tf_step_stats* st = stats ? stats : &local;
    rc = call_begin(ctx, st);
    if (rc != TF_OK) return rc;
    const size_t bytes = sizeof(double) * 3 * (size_t)ctx->N;
    TF_CK(cudaMemcpyAsync(ctx->un.p, x_n, bytes, host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, ctx->stream));
    if (grow) {
        rc = prologue(ctx, dt);
        if (rc != TF_OK) return rc;
    }
    ctx->warm_call = true;
    rc = newton_core(ctx, dt, st);
    ctx->warm_call = false;
    if (rc < 0) return rc;
    if (grow) ctx->sim_time += dt;  // runOneStep ends with currSimTimeSec += dt
    TF_CK(cudaMemcpyAsync(x_out, ctx->uk.p, bytes, host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, ctx->stream));
    const int rc2 = call_end(ctx, st);
    return rc2 != TF_OK ? rc2 : rc;
}

int tf_newton_step_device(tf_ctx* ctx, const double* d_x_n, double dt, double* d_x_out, tf_step_stats* stats) {
    return step_entry(ctx, d_x_n, dt, d_x_out, stats, false, false);
}

int tf_newton_step(tf_ctx* ctx, const double* x_n, double dt, double* x_out, tf_step_stats* stats) {
    return step_entry(ctx, x_n, dt, x_out, stats, true, false);
}

int tf_get_pattern(tf_ctx* ctx, int32_t* nnzb, int32_t* rowptr, int32_t* colidx) {
    if (!ctx) return TF_ERR_ARGUMENT;
    if (nnzb) *nnzb = (int32_t)ctx->nnzb;
    if (rowptr) std::memcpy(rowptr, ctx->rowptr.data(), sizeof(int32_t) * (ctx->N + 1));
    if (colidx) std::memcpy(colidx, ctx->colidx.data(), sizeof(int32_t) * (size_t)ctx->nnzb);
    return TF_OK;
}

int tf_assemble(tf_ctx* ctx, const double* uk, const double* un, double dt, double* g_out, double* bsr_vals_out) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    rc = activate_all(ctx);
    if (rc != TF_OK) return rc;
    if (!uk || !un || !g_out || !(dt > 0)) return TF_ERR_ARGUMENT;
    const size_t bytes = sizeof(double) * 3 * (size_t)ctx->N;
    TF_CK(cudaMemcpyAsync(ctx->uk.p, uk, bytes, cudaMemcpyHostToDevice, ctx->stream));
    TF_CK(cudaMemcpyAsync(ctx->un.p, un, bytes, cudaMemcpyHostToDevice, ctx->stream));
    TF_CK(cudaMemsetAsync(ctx->dflags.p, 0, sizeof(int32_t), ctx->stream));
    rc = assemble_system(ctx, dt);
    if (rc != TF_OK) return rc;
    TF_CK(cudaMemcpyAsync(g_out, ctx->g.p, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    if (bsr_vals_out)
        TF_CK(cudaMemcpyAsync(bsr_vals_out, ctx->vals.p, sizeof(double) * 9 * (size_t)ctx->nnzb, cudaMemcpyDeviceToHost,
                              ctx->stream));
    rc = read_flags(ctx);
    if (rc != TF_OK) return rc;
    if (*ctx->h_flags & DF_PATTERN_MISS) return set_error(ctx, TF_ERR_STATE, "routed entry outside the pattern");
    if (*ctx->h_flags & DF_NONFINITE) return TF_NONFINITE;
    return (*ctx->h_flags & DF_INVERTED) ? TF_ELEMENT_INVERTED : TF_OK;
}

int tf_solve(tf_ctx* ctx, const double* bsr_vals, const double* g, double* du, int32_t* iters, double* rel_res) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    rc = activate_all(ctx);
    if (rc != TF_OK) return rc;
    if (!bsr_vals || !g || !du) return TF_ERR_ARGUMENT;
    const size_t bytes = sizeof(double) * 3 * (size_t)ctx->N;
    TF_CK(cudaMemcpyAsync(ctx->vals.p, bsr_vals, sizeof(double) * 9 * (size_t)ctx->nnzb, cudaMemcpyHostToDevice, ctx->stream));
    TF_CK(cudaMemcpyAsync(ctx->g.p, g, bytes, cudaMemcpyHostToDevice, ctx->stream));
    TF_CK(cudaMemsetAsync(ctx->dflags.p, 0, sizeof(int32_t), ctx->stream));
    ctx->last_method = 0;
    ctx->cg_iters = 0;
    rc = krylov_solve(ctx);
    if (rc != TF_OK) return rc;
    KrylovScalars sc = *ctx->h_sc;
    int32_t total_iters = sc.iter;
    double rel = sc.bb > 0 ? std::sqrt(sc.rr / sc.bb) : 0.0;
    if (ctx->params.krylov_refine > 0 && sc.status == KS_CONVERGED && sc.bb > 0) {
        // Iterative refinement: r = g - J du in FP64, J d = r solved by the same Krylov solve, du += d.
        // The solve's relative tolerance bounds the correction's error, so each pass multiplies the
        // error of du by about kappa(J) x krylov_rtol until the residual reaches rounding level.
        KrylovWork w = make_work(ctx);
        TF_CK(dalloc(ctx->refine_acc, bytes));
        TF_CK(dalloc(ctx->refine_g, bytes));
        double* acc = dptr<double>(ctx->refine_acc);
        TF_CK(cudaMemcpyAsync(acc, ctx->du.p, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
        TF_CK(cudaMemcpyAsync(ctx->refine_g.p, ctx->g.p, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
        const double bb = sc.bb;
        for (int k = 0; k < ctx->params.krylov_refine; ++k) {
            TF_CK(launch_residual(w, acc, dptr<double>(ctx->refine_g), dptr<double>(ctx->g), ctx->stream));
            ctx->launches += 1;
            TF_CK(cudaMemcpyAsync(ctx->h_sc, ctx->sc.p, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, ctx->stream));
            TF_CK(cudaStreamSynchronize(ctx->stream));
            const double r2 = ctx->h_sc->du2;
            rel = std::sqrt(r2 / bb);
            if (!(r2 > 0.0)) break;  // exact (or non-finite: reported by the next solve's status)
            rc = krylov_solve(ctx);
            if (rc != TF_OK) break;
            const KrylovScalars sk = *ctx->h_sc;
            total_iters += sk.iter;
            if (sk.status != KS_CONVERGED) {
                sc.status = sk.status;
                break;
            }
            TF_CK(launch_axpy(3 * ctx->N, 1.0, dptr<double>(ctx->du), acc, ctx->stream));
            ctx->launches += 1;
        }
        // the refined du, g restored, and the true residual of the result
        TF_CK(cudaMemcpyAsync(ctx->du.p, acc, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
        TF_CK(launch_residual(w, acc, dptr<double>(ctx->refine_g), dptr<double>(ctx->g), ctx->stream));
        TF_CK(cudaMemcpyAsync(ctx->g.p, ctx->refine_g.p, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
        TF_CK(cudaMemcpyAsync(ctx->h_sc, ctx->sc.p, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, ctx->stream));
        TF_CK(cudaStreamSynchronize(ctx->stream));
        ctx->launches += 1;
        rel = std::sqrt(ctx->h_sc->du2 / bb);
        if (rc != TF_OK) return rc;
    }
    if (!ctx->slave.empty()) {
        KrylovWork w = make_work(ctx);
        // equate slaves only (no position update): reuse the update kernel on a scratch vector
        TF_CK(cudaMemsetAsync(ctx->xio.p, 0, bytes, ctx->stream));
        TF_CK(launch_newton_update(w, dptr<double>(ctx->xio), dptr<int32_t>(ctx->slaves_d), dptr<int32_t>(ctx->masters_d),
                                   (int32_t)ctx->slave.size(), ctx->stream));
    }
    TF_CK(cudaMemcpyAsync(du, ctx->du.p, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    TF_CK(cudaStreamSynchronize(ctx->stream));
    if (iters) *iters = total_iters;
    if (rel_res) *rel_res = rel;
    return krylov_status_to_tf(sc.status);
}

int tf_set_growth(tf_ctx* ctx, const double* fg, const double* rates, const double* angles,
                  const uint8_t* exposed, const uint8_t* peripodial) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    const size_t E = ctx->E;
    if (fg) {
        TF_CK(cudaMemcpy(ctx->fg.p, fg, sizeof(double) * 9 * E, cudaMemcpyHostToDevice));
        // keep InvFg consistent with Fg (growShapeByFg leaves both in step)
        std::vector<double> inv(9 * E);
        for (size_t e = 0; e < E; ++e) {
            const double* m = fg + e * 9;
            const double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                               m[2] * (m[3] * m[7] - m[4] * m[6]);
            if (det == 0.0 || !std::isfinite(det)) return TF_ERR_ARGUMENT;
            const double id = 1.0 / det;
            double* o = &inv[e * 9];
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
        rc = set_record_field(ctx, offsetof(ElemRecord, inv_fg), 9, inv.data());
        if (rc != TF_OK) return rc;
    }
    if (rates) TF_CK(cudaMemcpy(ctx->rates.p, rates, sizeof(double) * 3 * E, cudaMemcpyHostToDevice));
    if (angles) TF_CK(cudaMemcpy(ctx->angles.p, angles, sizeof(double) * E, cudaMemcpyHostToDevice));
    if (exposed) TF_CK(cudaMemcpy(ctx->exposed.p, exposed, E, cudaMemcpyHostToDevice));
    if (peripodial) TF_CK(cudaMemcpy(ctx->peripodial.p, peripodial, E, cudaMemcpyHostToDevice));
    return TF_OK;
}

int tf_get_growth(tf_ctx* ctx, double* fg, double* inv_fg) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    TF_CK(cudaStreamSynchronize(ctx->stream));
    if (fg) TF_CK(cudaMemcpy(fg, ctx->fg.p, sizeof(double) * 9 * (size_t)ctx->E, cudaMemcpyDeviceToHost));
    if (inv_fg) {
        std::vector<ElemRecord> rec(ctx->E);
        TF_CK(cudaMemcpy(rec.data(), ctx->elems.p, sizeof(ElemRecord) * (size_t)ctx->E, cudaMemcpyDeviceToHost));
        for (int e = 0; e < ctx->E; ++e) std::memcpy(inv_fg + (size_t)e * 9, rec[e].inv_fg, sizeof(double) * 9);
    }
    return TF_OK;
}

// GridBasedGrowthFunction's constructor (GrowthFunctionTypes.h:287-345) and
// preCalculateAnglesForCompatibleAveraging (:368-531): per cell, the four corners' growth and
// angles, angles of corners whose x / y growth ratio is below 1.1 left out, the others brought
// into [0, pi] and then within 45 degrees of the first kept corner, with x / y growth swapped
// where that took a 90-degree turn.
static void grid_cells(const tf_grid_growth& f, std::vector<GridCell>& cells) {
    const int nx = f.nx, ny = f.ny;
    auto gm = [&](int i, int j, int k) { return f.rates[((size_t)i * ny + j) * 3 + k]; };
    auto over = [&](int i, int j) {
        double AR = gm(i, j, 0) / gm(i, j, 1);
        if (AR < 0) AR *= -1.0;
        if (AR < 1.0) AR = 1 / AR;
        return !(AR < 1.1);
    };
    cells.assign((size_t)(nx - 1) * (ny - 1), GridCell());
    for (int IX = 0; IX < nx - 1; ++IX)
        for (int IY = 0; IY < ny - 1; ++IY) {
            GridCell& c = cells[(size_t)IX * (ny - 1) + IY];
            std::memset(&c, 0, sizeof(c));
            const int ci[4][2] = {{IX, IY}, {IX + 1, IY}, {IX, IY + 1}, {IX + 1, IY + 1}};
            double a[4] = {0, 0, 0, 0};
            bool elim[4] = {false, false, false, false};
            for (int q = 0; q < 4; ++q) {
                for (int k = 0; k < 3; ++k) c.g[q][k] = gm(ci[q][0], ci[q][1], k);
                if (over(ci[q][0], ci[q][1]))
                    a[q] = f.angles[(size_t)ci[q][0] * ny + ci[q][1]] * M_PI / 180.0;
                else
                    elim[q] = true;
            }
            for (int q = 0; q < 4; ++q) {
                while (a[q] < 0) a[q] += M_PI;
                while (a[q] > M_PI) a[q] -= M_PI;
            }
            int sel = 3;
            double tet = 0;
            for (int q = 0; q < 4; ++q)
                if (!elim[q]) {
                    tet = a[q];
                    sel = q;
                    break;
                }
            for (int q = sel; q < 4; ++q) {
                const double d = a[q] - tet;
                bool flip = false;
                if (d > 0) {
                    if (d >= M_PI / 4.0 && d < 3.0 * M_PI / 4.0) {
                        a[q] -= M_PI / 2.0;
                        flip = true;
                    } else if (d >= 3.0 * M_PI / 4.0 && d < 5.0 * M_PI / 4.0) {
                        a[q] -= M_PI;
                    } else if (d >= 5.0 * M_PI / 4.0 && d < 7.0 * M_PI / 4.0) {
                        a[q] -= 6.0 * M_PI / 4.0;
                        flip = true;
                    } else if (d >= 7.0 * M_PI / 4.0) {
                        a[q] -= 2.0 * M_PI;
                    }
                } else if (d < 0) {
                    if (d <= -M_PI / 4.0 && d > -3.0 * M_PI / 4.0) {
                        a[q] += M_PI / 2.0;
                        flip = true;
                    } else if (d <= -3.0 * M_PI / 4.0 && d > -5.0 * M_PI / 4.0) {
                        a[q] += M_PI;
                    } else if (d <= -5.0 * M_PI / 4.0 && d > -7.0 * M_PI / 4.0) {
                        a[q] += 6.0 * M_PI / 4.0;
                        flip = true;
                    } else if (d <= -7.0 * M_PI / 4.0) {
                        a[q] += 2.0 * M_PI;
                    }
                }
                if (flip) std::swap(c.g[q][0], c.g[q][1]);
            }
            for (int q = 0; q < 4; ++q) {
                c.a[q] = a[q];
                if (elim[q]) c.elim |= 1 << q;
            }
        }
}

int tf_set_grid_growth(tf_ctx* ctx, int32_t n_funcs, const tf_grid_growth* funcs, int32_t interpolation,
                       const double* rel_pos, const double* rel_z, const int32_t* elem_flags) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    if (n_funcs < 0 || (n_funcs > 0 && (!funcs || !rel_pos || !rel_z || !elem_flags)) ||
        (interpolation != 0 && interpolation != 1))
        return TF_ERR_ARGUMENT;
    for (int f = 0; f < n_funcs; ++f)
        if (funcs[f].nx < 2 || funcs[f].ny < 2 || !funcs[f].rates || !funcs[f].angles) return TF_ERR_ARGUMENT;
    for (auto& gf : ctx->grid_funcs) dfree(gf.cells);
    ctx->grid_funcs.clear();
    ctx->grid_interp = interpolation;
    if (n_funcs == 0) return TF_OK;
    const size_t E = (size_t)ctx->E;
    TF_CK(dalloc(ctx->grid_rel_pos, sizeof(double) * 2 * E));
    TF_CK(dalloc(ctx->grid_rel_z, sizeof(double) * E));
    TF_CK(dalloc(ctx->grid_eflags, sizeof(int32_t) * E));
    TF_CK(dalloc(ctx->grid_inc, sizeof(double) * 9 * E));
    TF_CK(cudaMemcpy(ctx->grid_rel_pos.p, rel_pos, sizeof(double) * 2 * E, cudaMemcpyHostToDevice));
    TF_CK(cudaMemcpy(ctx->grid_rel_z.p, rel_z, sizeof(double) * E, cudaMemcpyHostToDevice));
    TF_CK(cudaMemcpy(ctx->grid_eflags.p, elem_flags, sizeof(int32_t) * E, cudaMemcpyHostToDevice));
    std::vector<GridCell> cells;
    for (int f = 0; f < n_funcs; ++f) {
        tf_ctx::GridFuncHost h;
        h.t0 = funcs[f].t0;
        h.t1 = funcs[f].t1;
        h.zmin = funcs[f].z_min;
        h.zmax = funcs[f].z_max;
        h.nx = funcs[f].nx;
        h.ny = funcs[f].ny;
        h.flags = funcs[f].flags;
        grid_cells(funcs[f], cells);
        ctx->grid_funcs.push_back(h);
        TF_CK(dalloc(ctx->grid_funcs.back().cells, sizeof(GridCell) * cells.size()));
        TF_CK(cudaMemcpy(ctx->grid_funcs.back().cells.p, cells.data(), sizeof(GridCell) * cells.size(),
                         cudaMemcpyHostToDevice));
    }
    return TF_OK;
}

int tf_set_time(tf_ctx* ctx, double t) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    if (!std::isfinite(t)) return TF_ERR_ARGUMENT;
    ctx->sim_time = t;
    return TF_OK;
}

int tf_get_time(tf_ctx* ctx, double* t) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    if (!t) return TF_ERR_ARGUMENT;
    *t = ctx->sim_time;
    return TF_OK;
}

int tf_time_step_device(tf_ctx* ctx, const double* d_x_n, double dt, double* d_x_out, tf_step_stats* stats) {
    return step_entry(ctx, d_x_n, dt, d_x_out, stats, false, true);
}

int tf_time_step(tf_ctx* ctx, const double* x_n, double dt, double* x_out, tf_step_stats* stats) {
    return step_entry(ctx, x_n, dt, x_out, stats, true, true);
}

int tf_get_preconditioner(tf_ctx* ctx, int32_t* precond, int32_t* n_coarse, int32_t* coarse_refreshes) {
    if (!ctx) return TF_ERR_ARGUMENT;
    if (precond) *precond = ctx->ml_active ? TF_PRECOND_MULTILEVEL : ctx->params.precond;
    if (n_coarse) *n_coarse = (ctx->coarse_m > 0 || ctx->bc_active || ctx->ml_active) ? ctx->n_coarse : 0;
    if (coarse_refreshes) *coarse_refreshes = ctx->coarse_refreshes;
    return TF_OK;
}

int tf_get_krylov_method(tf_ctx* ctx, int32_t* method) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    if (!method) return TF_ERR_ARGUMENT;
    *method = ctx->last_method;
    return TF_OK;
}

int tf_get_smoother_block(tf_ctx* ctx, int32_t* nodes) {
    if (!ctx || !nodes) return TF_ERR_ARGUMENT;
    *nodes = use_persistent(ctx) ? ctx->smooth_G : 1;
    return TF_OK;
}

int tf_get_schedule(tf_ctx* ctx, int32_t* n_colours, int32_t* scatter, int32_t* elems_per_block) {
    if (!ctx) return TF_ERR_ARGUMENT;
    if (n_colours) *n_colours = ctx->n_colours;
    if (scatter) *scatter = ctx->scatter;
    if (elems_per_block) *elems_per_block = ctx->teams;
    return TF_OK;
}

int tf_autotune(tf_ctx* ctx, const double* x_n, double dt) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    rc = activate_all(ctx);
    if (rc != TF_OK) return rc;
    if (!x_n || !(dt > 0)) return TF_ERR_ARGUMENT;
    const size_t bytes = sizeof(double) * 3 * (size_t)ctx->N;
    TF_CK(cudaMemcpyAsync(ctx->uk.p, x_n, bytes, cudaMemcpyHostToDevice, ctx->stream));
    TF_CK(cudaMemcpyAsync(ctx->un.p, x_n, bytes, cudaMemcpyHostToDevice, ctx->stream));
    const int teams_opts[3] = {8, 16, 32};
    float best = 1e30f;
    int best_sc = TF_SCATTER_ATOMIC, best_t = 32;
    for (int sc = TF_SCATTER_ATOMIC; sc <= TF_SCATTER_STAGED; ++sc) {
        if (sc == TF_SCATTER_COLOURED && ctx->n_colours == 0) continue;
        if (ctx->params.scatter != TF_SCATTER_AUTO && sc != ctx->params.scatter) continue;
        for (int t : teams_opts) {
            if (ctx->params.elems_per_block > 0 && t != ctx->params.elems_per_block) continue;
            std::vector<float> times;
            for (int rep = 0; rep < 6; ++rep) {
                TF_CK(cudaMemsetAsync(ctx->vals.p, 0, sizeof(double) * 9 * (size_t)ctx->nnzb, ctx->stream));
                TF_CK(cudaMemsetAsync(ctx->g.p, 0, bytes, ctx->stream));
                TF_CK(cudaEventRecord(ctx->ev[0], ctx->stream));
                TF_CK(launch_elements(ctx, dt, sc, t));
                TF_CK(cudaEventRecord(ctx->ev[1], ctx->stream));
                TF_CK(cudaEventSynchronize(ctx->ev[1]));
                float ms;
                TF_CK(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
                if (rep > 0) times.push_back(ms);
            }
            std::sort(times.begin(), times.end());
            const float med = times[times.size() / 2];
            if (med < best) {
                best = med;
                best_sc = sc;
                best_t = t;
            }
        }
    }
    ctx->scatter = best_sc;
    ctx->teams = best_t;
    ctx->tuned = true;
    return TF_OK;
}

int tf_time_kernels(tf_ctx* ctx, int32_t reps, double* ms_element, double* ms_spmv) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    rc = activate_all(ctx);
    if (rc != TF_OK) return rc;
    if (reps <= 0) return TF_ERR_ARGUMENT;
    const double dt = 60.0;
    float ms = 0.0f;
    double tot = 0.0;
    for (int rep = 0; rep < reps; ++rep) {
        TF_CK(cudaMemsetAsync(ctx->vals.p, 0, sizeof(double) * 9 * (size_t)ctx->nnzb, ctx->stream));
        TF_CK(cudaMemsetAsync(ctx->g.p, 0, sizeof(double) * 3 * (size_t)ctx->N, ctx->stream));
        TF_CK(cudaEventRecord(ctx->ev[0], ctx->stream));
        TF_CK(launch_elements(ctx, dt, ctx->scatter, ctx->teams));
        TF_CK(cudaEventRecord(ctx->ev[1], ctx->stream));
        TF_CK(cudaEventSynchronize(ctx->ev[1]));
        TF_CK(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
        tot += ms;
    }
    if (ms_element) *ms_element = tot / reps;
    KrylovWork w = make_work(ctx);
    tot = 0.0;
    for (int rep = 0; rep < reps; ++rep) {
        TF_CK(cudaEventRecord(ctx->ev[0], ctx->stream));
        TF_CK(launch_spmv(w, dptr<double>(ctx->uk), dptr<double>(ctx->xio), ctx->stream));
        TF_CK(cudaEventRecord(ctx->ev[1], ctx->stream));
        TF_CK(cudaEventSynchronize(ctx->ev[1]));
        TF_CK(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
        tot += ms;
    }
    if (ms_spmv) *ms_spmv = tot / reps;
    return TF_OK;
}

int tf_solve_direct(tf_ctx* ctx, const double* bsr_vals, const double* g, double* du, double* ms_factor_solve,
                    int32_t* method) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    if (!bsr_vals || !g || !du) return TF_ERR_ARGUMENT;
    if (!ctx->slave.empty()) return set_error(ctx, TF_ERR_UNSUPPORTED, "direct solve: no slave-master pairs");
    if (ctx->pk_on && ctx->pk_pairs_n > 0) return set_error(ctx, TF_ERR_UNSUPPORTED, "direct solve: packing blocks");
    const size_t bytes = sizeof(double) * 3 * (size_t)ctx->N;
    TF_CK(cudaMemcpyAsync(ctx->vals.p, bsr_vals, sizeof(double) * 9 * (size_t)ctx->nnzb, cudaMemcpyHostToDevice, ctx->stream));
    TF_CK(cudaMemcpyAsync(ctx->g.p, g, bytes, cudaMemcpyHostToDevice, ctx->stream));
    float ms = 0.0f;
    int m = 0;
    const int drc = direct_solve_bsr3(ctx->N, ctx->nnzb, dptr<int32_t>(ctx->rowptr_d), dptr<int32_t>(ctx->colidx_d),
                                      dptr<double>(ctx->vals), dptr<double>(ctx->g), dptr<double>(ctx->du), ctx->stream,
                                      &ms, &m);
    if (drc == -3) return set_error(ctx, TF_ERR_OUT_OF_MEMORY, "direct solve: CSR buffers");
    if (drc < 0) return set_error(ctx, TF_ERR_CUDA, "direct solve: cuSOLVER failure");
    if (ms_factor_solve) *ms_factor_solve = ms;
    if (method) *method = m;
    if (drc == 4)
        return set_error(ctx, TF_ERR_UNSUPPORTED,
                         "direct solve: J is not positive definite (Cholesky failed) and too large for the QR fallback");
    TF_CK(cudaMemcpyAsync(du, ctx->du.p, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    TF_CK(cudaStreamSynchronize(ctx->stream));
    if (ms_factor_solve) *ms_factor_solve = ms;
    if (method) *method = m;
    return drc == 3 ? TF_KRYLOV_BREAKDOWN : TF_OK;
}

// One implicit time step on the device: un holds x_n and ctx->fg holds Fg_n on entry; after the
// call uk holds x_{n+1} and ctx->fg holds Fg_{n+1}.
static int device_time_step(tf_ctx* ctx, double dt, tf_step_stats* st) {
    int rc = prologue(ctx, dt);
    if (rc != TF_OK) return rc;
    tf_step_stats local;
    std::memset(&local, 0, sizeof(local));
    rc = newton_core(ctx, dt, &local);
    if (st) {
        st->newton_iters += local.newton_iters;
        st->krylov_iters_total += local.krylov_iters_total;
        st->krylov_iters_max = std::max(st->krylov_iters_max, local.krylov_iters_max);
        st->ms_assemble += local.ms_assemble;
        st->ms_solve += local.ms_solve;
        st->status = worse(st->status, local.status);
    }
    return rc;
}

int tf_adjoint_forward(tf_ctx* ctx, const double* x0, int32_t n_steps, double dt, int32_t checkpoint_every,
                       double* x_final, tf_step_stats* stats) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    if (!x0 || !x_final || n_steps <= 0 || checkpoint_every <= 0 || !(dt > 0)) return TF_ERR_ARGUMENT;
    if (ctx->has_visc || !ctx->slave.empty() || ctx->T != 1 || ctx->pk_on || ctx->lm_on)
        return set_error(ctx, TF_ERR_UNSUPPORTED,
                         "adjoint: single tissue without internal viscosity, slave-master pairs, packing or lumen");
    tf_step_stats local;
    tf_step_stats* st = stats ? stats : &local;
    rc = call_begin(ctx, st);
    if (rc != TF_OK) return rc;
    const size_t bx = sizeof(double) * 3 * (size_t)ctx->N, bf = sizeof(double) * 9 * (size_t)ctx->E;
    const int n_cp = (n_steps + checkpoint_every - 1) / checkpoint_every;
    ctx->cp_x.resize(n_cp);
    ctx->cp_fg.resize(n_cp);
    for (int i = 0; i < n_cp; ++i) {
        TF_CK(dalloc(ctx->cp_x[i], bx));
        TF_CK(dalloc(ctx->cp_fg[i], bf));
    }
    ctx->adj_steps = n_steps;
    ctx->adj_k = checkpoint_every;
    ctx->adj_dt = dt;
    TF_CK(cudaMemcpyAsync(ctx->un.p, x0, bx, cudaMemcpyHostToDevice, ctx->stream));
    for (int n = 0; n < n_steps; ++n) {
        if (n % checkpoint_every == 0) {
            TF_CK(cudaMemcpyAsync(ctx->cp_x[n / checkpoint_every].p, ctx->un.p, bx, cudaMemcpyDeviceToDevice, ctx->stream));
            TF_CK(cudaMemcpyAsync(ctx->cp_fg[n / checkpoint_every].p, ctx->fg.p, bf, cudaMemcpyDeviceToDevice, ctx->stream));
        }
        rc = device_time_step(ctx, dt, st);
        if (rc < 0) return rc;
        TF_CK(cudaMemcpyAsync(ctx->un.p, ctx->uk.p, bx, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    TF_CK(cudaMemcpyAsync(x_final, ctx->un.p, bx, cudaMemcpyDeviceToHost, ctx->stream));
    const int rc2 = call_end(ctx, st);
    return rc2 != TF_OK ? rc2 : st->status;
}

int tf_adjoint_backward(tf_ctx* ctx, const double* dL_dx_final, double* dL_drates, double* dL_dx0,
                        tf_step_stats* stats) {
    int rc = check_ctx(ctx);
    if (rc != TF_OK) return rc;
    if (!dL_dx_final || !dL_drates) return TF_ERR_ARGUMENT;
    if (ctx->adj_steps <= 0) return set_error(ctx, TF_ERR_STATE, "tf_adjoint_forward has not run");
    tf_step_stats local;
    tf_step_stats* st = stats ? stats : &local;
    rc = call_begin(ctx, st);
    if (rc != TF_OK) return rc;
    const int N = ctx->N, E = ctx->E, K = ctx->adj_k, S = ctx->adj_steps;
    const double dt = ctx->adj_dt;
    const size_t bx = sizeof(double) * 3 * (size_t)N, bf = sizeof(double) * 9 * (size_t)E;
    ctx->seg_x.resize(K + 1);
    ctx->seg_fg.resize(K + 1);
    for (int i = 0; i <= K; ++i) {
        TF_CK(dalloc(ctx->seg_x[i], bx));
        TF_CK(dalloc(ctx->seg_fg[i], bf));
    }
    TF_CK(dalloc(ctx->abar, bx));
    TF_CK(dalloc(ctx->abar2, bx));
    TF_CK(dalloc(ctx->mubar, bf));
    TF_CK(dalloc(ctx->dLdr, sizeof(double) * 3 * E));
    TF_CK(dalloc(ctx->qbuf, sizeof(double) * N));
    TF_CK(cudaMemcpyAsync(ctx->abar.p, dL_dx_final, bx, cudaMemcpyHostToDevice, ctx->stream));
    TF_CK(launch_mask_fixed(N, dptr<uint8_t>(ctx->fixmask), dptr<double>(ctx->abar), ctx->stream));
    TF_CK(cudaMemsetAsync(ctx->mubar.p, 0, bf, ctx->stream));
    TF_CK(cudaMemsetAsync(ctx->dLdr.p, 0, sizeof(double) * 3 * E, ctx->stream));
    const int n_seg = (S + K - 1) / K;
    for (int seg = n_seg - 1; seg >= 0; --seg) {
        const int s0 = seg * K, L = std::min(S, s0 + K) - s0;
        // recompute the segment's states from its checkpoint
        TF_CK(cudaMemcpyAsync(ctx->seg_x[0].p, ctx->cp_x[seg].p, bx, cudaMemcpyDeviceToDevice, ctx->stream));
        TF_CK(cudaMemcpyAsync(ctx->seg_fg[0].p, ctx->cp_fg[seg].p, bf, cudaMemcpyDeviceToDevice, ctx->stream));
        for (int j = 0; j < L; ++j) {
            TF_CK(cudaMemcpyAsync(ctx->un.p, ctx->seg_x[j].p, bx, cudaMemcpyDeviceToDevice, ctx->stream));
            TF_CK(cudaMemcpyAsync(ctx->fg.p, ctx->seg_fg[j].p, bf, cudaMemcpyDeviceToDevice, ctx->stream));
            rc = device_time_step(ctx, dt, st);
            if (rc < 0) return rc;
            TF_CK(cudaMemcpyAsync(ctx->seg_x[j + 1].p, ctx->uk.p, bx, cudaMemcpyDeviceToDevice, ctx->stream));
            TF_CK(cudaMemcpyAsync(ctx->seg_fg[j + 1].p, ctx->fg.p, bf, cudaMemcpyDeviceToDevice, ctx->stream));
        }
        // adjoint steps, last to first
        for (int j = L - 1; j >= 0; --j) {
            const double* x_n = dptr<double>(ctx->seg_x[j]);
            const double* x_n1 = dptr<double>(ctx->seg_x[j + 1]);
            TF_CK(launch_set_inv_fg(dptr<ElemRecord>(ctx->elems), E, dptr<double>(ctx->seg_fg[j + 1]), ctx->stream));
            TF_CK(launch_viscosity_surface(dptr<ElemRecord>(ctx->elems), E, N, x_n, dptr<uint8_t>(ctx->exposed),
                                           dptr<uint8_t>(ctx->peripodial), dptr<double>(ctx->visc_surface), ctx->stream));
            TF_CK(cudaMemcpyAsync(ctx->uk.p, x_n1, bx, cudaMemcpyDeviceToDevice, ctx->stream));
            TF_CK(cudaMemcpyAsync(ctx->un.p, x_n, bx, cudaMemcpyDeviceToDevice, ctx->stream));
            rc = activate_all(ctx);
            if (rc != TF_OK) return rc;
            rc = assemble_system(ctx, dt);  // J at the converged state of the step
            if (rc != TF_OK) return rc;
            // J^T lambda = abar (J is symmetric on this path); the solve reads its RHS from g
            TF_CK(cudaMemcpyAsync(ctx->g.p, ctx->abar.p, bx, cudaMemcpyDeviceToDevice, ctx->stream));
            rc = krylov_solve(ctx);
            if (rc != TF_OK) return rc;
            const KrylovScalars sc = *ctx->h_sc;
            st->krylov_iters_total += sc.iter;
            st->krylov_iters_max = std::max(st->krylov_iters_max, sc.iter);
            if (krylov_status_to_tf(sc.status) != TF_OK) st->status = worse(st->status, krylov_status_to_tf(sc.status));
            double* lam = dptr<double>(ctx->du);
            TF_CK(launch_mask_fixed(N, dptr<uint8_t>(ctx->fixmask), lam, ctx->stream));
            TF_CK(launch_growth_vjp(dptr<ElemRecord>(ctx->elems), E, lam, dptr<uint8_t>(ctx->fixmask), x_n1,
                                    dptr<double>(ctx->seg_fg[j]), dptr<double>(ctx->rates), dptr<double>(ctx->angles), dt,
                                    dptr<double>(ctx->mubar), dptr<double>(ctx->dLdr), ctx->stream));
            TF_CK(launch_position_vjp(dptr<ElemRecord>(ctx->elems), E, N, lam, dptr<uint8_t>(ctx->fixmask), x_n, x_n1,
                                      dptr<double>(ctx->visc_surface), dptr<double>(ctx->ext_visc),
                                      dptr<uint8_t>(ctx->exposed), dptr<uint8_t>(ctx->peripodial), dt,
                                      dptr<double>(ctx->qbuf), dptr<double>(ctx->abar2), ctx->stream));
            ctx->launches += 5;
            std::swap(ctx->abar, ctx->abar2);
        }
    }
    TF_CK(cudaMemcpyAsync(dL_drates, ctx->dLdr.p, sizeof(double) * 3 * E, cudaMemcpyDeviceToHost, ctx->stream));
    if (dL_dx0) TF_CK(cudaMemcpyAsync(dL_dx0, ctx->abar.p, bx, cudaMemcpyDeviceToHost, ctx->stream));
    const int rc2 = call_end(ctx, st);
    return rc2 != TF_OK ? rc2 : st->status;
}

const char* tf_last_error(tf_ctx* ctx) { return ctx ? ctx->last_error : g_create_error; }

}  // extern "C"
