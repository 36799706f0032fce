// capi_host.cpp -- a plain C++ host of the C ABI (include/tf_b200.h), linked against
// libtf_b200.so the way a C++ simulator links it: no Python, no CUDA or torch headers.
//
// It reads one tissue from a little-endian binary file, runs n implicit time steps
// (tf_time_step: growth prologue + Newton step) and writes the positions after the last step
// and the Newton iteration count of every step. tests/test_capi_host.py builds it with g++,
// feeds it the small rectangle and compares the output with the oracle.
//
// Input file, in order: int32 N, E, n_steps; double dt, newton_tol; int32 conn[E*6];
// double xref[E*18], x[N*3], lambda[E], mu[E], eta[E]; uint8 fixed[N*3]; double ext_visc[N*3],
// rates[E*3], angles[E]; uint8 exposed[E], peripodial[E].
// Output file: double x[N*3]; int32 newton_iters[n_steps].
#include <cstdint>
#include <cstdio>
#include <vector>

#include "tf_b200.h"

namespace {

template <class T>
bool read_n(FILE* f, std::vector<T>& v, size_t n) {
    v.resize(n);
    return n == 0 || std::fread(v.data(), sizeof(T), n, f) == n;
}

int fail(const char* what, int rc, tf_ctx* ctx) {
    std::fprintf(stderr, "%s failed: status %d (%s)\n", what, rc, tf_last_error(ctx));
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
        return 2;
    }
    FILE* in = std::fopen(argv[1], "rb");
    if (!in) return 2;
    int32_t hdr[3];
    double dtol[2];
    if (std::fread(hdr, sizeof(int32_t), 3, in) != 3 || std::fread(dtol, sizeof(double), 2, in) != 2) return 2;
    const size_t N = (size_t)hdr[0], E = (size_t)hdr[1];
    const int n_steps = hdr[2];
    std::vector<int32_t> conn;
    std::vector<double> xref, x, lam, mu, eta, ext, rates, angles;
    std::vector<uint8_t> fixed, exposed, peri;
    const bool ok = read_n(in, conn, E * 6) && read_n(in, xref, E * 18) && read_n(in, x, N * 3) && read_n(in, lam, E) &&
                    read_n(in, mu, E) && read_n(in, eta, E) && read_n(in, fixed, N * 3) && read_n(in, ext, N * 3) &&
                    read_n(in, rates, E * 3) && read_n(in, angles, E) && read_n(in, exposed, E) && read_n(in, peri, E);
    std::fclose(in);
    if (!ok) return 2;

    std::printf("%s\n", tf_version());
    tf_params p;
    tf_default_params(&p);
    p.newton_tol = dtol[1];
    p.krylov_rtol = 1e-14;
    tf_mesh_desc mesh = {(int32_t)N, (int32_t)E, conn.data(), xref.data()};
    tf_ctx* ctx = nullptr;
    int rc = tf_create(&mesh, &p, &ctx);
    if (rc != TF_OK) return fail("tf_create", rc, nullptr);
    if ((rc = tf_set_material(ctx, lam.data(), mu.data(), eta.data())) != TF_OK) return fail("tf_set_material", rc, ctx);
    if ((rc = tf_set_boundary(ctx, fixed.data(), ext.data(), nullptr, 0)) != TF_OK) return fail("tf_set_boundary", rc, ctx);
    if ((rc = tf_set_growth(ctx, nullptr, rates.data(), angles.data(), exposed.data(), peri.data())) != TF_OK)
        return fail("tf_set_growth", rc, ctx);
    std::vector<int32_t> iters;
    for (int s = 0; s < n_steps; ++s) {
        tf_step_stats st;
        rc = tf_time_step(ctx, x.data(), dtol[0], x.data(), &st);
        if (rc != TF_OK) return fail("tf_time_step", rc, ctx);
        iters.push_back(st.newton_iters);
        std::printf("step %d: %d Newton iterations, %d BiCGStab iterations, %.3f ms\n", s, st.newton_iters,
                    st.krylov_iters_total, st.ms_total);
    }
    tf_destroy(ctx);
    FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 2;
    std::fwrite(x.data(), sizeof(double), x.size(), out);
    std::fwrite(iters.data(), sizeof(int32_t), iters.size(), out);
    std::fclose(out);
    return 0;
}
