// Command-line harness around the reference's own hot path (Bem::ColocSim and friends),
// compiled from the reference sources against the oracle's Eigen-API shim.  Used to
// (1) generate golden vectors that pin the C restatement in bem_oracle.c and
// (2) time the reference's CPU path as the baseline arm of bench.py.
// Test infrastructure only: nothing in the product links or calls it.
//
// usage: ref_harness <action> <in.bin> <out.bin> [key=value ...]
//   in.bin : int64 N, int64 M, N*3 float64 vertices, M*3 int64 triangles, N float64 phi
//   actions:
//     assemble   -> G (N*N, column-major), H (N*N)
//     solve      -> psi_l = solve_system(G, H*phi)                (N)
//     position_t -> velocities (N*3)
//     pot_t      -> pot_t_multi(mesh, position_t(mesh, phi), t)   (N)
//     rk4        -> after each of `steps` RK4 steps: verts (N*3), phi (N), psi (N), time (1)
//     euler      -> same record layout as rk4, using evolve_system
//     stages     -> `steps` repetitions of one RK4 stage (position_t + pot_t_multi); writes the
//                   seconds of each repetition
//     rk4_timed  -> `warm` untimed RK4 steps (evolve_system_RK4), then up to `steps` timed ones (no new
//                   step once `budget` seconds of timed steps are spent, budget=0: no limit); writes
//                   the count K, per timed step: seconds, BiCGSTAB solves, BiCGSTAB iterations
//                   (timing sample of the reference's own step), then the final verts, phi, psi, time
//     exterior   -> exterior_pot(points) (LinLinSim.cpp:479-485: assemble, solve, compute_exterior_pot)
//     exterior_direct -> compute_exterior_pot(points, mesh, phi, psi) with the given psi
//   in.bin for exterior*: then int64 P, P*3 float64 points, and for exterior_direct N float64 psi
//   keys: p_inf epsilon sigma gamma V0 amp omega phase dt steps warm budget fixdt lu threads timing
//   amp/omega/phase define the far-field pressure p(x,t) = amp*sin(omega*t + phase).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <map>
#include <string>
#include <vector>

#include "Bem/Simulation/ColocSim.hpp"
#include <Eigen/IterativeLinearSolvers>

using namespace Bem;

static double g_amp = 0.0, g_omega = 0.0, g_phase = 0.0;
static real field(vec3 x, real t) {
    (void)x;
    return g_amp * std::sin(g_omega * t + g_phase);
}

static void die(const char* m) {
    std::fprintf(stderr, "ref_harness: %s\n", m);
    std::exit(2);
}

int main(int argc, char** argv) {
    if (argc < 4) die("usage: ref_harness <action> <in.bin> <out.bin> [key=value ...]");
    std::string action = argv[1];
    std::map<std::string, double> kv = {{"p_inf", 1.0}, {"epsilon", 1.0}, {"sigma", 0.0}, {"gamma", 1.0},
                                        {"V0", -1.0},   {"amp", 0.0},     {"omega", 0.0}, {"phase", 0.0},
                                        {"dt", 1e-3},   {"steps", 1},     {"fixdt", 1},   {"lu", 1},
                                        {"threads", 1}, {"t", 0.0},       {"timing", 0},  {"warm", 0},
                                        {"budget", 0.0}};
    for (int i = 4; i < argc; ++i) {
        const char* eq = std::strchr(argv[i], '=');
        if (!eq) die("bad key=value");
        kv[std::string(argv[i], (size_t)(eq - argv[i]))] = std::atof(eq + 1);
    }
    FILE* f = std::fopen(argv[2], "rb");
    if (!f) die("cannot open input");
    int64_t N = 0, M = 0;
    if (std::fread(&N, 8, 1, f) != 1 || std::fread(&M, 8, 1, f) != 1) die("bad header");
    std::vector<double> xyz((size_t)N * 3), phi((size_t)N);
    std::vector<int64_t> tri((size_t)M * 3);
    if (std::fread(xyz.data(), 8, xyz.size(), f) != xyz.size()) die("short verts");
    if (std::fread(tri.data(), 8, tri.size(), f) != tri.size()) die("short trigs");
    if (std::fread(phi.data(), 8, phi.size(), f) != phi.size()) die("short phi");
    std::vector<double> pts, psi_in;
    if (action == "exterior" || action == "exterior_direct") {
        int64_t P = 0;
        if (std::fread(&P, 8, 1, f) != 1) die("no points");
        pts.resize((size_t)P * 3);
        if (std::fread(pts.data(), 8, pts.size(), f) != pts.size()) die("short points");
        if (action == "exterior_direct") {
            psi_in.resize((size_t)N);
            if (std::fread(psi_in.data(), 8, psi_in.size(), f) != psi_in.size()) die("short psi");
        }
    }
    std::fclose(f);

    Mesh mesh;
    for (int64_t i = 0; i < N; ++i) mesh.verts.push_back(vec3(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
    for (int64_t j = 0; j < M; ++j)
        mesh.trigs.push_back(Triplet((size_t)tri[3 * j], (size_t)tri[3 * j + 1], (size_t)tri[3 * j + 2]));

    g_amp = kv["amp"];
    g_omega = kv["omega"];
    g_phase = kv["phase"];
    ColocSim sim(mesh, kv["p_inf"], kv["epsilon"], kv["sigma"], kv["gamma"], &field);
    sim.set_phi(phi);
    if (kv["V0"] > 0.0) sim.set_V_0(kv["V0"]);
    sim.set_bcgstab(kv["lu"] == 0.0);
    sim.set_num_threads((size_t)kv["threads"]);
    sim.set_time(kv["t"]);

    FILE* o = std::fopen(argv[3], "wb");
    if (!o) die("cannot open output");
    auto put = [&](const double* p, size_t n) {
        if (std::fwrite(p, 8, n, o) != n) die("write failed");
    };
    auto t0 = std::chrono::steady_clock::now();
    double t_asm = 0.0;
    if (action == "assemble") {
        Eigen::MatrixXd G, H;
        sim.assemble_matrices(G, H, sim.mesh);
        put(G.data(), (size_t)G.size());
        put(H.data(), (size_t)H.size());
    } else if (action == "solve") {
        Eigen::MatrixXd G, H;
        auto a0 = std::chrono::steady_clock::now();
        sim.assemble_matrices(G, H, sim.mesh);
        t_asm = std::chrono::duration<double>(std::chrono::steady_clock::now() - a0).count();
        Eigen::VectorXd b = H * make_copy(phi);
        Eigen::VectorXd x = sim.solve_system(G, b);
        put(x.data(), (size_t)x.size());
    } else if (action == "position_t") {
        PotVec p = phi;
        CoordVec v = sim.position_t(sim.mesh, p);
        for (auto const& e : v) {
            double d[3] = {e.x, e.y, e.z};
            put(d, 3);
        }
    } else if (action == "pot_t") {
        PotVec p = phi;
        CoordVec v = sim.position_t(sim.mesh, p);
        PotVec r = sim.pot_t_multi(sim.mesh, v, kv["t"]);
        put(r.data(), r.size());
    } else if (action == "rk4" || action == "euler") {
        int steps = (int)kv["steps"];
        for (int s = 0; s < steps; ++s) {
            if (action == "rk4")
                sim.evolve_system_RK4(kv["dt"], kv["fixdt"] != 0.0);
            else
                sim.evolve_system(kv["dt"], kv["fixdt"] != 0.0);
            for (auto const& e : sim.mesh.verts) {
                double d[3] = {e.x, e.y, e.z};
                put(d, 3);
            }
            PotVec ph = sim.get_phi(), ps = sim.get_psi();
            put(ph.data(), ph.size());
            put(ps.data(), ps.size());
            double tm = sim.get_time();
            put(&tm, 1);
        }
    } else if (action == "rk4_timed") {
        const int warm = (int)kv["warm"], steps = (int)kv["steps"];
        const double budget = kv["budget"];
        for (int s = 0; s < warm; ++s) sim.evolve_system_RK4(kv["dt"], kv["fixdt"] != 0.0);
        std::vector<double> recs;
        double spent = 0.0;
        for (int s = 0; s < steps && (budget <= 0.0 || spent < budget); ++s) {
            const long long s0 = Eigen::shim_detail::g_bicgstab_solves, i0 = Eigen::shim_detail::g_bicgstab_iters;
            auto a0 = std::chrono::steady_clock::now();
            sim.evolve_system_RK4(kv["dt"], kv["fixdt"] != 0.0);
            const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - a0).count();
            spent += sec;
            recs.push_back(sec);
            recs.push_back((double)(Eigen::shim_detail::g_bicgstab_solves - s0));
            recs.push_back((double)(Eigen::shim_detail::g_bicgstab_iters - i0));
        }
        const double count = (double)(recs.size() / 3);
        put(&count, 1);
        put(recs.data(), recs.size());
        for (auto const& e : sim.mesh.verts) {
            double d[3] = {e.x, e.y, e.z};
            put(d, 3);
        }
        PotVec ph = sim.get_phi(), ps = sim.get_psi();
        put(ph.data(), ph.size());
        put(ps.data(), ps.size());
        double tm = sim.get_time();
        put(&tm, 1);
    } else if (action == "stages") {
        int steps = (int)kv["steps"];
        PotVec p = phi;
        for (int s = 0; s < steps; ++s) {
            auto a0 = std::chrono::steady_clock::now();
            CoordVec v = sim.position_t(sim.mesh, p);
            PotVec r = sim.pot_t_multi(sim.mesh, v, kv["t"]);
            double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - a0).count();
            put(&sec, 1);
        }
    } else if (action == "exterior" || action == "exterior_direct") {
        CoordVec pos;
        for (size_t i = 0; i < pts.size() / 3; ++i) pos.push_back(vec3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]));
        PotVec r = action == "exterior" ? sim.exterior_pot(pos) : compute_exterior_pot(pos, sim.mesh, phi, psi_in);
        put(r.data(), r.size());
    } else {
        die("unknown action");
    }
    std::fclose(o);
    double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (kv["timing"] != 0.0) std::fprintf(stderr, "TIMING total_s=%.6f assemble_s=%.6f\n", el, t_asm);
    return 0;
}
