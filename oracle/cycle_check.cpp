// Remesh-and-step cycle of the reference's oscillations driver (oscillations.cpp:83-121), timed per part
// (test infrastructure).  Compiled against the reference's classes (CPU) and against the drop-in
// (GPU steps, GPU ray casting in the remesh projection).  Each iteration: export_mesh, remesh(0.12),
// four Euler steps with dp = 0.02 -- the driver's loop.  The driver's bubble sits at the origin,
// centred on its own wall image (a singular system); here it is moved to x = 3 (argument) so that the
// system is well posed.  Usage: cycle_check <ico.ply> <iterations> <x_offset> [mixed]
// Prints one line per iteration and a mean line over the iterations after the first.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>

#include <sys/resource.h>

#include "Bem/Mesh/MeshIO.hpp"
#include "Bem/Simulation/ColocSim.hpp"

using namespace Bem;
using clk = std::chrono::steady_clock;

static double ms(clk::time_point a, clk::time_point b) { return std::chrono::duration<double, std::milli>(b - a).count(); }

// the process's CPU time (user + system, ms) and context switches (voluntary, involuntary) so far: a
// slow iteration whose wall time the CPU time does not explain, with involuntary switches, was
// waiting for the host's cores, not for its own work
struct Usage {
    double cpu_ms;
    long vcsw, ivcsw;
};
static Usage usage() {
    rusage r{};
    getrusage(RUSAGE_SELF, &r);
    const double cpu = (r.ru_utime.tv_sec + r.ru_stime.tv_sec) * 1e3 + (r.ru_utime.tv_usec + r.ru_stime.tv_usec) * 1e-3;
    return {cpu, r.ru_nvcsw, r.ru_nivcsw};
}

static real K, Omega, Pa;
static real waveform(vec3 x, real t) { return Pa * std::sin(K * x.x - Omega * t); }

int main(int argc, char* argv[]) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: cycle_check <ico.ply> <iterations> <x_offset> [mixed]\n");
        return 2;
    }
    const int iters = std::atoi(argv[2]);
    // the driver's physical set-up (oscillations.cpp:30-67) at radius 3e-6 m, 5e4 Pa
    const real radius = 3e-6, pressure = 5e4, p_infty = 101325.0, sigma = 0.07275, c = 1481.0, f = 20e3;
    const real p_vap = 2300.0, rho = 998.2067, p_ref = p_infty - p_vap, t_ref = radius * std::sqrt(rho / p_ref);
    const real Sigma = sigma / (radius * p_ref), P_gas0 = 1.0 + 2.0 * Sigma, Gamma = 7.0 / 5.0;
    Omega = 2.0 * M_PI * f * t_ref;
    K = 2.0 * M_PI / (c / f / radius);
    Pa = pressure / p_ref;
    Mesh M;
    import_ply(argv[1], M);
    M.translate(vec3(std::atof(argv[3]), 0.0, 0.0));
    ColocSim sim(M, 1.0, P_gas0, Sigma, Gamma, &waveform);
    sim.set_min_dt(0.1 * M_PI / Omega);
    sim.set_phi(0.0);
    sim.set_damping_factor(0.2);
    sim.set_minimum_element_size(0.1);
    sim.set_maximum_element_size(0.9);
#ifdef CYCLE_DROPIN
    if (argc > 4 && std::string(argv[4]) == "mixed") sim.set_mixed_precision(true);
#endif
    double te = 0, tr = 0, ts = 0;
    for (int i = 0; i < iters; ++i) {
        const Usage u0 = usage();
        const auto t0 = clk::now();
        sim.export_mesh("cycle-mesh.ply");
        const auto t1 = clk::now();
        sim.remesh(0.12);
        const auto t2 = clk::now();
#ifdef CYCLE_DROPIN
        int64_t s0[6], s1[6];
        sim.gpu_stats(&s0[0], &s0[1], &s0[2], &s0[3], &s0[4], &s0[5]);
#endif
        for (int j = 0; j < 4; ++j) sim.evolve_system(0.02);
        const auto t3 = clk::now();
        const Usage u1 = usage();
        std::printf("iteration %d verts %zu export_ms %.2f remesh_ms %.2f steps_ms %.2f cpu_ms %.2f vcsw %ld ivcsw %ld", i,
                    sim.mesh.verts.size(), ms(t0, t1), ms(t1, t2), ms(t2, t3), u1.cpu_ms - u0.cpu_ms, u1.vcsw - u0.vcsw,
                    u1.ivcsw - u0.ivcsw);
#ifdef CYCLE_DROPIN
        // the GPU solver's work in this iteration's four steps
        sim.gpu_stats(&s1[0], &s1[1], &s1[2], &s1[3], &s1[4], &s1[5]);
        std::printf(" solves %lld iters %lld ns_steps %lld refreshes %lld fp64_fallbacks %lld gmres_fallbacks %lld",
                    (long long)(s1[0] - s0[0]), (long long)(s1[1] - s0[1]), (long long)(s1[2] - s0[2]),
                    (long long)(s1[3] - s0[3]), (long long)(s1[4] - s0[4]), (long long)(s1[5] - s0[5]));
#endif
        std::printf("\n");
        if (i > 0) {
            te += ms(t0, t1);
            tr += ms(t1, t2);
            ts += ms(t2, t3);
        }
    }
    const int n = iters - 1;
    if (n > 0)
        std::printf("mean iterations %d export_ms %.2f remesh_ms %.2f steps_ms %.2f total_ms %.2f verts %zu time %.17g\n",
                    n, te / n, tr / n, ts / n, (te + tr + ts) / n, sim.mesh.verts.size(), sim.get_time());
    return 0;
}
