// Parity driver for the drop-in C++ classes (test infrastructure).  The same source is compiled
// twice: against the reference's own Bem::Simulation / LinLinSim / ColocSim (CPU, Eigen-API shim)
// and against the drop-in classes over libbem_b200.so.  It exercises the public interface the
// reference's drivers use on a well-posed problem: a perturbed bubble well away from the wall
// image (MIRROR_MESH keeps its default), a host pressure-field callback, remeshing
// between steps, RK4 and Euler steps, the LU solver (set_bcgstab(false)) so that both builds solve to
// rounding.  Usage: dropin_check <in.ply> <out_prefix>; writes <out_prefix>-<k>.ply after each block.
#include <cmath>
#include <cstdio>
#include <iostream>
#include <string>

#include "Bem/Mesh/MeshIO.hpp"
#include "Bem/Simulation/ColocSim.hpp"

using namespace Bem;

static real field(vec3 x, real t) { return -0.3 * std::sin(0.7 * t + 0.2 * x.x); }

#ifdef CHECK_SUBCLASS
// A user's class derived from ColocSim (built with -DCHECK_SUBCLASS against the drop-in): the drop-in
// steps such classes through their virtual position_t and pot_t_multi, stage by stage, in the
// reference's RK4/Euler call sequence; the results must agree with ColocSim's own all-GPU step.
struct UserSim : ColocSim {
    using ColocSim::ColocSim;
};
using Sim = UserSim;
#else
using Sim = ColocSim;
#endif

int main(int argc, char* argv[]) {
    if (argc != 3) {
        std::cerr << "usage: dropin_check <in.ply> <out_prefix>" << std::endl;
        return 1;
    }
    Mesh M;
    import_ply(argv[1], M);
    const std::string out = argv[2];
    // radial perturbation 1 + 0.02 sin(3 theta)-like, deterministic, then away from the wall
    for (vec3& v : M.verts) v = v * (1.0 + 0.02 * std::sin(3.0 * v.z + v.y));
    M.translate(vec3(3.0, 0.0, 0.0));
    Sim sim(M, 1.0, 1.4, 0.0, 1.4, &field);
    sim.set_bcgstab(false);
    sim.set_phi(0.05);
    sim.set_damping_factor(0.2);
    sim.set_minimum_element_size(0.1);
    sim.set_maximum_element_size(0.9);
    sim.set_min_dt(5e-3);
    for (int k = 0; k < 3; ++k) {
        sim.remesh(0.25);
        sim.evolve_system_RK4(2e-3, true);
        sim.evolve_system_RK4(2e-3, false);
        sim.evolve_system(2e-3, false);
        std::cout << "block " << k << " time " << sim.get_time() << " volume " << sim.get_volume() << " verts "
                  << sim.mesh.verts.size() << std::endl;
        sim.export_mesh(out + "-" + std::to_string(k) + ".ply");
    }
    // the potential off the surface (LinLinSim::exterior_pot) at a few points around the bubble
    const CoordVec probe = {vec3(3.0, 0.0, 0.0), vec3(5.0, 0.5, -0.2), vec3(3.2, 2.5, 0.4), vec3(1.0, -0.3, 1.0)};
    const PotVec ext = sim.exterior_pot(probe);
    for (size_t i = 0; i < ext.size(); ++i) std::printf("exterior %zu %.17g\n", i, ext[i]);
    return 0;
}
