// Parity driver for the pinned-bubble class ColocSimPin (test infrastructure).  The same source is
// compiled twice: against the reference's own Bem::ColocSimPin (its ColocSimPin.cpp, CPU, Eigen-API
// shim) and against the drop-in ColocSimPin over libbem_b200.so.  A hemisphere on the wall x = 0
// (contact line on the wall), the wall image on (MIRROR_MESH default), a host pressure-field callback,
// the LU solver (set_bcgstab(false)) so that both builds solve to rounding; a first block of RK4 (fixed
// and adaptive dt) and Euler steps, then blocks that start with the contact-line-preserving remesh.
// Usage: pinned_check <in.ply> <out_prefix>; writes <out_prefix>-<k>.ply after each block and prints
// the pinned count and the potential at the pinned vertices.
#include <cmath>
#include <cstdio>
#include <iostream>
#include <string>

#include "Bem/Mesh/MeshIO.hpp"
#include "Bem/Simulation/ColocSimPin.hpp"

using namespace Bem;

static real field(vec3 x, real t) { return -0.3 * std::sin(0.7 * t + 0.2 * x.x); }

int main(int argc, char* argv[]) {
    if (argc != 3) {
        std::cerr << "usage: pinned_check <in.ply> <out_prefix>" << std::endl;
        return 1;
    }
    Mesh M;
    import_ply(argv[1], M);
    const std::string out = argv[2];
    ColocSimPin sim(M, 1.0, 1.4, 0.0, 1.4, &field);
    sim.set_bcgstab(false);
    sim.set_phi(0.05);
    sim.set_damping_factor(0.2);
    sim.set_minimum_element_size(0.1);
    sim.set_maximum_element_size(0.9);
    sim.set_min_dt(5e-3);
    for (int k = 0; k < 3; ++k) {
        if (k > 0) sim.remesh(0.3);
        sim.evolve_system_RK4(2e-3, true);
        sim.evolve_system_RK4(2e-3, false);
        sim.evolve_system(2e-3, false);
        std::printf("block %d time %.17g volume %.17g verts %zu npin %zu\n", k, sim.get_time(), sim.get_volume(),
                    sim.mesh.verts.size(), sim.N_pin);
        for (size_t i = sim.mesh.verts.size() - sim.N_pin; i < sim.mesh.verts.size(); ++i)
            std::printf("pinned %d %zu %.17g %.17g %.17g %.17g\n", k, i, sim.mesh.verts[i].x, sim.mesh.verts[i].y,
                        sim.mesh.verts[i].z, sim.get_phi(i));
        sim.export_mesh(out + "-" + std::to_string(k) + ".ply");
    }
    return 0;
}
