// Drop-in replacement of the reference's Bem::ColocSimPin (Bem/Simulation/ColocSimPin.hpp:13-66): a bubble
// sitting on the wall x = 0 whose contact line (the vertices on the wall) is pinned to the wall and
// slides along it with a contact-angle drift velocity.  The last N_pin vertices of the mesh are the
// contact line.  Assembly with the exchanged pinned columns, the solve, the velocities and the drift
// run on the GPU (bem_set_pinned, include/bem_b200.h); the contact-line-preserving remesh runs on the
// host with the user's mesh library, as in the reference.
//
// The reference header shares its include guard with ColocSim.hpp (COLOCSIM_HPP), so a translation
// unit there sees only one of the two classes; this header has its own guard, and code that includes
// only ColocSimPin.hpp compiles against either.
#ifndef COLOCSIMPIN_HPP
#define COLOCSIMPIN_HPP

#include <iostream>
#include <vector>

#include "LinLinSim.hpp"

#include <Eigen/Dense>

namespace Bem {

class ColocSimPin : public LinLinSim {
public:
    // The constructors move the vertices with |x| < 1e-5 to the end of the vertex list and set their
    // x to 0 (set_x_boundary); the second one permutes phi_init and psi_init along and takes them as
    // the initial state (ColocSimPin.hpp:17-50).
    ColocSimPin(Mesh const& initial, real p_inf = 1.0, real epsilon = 1.0, real sigma = 0.0, real gamma = 1.0,
                real (*pressurefield)(vec3 x, real t) = &default_field)
        : LinLinSim(initial, p_inf, epsilon, sigma, gamma, pressurefield), N_pin(0), index(0) {
        N_pin = set_x_boundary(mesh);
    }

    ColocSimPin(Mesh const& initial, PotVec phi_init, PotVec psi_init, real p_inf = 1.0, real epsilon = 1.0,
                real sigma = 0.0, real gamma = 1.0, real (*pressurefield)(vec3 x, real t) = &default_field)
        : LinLinSim(initial, p_inf, epsilon, sigma, gamma, pressurefield), N_pin(0), index(0) {
        N_pin = set_x_boundary(mesh, phi_init, psi_init);
        set_phi(phi_init);
        set_psi(psi_init);
    }

    virtual ~ColocSimPin() {}

    // G and H with the last N_pin columns exchanged (G(:,j) = -H(:,j), H(:,j) = -G(:,j)) after the
    // 4 pi rule (ColocSimPin.cpp:25-118), assembled on the GPU
    virtual void assemble_matrices(Eigen::MatrixXd& G, Eigen::MatrixXd& H, Mesh const& m) const override;

    // velocities with the drift velocity at the pinned vertices; pot receives the solved potential there
    // (ColocSimPin.cpp:139-194), on the GPU
    virtual CoordVec position_t(Mesh const& m, PotVec& pot) const override;

    // remeshing that keeps the contact line on the old one (ColocSimPin.cpp:289-619)
    virtual void remesh(real L) override;

    size_t N_pin;
    size_t index;  // counter of the boundary-projection exports of remesh

    void rearrange_boundary(Mesh& M, std::vector<bool> bound) const;
    size_t set_x_boundary(Mesh& M, PotVec& phi_t, PotVec& psi_t) const;
    size_t set_x_boundary(Mesh& M) const;

protected:
    virtual void configure_context(bem_ctx* c) const override;
};

}  // namespace Bem

#endif  // COLOCSIMPIN_HPP
