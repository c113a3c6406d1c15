// Drop-in replacement of the reference's Bem::LinLinSim (Bem/Simulation/LinLinSim.hpp:19-90):
// linear elements for phi and psi, RK4 and Euler time stepping on the GPU.
#ifndef LINLINSIM_HPP
#define LINLINSIM_HPP

#include <iostream>
#include <limits>
#include <vector>

#include "Simulation.hpp"

#include <Eigen/Dense>

// The reference selects linear elements and the wall image at compile time (LinLinSim.hpp:12-13).
// LINEAR must stay true (the GPU path integrates flat triangles); MIRROR_MESH keeps the reference's
// default and may be predefined to false to simulate free-space bubbles.
#define LINEAR true
#ifndef MIRROR_MESH
#define MIRROR_MESH true
#endif

namespace Bem {

PotVec compute_exterior_pot(CoordVec const& pos, Mesh M, PotVec phi, PotVec psi);

class LinLinSim : public Simulation {
public:
    // inline so that MIRROR_MESH takes the value of the including translation unit
    LinLinSim(Mesh const& initial, real p_inf = 1.0, real epsilon = 1.0, real sigma = 0.0, real gamma = 1.0,
              real (*pressurefield)(vec3 x, real t) = &default_field)
        : Simulation(initial, p_inf, epsilon, sigma, gamma, pressurefield),
          eps(1e-2),
          damping_factor(0.0),
          min_elm_size(0.0),
          max_elm_size(std::numeric_limits<real>::max()) {
        phi = Eigen::VectorXd::Zero((Eigen::Index)phi_dim());
        psi = Eigen::VectorXd::Zero((Eigen::Index)psi_dim());
        image_wall_ = MIRROR_MESH;
        curvature_params = curvature_param();
    }
    virtual ~LinLinSim() {}

    virtual size_t phi_dim() const override { return mesh.verts.size(); }
    virtual size_t psi_dim() const override { return mesh.verts.size(); }

    virtual void evolve_system(real dp, bool fixdt = false) override;
    virtual void evolve_system_RK4(real dp, bool fixdt = false);

    virtual void remesh(real L);

    void set_damping_factor(real value) { damping_factor = value; }
    void set_minimum_element_size(real value) { min_elm_size = value; }
    void set_maximum_element_size(real value) { max_elm_size = value; }

    std::vector<real> kappa(Mesh const& m) const;

    virtual CoordVec position_t(Mesh const& m, PotVec& pot) const;
    PotVec pot_t(Mesh const& m, CoordVec const& gradients, real t) const;
    PotVec pot_t_multi(Mesh const& m, CoordVec const& gradients, real t) const;

    PotVec exterior_pot(CoordVec const& positions) const;

    CoordVec nopenetration(real eps, real dt, CoordVec const& x0, CoordVec& c) const;

protected:
    real eps;

    void test_negative() const;

    // RK4 and Euler through the virtual position_t / pot_t_multi, for subclasses that override them
    // (the reference's own step sequence, LinLinSim.cpp:194-284); ColocSim itself steps on the GPU
    void evolve_rk4_virtual(real dp, bool fixdt);
    void evolve_euler_virtual(real dp, bool fixdt);

    std::vector<vec3> generate_tangent_gradients(Mesh const& m, std::vector<real> const& pot) const;

    std::vector<real> curvature_param() const;
    void update_curvature_params();  // damped, clamped curvature_params before a remesh

    real damping_factor;
    real min_elm_size, max_elm_size;
    PotVec curvature_params;
};

}  // namespace Bem

#endif  // LINLINSIM_HPP
