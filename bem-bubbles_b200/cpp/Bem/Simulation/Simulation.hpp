// Drop-in replacement of the reference's Bem::Simulation (Bem/Simulation/Simulation.hpp:26-210) whose
// hot path runs on the GPU through libbem_b200.so (include/bem_b200.h).
//
// The public interface -- constructor defaults, setters and getters, assemble/solve, the public
// member `mesh` -- keeps the reference's signatures so that its drivers compile unchanged.  The host
// copies of the state (mesh.verts, phi, psi, time) stay authoritative between calls; every hot-path
// call uploads them to the context's device state and reads the results back.
//
// Include root: this header is found as "Bem/Simulation/Simulation.hpp" with this directory's parent
// (cpp/) ahead of the user's bem-bubbles tree on the include path; Bem/basic, Bem/Mesh and
// Bem/Integration headers and Eigen come from that tree.
#ifndef SIMULATION_HPP
#define SIMULATION_HPP

#include <iostream>
#include <string>
#include <vector>

#include "Bem/basic/Bem.hpp"
#include "Bem/Mesh/Mesh.hpp"
#include "Bem/Integration/Integrator.hpp"
#include "Bem/Integration/quadrature.hpp"

#include <Eigen/Dense>

#include <cassert>

struct bem_ctx;

namespace Bem {

// functions for translating between PotVec and Eigen::VectorXd (Simulation.hpp:20-21)
std::vector<real> make_copy(Eigen::VectorXd const& vec);
Eigen::VectorXd make_copy(std::vector<real> const& vec);

// default pressure field (Simulation.hpp:24): zero everywhere
real default_field(vec3 x, real t);

class Simulation {
public:
    Simulation(Mesh const& initial, real p_inf = 1.0, real epsilon = 1.0, real sigma = 0.0, real gamma = 1.0,
               real (*pressurefield)(vec3 x, real t) = &default_field);
    virtual ~Simulation();
    Simulation(Simulation const&) = delete;
    Simulation& operator=(Simulation const&) = delete;

    virtual size_t phi_dim() const = 0;
    virtual size_t psi_dim() const = 0;

    virtual void assemble_matrices(Eigen::MatrixXd& G, Eigen::MatrixXd& H, Mesh const& m) const = 0;
    void assemble_matrices_prop(Eigen::MatrixXd& G, Eigen::MatrixXd& H) const { assemble_matrices(G, H, mesh); }

    // solving the system G*psi = H_phi for psi (Simulation.cpp:40-71), on the GPU
    Eigen::VectorXd solve_system(Eigen::MatrixXd const& G, Eigen::VectorXd const& H_phi) const;

    // psi from the current state (Simulation.hpp:73-77)
    void compute_psi();

    virtual void evolve_system(real dp, bool fixdt = false) = 0;

    void export_mesh(std::string fname) const;
    void export_mesh_values(std::string fname, std::vector<real> values) const;

    void set_phi(std::vector<real> const& value) {
        assert(value.size() == phi_dim());
        phi = make_copy(value);
    }
    void set_psi(std::vector<real> const& value) {
        assert(value.size() == psi_dim());
        psi = make_copy(value);
    }
    void set_phi(real value) { phi.fill(value); }
    void set_V_0(real value) { V_0 = value; }
    real get_phi(size_t index) const {
        assert(index < phi_dim());
        return phi((Eigen::Index)index);
    }
    real get_psi(size_t index) const {
        assert(index < psi_dim());
        return psi((Eigen::Index)index);
    }
    void set_time(real const& value) { time = value; }
    real get_time() const { return time; }
    real get_volume() const { return volume(mesh); }
    const std::vector<vec3>& get_vertices() { return mesh.verts; }
    std::vector<real> get_psi() { return make_copy(psi); }
    std::vector<real> get_phi() { return make_copy(phi); }
    void set_min_dt(real value) { min_dt = value; }
    void set_dp_balance(real value) { dp_balance = value; }
    void set_bcgstab(bool value) { bicgstab = value; }
    void set_num_threads(size_t num) { num_threads = num; }
    // Host-side integrator rules (used by subclasses that integrate on the host).  The GPU path
    // always integrates with the 7-point triangle rule and 7-point Gauss, the rules the reference
    // constructor selects (Simulation.hpp:44-45).
    void set_quadrature(std::vector<quadrature_2d> const& quad) { inter.set_quadrature(quad); }
    void set_quadrature(std::vector<quadrature_1d> const& quad) { inter.set_quadrature(quad); }

    // mixed precision (FP64 refinement on a low-precision inverse) instead of the FP64 solver
    void set_mixed_precision(bool value) { mixed = value; }
    // the GPU solver's counters since the context was created (bem_stats; all zero before the first step)
    void gpu_stats(int64_t* solves, int64_t* iterations, int64_t* ns_steps, int64_t* refreshes,
                   int64_t* fp64_fallbacks, int64_t* gmres_fallbacks) const;

protected:
    real get_dt(real dp, std::vector<vec3> const& gradients, std::vector<real> const& grad_potential) const;
    real potential_t(real grad_squared, real volume, real kappa, vec3 pos, real t) const;

    // physical constants, initial volume, far field, time stepping (Simulation.hpp:180-197)
    real p_inf, epsilon, sigma, gamma;
    real V_0;
    real (*pressurefield)(vec3 x, real t);
    real time;
    real min_dt;
    real dp_balance;
    bool bicgstab;
    size_t num_threads;
    bool mixed = false;

public:
    Mesh mesh;

protected:
    Integrator inter;
    // potential and its normal derivative on the surface, the reference's types (Simulation.hpp:204-208),
    // so that subclasses written against the reference (ColocSimPin) compile unchanged
    Eigen::VectorXd psi;
    Eigen::VectorXd phi;

    // ---- GPU context (one per simulation object) and its synchronisation with the host state
    mutable bem_ctx* ctx_ = nullptr;
    mutable std::vector<Triplet> ctx_trigs_;  // topology the context was built for
    bool image_wall_ = false;                 // wall image at x = 0 (the reference's MIRROR_MESH)
    bem_ctx* device_ctx() const;              // the context, created on first use (no mesh needed)
    bem_ctx* context(Mesh const& m) const;    // context whose topology is m's (rebuilt on change)
    virtual void configure_context(bem_ctx* c) const { (void)c; }  // subclass settings (pinned vertices)
    void push_state() const;                  // host mesh.verts, phi, psi, time, V_0, params -> device
    void pull_state();                        // device -> host
    void check(int status) const;             // status -> exception (std::out_of_range for x < 0)
};

}  // namespace Bem

#endif  // SIMULATION_HPP
