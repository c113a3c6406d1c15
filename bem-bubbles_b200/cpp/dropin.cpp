// Implementation of the drop-in Bem::Simulation / LinLinSim / ColocSim (Bem/Simulation/*.hpp in this
// directory) over the C ABI of libbem_b200.so.  The per-step hot path -- assembly, solve, vertex
// velocities, Bernoulli update, RK4/Euler combination -- runs on the GPU, and so do the exterior
// potential and the projection step of remeshing; the remesh's topology edits and the PLY export stay
// on the host with the user's Bem/Mesh library, as in the reference.
#include <cmath>
#include <cstdlib>
#include <set>
#include <stdexcept>
#include <typeinfo>

#include "Bem/Simulation/ColocSim.hpp"
#include "Bem/Simulation/ColocSimPin.hpp"
#include "Bem/Integration/Integrator.hpp"
#include "Bem/Mesh/HalfedgeMesh.hpp"
#include "Bem/Mesh/MeshIO.hpp"
#include "Bem/Mesh/MeshManip.hpp"
#include "../../include/bem_b200.h"
#include "dropin_util.hpp"

namespace Bem {

std::vector<real> make_copy(Eigen::VectorXd const& vec) {
    std::vector<real> out((size_t)vec.size());
    for (size_t i = 0; i < out.size(); ++i) out[i] = vec((Eigen::Index)i);
    return out;
}

Eigen::VectorXd make_copy(std::vector<real> const& vec) {
    Eigen::VectorXd out((Eigen::Index)vec.size());
    for (size_t i = 0; i < vec.size(); ++i) out((Eigen::Index)i) = vec[i];
    return out;
}

real default_field(vec3 x, real t) {
    (void)x;
    (void)t;
    return 0.0;
}

// ------------------------------------------------------------------ Simulation
Simulation::Simulation(Mesh const& initial, real p_inf, real epsilon, real sigma, real gamma,
                       real (*pressurefield)(vec3 x, real t))
    : p_inf(p_inf),
      epsilon(epsilon),
      sigma(sigma),
      gamma(gamma),
      V_0(volume(initial)),
      pressurefield(pressurefield),
      time(0.0),
      min_dt(-1.0),
      dp_balance(3.0),
      bicgstab(true),
      num_threads(100),
      mesh(initial) {
    inter.set_quadrature(quadrature_7);
    inter.set_quadrature(gauss_7);
}

Simulation::~Simulation() {
    if (ctx_) bem_destroy(ctx_);
}

void Simulation::check(int status) const {
    if (status == BEM_OK) return;
    if (status == BEM_ERR_NEGATIVE_X) {
        std::cout << "negative values occured" << std::endl;
        throw std::out_of_range("negative values");
    }
    std::string msg = ctx_ ? bem_last_error(ctx_) : "";
    throw std::runtime_error("bem_b200 error " + std::to_string(status) + ": " + msg);
}

static double field_trampoline(const double x[3], double t, void* user) {
    auto fn = reinterpret_cast<real (*)(vec3, real)>(user);
    return fn(vec3(x[0], x[1], x[2]), t);
}

using dropin::flat;
using dropin::unflat;

bem_ctx* Simulation::device_ctx() const {
    if (!ctx_) {
        int dev = 0;
        if (const char* e = std::getenv("BEM_DEVICE")) dev = std::atoi(e);
        check(bem_create(&ctx_, dev, nullptr));
    }
    return ctx_;
}

void Simulation::gpu_stats(int64_t* solves, int64_t* iterations, int64_t* ns_steps, int64_t* refreshes,
                           int64_t* fp64_fallbacks, int64_t* gmres_fallbacks) const {
    bem_stats st{};
    if (ctx_) check(bem_get_stats(ctx_, &st));
    *solves = st.solves;
    *iterations = st.total_iters;
    *ns_steps = st.ns_steps;
    *refreshes = st.precond_refresh;
    *fp64_fallbacks = st.fp64_fallbacks;
    *gmres_fallbacks = st.gmres_fallbacks;
}

bem_ctx* Simulation::context(Mesh const& m) const {
    device_ctx();
    bem_params p;
    bem_default_params(&p);
    p.p_inf = p_inf;
    p.epsilon = epsilon;
    p.sigma = sigma;
    p.gamma = gamma;
    p.min_dt = min_dt;
    p.dp_balance = dp_balance;
    p.mirror = image_wall_ ? 1 : 0;
    p.solver = mixed ? BEM_SOLVER_MIXED : (bicgstab ? BEM_SOLVER_BICGSTAB : BEM_SOLVER_LU);
    check(bem_set_params(ctx_, &p));
    bool same = ctx_trigs_.size() == m.trigs.size();
    for (size_t j = 0; same && j < m.trigs.size(); ++j) same = ctx_trigs_[j] == m.trigs[j];
    if (!same) {
        std::vector<int64_t> t(3 * m.trigs.size());
        for (size_t j = 0; j < m.trigs.size(); ++j)
            for (size_t k = 0; k < 3; ++k) t[3 * j + k] = (int64_t)m.trigs[j][k];
        std::vector<double> x = flat(m.verts);
        check(bem_set_mesh(ctx_, (int64_t)m.verts.size(), x.data(), (int64_t)m.trigs.size(), t.data()));
        ctx_trigs_ = m.trigs;
    }
    // the reference's pressure field is any function of (x, t); the zero default needs no callback
    if (pressurefield == &default_field)
        check(bem_set_field_callback(ctx_, nullptr, nullptr));
    else
        check(bem_set_field_callback(ctx_, &field_trampoline, reinterpret_cast<void*>(pressurefield)));
    configure_context(ctx_);
    return ctx_;
}

void Simulation::push_state() const {
    bem_ctx* c = context(mesh);
    std::vector<double> x = flat(mesh.verts);
    check(bem_set_state(c, x.data(), phi.data(), psi.data(), &time));
    check(bem_set_V0(c, V_0));
}

void Simulation::pull_state() {
    std::vector<double> x(3 * mesh.verts.size());
    check(bem_get_state(ctx_, x.data(), phi.data(), psi.data(), &time));
    mesh.verts = unflat(x);
}

Eigen::VectorXd Simulation::solve_system(Eigen::MatrixXd const& G, Eigen::VectorXd const& H_phi) const {
    if ((size_t)G.rows() != mesh.verts.size())
        throw std::invalid_argument("solve_system: the system size must equal the simulation's vertex count");
    bem_ctx* c = context(mesh);
    Eigen::VectorXd x(G.rows());
    check(bem_solve_system(c, G.data(), H_phi.data(), x.data()));
    return x;
}

void Simulation::compute_psi() {
    Eigen::MatrixXd G, H;
    assemble_matrices_prop(G, H);
    psi = solve_system(G, H * phi);
}

void Simulation::export_mesh(std::string fname) const {
    export_ply_float(fname, mesh, make_copy(phi), make_copy(psi));
}

void Simulation::export_mesh_values(std::string fname, std::vector<real> values) const {
    export_ply_float(fname, mesh, values);
}

// Simulation.cpp:73-75
real Simulation::potential_t(real grad_squared, real volume, real kappa, vec3 pos, real t) const {
    return 2.0 * sigma * kappa + 0.5 * grad_squared + p_inf - epsilon * std::pow(V_0 / volume, gamma) +
           pressurefield(pos, t);
}

// Simulation.cpp:77-92
real Simulation::get_dt(real dp, std::vector<vec3> const& gradients, std::vector<real> const& grad_potential) const {
    real max_pot = 0.0, max_vel = 0.0;
    for (size_t i = 0; i < gradients.size(); ++i) {
        max_pot = std::max(std::abs(grad_potential[i]), max_pot);
        max_vel = std::max(gradients[i].norm2(), max_vel);
    }
    real dt = dp / (max_pot + dp_balance * std::sqrt(max_vel));
    if (min_dt > 0.0) dt = std::min(dt, min_dt);
    return dt;
}

// ------------------------------------------------------------------ ColocSim
void ColocSim::assemble_matrices(Eigen::MatrixXd& G, Eigen::MatrixXd& H, Mesh const& m) const {
    bem_ctx* c = context(m);
    const Eigen::Index n = (Eigen::Index)m.verts.size();
    G.resize(n, n);
    H.resize(n, n);
    std::vector<double> x = flat(m.verts);
    check(bem_assemble(c, x.data(), G.data(), H.data()));
}

// ------------------------------------------------------------------ LinLinSim
void LinLinSim::test_negative() const {
    for (vec3 const& v : mesh.verts)
        if (v.x < 0.0) {
            std::cout << "negative values occured" << std::endl;
            throw std::out_of_range("negative values");
        }
}

// ColocSim and ColocSimPin step on the GPU in one call; another subclass (a user's class overriding
// position_t or assemble_matrices) steps through its virtual functions.
static bool steps_on_gpu(LinLinSim const* s) {
    return typeid(*s) == typeid(ColocSim) || typeid(*s) == typeid(ColocSimPin);
}

void LinLinSim::evolve_system_RK4(real dp, bool fixdt) {
    if (!steps_on_gpu(this)) {
        evolve_rk4_virtual(dp, fixdt);
        return;
    }
    std::cout << "begin_RK4" << std::endl;
    test_negative();
    push_state();
    double dt = 0.0;
    int rc = bem_evolve_rk4(ctx_, dp, fixdt ? 1 : 0, &dt);
    if (rc != BEM_OK && rc != BEM_ERR_NEGATIVE_X) check(rc);
    pull_state();
    std::cout << "end_RK4" << std::endl;
    test_negative();
}

void LinLinSim::evolve_system(real dp, bool fixdt) {
    if (!steps_on_gpu(this)) {
        evolve_euler_virtual(dp, fixdt);
        return;
    }
    push_state();
    double dt = 0.0;
    check(bem_evolve_euler(ctx_, dp, fixdt ? 1 : 0, &dt));
    pull_state();
}

// The reference's RK4 step (LinLinSim.cpp:194-257) through the virtual position_t: four stages, each
// pot_t_multi, the state-dependent potential passed by reference (a subclass may update entries of it,
// as ColocSimPin does for its pinned vertices), the wall treatment, psi from the averaged velocity.
// The call sequence and the vector expressions are the reference's, so that a subclass sees the same
// calls in the same order.
void LinLinSim::evolve_rk4_virtual(real dp, bool fixdt) {
    std::cout << "begin_RK4" << std::endl;
    test_negative();
    Mesh m2 = mesh, m3 = mesh, m4 = mesh;
    const CoordVec x1 = mesh.verts;
    PotVec p1 = get_phi();
    const CoordVec k1_x = position_t(mesh, p1);
    const PotVec k1_p = pot_t_multi(mesh, k1_x, time);
    const real dt = fixdt ? dp : get_dt(dp, k1_x, k1_p);
    m2.verts = x1 + (0.5 * dt) * k1_x;
    PotVec p2 = p1 + (0.5 * dt) * k1_p;
    const CoordVec k2_x = position_t(m2, p2);
    m3.verts = x1 + (0.5 * dt) * k2_x;
    const PotVec k2_p = pot_t_multi(m2, k2_x, time);
    PotVec p3 = p1 + (0.5 * dt) * k2_p;
    const CoordVec k3_x = position_t(m3, p3);
    m4.verts = x1 + dt * k3_x;
    const PotVec k3_p = pot_t_multi(m3, k3_x, time);
    PotVec p4 = p1 + dt * k3_p;
    CoordVec k4_x = position_t(m4, p4);
    CoordVec average = (k1_x + 2.0 * k2_x + 2.0 * k3_x + k4_x) * (1.0 / 6.0);
    const PotVec pf = p1 + (dt / 6.0) * (pot_t_multi(mesh, k1_x, time) + 2.0 * pot_t_multi(m2, k2_x, time) +
                                         2.0 * pot_t_multi(m3, k3_x, time) + pot_t_multi(m4, k4_x, time));
    mesh.verts = nopenetration(eps, dt, x1, average);
    const std::vector<vec3> normals = generate_vertex_normals(mesh);
    PotVec new_psi(average.size());
    for (size_t i = 0; i < average.size(); ++i) new_psi[i] = average[i].dot(normals[i]);
    set_psi(new_psi);
    set_phi(pf);
    time += dt;
    std::cout << "end_RK4" << std::endl;
    test_negative();
}

// The reference's Euler step (LinLinSim.cpp:260-284) through the virtual position_t.
void LinLinSim::evolve_euler_virtual(real dp, bool fixdt) {
    PotVec p = make_copy(phi);
    const CoordVec grads = position_t(mesh, p);
    const PotVec pot_derivative = pot_t_multi(mesh, grads, time);
    const real dt = fixdt ? dp : get_dt(dp, grads, pot_derivative);
    mesh.verts = mesh.verts + grads * dt;
    set_phi(p + dt * pot_derivative);
    time += dt;
}

CoordVec LinLinSim::position_t(Mesh const& m, PotVec& pot) const {
    bem_ctx* c = context(m);
    check(bem_set_V0(c, V_0));
    std::vector<double> x = flat(m.verts), vel(3 * m.verts.size());
    check(bem_position_t(c, x.data(), pot.data(), vel.data(), nullptr));
    return unflat(vel);
}

PotVec LinLinSim::pot_t_multi(Mesh const& m, CoordVec const& gradients, real t) const {
    bem_ctx* c = context(m);
    check(bem_set_V0(c, V_0));
    std::vector<double> x = flat(m.verts), g = flat(gradients);
    PotVec out(m.verts.size());
    check(bem_pot_t_multi(c, x.data(), g.data(), t, out.data()));
    return out;
}

// a single connected mesh is one loose part, so pot_t and pot_t_multi agree on it
PotVec LinLinSim::pot_t(Mesh const& m, CoordVec const& gradients, real t) const { return pot_t_multi(m, gradients, t); }

// LinLinSim::kappa (LinLinSim.cpp:122-146): per-triangle mean curvature averaged to the vertices
std::vector<real> LinLinSim::kappa(Mesh const& m) const {
    std::vector<real> kap, gam;
    curvatures(m, kap, gam);
    std::vector<real> out(m.verts.size(), 0.0), cnt(m.verts.size(), 0.0);
    for (size_t j = 0; j < m.trigs.size(); ++j)
        for (size_t k = 0; k < 3; ++k) {
            out[m.trigs[j][k]] += kap[j];
            cnt[m.trigs[j][k]] += 1.0;
        }
    for (size_t i = 0; i < out.size(); ++i) out[i] /= cnt[i];
    return out;
}

// LinLinSim::nopenetration (LinLinSim.cpp:162-190): exponential approach to the wall x = eps
CoordVec LinLinSim::nopenetration(real eps_, real dt, CoordVec const& x0, CoordVec& c) const {
    CoordVec xf(x0.size());
    for (size_t i = 0; i < x0.size(); ++i) xf[i] = x0[i] + dt * c[i];
    size_t applied = 0;
    for (size_t i = 0; i < x0.size(); ++i) {
        const real cx = c[i].x;
        if (cx * dt >= 0.0) continue;
        const real xpos = x0[i].x;
        bool moved = false;
        if (xpos < eps_) {
            xf[i].x = xpos * std::exp(cx / xpos * dt);
            moved = true;
        } else {
            const real te = (eps_ - xpos) / cx;
            if (std::abs(te) < std::abs(dt)) {
                xf[i].x = eps_ * std::exp(cx / eps_ * (dt - te));
                moved = true;
            }
        }
        if (moved) {
            c[i].x = (xf[i].x - xpos) / dt;
            ++applied;
        }
    }
    if (applied > 0) std::cout << "applied exponential " << applied << " times.      ##" << std::endl;
    return xf;
}

// LinLinSim::generate_tangent_gradients (LinLinSim.cpp:288-305): gradient of the linear interpolant
std::vector<vec3> LinLinSim::generate_tangent_gradients(Mesh const& m, std::vector<real> const& pot) const {
    std::vector<vec3> out;
    out.reserve(m.trigs.size());
    for (Triplet const& t : m.trigs) {
        const vec3 ab = m.verts[t.b] - m.verts[t.a], bc = m.verts[t.c] - m.verts[t.b];
        vec3 n = ab.vec(bc);
        n *= 1.0 / n.norm2();
        out.push_back((pot[t.c] - pot[t.b]) * n.vec(ab) + (pot[t.a] - pot[t.b]) * n.vec(bc));
    }
    return out;
}

// LinLinSim::curvature_param (LinLinSim.cpp:307-383): remeshing density from the maximal principal
// curvature and the potential's tangential gradient, smoothed over the two-ring
std::vector<real> LinLinSim::curvature_param() const {
    std::vector<real> param = max_curvature(mesh);
    const std::vector<vec3> grad = generate_tangent_gradients(mesh, make_copy(phi));
    std::vector<real> gsum(mesh.verts.size(), 0.0), cnt(mesh.verts.size(), 0.0);
    for (size_t j = 0; j < mesh.trigs.size(); ++j)
        for (size_t k = 0; k < 3; ++k) {
            gsum[mesh.trigs[j][k]] += grad[j].norm2();
            cnt[mesh.trigs[j][k]] += 1.0;
        }
    for (size_t i = 0; i < param.size(); ++i) param[i] = std::max(param[i], std::sqrt(1.0 + gsum[i] / cnt[i]));
    const std::vector<std::vector<size_t>> ring = generate_2_ring(mesh);
    std::vector<real> smooth(param.size());
    for (size_t i = 0; i < param.size(); ++i) {
        real s = 0.0;
        for (size_t j : ring[i]) s += param[j];
        smooth[i] = s / (real)ring[i].size();
    }
    return smooth;
}

// LinLinSim::remesh (LinLinSim.cpp:385-438): one split pass, then alternating flips, relaxation and
// collapses with the damped curvature parameter, then projection of the new vertices onto the old
// surface with interpolation of phi.  Host-side topology editing with the user's mesh library; the
// projection's ray casting on the GPU.
// The remeshing density: damped update d*old + (1-d)*new of curvature_params, clamped to the element
// size bounds (LinLinSim.cpp:387-394, ColocSimPin.cpp:297-304).  After an earlier remesh changed the
// vertex count only the common prefix carries the old values, as the reference's element-wise vector
// sum does.
void LinLinSim::update_curvature_params() {
    const std::vector<real> fresh = curvature_param();
    std::vector<real> mixed_params(fresh.size());
    for (size_t i = 0; i < fresh.size(); ++i)
        mixed_params[i] = (1.0 - damping_factor) * fresh[i] +
                          (i < curvature_params.size() ? damping_factor * curvature_params[i] : 0.0);
    curvature_params = mixed_params;
    if (min_elm_size > 0.0)
        for (real& c : curvature_params) c = std::max(std::min(c, 1.0 / min_elm_size), 1.0 / max_elm_size);
}

void LinLinSim::remesh(real L) {
    update_curvature_params();
    HalfedgeMesh he(generate_halfedges(mesh));
    split_edges(he, curvature_params, L * 0.75);
    flip_edges(he, 1);
    flip_edges(he, 1);
    relax_vertices(he);
    for (int round = 0; round < 4; ++round) {
        collapse_edges(he, curvature_params, L * 4.0 / 5.0);
        flip_edges(he, 1);
        flip_edges(he, 1);
        relax_vertices(he);
    }
    flip_edges(he, 1);
    relax_vertices(he);
    std::vector<real> new_phi;
    Mesh next = generate_mesh(he);
    dropin::project_interpolate(device_ctx(), next, generate_vertex_normals(next), mesh, make_copy(phi), new_phi,
                                nullptr, nullptr, true);
    mesh = next;
    phi = make_copy(new_phi);
    psi = Eigen::VectorXd::Zero((Eigen::Index)mesh.verts.size());
}

// compute_exterior_pot (LinLinSim.cpp:440-477): potential at points off the surface, 19-point rule, on
// the GPU (a context for the given mesh, released on return)
PotVec compute_exterior_pot(CoordVec const& pos, Mesh M, PotVec phi, PotVec psi) {
    PotVec out(pos.size(), 0.0);
    if (pos.empty()) return out;
    int dev = 0;
    if (const char* e = std::getenv("BEM_DEVICE")) dev = std::atoi(e);
    bem_ctx* c = nullptr;
    if (bem_create(&c, dev, nullptr) != BEM_OK) throw std::runtime_error("compute_exterior_pot: no CUDA device");
    struct Release {
        bem_ctx* c;
        ~Release() { bem_destroy(c); }
    } release{c};
    std::vector<int64_t> t(3 * M.trigs.size());
    for (size_t j = 0; j < M.trigs.size(); ++j)
        for (size_t k = 0; k < 3; ++k) t[3 * j + k] = (int64_t)M.trigs[j][k];
    std::vector<double> x = flat(M.verts), p = flat(pos);
    int rc = bem_set_mesh(c, (int64_t)M.verts.size(), x.data(), (int64_t)M.trigs.size(), t.data());
    if (rc == BEM_OK) rc = bem_exterior_potential(c, (int64_t)pos.size(), p.data(), phi.data(), psi.data(), out.data());
    if (rc != BEM_OK) throw std::runtime_error(std::string("compute_exterior_pot: ") + bem_last_error(c));
    return out;
}

// LinLinSim::exterior_pot (LinLinSim.cpp:479-485): psi solved at the current state, then the exterior
// potential, both on the GPU
PotVec LinLinSim::exterior_pot(CoordVec const& positions) const {
    PotVec out(positions.size(), 0.0);
    if (positions.empty()) return out;
    push_state();
    std::vector<double> p = flat(positions);
    check(bem_exterior_potential(ctx_, (int64_t)positions.size(), p.data(), nullptr, nullptr, out.data()));
    return out;
}

}  // namespace Bem
