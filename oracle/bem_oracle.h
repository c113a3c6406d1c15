/* CPU restatement of the bem-bubbles per-step hot path (the ORACLE).
 *
 * Test infrastructure only: tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load this library as the checker.  The product (libbem_b200.so) never links,
 * calls or falls back to it.
 *
 * Every function restates one reference function in plain C with the reference's
 * operation order, so that with one thread its results are bit-identical to the
 * reference compiled here (oracle/_ref, the reference sources built against the
 * Eigen-API shim).  That equality is checked by tests/test_oracle_pin.py against golden
 * vectors produced by oracle/_ref.
 *
 * Layouts: vertices are N x 3 row-major float64 (x,y,z per vertex, as std::vector<vec3>),
 * triangles M x 3 row-major int64, matrices N x N column-major float64 (Eigen's MatrixXd).
 */
#ifndef BEM_ORACLE_H
#define BEM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    double p_inf, epsilon, sigma, gamma, V0; /* Simulation.hpp:29-42, 180-183 */
    double field_amp, field_omega, field_phase; /* p_field(x,t) = amp*sin(omega*t + phase) */
    double min_dt, dp_balance;               /* Simulation.hpp:36-37 */
    double nopen_eps;                        /* LinLinSim.hpp:24 (1e-2) */
    int32_t mirror;                          /* LinLinSim.hpp:13 MIRROR_MESH */
    int32_t use_lu;                          /* Simulation.hpp:38 bicgstab = !use_lu */
} orc_params;

/* ColocSim::assemble_matrices (Bem/Simulation/ColocSim.cpp:21-102) */
int orc_assemble(int64_t N, int64_t M, const double* x, const int64_t* tri, int32_t mirror,
                 double* G, double* H);
/* H*phi as the shim's column-major GEMV (left-to-right column accumulation) */
void orc_gemv(int64_t N, const double* A, const double* v, double* y);
/* PartialPivLU solve (Simulation.cpp:57-60), shim's blocked algorithm */
int orc_solve_lu(int64_t N, const double* G, const double* b, double* x);
/* BiCGSTAB solve (Simulation.cpp:49-53), shim's restatement of Eigen's documented defaults */
int orc_solve_bicgstab(int64_t N, const double* G, const double* b, double* x,
                       int64_t* iters, double* rel_err);
/* generate_vertex_normals (Bem/Mesh/Mesh.cpp:141-163) */
void orc_vertex_normals(int64_t N, int64_t M, const double* x, const int64_t* tri, double* out);

/* compute_exterior_pot (LinLinSim.cpp:440-477): potential at P points off the surface from the surface
 * phi and psi (N each); 19-point rule, no wall image. */
void orc_exterior_pot(int64_t N, int64_t M, const double* x, const int64_t* tri, const double* phi,
                      const double* psi, int64_t P, const double* pts, double* out);
/* volume (Bem/Mesh/Mesh.cpp:206-218) */
double orc_volume(int64_t N, int64_t M, const double* x, const int64_t* tri);
/* LinLinSim::position_t (Bem/Simulation/LinLinSim.cpp:26-83); psi_l may be NULL */
int orc_position_t(int64_t N, int64_t M, const double* x, const int64_t* tri, const double* pot,
                   const orc_params* p, double* vel, double* psi_l);
/* LinLinSim::pot_t_multi (Bem/Simulation/LinLinSim.cpp:98-120) */
int orc_pot_t_multi(int64_t N, int64_t M, const double* x, const int64_t* tri, const double* grads,
                    double t, const orc_params* p, double* out);
/* LinLinSim::evolve_system_RK4 (LinLinSim.cpp:194-257); state updated in place.
 * Returns 0, or -2 when a vertex has x<0 (test_negative, LinLinSim.cpp:148-159). */
int orc_rk4_step(int64_t N, int64_t M, double* x, const int64_t* tri, double* phi, double* psi,
                 double* time, double dp, int32_t fixdt, const orc_params* p, double* dt_out);
/* LinLinSim::evolve_system (LinLinSim.cpp:260-284) */
int orc_euler_step(int64_t N, int64_t M, double* x, const int64_t* tri, double* phi, double* time,
                   double dp, int32_t fixdt, const orc_params* p, double* dt_out);

#ifdef __cplusplus
}
#endif
#endif
