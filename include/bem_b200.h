/* bem_b200 -- C ABI of the B200 (sm_100a) implementation of the bem-bubbles per-step hot path:
 * collocation influence-matrix assembly, the dense solve for dphi/dn, and the RK4 / Euler update
 * of vertex positions and surface potential.
 *
 * Plain C types only (pointers, sizes, doubles); no CUDA or torch types cross this boundary.
 * One context owns one simulation state (mesh, phi, psi, time, parameters) resident in GPU memory,
 * plus all device work buffers.  Calls on one context are serialised by the caller; distinct
 * contexts may be used from different threads.  Every function returns a bem_status; the text of
 * the last error of a context is available from bem_last_error().
 *
 * Host array layouts follow the reference's containers:
 *   vertices  N x 3 float64, row-major (std::vector<vec3>, Bem/basic/Bem.hpp:15)
 *   triangles M x 3 int64   (std::vector<Triplet>, Bem/basic/Triplet.hpp)
 *   scalars   N float64     (PotVec / Eigen::VectorXd)
 *   matrices  N x N float64, column-major (Eigen::MatrixXd)
 */
#ifndef BEM_B200_H
#define BEM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bem_ctx bem_ctx;

typedef enum {
    BEM_OK = 0,
    BEM_ERR_ARG = 1,          /* bad argument (null pointer, size mismatch, index out of range) */
    BEM_ERR_CUDA = 2,         /* CUDA runtime error */
    BEM_ERR_NEGATIVE_X = 3,   /* a vertex has x < 0: the reference throws std::out_of_range
                                 (LinLinSim::test_negative, Bem/Simulation/LinLinSim.cpp:148-159) */
    BEM_ERR_SINGULAR = 4,     /* zero pivot in the LU factorisation */
    BEM_ERR_NOT_CONVERGED = 5,/* iterative solver hit its iteration cap above tolerance */
    BEM_ERR_NOMEM = 6,        /* device allocation failed */
    BEM_ERR_STATE = 7         /* call order: no mesh set yet */
} bem_status;

typedef enum {
    BEM_SOLVER_BICGSTAB = 0,  /* the reference default (Simulation.hpp:38, Simulation.cpp:49-53) */
    BEM_SOLVER_LU = 1,        /* PartialPivLU (Simulation.cpp:57-60) */
    BEM_SOLVER_MIXED = 2      /* FP64 GMRES preconditioned by a low-precision inverse of G */
} bem_solver;

/* Physical and numerical parameters (Simulation ctor, Bem/Simulation/Simulation.hpp:29-54;
 * LinLinSim ctor, LinLinSim.hpp:22-27).  The far-field pressure of the reference is an arbitrary
 * function pointer real(*)(vec3 x, real t); here it is the family
 *     p_field(x, t) = field_amp * sin(field_kx * x.x + field_omega * t + field_phase)
 * evaluated on the device, or a host callback (bem_set_field_callback). */
typedef struct {
    double p_inf;        /* default 1 */
    double epsilon;      /* gas-pressure coefficient, default 1 */
    double sigma;        /* surface tension, default 0 */
    double gamma;        /* polytropic exponent, default 1 */
    double field_amp, field_kx, field_omega, field_phase;
    double min_dt;       /* Simulation::set_min_dt, default -1 (off) */
    double dp_balance;   /* Simulation::set_dp_balance, default 3 */
    double nopen_eps;    /* LinLinSim::eps (nopenetration wall distance), default 1e-2 */
    int32_t mirror;      /* image in the wall x = 0 (LinLinSim.hpp:13 MIRROR_MESH) */
    int32_t solver;      /* bem_solver */
    double mixed_tol;    /* relative residual target of BEM_SOLVER_MIXED, default 1e-12 */
    int32_t max_iters;   /* iteration cap for the iterative solvers, 0 = reference default (2N) */
    int32_t flags;       /* BEM_FLAG_* bits, default 0 */
} bem_params;

/* bem_params.flags: run the FP64 BiCGSTAB as separate kernels per iteration instead of the persistent
 * cooperative kernel (same iteration; for comparison, or where cooperative launches are unwanted). */
#define BEM_FLAG_BICGSTAB_MULTIKERNEL 1
/* bem_params.flags: start each RK4 stage solve of BEM_SOLVER_MIXED from the previous stage's solution
 * instead of the stage predictor (an extrapolation in time from the same stage of the last three
 * steps).  Either start converges to the same FP64 solution; the predictor saves refinement steps. */
#define BEM_FLAG_NO_STAGE_PREDICTOR 2
/* bem_params.flags: the step path (position_t, RK4, Euler) assembles H as well, with the column-group
 * kernel of bem_assemble, instead of the G-only triangle-patch kernel that forms b = H phi without
 * H.  Both give the same G and b to rounding; for comparison. */
#define BEM_FLAG_STEP_ASSEMBLE_H 4
/* bem_params.flags: run each round of BEM_SOLVER_MIXED's refinement steps as one cooperative kernel
 * with grid barriers instead of separate GEMV launches (the same tiles and summation order:
 * bit-identical results, with BEM_FLAG_NO_IR_GATE).  Measured slower than the separate launches on
 * B200 (0.36 against 0.27 ms per solve at N = 4002), so it is not the default. */
#define BEM_FLAG_REFINE_PERSISTENT 8
/* bem_params.flags: how BEM_SOLVER_MIXED builds its approximate inverse from scratch.  By default
 * (neither flag) large systems (N >= BEM_GJ_MIN_N) use blocked Gauss-Jordan elimination with row
 * partial pivoting in FP32, its rank-64 updates as split-precision tcgen05 GEMMs, polished by
 * Newton-Schulz steps; smaller ones use Newton-Schulz from a scaled identity.  The flags force one. */
#define BEM_FLAG_INVERSE_GJ 16
#define BEM_FLAG_INVERSE_NS 32
#define BEM_GJ_MIN_N 8192
/* bem_params.flags: no gated extra steps in the first round of BEM_SOLVER_MIXED's refinement.  By
 * default that round issues one or two steps beyond its estimate whose GEMVs a device-side check of
 * the convergence rule skips once it holds, so a short estimate does not cost a second round (a
 * read-back of the residual norms by the host and a new enqueue).  With the flag a round issues its
 * estimate only, as the cooperative round kernel of BEM_FLAG_REFINE_PERSISTENT does. */
#define BEM_FLAG_NO_IR_GATE 64

/* Fill *p with the reference's defaults. */
void bem_default_params(bem_params* p);

/* Create a context on CUDA device `device`.  Replaces the construction of Bem::ColocSim /
 * Bem::LinLinSim / Bem::Simulation (ColocSim.hpp:16, LinLinSim.hpp:22, Simulation.hpp:29). */
int bem_create(bem_ctx** out, int device, const bem_params* p);
int bem_destroy(bem_ctx* ctx);
const char* bem_last_error(const bem_ctx* ctx);
int bem_set_params(bem_ctx* ctx, const bem_params* p);
int bem_get_params(const bem_ctx* ctx, bem_params* p);

/* Set the mesh (topology + positions).  As in the Simulation ctor, V_0 := volume(mesh),
 * phi := 0, psi := 0 (Simulation.hpp:42, LinLinSim.hpp:28-29).  Replaces `Mesh mesh` set-up. */
int bem_set_mesh(bem_ctx* ctx, int64_t n_verts, const double* verts, int64_t n_trigs, const int64_t* trigs);
int bem_num_verts(const bem_ctx* ctx, int64_t* n);
/* mesh.verts read/write (public member Simulation::mesh, Simulation.hpp:202) */
int bem_set_vertices(bem_ctx* ctx, const double* verts);
int bem_get_vertices(bem_ctx* ctx, double* verts);
/* set_phi / get_phi / set_psi / get_psi (Simulation.hpp:92-143) */
int bem_set_phi(bem_ctx* ctx, const double* phi);
int bem_get_phi(bem_ctx* ctx, double* phi);
int bem_set_psi(bem_ctx* ctx, const double* psi);
int bem_get_psi(bem_ctx* ctx, double* psi);
/* The whole state in one call each way (any pointer may be NULL to skip that part).  bem_set_state
 * copies the arrays before returning and queues the device copies without waiting for them;
 * bem_get_state waits once for all of them.  The per-array calls above each wait on their own. */
int bem_set_state(bem_ctx* ctx, const double* verts, const double* phi, const double* psi, const double* time);
int bem_get_state(bem_ctx* ctx, double* verts, double* phi, double* psi, double* time);
/* set_time/get_time, set_V_0 (Simulation.hpp:106-126) */
int bem_set_time(bem_ctx* ctx, double t);
int bem_get_time(bem_ctx* ctx, double* t);
int bem_set_V0(bem_ctx* ctx, double v0);
int bem_get_V0(bem_ctx* ctx, double* v0);
/* get_volume: volume(mesh) (Simulation.hpp:128-130, Mesh.cpp:206-218) */
int bem_get_volume(bem_ctx* ctx, double* vol);

/* Host callback form of the reference's pressure-field function pointer (Simulation.hpp:186):
 * when set, it is evaluated on the host for every vertex at every RK4 stage (positions are copied
 * back for it), instead of the device-evaluated sine family.  Pass NULL to clear. */
typedef double (*bem_field_fn)(const double x[3], double t, void* user);
int bem_set_field_callback(bem_ctx* ctx, bem_field_fn fn, void* user);

/* ColocSim::assemble_matrices (Bem/Simulation/ColocSim.cpp:21-110) for the given vertex positions
 * (NULL = the context's mesh).  G and H are host N x N column-major outputs; either may be NULL. */
int bem_assemble(bem_ctx* ctx, const double* verts, double* G, double* H);
/* G and the right-hand side b = H*pot (after the 4 pi rule) as the step path forms them for
 * position_t (LinLinSim.cpp:26-83: assemble_matrices, then H*phi), for positions `verts` (NULL =
 * the context's mesh).  Single systems without pinned vertices use the G-only triangle-patch kernel,
 * which never forms H; otherwise the bem_assemble kernel.  G (N x N column-major) and b (N) are host
 * outputs; either may be NULL. */
int bem_assemble_rhs(bem_ctx* ctx, const double* verts, const double* pot, double* G, double* b);
/* Simulation::solve_system (Simulation.cpp:40-71): x = G^{-1} b with the context's solver. */
int bem_solve_system(bem_ctx* ctx, const double* G, const double* b, double* x);
/* LinLinSim::position_t (LinLinSim.cpp:26-83): vertex velocities for positions `verts` (NULL = mesh)
 * and potential `pot`.  psi_l (the solved dphi/dn) may be NULL. */
int bem_position_t(bem_ctx* ctx, const double* verts, const double* pot, double* vel, double* psi_l);
/* bem_position_t with pot in/out, as the reference's PotVec& argument: with pinned vertices
 * (bem_set_pinned) pot receives the solved potential at the pinned vertices (ColocSimPin.cpp:188). */
int bem_position_t_inout(bem_ctx* ctx, const double* verts, double* pot, double* vel, double* psi_l);

/* ---- Pinned contact line: the reference's ColocSimPin (Bem/Simulation/ColocSimPin.cpp:25-194),
 * replacing ColocSimPin::assemble_matrices and ColocSimPin::position_t.  The last n_pin vertices of the
 * mesh lie on the wall x = 0 (ColocSimPin::set_x_boundary moves them to the end).  With n_pin > 0:
 *  - every assembly (bem_assemble, the steps, the exterior potential's solve) exchanges the pinned
 *    columns after the 4 pi rule: G(:,j) = -H(:,j), H(:,j) = -G(:,j) (ColocSimPin.cpp:113-117);
 *  - position_t and the RK4/Euler stages use the stored psi (bem_set_psi) in place of the stage
 *    potential at the pinned vertices in H*pot (:146-148), move the pinned vertices with the drift
 *    velocity n_w * (beta (costheta_eq - c) + c_nonlinear c^3 / (c^2 - 1)), c = vertex normal . e_x,
 *    n_w the vertex normal with its x component removed, normalised (:126-136, :175-186), and set the
 *    stage potential at the pinned vertices to the solved unknowns (:188).
 * The reference's law: beta = 0.2, costheta_eq = cos(130 deg), c_nonlinear = 0.01 (:126-130).
 * n_pin = 0 switches pinning off; bem_set_mesh and bem_set_mesh_blocks reset it.  Single systems only;
 * the adjoint refuses pinned vertices. */
int bem_set_pinned(bem_ctx* ctx, int64_t n_pin, double beta, double costheta_eq, double c_nonlinear);
int bem_get_pinned(const bem_ctx* ctx, int64_t* n_pin);

/* ---- Remeshing support.  trace_mesh (Bem/Mesh/MeshManip.cpp:1250-1283) for P rays on the device, the
 * O(P x M) scan of project_and_interpolate (MeshManip.cpp:1426-1697): ray k starts at pos[3k..] with
 * direction dir[3k..]; among the triangles of the mesh (verts: nverts x 3, trigs: M x 3) whose closed
 * interior contains the intersection with the triangle's plane, the one with the smallest |s| is taken
 * (the first in triangle order on ties).  hit[3k..] receives the intersection, tri[k] the triangle and
 * ok[k] 1; a ray that hits nothing gets ok 0, hit (0,0,0) and triangle 0.  Results are bit-identical to
 * the host scan.  Uses the context's device and stream only (no mesh needed). */
int bem_trace_mesh(bem_ctx* ctx, int64_t nverts, const double* verts, int64_t M, const int64_t* trigs, int64_t P,
                   const double* pos, const double* dir, double* hit, int64_t* tri, int32_t* ok);
/* LinLinSim::pot_t_multi (LinLinSim.cpp:98-120): Dphi/Dt per vertex for positions `verts`
 * (NULL = mesh), vertex velocities `grads` and time t. */
int bem_pot_t_multi(bem_ctx* ctx, const double* verts, const double* grads, double t, double* out);
/* LinLinSim::evolve_system_RK4 (LinLinSim.cpp:194-257) and evolve_system (Euler, :260-284) on the
 * device-resident state.  fixdt != 0: dt = dp; else the adaptive Simulation::get_dt (Simulation.cpp:77-92).
 * *dt_out (may be NULL) receives the step taken.  BEM_ERR_NEGATIVE_X mirrors test_negative. */
int bem_evolve_rk4(bem_ctx* ctx, double dp, int32_t fixdt, double* dt_out);
int bem_evolve_euler(bem_ctx* ctx, double dp, int32_t fixdt, double* dt_out);
/* `steps` RK4 steps with fixed dt, without the x < 0 check and host synchronisation between steps (the
 * iterative solvers still read their residual norms back: the mixed solver once per stage). */
int bem_evolve_rk4_n(bem_ctx* ctx, double dt, int32_t steps);

/* ---- Batches of independent bubbles (a radius x pressure sweep as in the reference's
 * oscillations-array.sh, one process per point there).  No counterpart function in the reference:
 * each bubble follows the reference's single-bubble path (LinLinSim::evolve_system_RK4 with its own
 * V_0 and pressure field), and the bubbles do not interact.  The mesh is the concatenation of the
 * bubbles' meshes: bubble b owns vertices [vert_off[b], vert_off[b+1]) and only triangles among them.
 * G and H are block-diagonal (packed n_b x n_b blocks; bem_assemble returns them packed, block b at
 * offset sum_{b'<b} n_b'^2).  A batch always uses the mixed solver, batched over all bubbles without
 * host synchronisation; the pressure field is the device-evaluated family with per-bubble
 * parameters.  Replaces the mesh like bem_set_mesh; each bubble's V_0 starts as its own volume and
 * its field parameters as the context's. */
int bem_set_mesh_blocks(bem_ctx* ctx, int64_t N, const double* verts, int64_t M, const int64_t* trigs,
                        int32_t nblocks, const int64_t* vert_off);
int bem_num_blocks(const bem_ctx* ctx, int32_t* nblocks);
/* Per-bubble V_0 and field A*sin(kx*x + omega*t + phase); each array has nblocks entries or is NULL
 * (unchanged). */
int bem_set_block_params(bem_ctx* ctx, const double* V0, const double* amp, const double* kx,
                         const double* omega, const double* phase);
int bem_get_block_params(bem_ctx* ctx, double* V0, double* amp, double* kx, double* omega, double* phase);
/* Per-bubble statistics of the last batched solve: contraction per refinement step, final relative
 * residual, refinement steps used (any may be NULL). */
int bem_get_block_stats(bem_ctx* ctx, double* rho, double* rel_residual, int32_t* steps);
/* `steps` fixed-dt RK4 steps of a batch, each step one replay of a CUDA graph captured on the first
 * call (and again when dt changes).  After each step the host reads the per-bubble statistics:
 * stale approximate inverses are refreshed, and a bubble that missed the tolerance makes the step
 * run again from its start state.  bem_evolve_rk4_n on a batch takes the same steps without the graph. */
int bem_evolve_rk4_graph(bem_ctx* ctx, double dt, int32_t steps);
/* Assembly tile shape of a batch by measurement: column groups of 32 (x 128 rows), 48 and 64 (x 64
 * rows) and 16 (x 256 rows) are each planned and timed over three assemblies of the current state, and
 * the fastest is kept (remembered per device and batch shape).  *best_cg receives the width, ms[4] the
 * average times in that order (either may be NULL).  The state is kept; approximate inverses are
 * rebuilt on the next step. */
int bem_autotune_assembly(bem_ctx* ctx, int32_t* best_cg, double* ms);

/* Simulation::export_mesh (Simulation.cpp:94-96, export_ply_float MeshIO.cpp:263-298) of the current
 * state without waiting for the file: the state is packed to float32 on the device in stream order
 * (later steps may follow at once), copied to pinned memory on a separate stream and written by a
 * background thread.  Up to four files are in flight; a fifth call waits for the oldest.
 * bem_export_wait returns when every queued file is written, with the first write error if any. */
int bem_export_ply_async(bem_ctx* ctx, const char* path);
int bem_export_wait(bem_ctx* ctx);

/* Potential at P points off the surface (points: P x 3), compute_exterior_pot (LinLinSim.cpp:440-477):
 * sum over triangles of (-G psi + H phi)/(4 pi) with the 19-point rule, no wall image.  phi (N) NULL:
 * the context's phi.  psi (N) NULL: LinLinSim::exterior_pot (LinLinSim.cpp:479-485), i.e. psi solved
 * first from G psi = H phi with the context's solver at the current positions.  Points must lie off
 * the surface, as in the reference. */
int bem_exterior_potential(bem_ctx* ctx, int64_t P, const double* points, const double* phi, const double* psi,
                           double* out);

/* ---- Adjoint of fixed-dt RK4 trajectories.  No counterpart in the reference: reverse-mode
 * derivative of LinLinSim::evolve_system_RK4 (LinLinSim.cpp:194-257) as computed here, for
 * free-space bubbles (no wall image), sigma = 0 and the device-evaluated field; V_0 and the other
 * parameters are held fixed.  The transposed solves refine against the FP64 G through the mixed
 * solver's approximate inverse, which is built when the context uses another solver.
 * bem_adjoint_record runs `steps` RK4 steps from the current state (advancing it) and keeps one
 * checkpoint per step; it fails with BEM_ERR_STATE if a vertex comes within the wall treatment's
 * range (x < nopen_eps), which is not differentiated.  bem_adjoint_backward takes the adjoint of
 * the final state (d objective / d x_K as N x 3, d objective / d phi_K as N) and returns that of
 * the recorded initial state, recomputing each step's stages from its checkpoint. */
int bem_adjoint_record(bem_ctx* ctx, double dt, int32_t steps);
int bem_adjoint_backward(bem_ctx* ctx, const double* xbar_end, const double* phibar_end, double* xbar0,
                         double* phibar0);
/* The same with device arrays on the context's device, overwritten in place; returns after the
 * context's stream has finished. */
int bem_adjoint_backward_device(bem_ctx* ctx, double* xbar, double* phibar);
/* d(total enclosed volume)/d(vertex positions) at the current state, N x 3 host array
 * (Mesh.cpp:206-218 differentiated). */
int bem_volume_gradient(bem_ctx* ctx, double* xbar);
/* State from / to device arrays (N x 3 positions, N potentials) on the context's device; either
 * pointer may be NULL. */
int bem_set_state_device(bem_ctx* ctx, const double* x, const double* phi);
int bem_get_state_device(bem_ctx* ctx, double* x, double* phi);

/* Solver statistics of the most recent solve. */
typedef struct {
    int64_t solves;           /* solves since creation */
    int32_t last_iters;       /* iterations of the last iterative solve */
    int32_t precond_refresh;  /* refreshes of the mixed path's approximate inverse */
    double last_rel_residual; /* final relative residual of the last iterative solve */
    int64_t ns_steps;         /* Newton-Schulz steps taken by the mixed path (set-up and refreshes) */
    int64_t gmres_fallbacks;  /* mixed solves that handed over from refinement to GMRES */
    int64_t fp64_fallbacks;   /* mixed solves that fell back to the FP64 BiCGSTAB: no approximate inverse
                                 could be built, or GMRES missed the tolerance (a singular or nearly
                                 singular G, e.g. a bubble cut by its own wall image) */
    int64_t total_iters;      /* iterations of every iterative solve since creation (refinement steps of
                                 the mixed path, including its GMRES hand-overs; BiCGSTAB iterations) */
    int64_t wait_expired;     /* bounded grid-barrier waits of the persistent kernels (BiCGSTAB, LU
                                 panel) that gave up; each sent the context to the multi-kernel form */
    int64_t gj_inverses;      /* approximate inverses of the mixed path built by the tensor-core
                                 Gauss-Jordan elimination (the rest by Newton-Schulz from scratch) */
    int64_t ir_rounds;        /* rounds of refinement steps of the mixed path since creation (each ends
                                 with one read-back of the residual norms by the host) */
} bem_stats;
int bem_get_stats(bem_ctx* ctx, bem_stats* s);

/* Bound, in SM clock cycles, of every grid-wide barrier wait of the persistent kernels (the
 * cooperative BiCGSTAB, the cooperative refinement round, the row-distributed LU panel) and of the
 * LU cluster panel's mbarrier waits.  Default 2e9 (about a second at the B200's clock).  A wait that
 * runs out makes the kernel set its error word and return; the host reads it, counts it in
 * bem_stats.wait_expired and finishes the solve with the multi-kernel form (for the LU: the
 * single-CTA panel), which the context keeps for the rest of its life.  No counterpart in the reference (its solves
 * run on the host); exists so that this failure path can be tested without a GPU fault.
 * cycles <= 0 returns BEM_ERR_ARG. */
int bem_set_wait_limit(bem_ctx* ctx, int64_t cycles);

/* Synchronise the context's stream. */
int bem_sync(bem_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that time or order work around it. */
int bem_get_stream(bem_ctx* ctx, void** stream);

/* Device-time profile of the context's stream, recorded with CUDA events when enabled:
 * the regular/singular assembly kernel (the dominant kernel of a stage) and the whole solve
 * phase.  bem_get_profile synchronises the stream and returns the totals since the last reset. */
typedef struct {
    double assemble_ms;        /* summed duration of the assembly tile kernel */
    int64_t assemble_launches;
    double solve_ms;           /* summed duration of the solve phases */
    int64_t solve_calls;
    int64_t kernel_launches;   /* kernels of this library launched while profiling */
} bem_profile;
int bem_set_profiling(bem_ctx* ctx, int32_t on);
int bem_get_profile(bem_ctx* ctx, bem_profile* out);
int bem_reset_profile(bem_ctx* ctx);

/* Roofline denominators measured on `device` with FMA-loop kernels: dense FP64 and FP32
 * FMA throughput in TFLOP/s (2 flops per FMA).  Diagnostic; allocates and frees its own buffer. */
int bem_measure_fma_peaks(int device, double* fp64_tflops, double* fp32_tflops);

/* C = A * B for FP32 column-major n x n host matrices through the split-precision tensor-core GEMM
 * (tcgen05, bf16 hi/lo operand split, three MMAs per product, FP32 accumulation) that refreshes the
 * mixed solver's approximate inverse.  Exposed for verification; allocates its own device buffers. */
int bem_gemm_bf16x3(int device, int n, const float* A, const float* B, float* C);

/* Allocation-free form of bem_gemm_bf16x3, for callers that cannot allocate GPU memory (a host
 * framework that owns the device heap, loops that must not allocate after start-up, plug-ins that
 * only receive device pointers).  This entry point has no counterpart in the reference.
 * A, B, C: DEVICE pointers on `device` to FP32 column-major n x n matrices owned by the caller;
 * stream: a cudaStream_t that belongs to `device` (NULL = the legacy default stream).  The calling
 * thread's current device is the same after the call as before it.  The call allocates nothing: its scratch (four
 * bf16 operand planes and an error word) is a static device array of BEM_NOALLOC_GEMM_MAX_N^2 * 8
 * bytes + 256 bytes (8 MB) that every GPU loading this library holds until the process exits.
 * n > BEM_NOALLOC_GEMM_MAX_N returns BEM_ERR_ARG.  The first call on a device looks up the scratch's
 * device address (cudaGetSymbolAddress); make that first call before any stream capture.  All calls
 * share the one scratch array, which keeps the last call's contents: calls that overlap on the GPU
 * (other streams, other threads) race on it.  Returns after C is complete (synchronises `stream`). */
#define BEM_NOALLOC_GEMM_MAX_N 1024
int bem_gemm_bf16x3_noalloc(int device, int n, const float* A, const float* B, float* C, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* BEM_B200_H */
