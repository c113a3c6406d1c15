// Internal declarations shared by the CUDA translation units of libbem_b200.so.
// Nothing here crosses the C ABI (include/bem_b200.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/bem_b200.h"

namespace bemb {

// Kernel launches issued by this library (all contexts), for the bench's launch count.
extern std::atomic<long long> g_kernel_launches;
#define KLAUNCH() (::bemb::g_kernel_launches.fetch_add(1, std::memory_order_relaxed))

// Device-scoped one-time set-up (kernel attributes and __constant__ tables exist once per device,
// not once per process): runs setup() on the current device unless it already succeeded there for
// this mask.  Calls are serialised, so a second thread's first call waits until the set-up is
// complete instead of launching before it; the device's bit is set only after setup() returned
// true, so a failed set-up is tried again on the next call.  Returns whether the set-up is in place.
inline bool once_per_device(std::atomic<uint64_t>& mask, const std::function<bool()>& setup) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    const uint64_t bit = 1ull << (dev & 63);
    if (mask.load(std::memory_order_acquire) & bit) return true;
    static std::recursive_mutex m;
    std::lock_guard<std::recursive_mutex> lock(m);
    if (mask.load(std::memory_order_acquire) & bit) return true;
    if (!setup()) return false;
    mask.fetch_or(bit, std::memory_order_release);
    return true;
}

// Largest column-group width of the assembly tiles (a CTA owns up to CG_MAX columns of G and H);
// the width used for a mesh is Topology::cg, with the rows per CTA tied to it (see assemble.cu).
constexpr int CG_MAX = 64;
// Per (group, triangle): the owned slot of each of the 3 vertices in SLOT_BITS-bit fields,
// SLOT_NONE when the vertex belongs to another group.
constexpr int SLOT_BITS = 7;
constexpr int SLOT_NONE = 127;
// Triangle records staged per chunk in shared memory.
constexpr int ASM_TC = 40;
// Doubles per triangle record: 7 quadrature points (21), unit normal (3), area (1), pad (3).
constexpr int REC = 28;
// Triangle patches of the G-only assembly (the step path): every triangle belongs to exactly one
// patch of at most PT_MAX triangles touching at most PCOLS vertices (the patch's columns); a patch
// record of PREC doubles per triangle (288 bytes, a multiple of 16 for the bulk copy).
constexpr int PT_MAX = 32;
constexpr int PCOLS = 32;
constexpr int PREC = 36;
constexpr int PATCH_ROWS = 256;  // rows per CTA of the patch tiles
constexpr int RF_WORDS = 128;    // ints of Ctx::rf_bar (the refinement round kernel's barrier and error words,
                                 // the refinement's convergence gate)
// A patch: its triangles [t0, t0 + nt) of Topology::patch_tri, and the sub-system (block) it lies in:
// first vertex vbase and n vertices, G block at element mbase, row partials at pbase + row*np + lp
// (np patches in the block, lp this patch's index among them).
struct PatchInfo {
    int t0, nt, vbase, n, np, lp;
    long long mbase, pbase;
};
// A vertex whose G column sums the halo columns of several patches: cnt columns of n elements from
// element hpos of the halo buffer, in increasing patch order; its G column starts at element gpos.
// tick: its first ticket counter, one per row tile of its block (the patch CTA that draws the last
// ticket of a row tile sums that tile's rows).
struct PartialCol {
    long long hpos, gpos;
    int cnt, n, tick, pad;
};
// Fixed block count of the vector kernels, so reductions have a fixed, deterministic shape.
constexpr int VBLK = 128;
constexpr int VTHR = 256;

// Topology-derived, device-resident tables (rebuilt only when the triangle list changes).
struct Topology {
    int64_t N = 0, M = 0;
    int* tri = nullptr;          // M*3 int32, reference vertex order
    int* csr_off = nullptr;      // N+1, vertex -> incident triangles (increasing index)
    int* csr_idx = nullptr;      // 3M
    int ngroups = 0;             // assembly column groups
    int cg = 16;                 // vertices per column group
    int* grp_off = nullptr;      // ngroups+1 into grp_tri
    int* grp_tri = nullptr;      // triangles incident to the group's vertices, increasing
    int* grp_slot = nullptr;     // per grp_tri entry: 3 x SLOT_BITS owned-slot codes (SLOT_NONE = not owned)
    int* grp_vert = nullptr;     // ngroups*cg vertex of each slot, -1 padding
    int nparts = 0;              // loose parts (bubbles)
    int max_part_tris = 0;       // triangles of the largest part
    int* part_of_vert = nullptr; // N
    int* part_off = nullptr;     // nparts+1 into part_tidx
    int* part_tidx = nullptr;    // triangle ids grouped by part, increasing inside a part
    int* tri_rot = nullptr;      // M*3: triangles rotated so the largest vertex id comes first,
                                 // the vertex order split_by_loose_parts leaves (Mesh.cpp:410-426)
    std::vector<int> h_part_of_vert;
    // triangle patches of the G-only assembly (the whole mesh, or block by block for a batch)
    int npatch = 0;
    PatchInfo* pinfo = nullptr;     // npatch
    int* patch_tri = nullptr;       // M: triangle ids, patch by patch, increasing inside a patch
    int* patch_slot = nullptr;      // M: the column slots of the triangle's 3 vertices, 8 bits each
    int* patch_col = nullptr;       // npatch*PCOLS: vertex of each column slot, -1 padding
    long long* patch_dst = nullptr; // npatch*PCOLS: element offset of a partial slot's halo column, -1 complete
    int* patch_pk = nullptr;        // npatch*PCOLS: the partial vertex (index into pcol) of a slot, -1 complete
    unsigned* halo_tick = nullptr;  // ticket counters of the partial vertices' row tiles (zero between uses)
    int npartial = 0;               // vertices shared between patches
    PartialCol* pcol = nullptr;     // npartial
    int max_block_n = 0;            // rows of the largest block (the halo reduction's grid)
    long long halo_elems = 0;       // doubles of the halo columns
    int2* pwork = nullptr;          // tiles {patch, first row}, PATCH_ROWS rows each
    int nwork = 0;
};

// Control block of the iterative solvers and RK4 scalars, resident on the device.
struct DevScalars {
    double time;      // simulation time
    double dt;        // current step
    double V0;        // reference volume of the gas law
    double field;     // far-field pressure at the step-start time (x-independent family)
    // BiCGSTAB / GMRES scalars
    double rho, alpha, w, beta, r0_sq, rhs_sq, tol2, rr;
    int32_t iters, restarts, done, restart_flag, maxit, nonconv;
    int32_t pad[2];
};

// One independent sub-system of a block-diagonal batch (one bubble of a parameter sweep).  Its
// vertices are the contiguous range [vbase, vbase + n) of the shared arrays; its G and H blocks are
// n x n column-major at element offset mbase of the packed matrices; its column groups are
// [gbase, gbase + ngroups) with partial row sums at pbase; its GEMV row blocks start at rbase, its
// GEMV column splits number ncs with partials at pofs.
struct BlockInfo {
    int n, vbase, gbase, ngroups;
    int rbase, ncs, npatch, pad1;   // npatch: patches of the block (G-only assembly)
    long long mbase, pbase, pofs;
    long long ppbase;               // the G-only assembly's row partials of the block
};

struct Ctx;

// assemble.cu
struct QuadTables {
    double qc[7][3], quv[7][2], w[7], gc[7], gs[7], gw[7], orb[5];
    double q19[19][3];  // 19-point rule as (u, v, w): y = a + u (b - a) + v (c - b)
};
void quad_tables(QuadTables& t);
void launch_triangle_records(Ctx& c, const double* x, cudaStream_t s);
void launch_assemble(Ctx& c, const double* x, const double* phi, double* G, double* H, double* b,
                     cudaStream_t s, const double* x0 = nullptr,
                     double* r0 = nullptr);
void prepare_assemble(Ctx& c);  // kernel attributes and the persistent grid, outside any capture
// G and b (no H) through the triangle-patch kernels: systems without pinned vertices
void launch_assemble_g(Ctx& c, const double* x, const double* phi, double* b, cudaStream_t s,
                       const double* x0 = nullptr, double* r0 = nullptr);
void prepare_assemble_g(Ctx& c);  // its kernel attributes and constants, outside any capture

// stage.cu
void launch_velocity_prep(Ctx& c, const double* x, const double* pot, cudaStream_t s);
// stage >= 0: psil also goes into the stage predictor's history (the stage's solution)
void launch_velocity(Ctx& c, const double* psil, double* vel, cudaStream_t s, int stage = -1);
void launch_pot_t(Ctx& c, const double* x, const double* vel, const double* field_host, double* out,
                  cudaStream_t s);
void launch_part_volumes(Ctx& c, const double* x, double* vol, cudaStream_t s);
// xs = x1 + scale dt kx and ps = p1 + scale dt kp (an RK4 stage's state) in one launch
void launch_axpy_stage(Ctx& c, const double* kx, const double* kp, const double* coef_dev, double scale,
                       cudaStream_t s);
void launch_rk4_final(Ctx& c, cudaStream_t s, const int* skip = nullptr);
// Stage predictor of the mixed solve (stage.cu): depth of the history; the ring's stage times hold
// at PRED_CNT the number of steps that continue the current trajectory.  Start value of stage
// `stage` (0..3) extrapolated from the ring (launch_velocity stores the stage's solution), the end of a step;
// state copies that end the trajectory when a value changes.
constexpr int PRED_DEPTH = 3;
constexpr int PRED_CNT = PRED_DEPTH * 4;
void launch_stage_predict(Ctx& c, int stage, double* x, cudaStream_t s);
void launch_stage_advance(Ctx& c, const int* skip, cudaStream_t s);
void launch_state_accept(Ctx& c, int64_t n, const double* src, double* dst, cudaStream_t s);
void launch_time_accept(Ctx& c, double t, cudaStream_t s);
void launch_euler_final(Ctx& c, const double* vel, const double* potd, cudaStream_t s);
void launch_vertex_normals(Ctx& c, const double* x, double* out, cudaStream_t s);
void launch_get_dt(Ctx& c, const double* vel, const double* potd, double dp, cudaStream_t s);
void launch_any_negative(Ctx& c, const double* x, int* flag, cudaStream_t s);
void launch_curvature(Ctx& c, const double* x, double* kap, cudaStream_t s);

// pin.cu
void launch_pin_zero(Ctx& c, const double* pot, double* potz, cudaStream_t s);
void launch_pin_exchange(Ctx& c, const double* v, double* b, cudaStream_t s);
void launch_pin_finish(Ctx& c, const double* x, double* vel, double* pot, cudaStream_t s);

// bicg.cu
int bicgstab_persistent(Ctx& c, const double* A, const double* b, double* x, cudaStream_t s);
size_t pbicg_words(int64_t n);  // doubles of the persistent BiCGSTAB's dot and barrier scratch

// lu_panel.cu
// The panel of another column-major n x n matrix (only its columns [k0, k0+nb) are touched); piv and
// sing as c.piv and c.flag for c.LU.
struct PanelTarget {
    double* A;
    int n;
    int* piv;
    int* sing;
};
int lu_panel_rows(Ctx& c, int k0, int nb, cudaStream_t s, const PanelTarget* tgt = nullptr);
int lu_panel_cluster(Ctx& c, int k0, int nb, cudaStream_t s, const PanelTarget* tgt = nullptr);
// the panel's interchanges on the other columns of c.LU and on c.lu_perm; built: the (cluster) panel
// kernel composed them already
void lu_panel_swap_rest(Ctx& c, int k0, int nb, cudaStream_t s, bool built);
void lu_perm_init(Ctx& c, cudaStream_t s);  // c.lu_perm = identity, before the first panel
// lu_update.cu: A22 -= L21 U12 after the panel [k0, k0 + nb) of the column-major n x n A (FP64 tensor cores)
int lu_update(Ctx& c, int n, int k0, int nb, double* A, cudaStream_t s, int cb = -1, int ce = -1, bool narrow = false);
size_t lu_panel_words();   // doubles of Ctx::lu_aux
int* lu_panel_err(Ctx& c); // device error word of the row-distributed panels

// remesh.cu
int trace_mesh(Ctx& c, int64_t Nv, const double* verts, int64_t M, const int64_t* trigs, int64_t P, const double* pos,
               const double* dir, double* hit, int64_t* tri_out, int32_t* ok);

// Newton-Schulz job: X ~ A^-1 for an n x n column-major FP64 matrix A, with its FP32 copy G32 and
// FP32 work matrices T, P (all n x n).
struct NSJob {
    int n;
    const double* A;
    float* G32;
    float* X;
    float* T;
    float* P;
};
int ns_step(Ctx& c, const NSJob& j, cudaStream_t s, double* eres, int terms = 3);
int ns_from_scratch(Ctx& c, const NSJob& j, cudaStream_t s, bool classical);
// gj_inverse.cu: j.X ~ A^-1 by blocked Gauss-Jordan with tensor-core rank-64 updates (j.T as work)
int gj_inverse(Ctx& c, const NSJob& j, cudaStream_t s);
void to_f32(int64_t nn, const double* a, float* b, cudaStream_t s);

// tc_gemm.cu
// An operand of the general split-precision GEMM: S(r, k) = src[r*sr + k*sk] for r < rows, k < cols,
// times sign, zero for r in [zr0, zr1) or k in [zk0, zk1).
struct TcOperand {
    const float* src;
    long long sr, sk;
    int rows, cols;
    int zr0 = 0, zr1 = 0, zk0 = 0, zk1 = 0;
    float sign = 1.f;
};
void tc_split_op(const TcOperand& o, int rpad, int kpad, void* hi, void* lo, cudaStream_t s);
int tc_gemm_planes(Ctx& c, int m, int n, int mpad, int npad, int kpad, const void* ah, const void* al, const void* bh,
                   const void* bl, float* C, int ldc, bool acc, int* err, cudaStream_t s);
int tc_pad(int n);
int tc_gemm(Ctx& c, int n, const float* A, const float* B, float* C, void* planes, int* err, cudaStream_t s,
            int terms = 3);

// linalg.cu
void gemv(int64_t n, const double* A, const double* x, double* y, cudaStream_t s, double* part,
          unsigned* counters);
int bicgstab(Ctx& c, const double* A, const double* b, double* x, cudaStream_t s);
int lu_solve(Ctx& c, const double* A, const double* b, double* x, cudaStream_t s);
// Work that follows a solve and reads only its solution (an RK4 stage's velocity and Dphi/Dt).  The
// mixed solve enqueues it behind its first round of refinement steps, before the host waits for
// that round's residual norms, so the GPU runs it while the host decides; done says whether the
// enqueued work saw the final solution (else the caller enqueues it again).
struct SolveTail {
    std::function<int()> run;
    bool done = false;
};
int mixed_solve(Ctx& c, const double* A, const double* b, double* x, cudaStream_t s, SolveTail* tail = nullptr);

int mixed_refresh(Ctx& c, const double* A, cudaStream_t s, bool from_scratch);

// ctx.cu (shared with the adjoint)
int solve_dev(Ctx& c, const double* A, const double* b, double* x, cudaStream_t s);
int rk4_step_dev(Ctx& c, double dt, cudaStream_t s);
int ensure_mixed(Ctx& c);

// export.cu
int export_ply_async(Ctx& c, const char* path);
int export_wait(Ctx& c);
void exporter_release(Ctx& c);

// exterior.cu
int exterior_potential(Ctx& c, int64_t P, const double* pts_dev, const double* phi, const double* psi,
                       double* out_dev, cudaStream_t s);

// adjoint.cu
int adjoint_record(Ctx& c, double dt, int steps);
int adjoint_backward(Ctx& c, double* xbar, double* pbar);
int volume_gradient(Ctx& c, double* xbar);

// batch.cu
int batch_mixed_solve(Ctx& c, const double* A, const double* b, double* x, cudaStream_t s);
int batch_setup_solver(Ctx& c);
int batch_build_inverses(Ctx& c, cudaStream_t s);
int batch_after_step(Ctx& c, cudaStream_t s, bool* redo);
int batch_block_stats(Ctx& c, double* rho, double* rel, int32_t* steps);

}  // namespace bemb
