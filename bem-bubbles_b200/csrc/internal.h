// Internal declarations shared by the CUDA translation units of libbem_b200.so.
// Nothing here crosses the C ABI (include/bem_b200.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <vector>

#include "../../include/bem_b200.h"

namespace bemb {

// Kernel launches issued by this library (all contexts), for the bench's launch count.
extern std::atomic<long long> g_kernel_launches;
#define KLAUNCH() (::bemb::g_kernel_launches.fetch_add(1, std::memory_order_relaxed))

// Assembly CTA: ASM_THREADS threads, 1..4 full rows of G and H held in shared memory.
constexpr int ASM_THREADS = 256;
// Shared-memory budget of one assembly CTA (B200: up to 227 KB per CTA).
constexpr int ASM_SMEM_BUDGET = 225 * 1024;
// Fields of a triangle record (stored field-major): 7 quadrature points (21), unit normal (3),
// area (1), plane offset n.a (1).
constexpr int REC = 26;
// Fixed block count of the vector kernels, so reductions have a fixed, deterministic shape.
constexpr int VBLK = 128;
constexpr int VTHR = 256;

// Topology-derived, device-resident tables (rebuilt only when the triangle list changes).
struct Topology {
    int64_t N = 0, M = 0;
    int* tri = nullptr;          // M*3 int32, reference vertex order
    int* csr_off = nullptr;      // N+1, vertex -> incident triangles (increasing index)
    int* csr_idx = nullptr;      // 3M
    // assembly work list: the columns are split into nchunks ranges [ch_c0[k], ch_c0[k+1]); chunk k
    // lists every triangle touching its columns (entries ent_off[k]..ent_off[k+1]), grouped by
    // colour, where no two triangles of one colour share a vertex (col_off: nchunks*(ncolors+1))
    int nchunks = 0, ncolors = 0, asm_rows = 1;
    int64_t E = 0;               // total entries
    int* ch_c0 = nullptr;        // nchunks+1
    int* col_off = nullptr;      // nchunks*(ncolors+1), absolute entry offsets
    int4* ent = nullptr;         // E: (triangle, vertex a, vertex b, vertex c)
    std::vector<int> h_ch_c0;
    int nparts = 0;              // loose parts (bubbles)
    int* part_of_vert = nullptr; // N
    int* part_off = nullptr;     // nparts+1 into part_tidx
    int* part_tidx = nullptr;    // triangle ids grouped by part, increasing inside a part
    int* tri_rot = nullptr;      // M*3: triangles rotated so the largest vertex id comes first,
                                 // the vertex order split_by_loose_parts leaves (Mesh.cpp:410-426)
    std::vector<int> h_part_of_vert;
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

struct Ctx;

// assemble.cu
void launch_triangle_records(Ctx& c, const double* x, cudaStream_t s);
void launch_assemble(Ctx& c, const double* x, const double* phi, double* G, double* H, double* b,
                     cudaStream_t s);

// stage.cu
void launch_velocity_prep(Ctx& c, const double* x, const double* pot, cudaStream_t s);
void launch_velocity(Ctx& c, const double* psil, double* vel, cudaStream_t s);
void launch_pot_t(Ctx& c, const double* x, const double* vel, const double* field_host, double* out,
                  cudaStream_t s);
void launch_part_volumes(Ctx& c, const double* x, double* vol, cudaStream_t s);
void launch_axpy3(int64_t n, const double* a, const double* coef_dev, double scale, const double* k,
                  double* out, cudaStream_t s);
void launch_rk4_final(Ctx& c, cudaStream_t s);
void launch_euler_final(Ctx& c, const double* vel, const double* potd, cudaStream_t s);
void launch_vertex_normals(Ctx& c, const double* x, double* out, cudaStream_t s);
void launch_get_dt(Ctx& c, const double* vel, const double* potd, double dp, cudaStream_t s);
void launch_any_negative(Ctx& c, const double* x, int* flag, cudaStream_t s);
void launch_curvature(Ctx& c, const double* x, double* kap, cudaStream_t s);

// linalg.cu
void gemv(int64_t n, const double* A, const double* x, double* y, cudaStream_t s, double* part,
          unsigned* counters);
void transpose(int64_t n, const double* A, double* B, cudaStream_t s);
size_t assemble_smem_bytes(int rows, int cw);
int bicgstab(Ctx& c, const double* A, const double* b, double* x, cudaStream_t s);
int lu_solve(Ctx& c, const double* A, const double* b, double* x, cudaStream_t s);
int mixed_solve(Ctx& c, const double* A, const double* b, double* x, cudaStream_t s);

}  // namespace bemb
