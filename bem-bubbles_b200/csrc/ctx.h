// Context object behind the opaque bem_ctx handle: parameters, device-resident state and
// every device work buffer of one simulation.
#pragma once

#include <string>
#include <utility>
#include <vector>

#include "internal.h"

namespace bemb {

// Work of the adjoint (adjoint.cu): per-step checkpoints, per-stage records of the recomputed
// step, adjoint vectors and the partial sums of the assembly derivative.
struct AdjWork {
    int64_t N = 0;
    int cap = 0, steps = 0, rch = 1, tch = 1;
    double dt = 0.0, bb = 0.0;
    double *ckx = nullptr, *ckp = nullptr, *ckt = nullptr;                  // checkpoints
    double *xs = nullptr, *ps = nullptr, *ks = nullptr, *kps = nullptr;     // 4 stages
    double *psis = nullptr, *Gs = nullptr, *Hs = nullptr;                   // 4 stages
    double *kb = nullptr, *kpb = nullptr, *xb = nullptr, *pb = nullptr;     // adjoints
    double *xsb = nullptr, *psb = nullptr, *vb = nullptr, *wv = nullptr, *psib = nullptr, *mu = nullptr, *r = nullptr;
    double *tb = nullptr, *tp = nullptr, *rec = nullptr, *partA = nullptr, *partB = nullptr, *S = nullptr;
    double *red = nullptr, *tsave = nullptr, *iox = nullptr, *iop = nullptr;
};

struct PlyExporter;  // export.cu

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bem_params prm{};
    std::string err;
    Topology topo;
    bool have_mesh = false;

    // host pressure-field callback (reference: real(*pressurefield)(vec3, real))
    bem_field_fn field_cb = nullptr;
    void* field_user = nullptr;

    // ---- device state (mesh.verts, phi, psi) and scalars
    double* x = nullptr;    // N*3
    double* phi = nullptr;  // N
    double* psi = nullptr;  // N
    DevScalars* sc = nullptr;
    DevScalars* h_sc = nullptr;  // pinned mirror
    double* h_red = nullptr;     // pinned host copy of the mixed solve's residual-norm partials
    size_t h_red_cap = 0;        // its capacity in doubles

    // ---- per-stage work
    double* G = nullptr;       // N*N column-major
    double* H = nullptr;       // N*N column-major
    double* b = nullptr;       // N
    double* psil = nullptr;    // N, solved dphi/dn of the current stage
    double* rec = nullptr;     // M*REC triangle records (quadrature points, normal, area)
    double* tn = nullptr;      // M*3 triangle unit normals (Mesh.cpp formula)
    double* tg = nullptr;      // M*3 tangential gradients of the stage potential
    double* rowHp = nullptr;   // ngroups*N partial row sums of H
    double* bp = nullptr;      // ngroups*N partial H*phi
    double* vol = nullptr;     // nparts volumes
    double* vol_part = nullptr;  // nparts x 64 chunk sums of the volume reduction
    unsigned* vol_cnt = nullptr; // nparts completion counters of the volume reduction
    double* kap = nullptr;     // N mean curvature (sigma != 0)
    double* tk = nullptr;      // M per-triangle mean curvature
    double* fieldv = nullptr;  // N per-vertex field values (callback mode)
    int* flag = nullptr;       // device int flags

    // RK4 buffers
    double *x1 = nullptr, *xs = nullptr, *k1 = nullptr, *k2 = nullptr, *k3 = nullptr, *k4 = nullptr;
    double *p1 = nullptr, *ps = nullptr, *kp1 = nullptr, *kp2 = nullptr, *kp3 = nullptr, *kp4 = nullptr;
    double* vn = nullptr;  // N*3 vertex normals
    double* gp = nullptr;  // per-group partials of G x0 (the assembly's fused first residual)
    bool r0_ready = false; // c.r holds b - G x for the start value of the next mixed solve

    // ---- solver work
    double* part = nullptr;        // GEMV partials, up to 64*N
    unsigned* cnt = nullptr;       // GEMV completion counters
    double* red = nullptr;         // reduction partials (VBLK * 8)
    double *r = nullptr, *r0 = nullptr, *pv = nullptr, *vv = nullptr, *yv = nullptr, *zv = nullptr,
           *sv = nullptr, *tv = nullptr, *invd = nullptr;
    // LU
    double* LU = nullptr;  // N*N
    int* piv = nullptr;    // N
    int* lu_perm = nullptr;  // N: the factorisation's composed row permutation (row i of P A is row lu_perm[i])
    // the LU's look-ahead: the next panel on a high-priority stream beside the current trailing update
    cudaStream_t lu_side = nullptr;
    cudaEvent_t lu_ev[2] = {nullptr, nullptr};
    double* lu_aux = nullptr;  // row-distributed panels: candidates, diagonal rows, barrier and error words
    bool lu_rows_ok = true;    // the row-distributed panel is usable (cleared after a failed launch or wait)
    // mixed: approximate inverse (FP32), Krylov basis
    float* Xinv = nullptr;     // N*N column-major
    float* Tw = nullptr;       // N*N work for the Newton-Schulz refresh
    float* G32 = nullptr;      // N*N FP32 copy of G for the refresh GEMMs
    void* tcp = nullptr;       // 4 bf16 operand planes of the split-precision tensor-core GEMM
    int* tc_err = nullptr;     // error word of the tensor-core GEMM (bounded waits)
    double* V = nullptr;       // N*(m+1) Krylov basis
    double* Z = nullptr;       // N*m preconditioned directions
    double* hcol = nullptr;    // (m+2) Hessenberg column / dot results
    double* pbicg = nullptr;   // persistent BiCGSTAB: per-row-block dots, barrier and error words
    bool pbicg_ok = true;      // the persistent BiCGSTAB is usable (cleared after a failed launch or wait)
    int* rf_bar = nullptr;     // the mixed solve's round kernel: grid barrier words [0..1], error word [2]
    bool refine_ok = true;     // its cooperative launch is usable (cleared after a failed launch or wait)
    long long wait_limit = 2000000000LL;  // bound of the persistent kernels' grid-barrier waits, SM cycles
    // G-only assembly of the step path: patch-ordered triangle records, halo columns (nhalo x N; the
    // storage of H when nhalo <= N, since the step path does not write H), error word of its bulk copies
    double* prec = nullptr;
    double* halo = nullptr;
    int* asm_err = nullptr;
    bool xinv_valid = false;
    int mixed_backoff = 0;  // solves left that skip the mixed path after it failed (FP64 BiCGSTAB instead)
    int ir_base = -1;       // fewest refinement steps of a solve since the last refresh of X
    int ir_excess = 0;      // refinement steps paid above ir_base since the last refresh
    int ir_steps = 3;  // refinement steps issued per round of the mixed solve (adapted)
    // the same per RK4 stage of the step loop (stages differ in how good their start values are), and
    // whether that stage's last solve converged in its first round (then its consumers are enqueued
    // behind that round, see SolveTail); solve_stage: the stage of the current solve, or -1
    int ir_steps_stage[4] = {3, 3, 3, 3};
    bool stage_round0[4] = {false, false, false, false};
    // gated extra steps of the next first round per RK4 stage: 2 after a solve that used an extra step
    // or a second round, else 1
    int ir_extra_stage[4] = {2, 2, 2, 2};
    int solve_stage = -1;
    // Stage predictor of the mixed solve (single systems): the solutions of the RK4 stages of the last
    // PRED_DEPTH steps and the stage times, a ring over steps (pred_head: the slot the current step
    // writes, which holds the oldest step until then).  psih_t[PRED_CNT]: steps in the ring that
    // continue the current trajectory, kept on the device; a change of state from outside the step
    // loop clears it.
    double* psih = nullptr;    // [PRED_DEPTH][4][N]
    double* psih_t = nullptr;  // [PRED_DEPTH][4] + 1
    int pred_head = 0;
    int gmres_m = 30;

    // ---- block-diagonal batch (batch = true): independent sub-systems (bubbles) sharing the mesh
    // arrays; G and H are stored as packed n_b x n_b blocks
    bool batch = false;
    int batch_cg = 0;  // column-group width forced by the autotuner (0: default)
    int nblk = 1;
    std::vector<BlockInfo> h_blk;
    BlockInfo* blk = nullptr;  // device copy
    int* vblk = nullptr;       // N: block of each vertex
    int4* tiles = nullptr;     // assembly work list {group, first row, block, local group}
    int ntiles = 0;
    unsigned* tile_ctr = nullptr;
    int asm_grid = 0, asm_grid_cg = 0;  // persistent assembly grid and the tile shape it was sized for
    double* ppar = nullptr;    // per part {V0, field amp, kx, omega, phase}; null: the scalar parameters
    long long blk_elems = 0;   // sum of n_b^2
    // batched mixed solve (batch.cu)
    float* Xb = nullptr;        // packed FP32 approximate inverses
    int4* gv_items = nullptr;   // GEMV work list {block, row block, column split, 0}
    int gv_nitems = 0;
    int nrb_total = 0;          // sum of row blocks
    double* bpart = nullptr;    // batched GEMV column-split partials
    unsigned* bcnt = nullptr;   // batched GEMV row-block counters
    double* brnorm = nullptr;   // per row block residual norms
    int* bconv = nullptr;       // per block: converged in the current solve
    double* bstat = nullptr;    // per block: BSTAT_W doubles (norms, contraction)
    double* bstat_h = nullptr;  // pinned host mirror
    std::vector<char> bvalid;   // per block: inverse built
    std::vector<int> part_block;      // block of each loose part
    std::vector<double> h_ppar;       // host mirror of ppar
    std::vector<int64_t> h_trigs, h_voff;  // the batch's triangles and block offsets (re-planning)
    double* time_save = nullptr;      // device copy of the time at the start of a batched step
    float *bG32 = nullptr, *bT = nullptr, *bP = nullptr;  // Newton-Schulz work, largest block
    int bmax_n = 0;
    // CUDA graph of one batched RK4 step
    cudaGraphExec_t graph_exec = nullptr;
    double graph_dt = 0.0;
    long long graph_launches = 0;

    // ---- pinned contact line (pin.cu): the last n_pin vertices lie on the wall x = 0; drift-velocity
    // law beta (cos_eq - c) + c_nl c^3 / (c^2 - 1)
    int64_t n_pin = 0;
    double pin_beta = 0.0, pin_cos_eq = 0.0, pin_cnl = 0.0;
    double* potz = nullptr;  // N: stage potential with the pinned entries zeroed

    // pinned host staging of bem_set_state / bem_get_state (5N doubles) and the event of its last use
    double* h_stage = nullptr;
    size_t stage_cap = 0;
    cudaEvent_t stage_ev = nullptr;
    cudaEvent_t solve_ev = nullptr;  // end of the mixed solve's first-round norm readback

    // remesh ray casting (remesh.cu): one device buffer, grown on demand, kept across meshes
    void* trace_buf = nullptr;
    size_t trace_cap = 0;

    AdjWork adj;
    PlyExporter* exporter = nullptr;  // asynchronous PLY writer (export.cu)
    std::vector<int> h_tri;           // host copy of the triangles (M*3)

    // statistics
    bem_stats stats{};

    // device-time profiling (CUDA events on the context's stream)
    bool prof = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_asm, ev_solve;
    bem_profile prof_acc{};
    long long launches_at_reset = 0;
    cudaEvent_t take_event() {
        if (ev_pool.empty()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            return e;
        }
        cudaEvent_t e = ev_pool.back();
        ev_pool.pop_back();
        return e;
    }

    size_t bytes = 0;
    // device allocations of the current mesh, in allocation order, with their sizes
    std::vector<std::pair<void*, size_t>> allocs;
    // allocations of the previous mesh kept for re-use when the mesh changes (remeshing): the k-th
    // allocation of the new mesh takes the k-th block of the old one if it is large enough
    std::vector<std::pair<void*, size_t>> reuse;
    size_t reuse_pos = 0;

    int fail(int code, const std::string& m) {
        err = m;
        return code;
    }
};

// Device allocation recorded in the context (freed together by free_all).  When a mesh replaces
// another, the allocations are made in the same order as before, so the k-th one re-uses the k-th
// block of the previous mesh if it is large enough; a block that is too small is replaced by one with
// 1/8 headroom, since a remeshed surface's vertex count moves by a few per cent either way.
template <typename T>
inline int dalloc(Ctx& c, T** p, size_t count) {
    if (count == 0) count = 1;
    size_t bytes = count * sizeof(T);
    if (c.reuse_pos < c.reuse.size()) {
        const auto blk = c.reuse[c.reuse_pos];
        c.reuse[c.reuse_pos++] = {nullptr, 0};
        if (blk.second >= bytes) {
            *p = (T*)blk.first;
            c.allocs.push_back(blk);
            c.bytes += blk.second;
            return BEM_OK;
        }
        cudaFree(blk.first);
        bytes += bytes / 8;
    }
    cudaError_t e = cudaMalloc((void**)p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return c.fail(BEM_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    c.allocs.push_back({(void*)*p, bytes});
    c.bytes += bytes;
    return BEM_OK;
}
template <typename T>
inline int upload_vec(Ctx& c, T** dst, const std::vector<T>& src) {
    int rc = dalloc(c, dst, src.size());
    if (rc) return rc;
    if (cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
        return c.fail(BEM_ERR_CUDA, "cudaMemcpy (upload)");
    return BEM_OK;
}

// Record a CUDA error in the context and map it to a status.
#define BEM_CUDA(c, call)                                                              \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            return (c).fail(BEM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

}  // namespace bemb
