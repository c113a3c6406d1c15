// Block-diagonal batches: many independent bubbles (a radius x pressure sweep) stepped as one
// simulation whose systems do not couple.  The mesh arrays are shared (every per-vertex and
// per-triangle kernel of a stage runs once over all bubbles); G and H are packed n_b x n_b blocks.
//
// Solve: the mixed-precision refinement of linalg.cu, x <- x + X_b (b - G_b x) per block, issued
// without host synchronisation so that a whole RK4 step can be captured as one CUDA graph.  Each
// refinement step is three launches over all blocks: the FP64 residual GEMV (with per-row-block
// residual norms), a decision kernel (one warp per block: relative residual, contraction, converged
// flag) and the FP32 correction GEMV.  Blocks flagged converged drop out of the later GEMVs.  After
// the step the host reads the per-block contraction and refreshes the approximate inverses that
// have gone stale (Newton-Schulz on the tensor cores, outside the graph); a block that missed the
// tolerance makes the step run again from its saved start state after the refresh.
#include <math.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "ctx.h"

namespace bemb {

constexpr int BG_ROWS = 256;  // rows per CTA of the batched GEMV
constexpr int BG_COLS = 512;  // target columns per column split

static __device__ __forceinline__ double warp_sum_b(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// deterministic sum over a CTA of BG_ROWS threads; valid in thread 0
static __device__ double cta_sum_b(double v) {
    __shared__ double s_w[BG_ROWS / 32];
    v = warp_sum_b(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) s_w[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        r = (lane < BG_ROWS / 32) ? s_w[lane] : 0.0;
        r = warp_sum_b(r);
    }
    return r;
}

// y_b = cvec_b + sgn * A_b x_b (cvec null: y_b = A_b x_b) for every block not gated off.  Work list
// item {block, row block, column split}; the column-split partials of a row block are summed in a
// fixed order by the CTA that finishes last.  rnorm (optional): per row block, sum of y_i^2.
template <typename T>
__global__ void __launch_bounds__(BG_ROWS) k_bgemv(const int4* __restrict__ items, const BlockInfo* __restrict__ blk,
                                                   const T* __restrict__ A, const double* __restrict__ x, double* y,
                                                   double* __restrict__ part, unsigned* __restrict__ cnt,
                                                   const int* __restrict__ gate, const double* cvec, double sgn,
                                                   double* __restrict__ rnorm) {
    const int4 it = items[blockIdx.x];
    if (gate && gate[it.x]) return;
    const BlockInfo B = blk[it.x];
    const int n = B.n, rb = it.y, cs = it.z, ncs = B.ncs;
    const int il = rb * BG_ROWS + threadIdx.x;
    const int chunk = (n + ncs - 1) / ncs;
    const int c0 = cs * chunk, c1 = min(n, c0 + chunk);
    const double* xb = x + B.vbase;
    double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0, acc3 = 0.0;
    if (il < n) {
        const T* col = A + B.mbase + (size_t)c0 * n + il;
        int j = c0;
        for (; j + 3 < c1; j += 4) {
            T a0 = col[0], a1 = col[(size_t)n], a2 = col[2 * (size_t)n], a3 = col[3 * (size_t)n];
            acc0 = fma((double)a0, __ldg(xb + j), acc0);
            acc1 = fma((double)a1, __ldg(xb + j + 1), acc1);
            acc2 = fma((double)a2, __ldg(xb + j + 2), acc2);
            acc3 = fma((double)a3, __ldg(xb + j + 3), acc3);
            col += 4 * (size_t)n;
        }
        for (; j < c1; ++j) {
            acc0 = fma((double)col[0], __ldg(xb + j), acc0);
            col += n;
        }
        part[B.pofs + (size_t)cs * n + il] = (acc0 + acc1) + (acc2 + acc3);
    }
    __threadfence();
    __shared__ unsigned s_ticket;
    __syncthreads();
    if (threadIdx.x == 0) s_ticket = atomicAdd(&cnt[B.rbase + rb], 1u);
    __syncthreads();
    if (s_ticket != (unsigned)(ncs - 1)) return;
    __threadfence();
    double yi = 0.0;
    if (il < n) {
        for (int k = 0; k < ncs; ++k) yi += __ldcg(part + B.pofs + (size_t)k * n + il);
        if (cvec) yi = fma(sgn, yi, cvec[B.vbase + il]);
        y[B.vbase + il] = yi;
    }
    if (rnorm) {
        const double v = cta_sum_b(il < n ? yi * yi : 0.0);
        if (threadIdx.x == 0) rnorm[B.rbase + rb] = v;
    }
    if (threadIdx.x == 0) cnt[B.rbase + rb] = 0u;
}

// Per-block statistics (BSTAT_W doubles per block)
enum { BS_BB = 0, BS_FIRST = 1, BS_LAST = 2, BS_RHO = 3, BS_STEPS = 4, BS_CONV = 5, BSTAT_W = 8 };

// Start of a solve: ||b_b||^2, statistics reset; a zero right-hand side gives x_b = 0, converged.
__global__ void __launch_bounds__(BG_ROWS) k_binit(const BlockInfo* __restrict__ blk, const double* __restrict__ b,
                                                   double* __restrict__ x, double* __restrict__ st,
                                                   int* __restrict__ conv) {
    const BlockInfo B = blk[blockIdx.x];
    double s = 0.0;
    for (int i = threadIdx.x; i < B.n; i += BG_ROWS) s += b[B.vbase + i] * b[B.vbase + i];
    s = cta_sum_b(s);
    __shared__ double s_bb;
    if (threadIdx.x == 0) s_bb = s;
    __syncthreads();
    const double bb = s_bb;
    if (bb == 0.0)
        for (int i = threadIdx.x; i < B.n; i += BG_ROWS) x[B.vbase + i] = 0.0;
    if (threadIdx.x == 0) {
        double* q = st + (size_t)BSTAT_W * blockIdx.x;
        q[BS_BB] = bb;
        q[BS_FIRST] = q[BS_LAST] = 0.0;
        q[BS_RHO] = 0.0;
        q[BS_STEPS] = 0.0;
        q[BS_CONV] = bb == 0.0 ? 1.0 : 0.0;
        conv[blockIdx.x] = bb == 0.0 ? 1 : 0;
    }
}

// After the residual of refinement step k: relative residual, contraction (from steps still well
// above the tolerance), converged flag.  One warp per block.
__global__ void k_bdecide(int nblk, const BlockInfo* __restrict__ blk, const double* __restrict__ rnorm,
                          double* __restrict__ st, int* __restrict__ conv, int k, double tol) {
    const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (b >= nblk || conv[b]) return;
    const BlockInfo B = blk[b];
    const int nrb = (B.n + BG_ROWS - 1) / BG_ROWS;
    double rr = 0.0;
    for (int q = lane; q < nrb; q += 32) rr += rnorm[B.rbase + q];
    rr = warp_sum_b(rr);
    if (lane) return;
    double* q = st + (size_t)BSTAT_W * b;
    const double rel = sqrt(rr / q[BS_BB]);
    if (k == 0)
        q[BS_FIRST] = rel;
    else if (q[BS_LAST] > 1e3 * tol)
        q[BS_RHO] = fmax(q[BS_RHO], rel / q[BS_LAST]);
    q[BS_LAST] = rel;
    q[BS_STEPS] = (double)k;
    if (rel <= tol) {
        conv[b] = 1;
        q[BS_CONV] = 1.0;
    }
}

constexpr int BATCH_KMAX = 8;

int batch_mixed_solve(Ctx& c, const double* A, const double* b, double* x, cudaStream_t s) {
    const double tol = c.prm.mixed_tol > 0 ? c.prm.mixed_tol : 1e-12;
    const int nb = c.nblk;
    double* rn = c.brnorm;
    KLAUNCH(), k_binit<<<nb, BG_ROWS, 0, s>>>(c.blk, b, x, c.bstat, c.bconv);
    const int dgrid = (nb * 32 + 255) / 256;
    for (int k = 0; k <= BATCH_KMAX; ++k) {
        KLAUNCH(), k_bgemv<double><<<c.gv_nitems, BG_ROWS, 0, s>>>(c.gv_items, c.blk, A, x, c.r, c.bpart, c.bcnt, c.bconv,
                                                                  b, -1.0, rn);
        KLAUNCH(), k_bdecide<<<dgrid, 256, 0, s>>>(nb, c.blk, rn, c.bstat, c.bconv, k, tol);
        if (k == BATCH_KMAX) break;
        KLAUNCH(), k_bgemv<float><<<c.gv_nitems, BG_ROWS, 0, s>>>(c.gv_items, c.blk, c.Xb, c.r, x, c.bpart, c.bcnt, c.bconv,
                                                                 x, 1.0, nullptr);
    }
    c.stats.solves++;
    return BEM_OK;
}

// ------------------------------------------------------------------------------------------------
// Set-up of the batched solve: work lists and buffers (after the topology and blocks are known)
// ------------------------------------------------------------------------------------------------
int batch_setup_solver(Ctx& c) {
    std::vector<int4> items;
    int rbase = 0;
    long long pofs = 0;
    // column splits: at most BG_COLS columns per item, and for large blocks enough items to keep
    // four CTAs per SM busy by themselves in proportion to their share of the matrix elements
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
    double tot = 0.0;
    for (auto& B : c.h_blk) tot += (double)B.n * B.n;
    for (auto& B : c.h_blk) {
        const int nrb = (B.n + BG_ROWS - 1) / BG_ROWS;
        const int fill = (int)std::ceil(4.0 * sms * ((double)B.n * B.n / tot) / nrb);
        B.rbase = rbase;
        B.ncs = std::max(1, std::min(std::min(64, std::max(1, B.n / 16)), std::max((B.n + BG_COLS - 1) / BG_COLS, fill)));
        B.pofs = pofs;
        rbase += nrb;
        pofs += (long long)B.ncs * B.n;
    }
    // largest blocks first: the long work items start early
    std::vector<int> order((size_t)c.nblk);
    for (int b = 0; b < c.nblk; ++b) order[(size_t)b] = b;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return c.h_blk[(size_t)a].n > c.h_blk[(size_t)b].n; });
    for (int b : order) {
        const BlockInfo& B = c.h_blk[(size_t)b];
        const int nrb = (B.n + BG_ROWS - 1) / BG_ROWS;
        for (int cs = 0; cs < B.ncs; ++cs)
            for (int rb = 0; rb < nrb; ++rb) items.push_back(make_int4(b, rb, cs, 0));
    }
    c.gv_nitems = (int)items.size();
    c.nrb_total = rbase;
    int rc;
    if ((rc = upload_vec(c, &c.gv_items, items)) || (rc = upload_vec(c, &c.blk, c.h_blk)) ||
        (rc = dalloc(c, &c.bpart, (size_t)pofs)) || (rc = dalloc(c, &c.bcnt, (size_t)rbase)) ||
        (rc = dalloc(c, &c.brnorm, (size_t)rbase)) || (rc = dalloc(c, &c.bconv, (size_t)c.nblk)) ||
        (rc = dalloc(c, &c.bstat, (size_t)BSTAT_W * c.nblk)))
        return rc;
    BEM_CUDA(c, cudaMemset(c.bcnt, 0, sizeof(unsigned) * (size_t)rbase));
    BEM_CUDA(c, cudaMallocHost((void**)&c.bstat_h, sizeof(double) * BSTAT_W * (size_t)c.nblk));  // freed by free_all
    c.bmax_n = 0;
    for (auto& B : c.h_blk) c.bmax_n = std::max(c.bmax_n, B.n);
    const size_t mx = (size_t)c.bmax_n * c.bmax_n, np = (size_t)tc_pad(c.bmax_n) * tc_pad(c.bmax_n);
    uint16_t* planes = nullptr;
    if ((rc = dalloc(c, &c.Xb, (size_t)c.blk_elems)) || (rc = dalloc(c, &c.bG32, mx)) || (rc = dalloc(c, &c.bT, mx)) ||
        (rc = dalloc(c, &c.bP, mx)) || (rc = dalloc(c, &planes, 4 * np)) || (rc = dalloc(c, &c.tc_err, 1)))
        return rc;
    c.tcp = planes;
    BEM_CUDA(c, cudaMemset(c.tc_err, 0, sizeof(int)));
    c.bvalid.assign((size_t)c.nblk, 0);
    return BEM_OK;
}

// Newton-Schulz refresh of block b's approximate inverse against its current G block: one step
// from the stale inverse, or from scratch when there is none or the stale one no longer contracts.
static int refresh_block(Ctx& c, const double* A, int b, cudaStream_t s) {
    const BlockInfo& B = c.h_blk[(size_t)b];
    const NSJob j{B.n, A + B.mbase, c.bG32, c.Xb + B.mbase, c.bT, c.bP};
    to_f32((int64_t)B.n * B.n, j.A, c.bG32, s);
    if (c.bvalid[(size_t)b]) {
        double e = 0.0;
        int rc = ns_step(c, j, s, &e);
        if (rc) return rc;
        if (e < 0.9) {
            c.stats.precond_refresh++;
            return BEM_OK;
        }
    }
    c.bvalid[(size_t)b] = 0;
    int rc = ns_from_scratch(c, j, s, false);
    if (rc) return rc;
    c.bvalid[(size_t)b] = 1;
    c.stats.precond_refresh++;
    return BEM_OK;
}

// Approximate inverses of every block that has none, from the G blocks currently assembled.
int batch_build_inverses(Ctx& c, cudaStream_t s) {
    for (int b = 0; b < c.nblk; ++b)
        if (!c.bvalid[(size_t)b]) {
            int rc = refresh_block(c, c.G, b, s);
            if (rc) return rc;
        }
    return BEM_OK;
}

// After a batched step: per-block statistics of the last solve to the host.  Blocks whose
// contraction exceeded 0.02 get a refresh against the G blocks of that last solve; *redo is set when
// a block missed the tolerance within the refinement steps (the caller re-runs the step).
int batch_after_step(Ctx& c, cudaStream_t s, bool* redo) {
    *redo = false;
    BEM_CUDA(c, cudaMemcpyAsync(c.bstat_h, c.bstat, sizeof(double) * BSTAT_W * (size_t)c.nblk, cudaMemcpyDeviceToHost, s));
    BEM_CUDA(c, cudaStreamSynchronize(s));
    double worst = 0.0;
    for (int b = 0; b < c.nblk; ++b) {
        const double* q = c.bstat_h + (size_t)BSTAT_W * b;
        worst = std::max(worst, q[BS_LAST]);
        const bool ok = q[BS_CONV] != 0.0;
        if (!ok) *redo = true;
        if (!ok || q[BS_RHO] > 0.02) {
            int rc = refresh_block(c, c.G, b, s);
            if (rc) return rc;
        }
    }
    c.stats.last_rel_residual = worst;
    return BEM_OK;
}

int batch_block_stats(Ctx& c, double* rho, double* rel, int32_t* steps) {
    BEM_CUDA(c, cudaMemcpyAsync(c.bstat_h, c.bstat, sizeof(double) * BSTAT_W * (size_t)c.nblk, cudaMemcpyDeviceToHost,
                                c.stream));
    BEM_CUDA(c, cudaStreamSynchronize(c.stream));
    for (int b = 0; b < c.nblk; ++b) {
        const double* q = c.bstat_h + (size_t)BSTAT_W * b;
        if (rho) rho[b] = q[BS_RHO];
        if (rel) rel[b] = q[BS_LAST];
        if (steps) steps[b] = (int32_t)q[BS_STEPS];
    }
    return BEM_OK;
}

}  // namespace bemb
