// Dense solvers for G psi = H phi (Simulation::solve_system, Bem/Simulation/Simulation.cpp:40-71).
//
//   * BiCGSTAB (the reference default, Simulation.hpp:38): Jacobi preconditioner, zero start,
//     tolerance DBL_EPSILON on the recursive residual, at most 2N iterations, restart of the shadow
//     residual when rho vanishes -- the documented Eigen 3.4 BiCGSTAB<MatrixXd> behaviour.  All
//     scalars live on the device; the host only polls the done flag every few iterations.
//   * LU with row partial pivoting (PartialPivLU): right-looking blocked factorisation in FP64.
//   * MIXED: FP64 GMRES on G, right-preconditioned by an FP32 approximate inverse X ~ G^-1 kept
//     across stages and steps and refreshed by Newton-Schulz (X <- X(2I - G X)) when the Krylov
//     iteration count grows.  The answer is the FP64 G's solution to the relative residual
//     `mixed_tol` (checked on the true residual), whatever the quality of X.
//
// GEMV on the column-major N x N matrices is HBM-bound: a 2-D grid (row blocks x column splits),
// fixed-order reduction of the column-split partials by the last CTA of each row block.
#include <math.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "ctx.h"
#include "grid_barrier.cuh"

namespace bemb {

constexpr int GV_ROWS = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum n partials in a fixed order; result valid in every thread of the block.
__device__ double block_reduce_partials(const double* __restrict__ p, int n) {
    __shared__ double s_out;
    if (threadIdx.x < 32) {
        double a = 0.0;
        for (int k = threadIdx.x; k < n; k += 32) a += p[k];
        a = warp_sum(a);
        if (threadIdx.x == 0) s_out = a;
    }
    __syncthreads();
    double r = s_out;
    __syncthreads();
    return r;
}

// Deterministic block sum of per-thread values (blockDim.x a multiple of 32, <= 1024).
__device__ double block_sum(double v) {
    __shared__ double s_w[32];
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) s_w[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        r = (lane < (int)(blockDim.x >> 5)) ? s_w[lane] : 0.0;
        r = warp_sum(r);
        if (lane == 0) s_w[0] = r;
    }
    __syncthreads();
    r = s_w[0];
    __syncthreads();
    return r;
}

// L2 eviction policies of the GEMV's matrix loads (createpolicy, PTX ISA 7.4): the FP64 G streams
// through with evict_first, the FP32 approximate inverse X (half G's size) is loaded with evict_last
// so that it can stay in L2 across the refinement steps of one solve while G passes by.
__device__ __forceinline__ uint64_t l2_policy(bool keep) {
    uint64_t p;
    if (keep)
        asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    else
        asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// One matrix element through the read-only path, without L1 allocation, with the L2 policy pol.
__device__ __forceinline__ double ld_mat(const double* p, uint64_t pol) {
    double v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ double ld_mat(const float* p, uint64_t pol) {
    float v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return (double)v;
}

// y = A x; A column-major (T = double or float), x and y FP64.  grid (row blocks of GV_ROWS rows,
// column splits of `chunk` columns, a multiple of GV_UNR).  One row per thread; GV_UNR columns are
// loaded before they are used.  The column-split partials are summed in a fixed order by the last
// CTA of each row block (ticket counter), so the result is deterministic.
// Optional fused dots of the result: d1 = y.u, d2 = y.w partials per row block.
// y, u and w are not __restrict__: callers pass u == y to get y.y.  With cvec != null the result is
// y = cvec + sgn * (A x) (residuals b - A x, accumulations x + X r); cvec may alias y.
// Measured on B200 at n = 4002, back to back as in the refinement loop: one FP64 and one FP32 GEMV
// take 45 us together (256 rows x 64 column splits; wider vector loads per thread and TMA-staged
// columns were both slower, and the serial tail of the split sum cost 5-7 us before its loads were
// batched).
constexpr int GV_UNR = 8;
// One tile (row block rb, column split cs of `chunk` columns, ncs splits) of y = A x, the split sum
// by the last CTA of the row block, and its fused dots.  COHERENT: x, cvec and the partials may have
// been written earlier in the same kernel (the persistent refinement), so they are read through L2
// (ld.global.cg) rather than the read-only path; the arithmetic is the same either way.
template <typename T, bool COHERENT>
__device__ __forceinline__ void gemv_tile(int n, int chunk, int ncs, int rb, int cs, const T* __restrict__ A,
                                          const double* x, double* y, double* __restrict__ part,
                                          unsigned* __restrict__ cnt, const double* u, double* __restrict__ du,
                                          const double* w, double* __restrict__ dw, const double* cvec, double sgn,
                                          double* sx = nullptr) {
    const int i = rb * GV_ROWS + threadIdx.x;
    const int c0 = min(n, cs * chunk), c1 = min(n, c0 + chunk);
    if (COHERENT) {
        // the tile's slice of x, once through L2 into shared memory; the loop below reads it back as
        // broadcasts (sx - c0 + j is x[j])
        __syncthreads();
        for (int j = c0 + (int)threadIdx.x; j < c1; j += GV_ROWS) sx[j - c0] = __ldcg(x + j);
        __syncthreads();
    }
    const int xo = COHERENT ? c0 : 0;  // x[j] is xv[j - xo]
    const double* xv = COHERENT ? sx : x;
    if (i < n) {
        const uint64_t pol = l2_policy(sizeof(T) == 4);
        double acc0 = 0.0, acc1 = 0.0;
        const T* col = A + (size_t)c0 * n + i;
        int j = c0;
        for (; j + GV_UNR <= c1; j += GV_UNR) {
            double a[GV_UNR];
#pragma unroll
            for (int q = 0; q < GV_UNR; ++q) a[q] = ld_mat(col + (size_t)q * n, pol);
#pragma unroll
            for (int q = 0; q < GV_UNR; q += 2) {
                acc0 = fma(a[q], COHERENT ? xv[j + q - xo] : __ldg(xv + j + q), acc0);
                acc1 = fma(a[q + 1], COHERENT ? xv[j + q + 1 - xo] : __ldg(xv + j + q + 1), acc1);
            }
            col += (size_t)GV_UNR * n;
        }
        for (; j < c1; ++j) {
            acc0 = fma(ld_mat(col, pol), COHERENT ? xv[j - xo] : __ldg(xv + j), acc0);
            col += n;
        }
        part[(size_t)cs * n + i] = acc0 + acc1;
    }
    __threadfence();
    __shared__ unsigned s_ticket;
    __syncthreads();
    if (threadIdx.x == 0) s_ticket = atomicAdd(&cnt[rb], 1u);
    __syncthreads();
    if (s_ticket != (unsigned)(ncs - 1)) return;
    // last CTA of this row block: the column-split partials of each row summed in split order.  This
    // runs after every other CTA of the row block has finished, so its latency is the kernel's tail:
    // the partials are loaded 16 at a time before they are added, instead of one dependent L2 round
    // trip per split.
    __threadfence();
    constexpr int PB = 16;
    double yi = 0.0;
    if (i < n) {
        int k = 0;
        for (; k + PB <= ncs; k += PB) {
            double pv[PB];
#pragma unroll
            for (int q = 0; q < PB; ++q) pv[q] = __ldcg(part + (size_t)(k + q) * n + i);
#pragma unroll
            for (int q = 0; q < PB; ++q) yi += pv[q];
        }
        for (; k < ncs; ++k) yi += __ldcg(part + (size_t)k * n + i);
        if (cvec) yi = fma(sgn, yi, COHERENT ? __ldcg(cvec + i) : cvec[i]);
        y[i] = yi;
    }
    if (du) {
        const double v = block_sum((i < n) ? yi * (COHERENT ? __ldcg(u + i) : u[i]) : 0.0);
        if (threadIdx.x == 0) du[rb] = v;
    }
    if (dw) {
        const double v = block_sum((i < n) ? yi * (COHERENT ? __ldcg(w + i) : w[i]) : 0.0);
        if (threadIdx.x == 0) dw[rb] = v;
    }
    if (threadIdx.x == 0) cnt[rb] = 0u;
}

// y = A x; A column-major (T = double or float), x and y FP64.  grid (row blocks of GV_ROWS rows,
// column splits of `chunk` columns, a multiple of GV_UNR).  One row per thread; GV_UNR columns are
// loaded before they are used.  The column-split partials are summed in a fixed order by the last
// CTA of each row block (ticket counter), so the result is deterministic.
// Optional fused dots of the result: d1 = y.u, d2 = y.w partials per row block.
// y, u and w are not __restrict__: callers pass u == y to get y.y.  With cvec != null the result is
// y = cvec + sgn * (A x) (residuals b - A x, accumulations x + X r); cvec may alias y.
// Measured on B200 at n = 4002, back to back as in the refinement loop: one FP64 and one FP32 GEMV
// take 45 us together (256 rows x 64 column splits; wider vector loads per thread and TMA-staged
// columns were both slower, and the serial tail of the split sum cost 5-7 us before its loads were
// batched).
template <typename T>
__global__ void __launch_bounds__(GV_ROWS) k_gemv(int n, int chunk, const T* __restrict__ A,
                                                  const double* __restrict__ x, double* y,
                                                  double* __restrict__ part, unsigned* __restrict__ cnt,
                                                  const int* __restrict__ gate, int gate_val, const double* u,
                                                  double* __restrict__ du, const double* w, double* __restrict__ dw,
                                                  const double* cvec, double sgn) {
    if (gate && *gate != gate_val) return;
    gemv_tile<T, false>(n, chunk, gridDim.y, blockIdx.x, blockIdx.y, A, x, y, part, cnt, u, du, w, dw, cvec, sgn);
}

// Column splits: enough CTAs for about eight per SM, at most 64 (the partials buffer holds 64 n).
static int gemv_splits(int n) {
    const int rb = (n + GV_ROWS - 1) / GV_ROWS;
    int cs = std::max(1, std::min(64, (8 * 148 + rb - 1) / rb));
    cs = std::min(cs, std::max(1, n / 16));
    return cs;
}

template <typename T>
static void gemv_t(int n, const T* A, const double* x, double* y, cudaStream_t s, double* part, unsigned* cnt,
                   const int* gate = nullptr, int gate_val = 0, const double* u = nullptr, double* du = nullptr,
                   const double* w = nullptr, double* dw = nullptr, const double* cvec = nullptr, double sgn = 1.0) {
    const int ncs = gemv_splits(n);
    const int chunk = ((n + ncs - 1) / ncs + GV_UNR - 1) / GV_UNR * GV_UNR;
    dim3 grid((n + GV_ROWS - 1) / GV_ROWS, ncs);
    KLAUNCH(), k_gemv<T><<<grid, GV_ROWS, 0, s>>>(n, chunk, A, x, y, part, cnt, gate, gate_val, u, du, w, dw, cvec, sgn);
}

void gemv(int64_t n, const double* A, const double* x, double* y, cudaStream_t s, double* part, unsigned* cnt) {
    gemv_t<double>((int)n, A, x, y, s, part, cnt);
}

// ------------------------------------------------------------------------------------------------
// BiCGSTAB
// ------------------------------------------------------------------------------------------------
constexpr double DEPS = 2.220446049250313080847e-16;

// partial-sum slots inside Ctx::red (VBLK each)
enum { RS_RR = 0, RS_R0R = 1, RS_R0V = 2, RS_TT = 3, RS_TS = 4, RS_BB = 5, RS_N = 6 };

__global__ void k_bicg_init(int n, const double* __restrict__ A, const double* __restrict__ b,
                            double* __restrict__ x, double* __restrict__ r, double* __restrict__ r0,
                            double* __restrict__ p, double* __restrict__ v, double* __restrict__ invd,
                            double* __restrict__ red) {
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double d = A[(size_t)i * n + i];
        invd[i] = (d != 0.0) ? 1.0 / d : 1.0;
        x[i] = 0.0;
        r[i] = b[i];
        r0[i] = b[i];
        p[i] = 0.0;
        v[i] = 0.0;
        s += b[i] * b[i];
    }
    s = block_sum(s);
    if (threadIdx.x == 0) {
        red[RS_BB * VBLK + blockIdx.x] = s;
        red[RS_RR * VBLK + blockIdx.x] = s;
        red[RS_R0R * VBLK + blockIdx.x] = s;
    }
}

__global__ void k_bicg_init_scalars(DevScalars* sc, const double* __restrict__ red, int maxit) {
    double bb = block_reduce_partials(red + RS_BB * VBLK, VBLK);
    if (threadIdx.x == 0) {
        sc->rhs_sq = bb;
        sc->r0_sq = bb;
        sc->rho = 1.0;
        sc->alpha = 1.0;
        sc->w = 1.0;
        sc->tol2 = DEPS * DEPS * bb;
        sc->iters = 0;
        sc->restarts = 0;
        sc->done = (bb == 0.0) ? 1 : 0;
        sc->restart_flag = 0;
        sc->maxit = maxit;
        sc->nonconv = 0;
    }
}

// Loop test, rho, restart decision and beta (one CTA).
__global__ void k_bicg_begin(DevScalars* sc, const double* __restrict__ red) {
    double rr = block_reduce_partials(red + RS_RR * VBLK, VBLK);
    double r0r = block_reduce_partials(red + RS_R0R * VBLK, VBLK);
    if (threadIdx.x != 0 || sc->done) return;
    sc->rr = rr;
    if (!(rr > sc->tol2) || sc->iters >= sc->maxit) {
        sc->done = 1;
        sc->nonconv = (rr > sc->tol2) ? 1 : 0;
        return;
    }
    double rho_old = sc->rho;
    sc->beta = rho_old;  // kept for the restart path
    if (fabs(r0r) < DEPS * DEPS * sc->r0_sq) {
        sc->restart_flag = 1;
        return;
    }
    sc->restart_flag = 0;
    sc->rho = r0r;
    sc->beta = (r0r / rho_old) * (sc->alpha / sc->w);
}

// restart: r = b - t (t = A x), r0 = r, partial r.r
__global__ void k_bicg_restart_update(int n, const DevScalars* sc, const double* __restrict__ b,
                                      const double* __restrict__ t, double* __restrict__ r, double* __restrict__ r0,
                                      double* __restrict__ red) {
    if (sc->done || !sc->restart_flag) return;
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double ri = b[i] - t[i];
        r[i] = ri;
        r0[i] = ri;
        s += ri * ri;
    }
    s = block_sum(s);
    if (threadIdx.x == 0) red[RS_RR * VBLK + blockIdx.x] = s;
}

__global__ void k_bicg_restart_scalars(DevScalars* sc, const double* __restrict__ red) {
    double rr = block_reduce_partials(red + RS_RR * VBLK, VBLK);
    if (threadIdx.x != 0 || sc->done || !sc->restart_flag) return;
    double rho_old = sc->beta;
    sc->rho = rr;
    sc->r0_sq = rr;
    if (sc->restarts++ == 0) sc->iters = 0;
    sc->beta = (rr / rho_old) * (sc->alpha / sc->w);
    sc->restart_flag = 0;
}

// p = r + beta (p - w v); y = invd .* p
__global__ void k_bicg_p(int n, const DevScalars* sc, const double* __restrict__ r, double* __restrict__ p,
                         const double* __restrict__ v, const double* __restrict__ invd, double* __restrict__ y) {
    if (sc->done) return;
    const double beta = sc->beta, w = sc->w;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double pi = r[i] + beta * (p[i] - w * v[i]);
        p[i] = pi;
        y[i] = invd[i] * pi;
    }
}

// alpha = rho / (r0 . v); s = r - alpha v; z = invd .* s
__global__ void k_bicg_s(int n, int nrb, DevScalars* sc, const double* __restrict__ red_r0v,
                         const double* __restrict__ r, const double* __restrict__ v, const double* __restrict__ invd,
                         double* __restrict__ s, double* __restrict__ z) {
    if (sc->done) return;
    double r0v = block_reduce_partials(red_r0v, nrb);
    const double alpha = sc->rho / r0v;
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->alpha = alpha;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double si = r[i] - alpha * v[i];
        s[i] = si;
        z[i] = invd[i] * si;
    }
}

// w = (t.s)/(t.t); x += alpha y + w z; r = s - w t; partials r.r and r0.r; iteration count
__global__ void k_bicg_xr(int n, int nrb, DevScalars* sc, const double* __restrict__ red_tt,
                          const double* __restrict__ red_ts, const double* __restrict__ y,
                          const double* __restrict__ z, const double* __restrict__ s, const double* __restrict__ t,
                          const double* __restrict__ r0, double* __restrict__ x, double* __restrict__ r,
                          double* __restrict__ red) {
    if (sc->done) return;
    double tt = block_reduce_partials(red_tt, nrb);
    double ts = block_reduce_partials(red_ts, nrb);
    const double w = (tt > 0.0) ? ts / tt : 0.0;
    const double alpha = sc->alpha;
    double a = 0.0, b = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] += alpha * y[i] + w * z[i];
        double ri = s[i] - w * t[i];
        r[i] = ri;
        a += ri * ri;
        b += r0[i] * ri;
    }
    a = block_sum(a);
    b = block_sum(b);
    if (threadIdx.x == 0) {
        red[RS_RR * VBLK + blockIdx.x] = a;
        red[RS_R0R * VBLK + blockIdx.x] = b;
    }
    __syncthreads();
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc->w = w;
        sc->iters += 1;
    }
}

int bicgstab(Ctx& c, const double* A, const double* b, double* x, cudaStream_t s) {
    // one cooperative kernel per batch of iterations (bicg.cu); these launches are the fallback
    if (!c.batch && c.pbicg_ok && !(c.prm.flags & BEM_FLAG_BICGSTAB_MULTIKERNEL)) {
        const int rc = bicgstab_persistent(c, A, b, x, s);
        if (rc == BEM_OK || rc == BEM_ERR_NOT_CONVERGED) return rc;
        c.pbicg_ok = false;
    }
    const int n = (int)c.topo.N;
    const int nrb = (n + GV_ROWS - 1) / GV_ROWS;
    double* red = c.red;
    // GEMV dot partial slots (one per row block) after the VBLK-sized vector slots
    double* g_r0v = red + RS_N * VBLK;
    double* g_tt = g_r0v + nrb;
    double* g_ts = g_tt + nrb;
    const int maxit = c.prm.max_iters > 0 ? c.prm.max_iters : 2 * n;
    KLAUNCH(), k_bicg_init<<<VBLK, VTHR, 0, s>>>(n, A, b, x, c.r, c.r0, c.pv, c.vv, c.invd, red);
    KLAUNCH(), k_bicg_init_scalars<<<1, 32, 0, s>>>(c.sc, red, maxit);
    int* done_dev = &c.sc->done;
    int* rflag_dev = &c.sc->restart_flag;
    const int batch = 4;
    for (int it0 = 0;; it0 += batch) {
        for (int k = 0; k < batch; ++k) {
            KLAUNCH(), k_bicg_begin<<<1, 32, 0, s>>>(c.sc, red);
            // restart path (inactive unless the flag is set)
            gemv_t<double>(n, A, x, c.tv, s, c.part, c.cnt, rflag_dev, 1);
            KLAUNCH(), k_bicg_restart_update<<<VBLK, VTHR, 0, s>>>(n, c.sc, b, c.tv, c.r, c.r0, red);
            KLAUNCH(), k_bicg_restart_scalars<<<1, 32, 0, s>>>(c.sc, red);
            KLAUNCH(), k_bicg_p<<<VBLK, VTHR, 0, s>>>(n, c.sc, c.r, c.pv, c.vv, c.invd, c.yv);
            gemv_t<double>(n, A, c.yv, c.vv, s, c.part, c.cnt, done_dev, 0, c.r0, g_r0v);
            KLAUNCH(), k_bicg_s<<<VBLK, VTHR, 0, s>>>(n, nrb, c.sc, g_r0v, c.r, c.vv, c.invd, c.sv, c.zv);
            gemv_t<double>(n, A, c.zv, c.tv, s, c.part, c.cnt, done_dev, 0, c.tv, g_tt, c.sv, g_ts);
            KLAUNCH(), k_bicg_xr<<<VBLK, VTHR, 0, s>>>(n, nrb, c.sc, g_tt, g_ts, c.yv, c.zv, c.sv, c.tv, c.r0, x, c.r, red);
        }
        BEM_CUDA(c, cudaMemcpyAsync(c.h_sc, c.sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, s));
        BEM_CUDA(c, cudaStreamSynchronize(s));
        if (c.h_sc->done) break;
        if (it0 > 4 * maxit + 64) return c.fail(BEM_ERR_NOT_CONVERGED, "BiCGSTAB: loop guard");
    }
    c.stats.last_iters = c.h_sc->iters;
    c.stats.last_rel_residual = c.h_sc->rhs_sq > 0 ? sqrt(c.h_sc->rr / c.h_sc->rhs_sq) : 0.0;
    c.stats.total_iters += c.stats.last_iters;
    c.stats.solves++;
    return BEM_OK;
}


// ------------------------------------------------------------------------------------------------
// LU with row partial pivoting (FP64), right-looking, panel width LU_NB
// ------------------------------------------------------------------------------------------------
constexpr int LU_NB = 64;

// Panel factorisation of columns [k0, k0+nb), rows [k0, n), one CTA: pivot search (largest
// |entry|, first row on ties), row swap inside the panel, column scaling, rank-1 panel update.
__global__ void __launch_bounds__(1024) k_lu_panel(int n, int k0, int nb, double* __restrict__ A,
                                                   int* __restrict__ piv, int* __restrict__ sing) {
    __shared__ double s_v[32];
    __shared__ int s_i[32];
    __shared__ int s_p;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int j = k0; j < k0 + nb; ++j) {
        double best = -1.0;
        int bi = n;
        for (int i = j + tid; i < n; i += blockDim.x) {
            double v = fabs(A[(size_t)j * n + i]);
            if (v > best) {
                best = v;
                bi = i;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_xor_sync(0xffffffffu, best, o);
            int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) {
                best = ov;
                bi = oi;
            }
        }
        if (lane == 0) {
            s_v[wid] = best;
            s_i[wid] = bi;
        }
        __syncthreads();
        if (wid == 0) {
            best = (lane < (int)(blockDim.x >> 5)) ? s_v[lane] : -2.0;
            bi = (lane < (int)(blockDim.x >> 5)) ? s_i[lane] : n;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                double ov = __shfl_xor_sync(0xffffffffu, best, o);
                int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ov > best || (ov == best && oi < bi)) {
                    best = ov;
                    bi = oi;
                }
            }
            if (lane == 0) s_p = (bi < n) ? bi : j;
        }
        __syncthreads();
        const int p = s_p;
        if (tid == 0) piv[j] = p;
        if (p != j)
            for (int c = k0 + tid; c < k0 + nb; c += blockDim.x) {
                double t = A[(size_t)c * n + j];
                A[(size_t)c * n + j] = A[(size_t)c * n + p];
                A[(size_t)c * n + p] = t;
            }
        __syncthreads();
        const double d = A[(size_t)j * n + j];
        if (d != 0.0) {
            for (int i = j + 1 + tid; i < n; i += blockDim.x) A[(size_t)j * n + i] /= d;
        } else if (tid == 0) {
            *sing = 1;
        }
        __syncthreads();
        const int ncols = k0 + nb - j - 1, nrows = n - j - 1;
        for (int e = tid; e < ncols * nrows; e += blockDim.x) {
            int cc = e / nrows, rr = e - cc * nrows;
            int c = j + 1 + cc, i = j + 1 + rr;
            A[(size_t)c * n + i] -= A[(size_t)j * n + i] * A[(size_t)c * n + j];
        }
        __syncthreads();
    }
}

// Apply the panel's row interchanges to every column outside the panel.
__global__ void k_lu_laswp(int n, int k0, int nb, double* __restrict__ A, const int* __restrict__ piv) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n || (c >= k0 && c < k0 + nb)) return;
    double* col = A + (size_t)c * n;
    for (int j = k0; j < k0 + nb; ++j) {
        int p = piv[j];
        if (p != j) {
            double t = col[j];
            col[j] = col[p];
            col[p] = t;
        }
    }
}

// U12 = L11^-1 A12: one warp per column right of the panel, two panel rows per lane.
__global__ void __launch_bounds__(256) k_lu_trsm(int n, int k0, int nb, double* __restrict__ A) {
    __shared__ double L[LU_NB][LU_NB + 1];
    {
        // L11, all 16 loads of the thread in flight together
        double v[LU_NB * LU_NB / 256];
#pragma unroll
        for (int u = 0; u < LU_NB * LU_NB / 256; ++u) {
            const int e = threadIdx.x + 256 * u, r = e % LU_NB, c = e / LU_NB;
            v[u] = (r < nb && c < nb) ? A[(size_t)(k0 + c) * n + k0 + r] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < LU_NB * LU_NB / 256; ++u) {
            const int e = threadIdx.x + 256 * u;
            L[e % LU_NB][e / LU_NB] = v[u];
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    // each warp takes columns right of the panel, strided over the grid
    for (int col = k0 + nb + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); col < n;
         col += gridDim.x * (blockDim.x >> 5)) {
        double* a = A + (size_t)col * n + k0;
        double v0 = (lane < nb) ? a[lane] : 0.0, v1 = (lane + 32 < nb) ? a[lane + 32] : 0.0;
        for (int k = 0; k < nb; ++k) {
            double xk = (k < 32) ? __shfl_sync(0xffffffffu, v0, k) : __shfl_sync(0xffffffffu, v1, k - 32);
            if (lane > k && lane < nb) v0 -= L[lane][k] * xk;
            if (lane + 32 > k && lane + 32 < nb) v1 -= L[lane + 32][k] * xk;
        }
        if (lane < nb) a[lane] = v0;
        if (lane + 32 < nb) a[lane + 32] = v1;
    }
}

// Triangular solves of the factored system (x = P b, L y = x with unit L, U x = y) in blocks of TS_B
// columns, with the operations of the column-oriented substitution in the same order per element:
// each row subtracts the contributions of the columns in increasing order going forward and in
// decreasing order going back.  One launch per block: every CTA loads the block's diagonal part into
// shared memory and solves it with one warp (two rows per lane, the solved entry broadcast by a
// shuffle), CTA 0 writes the block's solution, and every CTA subtracts the block's columns from its
// rows outside the block.  The block's right-hand side is read, never written, in its own launch.
// Going back, each entry is multiplied by the reciprocal of its diagonal entry (formed before the
// sweep) instead of divided by it.
constexpr int TS_B = 64;
constexpr int TS_LD = TS_B + 1;

// y = P b: the recorded interchanges in order (one CTA, the vector in shared memory); the fallback
// when the factorisation kept no composed row permutation
__global__ void __launch_bounds__(1024) k_lu_permute(int n, const int* __restrict__ piv, const double* __restrict__ b,
                                                     double* __restrict__ y) {
    extern __shared__ double sy[];
    for (int i = threadIdx.x; i < n; i += blockDim.x) sy[i] = b[i];
    __syncthreads();
    if (threadIdx.x == 0)
        for (int j = 0; j < n; ++j) {
            const int p = piv[j];
            if (p != j) {
                const double t = sy[j];
                sy[j] = sy[p];
                sy[p] = t;
            }
        }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = sy[i];
}

// y = P b with the composed row permutation (row i of P A is row perm[i] of A)
__global__ void k_lu_gather(int n, const int* __restrict__ perm, const double* __restrict__ b, double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = b[perm[i]];
}

// forward: unit lower L on rows [k0, k0 + kb); y the running right-hand side (rows >= k0 + kb are
// updated), z the solution
__global__ void __launch_bounds__(256) k_trsv_fwd(int n, int k0, int kb, const double* __restrict__ A,
                                                  double* __restrict__ y, double* __restrict__ z) {
    __shared__ double sL[TS_B * TS_LD];  // [c][r]
    __shared__ double sx[TS_B];
    const int tid = threadIdx.x, k1 = k0 + kb;
    {
        // the diagonal block, all 16 loads of the thread in flight together
        double v[TS_B * TS_B / 256];
#pragma unroll
        for (int u = 0; u < TS_B * TS_B / 256; ++u) {
            const int e = tid + 256 * u, c = e / TS_B, r = e - c * TS_B;
            v[u] = (c < kb && r < kb) ? A[(size_t)(k0 + c) * n + k0 + r] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < TS_B * TS_B / 256; ++u) {
            const int e = tid + 256 * u, c = e / TS_B;
            sL[c * TS_LD + (e - c * TS_B)] = v[u];
        }
    }
    __syncthreads();
    if (tid < 32) {
        const int lane = tid;
        double v0 = lane < kb ? y[k0 + lane] : 0.0, v1 = lane + 32 < kb ? y[k0 + 32 + lane] : 0.0;
        for (int j = 0; j < kb; ++j) {
            const double xj = __shfl_sync(0xffffffffu, j < 32 ? v0 : v1, j & 31);
            if (lane > j && lane < kb) v0 -= sL[j * TS_LD + lane] * xj;
            if (lane + 32 > j && lane + 32 < kb) v1 -= sL[j * TS_LD + lane + 32] * xj;
        }
        if (lane < kb) sx[lane] = v0;
        if (lane + 32 < kb) sx[lane + 32] = v1;
    }
    __syncthreads();
    if (blockIdx.x == 0 && tid < kb) z[k0 + tid] = sx[tid];
    const int i = k1 + blockIdx.x * 256 + tid;
    if (i >= n) return;
    double acc = y[i];
    for (int j0 = 0; j0 < kb; j0 += 16) {  // 16 loads in flight, the subtractions in column order
        double lv[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) lv[u] = j0 + u < kb ? A[(size_t)(k0 + j0 + u) * n + i] : 0.0;
#pragma unroll
        for (int u = 0; u < 16; ++u)
            if (j0 + u < kb) acc -= lv[u] * sx[j0 + u];
    }
    y[i] = acc;
}

// backward: upper U on rows [k0, k0 + kb), columns from the last; y the running right-hand side
// (rows < k0 are updated), x the solution
__global__ void __launch_bounds__(256) k_trsv_bwd(int n, int k0, int kb, const double* __restrict__ A,
                                                  double* __restrict__ y, double* __restrict__ x) {
    __shared__ double sU[TS_B * TS_LD];  // [c][r]
    __shared__ double sx[TS_B];
    const int tid = threadIdx.x;
    {
        // the diagonal block, all 16 loads of the thread in flight together
        double v[TS_B * TS_B / 256];
#pragma unroll
        for (int u = 0; u < TS_B * TS_B / 256; ++u) {
            const int e = tid + 256 * u, c = e / TS_B, r = e - c * TS_B;
            v[u] = (c < kb && r < kb) ? A[(size_t)(k0 + c) * n + k0 + r] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < TS_B * TS_B / 256; ++u) {
            const int e = tid + 256 * u, c = e / TS_B;
            sU[c * TS_LD + (e - c * TS_B)] = v[u];
        }
    }
    __syncthreads();
    if (tid < 32) {
        const int lane = tid;
        double v0 = lane < kb ? y[k0 + lane] : 0.0, v1 = lane + 32 < kb ? y[k0 + 32 + lane] : 0.0;
        // reciprocals of the lane's two diagonal entries, formed before the sweep: a division per
        // step would sit on the sweep's critical path
        const double q0 = lane < kb ? 1.0 / sU[lane * TS_LD + lane] : 0.0;
        const double q1 = lane + 32 < kb ? 1.0 / sU[(lane + 32) * TS_LD + lane + 32] : 0.0;
        for (int j = kb - 1; j >= 0; --j) {
            if (lane == j) v0 *= q0;
            if (lane + 32 == j) v1 *= q1;
            const double xj = __shfl_sync(0xffffffffu, j < 32 ? v0 : v1, j & 31);
            if (lane < j) v0 -= sU[j * TS_LD + lane] * xj;
            if (lane + 32 < j) v1 -= sU[j * TS_LD + lane + 32] * xj;
        }
        if (lane < kb) sx[lane] = v0;
        if (lane + 32 < kb) sx[lane + 32] = v1;
    }
    __syncthreads();
    if (blockIdx.x == 0 && tid < kb) x[k0 + tid] = sx[tid];
    const int i = blockIdx.x * 256 + tid;
    if (i >= k0) return;
    double acc = y[i];
    for (int j1 = kb - 1; j1 >= 0; j1 -= 16) {  // 16 loads in flight, the subtractions from the last column
        double lv[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) lv[u] = j1 - u >= 0 ? A[(size_t)(k0 + j1 - u) * n + i] : 0.0;
#pragma unroll
        for (int u = 0; u < 16; ++u)
            if (j1 - u >= 0) acc -= lv[u] * sx[j1 - u];
    }
    y[i] = acc;
}

// x = U^-1 L^-1 P b with c.LU, c.piv (and c.lu_perm when the factorisation composed it); c.yv and
// c.zv are the work vectors
static void lu_substitute_blocked(Ctx& c, const double* b, double* x, cudaStream_t s, bool composed) {
    const int n = (int)c.topo.N;
    double* y = c.yv;
    double* z = c.zv;
    if (composed) {
        KLAUNCH(), k_lu_gather<<<(n + 255) / 256, 256, 0, s>>>(n, c.lu_perm, b, y);
    } else {
        static std::atomic<uint64_t> attr{0};
        once_per_device(attr, [] {
            return cudaFuncSetAttribute(k_lu_permute, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) ==
                   cudaSuccess;
        });
        KLAUNCH(), k_lu_permute<<<1, 1024, sizeof(double) * (size_t)n, s>>>(n, c.piv, b, y);
    }
    for (int k0 = 0; k0 < n; k0 += TS_B) {
        const int kb = std::min(TS_B, n - k0);
        const int rows = n - k0 - kb;
        KLAUNCH(), k_trsv_fwd<<<std::max(1, (rows + 255) / 256), 256, 0, s>>>(n, k0, kb, c.LU, y, z);
    }
    // z is now L^-1 P b; the backward sweep runs on it in place of y
    for (int k1 = n; k1 > 0; k1 -= TS_B) {
        const int k0 = std::max(0, k1 - TS_B);
        KLAUNCH(), k_trsv_bwd<<<std::max(1, (k0 + 255) / 256), 256, 0, s>>>(n, k0, k1 - k0, c.LU, z, x);
    }
}

// Blocked right-looking factorisation of c.LU (a copy of A).  rows: each panel on one thread-block
// cluster when its rows fit in the cluster's shared memory, else spread over the SMs with grid
// barriers (lu_panel.cu); the interchanges are composed per panel and applied to the other columns
// and to the row permutation c.lu_perm (*composed = true).  Otherwise the single-CTA panel and one
// interchange at a time.  The trailing update runs on the FP64 tensor cores (lu_update.cu).
static int lu_factor(Ctx& c, const double* A, cudaStream_t s, bool rows, bool* composed) {
    const int n = (int)c.topo.N;
    *composed = false;
    BEM_CUDA(c, cudaMemcpyAsync(c.LU, A, sizeof(double) * (size_t)n * n, cudaMemcpyDeviceToDevice, s));
    BEM_CUDA(c, cudaMemsetAsync(c.flag, 0, sizeof(int), s));
    // Look-ahead (row-distributed panels only): after panel k's interchanges and U12, the trailing
    // update first takes the next panel's columns; that panel is then factored on a high-priority side
    // stream while the rest of the update runs (in 64-row tiles, so that a panel CTA fits beside an
    // update CTA on an SM).  The side stream joins the main one before the next interchanges.
    cudaStream_t s2 = nullptr;
    if (rows) {
        BEM_CUDA(c, cudaMemsetAsync(lu_panel_err(c), 0, sizeof(int), s));
        lu_perm_init(c, s);
        if (!c.lu_side) {
            int lo = 0, hi = 0;
            BEM_CUDA(c, cudaDeviceGetStreamPriorityRange(&lo, &hi));
            BEM_CUDA(c, cudaStreamCreateWithPriority(&c.lu_side, cudaStreamNonBlocking, hi));
            for (cudaEvent_t& e : c.lu_ev) BEM_CUDA(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        }
        s2 = c.lu_side;
    }
    bool ahead = false, ahead_built = false;  // the current panel was factored by the look-ahead
    for (int k0 = 0; k0 < n; k0 += LU_NB) {
        const int nb = std::min(LU_NB, n - k0);
        bool built = false;
        if (rows) {
            if (ahead)
                built = ahead_built;
            else if (lu_panel_cluster(c, k0, nb, s) == BEM_OK)
                built = true;
            else if (lu_panel_rows(c, k0, nb, s) != BEM_OK)
                return BEM_ERR_CUDA;
            lu_panel_swap_rest(c, k0, nb, s, built);
        } else {
            KLAUNCH(), k_lu_panel<<<1, 1024, 0, s>>>(n, k0, nb, c.LU, c.piv, c.flag);
            KLAUNCH(), k_lu_laswp<<<(n + 255) / 256, 256, 0, s>>>(n, k0, nb, c.LU, c.piv);
        }
        ahead = false;
        const int rest = n - k0 - nb;
        if (rest <= 0) continue;
        KLAUNCH(), k_lu_trsm<<<std::min((rest + 7) / 8, 2 * 148), 256, 0, s>>>(n, k0, nb, c.LU);
        int rc;
        if (!rows) {
            if ((rc = lu_update(c, n, k0, nb, c.LU, s))) return rc;
            continue;
        }
        const int k1 = k0 + nb, nb2 = std::min(LU_NB, n - k1);
        if ((rc = lu_update(c, n, k0, nb, c.LU, s, k1, k1 + nb2))) return rc;  // the next panel's columns
        BEM_CUDA(c, cudaEventRecord(c.lu_ev[0], s));
        BEM_CUDA(c, cudaStreamWaitEvent(s2, c.lu_ev[0], 0));
        if (lu_panel_cluster(c, k1, nb2, s2) == BEM_OK)
            ahead_built = true;
        else if (lu_panel_rows(c, k1, nb2, s2) == BEM_OK)
            ahead_built = false;
        else
            return BEM_ERR_CUDA;  // nothing was enqueued on the side stream after the wait
        BEM_CUDA(c, cudaEventRecord(c.lu_ev[1], s2));
        rc = lu_update(c, n, k0, nb, c.LU, s, k1 + nb2, n, true);  // the rest, beside the next panel
        BEM_CUDA(c, cudaStreamWaitEvent(s, c.lu_ev[1], 0));
        if (rc) return rc;
        ahead = true;
    }
    if (rows) {
        int err = 0;
        BEM_CUDA(c, cudaMemcpyAsync(&err, lu_panel_err(c), sizeof(int), cudaMemcpyDeviceToHost, s));
        BEM_CUDA(c, cudaStreamSynchronize(s));
        if (err) {
            c.stats.wait_expired++;
            return BEM_ERR_CUDA;
        }
        *composed = true;
    }
    return BEM_OK;
}

int lu_solve(Ctx& c, const double* A, const double* b, double* x, cudaStream_t s) {
    const int n = (int)c.topo.N;
    int rc = BEM_ERR_CUDA;
    bool composed = false;
    if (c.lu_rows_ok && c.lu_aux) {
        rc = lu_factor(c, A, s, true, &composed);
        if (rc == BEM_ERR_CUDA) c.lu_rows_ok = false;  // factor again with the single-CTA panel
    }
    if (rc != BEM_OK) {
        if ((size_t)n * sizeof(double) > 200 * 1024)
            return c.fail(BEM_ERR_ARG,
                          "LU solver: N too large for the in-shared-memory interchange of b (N <= 25600)");
        rc = lu_factor(c, A, s, false, &composed);
        if (rc) return rc;
    }
    lu_substitute_blocked(c, b, x, s, composed);
    int sing = 0;
    BEM_CUDA(c, cudaMemcpyAsync(&sing, c.flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    BEM_CUDA(c, cudaStreamSynchronize(s));
    c.stats.solves++;
    c.stats.last_iters = 0;
    if (sing) return c.fail(BEM_ERR_SINGULAR, "LU: zero pivot (singular G)");
    return BEM_OK;
}

// ------------------------------------------------------------------------------------------------
// MIXED: FP64 GMRES right-preconditioned by an FP32 approximate inverse X, Newton-Schulz refresh
// ------------------------------------------------------------------------------------------------

__global__ void k_to_f32(int64_t nn, const double* __restrict__ a, float* __restrict__ b) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

// |G| column sums (norm-1 candidates) and row sums (norm-inf candidates)
__global__ void k_abs_colsum(int n, const double* __restrict__ A, double* __restrict__ cs) {
    int j = blockIdx.x;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += fabs(A[(size_t)j * n + i]);
    s = block_sum(s);
    if (threadIdx.x == 0) cs[j] = s;
}
__global__ void k_abs_rowsum(int n, const double* __restrict__ A, double* __restrict__ rs) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int j = 0; j < n; ++j) s += fabs(A[(size_t)j * n + i]);
    rs[i] = s;
}
__global__ void k_max_two(int n, const double* __restrict__ a, const double* __restrict__ b, double* out) {
    __shared__ double sa[1024], sb[1024];
    double ma = 0.0, mb = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        ma = fmax(ma, a[i]);
        mb = fmax(mb, b[i]);
    }
    sa[threadIdx.x] = ma;
    sb[threadIdx.x] = mb;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            sa[threadIdx.x] = fmax(sa[threadIdx.x], sa[threadIdx.x + w]);
            sb[threadIdx.x] = fmax(sb[threadIdx.x], sb[threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = 1.0 / (sa[0] * sb[0]);
}
// X0 = alpha * G^T (FP32), the classical Newton-Schulz start (Ben-Israel & Cohen 1966)
__global__ void k_scaled_transpose(int n, const double* __restrict__ A, const double* __restrict__ alpha,
                                   float* __restrict__ X) {
    __shared__ double tile[32][33];
    int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        int i = bx + threadIdx.x, j = by + k;
        tile[k][threadIdx.x] = (i < n && j < n) ? A[(size_t)j * n + i] : 0.0;
    }
    __syncthreads();
    const double a = *alpha;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        int i = by + threadIdx.x, j = bx + k;  // X(i,j) = G(j,i)
        if (i < n && j < n) X[(size_t)j * n + i] = (float)(a * tile[threadIdx.x][k]);
    }
}

// Xn = 2 X - P ; and partial ||I - T||_F^2 of the T = G X just used
__global__ void k_ns_combine(int64_t nn, const float* __restrict__ X, const float* __restrict__ P,
                             float* __restrict__ Xn) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x)
        Xn[i] = 2.f * X[i] - P[i];
}
__global__ void k_eye_resid(int n, const float* __restrict__ T, double* __restrict__ part) {
    double s = 0.0;
    const int64_t nn = (int64_t)n * n;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += (int64_t)gridDim.x * blockDim.x) {
        int64_t j = e / n, i = e - j * n;
        double d = (i == j ? 1.0 : 0.0) - (double)T[e];
        s += d * d;
    }
    s = block_sum(s);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}
__global__ void k_sum_partials(const double* __restrict__ p, int np, double* out) {
    double v = block_reduce_partials(p, np);
    if (threadIdx.x == 0) *out = v;
}

// One Newton-Schulz step X <- X (2I - G X) on job j; returns ||I - G X_old||_F / sqrt(n) (host
// value).  terms: precision of the two products (3 = BF16x3, 1 = bf16).
int ns_step(Ctx& c, const NSJob& j, cudaStream_t s, double* eres, int terms) {
    const int n = j.n;
    const int64_t nn = (int64_t)n * n;
    int rc = tc_gemm(c, n, j.G32, j.X, j.T, c.tcp, c.tc_err, s, terms);  // T = G X
    if (rc) return rc;
    KLAUNCH(), k_eye_resid<<<VBLK, VTHR, 0, s>>>(n, j.T, c.red);
    KLAUNCH(), k_sum_partials<<<1, 32, 0, s>>>(c.red, VBLK, c.red + VBLK);
    if ((rc = tc_gemm(c, n, j.X, j.T, j.P, c.tcp, c.tc_err, s, terms))) return rc;  // P = X T
    KLAUNCH(), k_ns_combine<<<4 * 148, 256, 0, s>>>(nn, j.X, j.P, j.X);
    double v = 0.0;
    int herr = 0;
    BEM_CUDA(c, cudaMemcpyAsync(&v, c.red + VBLK, sizeof(double), cudaMemcpyDeviceToHost, s));
    BEM_CUDA(c, cudaMemcpyAsync(&herr, c.tc_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    BEM_CUDA(c, cudaStreamSynchronize(s));
    if (herr) return c.fail(BEM_ERR_CUDA, "tensor-core GEMM: bounded wait expired (code " + std::to_string(herr) + ")");
    c.stats.ns_steps++;
    *eres = sqrt(v / n);
    return BEM_OK;
}

__global__ void k_fill(int n, double v, double* __restrict__ x) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = v;
}
// x = y / ||y|| from the per-row-block partials of y.y (every block sums them in the same order);
// lam = ||y||.
__global__ void k_scale_by_norm(int n, const double* __restrict__ part, int np, const double* __restrict__ y,
                                double* __restrict__ x, double* __restrict__ lam) {
    const double nrm = sqrt(block_reduce_partials(part, np));
    const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = y[i] * inv;
    if (blockIdx.x == 0 && threadIdx.x == 0) *lam = nrm;
}
// X = theta I (FP32)
__global__ void k_scaled_identity(int n, double theta, float* __restrict__ X) {
    const int64_t nn = (int64_t)n * n;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = e / n, i = e - j * n;
        X[e] = (i == j) ? (float)theta : 0.f;
    }
}

// Largest eigenvalue magnitude of A (n x n) by power iteration in FP64 (a handful of GEMVs).  The
// collocation single-layer matrix has a dominant constant mode separated from the next by a factor
// of about three, so a dozen iterations from the constant vector resolve it.
static int power_lambda(Ctx& c, int n, const double* A, cudaStream_t s, double* lam) {
    const int nrb = (n + GV_ROWS - 1) / GV_ROWS;
    double* y = c.r0;
    double* x = c.tv;
    double* dl = c.red + nrb;
    KLAUNCH(), k_fill<<<VBLK, VTHR, 0, s>>>(n, 1.0 / sqrt((double)n), x);
    for (int it = 0; it < 12; ++it) {
        gemv_t<double>(n, A, x, y, s, c.part, c.cnt, nullptr, 0, y, c.red);
        KLAUNCH(), k_scale_by_norm<<<VBLK, VTHR, 0, s>>>(n, c.red, nrb, y, x, dl);
    }
    BEM_CUDA(c, cudaMemcpyAsync(lam, dl, sizeof(double), cudaMemcpyDeviceToHost, s));
    BEM_CUDA(c, cudaStreamSynchronize(s));
    return BEM_OK;
}

// Approximate inverse X ~ G^-1 in FP32 by Newton-Schulz (Schulz 1933; E_{k+1} = E_k^2 with
// E = I - G X).  From scratch the start is X0 = I / lambda_max(G): the eigenvalues of the
// collocation single-layer matrix are positive (it discretises a positive operator), so E0 has
// spectral radius 1 - lambda_min/lambda_max and about log2(cond) steps suffice -- half of what the
// classical X0 = G^T / (||G||_1 ||G||_inf) needs (cond^2).  Steps whose residual is still above
// 0.25 run the GEMMs in plain bf16; the rest in BF16x3.  Should the scaled-identity start fail to
// contract (a matrix with eigenvalues off the positive axis), the classical start takes over.
// Expects j.G32 = fp32(j.A).
int ns_from_scratch(Ctx& c, const NSJob& j, cudaStream_t s, bool classical) {
    const int n = j.n;
    int terms = 3;
    if (!classical) {
        double lam = 0.0;
        int rc = power_lambda(c, n, j.A, s, &lam);
        if (rc) return rc;
        if (!(lam > 0.0) || !std::isfinite(lam)) return ns_from_scratch(c, j, s, true);
        KLAUNCH(), k_scaled_identity<<<4 * 148, 256, 0, s>>>(n, 1.0 / lam, j.X);
        terms = 1;
    } else {
        double* cs = c.red + 2 * VBLK;
        KLAUNCH(), k_abs_colsum<<<n, 256, 0, s>>>(n, j.A, c.r);
        KLAUNCH(), k_abs_rowsum<<<(n + 255) / 256, 256, 0, s>>>(n, j.A, c.r0);
        KLAUNCH(), k_max_two<<<1, 1024, 0, s>>>(n, c.r, c.r0, cs);
        dim3 tg((n + 31) / 32, (n + 31) / 32), tb(32, 8);
        KLAUNCH(), k_scaled_transpose<<<tg, tb, 0, s>>>(n, j.A, cs, j.X);
    }
    double emin = 1e300;
    for (int it = 0; it < 80; ++it) {
        double e = 1.0;
        int rc = ns_step(c, j, s, &e, terms);
        if (rc) return rc;
        if (terms == 3 && e < 1e-4) return BEM_OK;
        if (!std::isfinite(e) || (it >= 4 && e > 2.0 * emin)) break;  // not contracting
        emin = std::min(emin, e);
        if (terms == 1 && e < 0.25) terms = 3;
    }
    if (!classical) return ns_from_scratch(c, j, s, true);
    return c.fail(BEM_ERR_NOT_CONVERGED, "Newton-Schulz inverse did not converge");
}

void to_f32(int64_t nn, const double* a, float* b, cudaStream_t s) {
    KLAUNCH(), k_to_f32<<<4 * 148, 256, 0, s>>>(nn, a, b);
}

// v[i] in [-1, 1), a fixed hash of i
__global__ void k_fill_hash(int n, double* __restrict__ v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        unsigned h = (unsigned)i * 2654435761u + 0x9e3779b9u;
        h ^= h >> 16;
        h *= 0x85ebca6bu;
        h ^= h >> 13;
        v[i] = (double)(h >> 8) * (2.0 / 16777216.0) - 1.0;
    }
}

__global__ void k_rowblock_norm2(int n, const double* __restrict__ b, double* __restrict__ part);

// ||(I - G X) v|| / ||v|| for a fixed pseudo-random v (two GEMVs): an estimate of how much one
// refinement step with X contracts the error.
static int inverse_resid_estimate(Ctx& c, const NSJob& j, cudaStream_t s, double* est) {
    const int n = j.n, nrb = (n + GV_ROWS - 1) / GV_ROWS;
    double *v = c.r0, *w = c.tv, *r = c.yv;
    KLAUNCH(), k_fill_hash<<<VBLK, VTHR, 0, s>>>(n, v);
    gemv_t<float>(n, j.X, v, w, s, c.part, c.cnt);                                              // w = X v
    gemv_t<double>(n, j.A, w, r, s, c.part, c.cnt, nullptr, 0, r, c.red, nullptr, nullptr, v, -1.0);  // r = v - G w
    KLAUNCH(), k_rowblock_norm2<<<nrb, GV_ROWS, 0, s>>>(n, v, c.red + nrb);
    std::vector<double> h((size_t)2 * nrb);
    BEM_CUDA(c, cudaMemcpyAsync(h.data(), c.red, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s));
    BEM_CUDA(c, cudaStreamSynchronize(s));
    double rr = 0.0, vv = 0.0;
    for (int q = 0; q < nrb; ++q) {
        rr += h[(size_t)q];
        vv += h[(size_t)nrb + q];
    }
    *est = vv > 0.0 ? sqrt(rr / vv) : 1.0;
    return BEM_OK;
}

// X from scratch by the tensor-core Gauss-Jordan elimination.  When the estimate of ||(I - G X) v||
// is already below 1e-3 X is kept as it is; otherwise Newton-Schulz steps against G follow until
// ||I - G X|| is below 1e-2 before the last step (about 1e-4 after it, as the set-up by Newton-Schulz
// alone ends).
static int gj_polished(Ctx& c, const NSJob& j, cudaStream_t s) {
    int rc = gj_inverse(c, j, s);
    if (rc) return rc;
    double est = 1.0;
    if ((rc = inverse_resid_estimate(c, j, s, &est))) return rc;
    if (est < 1e-3) return BEM_OK;
    for (int it = 0; it < 8; ++it) {
        double e = 1.0;
        if ((rc = ns_step(c, j, s, &e, 3))) return rc;
        if (!(e < 0.9)) break;
        if (e < 1e-2) return BEM_OK;
    }
    return c.fail(BEM_ERR_NOT_CONVERGED, "Gauss-Jordan inverse: Newton-Schulz polish did not converge");
}

static bool use_gj(const Ctx& c, int n) {
    if (c.prm.flags & BEM_FLAG_INVERSE_NS) return false;
    if (c.prm.flags & BEM_FLAG_INVERSE_GJ) return true;
    return n >= BEM_GJ_MIN_N;
}

static int refresh_inverse(Ctx& c, const double* A, cudaStream_t s, bool from_scratch) {
    const int n = (int)c.topo.N;
    const int64_t nn = (int64_t)n * n;
    // LU buffer reused as FP32 scratch in the mixed path
    const NSJob j{n, A, c.G32, c.Xinv, c.Tw, reinterpret_cast<float*>(c.LU)};
    to_f32(nn, A, c.G32, s);
    if (from_scratch || !c.xinv_valid) {
        c.xinv_valid = false;
        int rc = BEM_ERR_CUDA;
        if (use_gj(c, n)) rc = gj_polished(c, j, s);
        if (rc != BEM_OK) rc = ns_from_scratch(c, j, s, false);  // the set-up without the elimination
        if (rc) return rc;
        c.xinv_valid = true;
    } else {
        double e = 0.0;
        int rc = ns_step(c, j, s, &e);
        if (rc) return rc;
        if (!(e < 0.9)) {  // diverging (stale X too far off): start over
            c.xinv_valid = false;
            return refresh_inverse(c, A, s, true);
        }
    }
    c.stats.precond_refresh++;
    return BEM_OK;
}

int mixed_refresh(Ctx& c, const double* A, cudaStream_t s, bool from_scratch) {
    return refresh_inverse(c, A, s, from_scratch);
}

// h[k] partials of V_k . w for k <= j (one partial per block per k)
__global__ void k_multidot(int n, int nv, const double* __restrict__ V, const double* __restrict__ w,
                           double* __restrict__ part) {
    for (int k = 0; k < nv; ++k) {
        double s = 0.0;
        const double* v = V + (size_t)k * n;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += v[i] * w[i];
        s = block_sum(s);
        if (threadIdx.x == 0) part[k * VBLK + blockIdx.x] = s;
    }
}
// h[k] (+)= sum of partials, one warp per k
__global__ void k_multidot_final(int nv, const double* __restrict__ part, double* __restrict__ h, int accumulate) {
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (k >= nv) return;
    double a = 0.0;
    for (int b = lane; b < VBLK; b += 32) a += part[k * VBLK + b];
    a = warp_sum(a);
    if (lane == 0) h[k] = accumulate ? h[k] + a : a;
}
// w -= sum_k V_k h[k]; partial ||w||^2 (slot nv*VBLK)
__global__ void k_orth_update(int n, int nv, const double* __restrict__ V, const double* __restrict__ h,
                              double* __restrict__ w, double* __restrict__ part) {
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double wi = w[i];
        for (int k = 0; k < nv; ++k) wi -= V[(size_t)k * n + i] * h[k];
        w[i] = wi;
        s += wi * wi;
    }
    s = block_sum(s);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}
// hn = sqrt(sum partials); V_next = w / hn; h[nv] = hn
__global__ void k_normalize(int n, const double* __restrict__ part, const double* __restrict__ w,
                            double* __restrict__ vnext, double* __restrict__ hslot) {
    double nrm2 = block_reduce_partials(part, VBLK);
    double hn = sqrt(nrm2);
    if (blockIdx.x == 0 && threadIdx.x == 0) *hslot = hn;
    double inv = (hn > 0.0) ? 1.0 / hn : 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) vnext[i] = w[i] * inv;
}
__global__ void k_scale(int n, const double* __restrict__ a, double f, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = a[i] * f;
}
// x += Z y
__global__ void k_combine(int n, int k, const double* __restrict__ Z, const double* __restrict__ y,
                          double* __restrict__ x) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = x[i];
        for (int q = 0; q < k; ++q) s += Z[(size_t)q * n + i] * y[q];
        x[i] = s;
    }
}
// r = b - t; partial ||r||^2 and ||b||^2
__global__ void k_resid(int n, const double* __restrict__ b, const double* __restrict__ t, double* __restrict__ r,
                        double* __restrict__ part) {
    double s = 0.0, bb = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double ri = b[i] - t[i];
        r[i] = ri;
        s += ri * ri;
        bb += b[i] * b[i];
    }
    s = block_sum(s);
    bb = block_sum(bb);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = s;
        part[VBLK + blockIdx.x] = bb;
    }
}
__global__ void k_resid_final(const double* __restrict__ part, double* out) {
    double a = block_reduce_partials(part, VBLK);
    double b = block_reduce_partials(part + VBLK, VBLK);
    if (threadIdx.x == 0) {
        out[0] = a;
        out[1] = b;
    }
}

static int gmres_solve(Ctx& c, const double* A, const double* b, double* x, cudaStream_t s) {
    const int n = (int)c.topo.N;
    const int m = c.gmres_m;
    const double tol = c.prm.mixed_tol > 0 ? c.prm.mixed_tol : 1e-12;
    if (!c.xinv_valid) {
        int rc = refresh_inverse(c, A, s, true);
        if (rc) return rc;
    }
    double* hp = c.red;                    // partial slots: up to (m+1)*VBLK
    double* hh = c.hcol;                   // device h column (m+2)
    std::vector<double> H((size_t)(m + 1) * m, 0.0), cs(m), sn(m), g(m + 1), hcol(m + 2);
    int total_it = 0;
    double relres = 1.0;
    for (int cycle = 0; cycle < 20; ++cycle) {
        // r = b - G x
        gemv_t<double>(n, A, x, c.tv, s, c.part, c.cnt);
        KLAUNCH(), k_resid<<<VBLK, VTHR, 0, s>>>(n, b, c.tv, c.r, hp);
        KLAUNCH(), k_resid_final<<<1, 32, 0, s>>>(hp, hh);
        double rb[2];
        BEM_CUDA(c, cudaMemcpyAsync(rb, hh, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
        BEM_CUDA(c, cudaStreamSynchronize(s));
        const double bnorm = sqrt(rb[1]);
        const double beta = sqrt(rb[0]);
        if (bnorm == 0.0) {
            relres = 0.0;
            break;
        }
        relres = beta / bnorm;
        if (relres <= tol) break;
        // V0 = r / beta
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int k = 0;
        KLAUNCH(), k_scale<<<VBLK, VTHR, 0, s>>>(n, c.r, 1.0 / beta, c.V);
        for (int j = 0; j < m; ++j) {
            double* vj = c.V + (size_t)j * n;
            double* zj = c.Z + (size_t)j * n;
            gemv_t<float>(n, c.Xinv, vj, zj, s, c.part, c.cnt);  // z = X v
            gemv_t<double>(n, A, zj, c.tv, s, c.part, c.cnt);    // w = G z
            KLAUNCH(), k_multidot<<<VBLK, VTHR, 0, s>>>(n, j + 1, c.V, c.tv, hp);
            KLAUNCH(), k_multidot_final<<<1, 32 * (j + 1), 0, s>>>(j + 1, hp, hh, 0);
            KLAUNCH(), k_orth_update<<<VBLK, VTHR, 0, s>>>(n, j + 1, c.V, hh, c.tv, hp + (size_t)(m + 1) * VBLK);
            // second Gram-Schmidt pass (CGS2)
            KLAUNCH(), k_multidot<<<VBLK, VTHR, 0, s>>>(n, j + 1, c.V, c.tv, hp);
            KLAUNCH(), k_multidot_final<<<1, 32 * (j + 1), 0, s>>>(j + 1, hp, hh + (m + 2), 0);
            KLAUNCH(), k_orth_update<<<VBLK, VTHR, 0, s>>>(n, j + 1, c.V, hh + (m + 2), c.tv, hp + (size_t)(m + 1) * VBLK);
            KLAUNCH(), k_normalize<<<VBLK, VTHR, 0, s>>>(n, hp + (size_t)(m + 1) * VBLK, c.tv, c.V + (size_t)(j + 1) * n,
                                              hh + j + 1);
            std::vector<double> h2(m + 2);
            BEM_CUDA(c, cudaMemcpyAsync(hcol.data(), hh, sizeof(double) * (j + 2), cudaMemcpyDeviceToHost, s));
            BEM_CUDA(c, cudaMemcpyAsync(h2.data(), hh + (m + 2), sizeof(double) * (j + 1), cudaMemcpyDeviceToHost, s));
            BEM_CUDA(c, cudaStreamSynchronize(s));
            for (int q = 0; q <= j; ++q) hcol[q] += h2[q];
            // Givens rotations on the new Hessenberg column
            for (int q = 0; q < j; ++q) {
                double t = cs[q] * hcol[q] + sn[q] * hcol[q + 1];
                hcol[q + 1] = -sn[q] * hcol[q] + cs[q] * hcol[q + 1];
                hcol[q] = t;
            }
            double den = hypot(hcol[j], hcol[j + 1]);
            cs[j] = (den > 0) ? hcol[j] / den : 1.0;
            sn[j] = (den > 0) ? hcol[j + 1] / den : 0.0;
            hcol[j] = den;
            hcol[j + 1] = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            for (int q = 0; q <= j; ++q) H[(size_t)q * m + j] = hcol[q];
            k = j + 1;
            ++total_it;
            if (fabs(g[j + 1]) / bnorm <= 0.5 * tol) break;
        }
        // y = R^-1 g
        std::vector<double> y(k);
        for (int q = k - 1; q >= 0; --q) {
            double acc = g[q];
            for (int r = q + 1; r < k; ++r) acc -= H[(size_t)q * m + r] * y[r];
            y[q] = acc / H[(size_t)q * m + q];
        }
        BEM_CUDA(c, cudaMemcpyAsync(hh, y.data(), sizeof(double) * k, cudaMemcpyHostToDevice, s));
        KLAUNCH(), k_combine<<<VBLK, VTHR, 0, s>>>(n, k, c.Z, hh, x);
    }
    c.stats.last_iters += total_it;
    c.stats.last_rel_residual = relres;
    if (relres > tol) return c.fail(BEM_ERR_NOT_CONVERGED, "mixed GMRES did not reach the tolerance");
    return BEM_OK;
}

// ||b||^2 partials with the GEMV's row-block shape (one partial per GV_ROWS rows)
__global__ void k_rowblock_norm2(int n, const double* __restrict__ b, double* __restrict__ part) {
    const int i = blockIdx.x * GV_ROWS + threadIdx.x;
    double v = (i < n) ? b[i] * b[i] : 0.0;
    v = block_sum(v);
    if (threadIdx.x == 0) part[blockIdx.x] = v;
}
// the same for two vectors in one launch (||b||^2 and the first residual's)
__global__ void k_rowblock_norm2x2(int n, const double* __restrict__ b, double* __restrict__ pb,
                                   const double* __restrict__ r, double* __restrict__ pr) {
    const int i = blockIdx.x * GV_ROWS + threadIdx.x;
    double v = (i < n) ? b[i] * b[i] : 0.0, w = (i < n) ? r[i] * r[i] : 0.0;
    v = block_sum(v);
    w = block_sum(w);
    if (threadIdx.x == 0) {
        pb[blockIdx.x] = v;
        pr[blockIdx.x] = w;
    }
}

// Mixed solve.  Iterative refinement x <- x + X (b - G x): the residual in FP64 against the FP64 G
// (so the limit is the FP64 solution), the correction through the FP32 approximate inverse X.
// Warm-started from the previous solution (the previous RK4 stage's psi); K steps are issued
// without host synchronisation, with the residual norms of every step kept on the device and read
// once.  A contraction too weak for refinement hands over to GMRES (same preconditioner, same
// start vector); a Newton-Schulz refresh of X follows the cost rule at the end.
// The FP64 BiCGSTAB (the reference's default solver) in place of the mixed solve, for a matrix the
// mixed path cannot handle: no approximate inverse converges (G singular or nearly so -- the
// reference's own BiCGSTAB then returns what it returns), or GMRES misses the tolerance.  After a
// failed inverse the next MIXED_BACKOFF solves go straight here instead of retrying the set-up.
constexpr int MIXED_BACKOFF = 16;
static int fp64_fallback(Ctx& c, const double* A, const double* b, double* x, cudaStream_t s, bool backoff) {
    c.stats.fp64_fallbacks++;
    c.stats.solves++;
    if (backoff) c.mixed_backoff = MIXED_BACKOFF;
    return bicgstab(c, A, b, x, s);
}

// One round of the refinement as one cooperative kernel (BEM_FLAG_REFINE_PERSISTENT; the separate
// launches below are the default, measured faster): for k < K, r = b - A x (its row-block norms
// into pr[k]; skipped for k = 0 when the assembly already left that residual) and x += X r, then the
// final r = b - A x (norms into pr[K]).  The GEMV tiles are k_gemv's (gemv_tile: the same split count,
// per-thread order and split sums), spread over co-resident CTAs and separated by grid barriers, so the
// result equals the multi-kernel round's bit for bit without its 2K+1 launches, their ramps and tails.
// A barrier wait that runs out sets *err and ends the kernel (grid_barrier); the host then repeats
// the round with separate launches.
// Ctx::rf_bar: the arrival count at word 0, the generation at RF_GEN and the error word at RF_ERR,
// each on its own 128-byte line (RF_WORDS ints)
constexpr int RF_GEN = 32, RF_ERR = 64, RF_GATE = 96;
static_assert(RF_GATE < RF_WORDS, "Ctx::rf_bar holds RF_WORDS ints");

// The host's convergence rule of the refinement on the device: with the row-block partials of |b|^2
// (pb) and of |r_k|^2 (prk) summed in the host's order, rel = sqrt(|r_k|^2 / |b|^2); the first k with
// rel <= tol is stored in *gate (which starts at -1), and the gated GEMVs that follow then return at
// once.  One thread: the same sums in the same order, so the device and the host decide alike.
__global__ void k_ir_check(int nrb, const double* __restrict__ pb, const double* __restrict__ prk, double tol,
                           int k, int* __restrict__ gate) {
    if (threadIdx.x != 0 || blockIdx.x != 0 || *gate >= 0) return;
    double bb = 0.0, a = 0.0;
    for (int q = 0; q < nrb; ++q) bb += pb[q];
    for (int q = 0; q < nrb; ++q) a += prk[q];
    if (bb != 0.0 && sqrt(a / bb) <= tol) *gate = k;
}
constexpr unsigned RF_SLEEP_NS = 32;  // polling interval of the waiting CTAs
constexpr int RF_CHUNK_MAX = 4096;    // columns of one tile's staged slice of the input vector
struct RFArgs {
    int n, chunk, ncs, K, skip_first;
    const double* A;
    const float* X;
    const double* b;
    double *x, *r, *part, *pr;
    unsigned* cnt;
    unsigned* bar;
    int* err;
    long long wait_limit;
};

__global__ void __launch_bounds__(GV_ROWS) k_refine_round(RFArgs a) {
    extern __shared__ double rf_x[];  // the current tile's slice of the input vector
    const int n = a.n, nrb = (n + GV_ROWS - 1) / GV_ROWS, ntiles = nrb * a.ncs;
    for (int k = 0; k <= a.K; ++k) {
        if (!(k == 0 && a.skip_first)) {
            for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
                gemv_tile<double, true>(n, a.chunk, a.ncs, t % nrb, t / nrb, a.A, a.x, a.r, a.part, a.cnt, a.r,
                                        a.pr + (size_t)k * nrb, nullptr, nullptr, a.b, -1.0, rf_x);
            if (k == a.K) break;
            if (!grid_barrier(a.bar, a.bar + RF_GEN, a.err, a.wait_limit, RF_SLEEP_NS)) return;
        }
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
            gemv_tile<float, true>(n, a.chunk, a.ncs, t % nrb, t / nrb, a.X, a.r, a.x, a.part, a.cnt, nullptr, nullptr,
                                   nullptr, nullptr, a.x, 1.0, rf_x);
        if (!grid_barrier(a.bar, a.bar + RF_GEN, a.err, a.wait_limit, RF_SLEEP_NS)) return;
    }
}

// Launches k_refine_round; BEM_ERR_CUDA when a cooperative launch of it is not possible (the caller
// uses separate launches).  Its barrier and error words are c.rf_bar (cleared with the mesh).
static int refine_round_persistent(Ctx& c, const double* A, const double* b, double* x, double* pr, int K,
                                   bool skip_first, cudaStream_t s) {
    const int n = (int)c.topo.N;
    if (!c.rf_bar) return BEM_ERR_CUDA;
    int sms = 0, coop = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c.device);
    const int ncs0 = gemv_splits(n);
    const size_t smem0 = sizeof(double) * (size_t)(((n + ncs0 - 1) / ncs0 + GV_UNR - 1) / GV_UNR * GV_UNR);
    if (!coop || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_refine_round, GV_ROWS, smem0) != cudaSuccess ||
        per_sm < 1) {
        cudaGetLastError();
        return BEM_ERR_CUDA;
    }
    RFArgs a{};
    a.n = n;
    a.ncs = gemv_splits(n);
    a.chunk = ((n + a.ncs - 1) / a.ncs + GV_UNR - 1) / GV_UNR * GV_UNR;
    if (a.chunk > RF_CHUNK_MAX) return BEM_ERR_CUDA;
    a.K = K;
    a.skip_first = skip_first ? 1 : 0;
    a.A = A;
    a.X = c.Xinv;
    a.b = b;
    a.x = x;
    a.r = c.r;
    a.part = c.part;
    a.pr = pr;
    a.cnt = c.cnt;
    a.bar = reinterpret_cast<unsigned*>(c.rf_bar);
    a.err = c.rf_bar + RF_ERR;
    a.wait_limit = c.wait_limit;
    const int nrb = (n + GV_ROWS - 1) / GV_ROWS;
    const int grid = std::min(nrb * a.ncs, per_sm * sms);
    void* args[] = {&a};
    KLAUNCH();
    const size_t smem = sizeof(double) * (size_t)a.chunk;
    if (cudaLaunchCooperativeKernel((void*)k_refine_round, grid, GV_ROWS, args, smem, s) != cudaSuccess) {
        cudaGetLastError();
        return BEM_ERR_CUDA;
    }
    return BEM_OK;
}

int mixed_solve(Ctx& c, const double* A, const double* b, double* x, cudaStream_t s, SolveTail* tail) {
    const int n = (int)c.topo.N;
    const double tol = c.prm.mixed_tol > 0 ? c.prm.mixed_tol : 1e-12;
    // the assembly already left r = b - A x for this start value in c.r (a stage of the step loop)
    bool r0_ready = c.r0_ready;
    c.r0_ready = false;
    if (c.mixed_backoff > 0) {
        --c.mixed_backoff;
        return fp64_fallback(c, A, b, x, s, false);
    }
    if (!c.xinv_valid) {
        r0_ready = false;  // the set-up uses c.r as scratch
        int rc = refresh_inverse(c, A, s, true);
        if (rc == BEM_ERR_NOT_CONVERGED) return fp64_fallback(c, A, b, x, s, true);
        if (rc) return rc;
    }
    const int nrb = (n + GV_ROWS - 1) / GV_ROWS;
    constexpr int KMAX = 12;
    double* pb = c.red;        // nrb
    double* pr = c.red + nrb;  // (KMAX+1)*nrb
    if (r0_ready)
        KLAUNCH(), k_rowblock_norm2x2<<<nrb, GV_ROWS, 0, s>>>(n, b, pb, c.r, pr);
    else
        KLAUNCH(), k_rowblock_norm2<<<nrb, GV_ROWS, 0, s>>>(n, b, pb);
    // The first round runs K steps and then up to IR_EXTRA more whose GEMVs are gated on the device:
    // a check after each residual from the K-th on stores the step at which the host's convergence
    // rule holds, and the gated GEMVs after it return at once.  A solve whose step count was guessed
    // one or two short then still ends in one round, without a second read-back, a recomputed
    // residual and a second enqueue of the solution's consumers.  A stage whose last solve needed
    // none of them gets one (a skipped gated GEMV still costs its launch).
    constexpr int IR_EXTRA = 2;
    const size_t red_cap = (size_t)(c.gmres_m + 8) * VBLK + 4096;  // doubles of c.red
    int* gate = (c.rf_bar && !(c.prm.flags & BEM_FLAG_NO_IR_GATE) && (size_t)(KMAX + IR_EXTRA + 2) * nrb <= red_cap)
                    ? c.rf_bar + RF_GATE
                    : nullptr;
    // the norms come back through pinned memory: a direct DMA the host sees as soon as it lands
    const size_t nh = (size_t)(KMAX + IR_EXTRA + 2) * nrb + 4;  // norms, the round kernel's error word, the gate
    if (c.h_red_cap < nh) {
        cudaFreeHost(c.h_red);
        c.h_red = nullptr;
        c.h_red_cap = 0;
        BEM_CUDA(c, cudaMallocHost((void**)&c.h_red, nh * sizeof(double)));
        c.h_red_cap = nh;
    }
    double* host = c.h_red;
    c.stats.last_iters = 0;
    const int st = c.solve_stage;
    int& ir_steps = st >= 0 ? c.ir_steps_stage[st] : c.ir_steps;
    int K = std::max(1, std::min(KMAX, ir_steps));
    if (tail && st >= 0 && !c.stage_round0[st]) tail = nullptr;  // not likely final after one round
    bool tail_valid = false;  // the tail was enqueued and x has not changed since
    double rho = 1.0, rel = 1.0, rel0 = -1.0;
    bool converged = false;
    bool r_fresh = false;  // c.r is b - A x for the current x, its relative norm rel (a later round skips it)
    int rounds = 0;
    int* herr = reinterpret_cast<int*>(host + (size_t)(KMAX + IR_EXTRA + 2) * nrb);
    int* hgate = herr + 1;
    for (int round = 0; round < 4; ++round) {
        ++rounds;
        ++c.stats.ir_rounds;
        tail_valid = false;  // a round changes x
        const bool skip_first = (round == 0 && r0_ready) || (round > 0 && r_fresh);
        const bool want = c.refine_ok && (c.prm.flags & BEM_FLAG_REFINE_PERSISTENT);
        const bool persistent = want && refine_round_persistent(c, A, b, x, pr, K, skip_first, s) == BEM_OK;
        const int E = (round == 0 && !persistent && gate) ? (st >= 0 ? c.ir_extra_stage[st] : IR_EXTRA) : 0;
        if (!persistent) {
            if (want) c.refine_ok = false;
            if (E) BEM_CUDA(c, cudaMemsetAsync(gate, 0xff, sizeof(int), s));  // -1: not converged
            for (int k = 0; k < K; ++k) {
                if (!(k == 0 && skip_first))
                    gemv_t<double>(n, A, x, c.r, s, c.part, c.cnt, nullptr, 0, c.r, pr + (size_t)k * nrb, nullptr,
                                   nullptr, b, -1.0);
                gemv_t<float>(n, c.Xinv, c.r, x, s, c.part, c.cnt, nullptr, 0, nullptr, nullptr, nullptr, nullptr, x,
                              1.0);
            }
            gemv_t<double>(n, A, x, c.r, s, c.part, c.cnt, nullptr, 0, c.r, pr + (size_t)K * nrb, nullptr, nullptr, b,
                           -1.0);
            for (int e = 0; e < E; ++e) {
                KLAUNCH(), k_ir_check<<<1, 32, 0, s>>>(nrb, pb, pr + (size_t)(K + e) * nrb, tol, K + e, gate);
                gemv_t<float>(n, c.Xinv, c.r, x, s, c.part, c.cnt, gate, -1, nullptr, nullptr, nullptr, nullptr, x,
                              1.0);
                gemv_t<double>(n, A, x, c.r, s, c.part, c.cnt, gate, -1, c.r, pr + (size_t)(K + e + 1) * nrb,
                               nullptr, nullptr, b, -1.0);
            }
            if (E) KLAUNCH(), k_ir_check<<<1, 32, 0, s>>>(nrb, pb, pr + (size_t)(K + E) * nrb, tol, K + E, gate);
        }
        BEM_CUDA(c, cudaMemcpyAsync(host, c.red, sizeof(double) * (size_t)(K + E + 2) * nrb, cudaMemcpyDeviceToHost,
                                    s));
        *herr = 0;
        *hgate = -1;
        if (persistent) BEM_CUDA(c, cudaMemcpyAsync(herr, c.rf_bar + RF_ERR, sizeof(int), cudaMemcpyDeviceToHost, s));
        if (E) BEM_CUDA(c, cudaMemcpyAsync(hgate, gate, sizeof(int), cudaMemcpyDeviceToHost, s));
        if (round == 0 && tail) {  // the solution's consumers, speculatively: x is final if this round converges
            if (!c.solve_ev) BEM_CUDA(c, cudaEventCreateWithFlags(&c.solve_ev, cudaEventDisableTiming));
            BEM_CUDA(c, cudaEventRecord(c.solve_ev, s));
            const int trc = tail->run();
            if (trc) return trc;
            tail_valid = true;
            BEM_CUDA(c, cudaEventSynchronize(c.solve_ev));
        } else {
            BEM_CUDA(c, cudaStreamSynchronize(s));
        }
        if (*herr) {
            // a barrier wait of the round kernel ran out: x holds some rows of this round's update and
            // r is incomplete.  Any x is a valid refinement iterate, so the round is repeated from x
            // with separate launches, which the context keeps from now on.
            // CTAs that had passed the last completed barrier may have drawn tickets of the next GEMV's
            // row blocks: clear them for the separate launches
            BEM_CUDA(c, cudaMemsetAsync(c.cnt, 0, sizeof(unsigned) * (size_t)(nrb + 1), s));
            c.stats.wait_expired++;
            c.refine_ok = false;
            r0_ready = false;
            r_fresh = false;
            tail_valid = false;
            --round;
            --rounds;
            continue;
        }
        // the steps this round made: K, or fewer than K + E when the gate closed at an extra step
        const int steps = (E && *hgate >= K) ? *hgate : K + E;
        if (round == 0 && E && st >= 0) c.ir_extra_stage[st] = (*hgate == K) ? 1 : IR_EXTRA;
        c.stats.last_iters += steps;
        double bb = 0.0;
        for (int q = 0; q < nrb; ++q) bb += host[(size_t)q];
        if (bb == 0.0) {
            tail_valid = false;
            BEM_CUDA(c, cudaMemsetAsync(x, 0, sizeof(double) * n, s));
            rel = 0.0;
            converged = true;
            break;
        }
        std::vector<double> rk((size_t)steps + 1);
        for (int k = 0; k <= steps; ++k) {
            double a = 0.0;
            for (int q = 0; q < nrb; ++q) a += host[(size_t)(1 + k) * nrb + q];
            rk[(size_t)k] = sqrt(a / bb);
        }
        if (round > 0 && skip_first) rk[0] = rel;  // the residual was not recomputed: its norm is the last one
        if (rel0 < 0) rel0 = rk[0];
        rel = rk[(size_t)steps];
        r_fresh = true;
        // contraction per step, from the steps still well above the FP64 floor of the residual
        rho = 0.0;
        for (int k = 0; k < steps; ++k)
            if (rk[(size_t)k] > 1e3 * tol) rho = std::max(rho, rk[(size_t)k + 1] / rk[(size_t)k]);
        if (rel <= tol) {
            converged = true;
            break;
        }
        if (!(rho < 0.3)) break;  // refinement too slow: GMRES below
        K = std::max(1, std::min(KMAX, (int)ceil(log(tol / rel) / log(std::max(rho, 1e-6))) + 1));
        if (rho == 0.0) K = 1;
    }
    int rc = BEM_OK;
    if (tail) tail->done = tail_valid && converged;
    if (!converged) {
        c.stats.gmres_fallbacks++;
        rc = gmres_solve(c, A, b, x, s);
        if (rc == BEM_ERR_NOT_CONVERGED) {
            c.xinv_valid = false;
            return fp64_fallback(c, A, b, x, s, true);
        }
        rho = 1.0;
    } else {
        c.stats.last_rel_residual = rel;
    }
    c.stats.total_iters += c.stats.last_iters;
    c.stats.solves++;
    // steps for the next solve from the observed contraction
    if (converged && rho > 0.0 && rel0 > tol)
        ir_steps = std::max(1, std::min(KMAX, (int)ceil(log(tol / rel0) / log(std::max(rho, 1e-6)))));
    if (st >= 0) c.stage_round0[st] = converged && rounds == 1;
    if (rc != BEM_OK) return rc;
    // Refresh policy.  X drifts from G^-1 as the surface moves, and each solve then needs a few more
    // refinement steps than right after a refresh.  A refresh (a Newton-Schulz step: two n^3 BF16x3
    // GEMMs) costs about REFRESH_COST refinement steps (two n^2 GEMVs); it is taken once the extra
    // steps paid since the last one add up to that cost (the rent-or-buy rule, within a factor two of
    // the best schedule in hindsight), or at once when the contraction is too weak for refinement.
    bool refresh = !converged || rho > 0.2;
    if (!refresh) {
        const int k = c.stats.last_iters;
        if (c.ir_base < 0 || k < c.ir_base) c.ir_base = k;
        c.ir_excess += k - c.ir_base;
        const double refresh_cost = 2.0 + n / 100.0;  // GEMM pair vs GEMV pair, measured rates on B200
        refresh = c.ir_excess > refresh_cost;
    }
    if (refresh) {
        c.ir_base = -1;
        c.ir_excess = 0;
        rc = refresh_inverse(c, A, s, false);
        if (rc == BEM_ERR_NOT_CONVERGED) {  // this solve stands; the next one starts over or falls back
            c.xinv_valid = false;
            c.mixed_backoff = MIXED_BACKOFF;
            rc = BEM_OK;
        }
    }
    return rc;
}

}  // namespace bemb
