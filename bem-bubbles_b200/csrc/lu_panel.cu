// Panel factorisation of the FP64 LU with row partial pivoting (Simulation::solve_system with
// set_bcgstab(false): Eigen's PartialPivLU, Simulation.cpp:57-60), spread over the SMs.
//
// The right-looking blocked LU in linalg.cu factors each panel of nb columns (rows k0..n-1) and then
// updates the trailing matrix.  Each pivot decision needs the whole column, so a panel takes nb
// steps that each see all rows.  Here the panel's rows are split over G co-resident CTAs (one
// cooperative launch per panel), each holding its rows of the nb panel columns in shared memory for
// the whole panel.  A column step is one grid barrier:
//   * every CTA finds its largest |entry| of column j among its rows at or below the diagonal
//     (first row on ties) and publishes it with the full candidate row; the owner of the diagonal row
//     publishes that row too (double-buffered by column parity, so the next step's writes never meet
//     this step's reads);
//   * after the barrier every CTA picks the same pivot from the candidates in CTA order (largest
//     |entry|, then smallest row: the single-CTA kernel's rule), the owners of the two rows exchange
//     them, and every CTA eliminates below the diagonal with the pivot row: l = a_ij / a_jj,
//     a_ik -= l * a_jk for the panel columns right of j (the arithmetic of the single-CTA kernel).
// At the end each CTA writes its rows back.  A barrier wait that expires sets an error word; the
// caller then factors the matrix again with the single-CTA panel.
#include <cooperative_groups.h>
#include <math.h>

#include <algorithm>

#include "ctx.h"
#include "grid_barrier.cuh"

namespace bemb {

namespace {

constexpr int LP_THREADS = 256;
constexpr int LP_NBMAX = 64;    // widest panel
constexpr int LP_GMAX = 1024;   // most CTAs of one panel

struct LPArgs {
    int n, k0, nb, rows_per;
    double* A;       // column-major n x n, factored in place
    int* piv;        // n: row interchanged with row k at step k
    int* sing;       // set on a zero pivot
    double* cand;    // 2 (parity) x G x (2 + nb): |entry|, row index, candidate row
    double* diag;    // 2 (parity) x nb: the diagonal row before the interchange
    unsigned* bar;   // grid barrier words
    int* err;        // barrier wait expired
    long long wait_limit;  // bound of each barrier wait, SM clock cycles
};

__global__ void __launch_bounds__(LP_THREADS) k_lu_panel_rows(LPArgs a) {
    extern __shared__ double sp[];  // [rows][ld], row-major; ld = nb + 1 (odd: no bank conflicts down a column)
    __shared__ double s_v[LP_THREADS / 32];
    __shared__ int s_i[LP_THREADS / 32];
    __shared__ int s_w[LP_THREADS / 32];
    __shared__ double s_prow[LP_NBMAX];
    const int n = a.n, nb = a.nb, G = gridDim.x, tid = threadIdx.x;
    const int r0 = a.k0 + blockIdx.x * a.rows_per, r1 = min(n, r0 + a.rows_per);
    const int nr = max(0, r1 - r0);
    const int stride = 2 + nb, ld = nb + 1;
    for (int e = tid; e < nr * nb; e += LP_THREADS) {
        const int c = e / nr, rr = e - c * nr;
        sp[rr * ld + c] = a.A[(size_t)(a.k0 + c) * n + r0 + rr];
    }
    __syncthreads();
    for (int j = 0; j < nb; ++j) {
        const int rowj = a.k0 + j;
        const int par = j & 1;
        double* cand = a.cand + (size_t)par * G * stride;
        double* diag = a.diag + (size_t)par * nb;
        // local pivot candidate: largest |a_ij| over owned rows i >= rowj, first row on ties
        double best = -1.0;
        int bi = n;
        for (int rr = tid; rr < nr; rr += LP_THREADS) {
            const int i = r0 + rr;
            if (i < rowj) continue;
            const double v = fabs(sp[rr * ld + j]);
            if (v > best || (v == best && i < bi)) {
                best = v;
                bi = i;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) {
                best = ov;
                bi = oi;
            }
        }
        if ((tid & 31) == 0) {
            s_v[tid >> 5] = best;
            s_i[tid >> 5] = bi;
        }
        __syncthreads();
        if (tid < 32) {
            best = tid < LP_THREADS / 32 ? s_v[tid] : -2.0;
            bi = tid < LP_THREADS / 32 ? s_i[tid] : n;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ov > best || (ov == best && oi < bi)) {
                    best = ov;
                    bi = oi;
                }
            }
            if (tid == 0) {
                s_v[0] = best;
                s_i[0] = bi;
            }
        }
        __syncthreads();
        best = s_v[0];
        bi = s_i[0];
        double* mine = cand + (size_t)blockIdx.x * stride;
        if (tid == 0) {
            mine[0] = best;
            mine[1] = (double)bi;
        }
        if (bi < n)
            for (int c = tid; c < nb; c += LP_THREADS) mine[2 + c] = sp[(bi - r0) * ld + c];
        if (rowj >= r0 && rowj < r1)
            for (int c = tid; c < nb; c += LP_THREADS) diag[c] = sp[(rowj - r0) * ld + c];
        if (!grid_barrier(a.bar, a.bar + 1, a.err, a.wait_limit)) return;
        // the pivot, the same in every CTA: largest |entry| over the candidates, then smallest row (an
        // order-independent rule, reduced over the threads)
        double pv = -1.0;
        int p = n, w = -1;
        for (int g = tid; g < G; g += LP_THREADS) {
            const double v = __ldcg(cand + (size_t)g * stride);
            const int i = (int)__ldcg(cand + (size_t)g * stride + 1);
            if (i < n && (v > pv || (v == pv && i < p))) {
                pv = v;
                p = i;
                w = g;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, pv, o);
            const int oi = __shfl_xor_sync(0xffffffffu, p, o);
            const int ow = __shfl_xor_sync(0xffffffffu, w, o);
            if (oi < n && (ov > pv || (ov == pv && oi < p))) {
                pv = ov;
                p = oi;
                w = ow;
            }
        }
        if ((tid & 31) == 0) {
            s_v[tid >> 5] = pv;
            s_i[tid >> 5] = p;
            s_w[tid >> 5] = w;
        }
        __syncthreads();
        if (tid < 32) {
            pv = tid < LP_THREADS / 32 ? s_v[tid] : -1.0;
            p = tid < LP_THREADS / 32 ? s_i[tid] : n;
            w = tid < LP_THREADS / 32 ? s_w[tid] : -1;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, pv, o);
                const int oi = __shfl_xor_sync(0xffffffffu, p, o);
                const int ow = __shfl_xor_sync(0xffffffffu, w, o);
                if (oi < n && (ov > pv || (ov == pv && oi < p))) {
                    pv = ov;
                    p = oi;
                    w = ow;
                }
            }
            if (tid == 0) {
                s_i[0] = p;
                s_w[0] = w;
            }
        }
        __syncthreads();
        p = s_i[0];
        w = s_w[0];
        if (p >= n) p = rowj;  // no candidate: keep the diagonal row
        const double* prow = (w >= 0) ? cand + (size_t)w * stride + 2 : diag;
        for (int c = tid; c < nb; c += LP_THREADS) s_prow[c] = __ldcg(prow + c);
        if (blockIdx.x == 0 && tid == 0) a.piv[rowj] = p;
        __syncthreads();
        // interchange: the pivot row goes to rowj, the old diagonal row to p
        if (p != rowj) {
            if (rowj >= r0 && rowj < r1)
                for (int c = tid; c < nb; c += LP_THREADS) sp[(rowj - r0) * ld + c] = s_prow[c];
            if (p >= r0 && p < r1)
                for (int c = tid; c < nb; c += LP_THREADS) sp[(p - r0) * ld + c] = __ldcg(diag + c);
        }
        __syncthreads();
        // eliminate below the diagonal with the pivot row
        const double d = s_prow[j];
        if (d == 0.0) {
            if (blockIdx.x == 0 && tid == 0) *a.sing = 1;
        }
        for (int rr = tid; rr < nr; rr += LP_THREADS) {
            const int i = r0 + rr;
            if (i <= rowj) continue;
            double l = sp[rr * ld + j];
            if (d != 0.0) {
                l /= d;
                sp[rr * ld + j] = l;
            }
            for (int c = j + 1; c < nb; ++c) sp[rr * ld + c] -= l * s_prow[c];
        }
        __syncthreads();
    }
    for (int e = tid; e < nr * nb; e += LP_THREADS) {
        const int c = e / nr, rr = e - c * nr;
        a.A[(size_t)(a.k0 + c) * n + r0 + rr] = sp[rr * ld + c];
    }
}

// One warp: tab_r[q] is a touched row, tab_s[q] the source row whose entries now sit there (both in
// shared memory, at most 2 nb entries).  Each transposition swaps the sources of its two rows; the
// lanes look a row up in parallel.  pairs[0] = m, then m (destination, source) pairs.
// A transposition whose partner row is not in (k0 + j, n) is skipped: it can only come from a panel
// whose bounded wait expired (an error the host reports), and skipping keeps every access in bounds.
__device__ void lu_build_pairs_warp(int n, int k0, int nb, const int* pj, int* tab_r, int* tab_s, int* pairs) {
    const int lane = threadIdx.x & 31;
    int cnt = 0;
    auto slot = [&](int r) {
        int found = -1;
        for (int q0 = 0; q0 < cnt && found < 0; q0 += 32) {
            const unsigned m = __ballot_sync(0xffffffffu, q0 + lane < cnt && tab_r[q0 + lane] == r);
            if (m) found = q0 + __ffs(m) - 1;
        }
        if (found >= 0) return found;
        if (lane == 0) {
            tab_r[cnt] = r;
            tab_s[cnt] = r;
        }
        __syncwarp();
        return cnt++;
    };
    for (int j = 0; j < nb; ++j) {
        const int rj = k0 + j, p = pj[j];
        if (p <= rj || p >= n) continue;
        const int a = slot(rj), b = slot(p);
        if (lane == 0) {
            const int t = tab_s[a];
            tab_s[a] = tab_s[b];
            tab_s[b] = t;
        }
        __syncwarp();
    }
    int m = 0;
    for (int q0 = 0; q0 < cnt; q0 += 32) {
        const int q = q0 + lane;
        const bool moved = q < cnt && tab_s[q] != tab_r[q];
        const unsigned bal = __ballot_sync(0xffffffffu, moved);
        if (moved) {
            const int k = m + __popc(bal & ((1u << lane) - 1u));
            pairs[1 + 2 * k] = tab_r[q];
            pairs[2 + 2 * k] = tab_s[q];
        }
        m += __popc(bal);
    }
    if (lane == 0) pairs[0] = m;
}

// The same panel on one thread-block cluster (up to 16 CTAs), for panels whose rows fit in the
// cluster's shared memory (about 5700 rows of a 64-column panel).  The candidates travel by push: a
// column step is
//   * each thread already holds the largest |entry| of the column among its rows (found while it
//     eliminated the previous column); one block barrier reduces them to the CTA's candidate;
//   * warp 0 writes the candidate (|entry|, row, the whole row) into slot `me` of every CTA's inbox,
//     the CTA owning the diagonal row writes that row into every CTA's diagonal box, and one lane per
//     destination arrives on the destination's mbarrier (release at cluster scope);
//   * warp 0 waits (bounded) on its own mbarrier for all CTAs' arrivals (acquire), then picks the
//     pivot from its inbox: largest |entry|, then smallest row (the single-CTA kernel's rule); the
//     pivot row and the diagonal row are already in its own shared memory; one block barrier;
//   * each thread takes its rows: the diagonal row's owner writes the pivot row there, the pivot
//     row's owner writes the old diagonal row in its place, and every row below the diagonal is
//     eliminated, l = a_ij * (1 / a_jj), a_ik -= l * a_jk, the next column first, so its candidate
//     comes with it.
// Inbox, diagonal box and mbarrier are double-buffered by column parity: a CTA writes column j + 2's
// candidates only after all CTAs' arrivals for column j + 1, which each CTA makes after it has read
// its column-j inbox.  A wait that runs out sets *err; the CTA still makes every write and arrival of
// the remaining columns (so no other CTA waits on it), and the caller factors again without the
// cluster.
constexpr int LC_MAX = 16;
constexpr size_t LC_SMEM = 220 * 1024;  // dynamic shared memory of one cluster CTA, at most

__device__ __forceinline__ uint32_t lp_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Bounded wait for phase `parity` of the local mbarrier `bar` (acquire at cluster scope): polls with
// the non-blocking test_wait and gives up after `limit` SM clock cycles.
__device__ __forceinline__ bool lp_bar_wait(uint32_t bar, uint32_t parity, long long limit) {
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > limit) return false;
    }
}

// pairs (may be null): CTA 0 also composes the panel's interchanges (lu_build_pairs_warp) at the end.
__global__ void __launch_bounds__(LP_THREADS) k_lu_panel_cluster(int n, int k0, int nb, int rows_per, double* A,
                                                                 int* piv, int* sing, int* pairs, int* err,
                                                                 long long wait_limit) {
    namespace cgx = cooperative_groups;
    cgx::cluster_group cl = cgx::this_cluster();
    // dynamic: [rows_per][ld] rows, inbox [2][C][2 + nb], diagonal box [2][nb]
    extern __shared__ double sp[];
    constexpr int NW = LP_THREADS / 32;
    __shared__ double s_v[NW];
    __shared__ int s_i[NW];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ double s_rcp;
    __shared__ int s_p, s_w, s_piv[LP_NBMAX], tab_r[2 * LP_NBMAX], tab_s[2 * LP_NBMAX];
    const int C = (int)cl.num_blocks(), me = (int)cl.block_rank(), tid = threadIdx.x;
    const int lane = tid & 31, wid = tid >> 5;
    const int ld = nb + 1, stride = 2 + nb;
    double* inbox = sp + (size_t)rows_per * ld;
    double* dbox = inbox + 2 * C * stride;
    const int r0 = k0 + me * rows_per, r1 = min(n, r0 + rows_per);
    const int nr = max(0, r1 - r0);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(lp_smem(&s_bar[0])), "r"(C));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(lp_smem(&s_bar[1])), "r"(C));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // the CTA's rows of the panel, 16 loads in flight per thread
    for (int e0 = tid; e0 < nr * nb; e0 += 16 * LP_THREADS) {
        double v[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            const int e = e0 + u * LP_THREADS, c = e / max(nr, 1), rr = e - c * nr;
            v[u] = e < nr * nb ? A[(size_t)(k0 + c) * n + r0 + rr] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            const int e = e0 + u * LP_THREADS, c = e / max(nr, 1), rr = e - c * nr;
            if (e < nr * nb) sp[rr * ld + c] = v[u];
        }
    }
    cl.sync();  // every CTA's mbarriers initialised before anyone arrives on them
    // this thread's candidate for column 0 (every row of the panel is at or below the diagonal)
    double best = -1.0;
    int bi = n;
    for (int rr = tid; rr < nr; rr += LP_THREADS) {
        const double v = fabs(sp[rr * ld]);
        if (v > best) {  // rows increase with rr: the first row wins ties
            best = v;
            bi = r0 + rr;
        }
    }
    bool ok = true;
    for (int j = 0; j < nb; ++j) {
        const int rowj = k0 + j, par = j & 1;
        const int owner_j = (rowj - k0) / rows_per;
        double* box = inbox + (size_t)par * C * stride;  // [C][2 + nb]
        double* dg = dbox + (size_t)par * nb;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
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
            double v = lane < NW ? s_v[lane] : -2.0;
            int i = lane < NW ? s_i[lane] : n;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, v, o);
                const int oi = __shfl_xor_sync(0xffffffffu, i, o);
                if (ov > v || (ov == v && oi < i)) {
                    v = ov;
                    i = oi;
                }
            }
            // the candidate row (two columns per lane) and, from the owner, the diagonal row
            const bool h0 = lane < nb, h1 = lane + 32 < nb;
            const double* crow = sp + (size_t)(i < n ? i - r0 : 0) * ld;
            const double c0v = (i < n && h0) ? crow[lane] : 0.0, c1v = (i < n && h1) ? crow[lane + 32] : 0.0;
            const bool own = me == owner_j;
            const double* drow_l = sp + (size_t)(own ? rowj - r0 : 0) * ld;
            const double d0v = (own && h0) ? drow_l[lane] : 0.0, d1v = (own && h1) ? drow_l[lane + 32] : 0.0;
            double* slot = box + (size_t)me * stride;
            for (int t = 0; t < C; ++t) {
                double* rs = cl.map_shared_rank(slot, t);
                if (lane == 0) {
                    rs[0] = v;
                    rs[1] = (double)i;
                }
                if (h0) rs[2 + lane] = c0v;
                if (h1) rs[2 + lane + 32] = c1v;
                if (own) {
                    double* rd = cl.map_shared_rank(dg, t);
                    if (h0) rd[lane] = d0v;
                    if (h1) rd[lane + 32] = d1v;
                }
            }
            asm volatile("fence.acq_rel.cluster;" ::: "memory");
            __syncwarp();
            if (lane < C) {
                uint32_t rb;
                asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(rb) : "r"(lp_smem(&s_bar[par])), "r"(lane));
                asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(rb) : "memory");
            }
            // all CTAs' candidates for this column, then the pivot (the same in every CTA)
            if (!lp_bar_wait(lp_smem(&s_bar[par]), (uint32_t)((j >> 1) & 1), wait_limit)) ok = false;
            double bv = -1.0;
            int bi2 = n, bw = -1;
            if (lane < C) {
                const double* rc = box + (size_t)lane * stride;
                const int ri = (int)rc[1];
                if (ri < n) {
                    bv = rc[0];
                    bi2 = ri;
                    bw = lane;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi2, o);
                const int ow = __shfl_xor_sync(0xffffffffu, bw, o);
                if (oi < n && (ov > bv || (ov == bv && oi < bi2))) {
                    bv = ov;
                    bi2 = oi;
                    bw = ow;
                }
            }
            if (bw >= 0 && (bi2 < rowj || bi2 >= n)) {  // not a row of this column's candidates: only
                bw = -1;                                // after an expired wait (garbage), never used
                bi2 = n;
                ok = false;
            }
            if (lane == 0) {
                const int p = (bi2 < n) ? bi2 : rowj;  // no candidate: keep the diagonal row
                const double d = (bw >= 0) ? box[(size_t)bw * stride + 2 + j] : dg[j];
                s_p = p;
                s_w = bw;
                s_rcp = d != 0.0 ? 1.0 / d : 0.0;
                s_piv[j] = p;
                if (me == 0) {
                    piv[rowj] = p;
                    if (d == 0.0) *sing = 1;
                }
            }
        }
        __syncthreads();
        const int p = s_p, w = s_w;
        const double rcp = s_rcp;
        const double* prow = (w >= 0) ? box + (size_t)w * stride + 2 : dg;
        best = -1.0;
        bi = n;
        for (int rr = tid; rr < nr; rr += LP_THREADS) {
            const int i = r0 + rr;
            if (i < rowj) continue;
            double* row = sp + rr * ld;
            // copies and updates go eight columns at a time, their loads before their stores (one
            // column at a time each load waits behind the previous store: the warp of the one lane
            // doing it then holds up the column step)
            if (i == rowj) {  // the pivot row moves here, multipliers of the earlier columns included
                if (p != rowj)
                    for (int cb = 0; cb < nb; cb += 8) {
                        double pv[8];
#pragma unroll
                        for (int u = 0; u < 8; ++u)
                            if (cb + u < nb) pv[u] = prow[cb + u];
#pragma unroll
                        for (int u = 0; u < 8; ++u)
                            if (cb + u < nb) row[cb + u] = pv[u];
                    }
                continue;
            }
            // the old diagonal row moves to the pivot's place: its earlier multipliers are copied and
            // the rest is eliminated straight from the diagonal box
            const double* src = row;
            if (i == p) {
                src = dg;
                for (int cb = 0; cb < j; cb += 8) {
                    double dv[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u)
                        if (cb + u < j) dv[u] = dg[cb + u];
#pragma unroll
                    for (int u = 0; u < 8; ++u)
                        if (cb + u < j) row[cb + u] = dv[u];
                }
            }
            double l = src[j];
            if (rcp != 0.0) l *= rcp;
            row[j] = l;
            if (j + 1 < nb) {
                const double v1 = src[j + 1] - l * prow[j + 1];
                row[j + 1] = v1;
                const double a1 = fabs(v1);
                if (a1 > best) {  // rows increase with rr
                    best = a1;
                    bi = i;
                }
            }
            for (int cb = j + 2; cb < nb; cb += 8) {
                double rv[8], pv[8];
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (cb + u < nb) {
                        rv[u] = src[cb + u];
                        pv[u] = prow[cb + u];
                    }
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (cb + u < nb) row[cb + u] = rv[u] - l * pv[u];
            }
        }
    }
    if (!ok && lane == 0) atomicExch(err, 1);
    cl.sync();  // no CTA leaves while another may still write into its shared memory
    for (int e = tid; e < nr * nb; e += LP_THREADS) {
        const int c = e / nr, rr = e - c * nr;
        A[(size_t)(k0 + c) * n + r0 + rr] = sp[rr * ld + c];
    }
    if (pairs && me == 0 && wid == 0) lu_build_pairs_warp(n, k0, nb, s_piv, tab_r, tab_s, pairs);
}

// Row interchanges of a panel applied to the columns outside it, as one permutation: the panel's
// transpositions (k0 + j, pj[j]) composed into (destination, source) row pairs by one warp, then one
// warp per column loads every source before storing any destination.
__global__ void __launch_bounds__(32) k_lu_perm_build(int n, int k0, int nb, const int* __restrict__ piv,
                                                      int* __restrict__ pairs) {
    __shared__ int tab_r[2 * LP_NBMAX], tab_s[2 * LP_NBMAX];
    lu_build_pairs_warp(n, k0, nb, piv + k0, tab_r, tab_s, pairs);
}

// perm (may be null): the composed row permutation so far, permuted like one more column
__global__ void k_lu_perm_apply(int n, int k0, int nb, const int* __restrict__ pairs, double* __restrict__ A,
                                int* __restrict__ perm) {
    const int col = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    const int m = pairs[0];
    constexpr int NQ = (2 * LP_NBMAX + 31) / 32;
    if (col == n && perm) {
        int v[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const int k = lane + 32 * q;
            if (k < m) v[q] = perm[pairs[2 + 2 * k]];
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const int k = lane + 32 * q;
            if (k < m) perm[pairs[1 + 2 * k]] = v[q];
        }
        return;
    }
    if (col >= n || (col >= k0 && col < k0 + nb)) return;
    double* a = A + (size_t)col * n;
    double v[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        const int k = lane + 32 * q;
        if (k < m) v[q] = a[pairs[2 + 2 * k]];
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        const int k = lane + 32 * q;
        if (k < m) a[pairs[1 + 2 * k]] = v[q];
    }
}

__global__ void k_iota_int(int n, int* __restrict__ v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

}  // namespace

// lu_aux layout: candidates (2 parities x LP_GMAX x (2 + nb)), diagonal rows (2 x LP_NBMAX),
// barrier words (2), error word
static double* lp_diag(Ctx& c) { return c.lu_aux + (size_t)2 * LP_GMAX * (2 + LP_NBMAX); }
static unsigned* lp_bar(Ctx& c) { return reinterpret_cast<unsigned*>(lp_diag(c) + 2 * LP_NBMAX); }

// then the interchange pairs of the last panel (1 + 2 x 2 LP_NBMAX ints)
static int* lp_pairs(Ctx& c) { return reinterpret_cast<int*>(lp_bar(c) + 4); }

size_t lu_panel_words() { return (size_t)2 * LP_GMAX * (2 + LP_NBMAX) + (size_t)2 * LP_NBMAX + 8 + 2 * LP_NBMAX + 8; }

// built: the panel kernel already composed the pairs (the cluster panel of c.LU does)
void lu_panel_swap_rest(Ctx& c, int k0, int nb, cudaStream_t s, bool built) {
    const int n = (int)c.topo.N;
    if (!built) KLAUNCH(), k_lu_perm_build<<<1, 32, 0, s>>>(n, k0, nb, c.piv, lp_pairs(c));
    KLAUNCH(), k_lu_perm_apply<<<(n + 1 + 7) / 8, 256, 0, s>>>(n, k0, nb, lp_pairs(c), c.LU, c.lu_perm);
}

void lu_perm_init(Ctx& c, cudaStream_t s) {
    const int n = (int)c.topo.N;
    KLAUNCH(), k_iota_int<<<(n + 255) / 256, 256, 0, s>>>(n, c.lu_perm);
}

// The panel on one thread-block cluster when its rows fit; BEM_ERR_CUDA when they do not or the
// cluster launch is unavailable.
int lu_panel_cluster(Ctx& c, int k0, int nb, cudaStream_t s, const PanelTarget* tgt) {
    const int n = tgt ? tgt->n : (int)c.topo.N;
    double* A = tgt ? tgt->A : c.LU;
    int* piv = tgt ? tgt->piv : c.piv;
    int* sing = tgt ? tgt->sing : c.flag;
    const int P = n - k0;
    if (nb > LP_NBMAX) return BEM_ERR_CUDA;
    const int C = std::max(1, std::min(LC_MAX, (P + 127) / 128));
    const int rows_per = (P + C - 1) / C;
    const size_t smem = sizeof(double) * ((size_t)rows_per * (nb + 1) + (size_t)2 * C * (2 + nb) + 2 * nb);
    if (smem > LC_SMEM) return BEM_ERR_CUDA;
    static std::atomic<uint64_t> attr{0};
    if (!once_per_device(attr, [] {
            return cudaFuncSetAttribute(k_lu_panel_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LC_SMEM) ==
                       cudaSuccess &&
                   cudaFuncSetAttribute(k_lu_panel_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
                       cudaSuccess;
        })) {
        cudaGetLastError();
        return BEM_ERR_CUDA;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C);
    cfg.blockDim = dim3(LP_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, k_lu_panel_cluster, &cfg) != cudaSuccess || clusters < 1) {
        cudaGetLastError();
        return BEM_ERR_CUDA;
    }
    KLAUNCH();
    int* pairs = tgt ? nullptr : lp_pairs(c);  // the interchange pairs of c.LU's panel, composed in the kernel
    if (cudaLaunchKernelEx(&cfg, k_lu_panel_cluster, n, k0, nb, rows_per, A, piv, sing, pairs, lu_panel_err(c),
                           (long long)c.wait_limit) != cudaSuccess) {
        cudaGetLastError();
        return BEM_ERR_CUDA;
    }
    return BEM_OK;
}

int* lu_panel_err(Ctx& c) { return reinterpret_cast<int*>(lp_bar(c) + 2); }

// Factor panel [k0, k0+nb) of c.LU (or of tgt's matrix) over rows k0..n-1.  Returns BEM_ERR_CUDA when the cooperative
// launch is unavailable or a barrier wait expired (the caller falls back to the single-CTA panel,
// from a fresh copy of the matrix).
int lu_panel_rows(Ctx& c, int k0, int nb, cudaStream_t s, const PanelTarget* tgt) {
    const int n = tgt ? tgt->n : (int)c.topo.N;
    int sms = 0, coop = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c.device);
    if (!coop) return BEM_ERR_CUDA;
    const int P = n - k0;
    const int G = std::max(1, std::min(sms, (P + 127) / 128));
    const int rows_per = (P + G - 1) / G;
    if (nb > LP_NBMAX || G > LP_GMAX) return BEM_ERR_CUDA;
    const size_t smem = sizeof(double) * (size_t)rows_per * (nb + 1);
    if (smem > 200 * 1024) return BEM_ERR_CUDA;
    static std::atomic<uint64_t> attr{0};
    if (!once_per_device(attr, [] {
            return cudaFuncSetAttribute(k_lu_panel_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) ==
                   cudaSuccess;
        })) {
        cudaGetLastError();
        return BEM_ERR_CUDA;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lu_panel_rows, LP_THREADS, smem) != cudaSuccess ||
        per_sm * sms < G)
        return BEM_ERR_CUDA;
    LPArgs a{};
    a.n = n;
    a.k0 = k0;
    a.nb = nb;
    a.rows_per = rows_per;
    a.A = tgt ? tgt->A : c.LU;
    a.piv = tgt ? tgt->piv : c.piv;
    a.sing = tgt ? tgt->sing : c.flag;
    a.cand = c.lu_aux;
    a.diag = lp_diag(c);
    a.bar = lp_bar(c);
    a.err = lu_panel_err(c);  // cleared once per factorisation by the caller
    a.wait_limit = c.wait_limit;
    BEM_CUDA(c, cudaMemsetAsync(a.bar, 0, 2 * sizeof(unsigned), s));
    void* args[] = {&a};
    KLAUNCH();
    cudaError_t e = cudaLaunchCooperativeKernel((void*)k_lu_panel_rows, G, LP_THREADS, args, smem, s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return BEM_ERR_CUDA;
    }
    return BEM_OK;
}

}  // namespace bemb
