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

// The same panel step on one thread-block cluster (up to 16 CTAs): the candidates, the diagonal row
// and the pivot row are read from the other CTAs' shared memory (distributed shared memory), and a
// column step is one hardware cluster barrier.  For panels whose rows fit in the cluster's shared
// memory (about 6000 rows of a 64-column panel).
constexpr int LC_MAX = 16;

__global__ void __launch_bounds__(LP_THREADS) k_lu_panel_cluster(int n, int k0, int nb, int rows_per, double* A,
                                                                 int* piv, int* sing) {
    namespace cgx = cooperative_groups;
    cgx::cluster_group cl = cgx::this_cluster();
    extern __shared__ double sp[];  // [rows_per][ld], then candidates [2][2 + nb] and diagonal rows [2][nb]
    __shared__ double s_v[LP_THREADS / 32];
    __shared__ int s_i[LP_THREADS / 32];
    __shared__ double s_prow[LP_NBMAX];
    __shared__ int s_pw[2];
    const int C = (int)cl.num_blocks(), me = (int)cl.block_rank(), tid = threadIdx.x;
    const int ld = nb + 1, stride = 2 + nb;
    double* cand = sp + (size_t)rows_per * ld;
    double* diag = cand + 2 * stride;
    const int r0 = k0 + me * rows_per, r1 = min(n, r0 + rows_per);
    const int nr = max(0, r1 - r0);
    for (int e = tid; e < nr * nb; e += LP_THREADS) {
        const int c = e / nr, rr = e - c * nr;
        sp[rr * ld + c] = A[(size_t)(k0 + c) * n + r0 + rr];
    }
    __syncthreads();
    for (int j = 0; j < nb; ++j) {
        const int rowj = k0 + j, par = j & 1;
        const int owner_j = (rowj - k0) / rows_per;
        double* mycand = cand + par * stride;
        double* mydiag = diag + par * nb;
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
        if (tid == 0) {
            mycand[0] = best;
            mycand[1] = (double)bi;
        }
        if (bi < n)
            for (int c = tid; c < nb; c += LP_THREADS) mycand[2 + c] = sp[(bi - r0) * ld + c];
        if (me == owner_j)
            for (int c = tid; c < nb; c += LP_THREADS) mydiag[c] = sp[(rowj - r0) * ld + c];
        cl.sync();
        // the pivot: the CTAs' candidates, largest |entry| then smallest row (the same in every CTA)
        if (tid < 32) {
            double v = -1.0;
            int i = n, w = -1;
            if (tid < C) {
                const double* rc = cl.map_shared_rank(mycand, tid);
                const int ri = (int)rc[1];
                if (ri < n) {
                    v = rc[0];
                    i = ri;
                    w = tid;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, v, o);
                const int oi = __shfl_xor_sync(0xffffffffu, i, o);
                const int ow = __shfl_xor_sync(0xffffffffu, w, o);
                if (oi < n && (ov > v || (ov == v && oi < i))) {
                    v = ov;
                    i = oi;
                    w = ow;
                }
            }
            if (tid == 0) {
                s_pw[0] = i;
                s_pw[1] = w;
            }
        }
        __syncthreads();
        int p = s_pw[0];
        const int w = s_pw[1];
        if (p >= n) p = rowj;
        const double* prow = (w >= 0) ? cl.map_shared_rank(mycand, w) + 2 : cl.map_shared_rank(mydiag, owner_j);
        const double* drow = cl.map_shared_rank(mydiag, owner_j);
        for (int c = tid; c < nb; c += LP_THREADS) s_prow[c] = prow[c];
        if (me == 0 && tid == 0) piv[rowj] = p;
        __syncthreads();
        if (p != rowj) {
            if (rowj >= r0 && rowj < r1)
                for (int c = tid; c < nb; c += LP_THREADS) sp[(rowj - r0) * ld + c] = s_prow[c];
            if (p >= r0 && p < r1)
                for (int c = tid; c < nb; c += LP_THREADS) sp[(p - r0) * ld + c] = drow[c];
        }
        __syncthreads();
        const double d = s_prow[j];
        if (d == 0.0 && me == 0 && tid == 0) *sing = 1;
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
    cl.sync();  // no CTA leaves while another may still read its shared memory
    for (int e = tid; e < nr * nb; e += LP_THREADS) {
        const int c = e / nr, rr = e - c * nr;
        A[(size_t)(k0 + c) * n + r0 + rr] = sp[rr * ld + c];
    }
}

// Row interchanges of a panel applied to the columns outside it, as one permutation: the panel's
// transpositions (j, piv[j]) composed into (destination, source) row pairs by one thread, then one
// warp per column loads every source before storing any destination.
__global__ void k_lu_perm_build(int k0, int nb, const int* __restrict__ piv, int* __restrict__ pairs) {
    // rows touched: the panel rows and their partners; content[r] = source row now at r
    int rows[2 * LP_NBMAX], src[2 * LP_NBMAX], cnt = 0;
    auto slot = [&](int r) {
        for (int q = 0; q < cnt; ++q)
            if (rows[q] == r) return q;
        rows[cnt] = r;
        src[cnt] = r;
        return cnt++;
    };
    for (int j = k0; j < k0 + nb; ++j) {
        const int p = piv[j];
        if (p == j) continue;
        const int a = slot(j), b = slot(p);
        const int t = src[a];
        src[a] = src[b];
        src[b] = t;
    }
    int m = 0;
    for (int q = 0; q < cnt; ++q)
        if (src[q] != rows[q]) {
            pairs[1 + 2 * m] = rows[q];
            pairs[2 + 2 * m] = src[q];
            ++m;
        }
    pairs[0] = m;
}

__global__ void k_lu_perm_apply(int n, int k0, int nb, const int* __restrict__ pairs, double* __restrict__ A) {
    const int col = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (col >= n || (col >= k0 && col < k0 + nb)) return;
    const int m = pairs[0];
    double* a = A + (size_t)col * n;
    double v[(2 * LP_NBMAX + 31) / 32];
#pragma unroll
    for (int q = 0; q < (2 * LP_NBMAX + 31) / 32; ++q) {
        const int k = lane + 32 * q;
        if (k < m) v[q] = a[pairs[2 + 2 * k]];
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < (2 * LP_NBMAX + 31) / 32; ++q) {
        const int k = lane + 32 * q;
        if (k < m) a[pairs[1 + 2 * k]] = v[q];
    }
}

}  // namespace

// lu_aux layout: candidates (2 parities x LP_GMAX x (2 + nb)), diagonal rows (2 x LP_NBMAX),
// barrier words (2), error word
static double* lp_diag(Ctx& c) { return c.lu_aux + (size_t)2 * LP_GMAX * (2 + LP_NBMAX); }
static unsigned* lp_bar(Ctx& c) { return reinterpret_cast<unsigned*>(lp_diag(c) + 2 * LP_NBMAX); }

// then the interchange pairs of the last panel (1 + 2 x 2 LP_NBMAX ints)
static int* lp_pairs(Ctx& c) { return reinterpret_cast<int*>(lp_bar(c) + 4); }

size_t lu_panel_words() { return (size_t)2 * LP_GMAX * (2 + LP_NBMAX) + (size_t)2 * LP_NBMAX + 8 + 2 * LP_NBMAX + 8; }

void lu_panel_swap_rest(Ctx& c, int k0, int nb, cudaStream_t s) {
    const int n = (int)c.topo.N;
    KLAUNCH(), k_lu_perm_build<<<1, 1, 0, s>>>(k0, nb, c.piv, lp_pairs(c));
    KLAUNCH(), k_lu_perm_apply<<<(n + 7) / 8, 256, 0, s>>>(n, k0, nb, lp_pairs(c), c.LU);
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
    const size_t smem = sizeof(double) * ((size_t)rows_per * (nb + 1) + 2 * (2 + nb) + 2 * nb);
    if (smem > 200 * 1024) return BEM_ERR_CUDA;
    static std::atomic<uint64_t> attr{0};
    if (!once_per_device(attr, [] {
            return cudaFuncSetAttribute(k_lu_panel_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) ==
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
    if (cudaLaunchKernelEx(&cfg, k_lu_panel_cluster, n, k0, nb, rows_per, A, piv, sing) != cudaSuccess) {
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
