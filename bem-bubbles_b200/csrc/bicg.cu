// Persistent BiCGSTAB: the iteration of linalg.cu's multi-kernel BiCGSTAB (the reference default
// solver, Simulation.cpp:49-53: Jacobi preconditioner, zero start, tolerance DBL_EPSILON on the
// recursive residual, at most 2N iterations, shadow-residual restart) as one cooperative kernel that
// runs a batch of iterations per launch.
//
// One BiCGSTAB iteration is two GEMVs and three vector updates; as separate launches it is about
// nine kernels, so for the small and medium systems of remeshed bubbles (N ~ 1000, G in L2) the
// launch and synchronisation overhead, not the matrix traffic, set the time.  Here the phases are
// separated by a grid-wide barrier (sense counter in global memory, bounded wait), the scalars are
// recomputed redundantly by every CTA from the same per-row-block partial sums (fixed order, so every
// CTA holds the same bits), and the host polls the done flag once per batch of iterations.
//
// Vectors written during the kernel are read with ld.global.cg (L2), never through the
// non-coherent L1 or the read-only path.  A barrier that waits longer than about a second sets an
// error word and every CTA returns; the caller then runs the multi-kernel path from the start.
#include <math.h>

#include <algorithm>

#include "ctx.h"
#include "grid_barrier.cuh"

namespace bemb {

namespace {

constexpr int PB_ROWS = 256;  // rows per row block, one thread per row
constexpr double PB_EPS = 2.220446049250313080847e-16;
enum { D_RR = 0, D_R0R = 1, D_R0V = 2, D_TT = 3, D_TS = 4, D_N = 5 };

struct PBArgs {
    int n, nrb, ncs, budget;
    const double* A;
    const double* b;
    const double* invd;
    double *x, *r, *r0, *p, *v, *y, *s, *z, *t;
    double* part;    // ncs x n column-split partials of the GEMVs
    unsigned* cnt;   // nrb row-block tickets (zero between uses)
    double* dots;    // D_N x nrb per-row-block partial dot products
    unsigned* bar;   // [0] arrivals, [1] generation
    int* err;        // barrier wait expired
    DevScalars* sc;  // scalars across launches
    long long wait_limit;  // bound of each barrier wait, SM clock cycles
};

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic CTA sum of per-thread values (PB_ROWS threads); valid in every thread.
__device__ double cta_sum(double v) {
    __shared__ double s_w[PB_ROWS / 32];
    __shared__ double s_r;
    v = wsum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) s_w[wid] = v;
    __syncthreads();
    if (wid == 0) {
        double r = lane < PB_ROWS / 32 ? s_w[lane] : 0.0;
        r = wsum(r);
        if (lane == 0) s_r = r;
    }
    __syncthreads();
    const double out = s_r;
    __syncthreads();
    return out;
}

// Fixed-order sum of the nrb row-block partials of dot k; the same bits in every CTA.
__device__ double dot_total(const PBArgs& a, int k) {
    __shared__ double s_d;
    if (threadIdx.x < 32) {
        double v = 0.0;
        for (int q = threadIdx.x; q < a.nrb; q += 32) v += __ldcg(a.dots + (size_t)k * a.nrb + q);
        v = wsum(v);
        if (threadIdx.x == 0) s_d = v;
    }
    __syncthreads();
    const double out = s_d;
    __syncthreads();
    return out;
}

__device__ __forceinline__ bool grid_sync(const PBArgs& a) { return grid_barrier(a.bar, a.bar + 1, a.err, a.wait_limit); }

// out = A in (column-major A), tiles (row block, column split) spread over the CTAs; the last CTA
// of a row block sums the splits in order, writes out and the row block's dots out.u0 -> dots[k0],
// out.u1 -> dots[k1] (u == out gives out.out).
constexpr int PB_CHUNK = 512;  // most columns of one GEMV tile (the staged slice of the input vector)

__device__ void gemv(const PBArgs& a, const double* in, double* out, const double* u0, int k0, const double* u1,
                     int k1) {
    __shared__ unsigned s_ticket;
    __shared__ double s_in[PB_CHUNK];
    const int n = a.n, ntiles = a.nrb * a.ncs, chunk = (n + a.ncs - 1) / a.ncs;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int rb = tile % a.nrb, cs = tile / a.nrb;
        const int i = rb * PB_ROWS + threadIdx.x;
        const int c0 = cs * chunk, c1 = min(n, c0 + chunk);
        __syncthreads();
        for (int j = c0 + threadIdx.x; j < c1; j += PB_ROWS) s_in[j - c0] = __ldcg(in + j);
        __syncthreads();
        if (i < n) {
            // eight independent column loads in flight per thread
            double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            const double* col = a.A + (size_t)c0 * n + i;
            int j = c0;
            for (; j + 7 < c1; j += 8) {
                double m[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) m[q] = __ldg(col + (size_t)q * n);
#pragma unroll
                for (int q = 0; q < 8; ++q) acc[q] = fma(m[q], s_in[j - c0 + q], acc[q]);
                col += 8 * (size_t)n;
            }
            for (; j < c1; ++j) {
                acc[0] = fma(__ldg(col), s_in[j - c0], acc[0]);
                col += n;
            }
            a.part[(size_t)cs * n + i] = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
        }
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) s_ticket = atomicAdd(a.cnt + rb, 1u);
        __syncthreads();
        if (s_ticket != (unsigned)(a.ncs - 1)) continue;
        __threadfence();
        double yi = 0.0;
        if (i < n) {
            for (int k = 0; k < a.ncs; ++k) yi += __ldcg(a.part + (size_t)k * n + i);
            out[i] = yi;
        }
        if (u0) {
            const double d = cta_sum(i < n ? yi * (u0 == out ? yi : __ldcg(u0 + i)) : 0.0);
            if (threadIdx.x == 0) a.dots[(size_t)k0 * a.nrb + rb] = d;
        }
        if (u1) {
            const double d = cta_sum(i < n ? yi * __ldcg(u1 + i) : 0.0);
            if (threadIdx.x == 0) a.dots[(size_t)k1 * a.nrb + rb] = d;
        }
        if (threadIdx.x == 0) a.cnt[rb] = 0u;
    }
}

__global__ void __launch_bounds__(PB_ROWS) k_pbicg(PBArgs a) {
    const int n = a.n;
    // scalars of the iteration, the same in every thread of every CTA
    double rho = __ldcg(&a.sc->rho), alpha = __ldcg(&a.sc->alpha), w = __ldcg(&a.sc->w);
    double beta = __ldcg(&a.sc->beta), r0_sq = __ldcg(&a.sc->r0_sq);
    const double tol2 = __ldcg(&a.sc->tol2);
    int iters = __ldcg(&a.sc->iters), restarts = __ldcg(&a.sc->restarts), done = __ldcg(&a.sc->done);
    int nonconv = __ldcg(&a.sc->nonconv);
    const int maxit = __ldcg(&a.sc->maxit);
    double rr = __ldcg(&a.sc->rr);
    for (int k = 0; k < a.budget && !done; ++k) {
        // loop test, rho, restart decision, beta
        rr = dot_total(a, D_RR);
        const double r0r = dot_total(a, D_R0R);
        if (!(rr > tol2) || iters >= maxit) {
            done = 1;
            nonconv = (rr > tol2) ? 1 : 0;
            break;
        }
        const double rho_old = rho;
        if (fabs(r0r) < PB_EPS * PB_EPS * r0_sq) {
            // restart: r = b - A x, r0 = r
            gemv(a, a.x, a.t, nullptr, 0, nullptr, 0);
            if (!grid_sync(a)) return;
            for (int rb = blockIdx.x; rb < a.nrb; rb += gridDim.x) {
                const int i = rb * PB_ROWS + threadIdx.x;
                double ri = 0.0;
                if (i < n) {
                    ri = __ldg(a.b + i) - __ldcg(a.t + i);
                    a.r[i] = ri;
                    a.r0[i] = ri;
                }
                const double d = cta_sum(ri * ri);
                if (threadIdx.x == 0) a.dots[(size_t)D_RR * a.nrb + rb] = d;
            }
            if (!grid_sync(a)) return;
            const double rr2 = dot_total(a, D_RR);
            rho = rr2;
            r0_sq = rr2;
            if (restarts++ == 0) iters = 0;
            beta = (rr2 / rho_old) * (alpha / w);
        } else {
            rho = r0r;
            beta = (r0r / rho_old) * (alpha / w);
        }
        // p = r + beta (p - w v); y = invd p
        for (int rb = blockIdx.x; rb < a.nrb; rb += gridDim.x) {
            const int i = rb * PB_ROWS + threadIdx.x;
            if (i < n) {
                const double pi = __ldcg(a.r + i) + beta * (__ldcg(a.p + i) - w * __ldcg(a.v + i));
                a.p[i] = pi;
                a.y[i] = __ldg(a.invd + i) * pi;
            }
        }
        if (!grid_sync(a)) return;
        // v = A y, r0.v
        gemv(a, a.y, a.v, a.r0, D_R0V, nullptr, 0);
        if (!grid_sync(a)) return;
        // alpha = rho / (r0.v); s = r - alpha v; z = invd s
        alpha = rho / dot_total(a, D_R0V);
        for (int rb = blockIdx.x; rb < a.nrb; rb += gridDim.x) {
            const int i = rb * PB_ROWS + threadIdx.x;
            if (i < n) {
                const double si = __ldcg(a.r + i) - alpha * __ldcg(a.v + i);
                a.s[i] = si;
                a.z[i] = __ldg(a.invd + i) * si;
            }
        }
        if (!grid_sync(a)) return;
        // t = A z, t.t, t.s
        gemv(a, a.z, a.t, a.t, D_TT, a.s, D_TS);
        if (!grid_sync(a)) return;
        // w = (t.s)/(t.t); x += alpha y + w z; r = s - w t; r.r and r0.r
        const double tt = dot_total(a, D_TT), ts = dot_total(a, D_TS);
        w = (tt > 0.0) ? ts / tt : 0.0;
        for (int rb = blockIdx.x; rb < a.nrb; rb += gridDim.x) {
            const int i = rb * PB_ROWS + threadIdx.x;
            double ri = 0.0, r0i = 0.0;
            if (i < n) {
                a.x[i] = __ldcg(a.x + i) + (alpha * __ldcg(a.y + i) + w * __ldcg(a.z + i));
                ri = __ldcg(a.s + i) - w * __ldcg(a.t + i);
                a.r[i] = ri;
                r0i = __ldcg(a.r0 + i);
            }
            const double d_rr = cta_sum(ri * ri);
            const double d_r0r = cta_sum(r0i * ri);
            if (threadIdx.x == 0) {
                a.dots[(size_t)D_RR * a.nrb + rb] = d_rr;
                a.dots[(size_t)D_R0R * a.nrb + rb] = d_r0r;
            }
        }
        ++iters;
        if (!grid_sync(a)) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.sc->rho = rho;
        a.sc->alpha = alpha;
        a.sc->w = w;
        a.sc->beta = beta;
        a.sc->r0_sq = r0_sq;
        a.sc->rr = rr;
        a.sc->iters = iters;
        a.sc->restarts = restarts;
        a.sc->done = done;
        a.sc->nonconv = nonconv;
    }
}

// Zero start: x = 0, r = r0 = b, p = v = 0, Jacobi diagonal, b.b per row block (as r.r and r0.r).
__global__ void __launch_bounds__(PB_ROWS) k_pbicg_init(PBArgs a) {
    const int rb = blockIdx.x, i = rb * PB_ROWS + threadIdx.x;
    double bi = 0.0;
    if (i < a.n) {
        const double d = a.A[(size_t)i * a.n + i];
        a.x[i] = 0.0;
        a.p[i] = 0.0;
        a.v[i] = 0.0;
        bi = a.b[i];
        a.r[i] = bi;
        a.r0[i] = bi;
        const_cast<double*>(a.invd)[i] = (d != 0.0) ? 1.0 / d : 1.0;
    }
    const double s = cta_sum(bi * bi);
    if (threadIdx.x == 0) {
        a.dots[(size_t)D_RR * a.nrb + rb] = s;
        a.dots[(size_t)D_R0R * a.nrb + rb] = s;
    }
    if (rb == 0 && threadIdx.x == 0) {
        a.bar[0] = 0u;
        a.bar[1] = 0u;
        *a.err = 0;
    }
}

__global__ void k_pbicg_init_scalars(PBArgs a, int maxit) {
    const double bb = dot_total(a, D_RR);
    if (threadIdx.x == 0) {
        DevScalars* sc = a.sc;
        sc->rhs_sq = bb;
        sc->r0_sq = bb;
        sc->rr = bb;
        sc->rho = 1.0;
        sc->alpha = 1.0;
        sc->w = 1.0;
        sc->beta = 0.0;
        sc->tol2 = PB_EPS * PB_EPS * bb;
        sc->iters = 0;
        sc->restarts = 0;
        sc->done = (bb == 0.0) ? 1 : 0;
        sc->restart_flag = 0;
        sc->maxit = maxit;
        sc->nonconv = 0;
    }
}

}  // namespace

size_t pbicg_words(int64_t n) { return (size_t)D_N * (size_t)((n + PB_ROWS - 1) / PB_ROWS) + 4; }

// Returns BEM_OK with the solution in x, or BEM_ERR_CUDA when the cooperative launch is unavailable
// or a barrier wait expired (the caller then uses the multi-kernel path; x is overwritten by it).
int bicgstab_persistent(Ctx& c, const double* A, const double* b, double* x, cudaStream_t s) {
    const int n = (int)c.topo.N;
    int sms = 0, per_sm = 0, coop = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c.device);
    if (!coop) return BEM_ERR_CUDA;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pbicg, PB_ROWS, 0) != cudaSuccess || per_sm < 1)
        return BEM_ERR_CUDA;
    PBArgs a{};
    a.n = n;
    a.nrb = (n + PB_ROWS - 1) / PB_ROWS;
    // CTAs: about 8K matrix entries per CTA and GEMV, at most four per SM; column splits so that the
    // tiles cover the CTAs, each at most PB_CHUNK columns wide
    const long long want = std::max(8LL, (long long)n * n / 8192);
    const int grid = (int)std::min<long long>(want, (long long)std::min(per_sm, 4) * sms);
    a.ncs = std::max({1, (grid + a.nrb - 1) / a.nrb, (n + PB_CHUNK - 1) / PB_CHUNK});
    a.ncs = std::min({a.ncs, 64, std::max(1, n / 16)});
    if ((n + a.ncs - 1) / a.ncs > PB_CHUNK) return BEM_ERR_CUDA;  // too large for the staged slice
    a.budget = 64;
    a.A = A;
    a.b = b;
    a.invd = c.invd;
    a.x = x;
    a.r = c.r;
    a.r0 = c.r0;
    a.p = c.pv;
    a.v = c.vv;
    a.y = c.yv;
    a.s = c.sv;
    a.z = c.zv;
    a.t = c.tv;
    a.part = c.part;
    a.cnt = c.cnt;
    // dots, then the barrier words and the error word (pbicg_words(n) doubles, allocated with the mesh)
    a.dots = c.pbicg;
    a.bar = reinterpret_cast<unsigned*>(c.pbicg + (size_t)D_N * a.nrb);
    a.err = reinterpret_cast<int*>(a.bar + 4);
    a.sc = c.sc;
    a.wait_limit = c.wait_limit;
    const int maxit = c.prm.max_iters > 0 ? c.prm.max_iters : 2 * n;
    KLAUNCH(), k_pbicg_init<<<a.nrb, PB_ROWS, 0, s>>>(a);
    KLAUNCH(), k_pbicg_init_scalars<<<1, 32, 0, s>>>(a, maxit);
    void* args[] = {&a};
    for (int launch = 0;; ++launch) {
        KLAUNCH();
        cudaError_t e = cudaLaunchCooperativeKernel((void*)k_pbicg, grid, PB_ROWS, args, 0, s);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return BEM_ERR_CUDA;
        }
        int err = 0;
        BEM_CUDA(c, cudaMemcpyAsync(c.h_sc, c.sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, s));
        BEM_CUDA(c, cudaMemcpyAsync(&err, a.err, sizeof(int), cudaMemcpyDeviceToHost, s));
        BEM_CUDA(c, cudaStreamSynchronize(s));
        if (err) {
            c.stats.wait_expired++;
            return c.fail(BEM_ERR_CUDA, "persistent BiCGSTAB: a grid barrier wait expired");
        }
        if (c.h_sc->done) break;
        if (launch * a.budget > 4 * maxit + 64) return c.fail(BEM_ERR_NOT_CONVERGED, "BiCGSTAB: loop guard");
    }
    c.stats.last_iters = c.h_sc->iters;
    c.stats.last_rel_residual = c.h_sc->rhs_sq > 0 ? sqrt(c.h_sc->rr / c.h_sc->rhs_sq) : 0.0;
    c.stats.total_iters += c.stats.last_iters;
    c.stats.solves++;
    return BEM_OK;
}

}  // namespace bemb
