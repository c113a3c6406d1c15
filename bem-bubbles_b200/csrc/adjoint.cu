// Adjoint (reverse mode) of fixed-dt RK4 trajectories of LinLinSim (LinLinSim.cpp:194-257): given
// the adjoint of the final state (xbar_K, phibar_K), the adjoint of the initial state.  There is no
// counterpart in the reference; this differentiates its forward map as the other kernels compute it.
//
// Forward: bem_adjoint_record runs the steps and keeps one checkpoint (x, phi, t) per step.
// Backward: per step, last first, the four stages are recomputed from the checkpoint (keeping
// each stage's G, H, psi, velocities) and reversed:
//   pot_t        Dphi/Dt = |v|^2/2 + p_inf - eps (V0/V_part)^gamma + A sin(kx x + w t + c)
//   position_t   v_i = mean over t of (g_t + psi_i n_t), g_t the tangent gradient, n_t the normal
//   solve        psi = G^-1 b, b = H_eff phi:  mu = G^-T psibar (refinement with X^T),
//                phibar += H_eff^T mu, Gbar_ij = -mu_i psi_j, Hbar_ij = mu_i (phi_j - phi_i) on the
//                raw entries (the 4 pi rule makes row i depend on phi_j - phi_i)
//   assembly     the derivative of every (row, triangle) integral with respect to the row's point
//                and the triangle's vertices, contracted with those weights on the fly.
// The assembly derivative runs as two passes that each recompute the pair terms: one thread per
// triangle over a chunk of rows (per-triangle sums), one thread per row over a chunk of triangles
// (per-row sums); partial sums are combined in a fixed order, so results are deterministic.
// Scope: free-space bubbles (no wall image), sigma = 0, device-evaluated field, single systems.
#include <math.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "ctx.h"

namespace bemb {

__constant__ double a_qc[7][3];   // basis weights (1-u, u-v, v) * w
__constant__ double a_quv[7][2];  // (u, v) of the points y = a + u (b - a) + v (c - b)
__constant__ double a_w[7];       // point weights
__constant__ double a_gc[7], a_gs[7], a_gw[7];

static void upload_adj_constants() {
    static std::atomic<uint64_t> done{0};
    once_per_device(done, [] {
        QuadTables t;
        quad_tables(t);
        return cudaMemcpyToSymbol(a_qc, t.qc, sizeof(t.qc)) == cudaSuccess &&
               cudaMemcpyToSymbol(a_quv, t.quv, sizeof(t.quv)) == cudaSuccess &&
               cudaMemcpyToSymbol(a_w, t.w, sizeof(t.w)) == cudaSuccess &&
               cudaMemcpyToSymbol(a_gc, t.gc, sizeof(t.gc)) == cudaSuccess &&
               cudaMemcpyToSymbol(a_gs, t.gs, sizeof(t.gs)) == cudaSuccess &&
               cudaMemcpyToSymbol(a_gw, t.gw, sizeof(t.gw)) == cudaSuccess;
    });
}

struct v3 {
    double x, y, z;
};
__device__ __forceinline__ v3 ld(const double* p, int i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ __forceinline__ v3 operator+(v3 a, v3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ v3 operator-(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ v3 operator*(double s, v3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ v3 cr(v3 a, v3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__device__ __forceinline__ double dt3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ void add3(double* p, int i, v3 v) {
    p[3 * i] += v.x;
    p[3 * i + 1] += v.y;
    p[3 * i + 2] += v.z;
}
__device__ __forceinline__ void put3(double* p, int i, v3 v) {
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}
// VJP of w = p x q: pbar += q x wbar, qbar += wbar x p
__device__ __forceinline__ void cross_vjp(v3 p, v3 q, v3 wb, v3& pb, v3& qb) {
    pb = pb + cr(q, wb);
    qb = qb + cr(wb, p);
}

// ------------------------------------------------------------------------------------------------
// Assembly derivative
// ------------------------------------------------------------------------------------------------
constexpr int AREC = 44;  // per-triangle record of the adjoint assembly
// y_q (21), N = ab x bc (3), |N|, N.a, Psi_q (7), Phi_q (7), a (3), pad
__global__ void k_adj_records(int M, const double* __restrict__ x, const int* __restrict__ tri,
                              const double* __restrict__ psi, const double* __restrict__ phi, double* __restrict__ rec) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M) return;
    const int ia = tri[3 * t], ib = tri[3 * t + 1], ic = tri[3 * t + 2];
    const v3 A = ld(x, ia), B = ld(x, ib), C = ld(x, ic);
    const v3 ab = B - A, bc = C - B;
    const v3 N = cr(ab, bc);
    double* r = rec + (size_t)t * AREC;
#pragma unroll
    for (int q = 0; q < 7; ++q) {
        const double u = a_quv[q][0], v = a_quv[q][1];
        r[3 * q] = (A.x + u * ab.x) + v * bc.x;
        r[3 * q + 1] = (A.y + u * ab.y) + v * bc.y;
        r[3 * q + 2] = (A.z + u * ab.z) + v * bc.z;
        r[30 + q] = a_qc[q][0] * psi[ia] + a_qc[q][1] * psi[ib] + a_qc[q][2] * psi[ic];
        r[37 + q] = a_qc[q][0] * phi[ia] + a_qc[q][1] * phi[ib] + a_qc[q][2] * phi[ic];
    }
    r[21] = N.x;
    r[22] = N.y;
    r[23] = N.z;
    r[24] = sqrt(dt3(N, N));
    r[25] = dt3(N, A);
    r[26] = A.x;
    r[27] = A.y;
    r[28] = A.z;
    r[29] = 0.0;
}

// One regular (row i, triangle t) pair, weights from mu_i, psi, phi:
//   J = |N| sum_q alpha_q / r_q - P sum_q eta_q / r_q^3,  P = N.(a - x_i),
//   alpha_q = -mu_i Psi_q,  eta_q = mu_i (Phi_q - phi_i w_q).
// Returns S1 = sum alpha/r, S3 = sum eta/r^3 and accumulates dJ/dz_q (z_q = y_q - x_i) into zb.
__device__ __forceinline__ void pair_terms(const double* __restrict__ r, v3 xi, double mu, double phii, double& S1,
                                           double& S3, v3* zb) {
    const double nrm = r[24];
    const double P = r[25] - (r[21] * xi.x + r[22] * xi.y + r[23] * xi.z);
    S1 = 0.0;
    S3 = 0.0;
#pragma unroll
    for (int q = 0; q < 7; ++q) {
        const v3 z = {r[3 * q] - xi.x, r[3 * q + 1] - xi.y, r[3 * q + 2] - xi.z};
        const double r2 = dt3(z, z);
        const double inv = 1.0 / sqrt(r2);
        const double inv3 = inv * inv * inv;
        const double al = -mu * r[30 + q];
        const double et = mu * (r[37 + q] - phii * a_w[q]);
        S1 = fma(al, inv, S1);
        S3 = fma(et, inv3, S3);
        const double cf = -nrm * al * inv3 + 3.0 * P * et * inv3 * inv * inv;
        zb[q] = zb[q] + cf * z;
    }
}

// Triangle side: thread per triangle over rows [r0, r1); partial sums per (row chunk, triangle):
// sum S1, sum S3, sum S3 x_i (3), dJ/dz_q (21).
constexpr int APART = 26;
__global__ void __launch_bounds__(128) k_adj_tri_pass(int M, int N, int rows_per_chunk, const double* __restrict__ rec,
                                                       const int* __restrict__ tri, const double* __restrict__ x,
                                                       const double* __restrict__ mu, const double* __restrict__ phi,
                                                       double* __restrict__ part) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int ch = blockIdx.y;
    if (t >= M) return;
    const int r0 = ch * rows_per_chunk, r1 = min(N, r0 + rows_per_chunk);
    const int ia = tri[3 * t], ib = tri[3 * t + 1], ic = tri[3 * t + 2];
    double rr[AREC];
#pragma unroll
    for (int k = 0; k < AREC; ++k) rr[k] = rec[(size_t)t * AREC + k];
    v3 zb[7];
#pragma unroll
    for (int q = 0; q < 7; ++q) zb[q] = {0.0, 0.0, 0.0};
    double s1 = 0.0, s3 = 0.0;
    v3 s3x = {0.0, 0.0, 0.0};
    for (int i = r0; i < r1; ++i) {
        if (i == ia || i == ib || i == ic) continue;  // singular pairs: k_adj_tri_final
        const v3 xi = ld(x, i);
        double S1, S3;
        pair_terms(rr, xi, mu[i], phi[i], S1, S3, zb);
        s1 += S1;
        s3 += S3;
        s3x = s3x + S3 * xi;
    }
    double* o = part + ((size_t)ch * M + t) * APART;
    o[0] = s1;
    o[1] = s3;
    o[2] = s3x.x;
    o[3] = s3x.y;
    o[4] = s3x.z;
#pragma unroll
    for (int q = 0; q < 7; ++q) {
        o[5 + 3 * q] = zb[q].x;
        o[6 + 3 * q] = zb[q].y;
        o[7 + 3 * q] = zb[q].z;
    }
}

// Row side: thread per row over triangles [t0, t1); xbar_i partial per (triangle chunk, row).
__global__ void __launch_bounds__(128) k_adj_row_pass(int N, int M, int tris_per_chunk, const double* __restrict__ rec,
                                                       const int* __restrict__ tri, const double* __restrict__ x,
                                                       const double* __restrict__ mu, const double* __restrict__ phi,
                                                       double* __restrict__ part) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int ch = blockIdx.y;
    if (i >= N) return;
    const int t0 = ch * tris_per_chunk, t1 = min(M, t0 + tris_per_chunk);
    const v3 xi = ld(x, i);
    const double m = mu[i], ph = phi[i];
    v3 acc = {0.0, 0.0, 0.0};
    for (int t = t0; t < t1; ++t) {
        if (i == tri[3 * t] || i == tri[3 * t + 1] || i == tri[3 * t + 2]) continue;
        const double* r = rec + (size_t)t * AREC;
        v3 zb[7];
#pragma unroll
        for (int q = 0; q < 7; ++q) zb[q] = {0.0, 0.0, 0.0};
        double S1, S3;
        pair_terms(r, xi, m, ph, S1, S3, zb);
        v3 zs = {0.0, 0.0, 0.0};
#pragma unroll
        for (int q = 0; q < 7; ++q) zs = zs + zb[q];
        const v3 Nv = {r[21], r[22], r[23]};
        acc = acc + (S3 * Nv - zs);
    }
    put3(part, ch * N + i, acc);
}

__global__ void k_adj_row_final(int N, int nch, const double* __restrict__ part, double* __restrict__ xbar) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    v3 s = {0.0, 0.0, 0.0};
    for (int c = 0; c < nch; ++c) s = s + ld(part, c * N + i);
    add3(xbar, i, s);
}

// Singular pair VJP: collocation vertex P0 of its own triangle (P0, P1, P2) (rotated as in the
// forward), G only:  J = (pi/8) |N| sum_q gamma_q / |cos_q ab + sin_q bc|,
// gamma_q = w_q (wg0 / cos + wg1 (cos - sin) / cos^2 + wg2 sin / cos^2),  wg_m = -mu_P0 psi_Pm.
__device__ void singular_vjp(v3 P0, v3 P1, v3 P2, double wg0, double wg1, double wg2, v3& b0, v3& b1, v3& b2) {
    const v3 ab = P1 - P0, bc = P2 - P1;
    const v3 N = cr(ab, bc);
    const double nrm = sqrt(dt3(N, N));
    const double k8 = 0.39269908169872415481;  // pi / 8
    double S = 0.0;
    v3 abb = {0.0, 0.0, 0.0}, bcb = {0.0, 0.0, 0.0};
#pragma unroll
    for (int q = 0; q < 7; ++q) {
        const double cx = a_gc[q], sx = a_gs[q];
        const double g = a_gw[q] * (wg0 / cx + wg1 * (cx - sx) / (cx * cx) + wg2 * sx / (cx * cx));
        const v3 D = cx * ab + sx * bc;
        const double d = sqrt(dt3(D, D));
        S += g / d;
        const v3 Db = (-k8 * nrm * g / (d * d * d)) * D;
        abb = abb + cx * Db;
        bcb = bcb + sx * Db;
    }
    const v3 Nb = (k8 * S / nrm) * N;
    cross_vjp(ab, bc, Nb, abb, bcb);
    b0 = b0 - abb;
    b1 = b1 + abb - bcb;
    b2 = b2 + bcb;
}

// Per triangle: the partial sums over row chunks in order, then the derivative with respect to its
// vertices a, b, c; plus its three singular pairs.  Output tb[t] = (abar, bbar, cbar) (overwritten).
__global__ void k_adj_tri_final(int M, int nch, const double* __restrict__ part, const double* __restrict__ rec,
                                const int* __restrict__ tri, const double* __restrict__ x,
                                const double* __restrict__ mu, const double* __restrict__ psi, double* __restrict__ tb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M) return;
    double s[APART];
#pragma unroll
    for (int k = 0; k < APART; ++k) s[k] = 0.0;
    for (int c = 0; c < nch; ++c) {
        const double* p = part + ((size_t)c * M + t) * APART;
#pragma unroll
        for (int k = 0; k < APART; ++k) s[k] += p[k];
    }
    const double* r = rec + (size_t)t * AREC;
    const int id[3] = {tri[3 * t], tri[3 * t + 1], tri[3 * t + 2]};
    const v3 A = ld(x, id[0]), B = ld(x, id[1]), C = ld(x, id[2]);
    const v3 ab = B - A, bc = C - B;
    const v3 N = {r[21], r[22], r[23]};
    const double nrm = r[24];
    // Nbar = (sum S1) N/|N| - (sum S3) a + sum S3 x_i
    const v3 Nb = ((s[0] / nrm) * N - s[1] * A) + v3{s[2], s[3], s[4]};
    v3 Ab = -s[1] * N, Bb = {0.0, 0.0, 0.0}, Cb = {0.0, 0.0, 0.0};
#pragma unroll
    for (int q = 0; q < 7; ++q) {
        const double u = a_quv[q][0], v = a_quv[q][1];
        const v3 z = {s[5 + 3 * q], s[6 + 3 * q], s[7 + 3 * q]};
        Ab = Ab + (1.0 - u) * z;
        Bb = Bb + (u - v) * z;
        Cb = Cb + v * z;
    }
    v3 abb = {0.0, 0.0, 0.0}, bcb = {0.0, 0.0, 0.0};
    cross_vjp(ab, bc, Nb, abb, bcb);
    Ab = Ab - abb;
    Bb = Bb + abb - bcb;
    Cb = Cb + bcb;
    // singular pairs: collocation vertex k, the triangle rotated to start there
    v3 out[3] = {Ab, Bb, Cb};
    const v3 P[3] = {A, B, C};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
        const double m = mu[id[k]];
        singular_vjp(P[k], P[k1], P[k2], -m * psi[id[k]], -m * psi[id[k1]], -m * psi[id[k2]], out[k], out[k1], out[k2]);
    }
    put3(tb, 3 * t, out[0]);
    put3(tb, 3 * t + 1, out[1]);
    put3(tb, 3 * t + 2, out[2]);
}

// ------------------------------------------------------------------------------------------------
// Pointwise stage derivatives
// ------------------------------------------------------------------------------------------------
// sum over the vertices of each loose part (one CTA per part, fixed order)
__global__ void k_part_sum(int N, const int* __restrict__ part, const double* __restrict__ v, double* __restrict__ out) {
    __shared__ double red[256];
    const int p = blockIdx.x;
    double s = 0.0;
    for (int i = threadIdx.x; i < N; i += 256)
        if (part[i] == p) s += v[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[p] = red[0];
}

// pot_t: vbar = kbar + kpbar_i v_i; xbar_i.x += kpbar_i A kx cos(kx x + w t + c)
__global__ void k_pot_vjp(int N, const double* __restrict__ x, const double* __restrict__ vel,
                          const double* __restrict__ kbar, const double* __restrict__ kpbar, const DevScalars* sc,
                          double famp, double fkx, double fomega, double fphase, double* __restrict__ vbar,
                          double* __restrict__ xbar) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double w = kpbar[i];
    put3(vbar, i, ld(kbar, i) + w * ld(vel, i));
    if (fkx != 0.0) xbar[3 * i] += w * famp * fkx * cos(fkx * x[3 * i] + fomega * sc->time + fphase);
}

// Volume term of pot_t through the part volumes: Vbar_p = S_p eps gamma (V0/V_p)^gamma / V_p with
// S_p the part's sum of kpbar; dV/da = (b x c)/6, dV/db = (c x a)/6, dV/dc = (a x b)/6.  With
// coef_only = 1: Vbar_p = 1 (the gradient of the volume itself).  tb[t] += contributions.
__global__ void k_vol_vjp(int M, const double* __restrict__ x, const int* __restrict__ tri,
                          const int* __restrict__ part, const double* __restrict__ vol, const double* __restrict__ S,
                          const DevScalars* __restrict__ sc, double eps_gas, double gamma, int coef_only,
                          double* __restrict__ tb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M) return;
    const int ia = tri[3 * t], ib = tri[3 * t + 1], ic = tri[3 * t + 2];
    const int p = part[ia];
    double vb = 1.0;
    if (!coef_only) {
        const double V = vol[p];
        vb = S[p] * eps_gas * gamma * pow(sc->V0 / V, gamma) / V;
    }
    const v3 A = ld(x, ia), B = ld(x, ib), C = ld(x, ic);
    const double f = vb / 6.0;
    add3(tb, 3 * t, f * cr(B, C));
    add3(tb, 3 * t + 1, f * cr(C, A));
    add3(tb, 3 * t + 2, f * cr(A, B));
}

// position_t, per vertex: psibar_i = (vbar_i / deg_i) . sum_t n_t; wv = (vbar_i / deg_i, psi_i vbar_i / deg_i)
__global__ void k_vel_vjp_vert(int N, const int* __restrict__ off, const int* __restrict__ idx,
                               const double* __restrict__ tn, const double* __restrict__ vbar,
                               const double* __restrict__ psi, double* __restrict__ wv, double* __restrict__ psibar) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    v3 sn = {0.0, 0.0, 0.0};
    for (int e = off[i]; e < off[i + 1]; ++e) sn = sn + ld(tn, idx[e]);
    const v3 w = (1.0 / (double)(off[i + 1] - off[i])) * ld(vbar, i);
    psibar[i] = dt3(w, sn);
    put3(wv, 2 * i, w);
    put3(wv, 2 * i + 1, psi[i] * w);
}

// position_t, per triangle: gbar = sum_k wv_k.0, nbar = sum_k wv_k.1, then the derivative of
// tn = m/|m| and g = s1 (m' x ab) + s2 (m' x bc), m = ab x bc, m' = m/|m|^2 (k_velocity_prep).
// tb[t] = (abar, bbar, cbar) (overwritten), tp[t] = (phibar_a, phibar_b, phibar_c).
__global__ void k_vel_vjp_tri(int M, const double* __restrict__ x, const int* __restrict__ tri,
                              const double* __restrict__ pot, const double* __restrict__ wv, double* __restrict__ tb,
                              double* __restrict__ tp) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M) return;
    const int ia = tri[3 * t], ib = tri[3 * t + 1], ic = tri[3 * t + 2];
    const v3 gb = (ld(wv, 2 * ia) + ld(wv, 2 * ib)) + ld(wv, 2 * ic);
    const v3 nb = (ld(wv, 2 * ia + 1) + ld(wv, 2 * ib + 1)) + ld(wv, 2 * ic + 1);
    const v3 A = ld(x, ia), B = ld(x, ib), C = ld(x, ic);
    const v3 ab = B - A, bc = C - B;
    const v3 m = cr(ab, bc);
    const double mm = dt3(m, m), mn = sqrt(mm);
    const v3 mp = (1.0 / mm) * m;
    const double s1 = pot[ic] - pot[ib], s2 = pot[ia] - pot[ib];
    const v3 u = cr(mp, ab), v = cr(mp, bc);
    const double s1b = dt3(gb, u), s2b = dt3(gb, v);
    v3 mpb = {0.0, 0.0, 0.0}, abb = {0.0, 0.0, 0.0}, bcb = {0.0, 0.0, 0.0};
    cross_vjp(mp, ab, s1 * gb, mpb, abb);
    cross_vjp(mp, bc, s2 * gb, mpb, bcb);
    // m' = m / |m|^2 and tn = m / |m|
    const v3 tn = (1.0 / mn) * m;
    v3 mb = (1.0 / mm) * mpb - (2.0 * dt3(m, mpb) / (mm * mm)) * m;
    mb = mb + (1.0 / mn) * (nb - dt3(tn, nb) * tn);
    cross_vjp(ab, bc, mb, abb, bcb);
    put3(tb, 3 * t, -1.0 * abb);
    put3(tb, 3 * t + 1, abb - bcb);
    put3(tb, 3 * t + 2, bcb);
    tp[3 * t] = s2b;
    tp[3 * t + 1] = -(s1b + s2b);
    tp[3 * t + 2] = s1b;
}

// triangle-corner contributions to vertices (through the incidence lists, fixed order)
__global__ void k_gather(int N, const int* __restrict__ off, const int* __restrict__ idx, const int* __restrict__ tri,
                         const double* __restrict__ tb, const double* __restrict__ tp, double* __restrict__ xbar,
                         double* __restrict__ pbar) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    v3 s = {0.0, 0.0, 0.0};
    double sp = 0.0;
    for (int e = off[i]; e < off[i + 1]; ++e) {
        const int t = idx[e];
        const int k = tri[3 * t] == i ? 0 : (tri[3 * t + 1] == i ? 1 : 2);
        s = s + ld(tb, 3 * t + k);
        if (tp) sp += tp[3 * t + k];
    }
    add3(xbar, i, s);
    if (pbar) pbar[i] += sp;
}

// y = cvec + sgn A^T x (A column-major n x n, T = double or float): one warp per column; part[b]:
// this CTA's sum of y_j^2 (optional).
template <typename T>
__global__ void __launch_bounds__(256) k_gemv_tcol(int n, const T* __restrict__ A, const double* __restrict__ x,
                                                   double* y, const double* cvec, double sgn, double* __restrict__ part) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int j = blockIdx.x * 8 + warp;
    double s = 0.0;
    if (j < n) {
        const T* col = A + (size_t)j * n;
        for (int i = lane; i < n; i += 32) s = fma((double)col[i], x[i], s);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ double sq[8];
    double yj = 0.0;
    if (j < n) {
        yj = cvec ? fma(sgn, s, cvec[j]) : s;
        if (lane == 0) y[j] = yj;
    }
    if (part) {
        if (lane == 0) sq[warp] = yj * yj;
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = 0.0;
            for (int w = 0; w < 8; ++w) a += sq[w];
            part[blockIdx.x] = a;
        }
    }
}

// RK4 reverse seeds: kbar_s = c_s dt xbar, kpbar_s = c_s dt pbar (c = 1/6, 1/3, 1/3, 1/6)
__global__ void k_rk4_seed(int N, double dt, const double* __restrict__ xb, const double* __restrict__ pb,
                           double* __restrict__ kb, double* __restrict__ kpb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double c[4] = {dt / 6.0, dt / 3.0, dt / 3.0, dt / 6.0};
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        for (int d = 0; d < 3; ++d) kb[(size_t)s * 3 * N + 3 * i + d] = c[s] * xb[3 * i + d];
        kpb[(size_t)s * N + i] = c[s] * pb[i];
    }
}
// after stage s: x1bar += xsbar, p1bar += psbar; k_{s-1}bar += h xsbar, kp_{s-1}bar += h psbar
__global__ void k_rk4_back(int N, double h, const double* __restrict__ xsb, const double* __restrict__ psb,
                           double* __restrict__ x1b, double* __restrict__ p1b, double* __restrict__ kprev,
                           double* __restrict__ kpprev) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    for (int d = 0; d < 3; ++d) {
        x1b[3 * i + d] += xsb[3 * i + d];
        if (kprev) kprev[3 * i + d] += h * xsb[3 * i + d];
    }
    p1b[i] += psb[i];
    if (kpprev) kpprev[i] += h * psb[i];
}
__global__ void k_stage_in(int n, const double* __restrict__ a, double h, const double* __restrict__ k,
                           double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = a[i] + h * k[i];
}
__global__ void k_any_below(int N, const double* __restrict__ x, double thr, int* flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N && x[3 * i] < thr) *flag = 1;
}

static inline int nbk(int64_t n, int t) { return (int)((n + t - 1) / t); }

// ------------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------------
static int adj_alloc(Ctx& c, int steps) {
    AdjWork& w = c.adj;
    const size_t N = (size_t)c.topo.N, M = (size_t)c.topo.M;
    if (w.N == (int64_t)N && w.cap >= steps) return BEM_OK;
    if (w.N != (int64_t)N) w = AdjWork{};  // buffers of an older mesh were freed with it
    const int cap = std::max(steps, w.cap);
    int rc;
    if ((rc = dalloc(c, &w.ckx, (size_t)cap * 3 * N)) || (rc = dalloc(c, &w.ckp, (size_t)cap * N)) ||
        (rc = dalloc(c, &w.ckt, (size_t)cap)))
        return rc;
    if (w.N != (int64_t)N) {
        // row chunks of the triangle pass and triangle chunks of the row pass: about four CTAs per SM
        // in each pass, at least 16 rows / triangles per chunk
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
        const int rch = std::max(1, std::min(nbk(4 * sms, nbk((int64_t)M, 128)), std::max(1, (int)N / 16)));
        const int tch = std::max(1, std::min(nbk(4 * sms, nbk((int64_t)N, 128)), std::max(1, (int)M / 16)));
        w.rch = rch;
        w.tch = tch;
        if ((rc = dalloc(c, &w.xs, 4 * 3 * N)) || (rc = dalloc(c, &w.ps, 4 * N)) || (rc = dalloc(c, &w.ks, 4 * 3 * N)) ||
            (rc = dalloc(c, &w.kps, 4 * N)) || (rc = dalloc(c, &w.psis, 4 * N)) || (rc = dalloc(c, &w.Gs, 4 * N * N)) ||
            (rc = dalloc(c, &w.Hs, 4 * N * N)) || (rc = dalloc(c, &w.kb, 4 * 3 * N)) || (rc = dalloc(c, &w.kpb, 4 * N)) ||
            (rc = dalloc(c, &w.xb, 3 * N)) || (rc = dalloc(c, &w.pb, N)) || (rc = dalloc(c, &w.xsb, 3 * N)) ||
            (rc = dalloc(c, &w.psb, N)) || (rc = dalloc(c, &w.vb, 3 * N)) || (rc = dalloc(c, &w.wv, 6 * N)) ||
            (rc = dalloc(c, &w.psib, N)) || (rc = dalloc(c, &w.mu, N)) || (rc = dalloc(c, &w.r, N)) ||
            (rc = dalloc(c, &w.tb, 9 * M)) || (rc = dalloc(c, &w.tp, 3 * M)) || (rc = dalloc(c, &w.rec, AREC * M)) ||
            (rc = dalloc(c, &w.partA, (size_t)rch * M * APART)) || (rc = dalloc(c, &w.partB, (size_t)tch * N * 3)) ||
            (rc = dalloc(c, &w.S, (size_t)c.topo.nparts + 1)) || (rc = dalloc(c, &w.red, (size_t)nbk(N, 8) * 16 + 64)) ||
            (rc = dalloc(c, &w.tsave, 2)) || (rc = dalloc(c, &w.iox, 3 * N)) || (rc = dalloc(c, &w.iop, N)))
            return rc;
    }
    w.N = (int64_t)N;
    w.cap = cap;
    return BEM_OK;
}

// mu = G^-T rhs by refinement mu <- mu + X^T (rhs - G^T mu) from mu = 0; the residual in FP64, the
// correction through the FP32 approximate inverse of the forward solves.
static int solve_transposed(Ctx& c, const double* G, const double* rhs, double* mu, cudaStream_t s) {
    AdjWork& w = c.adj;
    const int n = (int)c.topo.N;
    const int nb = nbk(n, 8);
    const double tol = c.prm.mixed_tol > 0 ? c.prm.mixed_tol : 1e-12;
    BEM_CUDA(c, cudaMemsetAsync(mu, 0, sizeof(double) * n, s));
    if (!c.xinv_valid) {  // forward solves by another solver: build the approximate inverse
        int rc = mixed_refresh(c, G, s, true);
        if (rc) return rc;
    }
    constexpr int K = 6;
    std::vector<double> h((size_t)(K + 2) * nb);
    double rel = 1.0;
    for (int round = 0; round < 6; ++round) {
        // residual norms of rhs (slot 0 of the first round: ||rhs||^2 via mu = 0) and of each step
        for (int k = 0; k <= K; ++k) {
            KLAUNCH(), k_gemv_tcol<double><<<nb, 256, 0, s>>>(n, G, mu, w.r, rhs, -1.0, w.red + (size_t)k * nb);
            if (k == K) break;
            KLAUNCH(), k_gemv_tcol<float><<<nb, 256, 0, s>>>(n, c.Xinv, w.r, mu, mu, 1.0, nullptr);
        }
        BEM_CUDA(c, cudaMemcpyAsync(h.data(), w.red, sizeof(double) * (size_t)(K + 1) * nb, cudaMemcpyDeviceToHost, s));
        BEM_CUDA(c, cudaStreamSynchronize(s));
        std::vector<double> rk((size_t)K + 1, 0.0);
        for (int k = 0; k <= K; ++k)
            for (int q = 0; q < nb; ++q) rk[(size_t)k] += h[(size_t)k * nb + q];
        if (round == 0) {
            w.bb = rk[0];
            if (w.bb == 0.0) return BEM_OK;
        }
        rel = sqrt(rk[K] / w.bb);
        if (rel <= tol) return BEM_OK;
        if (round == 1 || round == 3) {  // slow: refresh the approximate inverse against this G
            int rc = mixed_refresh(c, G, s, false);
            if (rc) return rc;
        }
    }
    return c.fail(BEM_ERR_NOT_CONVERGED, "adjoint: transposed solve did not reach the tolerance");
}

// forward stage s at (xs_s, ps_s): G_s, H_s, psi_s, k_s, kp_s
static int adj_stage_forward(Ctx& c, int st, cudaStream_t s) {
    AdjWork& w = c.adj;
    const int64_t N = c.topo.N;
    const double* xs = w.xs + 3 * N * st;
    const double* ps = w.ps + N * st;
    double* G = w.Gs + N * N * st;
    double* H = w.Hs + N * N * st;
    launch_assemble(c, xs, ps, G, H, c.b, s);
    int rc = solve_dev(c, G, c.b, c.psil, s);
    if (rc) return rc;
    BEM_CUDA(c, cudaMemcpyAsync(w.psis + N * st, c.psil, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
    launch_velocity_prep(c, xs, ps, s);
    launch_velocity(c, c.psil, w.ks + 3 * N * st, s);
    launch_pot_t(c, xs, w.ks + 3 * N * st, nullptr, w.kps + N * st, s);
    return BEM_OK;
}

// reverse of stage s: (kbar_s, kpbar_s) -> (xsbar, psbar)
static int adj_stage_reverse(Ctx& c, int st, cudaStream_t s) {
    AdjWork& w = c.adj;
    const int N = (int)c.topo.N, M = (int)c.topo.M;
    const Topology& T = c.topo;
    const double* xs = w.xs + 3 * (size_t)N * st;
    const double* ps = w.ps + (size_t)N * st;
    const double* vel = w.ks + 3 * (size_t)N * st;
    const double* psi = w.psis + (size_t)N * st;
    const double* G = w.Gs + (size_t)N * N * st;
    const double* H = w.Hs + (size_t)N * N * st;
    BEM_CUDA(c, cudaMemsetAsync(w.xsb, 0, sizeof(double) * 3 * N, s));
    BEM_CUDA(c, cudaMemsetAsync(w.psb, 0, sizeof(double) * N, s));
    // pot_t
    KLAUNCH(), k_pot_vjp<<<nbk(N, 128), 128, 0, s>>>(N, xs, vel, w.kb + 3 * (size_t)N * st, w.kpb + (size_t)N * st, c.sc,
                                                    c.prm.field_amp, c.prm.field_kx, c.prm.field_omega,
                                                    c.prm.field_phase, w.vb, w.xsb);
    launch_part_volumes(c, xs, c.vol, s);
    KLAUNCH(), k_part_sum<<<T.nparts, 256, 0, s>>>(N, T.part_of_vert, w.kpb + (size_t)N * st, w.S);
    // position_t: tangent gradients and normals at the stage
    launch_velocity_prep(c, xs, ps, s);
    KLAUNCH(), k_vel_vjp_vert<<<nbk(N, 128), 128, 0, s>>>(N, T.csr_off, T.csr_idx, c.tn, w.vb, psi, w.wv, w.psib);
    KLAUNCH(), k_vel_vjp_tri<<<nbk(M, 128), 128, 0, s>>>(M, xs, T.tri, ps, w.wv, w.tb, w.tp);
    KLAUNCH(), k_vol_vjp<<<nbk(M, 128), 128, 0, s>>>(M, xs, T.tri, T.part_of_vert, c.vol, w.S, c.sc, c.prm.epsilon,
                                                    c.prm.gamma, 0, w.tb);
    KLAUNCH(), k_gather<<<nbk(N, 128), 128, 0, s>>>(N, T.csr_off, T.csr_idx, T.tri, w.tb, w.tp, w.xsb, w.psb);
    // solve: mu = G^-T psibar; psbar += H^T mu
    int rc = solve_transposed(c, G, w.psib, w.mu, s);
    if (rc) return rc;
    KLAUNCH(), k_gemv_tcol<double><<<nbk(N, 8), 256, 0, s>>>(N, H, w.mu, w.psb, w.psb, 1.0, nullptr);
    // assembly derivative
    KLAUNCH(), k_adj_records<<<nbk(M, 128), 128, 0, s>>>(M, xs, T.tri, psi, ps, w.rec);
    const int rpc = nbk(N, w.rch), tpc = nbk(M, w.tch);
    KLAUNCH(), k_adj_tri_pass<<<dim3(nbk(M, 128), w.rch), 128, 0, s>>>(M, N, rpc, w.rec, T.tri, xs, w.mu, ps, w.partA);
    KLAUNCH(), k_adj_tri_final<<<nbk(M, 128), 128, 0, s>>>(M, w.rch, w.partA, w.rec, T.tri, xs, w.mu, psi, w.tb);
    KLAUNCH(), k_gather<<<nbk(N, 128), 128, 0, s>>>(N, T.csr_off, T.csr_idx, T.tri, w.tb, nullptr, w.xsb, nullptr);
    KLAUNCH(), k_adj_row_pass<<<dim3(nbk(N, 128), w.tch), 128, 0, s>>>(N, M, tpc, w.rec, T.tri, xs, w.mu, ps, w.partB);
    KLAUNCH(), k_adj_row_final<<<nbk(N, 128), 128, 0, s>>>(N, w.tch, w.partB, w.xsb);
    return BEM_OK;
}

static int adj_check_scope(Ctx& c) {
    if (c.batch) return c.fail(BEM_ERR_STATE, "adjoint: single systems only");
    if (c.prm.mirror) return c.fail(BEM_ERR_STATE, "adjoint: free-space bubbles only (no wall image)");
    if (c.prm.sigma != 0.0) return c.fail(BEM_ERR_STATE, "adjoint: sigma = 0 only");
    if (c.field_cb) return c.fail(BEM_ERR_STATE, "adjoint: device-evaluated field only");
    if (c.n_pin) return c.fail(BEM_ERR_STATE, "adjoint: no pinned vertices");
    return BEM_OK;
}

int adjoint_record(Ctx& c, double dt, int steps) {
    int rc = adj_check_scope(c);
    if (rc) return rc;
    if (steps < 1) return c.fail(BEM_ERR_ARG, "adjoint: steps >= 1");
    if ((rc = ensure_mixed(c)) || (rc = adj_alloc(c, steps))) return rc;
    upload_adj_constants();
    AdjWork& w = c.adj;
    cudaStream_t s = c.stream;
    const int64_t N = c.topo.N;
    int flag = 0;
    BEM_CUDA(c, cudaMemsetAsync(c.flag + 2, 0, sizeof(int), s));
    KLAUNCH(), k_any_below<<<nbk(N, 256), 256, 0, s>>>((int)N, c.x, c.prm.nopen_eps, c.flag + 2);
    BEM_CUDA(c, cudaMemcpyAsync(&flag, c.flag + 2, sizeof(int), cudaMemcpyDeviceToHost, s));
    BEM_CUDA(c, cudaStreamSynchronize(s));
    if (flag) {
        w.steps = 0;
        return c.fail(BEM_ERR_STATE, "adjoint: a vertex lies within the wall treatment's range (x < eps)");
    }
    for (int k = 0; k < steps; ++k) {
        BEM_CUDA(c, cudaMemcpyAsync(w.ckx + 3 * N * k, c.x, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, s));
        BEM_CUDA(c, cudaMemcpyAsync(w.ckp + N * k, c.phi, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
        BEM_CUDA(c, cudaMemcpyAsync(w.ckt + k, &c.sc->time, sizeof(double), cudaMemcpyDeviceToDevice, s));
        // the wall treatment (nopenetration) is not differentiated: every x must stay >= eps
        KLAUNCH(), k_any_below<<<nbk(N, 256), 256, 0, s>>>((int)N, c.x, c.prm.nopen_eps, c.flag + 2);
        if ((rc = rk4_step_dev(c, dt, s))) return rc;
    }
    KLAUNCH(), k_any_below<<<nbk(N, 256), 256, 0, s>>>((int)N, c.x, c.prm.nopen_eps, c.flag + 2);
    BEM_CUDA(c, cudaMemcpyAsync(&flag, c.flag + 2, sizeof(int), cudaMemcpyDeviceToHost, s));
    BEM_CUDA(c, cudaStreamSynchronize(s));
    w.steps = steps;
    w.dt = dt;
    if (flag) {
        w.steps = 0;
        return c.fail(BEM_ERR_STATE, "adjoint: a vertex came within the wall treatment's range (x < eps)");
    }
    return BEM_OK;
}

// xbar, pbar: device arrays (3N, N) on input the adjoint of the final state, on output of the initial.
int adjoint_backward(Ctx& c, double* xbar, double* pbar) {
    AdjWork& w = c.adj;
    if (w.steps < 1) return c.fail(BEM_ERR_STATE, "adjoint: no recorded trajectory");
    int rc = adj_check_scope(c);
    if (rc) return rc;
    cudaStream_t s = c.stream;
    const int64_t N = c.topo.N;
    const int n = (int)N;
    const double dt = w.dt;
    BEM_CUDA(c, cudaMemcpyAsync(w.tsave, &c.sc->time, sizeof(double), cudaMemcpyDeviceToDevice, s));
    BEM_CUDA(c, cudaMemcpyAsync(w.xb, xbar, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, s));
    BEM_CUDA(c, cudaMemcpyAsync(w.pb, pbar, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
    const double hs[4] = {0.0, 0.5, 0.5, 1.0};
    for (int k = w.steps - 1; k >= 0; --k) {
        // recompute the step's stages from its checkpoint
        BEM_CUDA(c, cudaMemcpyAsync(&c.sc->time, w.ckt + k, sizeof(double), cudaMemcpyDeviceToDevice, s));
        const double* x1 = w.ckx + 3 * N * k;
        const double* p1 = w.ckp + N * k;
        for (int st = 0; st < 4; ++st) {
            if (st == 0) {
                BEM_CUDA(c, cudaMemcpyAsync(w.xs, x1, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, s));
                BEM_CUDA(c, cudaMemcpyAsync(w.ps, p1, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
            } else {
                KLAUNCH(), k_stage_in<<<nbk(3 * N, 256), 256, 0, s>>>(3 * n, x1, hs[st] * dt, w.ks + 3 * N * (st - 1),
                                                                      w.xs + 3 * N * st);
                KLAUNCH(), k_stage_in<<<nbk(N, 256), 256, 0, s>>>(n, p1, hs[st] * dt, w.kps + N * (st - 1), w.ps + N * st);
            }
            if ((rc = adj_stage_forward(c, st, s))) return rc;
        }
        // reverse: seeds from (xbar, pbar), stages 4..1; x1bar, p1bar accumulate in xb, pb
        KLAUNCH(), k_rk4_seed<<<nbk(N, 128), 128, 0, s>>>(n, dt, w.xb, w.pb, w.kb, w.kpb);
        for (int st = 3; st >= 0; --st) {
            if ((rc = adj_stage_reverse(c, st, s))) return rc;
            KLAUNCH(), k_rk4_back<<<nbk(N, 128), 128, 0, s>>>(n, hs[st] * dt, w.xsb, w.psb, w.xb, w.pb,
                                                            st > 0 ? w.kb + 3 * N * (st - 1) : nullptr,
                                                            st > 0 ? w.kpb + N * (st - 1) : nullptr);
        }
    }
    BEM_CUDA(c, cudaMemcpyAsync(xbar, w.xb, sizeof(double) * 3 * N, cudaMemcpyDeviceToDevice, s));
    BEM_CUDA(c, cudaMemcpyAsync(pbar, w.pb, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
    BEM_CUDA(c, cudaMemcpyAsync(&c.sc->time, w.tsave, sizeof(double), cudaMemcpyDeviceToDevice, s));
    BEM_CUDA(c, cudaGetLastError());
    return BEM_OK;
}

// gradient of the total enclosed volume with respect to the vertices (xbar, device, overwritten)
int volume_gradient(Ctx& c, double* xbar) {
    const int N = (int)c.topo.N, M = (int)c.topo.M;
    int rc = adj_alloc(c, 1);
    if (rc) return rc;
    if (!xbar) xbar = c.adj.iox;
    cudaStream_t s = c.stream;
    BEM_CUDA(c, cudaMemsetAsync(c.adj.tb, 0, sizeof(double) * 9 * M, s));
    BEM_CUDA(c, cudaMemsetAsync(xbar, 0, sizeof(double) * 3 * N, s));
    KLAUNCH(), k_vol_vjp<<<nbk(M, 128), 128, 0, s>>>(M, c.x, c.topo.tri, c.topo.part_of_vert, c.vol, nullptr, c.sc, 0.0,
                                                    0.0, 1, c.adj.tb);
    KLAUNCH(), k_gather<<<nbk(N, 128), 128, 0, s>>>(N, c.topo.csr_off, c.topo.csr_idx, c.topo.tri, c.adj.tb, nullptr,
                                                    xbar, nullptr);
    return BEM_OK;
}

}  // namespace bemb
