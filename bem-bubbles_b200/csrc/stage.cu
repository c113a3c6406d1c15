// Per-stage pointwise work of LinLinSim (Bem/Simulation/LinLinSim.cpp) on the device:
// surface velocities (position_t), Bernoulli Dphi/Dt per bubble (pot_t_multi), vertex normals,
// adaptive dt, the RK4 / Euler combination and the wall treatment (nopenetration).
// All O(N) or O(M); memory-bound and tiny next to assembly and solve.
#include <math.h>

#include <algorithm>

#include "ctx.h"

namespace bemb {

struct d3 {
    double x, y, z;
};
__device__ __forceinline__ d3 ld3(const double* p, int i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ __forceinline__ void st3(double* p, int i, d3 v) {
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}
__device__ __forceinline__ d3 sub(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 cross(d3 a, d3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// generate_triangle_normals (Mesh.cpp:130-138) and generate_tangent_gradients (LinLinSim.cpp:288-305)
__global__ void k_velocity_prep(int M, const double* __restrict__ x, const int* __restrict__ tri,
                                const double* __restrict__ pot, double* __restrict__ tn, double* __restrict__ tg) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M) return;
    int a = tri[3 * t], b = tri[3 * t + 1], c = tri[3 * t + 2];
    d3 A = ld3(x, a), B = ld3(x, b), C = ld3(x, c);
    d3 n = cross(sub(B, A), sub(C, A));
    double inv = 1.0 / sqrt(dot(n, n));
    st3(tn, t, {n.x * inv, n.y * inv, n.z * inv});
    d3 ab = sub(B, A), bc = sub(C, B);
    d3 m = cross(ab, bc);
    double i2 = 1.0 / dot(m, m);
    m = {m.x * i2, m.y * i2, m.z * i2};
    double s1 = pot[c] - pot[b], s2 = pot[a] - pot[b];
    d3 u = cross(m, ab), v = cross(m, bc);
    st3(tg, t, {s1 * u.x + s2 * v.x, s1 * u.y + s2 * v.y, s1 * u.z + s2 * v.z});
}

// vertex gradient = mean over incident triangles of (tangent gradient + psi_i * normal)
// (LinLinSim.cpp:48-59)
// hist (may be null): the stage predictor's history row that receives psil, with the stage time
// t + c_s dt in *htime (one launch for both).
__global__ void k_velocity(int N, const int* __restrict__ off, const int* __restrict__ idx,
                           const double* __restrict__ tn, const double* __restrict__ tg,
                           const double* __restrict__ psil, double* __restrict__ vel, double* __restrict__ hist,
                           double* __restrict__ htime, double cs, const DevScalars* __restrict__ sc) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (hist && i == 0) *htime = sc->time + cs * sc->dt;
    if (i >= N) return;
    if (hist) hist[i] = psil[i];
    double gx = 0, gy = 0, gz = 0, num = 0;
    const double p = psil[i];
    for (int e = off[i]; e < off[i + 1]; ++e) {
        int t = idx[e];
        gx += tg[3 * t] + p * tn[3 * t];
        gy += tg[3 * t + 1] + p * tn[3 * t + 1];
        gz += tg[3 * t + 2] + p * tn[3 * t + 2];
        num += 1.0;
    }
    double s = 1.0 / num;
    st3(vel, i, {gx * s, gy * s, gz * s});
}

// Part volumes (Mesh.cpp:206-218), sum over the part's triangles of (a x b).c / 6, in two levels
// with a fixed shape: CTA (chunk, part) sums VOL_CHUNK consecutive triangles of the part's list by a
// tree; the last CTA of the part (completion counter) adds the chunk sums in chunk order.
constexpr int VOL_CHUNK = 256, VOL_MAXCH = 64;  // about one triangle per thread: the sum is latency-bound
__global__ void __launch_bounds__(256) k_part_volume(const double* __restrict__ x, const int* __restrict__ off,
                                                     const int* __restrict__ tidx, const int* __restrict__ ptri,
                                                     double* __restrict__ part_sums, unsigned* __restrict__ cnt,
                                                     double* __restrict__ vol) {
    __shared__ double red[256];
    __shared__ unsigned s_ticket;
    const int p = blockIdx.y, ch = blockIdx.x;
    const int b0 = off[p], b1 = off[p + 1];
    const int nch = min(VOL_MAXCH, max(1, (b1 - b0 + VOL_CHUNK - 1) / VOL_CHUNK));
    const int per = (b1 - b0 + nch - 1) / nch;  // triangles per chunk of this part
    if (ch >= nch) return;
    const int e0 = b0 + ch * per, e1 = min(b1, e0 + per);
    double acc = 0.0;
    for (int e = e0 + threadIdx.x; e < e1; e += 256) {
        const int t = tidx[e];
        d3 a = ld3(x, ptri[3 * t]), b = ld3(x, ptri[3 * t + 1]), c = ld3(x, ptri[3 * t + 2]);
        acc += dot(cross(a, b), c) / 6.0;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part_sums[(size_t)p * VOL_MAXCH + ch] = red[0];
        __threadfence();
        s_ticket = atomicAdd(&cnt[p], 1u);
    }
    __syncthreads();
    if (s_ticket != (unsigned)(nch - 1) || threadIdx.x != 0) return;
    __threadfence();
    double v = 0.0;
    for (int k = 0; k < nch; ++k) v += __ldcg(part_sums + (size_t)p * VOL_MAXCH + k);
    vol[p] = v;
    cnt[p] = 0u;
}

// potential_t (Simulation.cpp:73-75) per vertex:
// 2 sigma kappa + |grad|^2/2 + p_inf - epsilon (V0/V_part)^gamma + p_field(x, t_stepstart)
// ppar (optional, batches of independent bubbles): per part {V0, amp, kx, omega, phase} in place of
// the shared V0 and field parameters.
__global__ void k_pot_t(int N, const double* __restrict__ x, const double* __restrict__ vel,
                        const int* __restrict__ part, const double* __restrict__ vol,
                        const double* __restrict__ kap, const double* __restrict__ fieldv,
                        const DevScalars* __restrict__ sc, double p_inf, double eps_gas, double sigma,
                        double gamma, double famp, double fkx, double fomega, double fphase, double t_host,
                        int use_dev_time, const double* __restrict__ ppar, double* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    d3 g = ld3(vel, i);
    const int p = part[i];
    double V = vol[p];
    double t = use_dev_time ? sc->time : t_host;
    double V0 = sc->V0;
    if (ppar) {
        const double* q = ppar + 5 * p;
        V0 = q[0];
        famp = q[1];
        fkx = q[2];
        fomega = q[3];
        fphase = q[4];
    }
    double f;
    if (fieldv)
        f = fieldv[i];
    else
        f = famp * sin(fkx * x[3 * i] + fomega * t + fphase);
    double k = kap ? kap[i] : 0.0;
    out[i] = 2.0 * sigma * k + 0.5 * dot(g, g) + p_inf - eps_gas * pow(V0 / V, gamma) + f;
}

// out = a + (coef * scale) * k, coef from device memory (the step dt), elementwise.
// The positions and the potential of an RK4 stage in one launch: xs = x1 + scale dt kx (3N),
// ps = p1 + scale dt kp (N).
__global__ void k_axpy_stage(int N, const double* __restrict__ x1, const double* __restrict__ kx,
                             double* __restrict__ xs, const double* __restrict__ p1, const double* __restrict__ kp,
                             double* __restrict__ ps, const double* __restrict__ coef, double scale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double h = scale * *coef;
    if (i < 3 * N)
        xs[i] = x1[i] + h * kx[i];
    else if (i < 4 * N)
        ps[i - 3 * N] = p1[i - 3 * N] + h * kp[i - 3 * N];
}

// RK4 combination, phi update and nopenetration (LinLinSim.cpp:236-253, 162-190).
// avg = (k1 + 2k2 + 2k3 + k4)/6 is left in k1 for the psi update.
__global__ void k_rk4_final(int N, const double* __restrict__ x1, double* __restrict__ k1,
                            const double* __restrict__ k2, const double* __restrict__ k3,
                            const double* __restrict__ k4, const double* __restrict__ p1,
                            const double* __restrict__ q1, const double* __restrict__ q2,
                            const double* __restrict__ q3, const double* __restrict__ q4,
                            DevScalars* __restrict__ sc, double eps, double* __restrict__ x,
                            double* __restrict__ phi, const int* __restrict__ skip) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N || (skip && *skip)) return;
    const double dt = sc->dt;
    double av[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        int j = 3 * i + c;
        av[c] = (((k1[j] + 2.0 * k2[j]) + 2.0 * k3[j]) + k4[j]) * (1.0 / 6.0);
        x[j] = x1[j] + dt * av[c];
    }
    phi[i] = p1[i] + (dt / 6.0) * (((q1[i] + 2.0 * q2[i]) + 2.0 * q3[i]) + q4[i]);
    double cx = av[0];
    if (cx * dt < 0.0) {
        bool flag = false;
        double xpos = x1[3 * i];
        if (xpos < eps) {
            x[3 * i] = xpos * exp(cx / xpos * dt);
            flag = true;
        } else {
            double te = (eps - xpos) / cx;
            if (fabs(te) < fabs(dt)) {
                x[3 * i] = eps * exp(cx / eps * (dt - te));
                flag = true;
            }
        }
        if (flag) av[0] = (x[3 * i] - xpos) / dt;
    }
    k1[3 * i] = av[0];
    k1[3 * i + 1] = av[1];
    k1[3 * i + 2] = av[2];
}

__global__ void k_psi_from_avg(int N, const double* __restrict__ avg, const double* __restrict__ vn,
                               double* __restrict__ psi, DevScalars* __restrict__ sc, const int* __restrict__ skip) {
    if (skip && *skip) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) sc->time += sc->dt;
    if (i >= N) return;
    psi[i] = avg[3 * i] * vn[3 * i] + avg[3 * i + 1] * vn[3 * i + 1] + avg[3 * i + 2] * vn[3 * i + 2];
}

__global__ void k_euler_final(int N, const double* __restrict__ vel, const double* __restrict__ potd,
                              DevScalars* __restrict__ sc, double* __restrict__ x, double* __restrict__ phi) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double dt = sc->dt;
    if (i < N) {
        for (int c = 0; c < 3; ++c) x[3 * i + c] = x[3 * i + c] + vel[3 * i + c] * dt;
        phi[i] = phi[i] + dt * potd[i];
    }
}

__global__ void k_euler_time(DevScalars* sc) { sc->time += sc->dt; }

// Simulation::get_dt (Simulation.cpp:77-92): one CTA, deterministic max-reductions.
__global__ void k_get_dt(int N, const double* __restrict__ vel, const double* __restrict__ potd, double dp,
                         double dp_balance, double min_dt, DevScalars* __restrict__ sc) {
    __shared__ double mp[1024], mv[1024];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        a = fmax(fabs(potd[i]), a);
        d3 v = ld3(vel, i);
        b = fmax(dot(v, v), b);
    }
    mp[threadIdx.x] = a;
    mv[threadIdx.x] = b;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            mp[threadIdx.x] = fmax(mp[threadIdx.x], mp[threadIdx.x + w]);
            mv[threadIdx.x] = fmax(mv[threadIdx.x], mv[threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double dt = dp / (mp[0] + dp_balance * sqrt(mv[0]));
        if (min_dt > 0.0) dt = fmin(dt, min_dt);
        sc->dt = dt;
    }
}

__global__ void k_any_negative(int N, const double* __restrict__ x, int* flag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N && x[3 * i] < 0.0) *flag = 1;
}

static inline int nb(int64_t n, int t) { return (int)((n + t - 1) / t); }

void launch_velocity_prep(Ctx& c, const double* x, const double* pot, cudaStream_t s) {
    KLAUNCH(), k_velocity_prep<<<nb(c.topo.M, 128), 128, 0, s>>>((int)c.topo.M, x, c.topo.tri, pot, c.tn, c.tg);
}
// ring row of stage `stage` in the step `back` steps before the current one (back = 0: the current)
static int pred_row(const Ctx& c, int back, int stage) {
    return ((c.pred_head - back + 2 * PRED_DEPTH) % PRED_DEPTH) * 4 + stage;
}

// The current step's history row of stage `stage`, its time slot and the stage's offset c_s.
static void stage_history_row(Ctx& c, int stage, double** hist, double** htime, double* cs) {
    static const double stage_c[4] = {0.0, 0.5, 0.5, 1.0};
    const int row = pred_row(c, 0, stage);
    *hist = c.psih + (size_t)row * c.topo.N;
    *htime = c.psih_t + row;
    *cs = stage_c[stage];
}

void launch_velocity(Ctx& c, const double* psil, double* vel, cudaStream_t s, int stage) {
    double *hist = nullptr, *htime = nullptr;
    double cs = 0.0;
    if (stage >= 0) stage_history_row(c, stage, &hist, &htime, &cs);
    KLAUNCH(), k_velocity<<<nb(c.topo.N, 128), 128, 0, s>>>((int)c.topo.N, c.topo.csr_off, c.topo.csr_idx, c.tn, c.tg, psil,
                                                            vel, hist, htime, cs, c.sc);
}
void launch_part_volumes(Ctx& c, const double* x, double* vol, cudaStream_t s) {
    // chunks per part: enough for the largest part (the kernel exits early in smaller parts)
    const int nch = std::min(VOL_MAXCH, std::max(1, (c.topo.max_part_tris + VOL_CHUNK - 1) / VOL_CHUNK));
    dim3 grid(nch, c.topo.nparts);
    KLAUNCH(), k_part_volume<<<grid, 256, 0, s>>>(x, c.topo.part_off, c.topo.part_tidx, c.topo.tri_rot, c.vol_part,
                                                 c.vol_cnt, vol);
}
void launch_pot_t(Ctx& c, const double* x, const double* vel, const double* field_dev, double* out,
                  cudaStream_t s) {
    launch_part_volumes(c, x, c.vol, s);
    const double* kap = nullptr;
    if (c.prm.sigma != 0.0) {
        launch_curvature(c, x, c.kap, s);
        kap = c.kap;
    }
    KLAUNCH(), k_pot_t<<<nb(c.topo.N, 128), 128, 0, s>>>((int)c.topo.N, x, vel, c.topo.part_of_vert, c.vol, kap, field_dev,
                                               c.sc, c.prm.p_inf, c.prm.epsilon, c.prm.sigma, c.prm.gamma,
                                               c.prm.field_amp, c.prm.field_kx, c.prm.field_omega,
                                               c.prm.field_phase, 0.0, 1, c.ppar, out);
}
void launch_axpy_stage(Ctx& c, const double* kx, const double* kp, const double* coef_dev, double scale,
                       cudaStream_t s) {
    const int N = (int)c.topo.N;
    KLAUNCH(), k_axpy_stage<<<nb(4 * (int64_t)N, 256), 256, 0, s>>>(N, c.x1, kx, c.xs, c.p1, kp, c.ps, coef_dev, scale);
}
// skip (device flag, may be null): when set, the step leaves x, phi, psi and time untouched
void launch_rk4_final(Ctx& c, cudaStream_t s, const int* skip) {
    const int N = (int)c.topo.N;
    KLAUNCH(), k_rk4_final<<<nb(N, 128), 128, 0, s>>>(N, c.x1, c.k1, c.k2, c.k3, c.k4, c.p1, c.kp1, c.kp2, c.kp3, c.kp4, c.sc,
                                           c.prm.nopen_eps, c.x, c.phi, skip);
    launch_vertex_normals(c, c.x, c.vn, s);
    KLAUNCH(), k_psi_from_avg<<<nb(N, 128), 128, 0, s>>>(N, c.k1, c.vn, c.psi, c.sc, skip);
}
void launch_euler_final(Ctx& c, const double* vel, const double* potd, cudaStream_t s) {
    const int N = (int)c.topo.N;
    KLAUNCH(), k_euler_final<<<nb(N, 128), 128, 0, s>>>(N, vel, potd, c.sc, c.x, c.phi);
    KLAUNCH(), k_euler_time<<<1, 1, 0, s>>>(c.sc);
}
// ---------------------------------------------------------------- stage predictor (mixed solve)
// RK4 stage times relative to the step: t + c_s dt.
__constant__ double c_stage_c[4] = {0.0, 0.5, 0.5, 1.0};

// Start value of a stage solve: Lagrange extrapolation in time from the same stage of the last m
// steps (rows r0 newest, r1, r2 of the ring hist, times ht), x = sum_j w_j hist_j with
// w_j = prod_{k != j} (T - T_k) / (T_j - T_k) and T = t + c_s dt the stage's time.  m is the number
// of steps in the ring that continue the current trajectory (ht[PRED_CNT]); with none, x keeps the
// previous stage's solution.  Coinciding times or weights above 16 in magnitude (a step much longer
// than the history's) fall back to the newest value alone.  The refinement converges to the same
// FP64 solution from any start; a start whose error is O(dt^m) instead of the previous stage's
// O(dt) saves refinement steps.
__global__ void k_stage_predict(int N, const double* __restrict__ hist, const double* __restrict__ ht, int r0, int r1,
                                int r2, int stage, const DevScalars* __restrict__ sc, double* __restrict__ x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = min(PRED_DEPTH, (int)ht[PRED_CNT]);
    if (i >= N || m < 1) return;
    const double T = sc->time + c_stage_c[stage] * sc->dt;
    const int rows[3] = {r0, r1, r2};
    double Tk[3] = {0.0, 0.0, 0.0}, w[3] = {1.0, 0.0, 0.0};
    for (int j = 0; j < m; ++j) Tk[j] = ht[rows[j]];
    bool ok = true;
    for (int j = 0; j < m; ++j) {
        double wj = 1.0;
        for (int k = 0; k < m; ++k) {
            if (k == j) continue;
            const double d = Tk[j] - Tk[k];
            if (d == 0.0) ok = false;
            wj *= (T - Tk[k]) / d;
        }
        w[j] = wj;
        if (!(fabs(wj) <= 16.0)) ok = false;
    }
    if (!ok || m < 2) {
        x[i] = hist[(size_t)r0 * N + i];
        return;
    }
    double v = w[0] * hist[(size_t)r0 * N + i];
    for (int j = 1; j < m; ++j) v = fma(w[j], hist[(size_t)rows[j] * N + i], v);
    x[i] = v;
}

// End of a step: one more step in the ring, or none when the step's final update was skipped.
__global__ void k_stage_advance(double* ht, const int* skip) {
    ht[PRED_CNT] = (skip && *skip) ? 0.0 : fmin(ht[PRED_CNT] + 1.0, (double)PRED_DEPTH);
}

// dst <- src; a value that differs from the one held ends the predictor's trajectory.
__global__ void k_state_accept(int64_t n, const double* __restrict__ src, double* __restrict__ dst, double* ht) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = src[i];
        if (!(v == dst[i]) && ht) ht[PRED_CNT] = 0.0;
        dst[i] = v;
    }
}
__global__ void k_time_accept(double t, DevScalars* sc, double* ht) {
    if (!(t == sc->time) && ht) ht[PRED_CNT] = 0.0;
    sc->time = t;
}


void launch_stage_predict(Ctx& c, int stage, double* x, cudaStream_t s) {
    const int N = (int)c.topo.N;
    KLAUNCH(), k_stage_predict<<<nb(N, 256), 256, 0, s>>>(N, c.psih, c.psih_t, pred_row(c, 1, stage),
                                                          pred_row(c, 2, stage), pred_row(c, 3, stage), stage, c.sc, x);
}

void launch_stage_advance(Ctx& c, const int* skip, cudaStream_t s) {
    KLAUNCH(), k_stage_advance<<<1, 1, 0, s>>>(c.psih_t, skip);
    c.pred_head = (c.pred_head + 1) % PRED_DEPTH;
}

void launch_state_accept(Ctx& c, int64_t n, const double* src, double* dst, cudaStream_t s) {
    KLAUNCH(), k_state_accept<<<(int)std::min<int64_t>(nb(n, 256), 1184), 256, 0, s>>>(n, src, dst, c.psih_t);
}

void launch_time_accept(Ctx& c, double t, cudaStream_t s) {
    KLAUNCH(), k_time_accept<<<1, 1, 0, s>>>(t, c.sc, c.psih_t);
}

void launch_get_dt(Ctx& c, const double* vel, const double* potd, double dp, cudaStream_t s) {
    KLAUNCH(), k_get_dt<<<1, 1024, 0, s>>>((int)c.topo.N, vel, potd, dp, c.prm.dp_balance, c.prm.min_dt, c.sc);
}
void launch_any_negative(Ctx& c, const double* x, int* flag, cudaStream_t s) {
    KLAUNCH(), k_any_negative<<<nb(c.topo.N, 256), 256, 0, s>>>((int)c.topo.N, x, flag);
}

}  // namespace bemb
