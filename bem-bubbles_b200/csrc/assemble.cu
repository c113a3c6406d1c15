// Dense collocation assembly of G (single layer) and H (double layer) in FP64.
//
// Replaces ColocSim::assemble_matrices (Bem/Simulation/ColocSim.cpp:21-110) with the per-pair
// integrals of Integrator::integrate_Lin_coloc_local[_mir] (Bem/Integration/Integrator.cpp:237-283):
//   * regular pairs (vertex i not on triangle t): 7-point rule on the triangle
//     (integrate_disjoint_coloc[_mir], Integrator.hpp:471-513, kernel Integrator.hpp:116-119);
//   * singular pairs (i on t): polar rule with the analytic radial integral and 7-point Gauss in
//     the angle (integrate_identical_coloc[_mir], Integrator.cpp:13-89);
//   * the "4 pi rule" diagonal H(i,i) -= 4 pi + sum_j H(i,j) (ColocSim.cpp:85-97);
//   * the right-hand side b = H phi of position_t (LinLinSim.cpp:32), fused.
//
// Tiling (B200): one CTA owns R complete rows (collocation points) of G and H in shared memory
// (R*N*16 bytes, up to 225 KB) and walks every triangle exactly once.  Triangles are split into
// colour classes in which no two triangles share a vertex, so the threads of a colour scatter
// their three basis contributions into the shared rows without conflicts or atomics; one barrier
// separates colours.  Each thread evaluates its triangle's 7 quadrature points for all R rows (7R
// independent chains).  Triangle records are field-major so every warp load is one coalesced
// 256-byte line.  The epilogue reduces each row in a fixed order (row sum for the 4 pi rule,
// H.phi), fixes the diagonal and writes the rows contiguously: G and H are stored row-major.
// Nothing is evaluated twice and the result is bit-reproducible run to run.  Meshes too large for
// full rows in shared memory are split into column chunks (grid.y), finished by k_finish_rows.
#include <math.h>

#include <algorithm>

#include "ctx.h"

namespace bemb {

// c[q][k] = w_q * basis_k(u_q, v_q) for the 7-point rule mapped to the 45-degree unit triangle
// (u, v) = (qx + qy, qy), basis (1-u, u-v, v) (ResultTypes.hpp:111-117); u_q, v_q; Gauss-7 angle data.
__constant__ double c_qc[7][3];
__constant__ double c_quv[7][2];
__constant__ double c_gcos[7], c_gsin[7], c_gw[7];

// Reference tables (quadrature.hpp:30-38 gauss_7, :88-96 quadrature_7), evaluated on the host once.
static void upload_constants() {
    static bool done = false;
    if (done) return;
    const double Q[7][3] = {{0.33333333333333333, 0.33333333333333333, 0.22500000000000000 * 0.5},
                            {0.79742698535308720, 0.10128650732345633, 0.12593918054482717 * 0.5},
                            {0.10128650732345633, 0.79742698535308720, 0.12593918054482717 * 0.5},
                            {0.10128650732345633, 0.10128650732345633, 0.12593918054482717 * 0.5},
                            {0.05971587178976981, 0.47014206410511505, 0.13239415278850616 * 0.5},
                            {0.47014206410511505, 0.05971587178976981, 0.13239415278850616 * 0.5},
                            {0.47014206410511505, 0.47014206410511505, 0.13239415278850616 * 0.5}};
    const double GL[7][2] = {{0.5 * (1.0 + 0.0000000000000000), 0.5 * 0.4179591836734694},
                             {0.5 * (1.0 + 0.4058451513773972), 0.5 * 0.3818300505051189},
                             {0.5 * (1.0 - 0.4058451513773972), 0.5 * 0.3818300505051189},
                             {0.5 * (1.0 - 0.7415311855993945), 0.5 * 0.2797053914892766},
                             {0.5 * (1.0 + 0.7415311855993945), 0.5 * 0.2797053914892766},
                             {0.5 * (1.0 - 0.9491079123427585), 0.5 * 0.1294849661688697},
                             {0.5 * (1.0 + 0.9491079123427585), 0.5 * 0.1294849661688697}};
    double qc[7][3], quv[7][2], gc[7], gs[7], gw[7];
    for (int q = 0; q < 7; ++q) {
        double u = Q[q][0] + Q[q][1], v = Q[q][1], w = Q[q][2];
        quv[q][0] = u;
        quv[q][1] = v;
        qc[q][0] = (1.0 - u) * w;
        qc[q][1] = (u - v) * w;
        qc[q][2] = v * w;
        double th = GL[q][0] * 0.78539816339744830962;
        gc[q] = cos(th);
        gs[q] = sin(th);
        gw[q] = GL[q][1];
    }
    cudaMemcpyToSymbol(c_qc, qc, sizeof(qc));
    cudaMemcpyToSymbol(c_quv, quv, sizeof(quv));
    cudaMemcpyToSymbol(c_gcos, gc, sizeof(gc));
    cudaMemcpyToSymbol(c_gsin, gs, sizeof(gs));
    cudaMemcpyToSymbol(c_gw, gw, sizeof(gw));
    done = true;
}

// Per-entry triangle record, field-major (rec[f*E + e]): Interpolator (Interpolator.hpp:15-37)
// quantities, the 7 quadrature points y_q = a + u_q*ab + v_q*bc and the plane offset n.a.
__global__ void k_triangle_records(int64_t E, const double* __restrict__ x, const int4* __restrict__ ent,
                                   double* __restrict__ rec) {
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    const int4 t = ent[e];
    const int ia = t.y, ib = t.z, ic = t.w;
    double ax = x[3 * ia], ay = x[3 * ia + 1], az = x[3 * ia + 2];
    double abx = x[3 * ib] - ax, aby = x[3 * ib + 1] - ay, abz = x[3 * ib + 2] - az;
    double bcx = x[3 * ic] - x[3 * ib], bcy = x[3 * ic + 1] - x[3 * ib + 1], bcz = x[3 * ic + 2] - x[3 * ib + 2];
    double nx = aby * bcz - abz * bcy, ny = abz * bcx - abx * bcz, nz = abx * bcy - aby * bcx;
    double area = sqrt(nx * nx + ny * ny + nz * nz);
    double ia_ = 1.0 / area;
#pragma unroll
    for (int q = 0; q < 7; ++q) {
        double u = c_quv[q][0], v = c_quv[q][1];
        rec[(3 * q + 0) * E + e] = (ax + u * abx) + v * bcx;
        rec[(3 * q + 1) * E + e] = (ay + u * aby) + v * bcy;
        rec[(3 * q + 2) * E + e] = (az + u * abz) + v * bcz;
    }
    const double unx = nx * ia_, uny = ny * ia_, unz = nz * ia_;
    rec[21 * E + e] = unx;
    rec[22 * E + e] = uny;
    rec[23 * E + e] = unz;
    rec[24 * E + e] = area;
    // every quadrature point y_q satisfies y_q.n = a.n, so (y_q - x).n is one number per pair
    rec[25 * E + e] = ax * unx + ay * uny + az * unz;
}

// 1/sqrt(r2) for r2 > 0 in FP64: the hardware's approximate reciprocal square root
// (rsqrt.approx.ftz.f64) refined by the binomial series of (1-d)^(-1/2) = 1 + d/2 + 3d^2/8 + ...
// with d = 1 - r2*y0^2; the truncation error 5d^3/16 is far below the double rounding unit.
__device__ __forceinline__ double rsqrt_fp64(double r2) {
    double y0;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y0) : "d"(r2));
    const double t = r2 * y0;
    const double d = fma(-t, y0, 1.0);
    const double p = fma(0.375, d, 0.5);
    return fma(y0, d * p, y0);
}

// Singular pair: row i is vertex `shift` of triangle (ta, tb, tc).  Results in the triangle's
// original vertex order.  Reads the vertex positions from global memory (rare path).
template <bool MIRROR>
__device__ __noinline__ void singular_pair(const double* __restrict__ x, int ta, int tb, int tc, int shift,
                                           double& g0, double& g1, double& g2, double& h0, double& h1,
                                           double& h2) {
    int v[3] = {ta, tb, tc};
    int r0 = v[shift], r1 = v[(shift + 1) % 3], r2 = v[(shift + 2) % 3];
    double ax = x[3 * r0], ay = x[3 * r0 + 1], az = x[3 * r0 + 2];
    double abx = x[3 * r1] - ax, aby = x[3 * r1 + 1] - ay, abz = x[3 * r1 + 2] - az;
    double bcx = x[3 * r2] - x[3 * r1], bcy = x[3 * r2 + 1] - x[3 * r1 + 1], bcz = x[3 * r2 + 2] - x[3 * r1 + 2];
    double nx = aby * bcz - abz * bcy, ny = abz * bcx - abx * bcz, nz = abx * bcy - aby * bcx;
    double area = sqrt(nx * nx + ny * ny + nz * nz);
    double jac = 0.5 * area * 0.78539816339744830962;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
    for (int q = 0; q < 7; ++q) {
        double cx = c_gcos[q], sx = c_gsin[q];
        double dx = cx * abx + sx * bcx, dy = cx * aby + sx * bcy, dz = cx * abz + sx * bcz;
        double dist = sqrt(dx * dx + dy * dy + dz * dz);
        double of = jac * c_gw[q] / dist;
        double fac = 1.0 / (cx * cx);
        s0 += of * cx * fac;
        s1 += of * (cx - sx) * fac;
        s2 += of * sx * fac;
    }
    double rg[3] = {s0, s1, s2}, rh[3] = {0.0, 0.0, 0.0};
    if (MIRROR) {
        // regular rule over the mirrored own triangle, plain kernel, H sign flipped (Integrator.cpp:70-86)
        double bx = ax + abx, by = ay + aby, bz = az + abz;
        double cxp = bx + bcx, cyp = by + bcy, czp = bz + bcz;
        double max_ = -ax, mbx = -bx, mcx = -cxp;
        double mabx = mbx - max_, maby = by - ay, mabz = bz - az;
        double mbcx = mcx - mbx, mbcy = cyp - by, mbcz = czp - bz;
        double mnx = maby * mbcz - mabz * mbcy, mny = mabz * mbcx - mabx * mbcz, mnz = mabx * mbcy - maby * mbcx;
        double marea = sqrt(mnx * mnx + mny * mny + mnz * mnz);
        double mi = 1.0 / marea;
        mnx *= mi;
        mny *= mi;
        mnz *= mi;
        double a0 = 0, a1 = 0, a2 = 0, b0 = 0, b1 = 0, b2 = 0;
#pragma unroll
        for (int q = 0; q < 7; ++q) {
            double u = c_quv[q][0], w = c_quv[q][1];
            double zx = (max_ + u * mabx) + w * mbcx - ax;
            double zy = (ay + u * maby) + w * mbcy - ay;
            double zz = (az + u * mabz) + w * mbcz - az;
            double inv = 1.0 / sqrt(zx * zx + zy * zy + zz * zz);
            double hq = -(zx * mnx + zy * mny + zz * mnz) * inv * inv * inv;
            a0 += c_qc[q][0] * inv;
            a1 += c_qc[q][1] * inv;
            a2 += c_qc[q][2] * inv;
            b0 += c_qc[q][0] * hq;
            b1 += c_qc[q][1] * hq;
            b2 += c_qc[q][2] * hq;
        }
        rg[0] += a0 * marea;
        rg[1] += a1 * marea;
        rg[2] += a2 * marea;
        rh[0] = -(b0 * marea);
        rh[1] = -(b1 * marea);
        rh[2] = -(b2 * marea);
    }
    // rotated order (i first) back to the triangle's own order
    const int k0 = (3 - shift) % 3, k1 = (4 - shift) % 3, k2 = (5 - shift) % 3;
    g0 = rg[k0];
    g1 = rg[k1];
    g2 = rg[k2];
    h0 = rh[k0];
    h1 = rh[k1];
    h2 = rh[k2];
}

__device__ __forceinline__ double block_sum_fixed(double v, double* s_w) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) s_w[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        r = (lane < (int)(blockDim.x >> 5)) ? s_w[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
        if (lane == 0) s_w[0] = r;
    }
    __syncthreads();
    r = s_w[0];
    __syncthreads();
    return r;
}

template <bool MIRROR, int R>
__global__ void __launch_bounds__(ASM_THREADS) k_assemble_rows(
    int N, const int* __restrict__ ch_c0, int ncolors, const int* __restrict__ col_off, const int4* __restrict__ ent,
    int64_t E, const double* __restrict__ rec, const double* __restrict__ x, const double* __restrict__ phi,
    double* __restrict__ G, double* __restrict__ H, double* __restrict__ b, double* __restrict__ rowHp,
    double* __restrict__ bp, int single) {
    extern __shared__ __align__(16) double sm[];
    __shared__ double s_red[32];
    const int chunk = blockIdx.y;
    const int c0 = ch_c0[chunk], cw = ch_c0[chunk + 1] - c0;
    double* aG = sm;           // [R][cw]
    double* aH = sm + R * cw;  // [R][cw]
    const int r0 = blockIdx.x * R;
    for (int k = threadIdx.x; k < 2 * R * cw; k += ASM_THREADS) sm[k] = 0.0;
    double xr[R][3];
    int row[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = r0 + r;
        row[r] = (i < N) ? i : -1;
        const int ii = (i < N) ? i : r0;  // padding rows repeat a valid position; results are discarded
        xr[r][0] = x[3 * ii];
        xr[r][1] = x[3 * ii + 1];
        xr[r][2] = x[3 * ii + 2];
    }
    __syncthreads();
    const int* coff = col_off + (size_t)chunk * (ncolors + 1);
    for (int col = 0; col < ncolors; ++col) {
        const int e1 = coff[col + 1];
        for (int e = coff[col] + threadIdx.x; e < e1; e += ASM_THREADS) {
            const int4 tv = ent[e];
            const double nx = rec[21 * E + e], ny = rec[22 * E + e], nz = rec[23 * E + e];
            const double area = rec[24 * E + e], dt = rec[25 * E + e];
            double a[R][3], h[R][3], m[R][3];
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int k = 0; k < 3; ++k) a[r][k] = h[r][k] = m[r][k] = 0.0;
#pragma unroll
            for (int q = 0; q < 7; ++q) {
                const double yx = rec[(3 * q) * E + e], yy = rec[(3 * q + 1) * E + e], yz = rec[(3 * q + 2) * E + e];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const double zy = yy - xr[r][1], zz = yz - xr[r][2];
                    const double zx = yx - xr[r][0];
                    const double yz2 = fma(zy, zy, zz * zz);
                    const double inv = rsqrt_fp64(fma(zx, zx, yz2));
                    const double i3 = inv * inv * inv;
                    a[r][0] = fma(c_qc[q][0], inv, a[r][0]);
                    a[r][1] = fma(c_qc[q][1], inv, a[r][1]);
                    a[r][2] = fma(c_qc[q][2], inv, a[r][2]);
                    h[r][0] = fma(c_qc[q][0], i3, h[r][0]);
                    h[r][1] = fma(c_qc[q][1], i3, h[r][1]);
                    h[r][2] = fma(c_qc[q][2], i3, h[r][2]);
                    if (MIRROR) {
                        // image point (-y.x, y.y, y.z), image normal (-n.x, n.y, n.z) (Integrator.hpp:211-229)
                        const double mx = -yx - xr[r][0];
                        const double inv2 = rsqrt_fp64(fma(mx, mx, yz2));
                        const double j3 = inv2 * inv2 * inv2;
                        a[r][0] = fma(c_qc[q][0], inv2, a[r][0]);
                        a[r][1] = fma(c_qc[q][1], inv2, a[r][1]);
                        a[r][2] = fma(c_qc[q][2], inv2, a[r][2]);
                        m[r][0] = fma(c_qc[q][0], j3, m[r][0]);
                        m[r][1] = fma(c_qc[q][1], j3, m[r][1]);
                        m[r][2] = fma(c_qc[q][2], j3, m[r][2]);
                    }
                }
            }
            const int lv[3] = {tv.y - c0, tv.z - c0, tv.w - c0};
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (row[r] < 0) continue;
                double g0, g1, g2, h0, h1, h2;
                const int i = row[r];
                if (i == tv.y || i == tv.z || i == tv.w) {
                    const int shift = (i == tv.y) ? 0 : ((i == tv.z) ? 1 : 2);
                    singular_pair<MIRROR>(x, tv.y, tv.z, tv.w, shift, g0, g1, g2, h0, h1, h2);
                } else {
                    const double xn_yz = xr[r][1] * ny + xr[r][2] * nz;
                    const double sh = -(dt - fma(xr[r][0], nx, xn_yz)) * area;  // -(y - x).n * area
                    g0 = a[r][0] * area;
                    g1 = a[r][1] * area;
                    g2 = a[r][2] * area;
                    h0 = h[r][0] * sh;
                    h1 = h[r][1] * sh;
                    h2 = h[r][2] * sh;
                    if (MIRROR) {
                        // (y' - x).n' = n.a - (-x.x n.x + x.y n.y + x.z n.z)
                        const double sm2 = -(dt - fma(-xr[r][0], nx, xn_yz)) * area;
                        h0 = fma(m[r][0], sm2, h0);
                        h1 = fma(m[r][1], sm2, h1);
                        h2 = fma(m[r][2], sm2, h2);
                    }
                }
                double* rG = aG + r * cw;
                double* rH = aH + r * cw;
                if ((unsigned)lv[0] < (unsigned)cw) {
                    rG[lv[0]] += g0;
                    rH[lv[0]] += h0;
                }
                if ((unsigned)lv[1] < (unsigned)cw) {
                    rG[lv[1]] += g1;
                    rH[lv[1]] += h1;
                }
                if ((unsigned)lv[2] < (unsigned)cw) {
                    rG[lv[2]] += g2;
                    rH[lv[2]] += h2;
                }
            }
        }
        __syncthreads();
    }
    // epilogue: fixed-order row reductions, 4 pi diagonal, H.phi, contiguous row writes
#pragma unroll 1
    for (int r = 0; r < R; ++r) {
        const int i = row[r];
        if (i < 0) break;
        double* rG = aG + r * cw;
        double* rH = aH + r * cw;
        double sh = 0.0, sb = 0.0;
        for (int j = threadIdx.x; j < cw; j += ASM_THREADS) {
            const double hv = rH[j];
            sh += hv;
            sb = fma(hv, phi[c0 + j], sb);
        }
        sh = block_sum_fixed(sh, s_red);
        sb = block_sum_fixed(sb, s_red);
        if (single) {
            // H(i,i) -= 4 pi - val, val = -sum_j H(i,j)  (ColocSim.cpp:85-97)
            const double d = -(4.0 * 3.14159265358979323846 + sh);
            if (threadIdx.x == 0) {
                rH[i - c0] += d;
                if (b) b[i] = fma(d, phi[i], sb);
            }
            __syncthreads();
        } else if (threadIdx.x == 0) {
            rowHp[(size_t)chunk * N + i] = sh;
            bp[(size_t)chunk * N + i] = sb;
        }
        double* gG = G + (size_t)i * N + c0;
        double* gH = H + (size_t)i * N + c0;
        for (int j = threadIdx.x; j < cw; j += ASM_THREADS) {
            gG[j] = rG[j];
            gH[j] = rH[j];
        }
    }
}

// Multi-chunk finish: 4 pi diagonal and right-hand side from the per-chunk partials.
__global__ void k_finish_rows(int N, int nchunks, const double* __restrict__ rowHp, const double* __restrict__ bp,
                              const double* __restrict__ phi, double* __restrict__ H, double* __restrict__ b) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double sh = 0.0, sb = 0.0;
    for (int k = 0; k < nchunks; ++k) {
        sh += rowHp[(size_t)k * N + i];
        sb += bp[(size_t)k * N + i];
    }
    const double d = -(4.0 * 3.14159265358979323846 + sh);
    H[(size_t)i * N + i] += d;
    if (b) b[i] = fma(d, phi[i], sb);
}

void launch_triangle_records(Ctx& c, const double* x, cudaStream_t s) {
    upload_constants();
    const int64_t E = c.topo.E;
    KLAUNCH(), k_triangle_records<<<(unsigned)((E + 127) / 128), 128, 0, s>>>(E, x, c.topo.ent, c.rec);
}

size_t assemble_smem_bytes(int rows, int cw) { return sizeof(double) * 2 * (size_t)rows * cw; }

template <bool MIRROR, int R>
static void launch_rows(Ctx& c, const double* x, const double* phi, double* G, double* H, double* b, cudaStream_t s) {
    const Topology& t = c.topo;
    const int N = (int)t.N;
    int cwmax = 0;
    for (int k = 0; k < t.nchunks; ++k) cwmax = std::max(cwmax, t.h_ch_c0[k + 1] - t.h_ch_c0[k]);
    const size_t sm = assemble_smem_bytes(R, cwmax);
    static int attr_set = 0;
    if (attr_set < (int)sm) {
        cudaFuncSetAttribute(k_assemble_rows<MIRROR, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        attr_set = (int)sm;
    }
    dim3 grid((N + R - 1) / R, t.nchunks);
    KLAUNCH(), k_assemble_rows<MIRROR, R><<<grid, ASM_THREADS, sm, s>>>(N, t.ch_c0, t.ncolors, t.col_off, t.ent, t.E,
                                                                       c.rec, x, phi, G, H, b, c.rowHp, c.bp,
                                                                       t.nchunks == 1 ? 1 : 0);
}

template <bool MIRROR>
static void launch_rows_r(Ctx& c, const double* x, const double* phi, double* G, double* H, double* b, cudaStream_t s) {
    switch (c.topo.asm_rows) {
        case 4:
            launch_rows<MIRROR, 4>(c, x, phi, G, H, b, s);
            break;
        case 3:
            launch_rows<MIRROR, 3>(c, x, phi, G, H, b, s);
            break;
        case 2:
            launch_rows<MIRROR, 2>(c, x, phi, G, H, b, s);
            break;
        default:
            launch_rows<MIRROR, 1>(c, x, phi, G, H, b, s);
    }
}

void launch_assemble(Ctx& c, const double* x, const double* phi, double* G, double* H, double* b, cudaStream_t s) {
    const int N = (int)c.topo.N;
    launch_triangle_records(c, x, s);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c.prof) {
        e0 = c.take_event();
        e1 = c.take_event();
        cudaEventRecord(e0, s);
    }
    if (c.prm.mirror)
        launch_rows_r<true>(c, x, phi, G, H, b, s);
    else
        launch_rows_r<false>(c, x, phi, G, H, b, s);
    if (c.prof) {
        cudaEventRecord(e1, s);
        c.ev_asm.emplace_back(e0, e1);
    }
    if (c.topo.nchunks > 1)
        KLAUNCH(), k_finish_rows<<<(N + 255) / 256, 256, 0, s>>>(N, c.topo.nchunks, c.rowHp, c.bp, phi, H, b);
}

}  // namespace bemb
