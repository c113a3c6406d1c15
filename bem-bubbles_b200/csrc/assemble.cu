// Dense collocation assembly of G (single layer) and H (double layer) in FP64.
//
// Replaces ColocSim::assemble_matrices (Bem/Simulation/ColocSim.cpp:21-110) with the per-pair
// integrals of Integrator::integrate_Lin_coloc_local[_mir] (Bem/Integration/Integrator.cpp:237-283):
//   * regular pairs (vertex i not on triangle t): 7-point rule on the triangle
//     (integrate_disjoint_coloc[_mir], Integrator.hpp:471-513, kernel Integrator.hpp:116-119);
//   * singular pairs (i on t): polar rule with the analytic radial integral and 7-point Gauss in
//     the angle (integrate_identical_coloc[_mir], Integrator.cpp:13-89);
//   * the "4 pi rule" diagonal H(i,i) -= 4 pi + sum_j H(i,j) (ColocSim.cpp:85-97).
//
// Tiling (B200): a CTA owns one column group (cg vertices, i.e. cg columns of G and H) and a block
// of collocation rows, one row per thread.  It walks the triangles incident to its
// vertices in increasing index order (the reference's per-column summation order), with the
// triangle records staged in shared memory and read as broadcasts, and accumulates the cg columns
// of its rows in shared memory.  Column writes are coalesced (column-major, consecutive rows).
// No atomics: every entry is summed by exactly one thread in a fixed order, so the result is
// bit-reproducible run to run.  The same pass produces the per-group partial row sums of H and
// partial H*phi, so the 4 pi diagonal and the right-hand side need no second read of H.
#include <math.h>
#include <mutex>

#include "ctx.h"

namespace bemb {

// c[q][k] = w_q * basis_k(u_q, v_q) for the 7-point rule mapped to the 45-degree unit triangle
// (u, v) = (qx + qy, qy), basis (1-u, u-v, v) (ResultTypes.hpp:111-117); u_q, v_q; Gauss-7 angle data.
__constant__ double c_qc[7][3];
__constant__ double c_quv[7][2];
__constant__ double c_gcos[7], c_gsin[7], c_gw[7];
// The 7-point rule is symmetric: the centroid plus two orbits of three points whose barycentric
// weights are rotations of (alpha, beta, beta).  With S the orbit sum of kernel values and
// g_k the orbit point whose alpha sits on vertex k, sum_q w_q basis_k(q) K(q) =
//   C + dA * gA_k + dB * gB_k,   C = w0 b0 K(centroid) + cA*S_A + cB*S_B.
// c_orb = {w0*b0, cA, dA, cB, dB}.
__constant__ double c_orb[5];

// Reference tables (quadrature.hpp:30-38 gauss_7, :88-96 quadrature_7) in the forms the kernels use:
// per point the basis weights (1-u, u-v, v) * w of the triangle rule applied as (x+y, y) on the
// unit triangle, and cos, sin and weight of the Gauss angles on (0, pi/4).
void quad_tables(QuadTables& t) {
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
    for (int q = 0; q < 7; ++q) {
        double u = Q[q][0] + Q[q][1], v = Q[q][1], w = Q[q][2];
        t.quv[q][0] = u;
        t.quv[q][1] = v;
        t.w[q] = w;
        t.qc[q][0] = (1.0 - u) * w;
        t.qc[q][1] = (u - v) * w;
        t.qc[q][2] = v * w;
        double th = GL[q][0] * 0.78539816339744830962;
        t.gc[q] = cos(th);
        t.gs[q] = sin(th);
        t.gw[q] = GL[q][1];
    }
    // orbit form: point 0 is the centroid; points 3,1,2 carry alpha on vertex 0,1,2 (orbit A) and
    // points 6,4,5 (orbit B), with barycentric coordinates (1-u, u-v, v)
    const double w0 = Q[0][2], wA = Q[1][2], wB = Q[4][2];
    const double aA = 1.0 - (Q[3][0] + Q[3][1]), bA = Q[3][1];  // point 3: (alpha, beta, beta)
    const double aB = 1.0 - (Q[6][0] + Q[6][1]), bB = Q[6][1];  // point 6
    const double orb[5] = {w0 * (1.0 / 3.0), wA * bA, wA * (aA - bA), wB * bB, wB * (aB - bB)};
    for (int k = 0; k < 5; ++k) t.orb[k] = orb[k];
    // quadrature_19 (quadrature.hpp:126-146), the rule of compute_exterior_pot (LinLinSim.cpp:455)
    const double Q19[19][3] = {{0.33333333333333331, 0.33333333333333331, 9.71357962827961025e-2 * 0.5},
                               {2.06349616025259287e-2, 0.48968251919873701, 3.13347002271398278e-2 * 0.5},
                               {0.48968251919873701, 2.06349616025259287e-2, 3.13347002271398278e-2 * 0.5},
                               {0.48968251919873701, 0.48968251919873701, 3.13347002271398278e-2 * 0.5},
                               {0.12582081701412900, 0.43708959149293553, 7.78275410047754301e-2 * 0.5},
                               {0.43708959149293553, 0.12582081701412900, 7.78275410047754301e-2 * 0.5},
                               {0.43708959149293553, 0.43708959149293553, 7.78275410047754301e-2 * 0.5},
                               {0.62359292876193562, 0.18820353561903219, 7.96477389272090969e-2 * 0.5},
                               {0.18820353561903219, 0.62359292876193562, 7.96477389272090969e-2 * 0.5},
                               {0.18820353561903219, 0.18820353561903219, 7.96477389272090969e-2 * 0.5},
                               {0.91054097321109406, 4.47295133944529688e-2, 2.55776756586981006e-2 * 0.5},
                               {4.47295133944529688e-2, 0.91054097321109406, 2.55776756586981006e-2 * 0.5},
                               {4.47295133944529688e-2, 4.47295133944529688e-2, 2.55776756586981006e-2 * 0.5},
                               {0.74119859878449801, 3.68384120547362581e-2, 4.32835393772893970e-2 * 0.5},
                               {0.74119859878449801, 0.22196298916076573, 4.32835393772893970e-2 * 0.5},
                               {3.68384120547362581e-2, 0.74119859878449801, 4.32835393772893970e-2 * 0.5},
                               {3.68384120547362581e-2, 0.22196298916076573, 4.32835393772893970e-2 * 0.5},
                               {0.22196298916076573, 0.74119859878449801, 4.32835393772893970e-2 * 0.5},
                               {0.22196298916076573, 3.68384120547362581e-2, 4.32835393772893970e-2 * 0.5}};
    for (int q = 0; q < 19; ++q) {
        t.q19[q][0] = Q19[q][0] + Q19[q][1];
        t.q19[q][1] = Q19[q][1];
        t.q19[q][2] = Q19[q][2];
    }
}

static void upload_constants() {
    static std::atomic<uint64_t> done{0};
    once_per_device(done, [] {
        QuadTables t;
        quad_tables(t);
        return cudaMemcpyToSymbol(c_orb, t.orb, sizeof(t.orb)) == cudaSuccess &&
               cudaMemcpyToSymbol(c_qc, t.qc, sizeof(t.qc)) == cudaSuccess &&
               cudaMemcpyToSymbol(c_quv, t.quv, sizeof(t.quv)) == cudaSuccess &&
               cudaMemcpyToSymbol(c_gcos, t.gc, sizeof(t.gc)) == cudaSuccess &&
               cudaMemcpyToSymbol(c_gsin, t.gs, sizeof(t.gs)) == cudaSuccess &&
               cudaMemcpyToSymbol(c_gw, t.gw, sizeof(t.gw)) == cudaSuccess;
    });
}

// Per-triangle record: Interpolator (Interpolator.hpp:15-37) quantities and what the 7-point rule
// needs of the quadrature points y_q = a + w_q, w_q = u_q*ab + v_q*bc.  For a row x,
//   |y_q - x|^2 = |a - x|^2 + u_q (a - x).2ab + v_q (a - x).2bc + |w_q|^2,
// so a pair costs three dot products with a - x and then two FMAs and an add per point.  Layout:
// a (0-2), 2ab (3-5), 2bc (6-8), |w_q|^2 (9-15), y_q.x (16-22, for the wall image), unit normal
// (23-25), area (26), plane offset a.n (27).
__global__ void k_triangle_records(int M, const double* __restrict__ x, const int* __restrict__ tri,
                                   double* __restrict__ rec) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M) return;
    int ia = tri[3 * t], ib = tri[3 * t + 1], ic = tri[3 * t + 2];
    double ax = x[3 * ia], ay = x[3 * ia + 1], az = x[3 * ia + 2];
    double abx = x[3 * ib] - ax, aby = x[3 * ib + 1] - ay, abz = x[3 * ib + 2] - az;
    double bcx = x[3 * ic] - x[3 * ib], bcy = x[3 * ic + 1] - x[3 * ib + 1], bcz = x[3 * ic + 2] - x[3 * ib + 2];
    double nx = aby * bcz - abz * bcy, ny = abz * bcx - abx * bcz, nz = abx * bcy - aby * bcx;
    double area = sqrt(nx * nx + ny * ny + nz * nz);
    double ia_ = 1.0 / area;
    double* r = rec + (size_t)t * REC;
    r[0] = ax;
    r[1] = ay;
    r[2] = az;
    r[3] = 2.0 * abx;
    r[4] = 2.0 * aby;
    r[5] = 2.0 * abz;
    r[6] = 2.0 * bcx;
    r[7] = 2.0 * bcy;
    r[8] = 2.0 * bcz;
#pragma unroll
    for (int q = 0; q < 7; ++q) {
        const double u = c_quv[q][0], v = c_quv[q][1];
        const double wx = u * abx + v * bcx, wy = u * aby + v * bcy, wz = u * abz + v * bcz;
        r[9 + q] = wx * wx + wy * wy + wz * wz;
        r[16 + q] = ax + wx;
    }
    const double unx = nx * ia_, uny = ny * ia_, unz = nz * ia_;
    r[23] = unx;
    r[24] = uny;
    r[25] = unz;
    r[26] = area;
    // plane offset a.n: every quadrature point y_q satisfies y_q.n = a.n, so (y_q - x).n is one
    // number per (row, triangle) pair
    r[27] = ax * unx + ay * uny + az * unz;
}

// 1/sqrt(r2) for r2 > 0 in FP64: the hardware's approximate reciprocal square root
// (rsqrt.approx.ftz.f64) refined by the binomial series of (1-d)^(-1/2) = 1 + d/2 + 3d^2/8 + ...
// with d = 1 - r2*y0^2; truncation error 5d^3/16, far below the double rounding unit for the
// estimate's relative error.
__device__ __forceinline__ double rsqrt_fp64(double r2) {
    double y0;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y0) : "d"(r2));
    const double t = __dmul_rn(r2, y0);
    const double d = fma(-t, y0, 1.0);
    const double p = fma(0.375, d, 0.5);
    return fma(y0, __dmul_rn(d, p), y0);
}

// Orbit-form basis sums of the 7 kernel values k[0..6] (see c_orb): out_k = C + dA*kA_k + dB*kB_k.
__device__ __forceinline__ void orbit_sums(const double* k, double& o0, double& o1, double& o2) {
    const double SA = (k[1] + k[2]) + k[3], SB = (k[4] + k[5]) + k[6];
    const double C = fma(c_orb[0], k[0], fma(c_orb[1], SA, __dmul_rn(c_orb[3], SB)));
    o0 = fma(c_orb[2], k[3], fma(c_orb[4], k[6], C));
    o1 = fma(c_orb[2], k[1], fma(c_orb[4], k[4], C));
    o2 = fma(c_orb[2], k[2], fma(c_orb[4], k[5], C));
}

// Basis sums of one regular pair.  G_k = g_k * area; H_k = h_k * sh (+ m_k * sm with the wall image).
// The accumulation into the shared-memory sums is written with explicit fused multiply-adds, so every
// kernel that inlines this code produces the same bits (no contraction left to the compiler).
struct PairSums {
    double g[3], h[3], m[3];
    double area, sh, sm;
};

// Regular 7-point rule of one (row, triangle) pair.  All quadrature points lie in the triangle's
// plane, so (y_q - x).n = n.a - n.x is hoisted out of the quadrature loop (and likewise for the image
// triangle).
template <bool MIRROR>
__device__ __forceinline__ void regular_pair(const double* __restrict__ r, double xi0, double xi1, double xi2,
                                             PairSums& p) {
    const double nx = r[23], ny = r[24], nz = r[25], area = r[26], dt = r[27];
    const double xn_yz = fma(xi1, ny, __dmul_rn(xi2, nz));
    const double dn = dt - fma(xi0, nx, xn_yz);  // (y - x).n
    const double ax = r[0] - xi0, ay = r[1] - xi1, az = r[2] - xi2;
    const double A = fma(ax, ax, fma(ay, ay, __dmul_rn(az, az)));
    const double B = fma(ax, r[3], fma(ay, r[4], __dmul_rn(az, r[5])));
    const double C = fma(ax, r[6], fma(ay, r[7], __dmul_rn(az, r[8])));
    const double x4 = 4.0 * xi0;
    double kg[7], kh[7], km[7];
#pragma unroll
    for (int q = 0; q < 7; ++q) {
        const double r2 = fma(B, c_quv[q][0], fma(C, c_quv[q][1], A + r[9 + q]));
        const double inv = rsqrt_fp64(r2);
        kg[q] = inv;
        kh[q] = __dmul_rn(__dmul_rn(inv, inv), inv);
        if (MIRROR) {
            // image point (-y.x, y.y, y.z), image normal (-n.x, n.y, n.z) (Integrator.hpp:211-229):
            // |y' - x|^2 = |y - x|^2 + 4 x.x y.x
            const double inv2 = rsqrt_fp64(fma(x4, r[16 + q], r2));
            kg[q] += inv2;
            km[q] = __dmul_rn(__dmul_rn(inv2, inv2), inv2);
        }
    }
    orbit_sums(kg, p.g[0], p.g[1], p.g[2]);
    orbit_sums(kh, p.h[0], p.h[1], p.h[2]);
    p.area = area;
    p.sh = -__dmul_rn(dn, area);
    if (MIRROR) {
        orbit_sums(km, p.m[0], p.m[1], p.m[2]);
        // (y' - x).n' = n.a - (-x.x n.x + x.y n.y + x.z n.z)
        p.sm = -__dmul_rn(dt - fma(-xi0, nx, xn_yz), area);
    } else {
        p.m[0] = p.m[1] = p.m[2] = 0.0;
        p.sm = 0.0;
    }
}

template <bool MIRROR>
__device__ __forceinline__ double add_h(const PairSums& p, int k, double acc) {
    if (!MIRROR) return fma(p.h[k], p.sh, acc);
    return __dadd_rn(acc, fma(p.m[k], p.sm, __dmul_rn(p.h[k], p.sh)));
}

// Singular pair: row i is vertex `shift` of triangle (ta, tb, tc).  gg[m], hh[m]: the G and H
// contributions to the column of the triangle's vertex at position (m + shift) % 3.
template <bool MIRROR>
__device__ __forceinline__ void singular_sums(const double* __restrict__ x, int ta, int tb, int tc, int shift,
                                              double gg[3], double hh[3]) {
    const int r0 = shift == 0 ? ta : (shift == 1 ? tb : tc);
    const int r1 = shift == 0 ? tb : (shift == 1 ? tc : ta);
    const int r2 = shift == 0 ? tc : (shift == 1 ? ta : tb);
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
    double rg0 = s0, rg1 = s1, rg2 = s2, rh0 = 0.0, rh1 = 0.0, rh2 = 0.0;
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
        rg0 += a0 * marea;
        rg1 += a1 * marea;
        rg2 += a2 * marea;
        rh0 = -(b0 * marea);
        rh1 = -(b1 * marea);
        rh2 = -(b2 * marea);
    }
    gg[0] = rg0;
    gg[1] = rg1;
    gg[2] = rg2;
    hh[0] = rh0;
    hh[1] = rh1;
    hh[2] = rh2;
}

// Singular pairs of a row and the row's 4 pi rule, one warp per row (row i, il within its block of n
// vertices whose G/H block starts at element mbase and whose group partials are rowHp, bp).
//  * The lanes take the triangles around vertex i (the vertex-to-triangle lists are sorted), 32 at a
//    time, and evaluate their singular pairs in parallel: entries (lane, m) with column j and the G
//    and H contributions, staged in shared memory.
//  * The lane holding the first entry of each column j adds that column's entries to G(i, j) and
//    H(i, j) one by one in entry order (increasing triangle index), after the tile kernel has written
//    the regular part.  Entries of one column are never split between two lanes, so nothing races.
//  * The row's sums sum_j H(i, j) and sum_j H(i, j) phi_j are the group partials of the tiles (a fixed
//    butterfly order) plus the singular share (entry order); H(i, i) -= 4 pi + sum_j H(i, j) and
//    b_i = (H phi)_i follow (ColocSim.cpp:85-97).  Every sum has one fixed order, the same as with one
//    thread per row walking the triangles in order.
// A separate pass because inside the tile loop the rare singular branch cost a fifth of the tile
// kernel's time (divergent warps waiting at the staging barriers, and the call in the hot loop).
// GONLY (the G-only assembly of the step path, no H matrix): the partials bp are the regular pairs'
// share of sum_j H(i, j) (phi_j - phi_i) and rowHp is unused; the singular pairs add their H entries
// times (phi_j - phi_i), and b_i = that sum - 4 pi phi_i, which is the reference's
// sum_j H(i, j) phi_j after the 4 pi rule H(i, i) -= 4 pi + sum_j H(i, j) (ColocSim.cpp:85-97).
constexpr int SD_WARPS = 8;  // rows per CTA
template <bool MIRROR, bool GONLY = false>
__device__ __forceinline__ void singular_diag_row(int i, int il, int n, long long mbase, int vbase, int ngroups,
                                                  const double* __restrict__ rowHp, const double* __restrict__ bp,
                                                  const double* __restrict__ x, const int* __restrict__ tri,
                                                  const int* __restrict__ csr_off, const int* __restrict__ csr_idx,
                                                  const double* __restrict__ phi, double* __restrict__ G,
                                                  double* __restrict__ H, double* __restrict__ b,
                                                  const double* __restrict__ x0, const double* __restrict__ gp,
                                                  double* __restrict__ r0) {
    __shared__ int s_j[SD_WARPS][96];
    __shared__ double s_g[SD_WARPS][96], s_h[SD_WARPS][96];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double rs = 0.0, bsing = 0.0;  // (lane 0) the singular share of the H row sum and of H phi
    double gx = 0.0;               // (x0) this lane's share of (G x0)_i
    const int e0 = csr_off[i], e1 = csr_off[i + 1];
    for (int base = e0; base < e1; base += 32) {
        const int e = base + lane;
        int jj[3] = {-1, -1, -1};
        if (e < e1) {
            const int t = csr_idx[e];
            const int ta = tri[3 * t], tb = tri[3 * t + 1], tc = tri[3 * t + 2];
            const int shift = (i == ta) ? 0 : ((i == tb) ? 1 : 2);
            double gg[3], hh[3];
            singular_sums<MIRROR>(x, ta, tb, tc, shift, gg, hh);
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                jj[m] = tri[3 * t + (m + shift) % 3];
                s_g[w][3 * lane + m] = gg[m];
                s_h[w][3 * lane + m] = hh[m];
            }
        }
#pragma unroll
        for (int m = 0; m < 3; ++m) s_j[w][3 * lane + m] = jj[m];
        __syncwarp();
        const int ne = 3 * min(32, e1 - base);
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            const int j = jj[m], me = 3 * lane + m;
            if (j < 0) continue;
            bool first = true;
            for (int q = 0; q < me; ++q)
                if (s_j[w][q] == j) {
                    first = false;
                    break;
                }
            if (!first) continue;
            const size_t o = (size_t)mbase + (size_t)(j - vbase) * n + il;
            double gv = G[o], hv = (MIRROR && !GONLY) ? H[o] : 0.0, gsing = 0.0;
            for (int q = me; q < ne; ++q)
                if (s_j[w][q] == j) {
                    gv += s_g[w][q];
                    hv += s_h[w][q];
                    gsing += s_g[w][q];
                }
            G[o] = gv;
            if (x0) gx = fma(gsing, x0[j], gx);
            if (MIRROR && !GONLY) H[o] = hv;  // without the wall image the singular double layer vanishes (flat triangle)
        }
        if (MIRROR && lane == 0) {
            const double phii = GONLY ? phi[i] : 0.0;
            for (int q = 0; q < ne; ++q)
                if (s_j[w][q] >= 0) {
                    rs += s_h[w][q];
                    bsing = fma(s_h[w][q], GONLY ? phi[s_j[w][q]] - phii : phi[s_j[w][q]], bsing);
                }
        }
        __syncwarp();
    }
    // 4 pi rule and right-hand side: lane l sums the partials of groups l, l+32, ... and the warp adds
    // the lane sums in a fixed butterfly order (deterministic)
    double val = 0.0, bs = 0.0;
    const size_t pr = (size_t)il * ngroups;  // the row's partials, contiguous
    for (int g = lane; g < ngroups; g += 32) {
        if (!GONLY) val -= rowHp[pr + g];
        bs += bp[pr + g];
    }
    if (x0)
        for (int g = lane; g < ngroups; g += 32) gx += gp[pr + g];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        val += __shfl_xor_sync(0xffffffffu, val, o);
        bs += __shfl_xor_sync(0xffffffffu, bs, o);
        gx += __shfl_xor_sync(0xffffffffu, gx, o);
    }
    if (lane) return;
    bs += bsing;
    double bi;
    if (GONLY) {
        bi = fma(-4.0 * 3.14159265358979323846, phi[i], bs);
    } else {
        val -= rs;
        const double d = -(4.0 * 3.14159265358979323846 - val);
        const size_t oii = (size_t)mbase + (size_t)il * n + il;
        H[oii] += d;  // after the warp's singular update of H(i, i) (ordered by the last __syncwarp)
        bi = fma(d, phi[i], bs);
    }
    if (b) b[i] = bi;
    if (x0) r0[i] = bi - gx;  // the first residual b - G x0 of the solve that follows
}

template <bool MIRROR, bool GONLY = false>
__global__ void __launch_bounds__(32 * SD_WARPS)
    k_singular_diag(int N, int ngroups, const double* __restrict__ rowHp, const double* __restrict__ bp,
                    const double* __restrict__ x, const int* __restrict__ tri, const int* __restrict__ csr_off,
                    const int* __restrict__ csr_idx, const double* __restrict__ phi, double* __restrict__ G,
                    double* __restrict__ H, double* __restrict__ b, const double* __restrict__ x0,
                    const double* __restrict__ gp, double* __restrict__ r0) {
    const int i = blockIdx.x * SD_WARPS + (threadIdx.x >> 5);
    if (i >= N) return;
    singular_diag_row<MIRROR, GONLY>(i, i, N, 0, 0, ngroups, rowHp, bp, x, tri, csr_off, csr_idx, phi, G, H, b, x0,
                                     gp, r0);
}

// The same per block of a batch (rows of block vblk[i], its own groups and G/H block).
template <bool MIRROR>
__global__ void __launch_bounds__(32 * SD_WARPS)
    k_singular_diag_batch(int N, const int* __restrict__ vblk, const BlockInfo* __restrict__ blk,
                          const double* __restrict__ rowHp, const double* __restrict__ bp,
                          const double* __restrict__ x, const int* __restrict__ tri, const int* __restrict__ csr_off,
                          const int* __restrict__ csr_idx, const double* __restrict__ phi, double* __restrict__ G,
                          double* __restrict__ H, double* __restrict__ b) {
    const int i = blockIdx.x * SD_WARPS + (threadIdx.x >> 5);
    if (i >= N) return;
    const BlockInfo B = blk[vblk[i]];
    singular_diag_row<MIRROR>(i, i - B.vbase, B.n, B.mbase, B.vbase, B.ngroups, rowHp + B.pbase, bp + B.pbase, x,
                              tri, csr_off, csr_idx, phi, G, H, b, nullptr, nullptr, nullptr);
}

// Column-group tile: the columns of group g (local index gl within its block) for rows
// [row0, row0 + ROWS) clipped at rowend, of the block whose vertices start at vbase (n of them) and
// whose G/H block starts at element mbase.  CGT: vertices (columns) per group, ROWS: rows per CTA
// (one per thread).  Accumulators are thread-private columns of shared memory; the triangle
// records of the group are staged in shared memory ASM_TC at a time.
template <bool MIRROR, int CGT, int ROWS>
__device__ __forceinline__ void assemble_tile(double* smem, const double* __restrict__ x, const int* __restrict__ tri,
                                              const double* __restrict__ rec, const int* __restrict__ grp_off,
                                              const int* __restrict__ grp_tri, const int* __restrict__ grp_slot,
                                              const int* __restrict__ grp_vert, const double* __restrict__ phi,
                                              double* __restrict__ G, double* __restrict__ H,
                                              double* __restrict__ rowHp, double* __restrict__ bp, int g, int gl,
                                              int row0, int rowend, int n, int vbase, long long mbase,
                                              long long pbase, int ngrp, const double* __restrict__ x0,
                                              double* __restrict__ gp) {
    double* accG = smem;                      // [CGT][ROWS]
    double* accH = accG + CGT * ROWS;         // [CGT][ROWS]
    double* srec = accH + CGT * ROWS;         // [ASM_TC][REC]
    int* sinfo = reinterpret_cast<int*>(srec + ASM_TC * REC);  // [ASM_TC][4]
    const int tid = threadIdx.x;
    const int i = row0 + tid;
#pragma unroll 4
    for (int s = 0; s < CGT; ++s) {
        accG[s * ROWS + tid] = 0.0;
        accH[s * ROWS + tid] = 0.0;
    }
    double xi0 = 0.0, xi1 = 0.0, xi2 = 0.0;
    if (i < rowend) {
        xi0 = x[3 * i];
        xi1 = x[3 * i + 1];
        xi2 = x[3 * i + 2];
    }
    const int tb = grp_off[g], te = grp_off[g + 1];
    for (int c0 = tb; c0 < te; c0 += ASM_TC) {
        const int cnt = min(ASM_TC, te - c0);
        __syncthreads();
        for (int e = tid; e < cnt * (REC / 2); e += ROWS) {
            int tt = e / (REC / 2), w = e - tt * (REC / 2);
            const double2* src = reinterpret_cast<const double2*>(rec + (size_t)grp_tri[c0 + tt] * REC);
            reinterpret_cast<double2*>(srec + tt * REC)[w] = src[w];
        }
        for (int e = tid; e < cnt; e += ROWS) {
            int t = grp_tri[c0 + e];
            sinfo[4 * e] = grp_slot[c0 + e];
            sinfo[4 * e + 1] = tri[3 * t];
            sinfo[4 * e + 2] = tri[3 * t + 1];
            sinfo[4 * e + 3] = tri[3 * t + 2];
        }
        __syncthreads();
        if (i < rowend) {
            for (int tt = 0; tt < cnt; ++tt) {
                const int4 info = reinterpret_cast<const int4*>(sinfo)[tt];
                const int code = info.x;
                if (i == info.y || i == info.z || i == info.w) continue;  // singular: k_singular_diag
                PairSums p;
                regular_pair<MIRROR>(srec + tt * REC, xi0, xi1, xi2, p);
                const int s0 = code & SLOT_NONE, s1 = (code >> SLOT_BITS) & SLOT_NONE,
                          s2 = (code >> (2 * SLOT_BITS)) & SLOT_NONE;
                if (s0 != SLOT_NONE) {
                    accG[s0 * ROWS + tid] = fma(p.g[0], p.area, accG[s0 * ROWS + tid]);
                    accH[s0 * ROWS + tid] = add_h<MIRROR>(p, 0, accH[s0 * ROWS + tid]);
                }
                if (s1 != SLOT_NONE) {
                    accG[s1 * ROWS + tid] = fma(p.g[1], p.area, accG[s1 * ROWS + tid]);
                    accH[s1 * ROWS + tid] = add_h<MIRROR>(p, 1, accH[s1 * ROWS + tid]);
                }
                if (s2 != SLOT_NONE) {
                    accG[s2 * ROWS + tid] = fma(p.g[2], p.area, accG[s2 * ROWS + tid]);
                    accH[s2 * ROWS + tid] = add_h<MIRROR>(p, 2, accH[s2 * ROWS + tid]);
                }
            }
        }
    }
    if (i < rowend) {
        const int il = i - vbase;
        double rs = 0.0, bs = 0.0, gs = 0.0;
        for (int s = 0; s < CGT; ++s) {
            int v = grp_vert[g * CGT + s];
            if (v < 0) continue;
            double gv = accG[s * ROWS + tid], hv = accH[s * ROWS + tid];
            const size_t o = (size_t)mbase + (size_t)(v - vbase) * n + il;
            G[o] = gv;
            H[o] = hv;
            rs += hv;
            bs = fma(hv, phi[v], bs);
            if (x0) gs = fma(gv, x0[v], gs);
        }
        // row-major partials (row il, group gl of ngrp): the reduction over groups then reads each
        // row's partials as one contiguous run
        const size_t po = (size_t)pbase + (size_t)il * ngrp + gl;
        rowHp[po] = rs;
        bp[po] = bs;
        if (x0) gp[po] = gs;
    }
}

// Single system: one CTA per (column group, row tile).
template <bool MIRROR, int CGT, int ROWS, int MINB>
__global__ void __launch_bounds__(ROWS, MINB) k_assemble(int N, const double* __restrict__ x, const int* __restrict__ tri,
                                                         const double* __restrict__ rec, const int* __restrict__ grp_off,
                                                         const int* __restrict__ grp_tri, const int* __restrict__ grp_slot,
                                                         const int* __restrict__ grp_vert, const double* __restrict__ phi,
                                                         double* __restrict__ G, double* __restrict__ H,
                                                         double* __restrict__ rowHp, double* __restrict__ bp,
                                                         const double* __restrict__ x0, double* __restrict__ gp) {
    extern __shared__ __align__(16) double smem[];
    assemble_tile<MIRROR, CGT, ROWS>(smem, x, tri, rec, grp_off, grp_tri, grp_slot, grp_vert, phi, G, H, rowHp, bp,
                                     blockIdx.x, blockIdx.x, blockIdx.y * ROWS, N, N, 0, 0, 0, gridDim.x, x0, gp);
}

// Block-diagonal batch: one persistent launch over the work list of every block's tiles
// {group, first row, block, local group}; CTAs take tiles from an atomic counter, which the CTA
// that draws the last ticket resets for the next launch.
template <bool MIRROR, int CGT, int ROWS, int MINB>
__global__ void __launch_bounds__(ROWS, MINB)
    k_assemble_batch(const int4* __restrict__ tiles, int ntiles, unsigned* __restrict__ ctr,
                     const BlockInfo* __restrict__ blk, const double* __restrict__ x, const int* __restrict__ tri,
                     const double* __restrict__ rec, const int* __restrict__ grp_off, const int* __restrict__ grp_tri,
                     const int* __restrict__ grp_slot, const int* __restrict__ grp_vert, const double* __restrict__ phi,
                     double* __restrict__ G, double* __restrict__ H, double* __restrict__ rowHp,
                     double* __restrict__ bp) {
    extern __shared__ __align__(16) double smem[];
    __shared__ unsigned s_t;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) {
            s_t = atomicAdd(ctr, 1u);
            if (s_t == (unsigned)ntiles + gridDim.x - 1) *ctr = 0u;  // last ticket of this launch
        }
        __syncthreads();
        const unsigned t = s_t;
        if (t >= (unsigned)ntiles) break;
        const int4 td = tiles[t];
        const BlockInfo B = blk[td.z];
        assemble_tile<MIRROR, CGT, ROWS>(smem, x, tri, rec, grp_off, grp_tri, grp_slot, grp_vert, phi, G, H, rowHp,
                                         bp, td.x, td.w, td.y, B.vbase + B.n, B.n, B.vbase, B.mbase, B.pbase, B.ngroups,
                                         nullptr, nullptr);
    }
}

void launch_triangle_records(Ctx& c, const double* x, cudaStream_t s) {
    upload_constants();
    int M = (int)c.topo.M;
    KLAUNCH(), k_triangle_records<<<(M + 127) / 128, 128, 0, s>>>(M, x, c.topo.tri, c.rec);
}

template <bool MIRROR, int CGT, int ROWS, int MINB>
static void launch_tiles_t(Ctx& c, const double* x, const double* phi, double* G, double* H, cudaStream_t s,
                           const double* x0) {
    const int N = (int)c.topo.N;
    const size_t sm = sizeof(double) * (2 * CGT * ROWS + ASM_TC * REC) + sizeof(int) * 4 * ASM_TC;
    static std::atomic<uint64_t> attr{0};
    once_per_device(attr, [sm] {
        return cudaFuncSetAttribute(k_assemble<MIRROR, CGT, ROWS, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)sm) == cudaSuccess;
    });
    dim3 grid(c.topo.ngroups, (N + ROWS - 1) / ROWS);
    KLAUNCH(), k_assemble<MIRROR, CGT, ROWS, MINB><<<grid, ROWS, sm, s>>>(N, x, c.topo.tri, c.rec, c.topo.grp_off,
                                                                          c.topo.grp_tri, c.topo.grp_slot,
                                                                          c.topo.grp_vert, phi, G, H, c.rowHp, c.bp, x0,
                                                                          c.gp);
}

template <int CGT, int ROWS>
constexpr size_t tile_smem() {
    return sizeof(double) * (2 * CGT * ROWS + ASM_TC * REC) + sizeof(int) * 4 * ASM_TC;
}

template <bool MIRROR, int CGT, int ROWS, int MINB>
static void prepare_batch_t(Ctx& c) {
    const size_t sm = tile_smem<CGT, ROWS>();
    auto kern = k_assemble_batch<MIRROR, CGT, ROWS, MINB>;
    static std::atomic<uint64_t> attr{0};
    once_per_device(attr, [kern, sm] {
        return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) == cudaSuccess;
    });
    if (c.asm_grid_cg != CGT) {  // persistent grid: every CTA slot the SMs can hold
        int per_sm = 0, sms = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, ROWS, sm);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
        c.asm_grid = std::max(1, std::min(c.ntiles, std::max(1, per_sm) * sms));
        c.asm_grid_cg = CGT;
    }
}

template <bool MIRROR, int CGT, int ROWS, int MINB>
static void launch_batch_t(Ctx& c, const double* x, const double* phi, double* G, double* H, cudaStream_t s) {
    const size_t sm = tile_smem<CGT, ROWS>();
    auto kern = k_assemble_batch<MIRROR, CGT, ROWS, MINB>;
    prepare_batch_t<MIRROR, CGT, ROWS, MINB>(c);
    KLAUNCH(), kern<<<c.asm_grid, ROWS, sm, s>>>(c.tiles, c.ntiles, c.tile_ctr, c.blk, x, c.topo.tri, c.rec,
                                                c.topo.grp_off, c.topo.grp_tri, c.topo.grp_slot, c.topo.grp_vert, phi,
                                                G, H, c.rowHp, c.bp);
}

// Tile shapes: 16 columns x 256 rows (24 warps/SM, more boundary triangles), 32 x 128 (12 warps/SM),
// 48 x 64 and 64 x 64 (fewer boundary triangles, 6 warps/SM); all at 3 CTAs per SM within the 228 KB
// of shared memory.
void prepare_assemble_g(Ctx& c);

void prepare_assemble(Ctx& c) {
    if (c.topo.npatch > 0) prepare_assemble_g(c);
    if (!c.batch) return;
    c.asm_grid_cg = 0;
    if (c.prm.mirror) {
        if (c.topo.cg == 16) prepare_batch_t<true, 16, 256, 3>(c);
        else if (c.topo.cg == 64) prepare_batch_t<true, 64, 64, 3>(c);
        else if (c.topo.cg == 48) prepare_batch_t<true, 48, 64, 3>(c);
        else prepare_batch_t<true, 32, 128, 3>(c);
    } else {
        if (c.topo.cg == 16) prepare_batch_t<false, 16, 256, 3>(c);
        else if (c.topo.cg == 64) prepare_batch_t<false, 64, 64, 3>(c);
        else if (c.topo.cg == 48) prepare_batch_t<false, 48, 64, 3>(c);
        else prepare_batch_t<false, 32, 128, 3>(c);
    }
}

template <bool MIRROR>
static void launch_tiles(Ctx& c, const double* x, const double* phi, double* G, double* H, cudaStream_t s,
                         const double* x0) {
    if (c.batch) {
        switch (c.topo.cg) {
            case 16:
                launch_batch_t<MIRROR, 16, 256, 3>(c, x, phi, G, H, s);
                break;
            case 64:
                launch_batch_t<MIRROR, 64, 64, 3>(c, x, phi, G, H, s);
                break;
            case 48:
                launch_batch_t<MIRROR, 48, 64, 3>(c, x, phi, G, H, s);
                break;
            default:
                launch_batch_t<MIRROR, 32, 128, 3>(c, x, phi, G, H, s);
        }
        return;
    }
    switch (c.topo.cg) {
        case 16:
            launch_tiles_t<MIRROR, 16, 256, 3>(c, x, phi, G, H, s, x0);
            break;
        case 64:
            launch_tiles_t<MIRROR, 64, 64, 3>(c, x, phi, G, H, s, x0);
            break;
        case 48:
            launch_tiles_t<MIRROR, 48, 64, 3>(c, x, phi, G, H, s, x0);
            break;
        default:
            launch_tiles_t<MIRROR, 32, 128, 3>(c, x, phi, G, H, s, x0);
    }
}

// x0, r0 (single systems, may be null): with x0 the assembly also returns r0 = b - G x0, the first
// residual of a solve started from x0, from the G columns while they are in shared memory (per-group
// partials of G x0 beside those of H phi).
void launch_assemble(Ctx& c, const double* x, const double* phi, double* G, double* H, double* b, cudaStream_t s,
                     const double* x0, double* r0) {
    const int N = (int)c.topo.N;
    if (c.batch || !r0) x0 = nullptr;
    launch_triangle_records(c, x, s);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c.prof) {
        e0 = c.take_event();
        e1 = c.take_event();
        cudaEventRecord(e0, s);
    }
    if (c.prm.mirror)
        launch_tiles<true>(c, x, phi, G, H, s, x0);
    else
        launch_tiles<false>(c, x, phi, G, H, s, x0);
    // singular pairs and the 4 pi rule, one warp per row
    const Topology& T = c.topo;
    const int nbs = (N + SD_WARPS - 1) / SD_WARPS, nt = 32 * SD_WARPS;
    if (c.batch) {
        if (c.prm.mirror)
            KLAUNCH(), k_singular_diag_batch<true><<<nbs, nt, 0, s>>>(N, c.vblk, c.blk, c.rowHp, c.bp, x, T.tri, T.csr_off,
                                                                      T.csr_idx, phi, G, H, b);
        else
            KLAUNCH(), k_singular_diag_batch<false><<<nbs, nt, 0, s>>>(N, c.vblk, c.blk, c.rowHp, c.bp, x, T.tri,
                                                                       T.csr_off, T.csr_idx, phi, G, H, b);
    } else {
        if (c.prm.mirror)
            KLAUNCH(), k_singular_diag<true><<<nbs, nt, 0, s>>>(N, T.ngroups, c.rowHp, c.bp, x, T.tri, T.csr_off,
                                                                T.csr_idx, phi, G, H, b, x0, c.gp, r0);
        else
            KLAUNCH(), k_singular_diag<false><<<nbs, nt, 0, s>>>(N, T.ngroups, c.rowHp, c.bp, x, T.tri, T.csr_off,
                                                                 T.csr_idx, phi, G, H, b, x0, c.gp, r0);
    }
    if (c.prof) {  // the profile's assembly time: tiles, singular pairs and the 4 pi rule
        cudaEventRecord(e1, s);
        c.ev_asm.emplace_back(e0, e1);
    }
}


// ------------------------------------------------------------------------------------------------
// G-only assembly of the step path (triangle patches)
// ------------------------------------------------------------------------------------------------
// The RK4 step needs G and b = H phi (after the 4 pi rule), never H itself.  Each triangle belongs
// to exactly one patch (Topology::patch_*), so every regular (row, triangle) pair is evaluated once:
// a CTA owns one patch and ROWS rows, accumulates the patch's columns (at most PCOLS vertices) in
// shared memory and, per row, b's regular share sum_t sum_k H_k(i, t) (phi_k - phi_i) in a register.
// The patch's triangle records are contiguous (patch order) and arrive in shared memory by one bulk
// copy (cp.async.bulk, completion counted on an mbarrier) while the threads clear their accumulators.
// A column whose vertex has all its triangles in the patch is complete and goes straight to G; the
// columns of vertices shared with other patches go to halo columns.  For each shared vertex and row
// tile, the patch CTA that finishes last (a ticket counter) sums the halo slices in increasing patch
// order, while they are still in L2, and writes the G column.
// Without the wall image the singular pairs (3 per triangle, the polar rule of Integrator.cpp:13-41)
// are evaluated beside the records, one thread per (triangle, corner), and the tile loop adds them
// where the row is a vertex of the triangle; k_rhs_finish then sums each row's patch partials of b
// and adds the 4 pi term.  Per G entry the order is: the pairs of each patch, regular and singular,
// in increasing triangle order (for a column inside one patch, the reference's per-column order),
// then the patches in increasing order.  With the wall image the singular pairs carry an H part too;
// k_singular_diag<true, true> adds them after the tiles, with the 4 pi term.  No atomics on values,
// so results are bit-reproducible.

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// An mbarrier counting one arrival, initialised before any thread uses it.
__device__ __forceinline__ void copy_bar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One 1-D bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from global to
// shared memory, its completion counted on `bar` (the arrival that also announces the bytes).
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"((unsigned long long)__cvta_generic_to_global(src)), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// Bounded wait for phase `parity` of `bar`: false after `limit` polls.
__device__ __forceinline__ bool copy_bar_wait(uint64_t* bar, uint32_t parity, int limit) {
    const uint32_t a = smem_addr(bar);
    for (int it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
constexpr int COPY_WAIT_POLLS = 1 << 22;  // each poll may suspend the thread for a while: seconds in all

// Patch-order triangle records (PREC doubles): the k_triangle_records layout (0-27), the potential
// at the three vertices (28-30), the vertex ids (31, 21 bits each, as the bits of a double) and the
// column slots of the three vertices in the patch (32, 8 bits each).  Without the wall image the
// image points (16-22) are unused, and those doubles with 33-34 hold the triangle's singular pairs:
// for row = vertex k of the triangle, the G entry of the column of vertex v at sing_slot(3 k + v).
// 35 is padding.
__device__ __forceinline__ int sing_slot(int e) { return e < 7 ? 16 + e : 26 + e; }

// Threads [0, M): the records; without the wall image threads [M, 4M) also evaluate the singular
// pairs, one (triangle, corner) each (Integrator.cpp:13-41), into the record's singular slots.
template <bool MIRROR>
__global__ void k_patch_records(int M, const double* __restrict__ x, const double* __restrict__ phi,
                                const int* __restrict__ tri, const int* __restrict__ ptri,
                                const int* __restrict__ pslot, double* __restrict__ prec) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (!MIRROR && q >= M) {
        if (q >= 4 * M) return;
        const int p = (q - M) / 3, k = (q - M) - 3 * p;
        const int t = ptri[p];
        const int ta = tri[3 * t], tb = tri[3 * t + 1], tc = tri[3 * t + 2];
        double gg[3], hh[3];
        singular_sums<false>(x, ta, tb, tc, k, gg, hh);  // gg[m]: the column of vertex (m + k) % 3
        double* r = prec + (size_t)p * PREC;
#pragma unroll
        for (int m = 0; m < 3; ++m) r[sing_slot(3 * k + (m + k) % 3)] = gg[m];
        return;
    }
    const int p = q;
    if (p >= M) return;
    const int t = ptri[p];
    const int ia = tri[3 * t], ib = tri[3 * t + 1], ic = tri[3 * t + 2];
    const double ax = x[3 * ia], ay = x[3 * ia + 1], az = x[3 * ia + 2];
    const double abx = x[3 * ib] - ax, aby = x[3 * ib + 1] - ay, abz = x[3 * ib + 2] - az;
    const double bcx = x[3 * ic] - x[3 * ib], bcy = x[3 * ic + 1] - x[3 * ib + 1], bcz = x[3 * ic + 2] - x[3 * ib + 2];
    const double nx = aby * bcz - abz * bcy, ny = abz * bcx - abx * bcz, nz = abx * bcy - aby * bcx;
    const double area = sqrt(nx * nx + ny * ny + nz * nz);
    const double ia_ = 1.0 / area;
    double* r = prec + (size_t)p * PREC;
    r[0] = ax;
    r[1] = ay;
    r[2] = az;
    r[3] = 2.0 * abx;
    r[4] = 2.0 * aby;
    r[5] = 2.0 * abz;
    r[6] = 2.0 * bcx;
    r[7] = 2.0 * bcy;
    r[8] = 2.0 * bcz;
#pragma unroll
    for (int q2 = 0; q2 < 7; ++q2) {
        const double u = c_quv[q2][0], v = c_quv[q2][1];
        const double wx = u * abx + v * bcx, wy = u * aby + v * bcy, wz = u * abz + v * bcz;
        r[9 + q2] = wx * wx + wy * wy + wz * wz;
        if (MIRROR) r[16 + q2] = ax + wx;
    }
    const double unx = nx * ia_, uny = ny * ia_, unz = nz * ia_;
    r[23] = unx;
    r[24] = uny;
    r[25] = unz;
    r[26] = area;
    r[27] = ax * unx + ay * uny + az * unz;
    r[28] = phi[ia];
    r[29] = phi[ib];
    r[30] = phi[ic];
    r[31] = __longlong_as_double((long long)ia | ((long long)ib << 21) | ((long long)ic << 42));
    r[32] = __longlong_as_double((long long)pslot[p]);
    if (MIRROR) {
        r[33] = 0.0;
        r[34] = 0.0;
    }
    r[35] = 0.0;
}

template <int ROWS>
constexpr size_t patch_smem() {
    return sizeof(double) * ((size_t)PT_MAX * PREC + (size_t)PCOLS * ROWS);
}

// One CTA per tile {patch, first row} of the work list, ROWS rows of the patch's block, one row per
// thread.  G, the halo columns and the row partials are addressed through the patch's PatchInfo, so
// the same kernel serves a single system (one block) and a batch of independent bubbles.
template <bool MIRROR, int ROWS, int MINB>
__global__ void __launch_bounds__(ROWS, MINB)
    k_assemble_patch(const int2* __restrict__ work, const PatchInfo* __restrict__ pinfo,
                     const double* __restrict__ prec, const int* __restrict__ patch_col,
                     const long long* __restrict__ patch_dst, const double* __restrict__ x,
                     const double* __restrict__ phi, double* __restrict__ G, double* __restrict__ halo,
                     double* __restrict__ bp, const double* __restrict__ x0, double* __restrict__ gp,
                     int* __restrict__ err, const int* __restrict__ patch_pk, const PartialCol* __restrict__ pcol,
                     unsigned* __restrict__ halo_tick) {
    extern __shared__ __align__(16) double psmem[];
    double* srec = psmem;                  // [PT_MAX][PREC], the patch's records
    double* acc = psmem + PT_MAX * PREC;   // [PCOLS][ROWS], this CTA's rows of the patch's columns
    __shared__ __align__(8) uint64_t bar;
    __shared__ int s_col[PCOLS], s_pk[PCOLS];
    __shared__ long long s_dst[PCOLS];
    const int tid = threadIdx.x;
    const int2 wk = work[blockIdx.x];
    const int p = wk.x;
    const PatchInfo P = pinfo[p];
    const int i = wk.y + tid;  // row (global vertex index)
    if (tid == 0) copy_bar_init(&bar);
    __syncthreads();
    if (tid == 0) bulk_copy_g2s(srec, prec + (size_t)P.t0 * PREC, (uint32_t)(P.nt * PREC * sizeof(double)), &bar);
    if (tid < PCOLS) {
        s_col[tid] = patch_col[p * PCOLS + tid];
        s_dst[tid] = patch_dst[p * PCOLS + tid];
        s_pk[tid] = patch_pk[p * PCOLS + tid];
    }
#pragma unroll 8
    for (int s = 0; s < PCOLS; ++s) acc[s * ROWS + tid] = 0.0;
    const bool row = i < P.vbase + P.n;
    double xi0 = 0.0, xi1 = 0.0, xi2 = 0.0, phii = 0.0;
    if (row) {
        xi0 = x[3 * i];
        xi1 = x[3 * i + 1];
        xi2 = x[3 * i + 2];
        phii = phi[i];
    }
    if (!__syncthreads_and(copy_bar_wait(&bar, 0, COPY_WAIT_POLLS))) {
        // the records did not arrive in time: record the error, let the copy land (bounded) before the
        // CTA's shared memory is released, and leave this tile unwritten (the host reports the error)
        if (tid == 0) {
            atomicExch(err, 1);
            copy_bar_wait(&bar, 0, COPY_WAIT_POLLS);
        }
        return;
    }
    double hb = 0.0;  // sum over this patch's regular pairs of sum_k H_k (phi_k - phi_i)
    for (int t = 0; t < (row ? P.nt : 0); ++t) {
        const double* r = srec + t * PREC;
        const long long ids = __double_as_longlong(r[31]);
        const int code = (int)__double_as_longlong(r[32]);
        const int s0 = code & 255, s1 = (code >> 8) & 255, s2 = (code >> 16) & 255;
        const int ka = i == (int)(ids & 0x1FFFFF) ? 0 : (i == (int)((ids >> 21) & 0x1FFFFF) ? 1 : 2);
        if (ka < 2 || i == (int)(ids >> 42)) {
            // singular pair: without the wall image its G entries come with the records (the double
            // layer of the flat own triangle vanishes); with it, k_singular_diag<true, true> adds both
            if (!MIRROR) {
                acc[s0 * ROWS + tid] += r[sing_slot(3 * ka)];
                acc[s1 * ROWS + tid] += r[sing_slot(3 * ka + 1)];
                acc[s2 * ROWS + tid] += r[sing_slot(3 * ka + 2)];
            }
            continue;
        }
        PairSums ps;
        regular_pair<MIRROR>(r, xi0, xi1, xi2, ps);
        acc[s0 * ROWS + tid] = fma(ps.g[0], ps.area, acc[s0 * ROWS + tid]);
        acc[s1 * ROWS + tid] = fma(ps.g[1], ps.area, acc[s1 * ROWS + tid]);
        acc[s2 * ROWS + tid] = fma(ps.g[2], ps.area, acc[s2 * ROWS + tid]);
        const double e0 = r[28] - phii, e1 = r[29] - phii, e2 = r[30] - phii;
        hb = fma(fma(ps.h[0], e0, fma(ps.h[1], e1, __dmul_rn(ps.h[2], e2))), ps.sh, hb);
        if (MIRROR) hb = fma(fma(ps.m[0], e0, fma(ps.m[1], e1, __dmul_rn(ps.m[2], e2))), ps.sm, hb);
    }
    const int il = i - P.vbase;
    if (row) {
        double gs = 0.0;
        for (int s = 0; s < PCOLS; ++s) {
            const int v = s_col[s];
            if (v < 0) break;
            const double gv = acc[s * ROWS + tid];
            const long long h = s_dst[s];
            if (h < 0)
                G[P.mbase + (long long)(v - P.vbase) * P.n + il] = gv;
            else
                halo[h + il] = gv;
            if (x0) gs = fma(gv, x0[v], gs);
        }
        const long long po = P.pbase + (long long)il * P.np + P.lp;  // the row's partials are contiguous
        bp[po] = hb;
        if (x0) gp[po] = gs;
    }
    // shared vertices: one ticket per (vertex, row tile); the CTA drawing the last one sums the halo
    // slices of this row tile in increasing patch order (every slice was written before its ticket)
    const int rt = (wk.y - P.vbase) / ROWS;
    __threadfence();
    __syncthreads();
    __shared__ int s_nfin;
    static_assert(PCOLS == 32, "the finishing slots are drawn by one warp");
    static_assert(PT_MAX * PREC * sizeof(double) >= PCOLS * sizeof(PartialCol), "finishing slots fit the records");
    PartialCol* s_pc = reinterpret_cast<PartialCol*>(srec);  // the records are no longer read
    if (tid < PCOLS) {
        const int k = s_pk[tid];
        bool fin = false;
        PartialCol pc;
        if (k >= 0) {
            pc = pcol[k];
            fin = atomicAdd(&halo_tick[pc.tick + rt], 1u) == (unsigned)(pc.cnt - 1);
        }
        // the finishing columns, compacted in slot order
        const unsigned m = __ballot_sync(0xffffffffu, fin);
        if (fin) s_pc[__popc(m & ((1u << tid) - 1u))] = pc;
        if (tid == 0) s_nfin = __popc(m);
    }
    __syncthreads();
    const int nfin = s_nfin;
    if (nfin > 0) __threadfence();  // the other patches' slices, written before their tickets
    // four columns at a time, the first four slices of each loaded before any is summed (the slices
    // sit in L2: one round trip per four columns instead of one per column)
    constexpr int FC = 4, FS = 4;
    for (int f0 = 0; f0 < (row ? nfin : 0); f0 += FC) {
        double v[FC][FS];
#pragma unroll
        for (int f = 0; f < FC; ++f) {
            const PartialCol& pc = s_pc[f0 + f < nfin ? f0 + f : f0];
            const double* h = halo + pc.hpos + il;
#pragma unroll
            for (int c2 = 0; c2 < FS; ++c2) v[f][c2] = (f0 + f < nfin && c2 < pc.cnt) ? __ldcg(h + (size_t)c2 * pc.n) : 0.0;
        }
#pragma unroll
        for (int f = 0; f < FC; ++f) {
            if (f0 + f >= nfin) break;
            const PartialCol& pc = s_pc[f0 + f];
            double sum = v[f][0];
#pragma unroll
            for (int c2 = 1; c2 < FS; ++c2)
                if (c2 < pc.cnt) sum += v[f][c2];
            const double* h = halo + pc.hpos + il;
            for (int c2 = FS; c2 < pc.cnt; ++c2) sum += __ldcg(h + (size_t)c2 * pc.n);
            G[pc.gpos + il] = sum;
        }
    }
    if (tid < nfin) halo_tick[s_pc[tid].tick + rt] = 0u;  // for the next assembly
}

// The G-only singular pass of a batch: rows of block vblk[i], its patches' row partials.
template <bool MIRROR>
__global__ void __launch_bounds__(32 * SD_WARPS)
    k_singular_diag_batch_g(int N, const int* __restrict__ vblk, const BlockInfo* __restrict__ blk,
                            const double* __restrict__ bp, const double* __restrict__ x, const int* __restrict__ tri,
                            const int* __restrict__ csr_off, const int* __restrict__ csr_idx,
                            const double* __restrict__ phi, double* __restrict__ G, double* __restrict__ b) {
    const int i = blockIdx.x * SD_WARPS + (threadIdx.x >> 5);
    if (i >= N) return;
    const BlockInfo B = blk[vblk[i]];
    singular_diag_row<MIRROR, true>(i, i - B.vbase, B.n, B.mbase, B.vbase, B.npatch, nullptr, bp + B.ppbase, x, tri,
                                    csr_off, csr_idx, phi, G, nullptr, b, nullptr, nullptr, nullptr);
}

// b_i (and r0_i = b_i - (G x0)_i) of the G-only assembly without the wall image, one warp per row:
// the tiles already hold every pair of the row, so what is left is the sum of the row's patch partials
// (lane l takes patches l, l + 32, ..., the lanes add in a fixed butterfly order) and the 4 pi term,
// b_i = sum_j H(i, j) (phi_j - phi_i) - 4 pi phi_i (ColocSim.cpp:85-97).
__device__ __forceinline__ void rhs_finish_row(int i, int il, int np, const double* __restrict__ bp,
                                               const double* __restrict__ phi, double* __restrict__ b,
                                               const double* __restrict__ x0, const double* __restrict__ gp,
                                               double* __restrict__ r0) {
    const int lane = threadIdx.x & 31;
    const size_t pr = (size_t)il * np;  // the row's partials, contiguous
    double bs = 0.0, gx = 0.0;
    for (int g = lane; g < np; g += 32) bs += bp[pr + g];
    if (x0)
        for (int g = lane; g < np; g += 32) gx += gp[pr + g];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        bs += __shfl_xor_sync(0xffffffffu, bs, o);
        gx += __shfl_xor_sync(0xffffffffu, gx, o);
    }
    if (lane) return;
    const double bi = fma(-4.0 * 3.14159265358979323846, phi[i], bs);
    if (b) b[i] = bi;
    if (x0) r0[i] = bi - gx;
}

__global__ void __launch_bounds__(32 * SD_WARPS)
    k_rhs_finish(int N, int np, const double* __restrict__ bp, const double* __restrict__ phi,
                 double* __restrict__ b, const double* __restrict__ x0, const double* __restrict__ gp,
                 double* __restrict__ r0) {
    const int i = blockIdx.x * SD_WARPS + (threadIdx.x >> 5);
    if (i >= N) return;
    rhs_finish_row(i, i, np, bp, phi, b, x0, gp, r0);
}

__global__ void __launch_bounds__(32 * SD_WARPS)
    k_rhs_finish_batch(int N, const int* __restrict__ vblk, const BlockInfo* __restrict__ blk,
                       const double* __restrict__ bp, const double* __restrict__ phi, double* __restrict__ b) {
    const int i = blockIdx.x * SD_WARPS + (threadIdx.x >> 5);
    if (i >= N) return;
    const BlockInfo B = blk[vblk[i]];
    rhs_finish_row(i, i - B.vbase, B.npatch, bp + B.ppbase, phi, b, nullptr, nullptr, nullptr);
}

template <bool MIRROR>
static bool prepare_patch_t() {
    static std::atomic<uint64_t> attr{0};
    return once_per_device(attr, [] {
        return cudaFuncSetAttribute(k_assemble_patch<MIRROR, PATCH_ROWS, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)patch_smem<PATCH_ROWS>()) == cudaSuccess;
    });
}

// Kernel attributes and __constant__ tables of the G-only assembly, outside any stream capture.
void prepare_assemble_g(Ctx& c) {
    upload_constants();
    if (c.prm.mirror)
        prepare_patch_t<true>();
    else
        prepare_patch_t<false>();
}

// G (the context's G) and b = H phi after the 4 pi rule for positions x, potential phi, without H; with
// x0 (may be null; single systems) also r0 = b - G x0.  No pinned vertices.
void launch_assemble_g(Ctx& c, const double* x, const double* phi, double* b, cudaStream_t s, const double* x0,
                       double* r0) {
    const Topology& T = c.topo;
    const int N = (int)T.N, M = (int)T.M;
    if (!r0 || c.batch) x0 = nullptr;
    prepare_assemble_g(c);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c.prof) {
        e0 = c.take_event();
        e1 = c.take_event();
        cudaEventRecord(e0, s);
    }
    // records (and, without the wall image, the singular pairs)
    if (c.prm.mirror)
        KLAUNCH(), k_patch_records<true><<<(M + 127) / 128, 128, 0, s>>>(M, x, phi, T.tri, T.patch_tri,
                                                                          T.patch_slot, c.prec);
    else
        KLAUNCH(), k_patch_records<false><<<(4 * M + 127) / 128, 128, 0, s>>>(M, x, phi, T.tri, T.patch_tri,
                                                                               T.patch_slot, c.prec);
    constexpr size_t sm = patch_smem<PATCH_ROWS>();
    if (c.prm.mirror)
        KLAUNCH(), k_assemble_patch<true, PATCH_ROWS, 3><<<T.nwork, PATCH_ROWS, sm, s>>>(
                       T.pwork, T.pinfo, c.prec, T.patch_col, T.patch_dst, x, phi, c.G, c.halo, c.bp, x0, c.gp,
                       c.asm_err, T.patch_pk, T.pcol, T.halo_tick);
    else
        KLAUNCH(), k_assemble_patch<false, PATCH_ROWS, 3><<<T.nwork, PATCH_ROWS, sm, s>>>(
                       T.pwork, T.pinfo, c.prec, T.patch_col, T.patch_dst, x, phi, c.G, c.halo, c.bp, x0, c.gp,
                       c.asm_err, T.patch_pk, T.pcol, T.halo_tick);
    const int nbs = (N + SD_WARPS - 1) / SD_WARPS, nt = 32 * SD_WARPS;
    if (c.batch) {
        if (c.prm.mirror)
            KLAUNCH(), k_singular_diag_batch_g<true><<<nbs, nt, 0, s>>>(N, c.vblk, c.blk, c.bp, x, T.tri, T.csr_off,
                                                                        T.csr_idx, phi, c.G, b);
        else
            KLAUNCH(), k_rhs_finish_batch<<<nbs, nt, 0, s>>>(N, c.vblk, c.blk, c.bp, phi, b);
    } else if (c.prm.mirror) {
        KLAUNCH(), k_singular_diag<true, true><<<nbs, nt, 0, s>>>(N, T.npatch, nullptr, c.bp, x, T.tri, T.csr_off,
                                                                  T.csr_idx, phi, c.G, nullptr, b, x0, c.gp, r0);
    } else {
        KLAUNCH(), k_rhs_finish<<<nbs, nt, 0, s>>>(N, T.npatch, c.bp, phi, b, x0, c.gp, r0);
    }
    if (c.prof) {  // the profile's assembly time: records, tiles (with the shared columns' sums), singular pairs, 4 pi rule
        cudaEventRecord(e1, s);
        c.ev_asm.emplace_back(e0, e1);
    }
}

}  // namespace bemb
