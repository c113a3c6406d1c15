/* CPU restatement of the bem-bubbles per-step hot path -- the ORACLE (test infrastructure).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this file's
 * library; the product never does.  Each function follows one reference function with
 * the reference's floating-point operation order (cited per function), so results are
 * bit-identical to the reference compiled against the Eigen-API shim when the reference
 * runs on one thread.  Built without -march flags so that no FMA contraction happens.
 */
#include "bem_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#ifndef M_PI_4
#define M_PI_4 0.78539816339744830962
#endif

/* 7-point degree-5 triangle rule on the unit triangle (0,0),(1,0),(0,1), weights summing
 * to 1/2 (Bem/Integration/quadrature.hpp:88-96, the rule selected at Simulation.hpp:44). */
static const double QTRI[7][3] = {
    {0.33333333333333333, 0.33333333333333333, 0.22500000000000000 * 0.5},
    {0.79742698535308720, 0.10128650732345633, 0.12593918054482717 * 0.5},
    {0.10128650732345633, 0.79742698535308720, 0.12593918054482717 * 0.5},
    {0.10128650732345633, 0.10128650732345633, 0.12593918054482717 * 0.5},
    {0.05971587178976981, 0.47014206410511505, 0.13239415278850616 * 0.5},
    {0.47014206410511505, 0.05971587178976981, 0.13239415278850616 * 0.5},
    {0.47014206410511505, 0.47014206410511505, 0.13239415278850616 * 0.5}};
/* 7-point Gauss-Legendre on (0,1) (quadrature.hpp:30-38, selected at Simulation.hpp:45) */
/* quadrature_19 (quadrature.hpp:126-146), used by compute_exterior_pot (LinLinSim.cpp:455) */
static const double QTRI19[19][3] = {
    {0.33333333333333331, 0.33333333333333331, 9.71357962827961025e-2 * 0.5},
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

static const double GL7[7][2] = {
    {0.5 * (1.0 + 0.0000000000000000), 0.5 * 0.4179591836734694},
    {0.5 * (1.0 + 0.4058451513773972), 0.5 * 0.3818300505051189},
    {0.5 * (1.0 - 0.4058451513773972), 0.5 * 0.3818300505051189},
    {0.5 * (1.0 - 0.7415311855993945), 0.5 * 0.2797053914892766},
    {0.5 * (1.0 + 0.7415311855993945), 0.5 * 0.2797053914892766},
    {0.5 * (1.0 - 0.9491079123427585), 0.5 * 0.1294849661688697},
    {0.5 * (1.0 + 0.9491079123427585), 0.5 * 0.1294849661688697}};

typedef struct { double x, y, z; } v3;

static inline v3 mk(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline v3 vsub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vadd(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vscale(v3 a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline double vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 vcross(v3 a, v3 b) {  /* vector3d::vec, vector3d.hpp */
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline double vnorm(v3 a) { return sqrt(vdot(a, a)); }
static inline v3 vnormalize(v3 a) { return vscale(a, 1.0 / vnorm(a)); }
static inline v3 ld(const double* x, int64_t i) { return mk(x[3 * i], x[3 * i + 1], x[3 * i + 2]); }
static inline void st(double* x, int64_t i, v3 v) { x[3 * i] = v.x; x[3 * i + 1] = v.y; x[3 * i + 2] = v.z; }

/* Interpolator (Bem/Integration/Interpolator.hpp:15-37) */
typedef struct { v3 a, ab, bc, n; double area; } interp_t;
static interp_t mk_interp(v3 a, v3 b, v3 c) {
    interp_t t;
    t.a = a;
    t.ab = vsub(b, a);
    t.bc = vsub(c, b);
    t.n = vcross(t.ab, t.bc);
    t.area = vnorm(t.n);
    t.n = vscale(t.n, 1.0 / t.area);
    return t;
}
static inline v3 interp_at(const interp_t* t, double u, double v) {
    return vadd(vadd(t->a, vscale(t->ab, u)), vscale(t->bc, v));
}

/* integrand (Integrator.hpp:116-119): (1/|z|, -z.n/|z|^3) */
static inline void kern(v3 z, v3 n, double* g, double* h) {
    double inv = 1.0 / vnorm(z);
    *g = inv;
    *h = -vdot(z, n) * inv * inv * inv;
}

/* integrate_disjoint_coloc[_mir] (Integrator.hpp:471-513) with integrand_coloc[_mir]
 * (Integrator.hpp:197-229): 7-point rule on the 45-degree unit triangle, x (u,v) = (qx+qy, qy). */
static void disjoint_q(v3 x, const interp_t* t, int mirror, const double (*qt)[3], int nq, double G[3], double H[3]) {
    G[0] = G[1] = G[2] = 0.0;
    H[0] = H[1] = H[2] = 0.0;
    for (int q = 0; q < nq; ++q) {
        double y0 = qt[q][0] + qt[q][1], y1 = qt[q][1], w = qt[q][2];
        v3 y = interp_at(t, y0, y1);
        v3 n = t->n;
        double g, h;
        kern(vsub(y, x), n, &g, &h);
        if (mirror) {
            double g2, h2;
            y.x = -y.x;
            n.x = -n.x;
            kern(vsub(y, x), n, &g2, &h2);
            g += g2;
            h += h2;
        }
        double b[3] = {1.0 - y0, y0 - y1, y1}; /* get_linear_elements, ResultTypes.hpp:111-117 */
        for (int k = 0; k < 3; ++k) {
            G[k] += (b[k] * g) * w;
            H[k] += (b[k] * h) * w;
        }
    }
    for (int k = 0; k < 3; ++k) {
        G[k] *= t->area;
        H[k] *= t->area;
    }
}

static void disjoint(v3 x, const interp_t* t, int mirror, double G[3], double H[3]) {
    disjoint_q(x, t, mirror, QTRI, 7, G, H);
}

/* compute_exterior_pot (LinLinSim.cpp:440-477) with Integrator::get_exterior_potential
 * (Integrator.cpp:287-305): per evaluation point, the sum over triangles (in order) of
 * (-G.psi + H.phi)/(4 pi) over the 19-point rule, no wall image. */
void orc_exterior_pot(int64_t N, int64_t M, const double* x, const int64_t* tri, const double* phi,
                      const double* psi, int64_t P, const double* pts, double* out) {
    (void)N;
    for (int64_t i = 0; i < P; ++i) {
        v3 y = ld(pts, i);
        double val = 0.0;
        for (int64_t j = 0; j < M; ++j) {
            const int64_t* t = tri + 3 * j;
            interp_t it = mk_interp(ld(x, t[0]), ld(x, t[1]), ld(x, t[2]));
            double G[3], H[3];
            disjoint_q(y, &it, 0, QTRI19, 19, G, H);
            double integral = -G[0] * psi[t[0]] - G[1] * psi[t[1]] - G[2] * psi[t[2]] + H[0] * phi[t[0]] +
                              H[1] * phi[t[1]] + H[2] * phi[t[2]];
            integral *= (1.0 / (4.0 * M_PI));
            val += integral;
        }
        out[i] = val;
    }
}

/* integrate_identical_coloc<LinElm> (Integrator.cpp:13-41): x = vertex a of its own
 * triangle; polar coordinates, analytic radial integral, 7-point Gauss in theta on (0,pi/4). */
static void identical(const interp_t* t, double G[3]) {
    double jac = 0.5 * t->area * M_PI_4;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int q = 0; q < 7; ++q) {
        double px = GL7[q][0] * M_PI_4;
        double cx = cos(px), sx = sin(px);
        double dist = vnorm(vadd(vscale(t->ab, cx), vscale(t->bc, sx)));
        double of = jac * GL7[q][1] / dist;
        double fac = 1.0 / (cx * cx);
        acc[0] += of * cx * fac;
        acc[1] += of * (cx - sx) * fac;
        acc[2] += of * sx * fac;
    }
    G[0] = acc[0];
    G[1] = acc[1];
    G[2] = acc[2];
}

/* integrate_identical_coloc_mir (Integrator.cpp:44-89): singular part as above plus the
 * regular (non-image) rule over the mirrored own triangle, whose H flips sign. */
static void identical_mir(const interp_t* t, double G[3], double H[3]) {
    double Gs[3];
    identical(t, Gs);
    v3 a = interp_at(t, 0.0, 0.0);
    v3 x = a;
    v3 b = interp_at(t, 1.0, 0.0);
    v3 c = interp_at(t, 1.0, 1.0);
    a.x = -a.x;
    b.x = -b.x;
    c.x = -c.x;
    interp_t m = mk_interp(a, b, c);
    disjoint(x, &m, 0, G, H);
    for (int k = 0; k < 3; ++k) {
        H[k] *= -1.0;
        G[k] += Gs[k];
    }
}

int orc_assemble(int64_t N, int64_t M, const double* x, const int64_t* tri, int32_t mirror,
                 double* G, double* H) {
    memset(G, 0, sizeof(double) * (size_t)(N * N));
    memset(H, 0, sizeof(double) * (size_t)(N * N));
    /* triangle-major loop (ColocSim.cpp:49-79); on one thread the column scatter adds the
     * triangles in index order */
    for (int64_t j = 0; j < M; ++j) {
        const int64_t ta = tri[3 * j], tb = tri[3 * j + 1], tc = tri[3 * j + 2];
        for (int64_t i = 0; i < N; ++i) {
            double g[3], h[3];
            int64_t slot[3] = {ta, tb, tc};
            if (i == ta || i == tb || i == tc) {
                /* integrate_Lin_coloc_local[_mir] (Integrator.cpp:237-283): rotate so i is a */
                int shift = (i == ta) ? 0 : (i == tb ? 1 : 2);
                int64_t r[3] = {slot[shift], slot[(shift + 1) % 3], slot[(shift + 2) % 3]};
                interp_t t = mk_interp(ld(x, r[0]), ld(x, r[1]), ld(x, r[2]));
                if (mirror) {
                    identical_mir(&t, g, h);
                } else {
                    identical(&t, g);
                    h[0] = h[1] = h[2] = 0.0;
                }
                for (int k = 0; k < 3; ++k) {
                    int64_t col = slot[(k + shift) % 3];
                    G[col * N + i] += g[k];
                    H[col * N + i] += h[k];
                }
            } else {
                interp_t t = mk_interp(ld(x, ta), ld(x, tb), ld(x, tc));
                disjoint(ld(x, i), &t, mirror, g, h);
                for (int k = 0; k < 3; ++k) {
                    G[slot[k] * N + i] += g[k];
                    H[slot[k] * N + i] += h[k];
                }
            }
        }
    }
    /* 4-pi rule (ColocSim.cpp:85-97) */
    for (int64_t i = 0; i < N; ++i) {
        double val = 0.0;
        for (int64_t j = 0; j < N; ++j) val -= H[j * N + i];
        H[i * N + i] -= (4.0 * M_PI - val);
    }
    return 0;
}

void orc_gemv(int64_t N, const double* A, const double* v, double* y) {
    for (int64_t i = 0; i < N; ++i) y[i] = 0.0;
    for (int64_t j = 0; j < N; ++j) {
        const double vj = v[j];
        for (int64_t i = 0; i < N; ++i) y[i] += A[j * N + i] * vj;
    }
}

/* Blocked right-looking LU with row partial pivoting, panel width 64 (the shim's
 * PartialPivLU), then unit-lower / upper substitution. */
int orc_solve_lu(int64_t n, const double* G, const double* b, double* x) {
    const int64_t NB = 64;
    double* a = (double*)malloc(sizeof(double) * (size_t)(n * n));
    int64_t* perm = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
    if (!a || !perm) { free(a); free(perm); return -1; }
    memcpy(a, G, sizeof(double) * (size_t)(n * n));
#define A_(i, j) a[(i) + (j) * n]
    for (int64_t i = 0; i < n; ++i) perm[i] = i;
    int singular = 0;
    for (int64_t k0 = 0; k0 < n; k0 += NB) {
        const int64_t k1 = (k0 + NB < n) ? k0 + NB : n;
        for (int64_t k = k0; k < k1; ++k) {
            int64_t p = k;
            double best = fabs(A_(k, k));
            for (int64_t i = k + 1; i < n; ++i) {
                double v = fabs(A_(i, k));
                if (v > best) { best = v; p = i; }
            }
            if (p != k) {
                for (int64_t j = 0; j < n; ++j) { double t = A_(k, j); A_(k, j) = A_(p, j); A_(p, j) = t; }
                int64_t t = perm[k]; perm[k] = perm[p]; perm[p] = t;
            }
            const double piv = A_(k, k);
            if (piv != 0.0) {
                for (int64_t i = k + 1; i < n; ++i) A_(i, k) /= piv;
            } else {
                singular = 1;
            }
            for (int64_t j = k + 1; j < k1; ++j) {
                const double ukj = A_(k, j);
                for (int64_t i = k + 1; i < n; ++i) A_(i, j) -= A_(i, k) * ukj;
            }
        }
        if (k1 >= n) break;
        for (int64_t j = k1; j < n; ++j)
            for (int64_t k = k0; k < k1; ++k) {
                const double ukj = A_(k, j);
                for (int64_t i = k + 1; i < k1; ++i) A_(i, j) -= A_(i, k) * ukj;
            }
        for (int64_t j = k1; j < n; ++j)
            for (int64_t k = k0; k < k1; ++k) {
                const double ukj = A_(k, j);
                if (ukj == 0.0) continue;
                for (int64_t i = k1; i < n; ++i) A_(i, j) -= A_(i, k) * ukj;
            }
    }
    for (int64_t i = 0; i < n; ++i) x[i] = b[perm[i]];
    for (int64_t j = 0; j < n; ++j) {
        double xj = x[j];
        if (xj != 0.0)
            for (int64_t i = j + 1; i < n; ++i) x[i] -= A_(i, j) * xj;
    }
    for (int64_t j = n - 1; j >= 0; --j) {
        x[j] /= A_(j, j);
        double xj = x[j];
        if (xj != 0.0)
            for (int64_t i = 0; i < j; ++i) x[i] -= A_(i, j) * xj;
    }
#undef A_
    free(a);
    free(perm);
    return singular ? -3 : 0;
}

static double dotn(int64_t n, const double* u, const double* v) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += u[i] * v[i];
    return s;
}

/* Preconditioned BiCGSTAB with Eigen's documented defaults (Jacobi preconditioner,
 * tolerance = DBL_EPSILON, at most 2N iterations, zero start, shadow-residual restart). */
int orc_solve_bicgstab(int64_t n, const double* A, const double* b, double* x, int64_t* iters,
                       double* rel_err) {
    double* buf = (double*)calloc((size_t)(10 * n), sizeof(double));
    if (!buf) return -1;
    double *r = buf, *r0 = buf + n, *p = buf + 2 * n, *v = buf + 3 * n, *y = buf + 4 * n;
    double *z = buf + 5 * n, *s = buf + 6 * n, *t = buf + 7 * n, *invd = buf + 8 * n;
    for (int64_t i = 0; i < n; ++i) {
        double d = A[i + i * n];
        invd[i] = (d != 0.0) ? 1.0 / d : 1.0;
        x[i] = 0.0;
    }
    const double rhs2 = dotn(n, b, b);
    if (rhs2 == 0.0) {
        if (iters) *iters = 0;
        if (rel_err) *rel_err = 0.0;
        free(buf);
        return 0;
    }
    for (int64_t i = 0; i < n; ++i) r[i] = b[i];
    memcpy(r0, r, sizeof(double) * (size_t)n);
    double r0_sq = dotn(n, r0, r0);
    double rho = 1.0, alpha = 1.0, w = 1.0;
    const double eps = 2.220446049250313080847e-16;
    const double tol2 = eps * eps * rhs2, eps2 = eps * eps;
    const int64_t maxit = 2 * n;
    int64_t it = 0, restarts = 0;
    while (dotn(n, r, r) > tol2 && it < maxit) {
        double rho_old = rho;
        rho = dotn(n, r0, r);
        if (fabs(rho) < eps2 * r0_sq) {
            orc_gemv(n, A, x, t);
            for (int64_t i = 0; i < n; ++i) r[i] = b[i] - t[i];
            memcpy(r0, r, sizeof(double) * (size_t)n);
            rho = r0_sq = dotn(n, r, r);
            if (restarts++ == 0) it = 0;
        }
        double beta = (rho / rho_old) * (alpha / w);
        for (int64_t i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - w * v[i]);
        for (int64_t i = 0; i < n; ++i) y[i] = invd[i] * p[i];
        orc_gemv(n, A, y, v);
        alpha = rho / dotn(n, r0, v);
        for (int64_t i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
        for (int64_t i = 0; i < n; ++i) z[i] = invd[i] * s[i];
        orc_gemv(n, A, z, t);
        double tt = dotn(n, t, t);
        w = (tt > 0.0) ? dotn(n, t, s) / tt : 0.0;
        for (int64_t i = 0; i < n; ++i) x[i] += alpha * y[i] + w * z[i];
        for (int64_t i = 0; i < n; ++i) r[i] = s[i] - w * t[i];
        ++it;
    }
    if (iters) *iters = it;
    if (rel_err) *rel_err = sqrt(dotn(n, r, r) / rhs2);
    free(buf);
    return 0;
}

/* vertex -> incident triangles, increasing triangle order (Mesh.cpp:75-84) */
typedef struct { int64_t* off; int64_t* idx; } csr_t;
static int build_csr(int64_t N, int64_t M, const int64_t* tri, csr_t* c) {
    c->off = (int64_t*)calloc((size_t)(N + 1), sizeof(int64_t));
    c->idx = (int64_t*)malloc(sizeof(int64_t) * (size_t)(3 * M + 1));
    if (!c->off || !c->idx) return -1;
    for (int64_t j = 0; j < 3 * M; ++j) c->off[tri[j] + 1]++;
    for (int64_t i = 0; i < N; ++i) c->off[i + 1] += c->off[i];
    int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)(N + 1));
    if (!fill) return -1;
    memcpy(fill, c->off, sizeof(int64_t) * (size_t)(N + 1));
    for (int64_t j = 0; j < M; ++j)
        for (int k = 0; k < 3; ++k) c->idx[fill[tri[3 * j + k]]++] = j;
    free(fill);
    return 0;
}
static void free_csr(csr_t* c) { free(c->off); free(c->idx); }

/* Triplet::cyclic_reorder then (B x C)/(|B|^2 |C|^2) summed over the fan, normalised
 * (Mesh.cpp:141-163) */
static void vertex_normals_csr(int64_t N, const double* x, const int64_t* tri, const csr_t* c,
                               double* out) {
    for (int64_t i = 0; i < N; ++i) {
        v3 n = mk(0.0, 0.0, 0.0);
        for (int64_t e = c->off[i]; e < c->off[i + 1]; ++e) {
            const int64_t* t = tri + 3 * c->idx[e];
            int64_t a = t[0], b = t[1], cc = t[2];
            if (i == b) { int64_t o = a; a = b; b = cc; cc = o; }
            else if (i == cc) { int64_t o = a; a = cc; cc = b; b = o; }
            v3 B = vsub(ld(x, b), ld(x, a)), C = vsub(ld(x, cc), ld(x, a));
            n = vadd(n, vscale(vcross(B, C), 1.0 / (vdot(B, B) * vdot(C, C))));
        }
        st(out, i, vnormalize(n));
    }
}

void orc_vertex_normals(int64_t N, int64_t M, const double* x, const int64_t* tri, double* out) {
    csr_t c;
    if (build_csr(N, M, tri, &c) == 0) vertex_normals_csr(N, x, tri, &c, out);
    free_csr(&c);
}

double orc_volume(int64_t N, int64_t M, const double* x, const int64_t* tri) {
    (void)N;
    double vol = 0.0;
    for (int64_t j = 0; j < M; ++j) {
        v3 a = ld(x, tri[3 * j]), b = ld(x, tri[3 * j + 1]), c = ld(x, tri[3 * j + 2]);
        vol += vdot(vcross(a, b), c) / 6.0;
    }
    return vol;
}

static int solve_system(int64_t N, const double* G, const double* b, double* x, int use_lu) {
    if (use_lu) return orc_solve_lu(N, G, b, x);
    return orc_solve_bicgstab(N, G, b, x, NULL, NULL);
}

int orc_position_t(int64_t N, int64_t M, const double* x, const int64_t* tri, const double* pot,
                   const orc_params* p, double* vel, double* psi_out) {
    double* G = (double*)malloc(sizeof(double) * (size_t)(N * N));
    double* H = (double*)malloc(sizeof(double) * (size_t)(N * N));
    double* b = (double*)malloc(sizeof(double) * (size_t)N);
    double* psi = (double*)malloc(sizeof(double) * (size_t)N);
    v3* tn = (v3*)malloc(sizeof(v3) * (size_t)M);
    v3* tg = (v3*)malloc(sizeof(v3) * (size_t)M);
    csr_t c = {0, 0};
    int rc = -1;
    if (!G || !H || !b || !psi || !tn || !tg || build_csr(N, M, tri, &c)) goto done;
    orc_assemble(N, M, x, tri, p->mirror, G, H);
    orc_gemv(N, H, pot, b);                          /* H*make_copy(pot), LinLinSim.cpp:32 */
    rc = solve_system(N, G, b, psi, p->use_lu);
    for (int64_t j = 0; j < M; ++j) {
        const int64_t* t = tri + 3 * j;
        v3 A = ld(x, t[0]), B = ld(x, t[1]), C = ld(x, t[2]);
        tn[j] = vnormalize(vcross(vsub(B, A), vsub(C, A)));        /* Mesh.cpp:130-138 */
        v3 ab = vsub(B, A), bc = vsub(C, B);                         /* LinLinSim.cpp:288-305 */
        v3 n = vcross(ab, bc);
        n = vscale(n, 1.0 / vdot(n, n));
        tg[j] = vadd(vscale(vcross(n, ab), pot[t[2]] - pot[t[1]]),
                     vscale(vcross(n, bc), pot[t[0]] - pot[t[1]]));
    }
    for (int64_t i = 0; i < N; ++i) {                               /* LinLinSim.cpp:48-59 */
        double num = 0.0;
        v3 g = mk(0.0, 0.0, 0.0);
        for (int64_t e = c.off[i]; e < c.off[i + 1]; ++e) {
            int64_t j = c.idx[e];
            g = vadd(g, vadd(tg[j], vscale(tn[j], psi[i])));
            num += 1.0;
        }
        st(vel, i, vscale(g, 1.0 / num));
    }
    if (psi_out) memcpy(psi_out, psi, sizeof(double) * (size_t)N);
done:
    free(G); free(H); free(b); free(psi); free(tn); free(tg); free_csr(&c);
    return rc;
}

/* Full-pivoting LU solve of a (possibly tall) m x n system, the shim's FullPivLU. */
static void fullpiv_solve(int m, int n, double* a /* col-major m x n */, const double* rhs, double* x) {
    int rowp[16], colq[16];
    const int kmax = m < n ? m : n;
    for (int i = 0; i < m; ++i) rowp[i] = i;
    for (int j = 0; j < n; ++j) colq[j] = j;
    int rank = kmax, degenerate = 0;
    double maxpivot = 0.0;
#define F_(i, j) a[(i) + (j) * m]
    for (int k = 0; k < kmax; ++k) {
        int pr = k, pc = k;
        double best = -1.0;
        for (int j = k; j < n; ++j)
            for (int i = k; i < m; ++i) {
                double v = fabs(F_(i, j));
                if (v > best) { best = v; pr = i; pc = j; }
            }
        if (best == 0.0) { rank = k; degenerate = 1; break; }
        if (best > maxpivot) maxpivot = best;
        if (pr != k) {
            for (int j = 0; j < n; ++j) { double t = F_(k, j); F_(k, j) = F_(pr, j); F_(pr, j) = t; }
            int t = rowp[k]; rowp[k] = rowp[pr]; rowp[pr] = t;
        }
        if (pc != k) {
            for (int i = 0; i < m; ++i) { double t = F_(i, k); F_(i, k) = F_(i, pc); F_(i, pc) = t; }
            int t = colq[k]; colq[k] = colq[pc]; colq[pc] = t;
        }
        double piv = F_(k, k);
        for (int i = k + 1; i < m; ++i) F_(i, k) /= piv;
        for (int j = k + 1; j < n; ++j) {
            double ukj = F_(k, j);
            for (int i = k + 1; i < m; ++i) F_(i, j) -= F_(i, k) * ukj;
        }
    }
    if (!degenerate) {
        double thr = 2.220446049250313080847e-16 * (double)kmax;
        int r = 0;
        for (int k = 0; k < kmax; ++k)
            if (fabs(F_(k, k)) > thr * maxpivot) ++r;
        rank = r;
    }
    for (int j = 0; j < n; ++j) x[j] = 0.0;
    if (rank == 0) return;
    double c[16];
    for (int i = 0; i < m; ++i) c[i] = rhs[rowp[i]];
    for (int j = 0; j < kmax; ++j)
        for (int i = j + 1; i < kmax; ++i) c[i] -= F_(i, j) * c[j];
    for (int j = rank - 1; j >= 0; --j) {
        c[j] /= F_(j, j);
        for (int i = 0; i < j; ++i) c[i] -= F_(i, j) * c[j];
    }
    for (int i = 0; i < rank; ++i) x[colq[i]] = c[i];
#undef F_
}

/* LinLinSim::kappa -> curvatures (LinLinSim.cpp:122-146, Mesh.cpp:256-319) on one part */
static void part_kappa(int64_t n, int64_t m, const double* x, const int64_t* tri, double* kap) {
    double* vn = (double*)malloc(sizeof(double) * (size_t)(3 * n));
    double* w = (double*)calloc((size_t)n, sizeof(double));
    orc_vertex_normals(n, m, x, tri, vn);
    for (int64_t i = 0; i < n; ++i) kap[i] = 0.0;
    for (int64_t j = 0; j < m; ++j) {
        const int64_t* t = tri + 3 * j;
        v3 e0 = vsub(ld(x, t[1]), ld(x, t[0]));
        v3 e1 = vsub(ld(x, t[2]), ld(x, t[1]));
        v3 e2 = vsub(ld(x, t[0]), ld(x, t[2]));
        v3 u = vnormalize(e0);
        v3 nr = vnormalize(vcross(e0, e1));
        v3 v = vcross(nr, u);
        double A[18] = {0};
        double rows[6][3] = {{vdot(e0, u), vdot(e0, v), 0.0}, {0.0, vdot(e0, u), vdot(e0, v)},
                             {vdot(e1, u), vdot(e1, v), 0.0}, {0.0, vdot(e1, u), vdot(e1, v)},
                             {vdot(e2, u), vdot(e2, v), 0.0}, {0.0, vdot(e2, u), vdot(e2, v)}};
        for (int r = 0; r < 6; ++r)
            for (int cc = 0; cc < 3; ++cc) A[r + 6 * cc] = rows[r][cc];
        v3 na = ld(vn, t[0]), nb = ld(vn, t[1]), nc = ld(vn, t[2]);
        double rhs[6] = {vdot(vsub(nb, na), u), vdot(vsub(nb, na), v), vdot(vsub(nc, nb), u),
                         vdot(vsub(nc, nb), v), vdot(vsub(na, nc), u), vdot(vsub(na, nc), v)};
        double sol[3];
        fullpiv_solve(6, 3, A, rhs, sol);
        double mean = 0.5 * (sol[0] + sol[2]);
        for (int k = 0; k < 3; ++k) {
            kap[t[k]] += mean;
            w[t[k]] += 1.0;
        }
    }
    for (int64_t i = 0; i < n; ++i) kap[i] /= w[i];
    free(vn);
    free(w);
}

int orc_pot_t_multi(int64_t N, int64_t M, const double* x, const int64_t* tri, const double* grads,
                    double t, const orc_params* p, double* out) {
    /* split_by_loose_parts (Mesh.cpp:382-440): components in order of their smallest vertex;
     * inside a part vertices keep increasing global order, triangles increasing global order,
     * and every triangle ends rotated so that its largest global vertex comes first. */
    int64_t* comp = (int64_t*)malloc(sizeof(int64_t) * (size_t)N);
    int64_t* stack = (int64_t*)malloc(sizeof(int64_t) * (size_t)N);
    int64_t* local = (int64_t*)malloc(sizeof(int64_t) * (size_t)N);
    int64_t* pv = (int64_t*)malloc(sizeof(int64_t) * (size_t)N);
    int64_t* ptri = (int64_t*)malloc(sizeof(int64_t) * (size_t)(3 * M + 1));
    double* px = (double*)malloc(sizeof(double) * (size_t)(3 * N));
    double* kap = (double*)malloc(sizeof(double) * (size_t)N);
    csr_t c = {0, 0};
    int rc = -1;
    if (!comp || !stack || !local || !pv || !ptri || !px || !kap || build_csr(N, M, tri, &c)) goto done;
    for (int64_t i = 0; i < N; ++i) comp[i] = -1;
    const double field = p->field_amp * sin(p->field_omega * t + p->field_phase);
    int64_t ncomp = 0;
    for (int64_t s = 0; s < N; ++s) {
        if (comp[s] >= 0) continue;
        int64_t sp = 0;
        comp[s] = ncomp;
        stack[sp++] = s;
        while (sp) {
            int64_t v = stack[--sp];
            for (int64_t e = c.off[v]; e < c.off[v + 1]; ++e) {
                const int64_t* tt = tri + 3 * c.idx[e];
                for (int k = 0; k < 3; ++k)
                    if (comp[tt[k]] < 0) { comp[tt[k]] = ncomp; stack[sp++] = tt[k]; }
            }
        }
        ++ncomp;
    }
    for (int64_t cp = 0; cp < ncomp; ++cp) {
        int64_t n = 0, m = 0;
        for (int64_t i = 0; i < N; ++i)
            if (comp[i] == cp) { local[i] = n; pv[n] = i; st(px, n, ld(x, i)); ++n; }
        for (int64_t j = 0; j < M; ++j) {
            const int64_t* tt = tri + 3 * j;
            if (comp[tt[0]] != cp) continue;
            int r = 0;
            if (tt[1] > tt[r]) r = 1;
            if (tt[2] > tt[r]) r = 2;
            for (int k = 0; k < 3; ++k) ptri[3 * m + k] = local[tt[(r + k) % 3]];
            ++m;
        }
        double vol = orc_volume(n, m, px, ptri);
        if (p->sigma != 0.0) part_kappa(n, m, px, ptri, kap);
        else for (int64_t i = 0; i < n; ++i) kap[i] = 0.0;
        double gas = p->epsilon * pow(p->V0 / vol, p->gamma);
        for (int64_t i = 0; i < n; ++i) {
            v3 g = ld(grads, pv[i]);
            /* potential_t (Simulation.cpp:73-75) */
            out[pv[i]] = 2.0 * p->sigma * kap[i] + 0.5 * vdot(g, g) + p->p_inf - gas + field;
        }
    }
    rc = 0;
done:
    free(comp); free(stack); free(local); free(pv); free(ptri); free(px); free(kap); free_csr(&c);
    return rc;
}

static double get_dt(int64_t N, double dp, const double* vel, const double* pt, const orc_params* p) {
    double max_pot = 0.0, max_vel = 0.0;     /* Simulation.cpp:77-92 */
    for (int64_t i = 0; i < N; ++i) {
        max_pot = fmax(fabs(pt[i]), max_pot);
        v3 v = ld(vel, i);
        max_vel = fmax(vdot(v, v), max_vel);
    }
    max_vel = sqrt(max_vel);
    double dt = dp / (max_pot + p->dp_balance * max_vel);
    if (p->min_dt > 0.0) dt = fmin(dt, p->min_dt);
    return dt;
}

static int any_negative(int64_t N, const double* x) {
    for (int64_t i = 0; i < N; ++i)
        if (x[3 * i] < 0.0) return 1;
    return 0;
}

int orc_rk4_step(int64_t N, int64_t M, double* x, const int64_t* tri, double* phi, double* psi,
                 double* time, double dp, int32_t fixdt, const orc_params* p, double* dt_out) {
    if (any_negative(N, x)) return -2;
    const size_t n3 = (size_t)(3 * N), n1 = (size_t)N;
    double* buf = (double*)malloc(sizeof(double) * (n3 * 7 + n1 * 9));
    if (!buf) return -1;
    double *x1 = buf, *x2 = x1 + n3, *x3 = x2 + n3, *x4 = x3 + n3;
    double *k1x = x4 + n3, *k2x = k1x + n3, *k3x = k2x + n3;
    double *k4x = x2; /* reuses x2 once it is no longer needed? no: keep separate below */
    double *p1 = k3x + n3, *p2 = p1 + n1, *p3 = p2 + n1, *p4 = p3 + n1;
    double *k1p = p4 + n1, *k2p = k1p + n1, *k3p = k2p + n1, *k4p = k3p + n1, *nrm = k4p + n1;
    double* k4 = (double*)malloc(sizeof(double) * n3);
    double* vn = (double*)malloc(sizeof(double) * n3);
    (void)k4x;
    int rc = 0;
    if (!k4 || !vn) { rc = -1; goto done; }
    memcpy(x1, x, sizeof(double) * n3);
    memcpy(p1, phi, sizeof(double) * n1);
    const double t = *time;
    /* LinLinSim.cpp:200-238; every stage uses the step-start time t */
    if ((rc = orc_position_t(N, M, x1, tri, p1, p, k1x, NULL))) goto done;
    if ((rc = orc_pot_t_multi(N, M, x1, tri, k1x, t, p, k1p))) goto done;
    double dt = fixdt ? dp : get_dt(N, dp, k1x, k1p, p);
    for (size_t i = 0; i < n3; ++i) x2[i] = x1[i] + (0.5 * dt) * k1x[i];
    for (size_t i = 0; i < n1; ++i) p2[i] = p1[i] + (0.5 * dt) * k1p[i];
    if ((rc = orc_position_t(N, M, x2, tri, p2, p, k2x, NULL))) goto done;
    for (size_t i = 0; i < n3; ++i) x3[i] = x1[i] + (0.5 * dt) * k2x[i];
    if ((rc = orc_pot_t_multi(N, M, x2, tri, k2x, t, p, k2p))) goto done;
    for (size_t i = 0; i < n1; ++i) p3[i] = p1[i] + (0.5 * dt) * k2p[i];
    if ((rc = orc_position_t(N, M, x3, tri, p3, p, k3x, NULL))) goto done;
    for (size_t i = 0; i < n3; ++i) x4[i] = x1[i] + dt * k3x[i];
    if ((rc = orc_pot_t_multi(N, M, x3, tri, k3x, t, p, k3p))) goto done;
    for (size_t i = 0; i < n1; ++i) p4[i] = p1[i] + dt * k3p[i];
    if ((rc = orc_position_t(N, M, x4, tri, p4, p, k4, NULL))) goto done;
    if ((rc = orc_pot_t_multi(N, M, x4, tri, k4, t, p, k4p))) goto done;
    /* average = (k1 + 2 k2 + 2 k3 + k4) * (1/6) */
    double* avg = k1x;
    for (size_t i = 0; i < n3; ++i) avg[i] = (((k1x[i] + 2.0 * k2x[i]) + 2.0 * k3x[i]) + k4[i]) * (1.0 / 6.0);
    for (size_t i = 0; i < n1; ++i)
        phi[i] = p1[i] + (dt / 6.0) * (((k1p[i] + 2.0 * k2p[i]) + 2.0 * k3p[i]) + k4p[i]);
    /* nopenetration (LinLinSim.cpp:162-190); may modify avg[].x */
    const double eps = p->nopen_eps;
    for (int64_t i = 0; i < N; ++i) {
        for (int k = 0; k < 3; ++k) x[3 * i + k] = x1[3 * i + k] + dt * avg[3 * i + k];
        double cx = avg[3 * i];
        if (cx * dt < 0.0) {
            int flag = 0;
            double xpos = x1[3 * i];
            if (xpos < eps) {
                x[3 * i] = xpos * exp(cx / xpos * dt);
                flag = 1;
            } else {
                double te = (eps - xpos) / cx;
                if (fabs(te) < fabs(dt)) {
                    x[3 * i] = eps * exp(cx / eps * (dt - te));
                    flag = 1;
                }
            }
            if (flag) avg[3 * i] = (x[3 * i] - xpos) / dt;
        }
    }
    /* psi := average . vertex normal of the new mesh (LinLinSim.cpp:243-249) */
    orc_vertex_normals(N, M, x, tri, vn);
    for (int64_t i = 0; i < N; ++i) psi[i] = vdot(ld(avg, i), ld(vn, i));
    *time = t + dt;
    if (dt_out) *dt_out = dt;
    (void)nrm;
    if (any_negative(N, x)) rc = -2;
done:
    free(buf);
    free(k4);
    free(vn);
    return rc;
}

int orc_euler_step(int64_t N, int64_t M, double* x, const int64_t* tri, double* phi, double* time,
                   double dp, int32_t fixdt, const orc_params* p, double* dt_out) {
    const size_t n3 = (size_t)(3 * N), n1 = (size_t)N;
    double* g = (double*)malloc(sizeof(double) * n3);
    double* pt = (double*)malloc(sizeof(double) * n1);
    int rc = -1;
    if (!g || !pt) goto done;
    if ((rc = orc_position_t(N, M, x, tri, phi, p, g, NULL))) goto done;
    if ((rc = orc_pot_t_multi(N, M, x, tri, g, *time, p, pt))) goto done;
    double dt = fixdt ? dp : get_dt(N, dp, g, pt, p);
    for (size_t i = 0; i < n3; ++i) x[i] = x[i] + g[i] * dt;
    for (size_t i = 0; i < n1; ++i) phi[i] = phi[i] + dt * pt[i];
    *time += dt;
    if (dt_out) *dt_out = dt;
done:
    free(g);
    free(pt);
    return rc;
}
