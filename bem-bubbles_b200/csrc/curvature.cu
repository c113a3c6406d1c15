// Surface geometry that feeds discrete decisions: Max-1999 vertex normals and the per-triangle
// curvature tensor solved by complete-pivoting LU (Mesh.cpp:141-163, 256-319).  On symmetric meshes
// (an exact icosphere) the pivot search meets near-ties, and a pivot chosen differently gives another
// solution of the overdetermined 6x3 system.  This file is therefore compiled without fused
// multiply-add contraction (-fmad=false): every product and sum rounds as in the reference's C++, in
// the reference's operation order, so the same pivots are chosen.
#include <math.h>

#include "ctx.h"

namespace bemb {

struct g3 {
    double x, y, z;
};
__device__ __forceinline__ g3 ld3(const double* p, int i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ __forceinline__ void st3(double* p, int i, g3 v) {
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}
__device__ __forceinline__ g3 sub(g3 a, g3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ g3 cross(g3 a, g3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double dot(g3 a, g3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
using d3 = g3;

static inline int nb(int64_t n, int t) { return (int)((n + t - 1) / t); }

// Max-1999 vertex normals (Mesh.cpp:141-163)
__global__ void k_vertex_normals(int N, const double* __restrict__ x, const int* __restrict__ tri,
                                 const int* __restrict__ off, const int* __restrict__ idx, double* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double nx = 0, ny = 0, nz = 0;
    for (int e = off[i]; e < off[i + 1]; ++e) {
        int t = idx[e];
        int a = tri[3 * t], b = tri[3 * t + 1], c = tri[3 * t + 2];
        if (i == b) {
            int o = a;
            a = b;
            b = c;
            c = o;
        } else if (i == c) {
            int o = a;
            a = c;
            c = b;
            b = o;
        }
        d3 A = ld3(x, a);
        d3 B = sub(ld3(x, b), A), C = sub(ld3(x, c), A);
        d3 n = cross(B, C);
        double s = 1.0 / (dot(B, B) * dot(C, C));
        nx += n.x * s;
        ny += n.y * s;
        nz += n.z * s;
    }
    double inv = 1.0 / sqrt(nx * nx + ny * ny + nz * nz);
    st3(out, i, {nx * inv, ny * inv, nz * inv});
}

// Per-triangle curvature tensor (Rusinkiewicz least squares as written in Mesh.cpp:256-319):
// 6x3 system solved with complete pivoting, mean curvature 0.5*(x0+x2); averaged to vertices.
__global__ void k_tri_curvature(int M, const double* __restrict__ x, const int* __restrict__ tri,
                                const double* __restrict__ vn, double* __restrict__ tk) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M) return;
    int ia = tri[3 * t], ib = tri[3 * t + 1], ic = tri[3 * t + 2];
    d3 e0 = sub(ld3(x, ib), ld3(x, ia)), e1 = sub(ld3(x, ic), ld3(x, ib)), e2 = sub(ld3(x, ia), ld3(x, ic));
    double iu = 1.0 / sqrt(dot(e0, e0));
    d3 u = {e0.x * iu, e0.y * iu, e0.z * iu};
    d3 nr = cross(e0, e1);
    double inr = 1.0 / sqrt(dot(nr, nr));
    nr = {nr.x * inr, nr.y * inr, nr.z * inr};
    d3 v = cross(nr, u);
    double A[6][3] = {{dot(e0, u), dot(e0, v), 0.0}, {0.0, dot(e0, u), dot(e0, v)},
                      {dot(e1, u), dot(e1, v), 0.0}, {0.0, dot(e1, u), dot(e1, v)},
                      {dot(e2, u), dot(e2, v), 0.0}, {0.0, dot(e2, u), dot(e2, v)}};
    d3 na = ld3(vn, ia), nb = ld3(vn, ib), nc = ld3(vn, ic);
    double rhs[6] = {dot(sub(nb, na), u), dot(sub(nb, na), v), dot(sub(nc, nb), u),
                     dot(sub(nc, nb), v), dot(sub(na, nc), u), dot(sub(na, nc), v)};
    int rowp[6] = {0, 1, 2, 3, 4, 5}, colq[3] = {0, 1, 2};
    int rank = 3;
    double maxpiv = 0.0;
    bool degenerate = false;
    for (int k = 0; k < 3; ++k) {
        int pr = k, pc = k;
        double best = -1.0;
        for (int j = k; j < 3; ++j)
            for (int i = k; i < 6; ++i) {
                double a = fabs(A[i][j]);
                if (a > best) {
                    best = a;
                    pr = i;
                    pc = j;
                }
            }
        if (best == 0.0) {
            rank = k;
            degenerate = true;
            break;
        }
        maxpiv = fmax(maxpiv, best);
        if (pr != k) {
            for (int j = 0; j < 3; ++j) {
                double tmp = A[k][j];
                A[k][j] = A[pr][j];
                A[pr][j] = tmp;
            }
            int tmp = rowp[k];
            rowp[k] = rowp[pr];
            rowp[pr] = tmp;
        }
        if (pc != k) {
            for (int i = 0; i < 6; ++i) {
                double tmp = A[i][k];
                A[i][k] = A[i][pc];
                A[i][pc] = tmp;
            }
            int tmp = colq[k];
            colq[k] = colq[pc];
            colq[pc] = tmp;
        }
        double piv = A[k][k];
        for (int i = k + 1; i < 6; ++i) A[i][k] /= piv;
        for (int j = k + 1; j < 3; ++j)
            for (int i = k + 1; i < 6; ++i) A[i][j] -= A[i][k] * A[k][j];
    }
    if (!degenerate) {
        double thr = 2.220446049250313e-16 * 3.0;
        int r = 0;
        for (int k = 0; k < 3; ++k)
            if (fabs(A[k][k]) > thr * maxpiv) ++r;
        rank = r;
    }
    double c[6], sol[3] = {0, 0, 0};
    for (int i = 0; i < 6; ++i) c[i] = rhs[rowp[i]];
    for (int j = 0; j < 3; ++j)
        for (int i = j + 1; i < 3; ++i) c[i] -= A[i][j] * c[j];
    for (int j = rank - 1; j >= 0; --j) {
        c[j] /= A[j][j];
        for (int i = 0; i < j; ++i) c[i] -= A[i][j] * c[j];
    }
    for (int i = 0; i < rank; ++i) sol[colq[i]] = c[i];
    tk[t] = 0.5 * (sol[0] + sol[2]);
}

__global__ void k_vertex_avg(int N, const int* __restrict__ off, const int* __restrict__ idx,
                             const double* __restrict__ tk, double* __restrict__ kap) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double s = 0.0, w = 0.0;
    for (int e = off[i]; e < off[i + 1]; ++e) {
        s += tk[idx[e]];
        w += 1.0;
    }
    kap[i] = s / w;
}

void launch_vertex_normals(Ctx& c, const double* x, double* out, cudaStream_t s) {
    KLAUNCH(), k_vertex_normals<<<nb(c.topo.N, 128), 128, 0, s>>>((int)c.topo.N, x, c.topo.tri, c.topo.csr_off,
                                                        c.topo.csr_idx, out);
}
void launch_curvature(Ctx& c, const double* x, double* kap, cudaStream_t s) {
    // curvatures are computed on the loose parts, whose triangles carry the split's rotation
    launch_vertex_normals(c, x, c.vn, s);
    KLAUNCH(), k_tri_curvature<<<nb(c.topo.M, 128), 128, 0, s>>>((int)c.topo.M, x, c.topo.tri_rot, c.vn, c.tk);
    KLAUNCH(), k_vertex_avg<<<nb(c.topo.N, 128), 128, 0, s>>>((int)c.topo.N, c.topo.csr_off, c.topo.csr_idx, c.tk, kap);
}

}  // namespace bemb
