// Pinned contact line: the reference's ColocSimPin (Bem/Simulation/ColocSimPin.cpp:25-194) on the
// device.  The last n_pin vertices of the mesh lie on the wall x = 0 (the contact line of a bubble
// sitting on the wall).  psi is imposed (zero) there and their potential is the unknown, so after the
// 4 pi rule the pinned columns of G and H are exchanged with a sign change (ColocSimPin.cpp:113-117):
//   G(:,j) <- -H(:,j),  H(:,j) <- -G(:,j)          (j pinned)
// and the right-hand side H*pot takes the values at pinned vertices from the stored psi
// (ColocSimPin.cpp:146-148).  After the solve the pinned vertices move along the wall with the
// drift velocity of the contact angle (ColocSimPin.cpp:126-136, 175-186) and the solved unknowns,
// their potential, replace the stage potential there (ColocSimPin.cpp:188).
//
// Compiled without FMA contraction: the drift law and the in-wall normal round every operation as
// the reference's C++ does.  All three kernels are O(N * n_pin) or O(n_pin) next to the O(N^2)
// assembly; the exchange reads and writes the n_pin columns once, coalesced along the rows.
#include "ctx.h"

namespace bemb {

// potz = pot with the pinned entries zeroed: the assembly's fused H*pot then covers the free
// columns only, and the pinned columns' share is added after the exchange.
__global__ void k_pin_zero(int N, int first, const double* __restrict__ pot, double* __restrict__ potz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) potz[i] = i >= first ? 0.0 : pot[i];
}

// Column exchange of the pinned columns (after the 4 pi rule) and b(i) += sum_j G'(i,j) * v(j) over
// pinned j with G' the exchanged H' = -G: b = H' * pot with pot(j) = v(j) on the pinned vertices.
// One thread per row; the pinned columns are read along the rows (column-major storage).
__global__ void k_pin_exchange(int N, int first, double* __restrict__ G, double* __restrict__ H,
                               const double* __restrict__ v, double* __restrict__ b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double acc = 0.0;
    for (int j = first; j < N; ++j) {
        const size_t o = (size_t)j * N + i;
        const double g = G[o], h = H[o];
        G[o] = -h;
        H[o] = -g;
        acc += (-g) * v[j];
    }
    if (b) b[i] += acc;
}

// drift_velocity (ColocSimPin.cpp:126-136): beta (cos_eq - c) + c_nl c^3 / (c^2 - 1)
__device__ __forceinline__ double drift(double c, double beta, double ceq, double cnl) {
    return beta * (ceq - c) + cnl * (c * c * c) / (c * c - 1.0);
}

// Pinned vertices after the solve (ColocSimPin.cpp:175-189): velocity = in-wall part of the vertex
// normal, normalised, times the drift velocity of cos(theta) = normal.x; pot <- solved unknown.
__global__ void k_pin_finish(int N, int first, const double* __restrict__ vn, const double* __restrict__ psil,
                             double beta, double ceq, double cnl, double* __restrict__ vel,
                             double* __restrict__ pot) {
    const int i = first + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double c = vn[3 * i];
    double ny = vn[3 * i + 1], nz = vn[3 * i + 2];
    const double s = 1.0 / sqrt((0.0 * 0.0 + ny * ny) + nz * nz);  // vec3::normalize with x = 0
    ny *= s;
    nz *= s;
    const double d = drift(c, beta, ceq, cnl);
    vel[3 * i] = 0.0 * d;
    vel[3 * i + 1] = ny * d;
    vel[3 * i + 2] = nz * d;
    pot[i] = psil[i];
}

static inline int blocks(int64_t n, int t) { return (int)((n + t - 1) / t); }

void launch_pin_zero(Ctx& c, const double* pot, double* potz, cudaStream_t s) {
    const int N = (int)c.topo.N;
    KLAUNCH(), k_pin_zero<<<blocks(N, 256), 256, 0, s>>>(N, (int)(N - c.n_pin), pot, potz);
}

void launch_pin_exchange(Ctx& c, const double* v, double* b, cudaStream_t s) {
    const int N = (int)c.topo.N;
    KLAUNCH(), k_pin_exchange<<<blocks(N, 128), 128, 0, s>>>(N, (int)(N - c.n_pin), c.G, c.H, v, b);
}

void launch_pin_finish(Ctx& c, const double* x, double* vel, double* pot, cudaStream_t s) {
    const int N = (int)c.topo.N;
    launch_vertex_normals(c, x, c.vn, s);
    KLAUNCH(), k_pin_finish<<<blocks(c.n_pin, 128), 128, 0, s>>>(N, (int)(N - c.n_pin), c.vn, c.psil, c.pin_beta,
                                                                c.pin_cos_eq, c.pin_cnl, vel, pot);
}

}  // namespace bemb
