// Ray casting of the remesh projection on the device: trace_mesh (Bem/Mesh/MeshManip.cpp:1250-1283).
//
// After the topology edits of a remesh, every new vertex is projected onto the old surface along its
// vertex normal (project_and_interpolate, MeshManip.cpp:1426-1697): the ray p + s*d is intersected
// with the plane of every old triangle, and among the triangles whose (closed) interior contains the
// intersection the one with the smallest |s| is taken, the first in triangle order on ties.  The host
// scan is O(P * M); here one warp takes one ray, its lanes stride over the triangles in increasing
// order keeping their own first minimum, and a butterfly over (|s|, index) picks the global first
// minimum -- the same triangle the sequential scan keeps.
//
// Compiled without FMA contraction: every quantity rounds as the host C++ does (differences, cross
// and dot products, one division), so hit points and the chosen triangles are bit-identical to the
// reference's.  Rays that hit nothing report ok = 0, hit (0,0,0) and triangle 0, as the reference's
// caller then sees.
#include <math.h>

#include "ctx.h"

namespace bemb {

struct v3 {
    double x, y, z;
};
__device__ __forceinline__ v3 ldv(const double* p, int64_t i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ __forceinline__ v3 sub(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ v3 cross(v3 a, v3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

__global__ void k_trace_mesh(int64_t P, const double* __restrict__ x, const int64_t* __restrict__ tri, int64_t M,
                             const double* __restrict__ pos, const double* __restrict__ dir, double* __restrict__ hit,
                             int64_t* __restrict__ tri_out, int32_t* __restrict__ ok) {
    const int64_t ray = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (ray >= P) return;
    const v3 p = ldv(pos, ray), d = ldv(dir, ray);
    double best = -1.0;  // |s| of this lane's pick; negative: none yet
    int64_t bj = -1;
    v3 bx{0.0, 0.0, 0.0};
    for (int64_t j = lane; j < M; j += 32) {
        const v3 A = ldv(x, tri[3 * j]), B = ldv(x, tri[3 * j + 1]), C = ldv(x, tri[3 * j + 2]);
        const v3 a = sub(B, A), b = sub(C, B), c = sub(A, C);
        const v3 n = cross(a, b);
        const double s = dot(n, sub(A, p)) / dot(n, d);
        const v3 q = {p.x + s * d.x, p.y + s * d.y, p.z + s * d.z};
        if (fabs(s) < best || best < 0.0) {
            if (dot(cross(sub(A, q), a), n) >= 0 && dot(cross(sub(B, q), b), n) >= 0 &&
                dot(cross(sub(C, q), c), n) >= 0) {
                best = fabs(s);
                bj = j;
                bx = q;
            }
        }
    }
    // first minimum over the lanes: smallest |s|, then smallest triangle index
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const long long oj = __shfl_xor_sync(0xffffffffu, (long long)bj, o);
        const double ox = __shfl_xor_sync(0xffffffffu, bx.x, o);
        const double oy = __shfl_xor_sync(0xffffffffu, bx.y, o);
        const double oz = __shfl_xor_sync(0xffffffffu, bx.z, o);
        bool take;
        if (oj < 0)
            take = false;
        else if (bj < 0)
            take = true;
        else
            take = ob < best || (ob == best && oj < bj);
        if (take) {
            best = ob;
            bj = oj;
            bx = {ox, oy, oz};
        }
    }
    if (lane) return;
    const bool found = bj >= 0;
    hit[3 * ray] = found ? bx.x : 0.0;
    hit[3 * ray + 1] = found ? bx.y : 0.0;
    hit[3 * ray + 2] = found ? bx.z : 0.0;
    tri_out[ray] = found ? bj : 0;
    ok[ray] = found ? 1 : 0;
}

int trace_mesh(Ctx& c, int64_t Nv, const double* verts, int64_t M, const int64_t* trigs, int64_t P, const double* pos,
               const double* dir, double* hit, int64_t* tri_out, int32_t* ok) {
    // one allocation for the whole call: vertices, triangles, rays, results
    const size_t nb = sizeof(double) * (size_t)(3 * Nv + 9 * P) + sizeof(int64_t) * (size_t)(3 * M + P) +
                      sizeof(int32_t) * (size_t)P + 64;
    if (c.trace_cap < nb) {
        cudaFree(c.trace_buf);
        c.trace_buf = nullptr;
        c.trace_cap = 0;
        if (cudaMalloc(&c.trace_buf, nb) != cudaSuccess) return c.fail(BEM_ERR_NOMEM, "trace: device buffers");
        c.trace_cap = nb;
    }
    char* b = (char*)c.trace_buf;
    double* dx = (double*)b;
    double* dpos = dx + 3 * Nv;
    double* ddir = dpos + 3 * P;
    double* dhit = ddir + 3 * P;
    int64_t* dtri = (int64_t*)(dhit + 3 * P);
    int64_t* dout = dtri + 3 * M;
    int32_t* dok = (int32_t*)(dout + P);
    cudaStream_t s = c.stream;
    BEM_CUDA(c, cudaMemcpyAsync(dx, verts, sizeof(double) * 3 * Nv, cudaMemcpyHostToDevice, s));
    BEM_CUDA(c, cudaMemcpyAsync(dtri, trigs, sizeof(int64_t) * 3 * M, cudaMemcpyHostToDevice, s));
    BEM_CUDA(c, cudaMemcpyAsync(dpos, pos, sizeof(double) * 3 * P, cudaMemcpyHostToDevice, s));
    BEM_CUDA(c, cudaMemcpyAsync(ddir, dir, sizeof(double) * 3 * P, cudaMemcpyHostToDevice, s));
    const int threads = 256;
    const int64_t blocks = (32 * P + threads - 1) / threads;
    KLAUNCH(), k_trace_mesh<<<(unsigned)blocks, threads, 0, s>>>(P, dx, dtri, M, dpos, ddir, dhit, dout, dok);
    BEM_CUDA(c, cudaGetLastError());
    BEM_CUDA(c, cudaMemcpyAsync(hit, dhit, sizeof(double) * 3 * P, cudaMemcpyDeviceToHost, s));
    BEM_CUDA(c, cudaMemcpyAsync(tri_out, dout, sizeof(int64_t) * P, cudaMemcpyDeviceToHost, s));
    BEM_CUDA(c, cudaMemcpyAsync(ok, dok, sizeof(int32_t) * P, cudaMemcpyDeviceToHost, s));
    BEM_CUDA(c, cudaStreamSynchronize(s));
    return BEM_OK;
}

}  // namespace bemb
