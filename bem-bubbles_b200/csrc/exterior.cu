// Potential off the surface (LinLinSim::exterior_pot / compute_exterior_pot, LinLinSim.cpp:440-485,
// with Integrator::get_exterior_potential, Integrator.cpp:287-305): at every evaluation point x, the
// sum over triangles of (-G_k psi_k + H_k phi_k) / (4 pi) with the 19-point rule and no wall image.
//
// Per triangle the basis weights are folded with psi, phi, the area and 1/(4 pi) once:
//   A_q = -area w_q sum_k beta_k(q) psi_k / (4 pi),  B_q = -area w_q sum_k beta_k(q) phi_k / (4 pi),
// so that a (point, triangle) pair costs sum_q A_q / r_q + B_q dn / r_q^3, dn = n.a - n.x (all
// quadrature points lie in the triangle's plane).  One thread per point walks the triangles staged
// in shared memory; triangle chunks spread over gridDim.y when there are few points, and the chunk
// sums are added in a fixed order (deterministic).
#include <math.h>

#include <algorithm>
#include <atomic>

#include "ctx.h"

namespace bemb {

__constant__ double e_q19[19][3];

constexpr int EREC = 100;  // y_q (57), A_q (19), B_q (19), n (3), n.a (1), pad
constexpr int ETC = 16;    // triangles staged per round
constexpr int ETHREADS = 128;

static void upload_ext_constants() {
    static std::atomic<uint64_t> done{0};
    once_per_device(done, [] {
        QuadTables t;
        quad_tables(t);
        return cudaMemcpyToSymbol(e_q19, t.q19, sizeof(t.q19)) == cudaSuccess;
    });
}

__global__ void k_ext_records(int M, const double* __restrict__ x, const int* __restrict__ tri,
                              const double* __restrict__ phi, const double* __restrict__ psi, double* __restrict__ rec) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M) return;
    const int ia = tri[3 * t], ib = tri[3 * t + 1], ic = tri[3 * t + 2];
    const double ax = x[3 * ia], ay = x[3 * ia + 1], az = x[3 * ia + 2];
    const double abx = x[3 * ib] - ax, aby = x[3 * ib + 1] - ay, abz = x[3 * ib + 2] - az;
    const double bcx = x[3 * ic] - x[3 * ib], bcy = x[3 * ic + 1] - x[3 * ib + 1], bcz = x[3 * ic + 2] - x[3 * ib + 2];
    const double nx = aby * bcz - abz * bcy, ny = abz * bcx - abx * bcz, nz = abx * bcy - aby * bcx;
    const double area = sqrt(nx * nx + ny * ny + nz * nz);
    const double ia_ = 1.0 / area;
    double* r = rec + (size_t)t * EREC;
    const double s = -area / (4.0 * 3.14159265358979323846);
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        const double u = e_q19[q][0], v = e_q19[q][1], w = e_q19[q][2];
        r[3 * q] = (ax + u * abx) + v * bcx;
        r[3 * q + 1] = (ay + u * aby) + v * bcy;
        r[3 * q + 2] = (az + u * abz) + v * bcz;
        const double b0 = 1.0 - u, b1 = u - v, b2 = v;
        r[57 + q] = s * w * ((b0 * psi[ia] + b1 * psi[ib]) + b2 * psi[ic]);
        r[76 + q] = s * w * ((b0 * phi[ia] + b1 * phi[ib]) + b2 * phi[ic]);
    }
    r[95] = nx * ia_;
    r[96] = ny * ia_;
    r[97] = nz * ia_;
    r[98] = ax * r[95] + ay * r[96] + az * r[97];
    r[99] = 0.0;
}

__global__ void __launch_bounds__(ETHREADS) k_exterior(int P, const double* __restrict__ pts, int M, int tris_per_chunk,
                                                        const double* __restrict__ rec, double* __restrict__ part) {
    __shared__ __align__(16) double srec[ETC * EREC];
    const int i = blockIdx.x * ETHREADS + threadIdx.x;
    const int t0 = blockIdx.y * tris_per_chunk, t1 = min(M, t0 + tris_per_chunk);
    double x0 = 0.0, x1 = 0.0, x2 = 0.0;
    if (i < P) {
        x0 = pts[3 * i];
        x1 = pts[3 * i + 1];
        x2 = pts[3 * i + 2];
    }
    double val = 0.0;
    for (int c0 = t0; c0 < t1; c0 += ETC) {
        const int cnt = min(ETC, t1 - c0);
        __syncthreads();
        for (int e = threadIdx.x; e < cnt * (EREC / 2); e += ETHREADS) {
            const int tt = e / (EREC / 2), w = e - tt * (EREC / 2);
            reinterpret_cast<double2*>(srec + tt * EREC)[w] =
                reinterpret_cast<const double2*>(rec + (size_t)(c0 + tt) * EREC)[w];
        }
        __syncthreads();
        if (i < P) {
            for (int tt = 0; tt < cnt; ++tt) {
                const double* r = srec + tt * EREC;
                const double dn = r[98] - ((r[95] * x0 + r[96] * x1) + r[97] * x2);
                double sg = 0.0, sh = 0.0;
#pragma unroll
                for (int q = 0; q < 19; ++q) {
                    const double zx = r[3 * q] - x0, zy = r[3 * q + 1] - x1, zz = r[3 * q + 2] - x2;
                    const double inv = 1.0 / sqrt(zx * zx + zy * zy + zz * zz);
                    sg = fma(r[57 + q], inv, sg);
                    sh = fma(r[76 + q], inv * inv * inv, sh);
                }
                val += fma(sh, dn, sg);
            }
        }
    }
    if (i < P) part[(size_t)blockIdx.y * P + i] = val;
}

__global__ void k_ext_final(int P, int nch, const double* __restrict__ part, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    double s = 0.0;
    for (int c = 0; c < nch; ++c) s += part[(size_t)c * P + i];
    out[i] = s;
}

// out_dev[P] = exterior potential at pts_dev (P x 3, device) from the surface phi, psi (device, N).
int exterior_potential(Ctx& c, int64_t P, const double* pts_dev, const double* phi, const double* psi,
                       double* out_dev, cudaStream_t s) {
    upload_ext_constants();
    const int M = (int)c.topo.M;
    const int pb = (int)((P + ETHREADS - 1) / ETHREADS);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
    // triangle chunks: enough CTAs for about four per SM, whole rounds of ETC triangles each
    int nch = std::max(1, std::min((4 * sms + pb - 1) / pb, (M + ETC - 1) / ETC));
    const int per = ((M + nch - 1) / nch + ETC - 1) / ETC * ETC;
    nch = (M + per - 1) / per;
    double *rec = nullptr, *part = nullptr;
    if (cudaMalloc(&rec, sizeof(double) * EREC * (size_t)M) != cudaSuccess ||
        cudaMalloc(&part, sizeof(double) * (size_t)nch * (size_t)P) != cudaSuccess) {
        cudaFree(rec);
        return c.fail(BEM_ERR_NOMEM, "exterior potential: work buffers");
    }
    KLAUNCH(), k_ext_records<<<(M + 127) / 128, 128, 0, s>>>(M, c.x, c.topo.tri, phi, psi, rec);
    KLAUNCH(), k_exterior<<<dim3(pb, nch), ETHREADS, 0, s>>>((int)P, pts_dev, M, per, rec, part);
    KLAUNCH(), k_ext_final<<<pb, ETHREADS, 0, s>>>((int)P, nch, part, out_dev);
    const cudaError_t e = cudaStreamSynchronize(s);
    cudaFree(rec);
    cudaFree(part);
    if (e != cudaSuccess) return c.fail(BEM_ERR_CUDA, std::string("exterior potential: ") + cudaGetErrorString(e));
    return BEM_OK;
}

}  // namespace bemb
