// Trailing update of the blocked FP64 LU (Simulation::solve_system with set_bcgstab(false): Eigen's
// PartialPivLU, Simulation.cpp:57-60) on the FP64 tensor cores.
//
// After the panel of columns [k0, k0 + nb) is factored and U12 = L11^-1 A12 is in place, the trailing
// matrix takes A22 -= L21 U12 (rows and columns from k0 + nb).  Each CTA owns a 128 x 64 tile of
// A22: the panel's L21 rows (128 x nb) and U12 columns (nb x 64) are staged in shared memory, and
// eight warps each accumulate a 32 x 32 block with mma.sync m8n8k4 FP64 (DMMA: 8 x 8 x 4 per
// instruction), K = nb <= 64 in steps of 4, starting from the tile's own entries.  The tile of A22 is
// read and written once.
//
// m8n8k4 FP64 fragments (PTX ISA, mma.m8n8k4 .f64): lane l, g = l / 4, t = l % 4 holds A[g][t]
// (8 x 4, row-major), B[t][g] (4 x 8, column-major) and C/D[g][2t], C/D[g][2t + 1].
#include "ctx.h"

namespace bemb {

namespace {

constexpr int UB_M = 128, UB_N = 64, UB_K = 64;  // tile of A22, widest panel
constexpr int UA_LD = UB_M + 4;                  // sA[k][row]: +4 doubles, conflict-free fragment reads
constexpr int UBB_LD = UB_K + 4;                 // sB[col][k]
constexpr size_t UPD_SMEM = sizeof(double) * ((size_t)UB_K * UA_LD + (size_t)UB_N * UBB_LD);

__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(256, 2) k_lu_update(int n, int k0, int nb, double* __restrict__ A) {
    extern __shared__ __align__(16) double usm[];
    double* sA = usm;                       // [UB_K][UA_LD]: L21 rows of the tile, k-major
    double* sB = usm + UB_K * UA_LD;        // [UB_N][UBB_LD]: U12 columns of the tile, k contiguous
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int k1 = k0 + nb;
    const int r0 = k1 + blockIdx.x * UB_M, c0 = k1 + blockIdx.y * UB_N;
    const int kpad = (nb + 3) & ~3;
    const int g = lane >> 2, t = lane & 3;
    const int wr = (w & 3) * 32, wc = (w >> 2) * 32;  // the warp's 32 x 32 block in the tile
    // the accumulators start as the thread's 32 entries of the A22 tile and take -L21 U12 (the staged
    // L21 is negated), so the tile is read once, with every load in flight together
    double acc[4][4][2];
    const int gr0 = r0 + wr + g, gc0 = c0 + wc + 2 * t;
    double* const tile = A + (size_t)gc0 * n + gr0;  // entry (mi, ni, h) at (ni * 8 + h) * n + mi * 8
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const double* col = tile + (size_t)(ni * 8 + h) * n;
            const bool cok = gc0 + ni * 8 + h < n;
#pragma unroll
            for (int mi = 0; mi < 4; ++mi) acc[mi][ni][h] = (cok && gr0 + mi * 8 < n) ? col[mi * 8] : 0.0;
        }
    // staging, 8 independent loads of the thread before their stores
#pragma unroll
    for (int q = 0; q < UB_K * UB_M / 256; q += 8) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = tid + 256 * (q + u), k = e / UB_M, gr = r0 + (e - k * UB_M);
            v[u] = (k < nb && gr < n) ? -A[(size_t)(k0 + k) * n + gr] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = tid + 256 * (q + u), k = e / UB_M;
            if (k < kpad) sA[k * UA_LD + (e - k * UB_M)] = v[u];
        }
    }
#pragma unroll
    for (int q = 0; q < UB_N * UB_K / 256; q += 8) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = tid + 256 * (q + u), cc = e / UB_K, k = e - cc * UB_K, gc = c0 + cc;
            v[u] = (k < nb && gc < n) ? A[(size_t)gc * n + k0 + k] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = tid + 256 * (q + u), cc = e / UB_K;
            sB[cc * UBB_LD + (e - cc * UB_K)] = v[u];
        }
    }
    __syncthreads();
    for (int kk = 0; kk < kpad; kk += 4) {
        double a[4], b[4];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi) a[mi] = sA[(kk + t) * UA_LD + wr + mi * 8 + g];
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) b[ni] = sB[(wc + ni * 8 + g) * UBB_LD + kk + t];
#pragma unroll
        for (int mi = 0; mi < 4; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) dmma_8x8x4(acc[mi][ni][0], acc[mi][ni][1], a[mi], b[ni]);
    }
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            double* col = tile + (size_t)(ni * 8 + h) * n;
            if (gc0 + ni * 8 + h >= n) continue;
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
                if (gr0 + mi * 8 < n) col[mi * 8] = acc[mi][ni][h];
        }
}

}  // namespace

// A22 -= L21 U12 for the panel [k0, k0 + nb) of the column-major n x n matrix A (nb <= 64).
int lu_update(Ctx& c, int n, int k0, int nb, double* A, cudaStream_t s) {
    const int rest = n - k0 - nb;
    if (rest <= 0) return BEM_OK;
    if (nb > UB_K) return c.fail(BEM_ERR_ARG, "LU trailing update: panel wider than 64 columns");
    static std::atomic<uint64_t> attr{0};
    if (!once_per_device(attr, [] {
            return cudaFuncSetAttribute(k_lu_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)UPD_SMEM) ==
                   cudaSuccess;
        }))
        return c.fail(BEM_ERR_CUDA, "LU trailing update: shared-memory attribute refused");
    const dim3 grid((rest + UB_M - 1) / UB_M, (rest + UB_N - 1) / UB_N);
    KLAUNCH(), k_lu_update<<<grid, 256, UPD_SMEM, s>>>(n, k0, nb, A);
    return BEM_OK;
}

}  // namespace bemb
