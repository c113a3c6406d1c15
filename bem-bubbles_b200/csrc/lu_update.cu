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

constexpr int UB_N = 64, UB_K = 64;  // tile columns of A22, widest panel
constexpr int UBB_LD = UB_K + 4;     // sB[col][k]: +4 doubles, conflict-free fragment reads
// tile rows UB_M = 32 * WM (WM warps along the rows, two along the columns); sA[k][row] with +4 doubles
template <int WM>
constexpr size_t upd_smem() {
    return sizeof(double) * ((size_t)UB_K * (32 * WM + 4) + (size_t)UB_N * UBB_LD);
}

__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// columns [cb, ce) of A22 (cb >= k0 + nb)
template <int WM>
__global__ void __launch_bounds__(64 * WM, 2) k_lu_update(int n, int k0, int nb, int cb, int ce,
                                                           double* __restrict__ A) {
    constexpr int UB_M = 32 * WM, UA_LD = UB_M + 4, NT = 64 * WM;
    extern __shared__ __align__(16) double usm[];
    double* sA = usm;                       // [UB_K][UA_LD]: L21 rows of the tile, k-major
    double* sB = usm + UB_K * UA_LD;        // [UB_N][UBB_LD]: U12 columns of the tile, k contiguous
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int k1 = k0 + nb;
    const int r0 = k1 + blockIdx.x * UB_M, c0 = cb + blockIdx.y * UB_N;
    const int kpad = (nb + 3) & ~3;
    const int g = lane >> 2, t = lane & 3;
    const int wr = (w % WM) * 32, wc = (w / WM) * 32;  // the warp's 32 x 32 block in the tile
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
            const bool cok = gc0 + ni * 8 + h < ce;
#pragma unroll
            for (int mi = 0; mi < 4; ++mi) acc[mi][ni][h] = (cok && gr0 + mi * 8 < n) ? col[mi * 8] : 0.0;
        }
    // staging, 8 independent loads of the thread before their stores
#pragma unroll
    for (int q = 0; q < UB_K * UB_M / NT; q += 8) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = tid + NT * (q + u), k = e / UB_M, gr = r0 + (e - k * UB_M);
            v[u] = (k < nb && gr < n) ? -A[(size_t)(k0 + k) * n + gr] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = tid + NT * (q + u), k = e / UB_M;
            if (k < kpad) sA[k * UA_LD + (e - k * UB_M)] = v[u];
        }
    }
#pragma unroll
    for (int q = 0; q < UB_N * UB_K / NT; q += 8) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = tid + NT * (q + u), cc = e / UB_K, k = e - cc * UB_K, gc = c0 + cc;
            v[u] = (k < nb && gc < ce) ? A[(size_t)gc * n + k0 + k] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = tid + NT * (q + u), cc = e / UB_K;
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
            if (gc0 + ni * 8 + h >= ce) continue;
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
                if (gr0 + mi * 8 < n) col[mi * 8] = acc[mi][ni][h];
        }
}

}  // namespace

template <int WM>
static bool upd_prepare() {
    static std::atomic<uint64_t> attr{0};
    return once_per_device(attr, [] {
        return cudaFuncSetAttribute(k_lu_update<WM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)upd_smem<WM>()) == cudaSuccess;
    });
}

// A22 -= L21 U12 for the panel [k0, k0 + nb) of the column-major n x n matrix A (nb <= 64), on the
// columns [cb, ce) of A22 (all of them by default).  narrow: 64-row tiles of 128 threads and 70 KB of
// shared memory, so that a CTA of the cluster panel fits on the same SM (the look-ahead runs the next
// panel beside this update); else 128-row tiles of 256 threads and 102 KB.
int lu_update(Ctx& c, int n, int k0, int nb, double* A, cudaStream_t s, int cb, int ce, bool narrow) {
    if (cb < 0) cb = k0 + nb;
    if (ce < 0) ce = n;
    const int rest = n - k0 - nb, cols = ce - cb;
    if (rest <= 0 || cols <= 0) return BEM_OK;
    if (nb > UB_K) return c.fail(BEM_ERR_ARG, "LU trailing update: panel wider than 64 columns");
    if (narrow) {
        if (!upd_prepare<2>()) return c.fail(BEM_ERR_CUDA, "LU trailing update: shared-memory attribute refused");
        const dim3 grid((rest + 63) / 64, (cols + UB_N - 1) / UB_N);
        KLAUNCH(), k_lu_update<2><<<grid, 128, upd_smem<2>(), s>>>(n, k0, nb, cb, ce, A);
    } else {
        if (!upd_prepare<4>()) return c.fail(BEM_ERR_CUDA, "LU trailing update: shared-memory attribute refused");
        const dim3 grid((rest + 127) / 128, (cols + UB_N - 1) / UB_N);
        KLAUNCH(), k_lu_update<4><<<grid, 256, upd_smem<4>(), s>>>(n, k0, nb, cb, ce, A);
    }
    return BEM_OK;
}

}  // namespace bemb
