// Approximate inverse X ~ G^-1 for the mixed solver by blocked Gauss-Jordan elimination with row
// partial pivoting, in FP32 storage, the rank-nb updates as split-precision (BF16x3) tcgen05 GEMMs.
//
// Panel by panel (nb = 64 columns [k0, k1)), on the FP32 copy A of G:
//   * pivots: the panel's LU with row partial pivoting over rows k0..n-1 (the FP64 panel kernels of
//     lu_panel.cu on an FP64 copy of the panel), the same row choice as unblocked Gauss-Jordan;
//   * the interchanges applied to whole rows of A, and to the permutation perm;
//   * with B the panel's rows and O the others, b the panel's columns and o the others:
//       W = A_Bb^-1                       (in-place Gauss-Jordan of the pivoted block, FP64, one CTA)
//       P = -A_Ob W                       (tcgen05 GEMM, n x nb x nb)
//       R' = W A_Bo                       (tcgen05 GEMM, nb x n x nb)
//       A_Oo += P A_Bo                    (tcgen05 GEMM, n x n x nb, accumulating into A)
//       A_Ob = P, A_Bo = R', A_Bb = W.
//     The operands are masked (B rows of P, b columns of A_Bo are zero), so the accumulating GEMM
//     runs over the whole matrix and adds zero in the panel's rows and columns.
// At the end A holds (Pi G)^-1 for the row permutation Pi, and X[:, perm[j]] = A[:, j] is G^-1.
// Each product carries about 16 bits per operand (bf16 hi + lo), so X is accurate to about cond(G)
// times 1e-5; the caller polishes it with Newton-Schulz steps (X <- X (2I - G X)) against G.
// Cost: 2 n^3 tensor flops x 3 (BF16x3) and one read-modify-write of A per panel, against
// Newton-Schulz from scratch's 2 n^3 x 3 per step over about log2(cond(G)) steps.
#include <cuda_bf16.h>

#include <algorithm>

#include "ctx.h"

namespace bemb {

namespace {

constexpr int GJ_NB = 64;  // panel width (the FP64 panel kernels' widest)

// FP64 copy of the panel: Pm (m x nb, column-major, m = n - k0) = A[k0.., k0..k0+nb).
__global__ void k_gj_panel_copy(int n, int k0, int nb, const float* __restrict__ A, double* __restrict__ Pm) {
    const int m = n - k0;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)m * nb) return;
    const int c = (int)(e / m), r = (int)(e - (long long)c * m);
    Pm[e] = (double)A[(size_t)(k0 + c) * n + k0 + r];
}

// The panel's interchanges (step t: row k0+t with row k0+piv[t], in order) on every column of A,
// one thread per column, and on perm.
__global__ void k_gj_swap(int n, int k0, int nb, const int* __restrict__ piv, float* __restrict__ A,
                          int* __restrict__ perm) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) {
        float* col = A + (size_t)j * n + k0;
        for (int t = 0; t < nb; ++t) {
            const int p = piv[t];
            if (p != t && p > t && p < n - k0) {  // a partner outside the panel's rows only after an expired wait
                const float v = col[t];
                col[t] = col[p];
                col[p] = v;
            }
        }
    }
    if (j == 0)
        for (int t = 0; t < nb; ++t) {
            const int p = piv[t];
            if (p != t && p > t && p < n - k0) {
                const int v = perm[k0 + t];
                perm[k0 + t] = perm[k0 + p];
                perm[k0 + p] = v;
            }
        }
}

// W = A_Bb^-1 for the panel's nb x nb block of A after its interchanges, by in-place Gauss-Jordan
// without further pivoting in FP64 (the rows are already the partial-pivoting choice over the whole
// panel, so every pivot is the largest entry left in its column of the block): step k scales row k
// by 1/p and takes f_i times it from every other row i, all elements of a step in parallel.
__global__ void __launch_bounds__(1024) k_gj_block_inverse(int n, int k0, int nb, const float* __restrict__ A,
                                                           float* __restrict__ W, int* __restrict__ sing) {
    __shared__ double M[GJ_NB][GJ_NB + 1];
    __shared__ double s_f[GJ_NB];
    __shared__ double s_p;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < nb * nb; e += nt) {
        const int c = e / nb, r = e - c * nb;
        M[r][c] = (double)A[(size_t)(k0 + c) * n + k0 + r];
    }
    __syncthreads();
    for (int k = 0; k < nb; ++k) {
        if (tid < nb) s_f[tid] = M[tid][k];
        if (tid == 0) {
            s_p = M[k][k];
            if (s_p == 0.0) atomicExch(sing, 1);
        }
        __syncthreads();
        const double ip = s_p != 0.0 ? 1.0 / s_p : 0.0;
        if (tid < nb) M[k][tid] = (tid == k ? 1.0 : M[k][tid]) * ip;
        __syncthreads();
        for (int e = tid; e < nb * nb; e += nt) {
            const int i = e / nb, j = e - i * nb;
            if (i != k) M[i][j] = (j == k ? 0.0 : M[i][j]) - s_f[i] * M[k][j];
        }
        __syncthreads();
    }
    for (int e = tid; e < nb * nb; e += nt) {
        const int c = e / nb, r = e - c * nb;
        W[(size_t)c * nb + r] = (float)M[r][c];
    }
}

// After the accumulating GEMM: the panel's columns take P (zero in the panel's rows) and W in the
// panel's rows; the panel's rows outside its columns take R' (nb x n, leading dimension nb).
__global__ void k_gj_writeback(int n, int k0, int nb, const float* __restrict__ P, const float* __restrict__ Rn,
                               const float* __restrict__ W, float* __restrict__ A) {
    const long long tot = 2LL * n * nb;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        if (e < (long long)n * nb) {
            const int c = (int)(e / n), r = (int)(e - (long long)c * n);
            A[(size_t)(k0 + c) * n + r] = (r >= k0 && r < k0 + nb) ? W[(size_t)c * nb + (r - k0)] : P[(size_t)c * n + r];
        } else {
            const long long f = e - (long long)n * nb;
            const int j = (int)(f / nb), t = (int)(f - (long long)j * nb);
            if (j < k0 || j >= k0 + nb) A[(size_t)j * n + k0 + t] = Rn[(size_t)j * nb + t];
        }
    }
}

// X[:, perm[j]] = A[:, j]
__global__ void k_gj_permute_cols(int n, const int* __restrict__ perm, const float* __restrict__ A,
                                  float* __restrict__ X) {
    const int j = blockIdx.y;
    const float* src = A + (size_t)j * n;
    float* dst = X + (size_t)perm[j] * n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[i];
}

__global__ void k_iota(int n, int* __restrict__ v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

inline int round_up(int v, int m) { return (v + m - 1) / m * m; }



}  // namespace

// X (j.X) ~ G^-1 by the blocked Gauss-Jordan elimination above, from j.G32 = fp32(G); j.T is the
// working matrix.  Scratch: the upper half of c.LU (whose lower half is j.P) and the tensor-core
// operand planes c.tcp.  BEM_ERR_NOT_CONVERGED for a zero pivot, BEM_ERR_CUDA when a panel kernel
// cannot run or a bounded wait expired (the caller then builds X by Newton-Schulz from scratch).
int gj_inverse(Ctx& c, const NSJob& j, cudaStream_t s) {
    const int n = j.n;
    constexpr int NB = GJ_NB;
    if (!c.LU || !c.tcp || !c.lu_aux || n > 65535) return BEM_ERR_CUDA;
    float* A = j.T;
    BEM_CUDA(c, cudaMemcpyAsync(A, j.G32, sizeof(float) * (size_t)n * n, cudaMemcpyDeviceToDevice, s));
    // scratch, 256-byte aligned pieces in the upper half of c.LU
    char* base = reinterpret_cast<char*>(c.LU) + sizeof(float) * (size_t)n * n;
    const size_t avail = sizeof(float) * (size_t)n * n;
    size_t off = (256 - (reinterpret_cast<uintptr_t>(base) & 255)) & 255;
    auto take = [&](size_t bytes) {
        char* p = base + off;
        off += (bytes + 255) / 256 * 256;
        return p;
    };
    double* Pm = reinterpret_cast<double*>(take(sizeof(double) * (size_t)n * NB));
    float* P = reinterpret_cast<float*>(take(sizeof(float) * (size_t)n * NB));
    float* Rn = reinterpret_cast<float*>(take(sizeof(float) * (size_t)n * NB));
    float* W = reinterpret_cast<float*>(take(sizeof(float) * NB * NB));
    int* perm = reinterpret_cast<int*>(take(sizeof(int) * (size_t)n));
    int* piv = reinterpret_cast<int*>(take(sizeof(int) * NB));
    int* sing = reinterpret_cast<int*>(take(sizeof(int) * 4));
    if (off > avail) return BEM_ERR_CUDA;  // small n: the caller uses Newton-Schulz
    // operand planes
    const int mpad = round_up(n, 128), npad = round_up(n, 256), kpad = NB;
    __nv_bfloat16* pl = static_cast<__nv_bfloat16*>(c.tcp);
    __nv_bfloat16 *Ah = pl, *Al = Ah + (size_t)mpad * kpad;
    __nv_bfloat16 *Bh = Al + (size_t)mpad * kpad, *Bl = Bh + (size_t)npad * kpad;
    __nv_bfloat16 *Wah = Bl + (size_t)npad * kpad, *Wal = Wah + 128 * kpad;
    __nv_bfloat16 *Wbh = Wal + 128 * kpad, *Wbl = Wbh + 256 * kpad;
    KLAUNCH(), k_iota<<<(n + 255) / 256, 256, 0, s>>>(n, perm);
    BEM_CUDA(c, cudaMemsetAsync(sing, 0, sizeof(int), s));
    BEM_CUDA(c, cudaMemsetAsync(lu_panel_err(c), 0, sizeof(int), s));
    int rc = BEM_OK;
    for (int k0 = 0; k0 < n && rc == BEM_OK; k0 += NB) {
        const int nb = std::min(NB, n - k0), m = n - k0, k1 = k0 + nb;
        KLAUNCH(), k_gj_panel_copy<<<(int)(((long long)m * nb + 255) / 256), 256, 0, s>>>(n, k0, nb, A, Pm);
        const PanelTarget tgt{Pm, m, piv, sing};
        if (lu_panel_cluster(c, 0, nb, s, &tgt) != BEM_OK && lu_panel_rows(c, 0, nb, s, &tgt) != BEM_OK)
            return BEM_ERR_CUDA;
        KLAUNCH(), k_gj_swap<<<(n + 255) / 256, 256, 0, s>>>(n, k0, nb, piv, A, perm);
        KLAUNCH(), k_gj_block_inverse<<<1, 1024, 0, s>>>(n, k0, nb, A, W, sing);
        // P = -A_Ob W: A operand the panel's columns with its rows masked, B operand W (K x N = nb x nb)
        TcOperand a1{A + (size_t)k0 * n, 1, (long long)n, n, nb, k0, k1, 0, 0, -1.f};
        TcOperand b1{W, (long long)nb, 1, nb, nb};
        tc_split_op(a1, mpad, kpad, Ah, Al, s);
        tc_split_op(b1, 256, kpad, Wbh, Wbl, s);
        if ((rc = tc_gemm_planes(c, n, nb, mpad, 256, kpad, Ah, Al, Wbh, Wbl, P, n, false, c.tc_err, s))) break;
        // R' = W A_Bo: A operand W (nb x nb), B operand the panel's rows (K x N = nb x n) with its
        // columns masked; those B planes are also the accumulating GEMM's
        TcOperand a2{W, 1, (long long)nb, nb, nb};
        TcOperand b2{A + k0, (long long)n, 1, n, nb, k0, k1, 0, 0, 1.f};
        tc_split_op(a2, 128, kpad, Wah, Wal, s);
        tc_split_op(b2, npad, kpad, Bh, Bl, s);
        if ((rc = tc_gemm_planes(c, nb, n, 128, npad, kpad, Wah, Wal, Bh, Bl, Rn, nb, false, c.tc_err, s))) break;
        // A_Oo += P A_Bo over the whole matrix (zero in the panel's rows and columns)
        TcOperand a3{P, 1, (long long)n, n, nb, k0, k1, 0, 0, 1.f};
        tc_split_op(a3, mpad, kpad, Ah, Al, s);
        if ((rc = tc_gemm_planes(c, n, n, mpad, npad, kpad, Ah, Al, Bh, Bl, A, n, true, c.tc_err, s))) break;
        KLAUNCH(), k_gj_writeback<<<4 * 148, 256, 0, s>>>(n, k0, nb, P, Rn, W, A);
    }
    if (rc) return rc;
    int flags[3] = {0, 0, 0};
    BEM_CUDA(c, cudaMemcpyAsync(&flags[0], sing, sizeof(int), cudaMemcpyDeviceToHost, s));
    BEM_CUDA(c, cudaMemcpyAsync(&flags[1], lu_panel_err(c), sizeof(int), cudaMemcpyDeviceToHost, s));
    BEM_CUDA(c, cudaMemcpyAsync(&flags[2], c.tc_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    BEM_CUDA(c, cudaStreamSynchronize(s));
    if (flags[1] || flags[2]) {
        if (flags[1]) c.stats.wait_expired++;
        BEM_CUDA(c, cudaMemsetAsync(lu_panel_err(c), 0, sizeof(int), s));
        return c.fail(BEM_ERR_CUDA, "Gauss-Jordan inverse: a bounded wait expired");
    }
    if (flags[0]) return c.fail(BEM_ERR_NOT_CONVERGED, "Gauss-Jordan inverse: zero pivot (singular G)");
    KLAUNCH(), k_gj_permute_cols<<<dim3((n + 1023) / 1024, n), 256, 0, s>>>(n, perm, A, j.X);
    c.stats.gj_inverses++;
    return BEM_OK;
}

}  // namespace bemb
