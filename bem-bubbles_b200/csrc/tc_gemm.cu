// Split-precision tensor-core GEMM for sm_100a (tcgen05 + TMA + TMEM): C = A * B in FP32 from
// FP32 operands, each operand split into two bfloat16 parts (x = hi + lo, hi = bf16(x),
// lo = bf16(x - hi)) and the product formed as hi*hi + hi*lo + lo*hi with FP32 accumulation in
// tensor memory ("BF16x3": about 16 significant bits per operand, three bf16 MMAs per product).
// Used by the mixed solver's Newton-Schulz refresh of the approximate inverse (X <- X(2I - G X)).
// TERMS = 1 keeps only hi*hi (plain bf16 inputs, FP32 accumulation): the early Newton-Schulz steps
// of a from-scratch inverse, whose residual is still near 1, need no more.
//
// Structure: one CTA per 128 x BN tile of C, 128 threads.  Thread 0 issues TMA tile loads of the
// four operand planes (128B-swizzled, K-major) into a STAGES-deep shared-memory ring guarded by
// mbarriers; thread 32 issues the tcgen05.mma instructions (M=128, N=BN, K=16 per instruction)
// accumulating in TMEM and frees ring slots with tcgen05.commit; after the last k-block all four
// warps read their 32 TMEM lanes (tcgen05.ld 32x32b) and store FP32 C column-major.
// Every mbarrier wait is bounded: on timeout the kernel records an error code, drains its own
// in-flight copies (again bounded), releases TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "ctx.h"

namespace bemb {

constexpr int TC_BM = 128, TC_BK = 64, TC_THREADS = 128;
constexpr long long TC_SPIN_LIMIT = 1ll << 24;  // bounded waits (on the order of a second of polling)

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// returns true when the phase with the given parity has completed, false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (long long it = 0; it < TC_SPIN_LIMIT; ++it) {
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
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
// shared-memory matrix descriptor: K-major operand, 128-byte swizzle, 8-row atoms 1024 B apart
__device__ __forceinline__ uint64_t sdesc(const void* p) {
    const uint64_t addr = (smem_u32(p) & 0x3FFFF) >> 4;
    const uint64_t lbo = 1, sbo = 1024 >> 4;
    return addr | (lbo << 16) | (sbo << 32) | (1ull << 46) | (2ull << 61);
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accum)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// Instruction descriptor, kind::f16: D = F32 (bits 4-5 = 1), A = B = BF16 (bits 7-9, 10-12 = 1),
// both K-major (bits 15, 16 = 0), N >> 3 at bits 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// C (rows < m, columns < n, column-major with leading dimension ldc) = A B, or += A B with ACC.
template <int BN, int STAGES, int TERMS, bool ACC = false>
__global__ void __launch_bounds__(TC_THREADS, 1)
    k_gemm_bf16x3(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
                  const __grid_constant__ CUtensorMap mBh, const __grid_constant__ CUtensorMap mBl,
                  float* __restrict__ C, int m, int n, int ldc, int kblocks, int* __restrict__ err) {
    constexpr uint32_t A_BYTES = TC_BM * TC_BK * 2, B_BYTES = BN * TC_BK * 2;
    constexpr uint32_t STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    constexpr uint32_t STAGE_TX = TERMS == 1 ? A_BYTES + B_BYTES : STAGE_BYTES;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], done;
    __shared__ uint32_t tmem_base;
    __shared__ int abort_flag;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * TC_BM, n0 = blockIdx.x * BN;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&done, 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;

    int issued = 0;  // k-blocks whose loads the producer issued
    if (threadIdx.x == 0) {
        // TMA producer
        for (int kb = 0; kb < kblocks; ++kb) {
            const int s = kb % STAGES;
            if (kb >= STAGES && !mbar_wait(&empty[s], ((kb / STAGES) & 1) ^ 1)) {
                atomicExch(err, 1);
                abort_flag = 1;
                break;
            }
            uint8_t* st = smem + (size_t)s * STAGE_BYTES;
            mbar_expect_tx(&full[s], STAGE_TX);
            const int kx = kb * TC_BK;
            tma_load_2d(st, &mAh, kx, m0, &full[s]);
            tma_load_2d(st + 2 * A_BYTES, &mBh, kx, n0, &full[s]);
            if (TERMS == 3) {
                tma_load_2d(st + A_BYTES, &mAl, kx, m0, &full[s]);
                tma_load_2d(st + 2 * A_BYTES + B_BYTES, &mBl, kx, n0, &full[s]);
            }
            issued = kb + 1;
        }
        // drain: every issued stage must land before the CTA may exit
        if (abort_flag)
            for (int kb = (issued > STAGES ? issued - STAGES : 0); kb < issued; ++kb)
                (void)mbar_wait(&full[kb % STAGES], (kb / STAGES) & 1);
    } else if (threadIdx.x == 32) {
        // MMA issuer
        constexpr uint32_t idesc = idesc_bf16(TC_BM, BN);
        bool ok = true;
        for (int kb = 0; kb < kblocks; ++kb) {
            const int s = kb % STAGES;
            if (!mbar_wait(&full[s], (kb / STAGES) & 1)) {
                atomicExch(err, 2);
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            uint8_t* st = smem + (size_t)s * STAGE_BYTES;
#pragma unroll
            for (int k = 0; k < TC_BK / 16; ++k) {
                const uint64_t ah = sdesc(st + k * 32), al = sdesc(st + A_BYTES + k * 32);
                const uint64_t bh = sdesc(st + 2 * A_BYTES + k * 32), bl = sdesc(st + 2 * A_BYTES + B_BYTES + k * 32);
                umma_bf16(tmem, ah, bh, idesc, (kb > 0 || k > 0) ? 1u : 0u);
                if (TERMS == 3) {
                    umma_bf16(tmem, ah, bl, idesc, 1u);
                    umma_bf16(tmem, al, bh, idesc, 1u);
                }
            }
            umma_commit(&empty[s]);
        }
        umma_commit(&done);
        if (!ok) abort_flag = 1;
    }
    __syncwarp();
    // epilogue: TMEM lanes 32w..32w+31 hold rows m0+32w.., columns n0..n0+BN-1
    const bool have = mbar_wait(&done, 0);
    if (!have) atomicExch(err, 3);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    if (have && !abort_flag) {
        const int row = m0 + warp * 32 + lane;
        // 32 columns per round; with ACC the round's 32 values of C are loaded first, all in flight
        // together before the tensor-memory read (one memory latency per round, not one per element)
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 32) {
            float cv[32];
            if (ACC) {
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int col = n0 + c0 + j;
                    cv[j] = (row < m && col < n) ? C[(size_t)col * ldc + row] : 0.f;
                }
            }
            uint32_t r[32];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c0 + 16 * h);
                uint32_t* q = r + 16 * h;
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                    : "=r"(q[0]), "=r"(q[1]), "=r"(q[2]), "=r"(q[3]), "=r"(q[4]), "=r"(q[5]), "=r"(q[6]), "=r"(q[7]),
                      "=r"(q[8]), "=r"(q[9]), "=r"(q[10]), "=r"(q[11]), "=r"(q[12]), "=r"(q[13]), "=r"(q[14]),
                      "=r"(q[15])
                    : "r"(taddr));
            }
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < m) {
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int col = n0 + c0 + j;
                    if (col < n) C[(size_t)col * ldc + row] = ACC ? cv[j] + __uint_as_float(r[j]) : __uint_as_float(r[j]);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}

// Split an FP32 column-major n x n matrix into bf16 hi/lo planes of a padded npad x npad K-major
// layout.  trans = 0: plane[j*npad + i] = src(i, j) (the column-major matrix used as the B operand,
// K = row index); trans = 1: plane[i*npad + j] = src(i, j) (used as the A operand, K = column).
__global__ void k_split_bf16(int n, int npad, const float* __restrict__ src, __nv_bfloat16* __restrict__ hi,
                             __nv_bfloat16* __restrict__ lo, int trans) {
    __shared__ float tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;  // bx: row block of src, by: column block
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int i = bx + threadIdx.x, j = by + k;
        tile[k][threadIdx.x] = (i < n && j < n) ? src[(size_t)j * n + i] : 0.f;
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        int i, j;
        float v;
        if (!trans) {  // write plane[j*npad + i], consecutive threads -> consecutive i
            i = bx + threadIdx.x;
            j = by + k;
            v = tile[k][threadIdx.x];
            if (i < npad && j < npad) {
                const __nv_bfloat16 h = __float2bfloat16_rn(v);
                hi[(size_t)j * npad + i] = h;
                lo[(size_t)j * npad + i] = __float2bfloat16_rn(v - __bfloat162float(h));
            }
        } else {  // write plane[i*npad + j], consecutive threads -> consecutive j
            j = by + threadIdx.x;
            i = bx + k;
            v = tile[threadIdx.x][k];
            if (i < npad && j < npad) {
                const __nv_bfloat16 h = __float2bfloat16_rn(v);
                hi[(size_t)i * npad + j] = h;
                lo[(size_t)i * npad + j] = __float2bfloat16_rn(v - __bfloat162float(h));
            }
        }
    }
}

// An operand plane of the general GEMM: plane[r * kpad + k] = sign * S(r, k), bf16 hi/lo split, for
// r < rows and k < cols, zero in the padding (rpad x kpad) and for r in [zr0, zr1) or k in [zk0, zk1).
// S(r, k) = src[r * sr + k * sk]: (sr, sk) = (1, ld) reads an A operand stored column-major, (ld, 1) a
// B operand stored column-major (K x N; the plane's rows are its columns).  32 x 32 tiles, staged
// through shared memory when the plane's inner index is not the source's contiguous one.
__global__ void k_split_op(int rows, int cols, int rpad, int kpad, const float* __restrict__ src, long long sr,
                           long long sk, int zr0, int zr1, int zk0, int zk1, float sign,
                           __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo) {
    __shared__ float tile[32][33];
    const int k0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    auto value = [&](int r, int k) -> float {
        if (r >= rows || k >= cols || (r >= zr0 && r < zr1) || (k >= zk0 && k < zk1)) return 0.f;
        return sign * src[(long long)r * sr + (long long)k * sk];
    };
    auto put = [&](int r, int k, float v) {
        if (r < rpad && k < kpad) {
            const __nv_bfloat16 h = __float2bfloat16_rn(v);
            hi[(size_t)r * kpad + k] = h;
            lo[(size_t)r * kpad + k] = __float2bfloat16_rn(v - __bfloat162float(h));
        }
    };
    if (sr == 1) {  // contiguous along r: read along r, write along k through the tile
        for (int q = threadIdx.y; q < 32; q += blockDim.y) tile[q][threadIdx.x] = value(r0 + threadIdx.x, k0 + q);
        __syncthreads();
        for (int q = threadIdx.y; q < 32; q += blockDim.y) put(r0 + q, k0 + threadIdx.x, tile[threadIdx.x][q]);
    } else {  // contiguous along k (or neither): both along k
        for (int q = threadIdx.y; q < 32; q += blockDim.y) put(r0 + q, k0 + threadIdx.x, value(r0 + q, k0 + threadIdx.x));
    }
}

// ---------------------------------------------------------------- host side
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// 2-D bf16 plane of `rows` rows x kpad (K innermost), box {64, box_rows}, 128-byte swizzle
static bool make_map_rows(CUtensorMap* m, const void* base, int kpad, int rows, int box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)kpad, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)kpad * 2};
    cuuint32_t box[2] = {(cuuint32_t)TC_BK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// 2-D bf16 plane npad x npad (K innermost), box {64, rows}, 128-byte swizzle
static bool make_map(CUtensorMap* m, const void* base, int npad, int box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)npad, (cuuint64_t)npad};
    cuuint64_t strides[1] = {(cuuint64_t)npad * 2};
    cuuint32_t box[2] = {(cuuint32_t)TC_BK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

constexpr int TC_BN = 256, TC_STAGES = 2;

int tc_pad(int n) { return (n + 255) / 256 * 256; }

size_t tc_smem_bytes(int stages = TC_STAGES, int bn = TC_BN) {
    return (size_t)stages * (2 * TC_BM * TC_BK * 2 + 2 * bn * TC_BK * 2) + 1024;
}
constexpr int TC_BN_ACC = 128;  // the accumulating GEMM's tile width: three CTAs per SM with one stage

// C = A * B (all FP32, column-major n x n, leading dimension n).  Work buffers: four bf16 planes
// of tc_pad(n)^2 elements each (ah, al, bh, bl); err: device int (non-zero after a timeout).
// terms: 3 (BF16x3) or 1 (hi*hi only).
int tc_gemm(Ctx& c, int n, const float* A, const float* B, float* C, void* planes, int* err, cudaStream_t s,
            int terms) {
    const int npad = tc_pad(n);
    const size_t np = (size_t)npad * npad;
    __nv_bfloat16* ah = static_cast<__nv_bfloat16*>(planes);
    __nv_bfloat16 *al = ah + np, *bh = ah + 2 * np, *bl = ah + 3 * np;
    dim3 sg((npad + 31) / 32, (npad + 31) / 32), sb(32, 8);
    KLAUNCH(), k_split_bf16<<<sg, sb, 0, s>>>(n, npad, A, ah, al, 1);
    KLAUNCH(), k_split_bf16<<<sg, sb, 0, s>>>(n, npad, B, bh, bl, 0);
    CUtensorMap mAh, mAl, mBh, mBl;
    if (!make_map(&mAh, ah, npad, TC_BM) || !make_map(&mAl, al, npad, TC_BM) || !make_map(&mBh, bh, npad, TC_BN) ||
        !make_map(&mBl, bl, npad, TC_BN))
        return c.fail(BEM_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    const size_t sm = tc_smem_bytes();
    static std::atomic<uint64_t> attr{0};
    if (!once_per_device(attr, [sm] {
            return cudaFuncSetAttribute(k_gemm_bf16x3<TC_BN, TC_STAGES, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)sm) == cudaSuccess &&
                   cudaFuncSetAttribute(k_gemm_bf16x3<TC_BN, TC_STAGES, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)sm) == cudaSuccess;
        })) {
        cudaGetLastError();
        return c.fail(BEM_ERR_CUDA, "cudaFuncSetAttribute failed for the tensor-core GEMM");
    }
    dim3 grid(npad / TC_BN, npad / TC_BM);
    if (terms == 1)
        KLAUNCH(), k_gemm_bf16x3<TC_BN, TC_STAGES, 1><<<grid, TC_THREADS, sm, s>>>(mAh, mAl, mBh, mBl, C, n, n, n, npad / TC_BK, err);
    else
        KLAUNCH(), k_gemm_bf16x3<TC_BN, TC_STAGES, 3><<<grid, TC_THREADS, sm, s>>>(mAh, mAl, mBh, mBl, C, n, n, n, npad / TC_BK, err);
    // a launch refused for its configuration (shared memory, grid) leaves C unwritten: report it here,
    // since a later stream synchronisation does not
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) return c.fail(BEM_ERR_CUDA, std::string("tensor-core GEMM launch: ") + cudaGetErrorString(le));
    return BEM_OK;
}

void tc_split_op(const TcOperand& o, int rpad, int kpad, void* hi, void* lo, cudaStream_t s) {
    dim3 g((kpad + 31) / 32, (rpad + 31) / 32), b(32, 8);
    KLAUNCH(), k_split_op<<<g, b, 0, s>>>(o.rows, o.cols, rpad, kpad, o.src, o.sr, o.sk, o.zr0, o.zr1, o.zk0, o.zk1,
                                          o.sign, static_cast<__nv_bfloat16*>(hi), static_cast<__nv_bfloat16*>(lo));
}

// C (m x n, column-major, ldc) = A B, or += A B (acc), from operand planes made by tc_split_op:
// A planes mpad x kpad, B planes npad x kpad (mpad a multiple of 128, npad of 256, kpad of 64).
int tc_gemm_planes(Ctx& c, int m, int n, int mpad, int npad, int kpad, const void* ah, const void* al, const void* bh,
                   const void* bl, float* C, int ldc, bool acc, int* err, cudaStream_t s) {
    if (mpad % TC_BM || npad % TC_BN || kpad % TC_BK || m > mpad || n > npad)
        return c.fail(BEM_ERR_ARG, "tc_gemm_planes: plane shape");
    const int kb = kpad / TC_BK;
    const bool narrow = acc && kb == 1;  // the accumulating rank-64 update: 128-column tiles
    CUtensorMap mAh, mAl, mBh, mBl;
    const int bn = narrow ? TC_BN_ACC : TC_BN;
    if (!make_map_rows(&mAh, ah, kpad, mpad, TC_BM) || !make_map_rows(&mAl, al, kpad, mpad, TC_BM) ||
        !make_map_rows(&mBh, bh, kpad, npad, bn) || !make_map_rows(&mBl, bl, kpad, npad, bn))
        return c.fail(BEM_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    const size_t sm2 = tc_smem_bytes(2), sm1 = tc_smem_bytes(1), smn = tc_smem_bytes(1, TC_BN_ACC);
    static std::atomic<uint64_t> attr{0};
    if (!once_per_device(attr, [sm1, sm2, smn] {
            return cudaFuncSetAttribute(k_gemm_bf16x3<TC_BN, 2, 3, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)sm2) == cudaSuccess &&
                   cudaFuncSetAttribute(k_gemm_bf16x3<TC_BN, 2, 3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)sm2) == cudaSuccess &&
                   cudaFuncSetAttribute(k_gemm_bf16x3<TC_BN, 1, 3, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)sm1) == cudaSuccess &&
                   cudaFuncSetAttribute(k_gemm_bf16x3<TC_BN, 1, 3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)sm1) == cudaSuccess &&
                   cudaFuncSetAttribute(k_gemm_bf16x3<TC_BN_ACC, 1, 3, true>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smn) == cudaSuccess;
        })) {
        cudaGetLastError();
        return c.fail(BEM_ERR_CUDA, "cudaFuncSetAttribute failed for the tensor-core GEMM");
    }
    dim3 grid(npad / TC_BN, mpad / TC_BM);
    if (narrow) {
        dim3 gn(npad / TC_BN_ACC, mpad / TC_BM);
        KLAUNCH(), k_gemm_bf16x3<TC_BN_ACC, 1, 3, true><<<gn, TC_THREADS, smn, s>>>(mAh, mAl, mBh, mBl, C, m, n, ldc, kb,
                                                                                 err);
    } else if (kb == 1) {  // one k-block: a one-stage ring, half the shared memory, two CTAs per SM
        if (acc)
            KLAUNCH(), k_gemm_bf16x3<TC_BN, 1, 3, true><<<grid, TC_THREADS, sm1, s>>>(mAh, mAl, mBh, mBl, C, m, n, ldc, kb,
                                                                                 err);
        else
            KLAUNCH(), k_gemm_bf16x3<TC_BN, 1, 3, false><<<grid, TC_THREADS, sm1, s>>>(mAh, mAl, mBh, mBl, C, m, n, ldc, kb,
                                                                                  err);
    } else if (acc) {
        KLAUNCH(), k_gemm_bf16x3<TC_BN, 2, 3, true><<<grid, TC_THREADS, sm2, s>>>(mAh, mAl, mBh, mBl, C, m, n, ldc, kb, err);
    } else {
        KLAUNCH(), k_gemm_bf16x3<TC_BN, 2, 3, false><<<grid, TC_THREADS, sm2, s>>>(mAh, mAl, mBh, mBl, C, m, n, ldc, kb,
                                                                              err);
    }
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) return c.fail(BEM_ERR_CUDA, std::string("tensor-core GEMM launch: ") + cudaGetErrorString(le));
    return BEM_OK;
}

}  // namespace bemb

// Diagnostic entry point: C = A * B through the split-precision tensor-core GEMM, host buffers.
extern "C" int bem_gemm_bf16x3(int device, int n, const float* A, const float* B, float* C) {
    using namespace bemb;
    if (n <= 0 || !A || !B || !C) return BEM_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return BEM_ERR_CUDA;
    Ctx c;
    const size_t nn = (size_t)n * n;
    const size_t np = (size_t)tc_pad(n) * tc_pad(n);
    float *dA = nullptr, *dB = nullptr, *dC = nullptr;
    __nv_bfloat16* planes = nullptr;
    int* err = nullptr;
    int rc = BEM_OK;
    if (cudaMalloc(&dA, nn * 4) != cudaSuccess || cudaMalloc(&dB, nn * 4) != cudaSuccess ||
        cudaMalloc(&dC, nn * 4) != cudaSuccess || cudaMalloc(&planes, 4 * np * 2) != cudaSuccess ||
        cudaMalloc(&err, sizeof(int)) != cudaSuccess) {
        rc = BEM_ERR_NOMEM;
    } else {
        cudaMemcpy(dA, A, nn * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(dB, B, nn * 4, cudaMemcpyHostToDevice);
        cudaMemset(err, 0, sizeof(int));
        rc = tc_gemm(c, n, dA, dB, dC, planes, err, 0);
        int herr = 0;
        if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = BEM_ERR_CUDA;
        cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost);
        if (herr) rc = BEM_ERR_CUDA;
        if (rc == BEM_OK) cudaMemcpy(C, dC, nn * 4, cudaMemcpyDeviceToHost);
    }
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    cudaFree(planes);
    cudaFree(err);
    return rc;
}
