// QDHT products of the mixed-precision radial transform on the 5th-generation tensor
// cores (tcgen05, sm_100a): C = A B^T with FP32 A and C and a pre-split BF16 pair for B,
// as three BF16 products accumulated in FP32 in tensor memory:
//   A B ~ A_hi B_hi + A_hi B_lo + A_lo B_hi,   X_hi = bf16(X), X_lo = bf16(X - X_hi).
// The dropped A_lo B_lo term and the residual of the split are ~2^-16 relative, against
// the 2^-8 of a single BF16 product.
//
// Layout: A is the column-major 2Nw x K real view of a complex Nw x K array (element
// (r, m) at m*lda + r); B is row-major N x K (element (n, m) at n*K + m); C like A.
// One CTA computes a 128-row x BN-column tile. K is consumed in 64-deep chunks through a
// two-stage shared-memory ring: all threads convert their part of the next chunk to BF16
// (hi and lo) and write it in the K-major core-matrix layout (8 rows x 16 bytes per core
// matrix, no swizzle) while the previous chunk's MMAs run; one thread issues the
// 4 x 3 MMAs (M=128, N=BN, K=16) of a chunk and commits them to the stage's mbarrier.
// The accumulator (128 lanes x BN FP32 columns) is read back with tcgen05.ld by all
// eight warps (warp w: lanes 32*(w%4).., column half w/4).
//
// Every wait on an mbarrier is bounded; on expiry the kernel raises ST_WAIT_TIMEOUT in
// *flags, waits (bounded) for its last commit, frees its tensor memory and returns.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "common.cuh"

namespace luna {

#define TC_BM 128
#define TC_KC 64
#define TC_THREADS 256
#define TC_WAIT_CYCLES (2000000000LL)  // ~1 s at the B200 boost clock

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// tcgen05 shared-memory matrix descriptor: K-major, no swizzle (canonical layout
// ((8,n),2):((16B,SBO),LBO)), version 1 (sm_100).
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 accumulator.
__host__ __device__ constexpr uint32_t tc_idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tc_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of an mbarrier; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_try(mbar, parity)) {
        if (clock64() - t0 > TC_WAIT_CYCLES) return false;
    }
    return true;
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&v);
}

// 32 consecutive FP32 accumulator columns of this thread's lane.
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

// Shared memory of one stage: A hi, A lo (128 x 64 BF16 each), B hi, B lo (BN x 64 each).
template <int BN>
struct TcStage {
    static constexpr int A_BYTES = TC_BM * TC_KC * 2;
    static constexpr int B_BYTES = BN * TC_KC * 2;
    static constexpr int BYTES = 2 * A_BYTES + 2 * B_BYTES;
};

template <int BN>
constexpr int tc_smem_bytes() {
    return 2 * TcStage<BN>::BYTES + 1024;  // two stages + alignment slack
}

// byte offset of the 16-byte chunk (row, kchunk) of a 64-deep K-major tile
__device__ __forceinline__ uint32_t tc_off(int row, int kch) {
    return (uint32_t)((row >> 3) * 1024 + kch * 128 + (row & 7) * 16);
}

// C[r, n0 + j] = sum_m A[m*lda + r] B[(n0 + j)*K + m] for r < rows, j < BN (K % 64 == 0,
// N % BN == 0). Grid: (ceil(rows/128), N/BN).
template <int BN>
__global__ void __launch_bounds__(TC_THREADS, 1)
tc_gemm_3xbf16(const float* __restrict__ A, int lda, int rows, const __nv_bfloat16* __restrict__ Bhi,
               const __nv_bfloat16* __restrict__ Blo, float* __restrict__ C, int K, const int* finished,
               int* flags) {
    static_assert(BN % 64 == 0 && BN >= 64 && BN <= 256, "BN must be 64, 128 or 256");
    if (finished && *finished) return;
    extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_base_sh;
    unsigned char* sm = (unsigned char*)(((uintptr_t)tc_smem_raw + 1023) & ~(uintptr_t)1023);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int r0 = blockIdx.x * TC_BM, n0 = blockIdx.y * BN;
    constexpr uint32_t TCOLS = (BN <= 32) ? 32 : (BN <= 64) ? 64 : (BN <= 128) ? 128 : 256;
    constexpr uint32_t idesc = tc_idesc_bf16(TC_BM, BN);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_sh;

    const int nk = K / TC_KC;
    bool ok = true;   // uniform across the CTA
    int issued = 0;   // chunks whose MMAs have been issued and committed
    for (int kc = 0; kc < nk; ++kc) {
        const int s = kc & 1;
        unsigned char* st = sm + s * TcStage<BN>::BYTES;
        unsigned char* sAh = st;
        unsigned char* sAl = st + TcStage<BN>::A_BYTES;
        unsigned char* sBh = st + 2 * TcStage<BN>::A_BYTES;
        unsigned char* sBl = sBh + TcStage<BN>::B_BYTES;
        if (kc >= 2) {  // the stage's previous MMAs must have finished reading it
            const bool w = mbar_wait(smem_u32(&mbar[s]), ((kc - 2) >> 1) & 1);
            ok = __syncthreads_and(w) != 0;
            if (!ok) break;
        }
        // A chunk: 128 rows x 8 k-chunks of 8; unit u -> (row u%128, kchunk u/128)
        const int m0 = kc * TC_KC;
#pragma unroll
        for (int q = 0; q < (TC_BM * 8) / TC_THREADS; ++q) {
            const int u = tid + TC_THREADS * q;
            const int row = u & (TC_BM - 1), kch = u >> 7;
            const int r = r0 + row;
            float v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = (r < rows) ? __ldg(A + (size_t)(m0 + kch * 8 + j) * lda + r) : 0.0f;
            uint4 h, l;
            float lo[8];
            uint32_t* hp = &h.x;
#pragma unroll
            for (int j = 0; j < 8; j += 2) {
                __nv_bfloat162 b = __floats2bfloat162_rn(v[j], v[j + 1]);
                hp[j / 2] = *reinterpret_cast<uint32_t*>(&b);
                lo[j] = v[j] - __bfloat162float(b.x);
                lo[j + 1] = v[j + 1] - __bfloat162float(b.y);
            }
            l.x = pack_bf16(lo[0], lo[1]);
            l.y = pack_bf16(lo[2], lo[3]);
            l.z = pack_bf16(lo[4], lo[5]);
            l.w = pack_bf16(lo[6], lo[7]);
            const uint32_t o = tc_off(row, kch);
            *reinterpret_cast<uint4*>(sAh + o) = h;
            *reinterpret_cast<uint4*>(sAl + o) = l;
        }
        // B chunk: BN rows x 8 k-chunks, 16-byte copies
        for (int u = tid; u < BN * 8; u += TC_THREADS) {
            const int row = u >> 3, kch = u & 7;
            const size_t g = (size_t)(n0 + row) * K + m0 + kch * 8;
            const uint32_t o = tc_off(row, kch);
            *reinterpret_cast<uint4*>(sBh + o) = __ldg(reinterpret_cast<const uint4*>(Bhi + g));
            *reinterpret_cast<uint4*>(sBl + o) = __ldg(reinterpret_cast<const uint4*>(Blo + g));
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t aH = smem_u32(sAh), aL = smem_u32(sAl), bH = smem_u32(sBh), bL = smem_u32(sBl);
#pragma unroll
            for (int kk = 0; kk < TC_KC / 16; ++kk) {
                const uint32_t off = kk * 256;  // two 16-byte k-chunks per K=16 step
                const uint64_t dAh = tc_desc(aH + off, 128, 1024), dAl = tc_desc(aL + off, 128, 1024);
                const uint64_t dBh = tc_desc(bH + off, 128, 1024), dBl = tc_desc(bL + off, 128, 1024);
                tc_mma(tmem, dAh, dBh, idesc, (kc > 0 || kk > 0) ? 1u : 0u);
                tc_mma(tmem, dAh, dBl, idesc, 1u);
                tc_mma(tmem, dAl, dBh, idesc, 1u);
            }
            tc_commit(smem_u32(&mbar[s]));
        }
        issued = kc + 1;
    }
    // wait for the last issued chunk (its commit covers every earlier MMA), also after a
    // timeout, so that no MMA is in flight when the tensor memory is freed
    if (issued > 0) {
        const bool w = mbar_wait(smem_u32(&mbar[(issued - 1) & 1]), ((issued - 1) >> 1) & 1);
        ok = (__syncthreads_and(w) != 0) && ok && issued == nk;
    }
    if (!ok && tid == 0 && flags) atomicOr(flags, 1 << ST_WAIT_TIMEOUT);
    tc_fence_after();
    if (ok) {
        const int quarter = warp & 3, half = warp >> 2;
        const int row = quarter * 32 + (tid & 31);
        const int r = r0 + row;
        constexpr int CPW = BN / 2;  // columns per warp
#pragma unroll
        for (int c0 = 0; c0 < CPW; c0 += 32) {
            const int col = half * CPW + c0;
            float v[32];
            tc_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)col, v);
            if (r < rows) {
#pragma unroll
                for (int j = 0; j < 32; ++j) C[(size_t)(n0 + col + j) * lda + r] = v[j];
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS));
}

}  // namespace luna
