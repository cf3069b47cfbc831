// QDHT products of the mixed-precision radial transform on the 5th-generation tensor
// cores (tcgen05, sm_100a): C = A B^T with FP32 A and C and a pre-split BF16 pair for B,
// as three BF16 products accumulated in FP32 in tensor memory:
//   A B ~ A_hi B_hi + A_hi B_lo + A_lo B_hi,   X_hi = bf16(X), X_lo = bf16(X - X_hi).
// The dropped A_lo B_lo term and the residual of the split are ~2^-16 relative, against
// the 2^-8 of a single BF16 product.
//
// Layout: A is the column-major 2Nw x K real view of a complex Nw x K array (element
// (r, m) at m*lda + r); B is N x K, stored pre-tiled (tc_btile_index: one contiguous block
// of BN rows x 64 k per (n tile, k chunk), BF16 hi then lo, each in the K-major
// core-matrix layout the MMA reads: 8 rows x 16 bytes per core matrix, no swizzle); C like A.
// One CTA computes a 128-row x BN-column tile. Its FP32 A chunks (64 k x 128 rows) stream
// into a ring of TC_RAW shared-memory slots by 8-byte cp.async, TC_RAW - 1 chunks ahead of
// their use; each chunk is converted in shared memory to BF16 hi and lo in the core-matrix
// layout of one of two stages, whose B block arrives by one bulk copy (cp.async.bulk,
// completion counted in bytes on the stage's mbarrier). One thread issues the 4 x 3 MMAs
// (M=128, N=BN, K=16) of a chunk and commits them to the stage's other mbarrier.
// The accumulator (128 lanes x BN FP32 columns) is read back with tcgen05.ld: warp w takes
// lanes 32*(w%4).. and, for BN >= 64, the column half w/4 (warps 4-7 idle for BN = 32).
//
// Every wait on an mbarrier is bounded; on expiry the kernel raises ST_WAIT_TIMEOUT in
// *flags, waits (bounded) for its last commit and its last bulk copy, drains its cp.async
// groups, frees its tensor memory and returns.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "common.cuh"

namespace luna {

#define TC_BM 128
#define TC_KC 64
#define TC_THREADS 256
#define TC_WAIT_CYCLES (2000000000LL)  // ~1 s at the B200 boost clock
#define TC_RAW 3                        // FP32 A chunks in the shared-memory ring

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

// Shared memory of one stage: A hi, A lo (128 x 64 BF16 each), B hi, B lo (BN x 64 each);
// after the two stages, the ring of TC_RAW FP32 A chunks (64 k x 128 rows each).
template <int BN>
struct TcStage {
    static constexpr int A_BYTES = TC_BM * TC_KC * 2;
    static constexpr int B_BYTES = BN * TC_KC * 2;
    static constexpr int BYTES = 2 * A_BYTES + 2 * B_BYTES;
    static constexpr int RAW_BYTES = TC_KC * TC_BM * 4;
};

template <int BN>
constexpr int tc_smem_bytes() {
    return 2 * TcStage<BN>::BYTES + TC_RAW * TcStage<BN>::RAW_BYTES + 1024;  // + alignment slack
}

// Element index, in the pre-tiled B of tc_gemm_3xbf16<BN> (N x K, K % 64 == 0), of the hi
// half of B[n, m]; the lo half of the same element sits BN*64 elements later. Blocks of
// BN rows x 64 k in the order (n tile, k chunk), hi then lo, each in the layout of tc_off.
template <int BN>
inline size_t tc_btile_index(int n, int m, int K) {
    const int t = n / BN, row = n % BN, kc = m / TC_KC, k = m % TC_KC;
    const size_t blk = ((size_t)t * (K / TC_KC) + kc) * (size_t)(2 * BN * TC_KC);
    return blk + (size_t)((((row >> 3) * 1024 + (k >> 3) * 128 + (row & 7) * 16) >> 1) + (k & 7));
}

// byte offset of the 16-byte chunk (row, kchunk) of a 64-deep K-major tile
__device__ __forceinline__ uint32_t tc_off(int row, int kch) {
    return (uint32_t)((row >> 3) * 1024 + kch * 128 + (row & 7) * 16);
}

// C[r, n0 + j] = sum_m A[m*lda + r] B[n0 + j, m] for r < rows, j < BN, with B pre-tiled
// as tc_btile_index<BN> lays it out (K % 64 == 0, N % BN == 0; A 8-byte aligned, lda
// even). Grid: (ceil(rows/128), N/BN).
template <int BN>
__global__ void __launch_bounds__(TC_THREADS, 1)
tc_gemm_3xbf16(const float* __restrict__ A, int lda, int rows, const __nv_bfloat16* __restrict__ Bt,
               float* __restrict__ C, int K, const int* finished, int* flags) {
    static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "BN must be a multiple of 32 in 32..256");
    if (finished && *finished) return;
    extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
    __shared__ __align__(8) uint64_t mbar[4];  // 0, 1: MMAs of stage s done; 2, 3: B of stage s landed
    __shared__ uint32_t tmem_base_sh;
    unsigned char* sm = (unsigned char*)(((uintptr_t)tc_smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char* raw = sm + 2 * TcStage<BN>::BYTES;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int r0 = blockIdx.x * TC_BM;
    constexpr uint32_t TCOLS = (BN <= 32) ? 32 : (BN <= 64) ? 64 : (BN <= 128) ? 128 : 256;
    constexpr uint32_t idesc = tc_idesc_bf16(TC_BM, BN);
    constexpr uint32_t BBLK = 2 * TcStage<BN>::B_BYTES;  // bytes of one pre-tiled B block (hi + lo)

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int q = 0; q < 4; ++q) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[q])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_sh;
    const int nk = K / TC_KC;

    // FP32 chunk kc of A into ring slot kc % TC_RAW ([k][row], 512 bytes per k): one 8-byte
    // cp.async per row pair, zero-filled past `rows`; one commit group per call (empty past
    // the last chunk, so that the group count stays uniform).
    auto fetch = [&](int kc) {
        if (kc < nk) {
            const uint32_t dst = smem_u32(raw + (kc % TC_RAW) * TcStage<BN>::RAW_BYTES);
            const size_t m0 = (size_t)kc * TC_KC;
#pragma unroll 4
            for (int q = 0; q < (TC_KC * TC_BM / 2) / TC_THREADS; ++q) {
                const int u = tid + TC_THREADS * q;
                const int pr = u & (TC_BM / 2 - 1), k = u / (TC_BM / 2);
                const int r = r0 + 2 * pr;
                const uint32_t nb = (r + 1 < rows) ? 8u : (r < rows) ? 4u : 0u;
                const float* src = nb ? A + (m0 + k) * (size_t)lda + r : A;
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst + (uint32_t)(k * TC_BM + 2 * pr) * 4u),
                             "l"(src), "r"(nb)
                             : "memory");
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    for (int j = 0; j < TC_RAW - 1; ++j) fetch(j);

    bool ok = true;   // uniform across the CTA
    int issued = 0;   // chunks whose MMAs have been issued and committed
    int bcopies = 0;  // chunks whose B block copy was issued
    int bwaited = 0;  // chunks whose B block copy was seen complete
    for (int kc = 0; kc < nk; ++kc) {
        const int s = kc & 1;
        unsigned char* st = sm + s * TcStage<BN>::BYTES;
        unsigned char* sAh = st;
        unsigned char* sAl = st + TcStage<BN>::A_BYTES;
        unsigned char* sBh = st + 2 * TcStage<BN>::A_BYTES;
        // the ring slot of chunk kc + TC_RAW - 1 held chunk kc - 1, converted before the last barrier
        fetch(kc + TC_RAW - 1);
        if (kc >= 2) {  // the stage's previous MMAs must have finished reading it
            const bool w = mbar_wait(smem_u32(&mbar[s]), ((kc - 2) >> 1) & 1);
            ok = __syncthreads_and(w) != 0;
            if (!ok) break;
        }
        if (tid == 0) {  // B hi and lo of (n tile, chunk kc): one contiguous block, one bulk copy
            const uint32_t fb = smem_u32(&mbar[2 + s]);
            const __nv_bfloat16* src = Bt + ((size_t)blockIdx.y * nk + kc) * (size_t)(2 * BN * TC_KC);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb), "r"(BBLK) : "memory");
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                             smem_u32(sBh)),
                         "l"(src), "r"(BBLK), "r"(fb)
                         : "memory");
        }
        bcopies = kc + 1;
        asm volatile("cp.async.wait_group %0;" ::"n"(TC_RAW - 1) : "memory");  // this thread's part of chunk kc
        __syncthreads();
        // A chunk: 128 rows x 8 k-chunks of 8 from the ring; unit u -> (row u%128, kchunk u/128)
        const float* rw = reinterpret_cast<const float*>(raw + (kc % TC_RAW) * TcStage<BN>::RAW_BYTES);
#pragma unroll
        for (int q = 0; q < (TC_BM * 8) / TC_THREADS; ++q) {
            const int u = tid + TC_THREADS * q;
            const int row = u & (TC_BM - 1), kch = u >> 7;
            float v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = rw[(kch * 8 + j) * TC_BM + row];
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
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        {  // the stage's B block has landed (and every thread's A writes are done)
            const bool w = mbar_wait(smem_u32(&mbar[2 + s]), (kc >> 1) & 1);
            ok = __syncthreads_and(w) != 0;
            if (!ok) break;
            bwaited = kc + 1;
        }
        if (tid == 0) {
            tc_fence_after();
            const uint32_t aH = smem_u32(sAh), aL = smem_u32(sAl);
            const uint32_t bH = smem_u32(sBh), bL = bH + TcStage<BN>::B_BYTES;
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
    asm volatile("cp.async.wait_all;" ::: "memory");
    // wait for the last issued chunk (its commit covers every earlier MMA) and for a B copy
    // not yet seen complete, also after a timeout, so that no MMA or copy is in flight when
    // the tensor memory is freed and the CTA leaves
    if (issued > 0) {
        const bool w = mbar_wait(smem_u32(&mbar[(issued - 1) & 1]), ((issued - 1) >> 1) & 1);
        ok = (__syncthreads_and(w) != 0) && ok && issued == nk;
    }
    if (bcopies > bwaited) {
        const int c = bcopies - 1;
        const bool w = mbar_wait(smem_u32(&mbar[2 + (c & 1)]), (c >> 1) & 1);
        ok = (__syncthreads_and(w) != 0) && ok;
    }
    if (!ok && tid == 0 && flags) atomicOr(flags, 1 << ST_WAIT_TIMEOUT);
    tc_fence_after();
    constexpr int HALVES = (BN >= 64) ? 2 : 1;
    const int quarter = warp & 3, half = warp >> 2;
    if (ok && half < HALVES) {
        const int row = quarter * 32 + (tid & 31);
        const int r = r0 + row;
        const int n0 = blockIdx.y * BN;
        constexpr int CPW = BN / HALVES;  // columns per warp
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
