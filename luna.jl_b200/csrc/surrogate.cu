// Learned surrogate of the capillary scan (no counterpart in the reference): an ensemble
// of multilayer perceptrons mapping the scan parameters and z to the log spectrum and
// temporal envelope, trained and evaluated by the kernels of this file.
//
//   * sg_gemm<AT, BT>: C[m, n] = sum_k A(m, k) B(n, k) on the 5th-generation tensor cores
//     (tcgen05.mma kind::f16, BF16 operands, FP32 accumulator in tensor memory) for the
//     three products of a linear layer: forward Y = X W^T (A = X, B = W, both stored with
//     k contiguous), backward data dX = dZ W (B = W read with n contiguous) and backward
//     weights dW = dZ^T X (both read with the batch index contiguous). The CTA's threads
//     stage 128 x 64 tiles of A and B into shared memory in the K-major core-matrix layout
//     (asynchronous 16-byte copies where k is contiguous, through registers where the source
//     is stored the other way), one thread issues the MMAs, and a three-stage ring keeps two
//     chunks in flight while the MMAs of a third run.
//     Fused epilogues: bias + SiLU with the pre-activation kept (forward), the SiLU
//     derivative of the layer input (backward data), plain FP32 (backward weights).
//     blockIdx.z runs over ensemble members (strided operands).
//   * Fourier-feature input, MSE loss and output gradient, bias gradient, Adam with FP32
//     master weights writing the BF16 working copy, ensemble mean and spread.
//
// All dimensions are multiples of 128 (the batch and the layer widths) and of 64 (the
// reduction); the host checks them. Every mbarrier wait is bounded (about 1 s); on expiry
// the kernel sets *err, waits (bounded) for its last commit, frees its tensor memory and
// returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/luna_surrogate.h"
#include "tc_gemm.cuh"

using namespace luna;
typedef __nv_bfloat16 bf16;

namespace {

constexpr int SG_BM = 128, SG_BN = 128, SG_KC = 64, SG_THREADS = 256;
constexpr int SG_TILE_BYTES = SG_BM * SG_KC * 2;      // one 128 x 64 BF16 tile
constexpr int SG_STAGE_BYTES = 2 * SG_TILE_BYTES;     // A and B
constexpr int SG_STAGES = 3;                          // ring depth: two chunks in flight
constexpr int SG_SMEM = SG_STAGES * SG_STAGE_BYTES + 1024;  // stages + alignment slack

enum { EPI_F32 = 0, EPI_FWD = 1, EPI_BWD_DATA = 2 };

struct SgArgs {
    const bf16* A; long long lda, sA;   // element (m, k): AT ? A[k*lda + m] : A[m*lda + k]
    const bf16* B; long long ldb, sB;   // element (n, k): BT ? B[k*ldb + n] : B[n*ldb + k]
    int M, N, K;
    int epi;
    float* C; long long ldc, sC;        // EPI_F32: C[m*ldc + n]
    const float* bias; long long sbias; // EPI_FWD: + bias[n]
    int act;                            // EPI_FWD: 1 SiLU, 0 identity
    bf16* Y; long long ldy, sY;         // EPI_FWD: act(v) as BF16 (may be null)
    bf16* Z; long long sZ;              // EPI_FWD: pre-activation as BF16 (ld = ldy; may be null)
    float* Yf; long long sYf;           // EPI_FWD: act(v) as FP32 (ld = ldy; may be null)
    const bf16* Zp; long long sZp;      // EPI_BWD_DATA: pre-activation of the layer input
                                        // (ld = ldy); writes v * silu'(Zp) to Y
};

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// Stage rows [r0, r0+128) x k [k0, k0+64) of an operand into the K-major core-matrix layout.
template <bool T>
__device__ __forceinline__ void sg_stage(const bf16* __restrict__ src, long long ld, int r0, int k0, unsigned char* dst,
                                         int tid) {
    if (!T) {
        // k contiguous: one 16-byte chunk (8 consecutive k) per unit
#pragma unroll
        for (int q = 0; q < (SG_BM * 8) / SG_THREADS; ++q) {
            const int u = tid + SG_THREADS * q;
            const int row = u >> 3, kch = u & 7;
            const uint4 v = __ldg(reinterpret_cast<const uint4*>(src + (size_t)(r0 + row) * ld + k0 + kch * 8));
            *reinterpret_cast<uint4*>(dst + tc_off(row, kch)) = v;
        }
    } else {
        // rows contiguous: a pair of rows (4 bytes) at each of 8 consecutive k per unit,
        // repacked into the two rows' 16-byte chunks
#pragma unroll
        for (int q = 0; q < (SG_BM / 2 * 8) / SG_THREADS; ++q) {
            const int u = tid + SG_THREADS * q;
            const int rp = u & (SG_BM / 2 - 1), kch = u >> 6;
            const int row = 2 * rp;
            uint32_t w[8];
#pragma unroll
            for (int j = 0; j < 8; ++j)
                w[j] = __ldg(reinterpret_cast<const unsigned int*>(src + (size_t)(k0 + kch * 8 + j) * ld + r0 + row));
            uint4 c0, c1;
            c0.x = (w[0] & 0xFFFFu) | (w[1] << 16);
            c0.y = (w[2] & 0xFFFFu) | (w[3] << 16);
            c0.z = (w[4] & 0xFFFFu) | (w[5] << 16);
            c0.w = (w[6] & 0xFFFFu) | (w[7] << 16);
            c1.x = (w[0] >> 16) | (w[1] & 0xFFFF0000u);
            c1.y = (w[2] >> 16) | (w[3] & 0xFFFF0000u);
            c1.z = (w[4] >> 16) | (w[5] & 0xFFFF0000u);
            c1.w = (w[6] >> 16) | (w[7] & 0xFFFF0000u);
            *reinterpret_cast<uint4*>(dst + tc_off(row, kch)) = c0;
            *reinterpret_cast<uint4*>(dst + tc_off(row + 1, kch)) = c1;
        }
    }
}

// Asynchronous form of sg_stage for an operand stored with k contiguous: one 16-byte
// cp.async per core-matrix row (no register round trip); other layouts are staged through
// registers (sg_stage<true>).
template <bool T>
__device__ __forceinline__ void sg_load(const bf16* __restrict__ src, long long ld, int r0, int k0, unsigned char* dst,
                                        int tid) {
    if constexpr (T) {
        sg_stage<true>(src, ld, r0, k0, dst, tid);
    } else {
#pragma unroll
        for (int q = 0; q < (SG_BM * 8) / SG_THREADS; ++q) {
            const int u = tid + SG_THREADS * q;
            const int row = u >> 3, kch = u & 7;
            const bf16* g = src + (size_t)(r0 + row) * ld + k0 + kch * 8;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst + tc_off(row, kch))), "l"(g)
                         : "memory");
        }
    }
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ uint4 pack8(const float* v) {
    uint4 o;
    o.x = pack_bf16(v[0], v[1]);
    o.y = pack_bf16(v[2], v[3]);
    o.z = pack_bf16(v[4], v[5]);
    o.w = pack_bf16(v[6], v[7]);
    return o;
}

__device__ __forceinline__ void unpack8(uint4 u, float* v) {
    const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        v[2 * j] = __uint_as_float(w[j] << 16);
        v[2 * j + 1] = __uint_as_float(w[j] & 0xFFFF0000u);
    }
}

// Grid (M/128, N/128, members), 256 threads.
template <bool AT, bool BT>
__global__ void __launch_bounds__(SG_THREADS, 2) sg_gemm(const SgArgs a, int* err) {
    extern __shared__ __align__(1024) unsigned char sg_smem_raw[];
    __shared__ __align__(8) uint64_t mbar[SG_STAGES];
    __shared__ uint32_t tmem_base_sh;
    unsigned char* sm = (unsigned char*)(((uintptr_t)sg_smem_raw + 1023) & ~(uintptr_t)1023);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int m0 = blockIdx.x * SG_BM, n0 = blockIdx.y * SG_BN, z = blockIdx.z;
    const bf16* A = a.A + (size_t)z * a.sA;
    const bf16* B = a.B + (size_t)z * a.sB;
    constexpr uint32_t TCOLS = SG_BN;
    constexpr uint32_t idesc = tc_idesc_bf16(SG_BM, SG_BN);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                     "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < SG_STAGES; ++q) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[q])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_sh;

    // chunk c of K lives in stage c % SG_STAGES; the MMAs of chunk c commit to that stage's
    // mbarrier (phase c / SG_STAGES), which frees the stage for chunk c + SG_STAGES
    const int nk = a.K / SG_KC;
    auto stA = [&](int c) { return sm + (c % SG_STAGES) * SG_STAGE_BYTES; };
    bool ok = true;
    int issued = 0;
#pragma unroll
    for (int c = 0; c < SG_STAGES - 1; ++c) {
        if (c < nk) {
            sg_load<AT>(A, a.lda, m0, c * SG_KC, stA(c), tid);
            sg_load<BT>(B, a.ldb, n0, c * SG_KC, stA(c) + SG_TILE_BYTES, tid);
        }
        cp_async_commit();
    }
    for (int kc = 0; kc < nk; ++kc) {
        const int nxt = kc + SG_STAGES - 1;
        if (nxt < nk) {
            if (nxt >= SG_STAGES) {  // the stage's previous chunk (kc - 1) must be consumed
                const bool w = mbar_wait(smem_u32(&mbar[nxt % SG_STAGES]), ((nxt - SG_STAGES) / SG_STAGES) & 1);
                ok = __syncthreads_and(w) != 0;
                if (!ok) break;
            }
            sg_load<AT>(A, a.lda, m0, nxt * SG_KC, stA(nxt), tid);
            sg_load<BT>(B, a.ldb, n0, nxt * SG_KC, stA(nxt) + SG_TILE_BYTES, tid);
        }
        cp_async_commit();
        cp_async_wait<SG_STAGES - 1>();  // this thread's copies of chunk kc have landed
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t aa = smem_u32(stA(kc)), bb = aa + SG_TILE_BYTES;
#pragma unroll
            for (int kk = 0; kk < SG_KC / 16; ++kk) {
                const uint32_t off = kk * 256;  // two 16-byte k-chunks per K=16 step
                tc_mma(tmem, tc_desc(aa + off, 128, 1024), tc_desc(bb + off, 128, 1024), idesc,
                       (kc > 0 || kk > 0) ? 1u : 0u);
            }
            tc_commit(smem_u32(&mbar[kc % SG_STAGES]));
        }
        issued = kc + 1;
    }
    cp_async_wait<0>();  // no copy in flight past this point
    if (issued > 0) {
        const int c = issued - 1;
        const bool w = mbar_wait(smem_u32(&mbar[c % SG_STAGES]), (c / SG_STAGES) & 1);
        ok = (__syncthreads_and(w) != 0) && ok && issued == nk;
    }
    if (!ok && tid == 0 && err) atomicOr(err, 1);
    tc_fence_after();
    if (ok) {
        const int quarter = warp & 3, half = warp >> 2;
        const int row = m0 + quarter * 32 + (tid & 31);
#pragma unroll 1
        for (int c0 = 0; c0 < SG_BN / 2; c0 += 32) {
            const int col = n0 + half * (SG_BN / 2) + c0;
            float v[32];
            tc_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(half * (SG_BN / 2) + c0), v);
            if (a.epi == EPI_F32) {
                float* c = a.C + (size_t)z * a.sC + (size_t)row * a.ldc + col;
#pragma unroll
                for (int j = 0; j < 32; j += 4) *reinterpret_cast<float4*>(c + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
            } else if (a.epi == EPI_FWD) {
                const float* bias = a.bias + (size_t)z * a.sbias + col;
                const size_t o = (size_t)row * a.ldy + col;
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] += __ldg(bias + j);
                if (a.Z) {
                    bf16* zp = a.Z + (size_t)z * a.sZ + o;
#pragma unroll
                    for (int j = 0; j < 32; j += 8) *reinterpret_cast<uint4*>(zp + j) = pack8(v + j);
                }
                if (a.act == 1) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) v[j] = silu(v[j]);
                }
                if (a.Y) {
                    bf16* yp = a.Y + (size_t)z * a.sY + o;
#pragma unroll
                    for (int j = 0; j < 32; j += 8) *reinterpret_cast<uint4*>(yp + j) = pack8(v + j);
                }
                if (a.Yf) {
                    float* yf = a.Yf + (size_t)z * a.sYf + o;
#pragma unroll
                    for (int j = 0; j < 32; j += 4) *reinterpret_cast<float4*>(yf + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
                }
            } else {  // EPI_BWD_DATA
                const size_t o = (size_t)row * a.ldy + col;
                const bf16* zp = a.Zp + (size_t)z * a.sZp + o;
#pragma unroll
                for (int j = 0; j < 32; j += 8) {
                    float zz[8];
                    unpack8(__ldg(reinterpret_cast<const uint4*>(zp + j)), zz);
#pragma unroll
                    for (int q = 0; q < 8; ++q) v[j + q] *= dsilu(zz[q]);
                }
                bf16* yp = a.Y + (size_t)z * a.sY + o;
#pragma unroll
                for (int j = 0; j < 32; j += 8) *reinterpret_cast<uint4*>(yp + j) = pack8(v + j);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS));
}

// Fourier-feature input: out[b, 0:8] = x, out[b, 8 + j] = sin(2 pi f_j . x),
// out[b, 8 + nf + j] = cos(2 pi f_j . x), j < nf = (ld - 8) / 2; f [nf x 8]. One thread per
// (b, j); members share the features.
__global__ void sg_features(const float* __restrict__ x, int B, const float* __restrict__ f, int nf, bf16* out, int ld) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)B * (nf + 8)) return;
    const int b = (int)(t / (nf + 8)), j = (int)(t % (nf + 8));
    const float* xb = x + (size_t)b * 8;
    bf16* o = out + (size_t)b * ld;
    if (j < 8) {
        o[j] = __float2bfloat16(xb[j]);
        return;
    }
    const int q = j - 8;
    float d = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) d += f[q * 8 + i] * xb[i];
    float s, c;
    sincospif(2.0f * d, &s, &c);
    o[8 + q] = __float2bfloat16(s);
    o[8 + nf + q] = __float2bfloat16(c);
}

// MSE over [members, B, N]: dY = 2 (Y - T) / (B N) as BF16, loss[z] += sum (Y - T)^2 / (B N).
__global__ void sg_mse(const float* __restrict__ Y, const float* __restrict__ T, long long sT, int B, int N,
                       bf16* dY, double* loss) {
    __shared__ double red[8];
    const int z = blockIdx.y;
    const long long n = (long long)B * N;
    const float* y = Y + (size_t)z * n;
    const float* tt = T + (size_t)z * sT;
    bf16* d = dY + (size_t)z * n;
    const float sc = 1.0f / (float)n;
    double acc = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float e = y[i] - tt[i];
        d[i] = __float2bfloat16(2.0f * e * sc);
        acc += (double)e * e;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        atomicAdd(loss + z, s / (double)n);
    }
}

// db[z, c] = sum_b dZ[z, b, c] (column sums), one thread per column.
__global__ void sg_colsum(const bf16* __restrict__ dZ, int B, int N, float* db) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x, z = blockIdx.y;
    if (c >= N) return;
    const bf16* p = dZ + (size_t)z * B * N + c;
    float s = 0;
    for (int b = 0; b < B; ++b) s += __bfloat162float(p[(size_t)b * N]);
    db[(size_t)z * N + c] = s;
}

// Adam (bias-corrected) on FP32 master parameters; wbf (may be null) receives the BF16
// working copy.
__global__ void sg_adam(float* p, float* m, float* v, const float* g, long long n, float lr, float b1, float b2,
                        float eps, float c1, float c2, bf16* wbf) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] = pi;
        if (wbf) wbf[i] = __float2bfloat16(pi);
    }
}

// Ensemble statistics of [members, B, N] outputs: mean[b, n], and per point the largest
// standard deviation over the first nspec columns (the spectral bins).
__global__ void sg_ensemble(const float* __restrict__ Y, int members, int B, int N, int nspec, float* mean,
                            float* spread) {
    __shared__ float red[8];
    const int b = blockIdx.x;
    float smax = 0;
    for (int c = threadIdx.x; c < N; c += blockDim.x) {
        float s = 0, s2 = 0;
        for (int z = 0; z < members; ++z) {
            const float y = Y[((size_t)z * B + b) * N + c];
            s += y;
            s2 += y * y;
        }
        const float mu = s / members;
        mean[(size_t)b * N + c] = mu;
        if (c < nspec && members > 1) smax = fmaxf(smax, sqrtf(fmaxf(s2 / members - mu * mu, 0.0f)));
    }
    for (int o = 16; o > 0; o >>= 1) smax = fmaxf(smax, __shfl_xor_sync(0xffffffffu, smax, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = smax;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s = fmaxf(s, red[w]);
        spread[b] = s;
    }
}

int launch_gemm(const SgArgs& a, int members, int* err, cudaStream_t st, bool at, bool bt) {
    if (a.M % SG_BM || a.N % SG_BN || a.K % SG_KC || members < 1) return 16;
    dim3 grid(a.M / SG_BM, a.N / SG_BN, members);
    cudaError_t e;
    if (!at && !bt) {
        e = cudaFuncSetAttribute(sg_gemm<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, SG_SMEM);
        if (e == cudaSuccess) sg_gemm<false, false><<<grid, SG_THREADS, SG_SMEM, st>>>(a, err);
    } else if (!at && bt) {
        e = cudaFuncSetAttribute(sg_gemm<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SG_SMEM);
        if (e == cudaSuccess) sg_gemm<false, true><<<grid, SG_THREADS, SG_SMEM, st>>>(a, err);
    } else if (at && bt) {
        e = cudaFuncSetAttribute(sg_gemm<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SG_SMEM);
        if (e == cudaSuccess) sg_gemm<true, true><<<grid, SG_THREADS, SG_SMEM, st>>>(a, err);
    } else {
        return 16;
    }
    if (e != cudaSuccess) return 18;
    return cudaGetLastError() == cudaSuccess ? 0 : 18;
}

}  // namespace

extern "C" {

// Forward of one linear layer for `members` ensemble members at once (device pointers,
// BF16 unless stated): Z = X W^T + b, Y = act(Z) (act 1: SiLU, 0: identity). X [B x K]
// (member stride sX), W [N x K] (stride N*K), b FP32 [N] (stride N); outputs [B x N] with
// member stride B*N: Y BF16 (may be null), Zout BF16 pre-activation (may be null), Yf FP32
// (may be null). B, N multiples of 128, K of 64. err: device int set on a wait timeout.
int luna_sg_linear_fwd(const void* X, long long sX, const void* W, const float* b, int B, int K, int N, int act,
                       void* Y, void* Zout, float* Yf, int members, int* err, void* stream) {
    SgArgs a = {};
    a.A = (const bf16*)X; a.lda = K; a.sA = sX;
    a.B = (const bf16*)W; a.ldb = K; a.sB = (long long)N * K;
    a.M = B; a.N = N; a.K = K;
    a.epi = EPI_FWD;
    a.bias = b; a.sbias = N; a.act = act;
    a.Y = (bf16*)Y; a.ldy = N; a.sY = (long long)B * N;
    a.Z = (bf16*)Zout; a.sZ = (long long)B * N;
    a.Yf = Yf; a.sYf = (long long)B * N;
    return launch_gemm(a, members, err, (cudaStream_t)stream, false, false);
}

// Backward data: dXpre = (dZ W) * silu'(Zprev) as BF16 [B x K] (member stride B*K), for the
// layer whose input was SiLU(Zprev); dZ [B x N] (stride B*N), W [N x K] (stride N*K).
int luna_sg_linear_bwd_data(const void* dZ, const void* W, const void* Zprev, int B, int K, int N, void* dXpre,
                            int members, int* err, void* stream) {
    SgArgs a = {};
    a.A = (const bf16*)dZ; a.lda = N; a.sA = (long long)B * N;
    a.B = (const bf16*)W; a.ldb = K; a.sB = (long long)N * K;   // element (k, n) = W[n*K + k]
    a.M = B; a.N = K; a.K = N;
    a.epi = EPI_BWD_DATA;
    a.Y = (bf16*)dXpre; a.ldy = K; a.sY = (long long)B * K;
    a.Zp = (const bf16*)Zprev; a.sZp = (long long)B * K;
    return launch_gemm(a, members, err, (cudaStream_t)stream, false, true);
}

// Backward weights: dW = dZ^T X as FP32 [N x K] (stride N*K), db = column sums of dZ FP32
// [N] (stride N); dZ [B x N] (stride B*N), X [B x K] (stride sX).
int luna_sg_linear_bwd_weight(const void* dZ, const void* X, long long sX, int B, int K, int N, float* dW, float* db,
                              int members, int* err, void* stream) {
    SgArgs a = {};
    a.A = (const bf16*)dZ; a.lda = N; a.sA = (long long)B * N;  // element (n, b) = dZ[b*N + n]
    a.B = (const bf16*)X; a.ldb = K; a.sB = sX;                 // element (k, b) = X[b*K + k]
    a.M = N; a.N = K; a.K = B;
    a.epi = EPI_F32;
    a.C = dW; a.ldc = K; a.sC = (long long)N * K;
    int rc = launch_gemm(a, members, err, (cudaStream_t)stream, true, true);
    if (rc) return rc;
    sg_colsum<<<dim3((N + 255) / 256, members), 256, 0, (cudaStream_t)stream>>>((const bf16*)dZ, B, N, db);
    return cudaGetLastError() == cudaSuccess ? 0 : 18;
}

// Fourier features of x [B x 8] FP32 into out [B x ld] BF16 (ld = 8 + 2 nf, f [nf x 8]).
int luna_sg_features(const float* x, int B, const float* f, int nf, void* out, int ld, void* stream) {
    if (ld != 8 + 2 * nf || B < 1) return 16;
    const long long n = (long long)B * (nf + 8);
    sg_features<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(x, B, f, nf, (bf16*)out, ld);
    return cudaGetLastError() == cudaSuccess ? 0 : 18;
}

// Mean squared error of Y [members x B x N] FP32 against T (member stride sT, 0 to share):
// dY BF16 (same shape) and loss[z] += mean squared error of member z (FP64).
int luna_sg_mse(const float* Y, const float* T, long long sT, int B, int N, void* dY, double* loss, int members,
                void* stream) {
    sg_mse<<<dim3(256, members), 256, 0, (cudaStream_t)stream>>>(Y, T, sT, B, N, (bf16*)dY, loss);
    return cudaGetLastError() == cudaSuccess ? 0 : 18;
}

// One Adam step (step number t >= 1) on n FP32 parameters; wbf (may be null) gets BF16.
int luna_sg_adam(float* p, float* m, float* v, const float* g, long long n, float lr, float b1, float b2, float eps,
                 int t, void* wbf, void* stream) {
    const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
    sg_adam<<<592, 256, 0, (cudaStream_t)stream>>>(p, m, v, g, n, lr, b1, b2, eps, c1, c2, (bf16*)wbf);
    return cudaGetLastError() == cudaSuccess ? 0 : 18;
}

// Ensemble mean [B x N] and per-point spread (largest member standard deviation over the
// first nspec outputs) of Y [members x B x N].
int luna_sg_ensemble(const float* Y, int members, int B, int N, int nspec, float* mean, float* spread, void* stream) {
    sg_ensemble<<<B, 256, 0, (cudaStream_t)stream>>>(Y, members, B, N, nspec, mean, spread);
    return cudaGetLastError() == cudaSuccess ? 0 : 18;
}

}  // extern "C"
