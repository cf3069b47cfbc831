// FMA throughput of this GPU in FP32 and FP64 (the compute ceilings of the solver's
// roofline), measured with CUDA events. Each thread runs 8 independent multiply-add chains
// in registers (no memory traffic inside the timed loop); one store per thread at the end
// keeps the chains alive. Grid: 8 CTAs of 256 threads per SM, a multiple of the SM count.
#include <cuda_runtime.h>

namespace {

template <typename T>
__global__ void __launch_bounds__(256) fma_chains(T* out, int iters, T a, T b) {
    T x0 = (T)threadIdx.x, x1 = x0 + (T)1, x2 = x0 + (T)2, x3 = x0 + (T)3;
    T x4 = x0 + (T)4, x5 = x0 + (T)5, x6 = x0 + (T)6, x7 = x0 + (T)7;
#pragma unroll 1
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
}

template <typename T>
int run(double* tflops, float* ms_out, int iters) {
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 1;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 1;
    const int blocks = nsm * 8, threads = 256;
    T* out = nullptr;
    if (cudaMalloc(&out, sizeof(T) * blocks * threads) != cudaSuccess) return 1;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    // a = 1 - 2^-20, b = 2^-20 keep every chain finite and away from denormals
    const T a = (T)(1.0 - 1.0 / 1048576.0), b = (T)(1.0 / 1048576.0);
    fma_chains<T><<<blocks, threads>>>(out, iters / 8 + 1, a, b);  // warm-up
    float best = 1e30f;
    for (int r = 0; r < 5; ++r) {
        cudaEventRecord(e0);
        fma_chains<T><<<blocks, threads>>>(out, iters, a, b);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return 1;
    const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    *ms_out = best;
    return 0;
}

}  // namespace

extern "C" {
// Peak FMA throughput (2 flops per FMA) in TFLOP/s: fp64 != 0 for FP64, else FP32. The
// fastest of 5 launches of `iters` x 128 FMAs per thread. Returns 0 on success.
int luna_peaks_fma(int fp64, int iters, double* tflops, float* ms) {
    if (!tflops || !ms || iters < 1) return 1;
    return fp64 ? run<double>(tflops, ms, iters) : run<float>(tflops, ms, iters);
}
}
