// FP32 fused multiply-add throughput of the current device, measured: the
// denominator for the arithmetic rate of the convolutions (whose bit-exact
// taps are a separate multiply and add each, i.e. half the fused rate at best).
#include "kernels.cuh"

namespace aprb {

namespace {

constexpr int kChains = 16;  // independent FMA chains per thread (latency cover)

__global__ void __launch_bounds__(256) fma_peak_kernel(const float *__restrict__ seed, float *__restrict__ sink,
                                                       int iters) {
    const float b = seed[0], c = seed[1];
    float a[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = seed[2] + 1e-7f * (float)(threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) a[k] = __fmaf_rn(a[k], b, c);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += a[k];
    if (s == -1.0f) sink[blockIdx.x * blockDim.x + threadIdx.x] = s;  // never true: keeps the chains live
}

}  // namespace

double measure_fp32_fma_tflops(cudaStream_t s) {
    static thread_local DevBuf buf;
    float *d = buf.as<float>(4);
    const float h[4] = {0.9990234375f, 0.0009765625f, 0.5f, 0.0f};  // a -> c / (1 - b) = 1: finite, normal
    APRB_CUDA(cudaMemcpyAsync(d, h, sizeof(h), cudaMemcpyHostToDevice, s));
    int dev = 0, sms = 0;
    APRB_CUDA(cudaGetDevice(&dev));
    APRB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = sms * 8, threads = 256, iters = 8192;
    cudaEvent_t e0, e1;
    APRB_CUDA(cudaEventCreate(&e0));
    APRB_CUDA(cudaEventCreate(&e1));
    fma_peak_kernel<<<blocks, threads, 0, s>>>(d, d, iters);  // warm-up
    APRB_CUDA(cudaEventRecord(e0, s));
    fma_peak_kernel<<<blocks, threads, 0, s>>>(d, d, iters);
    APRB_CUDA(cudaEventRecord(e1, s));
    count_launch(2);
    APRB_CHECK_LAUNCH();
    APRB_CUDA(cudaEventSynchronize(e1));
    float ms = 0.0f;
    APRB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double flops = 2.0 * kChains * (double)iters * blocks * threads;
    return flops / (ms * 1e-3) / 1e12;
}

}  // namespace aprb
