// FP64 peak micro-benchmark: DFMA on the CUDA cores and mma.sync.m8n8k4.f64 (the FP64 tensor
// instruction the DWT kernels use), each as many independent chains over all SMs. Prints the
// achieved TFLOP/s; the DWT roofline uses the larger of the two. Built and run by
// `python -m pfsoftlib_b200.peaks`.
#include <cstdio>
#include <cuda_runtime.h>
__global__ void dfma_kernel(double* out, int iters, double a, double b) {
    double x[16];
    for (int i = 0; i < 16; ++i) x[i] = threadIdx.x * 1e-3 + i;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 16; ++i) x[i] = fma(x[i], a, b);
    }
    double s = 0; for (int i = 0; i < 16; ++i) s += x[i];
    if (s == 12345.678) out[threadIdx.x] = s;
}
__global__ void dmma_kernel(double* out, int iters) {
    double a = threadIdx.x * 1e-3, b = 1.0 + threadIdx.x * 1e-4;
    double c[8][2];
    for (int i = 0; i < 8; ++i) { c[i][0] = 0; c[i][1] = 0; }
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                         : "+d"(c[i][0]), "+d"(c[i][1]) : "d"(a), "d"(b));
    }
    double s = 0; for (int i = 0; i < 8; ++i) s += c[i][0] + c[i][1];
    if (s == 12345.678) out[threadIdx.x] = s;
}
int main() {
    int sms; cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    double* out; cudaMalloc(&out, 1 << 20);
    cudaEvent_t e0, e1; cudaEventCreate(&e0); cudaEventCreate(&e1);
    int blocks = sms * 4, threads = 256, iters = 20000;
    for (int rep = 0; rep < 2; ++rep) {
        cudaEventRecord(e0);
        dfma_kernel<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
        cudaEventRecord(e1); cudaEventSynchronize(e1);
        float ms; cudaEventElapsedTime(&ms, e0, e1);
        double flops = 2.0 * 16 * iters * (double)blocks * threads;
        if (rep) printf("DFMA: %.2f TFLOP/s (%.3f ms)\n", flops / ms / 1e9, ms);
    }
    for (int rep = 0; rep < 2; ++rep) {
        cudaEventRecord(e0);
        dmma_kernel<<<blocks, threads>>>(out, iters / 4);
        cudaEventRecord(e1); cudaEventSynchronize(e1);
        float ms; cudaEventElapsedTime(&ms, e0, e1);
        double flops = 2.0 * 256 * 8 * (iters / 4) * (double)blocks * threads / 32;
        if (rep) printf("DMMA m8n8k4: %.2f TFLOP/s (%.3f ms)\n", flops / ms / 1e9, ms);
    }
    printf("err %s\n", cudaGetErrorString(cudaGetLastError()));
    return 0;
}
