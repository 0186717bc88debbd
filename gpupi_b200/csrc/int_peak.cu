// Integer-pipe peaks of the GPU this runs on: the ceiling the limb kernels
// are measured against (the NTT passes execute ~66 integer instructions per
// point and move 12 bytes, so HBM bandwidth is not what bounds them).
//
//   k_peak_imad: 32-bit multiply-adds (mad.lo.u32 -> IMAD, the FMA-heavy
//                pipe), eight independent chains per thread;
//   k_peak_alu:  three-input logic (LOP3, the ALU pipe), eight chains.
// Both run two CTAs of 1024 threads per SM for `iters` iterations; the rate
// is warp instructions per second (thread operations / 32), timed with CUDA
// events after a warm-up launch.  The chains' results are stored so that
// nothing is optimised away.
#include "common.cuh"

namespace gpupi {
namespace {

__global__ void __launch_bounds__(1024) k_peak_imad(uint32_t *out, uint32_t iters, uint32_t seed) {
    uint32_t a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + threadIdx.x * 8u + k;
    const uint32_t m = seed | 1u, c = seed ^ 0x9e3779b9u;
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[k]) : "r"(m), "r"(c));
    }
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s ^= a[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(1024) k_peak_alu(uint32_t *out, uint32_t iters, uint32_t seed) {
    uint32_t a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + threadIdx.x * 8u + k;
    const uint32_t b = seed | 1u, c = seed ^ 0x9e3779b9u;
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k)
            asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(a[k]) : "r"(b), "r"(c));   // a ^ b ^ c
    }
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s ^= a[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

// Warp instructions per second of each pipe (best of `reps` launches).
cudaError_t int_peak(double *imad_winst_per_s, double *alu_winst_per_s) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned blocks = 2u * (unsigned)sms, threads = 1024u;
    const uint32_t iters = 1u << 14;
    uint32_t *out = nullptr;
    cudaError_t err = cudaMalloc(&out, (size_t)blocks * threads * 4);
    if (err != cudaSuccess) return err;
    cudaStream_t st = current_stream();
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const double winst = (double)blocks * threads / 32.0 * iters * 8.0;
    for (int pipe = 0; pipe < 2; ++pipe) {
        float best = 1e30f;
        for (int r = 0; r < 4; ++r) {
            cudaEventRecord(e0, st);
            if (pipe == 0)
                k_peak_imad<<<blocks, threads, 0, st>>>(out, iters, 12345u + r);
            else
                k_peak_alu<<<blocks, threads, 0, st>>>(out, iters, 12345u + r);
            count_launch();
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (r > 0) best = std::min(best, ms);   // the first launch warms up
        }
        const double rate = winst / (best * 1e-3);
        if (pipe == 0 && imad_winst_per_s) *imad_winst_per_s = rate;
        if (pipe == 1 && alu_winst_per_s) *alu_winst_per_s = rate;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    err = cudaGetLastError();
    cudaFree(out);
    return err;
}

}  // namespace gpupi
