// Batched signed bit shift (gpupi batch_shift.cu:22-112).
//
// out_j = bits [32j - s, 32j - s + 32) of A (s = shift, positive = left),
// with A read as zero outside [0, L_in) and the result truncated to L_out
// limbs.  Pure gather: each thread produces 4 consecutive output limbs from
// at most 5 input limbs, so loads and stores are contiguous across a warp.
// HBM-bound: algorithmic bytes = 4 * (N*L_in_read + N*L_out).
#include "common.cuh"
#include "batch_shift.h"

namespace gpupi {

constexpr uint32_t kShiftPerThread = 4;

__global__ void __launch_bounds__(256) shift_bits_kernel(const uint32_t *__restrict__ A,
                                                         uint32_t *__restrict__ B, uint32_t N,
                                                         uint32_t L_in, uint32_t L_out,
                                                         uint64_t s_in, uint64_t s_out,
                                                         int32_t shift_bits,
                                                         uint32_t chunks_per_row) {
    const uint64_t total = (uint64_t)N * chunks_per_row;
    // Left shift by s: out_j = (a_{j-w} << b) | (a_{j-w-1} >> (32-b)).
    // Right shift by s: out_j = (a_{j+w} >> b) | (a_{j+w+1} << (32-b)).
    const bool left = shift_bits >= 0;
    const uint32_t mag = left ? (uint32_t)shift_bits : (uint32_t)(-(int64_t)shift_bits);
    const uint32_t w = mag >> 5;
    const uint32_t b = mag & 31u;
    for (uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t row = (uint32_t)(idx / chunks_per_row);
        const uint32_t j0 = (uint32_t)(idx - (uint64_t)row * chunks_per_row) * kShiftPerThread;
        const uint32_t *a = A + row * s_in;
        uint32_t *o = B + row * s_out;
        // source window: for left, limbs j0-w-1 .. j0-w+3; for right j0+w .. j0+w+4
        int64_t src0 = left ? (int64_t)j0 - (int64_t)w - 1 : (int64_t)j0 + (int64_t)w;
        uint32_t win[kShiftPerThread + 1];
#pragma unroll
        for (uint32_t k = 0; k <= kShiftPerThread; ++k) {
            const int64_t s = src0 + k;
            win[k] = (s >= 0 && s < (int64_t)L_in) ? a[s] : 0u;
        }
#pragma unroll
        for (uint32_t k = 0; k < kShiftPerThread; ++k) {
            const uint32_t j = j0 + k;
            if (j >= L_out) break;
            uint32_t r;
            if (left) {
                r = (b == 0u) ? win[k + 1] : ((win[k + 1] << b) | (win[k] >> (32u - b)));
            } else {
                r = (b == 0u) ? win[k] : ((win[k] >> b) | (win[k + 1] << (32u - b)));
            }
            o[j] = r;
        }
    }
}

}  // namespace gpupi

void batch_shift_bits(const uint32_t *A, uint32_t *B, uint32_t N, uint32_t L_in, uint32_t L_out,
                      uint32_t stride_in, uint32_t stride_out, int32_t shift_bits) {
    using namespace gpupi;
    if (N == 0u || L_out == 0u) return;
    const uint32_t chunks = (L_out + kShiftPerThread - 1) / kShiftPerThread;
    const uint64_t total = (uint64_t)N * chunks;
    KernelTimed kt("shift", 8.0 * N * (double)L_out);
    shift_bits_kernel<<<grid_for(total, 256, kNumSMs * 32), 256, 0, current_stream()>>>(
        A, B, N, L_in, L_out, stride_in, stride_out, shift_bits, chunks);
    GPUPI_LAUNCH_CHECK();
}
