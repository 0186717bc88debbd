// Largest used bit / limb length over a batch (gpupi batch_bitlength.cu:33-245).
//
// One warp per row scans down from the top limb, 32 limbs per step, and stops
// at the first non-zero limb, so a row whose top limb is set costs one 128-byte
// read instead of a full pass.  Per-CTA maxima are combined with one
// atomicMax into a device word that the host then reads (the API returns the
// value synchronously, like the reference).
#include "common.cuh"
#include "batch_bitlength.h"

namespace gpupi {

template <bool BITS>
__global__ void __launch_bounds__(256) length_max_kernel(const uint32_t *__restrict__ A,
                                                         uint32_t *result, uint32_t N, uint32_t L,
                                                         uint64_t stride) {
    __shared__ uint32_t cta_max;
    if (threadIdx.x == 0) cta_max = 0u;
    __syncthreads();
    const uint32_t lane = lane_id();
    const uint32_t wpc = blockDim.x >> 5;
    uint32_t best = 0u;
    for (uint32_t row = blockIdx.x * wpc + (threadIdx.x >> 5); row < N; row += gridDim.x * wpc) {
        const uint32_t *a = A + row * stride;
        for (int64_t top = (int64_t)L - 1; top >= 0; top -= 32) {
            const int64_t j = top - lane;
            const uint32_t v = (j >= 0) ? a[j] : 0u;
            const uint32_t nz = __ballot_sync(0xffffffffu, v != 0u);
            if (nz != 0u) {
                const uint32_t hl = (uint32_t)(__ffs(nz) - 1);  // lowest lane = highest limb
                const uint32_t limb = (uint32_t)(top - hl);
                const uint32_t topv = __shfl_sync(0xffffffffu, v, hl);
                const uint32_t len = BITS ? limb * 32u + (32u - __clz(topv)) : limb + 1u;
                best = max(best, len);
                break;
            }
        }
    }
    if (lane == 0 && best) atomicMax(&cta_max, best);
    __syncthreads();
    if (threadIdx.x == 0 && cta_max) atomicMax(result, cta_max);
}

template <bool BITS>
static uint32_t length_max(const uint32_t *A, uint32_t *workspace, uint32_t N, uint32_t L,
                           uint32_t stride) {
    if (N == 0u || L == 0u) return 0u;
    cudaStream_t st = current_stream();
    cudaMemsetAsync(workspace, 0, sizeof(uint32_t), st);
    length_max_kernel<BITS><<<grid_for(N, 8, kNumSMs * 8), 256, 0, st>>>(A, workspace, N, L, stride);
    GPUPI_LAUNCH_CHECK();
    uint32_t h = 0u;
    cudaMemcpyAsync(&h, workspace, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    note_d2h(sizeof(uint32_t));
    cudaStreamSynchronize(st);
    return h;
}

}  // namespace gpupi

uint32_t batch_bitlength_max(const uint32_t *A, uint32_t *workspace, uint32_t N, uint32_t L,
                             uint32_t stride_A) {
    return gpupi::length_max<true>(A, workspace, N, L, stride_A);
}

uint32_t batch_limblength_max(const uint32_t *A, uint32_t *workspace, uint32_t N, uint32_t L,
                              uint32_t stride_A) {
    return gpupi::length_max<false>(A, workspace, N, L, stride_A);
}

size_t batch_bitlength_workspace_size(uint32_t N, uint32_t L) {
    (void)N;
    (void)L;
    return 4;
}
