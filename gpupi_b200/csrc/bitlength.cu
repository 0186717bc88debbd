// Largest used bit / limb length over a batch (gpupi batch_bitlength.cu:33-245).
//
// One warp per row scans down from the top limb, 32 limbs per step, and stops
// at the first non-zero limb, so a row whose top limb is set costs one 128-byte
// read instead of a full pass.  Per-CTA maxima meet in one device word; the
// last CTA to finish (ticket counter) moves the result straight into pinned,
// mapped host memory and re-zeroes the word and the counter, so a call is one
// launch plus one stream synchronisation — no memset, no device-to-host copy.
// The two device words belong to the library (one pair per device, zeroed when
// first created) and return to zero after every call.  Calls are issued on the
// library's single stream, so they never overlap.
#include "common.cuh"
#include "batch_bitlength.h"

#include <mutex>

namespace gpupi {

template <bool BITS>
__global__ void __launch_bounds__(256) length_max_kernel(const uint32_t *__restrict__ A, uint32_t N, uint32_t L,
                                                         uint64_t stride, uint32_t *dev_max, uint32_t *dev_count,
                                                         volatile uint32_t *host_out) {
    __shared__ uint32_t cta_max;
    __shared__ bool last;
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
                const uint32_t hl = (uint32_t)(__ffs(nz) - 1);   // lowest lane = highest limb
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
    if (threadIdx.x == 0) {
        if (cta_max) atomicMax(dev_max, cta_max);
        __threadfence();
        const uint32_t ticket = atomicAdd(dev_count, 1u);
        last = (ticket == gridDim.x - 1u);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        const uint32_t v = atomicExch(dev_max, 0u);
        *host_out = v;
        __threadfence_system();
        atomicExch(dev_count, 0u);
    }
}

namespace {
struct LengthState {
    uint32_t *dev = nullptr;            // [0] = max, [1] = ticket counter
    volatile uint32_t *host = nullptr;  // pinned, mapped
    uint32_t *host_dev = nullptr;       // device view of host
};
LengthState g_len[64];
std::mutex g_len_mu;

LengthState *length_state() {
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 64) return nullptr;
    std::lock_guard<std::mutex> g(g_len_mu);
    LengthState &s = g_len[d];
    if (!s.dev) {
        uint32_t *dev = nullptr;
        void *host = nullptr;
        if (cudaMalloc(&dev, 2 * sizeof(uint32_t)) != cudaSuccess) return nullptr;
        if (cudaMemset(dev, 0, 2 * sizeof(uint32_t)) != cudaSuccess ||
            cudaHostAlloc(&host, sizeof(uint32_t), cudaHostAllocMapped) != cudaSuccess) {
            cudaFree(dev);
            return nullptr;
        }
        uint32_t *hd = nullptr;
        if (cudaHostGetDevicePointer((void **)&hd, host, 0) != cudaSuccess) {
            cudaFree(dev);
            cudaFreeHost(host);
            return nullptr;
        }
        cudaDeviceSynchronize();
        s.dev = dev;
        s.host = (volatile uint32_t *)host;
        s.host_dev = hd;
    }
    return &s;
}
}  // namespace

template <bool BITS>
static uint32_t length_max(const uint32_t *A, uint32_t *workspace, uint32_t N, uint32_t L, uint32_t stride) {
    (void)workspace;
    if (N == 0u || L == 0u) return 0u;
    LengthState *s = length_state();
    if (!s) return 0u;
    cudaStream_t st = current_stream();
    *s->host = 0xffffffffu;
    length_max_kernel<BITS><<<grid_for(N, 8, kNumSMs * 8), 256, 0, st>>>(A, N, L, stride, s->dev, s->dev + 1,
                                                                        s->host_dev);
    count_launch();
    cudaStreamSynchronize(st);
    note_d2h(sizeof(uint32_t));
    return *s->host;
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
