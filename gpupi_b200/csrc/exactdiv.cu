// In-place exact division by an odd 32-bit divisor, modulo 2^(32L)
// (gpupi batch_exactdiv_small.cu:15-141).
//
// Hensel (2-adic) division, least significant limb first:
//   t_i = a_i - c_i;  q_i = t_i * B^-1 mod 2^32;  c_{i+1} = hi(q_i * B) + [a_i < c_i]
// which yields the unique q with q*B == A mod 2^(32L) (the quotient when B | A).
// One thread per row; rows are staged through shared memory 32 limbs at a
// time so that global loads and stores stay coalesced.
#include "common.cuh"
#include "batch_exactdiv_small.h"

namespace gpupi {

constexpr uint32_t kDivRows = 32;   // rows per warp
constexpr uint32_t kDivWarps = 4;

__global__ void __launch_bounds__(kDivRows * kDivWarps) exactdiv_kernel(uint32_t *A, uint32_t B,
                                                                      uint32_t Binv, uint32_t N,
                                                                      uint32_t L, uint64_t stride) {
    __shared__ uint32_t tile[kDivWarps][32][33];
    const uint32_t lane = lane_id();
    const uint32_t w = threadIdx.x >> 5;
    for (uint64_t base = ((uint64_t)blockIdx.x * kDivWarps + w) * kDivRows; base < N;
         base += (uint64_t)gridDim.x * kDivWarps * kDivRows) {
        const uint32_t rows = (uint32_t)((N - base) < kDivRows ? (N - base) : kDivRows);
        uint32_t c = 0u;
        for (uint32_t l0 = 0; l0 < L; l0 += 32u) {
            const uint32_t len = min(32u, L - l0);
            // coalesced load: lane = limb, loop over rows
            for (uint32_t r = 0; r < rows; ++r)
                tile[w][r][lane] = (lane < len) ? A[(base + r) * stride + l0 + lane] : 0u;
            __syncwarp();
            if (lane < rows) {
                for (uint32_t k = 0; k < len; ++k) {
                    const uint32_t a = tile[w][lane][k];
                    const uint32_t t = a - c;
                    const uint32_t q = t * Binv;
                    c = __umulhi(q, B) + (a < c ? 1u : 0u);
                    tile[w][lane][k] = q;
                }
            }
            __syncwarp();
            for (uint32_t r = 0; r < rows; ++r)
                if (lane < len) A[(base + r) * stride + l0 + lane] = tile[w][r][lane];
            __syncwarp();
        }
    }
}

static uint32_t inverse_mod_2_32(uint32_t b) {
    uint32_t x = b;  // correct to 3 bits for odd b
    for (int i = 0; i < 5; ++i) x *= 2u - b * x;
    return x;
}

}  // namespace gpupi

void batch_exactdiv_small(uint32_t *A, uint32_t B, uint32_t N, uint32_t L, uint32_t stride_A) {
    using namespace gpupi;
    if (N == 0u || L == 0u || (B & 1u) == 0u) return;
    const uint32_t binv = inverse_mod_2_32(B);
    exactdiv_kernel<<<grid_for(N, kDivRows * kDivWarps, kNumSMs * 8), kDivRows * kDivWarps, 0,
                      current_stream()>>>(A, B, binv, N, L, stride_A);
    GPUPI_LAUNCH_CHECK();
}
