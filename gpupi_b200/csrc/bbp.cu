// BBP hex digits of pi at arbitrary positions, an independent spot check of
// RET (the pipeline's binary fraction of pi).  Integer fixed point only.
//
//   frac(16^n pi) = frac(4 S1 - 2 S4 - S5 - S6),
//   S_j = sum_{k<=n} frac(16^(n-k) / (8k+j)) + sum_{k>n} 16^(n-k) / (8k+j)
//
// Every term is carried as floor(2^64 * frac(.)) in a uint64, so sums wrap
// modulo 1 exactly as the fractional part does.  The denominators 8k+4 and
// 8k+6 are even; with e = n - k >= 1 their terms are rewritten over odd
// moduli: 16^e/(8k+4) = 4 16^(e-1)/(2k+1), 16^e/(8k+6) = 8 16^(e-1)/(4k+3).
// So every term of the first sum is frac(2^E / m) with m odd, computed as
//   t = 2^E * 2^64 mod m   (left-to-right powering in Montgomery form,
//                           R = 2^64, doubling = shift and subtract)
//   floor(2^64 frac(2^E/m)) = (v 2^64 - t) / m = -t * m^-1 mod 2^64
// (the division is exact, so it is one multiplication by the inverse).
// Each term is truncated, so the sum of 4(n+17) terms with weights
// 4, 2, 1, 1 is within 8 (n + 17) units of 2^-64 of the exact fraction;
// callers compare only bits that this bound cannot flip.
#include "common.cuh"

#include <vector>

namespace gpupi {
namespace {

// x * y / 2^64 mod m for odd m < 2^34, x, y < m; mneg = -m^-1 mod 2^64.
__device__ __forceinline__ uint64_t mont64(uint64_t x, uint64_t y, uint64_t m, uint64_t mneg) {
    const uint64_t lo = x * y;
    const uint64_t hi = __umul64hi(x, y);
    const uint64_t u = lo * mneg;   // lo + lo(u m) = 0 mod 2^64
    const uint64_t r = hi + __umul64hi(u, m) + (lo != 0u ? 1u : 0u);
    return r >= m ? r - m : r;
}

// floor(2^64 * frac(2^E / m)), m odd, 1 <= m < 2^34
__device__ __forceinline__ uint64_t frac_pow2(uint64_t E, uint64_t m) {
    uint64_t inv = m;   // m^-1 mod 2^64: m m = 1 mod 8, each Newton step doubles the bits
#pragma unroll
    for (int i = 0; i < 5; ++i) inv *= 2u - m * inv;
    const uint64_t mneg = 0u - inv;
    uint64_t x = (0u - m) % m;   // 2^64 mod m: Montgomery form of 1
    if (E != 0u) {
        const int top = 63 - __clzll((long long)E);
        x <<= 1;   // leading bit: 2^1
        if (x >= m) x -= m;
        for (int b = top - 1; b >= 0; --b) {
            x = mont64(x, x, m, mneg);
            if ((E >> b) & 1u) {
                x <<= 1;
                if (x >= m) x -= m;
            }
        }
    }
    return (0u - x) * inv;
}

// floor(2^64 / m), m >= 2
__device__ __forceinline__ uint64_t recip64(uint64_t m) {
    const uint64_t all = ~0ull;
    uint64_t q = all / m;
    if (all % m == m - 1u) ++q;   // m divides 2^64
    return q;
}

__global__ void __launch_bounds__(256) bbp_kernel(uint64_t n, unsigned long long *acc) {
    uint64_t sum = 0u;
    const uint64_t terms = 4u * (n + 1u);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < terms; t += stride) {
        const uint64_t k = t >> 2;
        const uint32_t which = (uint32_t)(t & 3u);   // j = 1, 4, 5, 6
        const uint64_t e = n - k;
        uint64_t q;
        if ((which == 1u || which == 3u) && e == 0u) {
            q = recip64(8u * n + (which == 1u ? 4u : 6u));   // k = n: 1/(8n+j) itself
        } else {
            uint64_t E, m;
            if (which == 0u) {
                E = 4u * e;
                m = 8u * k + 1u;
            } else if (which == 1u) {
                E = 4u * e - 2u;
                m = 2u * k + 1u;
            } else if (which == 2u) {
                E = 4u * e;
                m = 8u * k + 5u;
            } else {
                E = 4u * e - 1u;
                m = 4u * k + 3u;
            }
            q = frac_pow2(E, m);
        }
        sum += (which == 0u) ? (q << 2) : (which == 1u ? (0u - (q << 1)) : (0u - q));
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // tail k > n: 16^(n-k) / (8k+j) = 2^(64 - 4d) / (8k+j) units, d = k - n < 16
        for (uint64_t d = 1; d < 16; ++d) {
            const uint64_t k = n + d;
            const uint64_t num = 1ull << (64 - 4 * d);
            sum += (num / (8u * k + 1u)) << 2;
            sum -= (num / (8u * k + 4u)) << 1;
            sum -= num / (8u * k + 5u);
            sum -= num / (8u * k + 6u);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
    if (lane_id() == 0) atomicAdd(acc, (unsigned long long)sum);
}

}  // namespace

// fractions[i] = floor-ish(2^64 frac(16^positions[i] pi)), within
// 8 (positions[i] + 17) units of the exact value.
cudaError_t bbp_fractions(const uint64_t *positions, uint32_t count, uint64_t *fractions) {
    if (count == 0u) return cudaSuccess;
    if (!positions || !fractions) return cudaErrorInvalidValue;
    for (uint32_t i = 0; i < count; ++i)
        if (positions[i] > (1ull << 30)) return cudaErrorInvalidValue;   // moduli stay below 2^34
    cudaStream_t st = current_stream();
    unsigned long long *acc = nullptr;
    cudaError_t err = scratch_alloc((void **)&acc, (size_t)count * 8u);
    if (err != cudaSuccess) return err;
    err = cudaMemsetAsync(acc, 0, (size_t)count * 8u, st);
    for (uint32_t i = 0; i < count && err == cudaSuccess; ++i) {
        bbp_kernel<<<kNumSMs * 8, 256, 0, st>>>(positions[i], acc + i);
        count_launch();
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpyAsync(fractions, acc, (size_t)count * 8u, cudaMemcpyDeviceToHost, st);
    note_d2h((size_t)count * 8u);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
    scratch_free(acc);
    return err;
}

}  // namespace gpupi
