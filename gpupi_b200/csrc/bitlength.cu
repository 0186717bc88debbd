// Largest used bit / limb length over a batch (gpupi batch_bitlength.cu:33-245).
//
// Long rows (unless there are very many): 4096-limb chunks scanned from the
// top by all CTAs; a CTA stops at the first chunk that cannot beat the best
// length found so far (every later chunk of its sequence lies lower).  Short rows, or very many rows: one thread per row, bounded by the
// best length seen so far.  Per-CTA maxima meet in one device word; the
// last CTA to finish (ticket counter) moves the result straight into pinned,
// mapped host memory and re-zeroes the word and the counter, so a call is one
// launch plus one stream synchronisation — no memset, no device-to-host copy.
// The two device words belong to the library (one pair per device and
// stream, zeroed when first created) and return to zero after every call.
// Calls on one stream run in order, so a pair is never used by two scans at
// once; scans on different streams (the splitting tree's graph on its own
// stream, other work beside it) use different pairs.
#include "common.cuh"
#include "batch_bitlength.h"

#include <deque>
#include <mutex>

namespace gpupi {

// Few (long) rows: the rows are cut into 4096-limb chunks counted from the
// top; work item w = (chunk c, row) with c major, so the first wave of CTAs
// reads the top chunk of every row.  A chunk is skipped when even its top
// limb could not beat the best length already published in dev_max, so a
// call usually reads one wave of chunks however long the zero run above the
// highest set limb is.
constexpr uint32_t kChunk = 4096;   // 256 threads x 16 limbs

template <bool BITS>
__global__ void __launch_bounds__(256) length_max_chunks_kernel(const uint32_t *__restrict__ A, uint32_t N,
                                                                uint32_t L, uint64_t stride, uint64_t items,
                                                                uint32_t *dev_max, uint32_t *dev_count,
                                                                volatile uint32_t *host_out) {
    __shared__ uint32_t cta_max;
    __shared__ bool last;
    __shared__ bool skip;
    for (uint64_t w = blockIdx.x; w < items; w += gridDim.x) {
        const uint32_t row = (uint32_t)(w % N);
        const uint64_t c = w / N;
        const int64_t hi = (int64_t)L - (int64_t)(c * kChunk);   // chunk covers [hi - 4096, hi)
        if (threadIdx.x == 0) {
            const uint32_t cur = *((volatile uint32_t *)dev_max);
            const uint64_t best_possible = BITS ? (uint64_t)hi * 32u : (uint64_t)hi;
            skip = best_possible <= cur;
            cta_max = 0u;
        }
        __syncthreads();
        // items run top chunk first (chunk index major): once a chunk cannot
        // beat the best length, no later item of this CTA can either
        if (skip) break;
        {
            const uint32_t *a = A + row * stride;
            uint32_t best = 0u;
#pragma unroll 4
            for (int k = 0; k < 16; ++k) {
                // k-th 256-limb slab from the top of the chunk, coalesced across the CTA
                const int64_t j = hi - 1 - (int64_t)k * 256 - (int64_t)threadIdx.x;
                if (j >= 0 && j > hi - 1 - (int64_t)kChunk) {
                    const uint32_t v = a[j];
                    if (v != 0u) {
                        const uint32_t len = BITS ? (uint32_t)j * 32u + (32u - __clz(v)) : (uint32_t)j + 1u;
                        best = max(best, len);
                    }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
            if (lane_id() == 0 && best) atomicMax(&cta_max, best);
            __syncthreads();
            if (threadIdx.x == 0 && cta_max) atomicMax(dev_max, cta_max);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
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

// Many rows: one thread per row, reading down from the top limb only while
// the row could still beat the longest length this thread has seen (after
// the first row that is usually a single 4-byte read per row).
template <bool BITS>
__global__ void __launch_bounds__(256) length_max_rows_kernel(const uint32_t *__restrict__ A, uint32_t N,
                                                              uint32_t L, uint64_t stride, uint32_t *dev_max,
                                                              uint32_t *dev_count, volatile uint32_t *host_out) {
    __shared__ uint32_t cta_max;
    __shared__ bool last;
    if (threadIdx.x == 0) cta_max = 0u;
    __syncthreads();
    uint32_t best = 0u;
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < N; row += gridDim.x * blockDim.x) {
        const uint32_t *a = A + row * stride;
        const int64_t floor_limb = BITS ? (int64_t)(best >> 5) : (int64_t)best;
        for (int64_t j = (int64_t)L - 1; j >= floor_limb; --j) {
            const uint32_t v = a[j];
            if (v != 0u) {
                const uint32_t len = BITS ? (uint32_t)j * 32u + (32u - __clz(v)) : (uint32_t)j + 1u;
                best = max(best, len);
                break;
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
    if (lane_id() == 0 && best) atomicMax(&cta_max, best);
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
    int dev_id = -1;
    cudaStream_t stream = nullptr;
    uint32_t *dev = nullptr;            // [0] = max, [1] = ticket counter
    volatile uint32_t *host = nullptr;  // pinned, mapped
    uint32_t *host_dev = nullptr;       // device view of host
};
// Entries are never removed: graphs captured on a stream keep their pair's
// addresses.  A deque keeps them in place as it grows.
std::deque<LengthState> g_len;
std::mutex g_len_mu;

LengthState *length_state() {
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0) return nullptr;
    const cudaStream_t st = current_stream();
    std::lock_guard<std::mutex> g(g_len_mu);
    for (LengthState &e : g_len)
        if (e.dev_id == d && e.stream == st) return &e;
    g_len.push_back(LengthState{});
    LengthState &s = g_len.back();
    s.dev_id = d;
    s.stream = st;
    {
        uint32_t *dev = nullptr;
        void *host = nullptr;
        if (cudaMalloc(&dev, 2 * sizeof(uint32_t)) != cudaSuccess) {
            g_len.pop_back();
            return nullptr;
        }
        if (cudaMemset(dev, 0, 2 * sizeof(uint32_t)) != cudaSuccess ||
            cudaHostAlloc(&host, sizeof(uint32_t), cudaHostAllocMapped) != cudaSuccess) {
            cudaFree(dev);
            g_len.pop_back();
            return nullptr;
        }
        uint32_t *hd = nullptr;
        if (cudaHostGetDevicePointer((void **)&hd, host, 0) != cudaSuccess) {
            cudaFree(dev);
            cudaFreeHost(host);
            g_len.pop_back();
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
    // one thread per row only for short rows or very many rows: a thread
    // reads its row from the top one limb at a time, which for rows of
    // thousands of limbs that are shorter than the batch's length is a long
    // serial scan (up to 7 ms for 4096 rows of 60K limbs); the chunked
    // kernel reads such rows in coalesced 4096-limb chunks
    if (L <= 64u || N >= 65536u)
        length_max_rows_kernel<BITS><<<grid_for(N, 256, kNumSMs * 8), 256, 0, st>>>(A, N, L, stride, s->dev,
                                                                                  s->dev + 1, s->host_dev);
    else {
        const uint64_t items = (uint64_t)N * ((L + kChunk - 1u) / kChunk);
        length_max_chunks_kernel<BITS><<<grid_for(items, 1, kNumSMs * 8), 256, 0, st>>>(
            A, N, L, stride, items, s->dev, s->dev + 1, s->host_dev);
    }
    count_launch();
    cudaStreamSynchronize(st);
    note_d2h(sizeof(uint32_t));
    return *s->host;
}

// Creates the current stream's pair of words ahead of a stream capture (their
// creation synchronises the device, which a capture does not allow).
cudaError_t limb_length_prepare() { return length_state() ? cudaSuccess : cudaErrorMemoryAllocation; }

// The limb length of a batch written to device memory (d_out), without a
// host synchronisation: the same scans, the result stored where one later
// copy reads it.  Calls on one stream run in order and each stream has its
// own max / ticket words, so a pair is never used by two scans at once.
cudaError_t limb_length_to_device(const uint32_t *A, uint32_t N, uint32_t L, uint32_t stride, uint32_t *d_out) {
    LengthState *s = length_state();
    if (!s) return cudaErrorMemoryAllocation;
    cudaStream_t st = current_stream();
    if (N == 0u || L == 0u) return cudaMemsetAsync(d_out, 0, sizeof(uint32_t), st);
    if (L <= 64u || N >= 65536u)
        length_max_rows_kernel<false><<<grid_for(N, 256, kNumSMs * 8), 256, 0, st>>>(A, N, L, stride, s->dev,
                                                                                   s->dev + 1, d_out);
    else {
        const uint64_t items = (uint64_t)N * ((L + kChunk - 1u) / kChunk);
        length_max_chunks_kernel<false><<<grid_for(items, 1, kNumSMs * 8), 256, 0, st>>>(
            A, N, L, stride, items, s->dev, s->dev + 1, d_out);
    }
    count_launch();
    return cudaGetLastError();
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
