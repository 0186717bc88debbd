// Block- and grid-level binary carry resolution shared by every kernel that
// ends in a carry pass (carry-chain ops, NTT CRT stage, schoolbook).
//
// Scheme for a row split into tiles of `span` limbs, one CTA per tile:
//   1. the CTA computes its tile assuming carry-in 0, resolving carries
//      between its threads with ballots (block_resolve), and publishes
//      flags = G | P << 1 | prefix << 2 where G = carry out, P = the tile
//      result is all ones (all zeros for subtraction) and prefix = number of
//      low limbs of the tile result that are all ones (all zeros);
//   2. carry_fixup (one warp per row) scans the flags of the row and adds the
//      incoming carry to tiles that receive one by rewriting their prefix and
//      bumping the next limb.
// No CTA ever waits for another, so there is no spin loop to bound.
#pragma once

#include "common.cuh"

namespace gpupi {

struct BlockCarry {
    uint32_t cin;   // carry into this thread's chunk (tile carry-in 0)
    uint32_t G;     // tile generates a carry
    uint32_t P;     // tile propagates a carry
};

// g/p: this thread's chunk generates / propagates.  Threads are ordered by
// threadIdx.x (low limbs first).  NWARPS <= 32.  Uses 2*NWARPS shared words.
template <int NWARPS>
__device__ __forceinline__ BlockCarry block_resolve(bool g, bool p, uint32_t *sh_g, uint32_t *sh_p) {
    const uint32_t lane = lane_id();
    const uint32_t w = threadIdx.x >> 5;
    const uint32_t gm = __ballot_sync(0xffffffffu, g);
    const uint32_t pm = __ballot_sync(0xffffffffu, p);
    const GroupCarry wc = resolve_group(gm, pm, 0u);
    if (lane == 0) {
        sh_g[w] = wc.carry_out;
        sh_p[w] = (pm == 0xffffffffu) ? 1u : 0u;
    }
    __syncthreads();
    uint32_t wg = 0u, wp = 0u;
#pragma unroll
    for (int k = 0; k < NWARPS; ++k) {
        wg |= sh_g[k] << k;
        wp |= sh_p[k] << k;
    }
    const GroupCarry bc = resolve_group_n(wg, wp, 0u, NWARPS);
    const uint32_t cin_w = (bc.carry_in_mask >> w) & 1u;
    const GroupCarry wc2 = resolve_group(gm, pm, cin_w);
    BlockCarry r;
    r.cin = (wc2.carry_in_mask >> lane) & 1u;
    r.G = bc.carry_out;
    r.P = (wp == ((NWARPS == 32) ? 0xffffffffu : ((1u << NWARPS) - 1u))) ? 1u : 0u;
    return r;
}

// Tile prefix: `local` = index (within this thread's V-limb chunk) of the first
// limb that is not all ones, or V if the whole chunk is all ones.  Returns, in
// every thread, the tile prefix length (NWARPS*32*V when the tile is all ones).
template <int NWARPS, int V>
__device__ __forceinline__ uint32_t block_prefix(uint32_t local, uint32_t *sh) {
    const uint32_t lane = lane_id();
    const uint32_t w = threadIdx.x >> 5;
    const uint32_t stop = __ballot_sync(0xffffffffu, local < (uint32_t)V);
    uint32_t wpre = 32u * V;
    if (stop != 0u) {
        const uint32_t first = (uint32_t)(__ffs(stop) - 1);
        wpre = first * V + __shfl_sync(0xffffffffu, local, first);
    }
    __syncthreads();
    if (lane == 0) sh[w] = wpre;
    __syncthreads();
    uint32_t pre = 0u;
    for (int k = 0; k < NWARPS; ++k) {
        pre += sh[k];
        if (sh[k] != 32u * V) break;
    }
    return pre;
}

// Cross-tile carry fix-up.  One warp per row; flags[row*tiles + t].
template <bool SUB>
__global__ void carry_fixup_kernel(uint32_t *C, uint64_t sC, uint32_t N, uint32_t Lc,
                                   uint32_t tiles_per_row, uint32_t span, const uint32_t *flags) {
    const uint32_t lane = lane_id();
    const uint32_t gwarp = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t row = gwarp; row < N; row += nwarps) {
        uint32_t cin = 0u;
        uint32_t *out = C + row * sC;
        for (uint32_t base = 0; base < tiles_per_row; base += 32u) {
            const uint32_t t = base + lane;
            uint32_t f = 0u;
            if (t < tiles_per_row) f = flags[(uint64_t)row * tiles_per_row + t];
            const uint32_t gm = __ballot_sync(0xffffffffu, (f & 1u) != 0u);
            const uint32_t pm = __ballot_sync(0xffffffffu, (f & 2u) != 0u);
            const GroupCarry gc = resolve_group(gm, pm, cin);
            cin = gc.carry_out;
            if (t < tiles_per_row && ((gc.carry_in_mask >> lane) & 1u)) {
                const uint64_t start = (uint64_t)t * span;
                const uint32_t pre = f >> 2;
                for (uint32_t k = 0; k < pre && start + k < Lc; ++k)
                    out[start + k] = SUB ? 0xffffffffu : 0u;
                if (pre < span && start + pre < Lc)
                    out[start + pre] = SUB ? out[start + pre] - 1u : out[start + pre] + 1u;
            }
        }
    }
}

// Cross-tile carry fix-up for long rows: one 1024-thread CTA per row walks
// the row's flags 1024 tiles at a time (block-wide ballot resolution, the
// next chunk's flags loaded while the current one resolves), so a row of T
// tiles costs T/1024 dependent steps instead of T/32.
template <bool SUB>
__global__ void __launch_bounds__(1024) carry_fixup_rows_kernel(uint32_t *C, uint64_t sC, uint32_t Lc,
                                                                uint32_t tiles_per_row, uint32_t span,
                                                                const uint32_t *flags) {
    __shared__ uint32_t sg[32], sp[32];
    const uint32_t row = blockIdx.x;
    const uint32_t *fr = flags + (uint64_t)row * tiles_per_row;
    uint32_t *out = C + row * sC;
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t wmask = (1u << w) - 1u;
    uint32_t cin = 0u;
    uint32_t fnext = (threadIdx.x < tiles_per_row) ? fr[threadIdx.x] : 0u;
    for (uint32_t base = 0; base < tiles_per_row; base += 1024u) {
        const uint32_t t = base + threadIdx.x;
        const uint32_t f = fnext;   // 0 beyond the row: neither generates nor propagates
        const uint32_t tn = t + 1024u;
        fnext = (tn < tiles_per_row) ? fr[tn] : 0u;
        const bool p = ((f >> 1) & 1u) != 0u;
        const BlockCarry bc = block_resolve<32>((f & 1u) != 0u, p, sg, sp);
        // carry into this tile when the chunk itself receives cin: every
        // earlier tile of the chunk must propagate
        const uint32_t pm = __ballot_sync(0xffffffffu, p);
        uint32_t wp = 0u;
#pragma unroll
        for (int k = 0; k < 32; ++k) wp |= sp[k] << k;
        const bool prev_all = ((pm & lt) == lt) && ((wp & wmask) == wmask);
        const uint32_t tin = bc.cin | (prev_all ? cin : 0u);
        if (t < tiles_per_row && tin) {
            const uint64_t start = (uint64_t)t * span;
            const uint32_t pre = f >> 2;
            for (uint32_t k = 0; k < pre && start + k < Lc; ++k) out[start + k] = SUB ? 0xffffffffu : 0u;
            if (pre < span && start + pre < Lc)
                out[start + pre] = SUB ? out[start + pre] - 1u : out[start + pre] + 1u;
        }
        cin = bc.G | (bc.P & cin);
        __syncthreads();   // sg / sp are rewritten by the next chunk
    }
}

inline void launch_carry_fixup(bool sub, uint32_t *C, uint64_t sC, uint32_t N, uint32_t Lc,
                               uint32_t tiles_per_row, uint32_t span, const uint32_t *flags,
                               cudaStream_t st) {
    if (tiles_per_row > 64u) {
        if (sub)
            carry_fixup_rows_kernel<true><<<N, 1024, 0, st>>>(C, sC, Lc, tiles_per_row, span, flags);
        else
            carry_fixup_rows_kernel<false><<<N, 1024, 0, st>>>(C, sC, Lc, tiles_per_row, span, flags);
    } else {
        const unsigned grid = grid_for(N, 4, kNumSMs * 8);
        if (sub)
            carry_fixup_kernel<true><<<grid, 128, 0, st>>>(C, sC, N, Lc, tiles_per_row, span, flags);
        else
            carry_fixup_kernel<false><<<grid, 128, 0, st>>>(C, sC, N, Lc, tiles_per_row, span, flags);
    }
    count_launch();
}

// Chunk arithmetic for kernels whose per-position values are up to 96 bits
// (convolution coefficients, schoolbook column sums).
//   S = sum_v c[v] * 2^(32v)   (V+3 limbs)
template <int V>
__device__ __forceinline__ void chunk_sum3(const uint32_t (&c)[V][3], uint32_t (&S)[V + 3]) {
    uint64_t carry = 0;
#pragma unroll
    for (int k = 0; k < V + 3; ++k) {
        uint64_t s = carry;
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int d = k - v;
            if (d >= 0 && d <= 2) s += c[v][d];
        }
        S[k] = (uint32_t)s;
        carry = s >> 32;
    }
}

// X = S[0..V) + H (3 limbs spilled from the previous chunk); returns carry out.
template <int V>
__device__ __forceinline__ uint32_t chunk_add_spill(const uint32_t (&S)[V + 3], const uint32_t (&H)[3],
                                                    uint32_t (&X)[V]) {
    uint64_t t = 0;
#pragma unroll
    for (int k = 0; k < V; ++k) {
        t += (uint64_t)S[k] + (k < 3 ? H[k] : 0u);
        X[k] = (uint32_t)t;
        t >>= 32;
    }
    static_assert(V >= 3, "the 3-limb spill must fit in one chunk");
    return (uint32_t)t;
}

template <int V>
__device__ __forceinline__ void chunk_increment(uint32_t (&X)[V], uint32_t cin) {
    uint32_t c = cin;
#pragma unroll
    for (int k = 0; k < V; ++k) {
        const uint32_t s = X[k] + c;
        c = (s < X[k]) ? 1u : 0u;
        X[k] = s;
    }
}

template <int V>
__device__ __forceinline__ uint32_t chunk_first_not_ones(const uint32_t (&X)[V]) {
    uint32_t first = V;
#pragma unroll
    for (int k = V - 1; k >= 0; --k)
        if (X[k] != 0xffffffffu) first = k;
    return first;
}

}  // namespace gpupi
