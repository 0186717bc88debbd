// Carry-chain family: add, sub, add_small, sub_small, mul_small, shift_add,
// shift_sub (gpupi batch_add.cu, batch_sub.cu, batch_add_small.cu,
// batch_sub_small.cu, batch_mul_small.cu, batch_shift_add.cu,
// batch_shift_sub.cu).
//
// Every one of these is "out_j = x_j +/- y_j +/- carry" over j < L_c with a
// carry of at most one bit, once the operands are written as two limb
// streams:
//   add/sub         x = A_j,                         y = B_j
//   add/sub_small   x = A_j,                         y = (j == 0) ? b : 0
//   mul_small       x = lo(A_j * b),                 y = hi(A_{j-1} * b)
//   shift_add/sub   x = (A << s)_j (two limbs of A), y = B_j
// so one engine serves them all.  Limbs past an operand's length read as 0,
// which gives the reference's "computed over max+1 limbs, truncated or
// zero-extended to L_c" semantics directly.
//
// Launch shapes (all sm_100a, no inter-CTA waiting):
//   * lanes per row    - short rows (L_c <= 32) in huge batches: 8, 16 or
//                        32 lanes per row, one ballot pair;
//   * warp per row     - 32-limb groups resolved with two ballots and one
//                        64-bit add (common.cuh), carry kept warp-uniform;
//   * tiles + fix-up   - long rows: each CTA owns a 4096-limb tile, writes its
//                        result assuming carry-in 0 plus (generate, propagate,
//                        ones-prefix) flags; a second kernel scans the flags
//                        of each row and patches only the all-ones prefix of
//                        tiles that receive a carry (usually one limb).
// Traffic is the algorithmic minimum (read operands once, write C once)
// except for the few fix-up limbs.
#include "common.cuh"
#include "carry_tile.cuh"

#include "batch_add.h"
#include "batch_add_small.h"
#include "batch_mul_small.h"
#include "batch_shift_add.h"
#include "batch_shift_sub.h"
#include "batch_sub.h"
#include "batch_sub_small.h"

namespace gpupi {

// ---------------------------------------------------------------------------
// Operand generators
// ---------------------------------------------------------------------------
struct GenTwo {
    const uint32_t *A;
    const uint32_t *B;
    uint32_t La, Lb;
    uint64_t sA, sB;
    __device__ __forceinline__ void operator()(uint32_t row, uint32_t j, uint32_t &x,
                                               uint32_t &y) const {
        x = (j < La) ? A[row * sA + j] : 0u;
        y = (j < Lb) ? B[row * sB + j] : 0u;
    }
    double read_limbs(uint32_t Lc) const { return (double)std::min(La, Lc) + std::min(Lb, Lc); }
};

struct GenSmall {
    const uint32_t *A;
    uint32_t b;
    uint32_t La;
    uint64_t sA;
    __device__ __forceinline__ void operator()(uint32_t row, uint32_t j, uint32_t &x,
                                               uint32_t &y) const {
        x = (j < La) ? A[row * sA + j] : 0u;
        y = (j == 0u) ? b : 0u;
    }
    double read_limbs(uint32_t Lc) const { return (double)std::min(La, Lc); }
};

struct GenMulSmall {
    const uint32_t *A;
    uint32_t b;
    uint32_t La;
    uint64_t sA;
    __device__ __forceinline__ void operator()(uint32_t row, uint32_t j, uint32_t &x,
                                               uint32_t &y) const {
        const uint32_t *r = A + row * sA;
        x = (j < La) ? r[j] * b : 0u;
        y = (j >= 1u && j - 1u < La) ? __umulhi(r[j - 1u], b) : 0u;
    }
    double read_limbs(uint32_t Lc) const { return (double)std::min(La, Lc); }
};

struct GenShiftTwo {
    const uint32_t *A;
    const uint32_t *B;
    uint32_t La, Lb;
    uint64_t sA, sB;
    uint32_t word, bit;
    __device__ __forceinline__ void operator()(uint32_t row, uint32_t j, uint32_t &x,
                                               uint32_t &y) const {
        const uint32_t *r = A + row * sA;
        uint32_t lo = 0u, prev = 0u;
        if (j >= word) {
            const uint32_t src = j - word;
            lo = (src < La) ? r[src] : 0u;
            prev = (bit != 0u && src >= 1u && src - 1u < La) ? r[src - 1u] : 0u;
        }
        x = (bit == 0u) ? lo : ((lo << bit) | (prev >> (32u - bit)));
        y = (j < Lb) ? B[row * sB + j] : 0u;
    }
    double read_limbs(uint32_t Lc) const { return (double)std::min(La, Lc) + std::min(Lb, Lc); }
};

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
// G lanes per row (G = 8, 16, 32; L_c <= G), 32 / G rows per warp: the
// short rows of the splitting tree's lower levels (millions of 6..32-limb
// rows) with whole groups of lanes reading and writing each row's limbs
// contiguously.
template <class Gen, bool SUB, int G>
__global__ void carry_seg_rows(Gen gen, uint32_t *C, uint64_t sC, uint32_t N, uint32_t Lc) {
    constexpr uint32_t kMask = (G == 32) ? 0xffffffffu : ((1u << G) - 1u);
    const uint32_t lane = lane_id();
    const uint32_t grp = lane / G, gl = lane % G;
    const uint32_t warps_per_cta = blockDim.x >> 5;
    const uint64_t gwarp = (uint64_t)blockIdx.x * warps_per_cta + (threadIdx.x >> 5);
    const uint64_t nwarps = (uint64_t)gridDim.x * warps_per_cta;
    // the whole warp runs every iteration (ballots); rows past N do nothing
    for (uint64_t base = gwarp * (32 / G); base < N; base += nwarps * (32 / G)) {
        const uint64_t row = base + grp;
        const bool valid = row < N && gl < Lc;
        uint32_t x = 0u, y = 0u;
        if (valid) gen((uint32_t)row, gl, x, y);
        bool g, p;
        const uint32_t s = raw_limb<SUB>(x, y, g, p);
        if (!valid) g = p = false;
        const uint32_t gm = (__ballot_sync(0xffffffffu, g) >> (grp * G)) & kMask;
        const uint32_t pm = (__ballot_sync(0xffffffffu, p) >> (grp * G)) & kMask;
        const GroupCarry gc = resolve_group_n(gm, pm, 0u, G);
        const uint32_t r = apply_carry<SUB>(s, (gc.carry_in_mask >> gl) & 1u);
        if (valid) C[row * sC + gl] = r;
    }
}

template <class Gen, bool SUB, int UNROLL>
__global__ void carry_warp_rows(Gen gen, uint32_t *C, uint64_t sC, uint32_t N, uint32_t Lc) {
    const uint32_t lane = lane_id();
    const uint32_t warps_per_cta = blockDim.x >> 5;
    const uint32_t gwarp = blockIdx.x * warps_per_cta + (threadIdx.x >> 5);
    const uint32_t nwarps = gridDim.x * warps_per_cta;
    for (uint32_t row = gwarp; row < N; row += nwarps) {
        uint32_t cin = 0u;
        uint32_t *out = C + row * sC;
        for (uint32_t base = 0; base < Lc; base += 32u * UNROLL) {
            uint32_t s[UNROLL], gm[UNROLL], pm[UNROLL];
#pragma unroll
            for (int u = 0; u < UNROLL; ++u) {
                const uint32_t j = base + u * 32u + lane;
                uint32_t x = 0u, y = 0u;
                if (j < Lc) gen(row, j, x, y);
                bool g, p;
                s[u] = raw_limb<SUB>(x, y, g, p);
                if (j >= Lc) g = p = false;
                gm[u] = __ballot_sync(0xffffffffu, g);
                pm[u] = __ballot_sync(0xffffffffu, p);
            }
#pragma unroll
            for (int u = 0; u < UNROLL; ++u) {
                const uint32_t j = base + u * 32u + lane;
                const GroupCarry gc = resolve_group(gm[u], pm[u], cin);
                cin = gc.carry_out;
                const uint32_t r = apply_carry<SUB>(s[u], (gc.carry_in_mask >> lane) & 1u);
                if (j < Lc) out[j] = r;
            }
        }
    }
}

constexpr int kTileWarps = 8;
constexpr int kTileGroups = 16;                          // 32-limb groups per warp
constexpr uint32_t kWarpSpan = 32u * kTileGroups;        // 512 limbs
constexpr uint32_t kTileSpan = kWarpSpan * kTileWarps;   // 4096 limbs

// Per-tile flags: bit 0 = generates a carry with carry-in 0, bit 1 = lets a
// carry through (result with carry-in 0 is all ones / all zeros for sub),
// bits 2.. = length of the all-ones (all-zeros) prefix of the tile result.
template <class Gen, bool SUB>
__global__ void __launch_bounds__(kTileWarps * 32)
carry_tiles(Gen gen, uint32_t *C, uint64_t sC, uint32_t Lc, uint32_t tiles_per_row,
            uint32_t *flags) {
    __shared__ uint32_t warp_g[kTileWarps], warp_p[kTileWarps], warp_prefix[kTileWarps];
    const uint32_t lane = lane_id();
    const uint32_t w = threadIdx.x >> 5;
    const uint32_t tile = blockIdx.x;
    const uint32_t row = tile / tiles_per_row;
    const uint32_t t = tile - row * tiles_per_row;
    const uint32_t wbase = t * kTileSpan + w * kWarpSpan;
    uint32_t *out = C + row * sC;

    uint32_t s[kTileGroups], gm[kTileGroups], pm[kTileGroups];
    const uint32_t ones = SUB ? 0u : 0xffffffffu;
#pragma unroll
    for (int u = 0; u < kTileGroups; ++u) {
        const uint32_t j = wbase + u * 32u + lane;
        uint32_t x = 0u, y = 0u;
        if (j < Lc) gen(row, j, x, y);
        bool g, p;
        s[u] = raw_limb<SUB>(x, y, g, p);
        if (j >= Lc) g = p = false;
        gm[u] = __ballot_sync(0xffffffffu, g);
        pm[u] = __ballot_sync(0xffffffffu, p);
    }
    // Pass 1: carry-in 0 for this warp's span.
    uint32_t c = 0u;
    bool all_p = true;
#pragma unroll
    for (int u = 0; u < kTileGroups; ++u) {
        c = resolve_group(gm[u], pm[u], c).carry_out;
        all_p = all_p && (pm[u] == 0xffffffffu);
    }
    if (lane == 0) {
        warp_g[w] = c;
        warp_p[w] = all_p ? 1u : 0u;
    }
    __syncthreads();
    // Carry into each warp of the tile (tile carry-in assumed 0).
    uint32_t gmask = 0u, pmask = 0u;
#pragma unroll
    for (int k = 0; k < kTileWarps; ++k) {
        gmask |= warp_g[k] << k;
        pmask |= warp_p[k] << k;
    }
    const GroupCarry tc = resolve_group_n(gmask, pmask, 0u, kTileWarps);
    uint32_t cin = (tc.carry_in_mask >> w) & 1u;
    // Pass 2: final values, stored, and this warp's ones-prefix.
    uint32_t prefix = kWarpSpan;
    bool prefix_open = true;
#pragma unroll
    for (int u = 0; u < kTileGroups; ++u) {
        const uint32_t j = wbase + u * 32u + lane;
        const GroupCarry gc = resolve_group(gm[u], pm[u], cin);
        cin = gc.carry_out;
        const uint32_t r = apply_carry<SUB>(s[u], (gc.carry_in_mask >> lane) & 1u);
        if (j < Lc) out[j] = r;
        const uint32_t not_ones = __ballot_sync(0xffffffffu, (r != ones) || (j >= Lc));
        if (prefix_open && not_ones != 0u) {
            prefix = u * 32u + (uint32_t)(__ffs(not_ones) - 1);
            prefix_open = false;
        }
    }
    if (lane == 0) warp_prefix[w] = prefix;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t pre = 0u;
        for (int k = 0; k < kTileWarps; ++k) {
            pre += warp_prefix[k];
            if (warp_prefix[k] != kWarpSpan) break;
        }
        // tile generate/propagate: warp 7's outgoing carry with tile cin 0
        const uint32_t G = tc.carry_out;
        const uint32_t P = (pmask == 0xffu) ? 1u : 0u;
        flags[tile] = G | (P << 1) | (pre << 2);
    }
}

// ---------------------------------------------------------------------------
// Dispatch
// ---------------------------------------------------------------------------
enum class CarryPlan { Lanes, Warp, Tiles };

static CarryPlan plan_for(uint32_t N, uint32_t Lc) {
    if (Lc <= 32u && N >= 2048u) return CarryPlan::Lanes;
    if (Lc <= kTileSpan || (uint64_t)N >= (uint64_t)kNumSMs * 64u) return CarryPlan::Warp;
    return CarryPlan::Tiles;
}

static size_t carry_workspace_bytes(uint32_t N, uint32_t Lc) {
    if (N == 0u || Lc == 0u || plan_for(N, Lc) != CarryPlan::Tiles) return 0;
    const uint64_t tiles = (Lc + kTileSpan - 1u) / kTileSpan;
    return (size_t)N * tiles * sizeof(uint32_t);
}

template <class Gen, bool SUB>
static void run_carry(const Gen &gen, uint32_t *C, uint32_t N, uint32_t Lc, uint32_t sC,
                      uint32_t *workspace) {
    if (N == 0u || Lc == 0u) return;
    cudaStream_t st = current_stream();
    const CarryPlan plan = plan_for(N, Lc);
    KernelTimed kt("carry_chain", 4.0 * N * (gen.read_limbs(Lc) + (double)Lc));
    if (plan == CarryPlan::Lanes) {
        // rows per 256-thread CTA: 8 warps x 32 / G
        if (Lc <= 8u)
            carry_seg_rows<Gen, SUB, 8><<<grid_for(N, 32, kNumSMs * 32), 256, 0, st>>>(gen, C, sC, N, Lc);
        else if (Lc <= 16u)
            carry_seg_rows<Gen, SUB, 16><<<grid_for(N, 16, kNumSMs * 32), 256, 0, st>>>(gen, C, sC, N, Lc);
        else
            carry_seg_rows<Gen, SUB, 32><<<grid_for(N, 8, kNumSMs * 32), 256, 0, st>>>(gen, C, sC, N, Lc);
        GPUPI_LAUNCH_CHECK();
    } else if (plan == CarryPlan::Warp) {
        const unsigned warps = 8;
        if (Lc <= 64u) {
            carry_warp_rows<Gen, SUB, 2><<<grid_for(N, warps), warps * 32, 0, st>>>(gen, C, sC, N, Lc);
        } else if (Lc <= 1024u) {
            carry_warp_rows<Gen, SUB, 4><<<grid_for(N, warps), warps * 32, 0, st>>>(gen, C, sC, N, Lc);
        } else {
            // long rows: more 32-limb groups in flight per warp
            carry_warp_rows<Gen, SUB, 8><<<grid_for(N, warps), warps * 32, 0, st>>>(gen, C, sC, N, Lc);
        }
        GPUPI_LAUNCH_CHECK();
    } else {
        const uint32_t tiles = (Lc + kTileSpan - 1u) / kTileSpan;
        const uint64_t total = (uint64_t)tiles * N;
        carry_tiles<Gen, SUB><<<(unsigned)total, kTileWarps * 32, 0, st>>>(gen, C, sC, Lc, tiles,
                                                                         workspace);
        GPUPI_LAUNCH_CHECK();
        launch_carry_fixup(SUB, C, sC, N, Lc, tiles, kTileSpan, workspace, st);
    }
}

}  // namespace gpupi

using namespace gpupi;

// ---------------------------------------------------------------------------
// Reference-compatible entry points
// ---------------------------------------------------------------------------
void batch_add_simple(uint32_t *A, uint32_t *B, uint32_t *C, uint32_t *workspace, uint32_t N,
                      uint32_t L_a, uint32_t L_b, uint32_t L_c, uint32_t stride_A,
                      uint32_t stride_B, uint32_t stride_C) {
    GenTwo g{A, B, L_a, L_b, stride_A, stride_B};
    run_carry<GenTwo, false>(g, C, N, L_c, stride_C, workspace);
}

size_t batch_add_simple_workspace_size(uint32_t N, uint32_t L_a, uint32_t L_b, uint32_t L_c) {
    (void)L_a;
    (void)L_b;
    return carry_workspace_bytes(N, L_c);
}

void batch_sub_simple(uint32_t *A, uint32_t *B, uint32_t *C, uint32_t *workspace, uint32_t N,
                      uint32_t L_a, uint32_t L_b, uint32_t L_c, uint32_t stride_A,
                      uint32_t stride_B, uint32_t stride_C) {
    GenTwo g{A, B, L_a, L_b, stride_A, stride_B};
    run_carry<GenTwo, true>(g, C, N, L_c, stride_C, workspace);
}

size_t batch_sub_simple_workspace_size(uint32_t N, uint32_t L_a, uint32_t L_b, uint32_t L_c) {
    (void)L_a;
    (void)L_b;
    return carry_workspace_bytes(N, L_c);
}

void batch_add_small(const uint32_t *A, uint32_t B, uint32_t *C, uint32_t *workspace, uint32_t N,
                     uint32_t L_a, uint32_t L_c, uint32_t stride_A, uint32_t stride_C) {
    GenSmall g{A, B, L_a, stride_A};
    run_carry<GenSmall, false>(g, C, N, L_c, stride_C, workspace);
}

size_t batch_add_small_workspace_size(uint32_t N, uint32_t L_a, uint32_t L_c) {
    (void)L_a;
    return carry_workspace_bytes(N, L_c);
}

void batch_sub_small(const uint32_t *A, uint32_t B, uint32_t *C, uint32_t *workspace, uint32_t N,
                     uint32_t L_a, uint32_t L_c, uint32_t stride_A, uint32_t stride_C) {
    GenSmall g{A, B, L_a, stride_A};
    run_carry<GenSmall, true>(g, C, N, L_c, stride_C, workspace);
}

size_t batch_sub_small_workspace_size(uint32_t N, uint32_t L_a, uint32_t L_c) {
    (void)L_a;
    return carry_workspace_bytes(N, L_c);
}

void batch_mul_small(const uint32_t *A, uint32_t B, uint32_t *C, uint32_t *workspace, uint32_t N,
                     uint32_t L_a, uint32_t L_c, uint32_t stride_A, uint32_t stride_C) {
    GenMulSmall g{A, B, L_a, stride_A};
    run_carry<GenMulSmall, false>(g, C, N, L_c, stride_C, workspace);
}

size_t batch_mul_small_workspace_size(uint32_t N, uint32_t L_a, uint32_t L_c) {
    (void)L_a;
    return carry_workspace_bytes(N, L_c);
}

void batch_shift_add_simple(const uint32_t *A, const uint32_t *B, uint32_t *C, uint32_t *workspace,
                            uint32_t shift, uint32_t N, uint32_t L_a, uint32_t L_b, uint32_t L_c,
                            uint32_t stride_A, uint32_t stride_B, uint32_t stride_C) {
    GenShiftTwo g{A, B, L_a, L_b, stride_A, stride_B, shift >> 5, shift & 31u};
    run_carry<GenShiftTwo, false>(g, C, N, L_c, stride_C, workspace);
}

size_t batch_shift_add_simple_workspace_size(uint32_t N, uint32_t L_a, uint32_t L_b, uint32_t L_c,
                                             uint32_t shift) {
    (void)L_a;
    (void)L_b;
    (void)shift;
    return carry_workspace_bytes(N, L_c);
}

void batch_shift_sub_simple(const uint32_t *A, const uint32_t *B, uint32_t *C, uint32_t *workspace,
                            uint32_t shift, uint32_t N, uint32_t L_a, uint32_t L_b, uint32_t L_c,
                            uint32_t stride_A, uint32_t stride_B, uint32_t stride_C) {
    GenShiftTwo g{A, B, L_a, L_b, stride_A, stride_B, shift >> 5, shift & 31u};
    run_carry<GenShiftTwo, true>(g, C, N, L_c, stride_C, workspace);
}

size_t batch_shift_sub_simple_workspace_size(uint32_t N, uint32_t L_a, uint32_t L_b, uint32_t L_c,
                                             uint32_t shift) {
    (void)L_a;
    (void)L_b;
    (void)shift;
    return carry_workspace_bytes(N, L_c);
}

// ---------------------------------------------------------------------------
// Allocation-free batched addition (gpupi_mp_add_noalloc in gpupi_c.h).
//
// Some callers cannot allocate device memory at the moment they need an add:
// code that runs with all device memory already handed to another allocator
// (a pre-sized pool it must not grow), and latency-critical loops that must
// not call cudaMalloc/cudaFree because those calls can synchronise the whole
// device.  For them the per-tile carry flags of long rows live in the fixed
// array below, compiled into the library, instead of a context workspace.
//
// Limit: kNoAllocMaxTiles flag words (256 KiB), i.e. N * ceil(L_c / 4096) tiles
// for rows on the multi-tile path; larger requests are rejected.
// The array is shared by every call and keeps the previous call's flags; no
// word has to start at zero because each tile's CTA writes its flag before
// the fix-up kernel reads it.  Calls whose kernels overlap on the GPU (two
// streams, two host threads) would race on the array.
// ---------------------------------------------------------------------------
#include "gpupi_c.h"

#include <mutex>

namespace gpupi {

constexpr uint64_t kNoAllocMaxTiles = 65536;
static __device__ __align__(256) uint32_t g_noalloc_flags[kNoAllocMaxTiles];

// Device address of g_noalloc_flags, looked up once per device (with that
// device current) on the first call that needs it.
static uint32_t *g_noalloc_addr[64];
static std::mutex g_noalloc_mu;

static cudaError_t noalloc_flags_address(uint32_t **out) {
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (g_noalloc_addr[dev] == nullptr) {
        void *p = nullptr;
        err = cudaGetSymbolAddress(&p, g_noalloc_flags);
        if (err != cudaSuccess) return err;
        g_noalloc_addr[dev] = static_cast<uint32_t *>(p);
    }
    *out = g_noalloc_addr[dev];
    return cudaSuccess;
}

static bool noalloc_view_ok(const uint32_t *d, uint32_t len, uint32_t n, uint32_t stride) {
    if (n == 0u) return len <= stride;
    if (d == nullptr) return false;
    return stride == 0u || len <= stride;
}

}  // namespace gpupi

extern "C" int gpupi_mp_add_noalloc(uint32_t N, const uint32_t *d_A, uint32_t L_a, uint32_t stride_A,
                                    const uint32_t *d_B, uint32_t L_b, uint32_t stride_B, uint32_t *d_C,
                                    uint32_t L_c, uint32_t stride_C) {
    using namespace gpupi;
    if (!noalloc_view_ok(d_A, L_a, N, stride_A) || !noalloc_view_ok(d_B, L_b, N, stride_B) ||
        !noalloc_view_ok(d_C, L_c, N, stride_C))
        return (int)cudaErrorInvalidValue;
    if (N == 0u || L_c == 0u) return 0;
    uint32_t *flags = nullptr;
    if (plan_for(N, L_c) == CarryPlan::Tiles) {
        const uint64_t tiles = (uint64_t)N * ((L_c + kTileSpan - 1u) / kTileSpan);
        if (tiles > kNoAllocMaxTiles) return (int)cudaErrorInvalidValue;   // beyond the fixed array
        const cudaError_t err = noalloc_flags_address(&flags);
        if (err != cudaSuccess) return (int)err;
    }
    GenTwo g{d_A, d_B, L_a, L_b, stride_A, stride_B};
    run_carry<GenTwo, false>(g, d_C, N, L_c, stride_C, flags);
    return (int)cudaGetLastError();
}
