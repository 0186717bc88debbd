// Shared device/host helpers for the gpupi_b200 limb kernels (sm_100a).
//
// Numbers are little-endian arrays of 32-bit limbs.  A batch of N numbers
// lives at data + row * stride (stride 0 broadcasts one row to every item),
// exactly as BatchMPArray describes it (gpupi batch_arith.h:10-22).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <algorithm>

namespace gpupi {

constexpr int kWarp = 32;
constexpr int kNumSMs = 148;  // B200: 2 dies x 74 SMs

// Grid size for grid-stride kernels: enough CTAs to fill every SM several
// times, never more than the work needs.
inline unsigned grid_for(uint64_t work_items, unsigned per_cta, unsigned max_ctas = kNumSMs * 16) {
    uint64_t ctas = (work_items + per_cta - 1) / per_cta;
    if (ctas == 0) ctas = 1;
    return (unsigned)std::min<uint64_t>(ctas, max_ctas);
}

// Host-side stream used by every launch.  The legacy default stream keeps the
// reference's implicit ordering for callers that never set one.
cudaStream_t current_stream();
void set_current_stream(cudaStream_t s);

// Counts kernel launches issued by this library (for launch-count claims).
uint64_t launch_counter();
void count_launch();
void add_launches(int64_t n);   // kernels a CUDA graph launch runs (or un-count a capture)

// Host<->device bytes moved by this library (pipeline inputs/results,
// compact() results, base-case round trips).
void note_h2d(uint64_t bytes);
void note_d2h(uint64_t bytes);
void transfer_bytes(uint64_t *h2d, uint64_t *d2h);

// Device scratch for the library's temporaries: a per-stream arena with no
// driver call in steady state (scratch.cu).  Freed ranges are reused only by
// work issued later on the same stream.
cudaError_t scratch_alloc(void **p, size_t bytes);
void scratch_free(void *p);
void scratch_reserve(size_t bytes);   // grow the idle arena of the current stream
void scratch_context_opened();
void scratch_context_closed();
void scratch_stats(uint64_t *block_bytes, uint64_t *high_water, uint64_t *spills);
uint64_t scratch_live_bytes();
// A caller-owned block standing in for the arena on this host thread (no
// spills: a request that does not fit fails); see scratch.cu.
void scratch_private_begin(void *base, size_t cap);
bool scratch_private_end();   // false: a request did not fit
void scratch_private_drop(void *base);
void scratch_window_begin();
size_t scratch_window_peak();

// Host-side allocation-failure injection (tests of the error paths; no GPU
// fault is involved): fail_alloc_arm(mask, n) makes the n-th following
// device allocation whose category is in mask return
// cudaErrorMemoryAllocation, once, without allocating.  Categories:
enum AllocKind : uint32_t {
    kAllocScratch = 1u,     // scratch arena requests (scratch_alloc)
    kAllocWorkspace = 2u,   // growth of a context's workspace
    kAllocArray = 4u,       // batch_mp_array_create
};
void fail_alloc_arm(uint32_t mask, uint32_t nth);
bool fail_alloc_now(AllocKind kind);   // true: this allocation must fail

// Optional per-kernel timing: when enabled, the launch sites bracket each
// launch with CUDA events on the current stream and record the launch's
// algorithmic HBM bytes.  Resolved (after a synchronisation) by
// kernel_timer_report().  Off by default: no events are recorded.
bool kernel_timer_enabled();
void kernel_timer_enable(bool on);
void kernel_timer_reset();
int kernel_timer_begin(const char *name);           // returns a slot or -1
void kernel_timer_end(int slot, double algo_bytes);
size_t kernel_timer_report(char *buf, size_t cap);  // "name launches ms bytes" lines

struct KernelTimed {
    int slot;
    double bytes;
    KernelTimed(const char *name, double algo_bytes) : slot(kernel_timer_begin(name)), bytes(algo_bytes) {}
    ~KernelTimed() { kernel_timer_end(slot, bytes); }
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// One product of a ragged batch: operand offsets and lengths (limbs) and the
// offset of its L_a + L_b output limbs.
struct RaggedRow {
    uint64_t offA, offB, offC;
    uint32_t La, Lb;
};

// ---------------------------------------------------------------------------
// Binary carry resolution across a warp.
//
// Each lane holds one limb position of a 32-limb group, ordered by lane.  For
// an addition the lane's raw sum s = x + y either generates a carry (g), lets
// an incoming carry through (p: s == 0xffffffff) or absorbs it.  Treating the
// lanes as the bits of a 32-bit word, carry propagation is itself a binary
// addition: with a = g|p and b = g, the carry INTO lane i is bit i of
// (a + b + cin) ^ a ^ b, and bit 32 of the sum is the carry out of the group.
// Subtraction is the same with borrows (g: x < y, p: x == y).
// ---------------------------------------------------------------------------
struct GroupCarry {
    uint32_t carry_in_mask;  // bit i = carry into lane i
    uint32_t carry_out;      // 0/1 carry out of lane 31
};

__device__ __forceinline__ GroupCarry resolve_group(uint32_t gmask, uint32_t pmask, uint32_t cin) {
    const uint64_t a = (uint64_t)(gmask | pmask);
    const uint64_t b = (uint64_t)gmask;
    const uint64_t sum = a + b + (uint64_t)cin;
    GroupCarry r;
    r.carry_in_mask = (uint32_t)(sum ^ a ^ b);
    r.carry_out = (uint32_t)(sum >> 32);
    return r;
}

// Raw limb op: returns s and sets g/p for the carry scan.
// Same resolution for a group of n <= 32 members held in bits [0, n).  The
// members are moved to the top bits and the free low bits are marked
// "propagate", so cin still enters at bit 0 and the carry out is bit 32.
// Returns the carry into member i in bit i.
__device__ __forceinline__ GroupCarry resolve_group_n(uint32_t gmask, uint32_t pmask, uint32_t cin,
                                                      int n) {
    const int pad = 32 - n;
    const uint32_t low = pad ? ((1u << pad) - 1u) : 0u;
    GroupCarry r = resolve_group(pad ? (gmask << pad) : gmask,
                                 pad ? ((pmask << pad) | low) : pmask, cin);
    r.carry_in_mask = pad ? (r.carry_in_mask >> pad) : r.carry_in_mask;
    return r;
}

template <bool SUB>
__device__ __forceinline__ uint32_t raw_limb(uint32_t x, uint32_t y, bool &g, bool &p) {
    if (SUB) {
        const uint32_t d = x - y;
        g = x < y;
        p = (d == 0u);
        return d;
    } else {
        const uint32_t s = x + y;
        g = s < x;
        p = (s == 0xffffffffu);
        return s;
    }
}

template <bool SUB>
__device__ __forceinline__ uint32_t apply_carry(uint32_t s, uint32_t c) {
    return SUB ? s - c : s + c;
}

}  // namespace gpupi

#define GPUPI_LAUNCH_CHECK() \
    do { ::gpupi::count_launch(); } while (0)
