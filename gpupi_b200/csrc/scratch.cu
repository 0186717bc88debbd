// Device scratch memory for the library's temporaries (pi pipeline levels,
// decimal conversion buffers, power tables).
//
// One arena per (device, stream): a single device block carved best-fit with
// coalescing of freed neighbours, all bookkeeping on the host.  A free is
// immediate on the host; the range is handed out again only to work issued
// later on the same stream, which the stream runs after every earlier use
// of it, so no event or synchronisation is needed.
//
// A request that does not fit is served by cudaMallocAsync (and released
// with cudaFreeAsync).  When the arena's live bytes return to zero after
// such a spill, the block is replaced by one sized from the high-water mark
// of live bytes, so a repeated workload (the same pi computation again) runs
// entirely inside the arena after its first call; callers that know their
// footprint reserve it up front (scratch_reserve).
//
// Why not the stream-ordered pool for everything: on B200 (driver 580) a
// large cudaMallocAsync that maps new memory costs about 6.5 ms of host time
// per GB, and pool allocations of about 1 GB took 2 to 300 ms each even with
// the pool told to keep its memory, while the device sat idle.  cudaMalloc
// maps 21 GB in 3 to 6 ms, so the block comes from cudaMalloc (its free
// synchronises the device, which only a regrow or the last context's
// close does).
//
// Blocks are released when the last BatchMPContext is destroyed.
#include "common.cuh"
#include "range_map.h"

#include <map>
#include <mutex>
#include <unordered_map>
#include <utility>

namespace gpupi {
namespace {

constexpr size_t kAlign = 256;
constexpr size_t kGrain = 2u << 20;

size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct Arena {
    cudaStream_t stream = nullptr;
    char *base = nullptr;
    size_t cap = 0;
    RangeMap free;                                  // free ranges of the block
    std::unordered_map<void *, size_t> live;        // arena blocks: ptr -> size
    std::unordered_map<void *, size_t> spilled;     // cudaMallocAsync blocks: ptr -> size
    size_t live_bytes = 0, high = 0;
    size_t win_base = 0, win_peak = 0;   // live bytes at a window's start, peak above it
    uint64_t spills = 0;   // requests ever served outside the block
    bool grow = false;

    void note_peak() {
        high = std::max(high, live_bytes);
        if (live_bytes > win_base) win_peak = std::max(win_peak, live_bytes - win_base);
    }

    void reset_block(char *p, size_t bytes) {
        base = p;
        cap = p ? bytes : 0;
        free.reset(cap);
    }

    cudaError_t alloc(void **out, size_t bytes) {
        const size_t need = round_up(bytes ? bytes : 1, kAlign);
        size_t off = 0;
        if (base && free.take(need, &off)) {
            void *p = base + off;
            live.emplace(p, need);
            live_bytes += need;
            note_peak();
            *out = p;
            return cudaSuccess;
        }
        void *p = nullptr;
        const cudaError_t err = cudaMallocAsync(&p, need, stream);
        if (err != cudaSuccess) return err;
        spilled.emplace(p, need);
        ++spills;
        live_bytes += need;
        note_peak();
        grow = true;
        *out = p;
        return cudaSuccess;
    }

    // false when p is not one of this arena's blocks
    bool release(void *p) {
        auto a = live.find(p);
        if (a != live.end()) {
            free.give((size_t)((char *)p - base), a->second);
            live_bytes -= a->second;
            live.erase(a);
        } else {
            auto s = spilled.find(p);
            if (s == spilled.end()) return false;
            cudaFreeAsync(p, stream);
            live_bytes -= s->second;
            spilled.erase(s);
        }
        if (live_bytes == 0u && grow) regrow();
        return true;
    }

    // Everything is free: replace the block by one with room for the
    // high-water mark plus a quarter for fragmentation (and never smaller
    // than one and a half times the old block, so repeated spills converge).
    void regrow() {
        grow = false;
        replace_block(round_up(std::max(high + high / 4, cap + cap / 2), kGrain));
    }

    // Only while nothing is live.  cudaFree waits for queued work that may
    // still use the old block.
    void replace_block(size_t bytes) {
        if (base) cudaFree(base);
        reset_block(nullptr, 0);
        char *p = nullptr;
        if (cudaMalloc((void **)&p, bytes) != cudaSuccess) {
            cudaGetLastError();   // keep serving requests by spilling
            return;
        }
        reset_block(p, bytes);
    }

    // after a device synchronisation (the stream itself may be gone)
    void drop() {
        for (auto &kv : spilled) cudaFree(kv.first);
        spilled.clear();
        if (base) cudaFree(base);
        live.clear();
        reset_block(nullptr, 0);
        live_bytes = high = 0;
        grow = false;
    }
};

// A caller-owned device block carved like an arena but never spilling: the
// splitting tree's temporaries while the tree is captured into a CUDA graph
// (pi_engine.cu), so that every replay of the graph finds them at the same
// addresses.  Selected per host thread; its ranges are recognised by
// address when freed later.
struct Private {
    char *base = nullptr;
    size_t cap = 0;
    RangeMap free;
    std::unordered_map<void *, size_t> live;
    bool exhausted = false;   // a request did not fit
};

struct Registry {
    std::mutex mu;
    std::map<std::pair<int, cudaStream_t>, Arena> arenas;
    std::map<char *, Private> privates;   // by base
    int contexts = 0;
};

thread_local char *t_private = nullptr;   // base of this thread's active private block
Registry &registry() {
    static Registry r;
    return r;
}

}  // namespace

namespace {
std::mutex g_fail_mu;
uint32_t g_fail_mask = 0u, g_fail_left = 0u;
}  // namespace

void fail_alloc_arm(uint32_t mask, uint32_t nth) {
    std::lock_guard<std::mutex> g(g_fail_mu);
    g_fail_mask = nth ? mask : 0u;
    g_fail_left = nth;
}

bool fail_alloc_now(AllocKind kind) {
    std::lock_guard<std::mutex> g(g_fail_mu);
    if (!(g_fail_mask & kind) || g_fail_left == 0u) return false;
    if (--g_fail_left != 0u) return false;
    g_fail_mask = 0u;
    return true;
}

cudaError_t scratch_alloc(void **p, size_t bytes) {
    if (!p) return cudaErrorInvalidValue;
    if (fail_alloc_now(kAllocScratch)) return cudaErrorMemoryAllocation;
    if (t_private) {
        Registry &r = registry();
        std::lock_guard<std::mutex> g(r.mu);
        Private &pv = r.privates[t_private];
        const size_t need = round_up(bytes ? bytes : 1, kAlign);
        size_t off = 0;
        if (!pv.free.take(need, &off)) {
            pv.exhausted = true;
            return cudaErrorMemoryAllocation;
        }
        *p = pv.base + off;
        pv.live.emplace(*p, need);
        return cudaSuccess;
    }
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    Registry &r = registry();
    std::lock_guard<std::mutex> g(r.mu);
    const cudaStream_t st = current_stream();
    Arena &a = r.arenas[{dev, st}];
    a.stream = st;
    return a.alloc(p, bytes);
}

void scratch_free(void *p) {
    if (!p) return;
    Registry &r = registry();
    std::lock_guard<std::mutex> g(r.mu);
    if (!r.privates.empty()) {
        auto it = r.privates.upper_bound((char *)p);
        if (it != r.privates.begin()) {
            --it;
            Private &pv = it->second;
            if ((char *)p < pv.base + pv.cap) {
                auto a = pv.live.find(p);
                if (a != pv.live.end()) {
                    pv.free.give((size_t)((char *)p - pv.base), a->second);
                    pv.live.erase(a);
                }
                return;
            }
        }
    }
    for (auto &kv : r.arenas)
        if (kv.second.release(p)) return;
}

// Start carving the calling thread's scratch requests from [base, base + cap)
// (freshly: every range free); scratch_private_end() returns to the stream
// arenas and reports whether every request fitted.
void scratch_private_begin(void *base, size_t cap) {
    Registry &r = registry();
    std::lock_guard<std::mutex> g(r.mu);
    Private &pv = r.privates[(char *)base];
    pv.base = (char *)base;
    pv.cap = cap;
    pv.free.reset(cap);
    pv.live.clear();
    pv.exhausted = false;
    t_private = (char *)base;
}

bool scratch_private_end() {
    Registry &r = registry();
    std::lock_guard<std::mutex> g(r.mu);
    const bool ok = t_private ? !r.privates[t_private].exhausted : true;
    t_private = nullptr;
    return ok;
}

// Forget a private block (its memory is the caller's to free).
void scratch_private_drop(void *base) {
    Registry &r = registry();
    std::lock_guard<std::mutex> g(r.mu);
    r.privates.erase((char *)base);
}

// Peak of live scratch bytes on the current stream's arena above the level
// at scratch_window_begin().
void scratch_window_begin() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    Registry &r = registry();
    std::lock_guard<std::mutex> g(r.mu);
    Arena &a = r.arenas[{dev, current_stream()}];
    a.stream = current_stream();
    a.win_base = a.live_bytes;
    a.win_peak = 0;
}

size_t scratch_window_peak() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    Registry &r = registry();
    std::lock_guard<std::mutex> g(r.mu);
    return r.arenas[{dev, current_stream()}].win_peak;
}

void scratch_reserve(size_t bytes) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    Registry &r = registry();
    std::lock_guard<std::mutex> g(r.mu);
    const cudaStream_t st = current_stream();
    Arena &a = r.arenas[{dev, st}];
    a.stream = st;
    if (a.live_bytes != 0u || a.cap >= bytes) return;
    a.replace_block(round_up(bytes, kGrain));
}

void scratch_context_opened() {
    Registry &r = registry();
    std::lock_guard<std::mutex> g(r.mu);
    ++r.contexts;
}

void scratch_context_closed() {
    Registry &r = registry();
    std::lock_guard<std::mutex> g(r.mu);
    if (r.contexts > 0) --r.contexts;
    if (r.contexts != 0) return;
    int cur = 0;
    cudaGetDevice(&cur);
    for (auto &kv : r.arenas) {
        if (kv.first.first != cur) cudaSetDevice(kv.first.first);
        cudaDeviceSynchronize();
        kv.second.drop();
    }
    cudaSetDevice(cur);
    r.arenas.clear();
}

uint64_t scratch_live_bytes() {
    Registry &r = registry();
    std::lock_guard<std::mutex> g(r.mu);
    uint64_t live = 0;
    for (auto &kv : r.arenas) live += kv.second.live_bytes;
    return live;
}

void scratch_stats(uint64_t *block_bytes, uint64_t *high_water, uint64_t *spills) {
    Registry &r = registry();
    std::lock_guard<std::mutex> g(r.mu);
    uint64_t b = 0, h = 0, s = 0;
    for (auto &kv : r.arenas) {
        b += kv.second.cap;
        h = std::max<uint64_t>(h, kv.second.high);
        s += kv.second.spills;
    }
    if (block_bytes) *block_bytes = b;
    if (high_water) *high_water = h;
    if (spills) *spills = s;
}

}  // namespace gpupi
