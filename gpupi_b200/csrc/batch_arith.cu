// Batched-MP API: context, array views, validation and multiply dispatch
// (gpupi batch_arith.cu:1-424, header batch_arith.h:8-152).
//
// Same contract as the reference: views are validated (cudaErrorInvalidValue
// on malformed metadata), scratch comes from one grow-only context
// workspace, and every op is issued on the library's current stream.  The
// multiply picks schoolbook below a crossover and the three-prime NTT above it.
#include "common.cuh"
#include "batch_add.h"
#include "batch_add_small.h"
#include "batch_arith.h"
#include "batch_bitlength.h"
#include "batch_exactdiv_small.h"
#include "batch_mul_naive.h"
#include "batch_mul_ntt.h"
#include "batch_mul_small.h"
#include "batch_shift.h"
#include "batch_shift_add.h"
#include "batch_shift_sub.h"
#include "batch_sub.h"
#include "batch_sub_small.h"

#include <string.h>

#include <atomic>
#include <chrono>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

namespace gpupi {

static cudaStream_t g_stream = 0;
static std::atomic<uint64_t> g_launches{0};

cudaStream_t current_stream() { return g_stream; }
void set_current_stream(cudaStream_t s) { g_stream = s; }
uint64_t launch_counter() { return g_launches.load(); }
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void add_launches(int64_t n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }

static std::atomic<uint64_t> g_h2d{0}, g_d2h{0};
void note_h2d(uint64_t b) { g_h2d.fetch_add(b, std::memory_order_relaxed); }
void note_d2h(uint64_t b) { g_d2h.fetch_add(b, std::memory_order_relaxed); }
void transfer_bytes(uint64_t *h2d, uint64_t *d2h) {
    if (h2d) *h2d = g_h2d.load();
    if (d2h) *d2h = g_d2h.load();
}

namespace {
struct TimerRec {
    const char *name;
    cudaEvent_t a, b;
    double bytes;
    double host_a, host_b;   // host clock (ms) when a and b were recorded
};
double host_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
struct TimerState {
    std::mutex mu;
    bool on = false;
    std::vector<TimerRec> recs;
    std::vector<cudaEvent_t> pool;
    size_t used = 0;
};
TimerState &timer() {
    static TimerState t;
    return t;
}
cudaEvent_t pool_event(TimerState &t) {
    if (t.used == t.pool.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        t.pool.push_back(e);
    }
    return t.pool[t.used++];
}
}  // namespace

bool kernel_timer_enabled() { return timer().on; }
void kernel_timer_enable(bool on) { timer().on = on; }
void kernel_timer_reset() {
    TimerState &t = timer();
    std::lock_guard<std::mutex> g(t.mu);
    t.recs.clear();
    t.used = 0;
}
int kernel_timer_begin(const char *name) {
    TimerState &t = timer();
    if (!t.on) return -1;
    std::lock_guard<std::mutex> g(t.mu);
    TimerRec r{name, pool_event(t), pool_event(t), 0.0, host_ms(), 0.0};
    cudaEventRecord(r.a, g_stream);
    t.recs.push_back(r);
    return (int)t.recs.size() - 1;
}
void kernel_timer_end(int slot, double bytes) {
    if (slot < 0) return;
    TimerState &t = timer();
    std::lock_guard<std::mutex> g(t.mu);
    cudaEventRecord(t.recs[slot].b, g_stream);
    t.recs[slot].bytes = bytes;
    t.recs[slot].host_b = host_ms();
}
size_t kernel_timer_report(char *buf, size_t cap) {
    TimerState &t = timer();
    std::lock_guard<std::mutex> g(t.mu);
    cudaDeviceSynchronize();
    struct Agg {
        uint64_t n = 0;
        double ms = 0, bytes = 0;
    };
    std::map<std::string, Agg> agg;
    for (const TimerRec &r : t.recs) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.a, r.b);
        Agg &x = agg[r.name];
        x.n++;
        x.ms += ms;
        x.bytes += r.bytes;
    }
    // Time between consecutive timed launches, keyed by the two families:
    // untimed kernels, host synchronisations and launch starvation.  The
    // host figure is the host clock between recording the two events; a
    // device gap close to it means the device waited for the host.
    struct Gap {
        uint64_t n = 0;
        double ms = 0, host = 0;
    };
    std::map<std::string, Gap> gaps;
    for (size_t i = 1; i < t.recs.size(); ++i) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, t.recs[i - 1].b, t.recs[i].a) != cudaSuccess) continue;
        Gap &x = gaps[std::string(t.recs[i - 1].name) + ">" + t.recs[i].name];
        x.n++;
        x.ms += ms;
        x.host += t.recs[i].host_a - t.recs[i - 1].host_b;
    }
    std::string out;
    char line[256];
    for (auto &kv : agg) {
        snprintf(line, sizeof(line), "%s %llu %.6f %.0f\n", kv.first.c_str(), (unsigned long long)kv.second.n,
                 kv.second.ms, kv.second.bytes);
        out += line;
    }
    for (auto &kv : gaps) {
        snprintf(line, sizeof(line), "gap:%s %llu %.6f %.6f\n", kv.first.c_str(), (unsigned long long)kv.second.n,
                 kv.second.ms, kv.second.host);
        out += line;
    }
    if (buf && cap) {
        const size_t n = std::min(cap - 1, out.size());
        memcpy(buf, out.data(), n);
        buf[n] = 0;
    }
    return out.size();
}

void school_mul(const uint32_t *A, const uint32_t *B, uint32_t *C, uint32_t N, uint32_t La,
                uint32_t Lb, uint64_t sA, uint64_t sB, uint64_t sC);
bool school_thread_fits(uint32_t La, uint32_t Lb);
cudaError_t tc_mul(const uint32_t *A, const uint32_t *B, uint32_t *C, uint32_t N, uint32_t La, uint32_t Lb,
                   uint64_t sA, uint64_t sB, uint64_t sC);
enum MulKind { kSchool = 0, kTensor = 1, kNtt = 2 };
int mul_kind(uint32_t La, uint32_t Lb, bool public_api);   // tune.cu: school / tc / ntt per length bucket
void tune_load_default();

// Largest L_a + L_b handled by schoolbook.  The public batch_mp_mul keeps the
// reference's rule (schoolbook up to 1024, batch_arith.cu:181: such products
// never grow the context workspace, which gpupi's own tests check), with the
// tensor-core schoolbook where the tune table says it is faster.  The
// library's own algorithms (pi pipeline, decimal conversion, ragged batches)
// use mul_tuned: the tune table's kernel per length bucket (tune.cu), else
// the built-in rule: on B200 this library's NTT overtakes its CUDA-core
// schoolbook between 384 and 512 limbs (batched products of 2^27 limbs in
// total: 384 -> 3.8 ms school / 4.7 ms NTT, 512 -> 4.6 / 3.7 ms), so its
// switch is at 448.  The product is exact either way.  The built-in switch is
// overridable with gpupi_set_mul_crossover().
constexpr uint32_t kRefSchoolMax = 1024u;
static uint32_t g_school_max = 448u;

}  // namespace gpupi

struct BatchMPContext {
    NTTPrecomputedTables ntt_tables;
    uint32_t *workspace;
    size_t workspace_size_bytes;
};

namespace {

cudaError_t allocate_tables(BatchMPContext *ctx) {
    cudaError_t err = cudaMalloc(&ctx->ntt_tables.roots_table_lv1, 65536 * sizeof(uint3));
    if (err != cudaSuccess) return err;
    err = cudaMalloc(&ctx->ntt_tables.roots_table_lv2, 65536 * sizeof(uint3));
    if (err != cudaSuccess) return err;
    err = cudaMalloc(&ctx->ntt_tables.inv2n_table, 33 * sizeof(uint3));
    if (err != cudaSuccess) return err;
    init_ntt_precomputed_tables(&ctx->ntt_tables);
    err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    return cudaDeviceSynchronize();
}

cudaError_t ensure_workspace(BatchMPContext *ctx, size_t bytes) {
    if (bytes <= ctx->workspace_size_bytes) return cudaSuccess;
    uint32_t *p = nullptr;
    // the old buffer may still be in use by queued work
    cudaError_t err = cudaStreamSynchronize(gpupi::current_stream());
    if (err != cudaSuccess) return err;
    if (gpupi::fail_alloc_now(gpupi::kAllocWorkspace)) return cudaErrorMemoryAllocation;
    err = cudaMalloc(&p, bytes);
    if (err != cudaSuccess) return err;
    if (ctx->workspace) cudaFree(ctx->workspace);
    ctx->workspace = p;
    ctx->workspace_size_bytes = bytes;
    return cudaSuccess;
}

void release_context(BatchMPContext *ctx) {
    if (ctx->workspace) cudaFree(ctx->workspace);
    ctx->workspace = nullptr;
    ctx->workspace_size_bytes = 0;
    if (ctx->ntt_tables.roots_table_lv1) cudaFree(ctx->ntt_tables.roots_table_lv1);
    if (ctx->ntt_tables.roots_table_lv2) cudaFree(ctx->ntt_tables.roots_table_lv2);
    if (ctx->ntt_tables.inv2n_table) cudaFree(ctx->ntt_tables.inv2n_table);
    ctx->ntt_tables = NTTPrecomputedTables{};
}

// batch_arith.cu:89-104
bool valid_array(const BatchMPArray &a) {
    if (a.batch_size == 0u) return a.length <= a.stride;
    if (a.data == nullptr) return false;
    if (a.stride == 0u) return true;
    return a.length <= a.stride;
}

bool same_batch(const BatchMPArray &a, const BatchMPArray &b) { return a.batch_size == b.batch_size; }

}  // namespace

BatchMPArray batch_mp_array_create(uint32_t batch_size, uint32_t length, uint32_t stride) {
    BatchMPArray a{};
    a.length = length;
    a.batch_size = batch_size;
    a.stride = (stride == 0u) ? length : stride;
    if (a.length > a.stride) return BatchMPArray{};
    const size_t bytes = (size_t)a.batch_size * a.stride * sizeof(uint32_t);
    if (bytes == 0u) return a;
    if (gpupi::fail_alloc_now(gpupi::kAllocArray) || cudaMalloc(&a.data, bytes) != cudaSuccess) a = BatchMPArray{};
    return a;
}

void batch_mp_array_release(BatchMPArray array) {
    if (array.data) cudaFree(array.data);
}

BatchMPContext *batch_mp_init() {
    gpupi::tune_load_default();
    BatchMPContext *ctx = new (std::nothrow) BatchMPContext{};
    if (!ctx) return nullptr;
    if (allocate_tables(ctx) != cudaSuccess) {
        release_context(ctx);
        delete ctx;
        return nullptr;
    }
    gpupi::scratch_context_opened();
    return ctx;
}

namespace gpupi {
void pi_forget_context(const BatchMPContext *ctx);   // pi_engine.cu: graphs that use its tables
}

void batch_mp_destroy(BatchMPContext *ctx) {
    if (!ctx) return;
    gpupi::pi_forget_context(ctx);
    release_context(ctx);
    delete ctx;
    gpupi::scratch_context_closed();
}

size_t batch_mp_workspace_size(const BatchMPContext *ctx) { return ctx ? ctx->workspace_size_bytes : 0u; }

cudaError_t batch_mp_ensure_workspace(BatchMPContext *ctx, size_t required_bytes) {
    if (!ctx) return cudaErrorInvalidValue;
    return ensure_workspace(ctx, required_bytes);
}

namespace gpupi {
static cudaError_t mul_with(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, BatchMPArray C,
                            uint32_t school_max) {
    if (!ctx || !valid_array(A) || !valid_array(B) || !valid_array(C)) return cudaErrorInvalidValue;
    if (!same_batch(A, B) || !same_batch(A, C)) return cudaErrorInvalidValue;
    if ((uint64_t)C.length != (uint64_t)A.length + B.length) return cudaErrorInvalidValue;
    if (A.batch_size == 0u || C.length == 0u) return cudaSuccess;
    const int kind = gpupi::mul_kind(A.length, B.length, school_max == kRefSchoolMax);
    if (kind == gpupi::kSchool) {
        gpupi::school_mul(A.data, B.data, C.data, A.batch_size, A.length, B.length, A.stride, B.stride,
                          C.stride);
        return cudaGetLastError();
    }
    if (kind == gpupi::kTensor)
        return gpupi::tc_mul(A.data, B.data, C.data, A.batch_size, A.length, B.length, A.stride, B.stride,
                             C.stride);
    cudaError_t err = ensure_workspace(ctx, batch_mul_ntt_workspace_size(A.batch_size, A.length, B.length));
    if (err != cudaSuccess) return err;
    batch_mul_ntt(A.data, B.data, C.data, ctx->workspace, ctx->ntt_tables, A.batch_size, A.length,
                  B.length, A.stride, B.stride, C.stride);
    return cudaGetLastError();
}
cudaError_t mul_tuned(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, BatchMPArray C) {
    return mul_with(ctx, A, B, C, g_school_max);
}
}  // namespace gpupi

cudaError_t batch_mp_mul(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, BatchMPArray C) {
    return gpupi::mul_with(ctx, A, B, C, gpupi::kRefSchoolMax);
}

cudaError_t batch_mp_mul_small(BatchMPContext *ctx, BatchMPArray A, uint32_t B, BatchMPArray C) {
    if (!ctx || !valid_array(A) || !valid_array(C)) return cudaErrorInvalidValue;
    if (!same_batch(A, C)) return cudaErrorInvalidValue;
    cudaError_t err = ensure_workspace(ctx, batch_mul_small_workspace_size(A.batch_size, A.length, C.length));
    if (err != cudaSuccess) return err;
    batch_mul_small(A.data, B, C.data, ctx->workspace, A.batch_size, A.length, C.length, A.stride, C.stride);
    return cudaGetLastError();
}

cudaError_t batch_mp_exactdiv_small(BatchMPContext *ctx, BatchMPArray A, uint32_t B) {
    if (!ctx || !valid_array(A)) return cudaErrorInvalidValue;
    if (B == 0u || (B & 1u) == 0u || A.length > 128u) return cudaErrorInvalidValue;
    batch_exactdiv_small(A.data, B, A.batch_size, A.length, A.stride);
    return cudaGetLastError();
}

cudaError_t batch_mp_add(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, BatchMPArray C) {
    if (!ctx || !valid_array(A) || !valid_array(B) || !valid_array(C)) return cudaErrorInvalidValue;
    if (!same_batch(A, B) || !same_batch(A, C)) return cudaErrorInvalidValue;
    cudaError_t err = ensure_workspace(
        ctx, batch_add_simple_workspace_size(A.batch_size, A.length, B.length, C.length));
    if (err != cudaSuccess) return err;
    batch_add_simple(A.data, B.data, C.data, ctx->workspace, A.batch_size, A.length, B.length, C.length,
                     A.stride, B.stride, C.stride);
    return cudaGetLastError();
}

cudaError_t batch_mp_add_small(BatchMPContext *ctx, BatchMPArray A, uint32_t B, BatchMPArray C) {
    if (!ctx || !valid_array(A) || !valid_array(C)) return cudaErrorInvalidValue;
    if (!same_batch(A, C)) return cudaErrorInvalidValue;
    cudaError_t err = ensure_workspace(ctx, batch_add_small_workspace_size(A.batch_size, A.length, C.length));
    if (err != cudaSuccess) return err;
    batch_add_small(A.data, B, C.data, ctx->workspace, A.batch_size, A.length, C.length, A.stride, C.stride);
    return cudaGetLastError();
}

cudaError_t batch_mp_shift_add(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, uint32_t shift,
                               BatchMPArray C) {
    if (!ctx || !valid_array(A) || !valid_array(B) || !valid_array(C)) return cudaErrorInvalidValue;
    if (!same_batch(A, B) || !same_batch(A, C)) return cudaErrorInvalidValue;
    if (C.data == A.data || C.data == B.data) return cudaErrorInvalidValue;
    cudaError_t err = ensure_workspace(
        ctx, batch_shift_add_simple_workspace_size(A.batch_size, A.length, B.length, C.length, shift));
    if (err != cudaSuccess) return err;
    batch_shift_add_simple(A.data, B.data, C.data, ctx->workspace, shift, A.batch_size, A.length, B.length,
                           C.length, A.stride, B.stride, C.stride);
    return cudaGetLastError();
}

cudaError_t batch_mp_shift_sub(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, uint32_t shift,
                               BatchMPArray C) {
    if (!ctx || !valid_array(A) || !valid_array(B) || !valid_array(C)) return cudaErrorInvalidValue;
    if (!same_batch(A, B) || !same_batch(A, C)) return cudaErrorInvalidValue;
    if (C.data == A.data || C.data == B.data) return cudaErrorInvalidValue;
    cudaError_t err = ensure_workspace(
        ctx, batch_shift_sub_simple_workspace_size(A.batch_size, A.length, B.length, C.length, shift));
    if (err != cudaSuccess) return err;
    batch_shift_sub_simple(A.data, B.data, C.data, ctx->workspace, shift, A.batch_size, A.length, B.length,
                           C.length, A.stride, B.stride, C.stride);
    return cudaGetLastError();
}

cudaError_t batch_mp_sub(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, BatchMPArray C) {
    if (!ctx || !valid_array(A) || !valid_array(B) || !valid_array(C)) return cudaErrorInvalidValue;
    if (!same_batch(A, B) || !same_batch(A, C)) return cudaErrorInvalidValue;
    cudaError_t err = ensure_workspace(
        ctx, batch_sub_simple_workspace_size(A.batch_size, A.length, B.length, C.length));
    if (err != cudaSuccess) return err;
    batch_sub_simple(A.data, B.data, C.data, ctx->workspace, A.batch_size, A.length, B.length, C.length,
                     A.stride, B.stride, C.stride);
    return cudaGetLastError();
}

cudaError_t batch_mp_sub_small(BatchMPContext *ctx, BatchMPArray A, uint32_t B, BatchMPArray C) {
    if (!ctx || !valid_array(A) || !valid_array(C)) return cudaErrorInvalidValue;
    if (!same_batch(A, C)) return cudaErrorInvalidValue;
    cudaError_t err = ensure_workspace(ctx, batch_sub_small_workspace_size(A.batch_size, A.length, C.length));
    if (err != cudaSuccess) return err;
    batch_sub_small(A.data, B, C.data, ctx->workspace, A.batch_size, A.length, C.length, A.stride, C.stride);
    return cudaGetLastError();
}

cudaError_t batch_mp_shift_bits(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, int32_t shift_bits) {
    if (!ctx || !valid_array(A) || !valid_array(B)) return cudaErrorInvalidValue;
    if (!same_batch(A, B)) return cudaErrorInvalidValue;
    batch_shift_bits(A.data, B.data, A.batch_size, A.length, B.length, A.stride, B.stride, shift_bits);
    return cudaGetLastError();
}

cudaError_t batch_mp_bitlength_max(BatchMPContext *ctx, BatchMPArray A, uint32_t *result) {
    if (!ctx || !valid_array(A) || !result) return cudaErrorInvalidValue;
    cudaError_t err = ensure_workspace(ctx, batch_bitlength_workspace_size(A.batch_size, A.length));
    if (err != cudaSuccess) return err;
    *result = batch_bitlength_max(A.data, ctx->workspace, A.batch_size, A.length, A.stride);
    return cudaGetLastError();
}

cudaError_t batch_mp_limblength_max(BatchMPContext *ctx, BatchMPArray A, uint32_t *result) {
    if (!ctx || !valid_array(A) || !result) return cudaErrorInvalidValue;
    cudaError_t err = ensure_workspace(ctx, batch_bitlength_workspace_size(A.batch_size, A.length));
    if (err != cudaSuccess) return err;
    *result = batch_limblength_max(A.data, ctx->workspace, A.batch_size, A.length, A.stride);
    return cudaGetLastError();
}

cudaError_t BatchMPArray::compact(BatchMPContext *ctx) {
    uint32_t len = 0u;
    cudaError_t err = batch_mp_limblength_max(ctx, *this, &len);
    if (err != cudaSuccess) return err;
    length = len;
    return cudaSuccess;
}

namespace gpupi {
// NTT product regardless of the crossover (testing and tuning entry point).
cudaError_t mul_ntt_direct(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, BatchMPArray C) {
    if (!ctx || !valid_array(A) || !valid_array(B) || !valid_array(C)) return cudaErrorInvalidValue;
    if (!same_batch(A, B) || !same_batch(A, C)) return cudaErrorInvalidValue;
    if ((uint64_t)C.length != (uint64_t)A.length + B.length) return cudaErrorInvalidValue;
    cudaError_t err = ensure_workspace(ctx, batch_mul_ntt_workspace_size(A.batch_size, A.length, B.length));
    if (err != cudaSuccess) return err;
    batch_mul_ntt(A.data, B.data, C.data, ctx->workspace, ctx->ntt_tables, A.batch_size, A.length, B.length,
                  A.stride, B.stride, C.stride);
    return cudaGetLastError();
}
const NTTPrecomputedTables &context_tables(const BatchMPContext *ctx) { return ctx->ntt_tables; }
const void *context_workspace(const BatchMPContext *ctx) { return ctx ? ctx->workspace : nullptr; }
void set_school_max(uint32_t v) { g_school_max = v; }
uint32_t school_max() { return g_school_max; }
}  // namespace gpupi
