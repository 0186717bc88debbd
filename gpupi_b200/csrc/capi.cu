// extern "C" boundary of libgpupi_b200.so (declared in include/gpupi_c.h).
// Thin adapters from plain pointers/sizes to the BatchMPArray API.
#include "common.cuh"
#include "batch_arith.h"
#include "batch_decimal_naive.h"
#include "batch_mul_naive.h"
#include "batch_mul_ntt.h"
#include "convert_decimal.h"
#include "gpupi_c.h"
#include "pi_engine.h"
#include "spectrum.h"

#include <string.h>

#include <algorithm>
#include <string>

struct gpupi_ctx {
    BatchMPContext *ctx;
};

namespace gpupi {
cudaError_t bbp_fractions(const uint64_t *positions, uint32_t count, uint64_t *fractions);
cudaError_t tc_mul(const uint32_t *A, const uint32_t *B, uint32_t *C, uint32_t N, uint32_t La, uint32_t Lb,
                   uint64_t sA, uint64_t sB, uint64_t sC);
bool tc_fits(uint32_t La, uint32_t Lb);
uint32_t tc_error();
cudaError_t tc_selftest_timeout(uint32_t *seen, uint32_t *after);
int mul_kind(uint32_t La, uint32_t Lb, bool public_api);
cudaError_t int_peak(double *imad_winst_per_s, double *alu_winst_per_s);
void ntt_shape_of(uint32_t La, uint32_t Lb, int *log_k, int *M);
int tune_load(const char *path);
int tune_load_text(const char *text);
void tune_reset();
std::string tune_describe();
cudaError_t autotune(BatchMPContext *ctx, const char *path, uint64_t budget_limbs, std::string *report);
cudaError_t mul_ragged(BatchMPContext *ctx, uint32_t N, const uint32_t *A, const uint64_t *offA, const uint32_t *La,
                       const uint32_t *B, const uint64_t *offB, const uint32_t *Lb, uint32_t *C,
                       const uint64_t *offC);
}

namespace {
inline BatchMPArray view(const uint32_t *d, uint32_t len, uint32_t n, uint32_t stride) {
    return BatchMPArray{const_cast<uint32_t *>(d), len, n, stride};
}
inline BatchMPContext *raw(gpupi_ctx *c) { return c ? c->ctx : nullptr; }
}  // namespace

extern "C" {

const char *gpupi_version(void) { return "gpupi_b200 0.1 (sm_100a, three-prime NTT)"; }

uint64_t gpupi_launch_count(void) { return gpupi::launch_counter(); }

int gpupi_set_stream(void *s) {
    gpupi::set_current_stream((cudaStream_t)s);
    return 0;
}

int gpupi_device_sync(void) { return (int)cudaDeviceSynchronize(); }

gpupi_ctx *gpupi_ctx_create(void) {
    BatchMPContext *c = batch_mp_init();
    if (!c) return nullptr;
    gpupi_ctx *h = new gpupi_ctx{c};
    return h;
}

void gpupi_ctx_destroy(gpupi_ctx *ctx) {
    if (!ctx) return;
    batch_mp_destroy(ctx->ctx);
    delete ctx;
}

size_t gpupi_ctx_workspace_size(const gpupi_ctx *ctx) { return ctx ? batch_mp_workspace_size(ctx->ctx) : 0; }

int gpupi_ctx_ensure_workspace(gpupi_ctx *ctx, size_t bytes) {
    return (int)batch_mp_ensure_workspace(raw(ctx), bytes);
}

int gpupi_mp_mul(gpupi_ctx *ctx, uint32_t N, const uint32_t *A, uint32_t La, uint32_t sA, const uint32_t *B,
                 uint32_t Lb, uint32_t sB, uint32_t *C, uint32_t Lc, uint32_t sC) {
    return (int)batch_mp_mul(raw(ctx), view(A, La, N, sA), view(B, Lb, N, sB), view(C, Lc, N, sC));
}

int gpupi_mp_mul_spectra(gpupi_ctx *ctx, uint32_t N, const uint32_t *A, uint32_t La, const uint32_t *B,
                         uint32_t Lb, const uint32_t *D, uint32_t Ld, const uint32_t *E, uint32_t Le, uint32_t *C,
                         uint32_t Lc) {
    BatchMPContext *c = raw(ctx);
    if (!c || !A || !B || !C || N == 0u || La == 0u || Lb == 0u) return (int)cudaErrorInvalidValue;
    const bool two = D != nullptr;
    if (two && (!E || Ld == 0u || Le == 0u)) return (int)cudaErrorInvalidValue;
    const uint64_t need = std::max<uint64_t>((uint64_t)La + Lb, two ? (uint64_t)Ld + Le + 1u : 0u);
    if (Lc < need) return (int)cudaErrorInvalidValue;
    const gpupi::SpectrumShape S = gpupi::spectrum_shape(Lc - 1u);
    const uint32_t las[2] = {La, Ld}, lbs[2] = {Lb, Le};
    if (S.M == 0 || !gpupi::spectrum_sum_fits(las, lbs, two ? 2 : 1)) return (int)cudaErrorInvalidValue;
    const uint64_t words = gpupi::spectrum_words(S, N);
    uint32_t *F[4] = {nullptr, nullptr, nullptr, nullptr}, *flags = nullptr;
    cudaError_t err = cudaSuccess;
    for (int i = 0; i < (two ? 4 : 2) && err == cudaSuccess; ++i) err = gpupi::scratch_alloc((void **)&F[i], words * 4);
    if (err == cudaSuccess) err = gpupi::scratch_alloc((void **)&flags, gpupi::spectrum_flag_words(N, Lc) * 4);
    if (err == cudaSuccess) {
        const NTTPrecomputedTables &t = gpupi::context_tables(c);
        gpupi::spectrum_forward(t, S, N, A, La, La, F[0], B, Lb, Lb, F[1]);
        if (two) gpupi::spectrum_forward(t, S, N, D, Ld, Ld, F[2], E, Le, Le, F[3]);
        const uint32_t *X[2] = {F[0], F[2]}, *Y[2] = {F[1], F[3]};
        gpupi::spectrum_inverse(t, S, N, two ? 2 : 1, X, Y, F[0], C, Lc, Lc, flags);
        err = cudaGetLastError();
    }
    for (int i = 0; i < 4; ++i) gpupi::scratch_free(F[i]);
    gpupi::scratch_free(flags);
    return (int)err;
}

int gpupi_mp_add(gpupi_ctx *ctx, uint32_t N, const uint32_t *A, uint32_t La, uint32_t sA, const uint32_t *B,
                 uint32_t Lb, uint32_t sB, uint32_t *C, uint32_t Lc, uint32_t sC) {
    return (int)batch_mp_add(raw(ctx), view(A, La, N, sA), view(B, Lb, N, sB), view(C, Lc, N, sC));
}

int gpupi_mp_sub(gpupi_ctx *ctx, uint32_t N, const uint32_t *A, uint32_t La, uint32_t sA, const uint32_t *B,
                 uint32_t Lb, uint32_t sB, uint32_t *C, uint32_t Lc, uint32_t sC) {
    return (int)batch_mp_sub(raw(ctx), view(A, La, N, sA), view(B, Lb, N, sB), view(C, Lc, N, sC));
}

int gpupi_mp_shift_add(gpupi_ctx *ctx, uint32_t N, const uint32_t *A, uint32_t La, uint32_t sA,
                       const uint32_t *B, uint32_t Lb, uint32_t sB, uint32_t shift, uint32_t *C, uint32_t Lc,
                       uint32_t sC) {
    return (int)batch_mp_shift_add(raw(ctx), view(A, La, N, sA), view(B, Lb, N, sB), shift, view(C, Lc, N, sC));
}

int gpupi_mp_shift_sub(gpupi_ctx *ctx, uint32_t N, const uint32_t *A, uint32_t La, uint32_t sA,
                       const uint32_t *B, uint32_t Lb, uint32_t sB, uint32_t shift, uint32_t *C, uint32_t Lc,
                       uint32_t sC) {
    return (int)batch_mp_shift_sub(raw(ctx), view(A, La, N, sA), view(B, Lb, N, sB), shift, view(C, Lc, N, sC));
}

int gpupi_mp_add_small(gpupi_ctx *ctx, uint32_t N, const uint32_t *A, uint32_t La, uint32_t sA, uint32_t b,
                       uint32_t *C, uint32_t Lc, uint32_t sC) {
    return (int)batch_mp_add_small(raw(ctx), view(A, La, N, sA), b, view(C, Lc, N, sC));
}

int gpupi_mp_sub_small(gpupi_ctx *ctx, uint32_t N, const uint32_t *A, uint32_t La, uint32_t sA, uint32_t b,
                       uint32_t *C, uint32_t Lc, uint32_t sC) {
    return (int)batch_mp_sub_small(raw(ctx), view(A, La, N, sA), b, view(C, Lc, N, sC));
}

int gpupi_mp_mul_small(gpupi_ctx *ctx, uint32_t N, const uint32_t *A, uint32_t La, uint32_t sA, uint32_t b,
                       uint32_t *C, uint32_t Lc, uint32_t sC) {
    return (int)batch_mp_mul_small(raw(ctx), view(A, La, N, sA), b, view(C, Lc, N, sC));
}

int gpupi_mp_exactdiv_small(gpupi_ctx *ctx, uint32_t N, uint32_t *A, uint32_t La, uint32_t sA, uint32_t b) {
    return (int)batch_mp_exactdiv_small(raw(ctx), view(A, La, N, sA), b);
}

int gpupi_mp_shift_bits(gpupi_ctx *ctx, uint32_t N, const uint32_t *A, uint32_t La, uint32_t sA, uint32_t *B,
                        uint32_t Lb, uint32_t sB, int32_t shift_bits) {
    return (int)batch_mp_shift_bits(raw(ctx), view(A, La, N, sA), view(B, Lb, N, sB), shift_bits);
}

int gpupi_mp_bitlength_max(gpupi_ctx *ctx, uint32_t N, const uint32_t *A, uint32_t La, uint32_t sA,
                           uint32_t *h_result) {
    return (int)batch_mp_bitlength_max(raw(ctx), view(A, La, N, sA), h_result);
}

int gpupi_mp_limblength_max(gpupi_ctx *ctx, uint32_t N, const uint32_t *A, uint32_t La, uint32_t sA,
                            uint32_t *h_result) {
    return (int)batch_mp_limblength_max(raw(ctx), view(A, La, N, sA), h_result);
}

int gpupi_mul_naive(uint32_t N, const uint32_t *A, uint32_t La, uint32_t sA, const uint32_t *B, uint32_t Lb,
                    uint32_t sB, uint32_t *C, uint32_t sC) {
    if ((uint64_t)La + Lb > (uint64_t)BATCH_MUL_NAIVE_L_MAX) return (int)cudaErrorInvalidValue;
    batch_mul_naive(const_cast<uint32_t *>(A), const_cast<uint32_t *>(B), C, (int)N, (int)La, (int)Lb, (int)sA,
                    (int)sB, (int)sC);
    return (int)cudaGetLastError();
}

int gpupi_mul_tc(uint32_t N, const uint32_t *A, uint32_t La, uint32_t sA, const uint32_t *B, uint32_t Lb,
                 uint32_t sB, uint32_t *C, uint32_t sC) {
    if (!gpupi::tc_fits(La, Lb) || (sA && sA < La) || (sB && sB < Lb) || (N > 1u && sC < La + Lb))
        return (int)cudaErrorInvalidValue;
    return (int)gpupi::tc_mul(A, B, C, N, La, Lb, sA, sB, sC);
}

int gpupi_tc_error(void) { return (int)gpupi::tc_error(); }

int gpupi_tc_selftest_timeout(uint32_t *seen, uint32_t *after) {
    if (!seen || !after) return (int)cudaErrorInvalidValue;
    return (int)gpupi::tc_selftest_timeout(seen, after);
}

int gpupi_tree_graph_stats(uint64_t *out5) {
    if (!out5) return (int)cudaErrorInvalidValue;
    const gpupi::TreeGraphStats t = gpupi::tree_graph_stats();
    out5[0] = t.recorded;
    out5[1] = t.captured;
    out5[2] = t.replayed;
    out5[3] = t.fallbacks;
    out5[4] = t.disabled;
    return 0;
}

int gpupi_tree_graph_perturb(void) {
    gpupi::tree_graph_perturb();
    return 0;
}

int gpupi_fail_alloc(uint32_t kind_mask, uint32_t nth) {
    gpupi::fail_alloc_arm(kind_mask, nth);
    return 0;
}

uint64_t gpupi_scratch_live_bytes(void) { return gpupi::scratch_live_bytes(); }

int gpupi_int_peak(double *imad_winst_per_s, double *alu_winst_per_s) {
    return (int)gpupi::int_peak(imad_winst_per_s, alu_winst_per_s);
}

int gpupi_tune_load(const char *path) { return gpupi::tune_load(path); }
int gpupi_tune_load_text(const char *text) { return gpupi::tune_load_text(text); }
int gpupi_tune_reset(void) {
    gpupi::tune_reset();
    return 0;
}
size_t gpupi_tune_describe(char *buf, size_t cap) {
    const std::string s = gpupi::tune_describe();
    if (buf && cap) {
        const size_t n = std::min(cap - 1, s.size());
        memcpy(buf, s.data(), n);
        buf[n] = 0;
    }
    return s.size();
}
int gpupi_mul_kind(uint32_t La, uint32_t Lb, int public_api) { return gpupi::mul_kind(La, Lb, public_api != 0); }
int gpupi_ntt_shape(uint32_t La, uint32_t Lb, int *log_k, int *M) {
    if (!log_k || !M || La == 0u || Lb == 0u) return (int)cudaErrorInvalidValue;
    gpupi::ntt_shape_of(La, Lb, log_k, M);
    return 0;
}
int gpupi_autotune(gpupi_ctx *ctx, const char *path, uint64_t budget_limbs) {
    return (int)gpupi::autotune(raw(ctx), path, budget_limbs, nullptr);
}

int gpupi_mp_mul_ragged(gpupi_ctx *ctx, uint32_t N, const uint32_t *A, const uint64_t *offA, const uint32_t *La,
                        const uint32_t *B, const uint64_t *offB, const uint32_t *Lb, uint32_t *C,
                        const uint64_t *offC) {
    return (int)gpupi::mul_ragged(raw(ctx), N, A, offA, La, B, offB, Lb, C, offC);
}

int gpupi_mul_ntt(gpupi_ctx *ctx, uint32_t N, const uint32_t *A, uint32_t La, uint32_t sA, const uint32_t *B,
                  uint32_t Lb, uint32_t sB, uint32_t *C, uint32_t sC) {
    return (int)gpupi::mul_ntt_direct(raw(ctx), view(A, La, N, sA), view(B, Lb, N, sB),
                                      view(C, La + Lb, N, sC));
}

int gpupi_decimal_naive(uint32_t N, const uint32_t *A, uint32_t L_limb, uint32_t sA, char *out, uint32_t L_dec,
                        uint32_t sO) {
    if (L_limb > (uint32_t)BATCH_DECIMAL_NAIVE_L_LIMB_MAX) return (int)cudaErrorInvalidValue;
    batch_decimal_naive(A, out, N, (int)L_limb, sA, (int)L_dec, sO);
    return (int)cudaGetLastError();
}

int gpupi_convert_decimal(gpupi_ctx *ctx, const uint32_t *X, uint32_t Lx, uint32_t input_bits,
                          uint32_t total_digits, uint32_t leaf_digits, char *out) {
    BatchMPContext *c = raw(ctx);
    if (!c || leaf_digits == 0u || total_digits % leaf_digits) return (int)cudaErrorInvalidValue;
    uint32_t ratio = total_digits / leaf_digits, levels = 0u;
    while (ratio > 1u && (ratio & 1u) == 0u) {
        ratio >>= 1;
        ++levels;
    }
    if (ratio != 1u) return (int)cudaErrorInvalidValue;
    ConvertDecimalPowerTable t{};
    cudaError_t err = convert_decimal_precompute_powers(c, &t, leaf_digits, levels);
    if (err == cudaSuccess)
        err = convert_decimal_equal_split(c, view(X, Lx, 1, Lx), input_bits, total_digits, leaf_digits, &t, out);
    convert_decimal_release_powers(&t);
    return (int)err;
}

namespace {
struct StreamSink {
    gpupi_digit_sink fn;
    void *user;
};
}  // namespace

int gpupi_pi_stream(gpupi_ctx *ctx, uint32_t digits, uint32_t flags, gpupi_digit_sink sink, void *user,
                    size_t chunk, uint32_t *info) {
    if (!sink) return (int)cudaErrorInvalidValue;
    StreamSink k{sink, user};
    gpupi::PiRequest req;
    req.digits = digits;
    req.ctx = raw(ctx);
    req.plain = (flags & 4u) != 0u;
    req.sink = [](const char *data, size_t n, void *u) {
        StreamSink *s = static_cast<StreamSink *>(u);
        return s->fn(data, n, s->user) == 0;
    };
    req.sink_user = &k;
    if (chunk) req.sink_chunk = chunk;
    gpupi::PiOutput out;
    const cudaError_t err = gpupi::pi_run(req, out);
    if (err != cudaSuccess) return (int)err;
    if (info) {
        uint32_t leaf = 0u;
        gpupi::round_up_decimal_digits(digits, &leaf);
        info[0] = out.convert_digits;
        info[1] = out.ret_len;
        memcpy(&info[2], &out.elapsed_ms, 4);
        info[3] = (uint32_t)(out.workspace_bytes >> 20);
        info[4] = 0u;
        info[5] = leaf;
        memcpy(&info[6], &out.output_ms, 4);
        info[7] = 0u;
    }
    return 0;
}

int gpupi_pi_compute_checkpointed(gpupi_ctx *ctx, uint32_t digits, uint32_t flags, const char *checkpoint,
                                  uint32_t *h_ret, size_t ret_cap, char *h_digits, size_t digits_cap,
                                  uint32_t *info) {
    if (!checkpoint) return (int)cudaErrorInvalidValue;
    gpupi::PiRequest req;
    req.digits = digits;
    req.profile_stages = (flags & 1u) != 0u;
    req.copy_digits = h_digits ? (uint32_t)std::min<size_t>(digits_cap, digits) : 0u;
    req.ctx = raw(ctx);
    req.device_only = (flags & 2u) != 0u;
    req.plain = (flags & 4u) != 0u;
    req.host_digits = h_digits;
    req.host_ret = h_ret;
    req.host_ret_cap = h_ret ? ret_cap : 0;
    req.checkpoint = checkpoint;
    gpupi::PiOutput out;
    cudaError_t err = gpupi::pi_run(req, out);
    if (err != cudaSuccess) return (int)err;
    if (info) {
        uint32_t leaf = 0u;
        gpupi::round_up_decimal_digits(digits, &leaf);
        info[0] = out.convert_digits;
        info[1] = out.ret_len;
        memcpy(&info[2], &out.elapsed_ms, 4);
        info[3] = (uint32_t)(out.workspace_bytes >> 20);
        info[4] = (uint32_t)out.stages.size();
        info[5] = leaf;
        info[6] = 0u;
        info[7] = (uint32_t)out.checkpoint;
    }
    return 0;
}

int gpupi_pi_compute(gpupi_ctx *ctx, uint32_t digits, uint32_t flags, uint32_t *h_ret, size_t ret_cap,
                     char *h_digits, size_t digits_cap, uint32_t *info) {
    gpupi::PiRequest req;
    req.digits = digits;
    req.profile_stages = (flags & 1u) != 0u;
    req.copy_digits = h_digits ? (uint32_t)std::min<size_t>(digits_cap, digits) : 0u;
    req.ctx = raw(ctx);
    req.device_only = (flags & 2u) != 0u;
    req.plain = (flags & 4u) != 0u;
    req.host_digits = h_digits;
    req.host_ret = h_ret;
    req.host_ret_cap = h_ret ? ret_cap : 0;
    gpupi::PiOutput out;
    cudaError_t err = gpupi::pi_run(req, out);
    if (err != cudaSuccess) return (int)err;
    if (info) {
        uint32_t leaf = 0u;
        gpupi::round_up_decimal_digits(digits, &leaf);
        info[0] = out.convert_digits;
        info[1] = out.ret_len;
        memcpy(&info[2], &out.elapsed_ms, 4);
        info[3] = (uint32_t)(out.workspace_bytes >> 20);
        info[4] = (uint32_t)out.stages.size();
        info[5] = leaf;
        info[6] = 0u;
        info[7] = 0u;
    }
    return 0;
}

int gpupi_timer_enable(int on) {
    gpupi::kernel_timer_enable(on != 0);
    return 0;
}

int gpupi_timer_reset(void) {
    gpupi::kernel_timer_reset();
    return 0;
}

size_t gpupi_timer_report(char *buf, size_t cap) { return gpupi::kernel_timer_report(buf, cap); }

int gpupi_bbp_fractions(const uint64_t *positions, uint32_t count, uint64_t *fractions) {
    return (int)gpupi::bbp_fractions(positions, count, fractions);
}

int gpupi_transfer_bytes(uint64_t *h2d, uint64_t *d2h) {
    gpupi::transfer_bytes(h2d, d2h);
    return 0;
}

int gpupi_scratch_stats(uint64_t *block_bytes, uint64_t *high_water, uint64_t *spills) {
    gpupi::scratch_stats(block_bytes, high_water, spills);
    return 0;
}

int gpupi_set_mul_crossover(uint32_t v) {
    if (v > (uint32_t)BATCH_MUL_NAIVE_L_MAX) return (int)cudaErrorInvalidValue;
    gpupi::set_school_max(v);
    return 0;
}

}  // extern "C"
