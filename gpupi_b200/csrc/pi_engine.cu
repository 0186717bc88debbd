// Chudnovsky pi pipeline driver (gpupi pi_bs_gpu.cu:36-131, 504-792,
// 1143-1685, 2073-2431).
//
// Host C++ drives the same sequence of batched operations as the reference,
// with the same operand lengths (including every compact()-derived length),
// so every intermediate integer, the RET value and the digits are identical.
// All limb work is done by this library's kernels on the current stream.
// Temporary device buffers come from the stream's scratch arena (scratch.cu):
// per-level allocation costs neither a device synchronisation nor, after
// the first call, any driver call.
#include "common.cuh"
#include "batch_arith.h"
#include "batch_mul_naive.h"
#include "batch_mul_ntt.h"
#include "convert_decimal.h"
#include "pi_engine.h"
#include "spectrum.h"
#include "checkpoint_file.h"

#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <mutex>
#include <string>
#include <vector>

namespace gpupi {

// ---------------------------------------------------------------------------
// Leaves (pi_bs_gpu.cu:17-131): P (3 limbs), Q (4), R (6) per term, after the
// same common-factor reductions by 5, 3, 23, 29.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void reduce_pair(uint32_t &a, uint32_t &b) {
    if (a % 3u == 0u && b % 3u == 0u) { a /= 3u; b /= 3u; }
    if (a % 5u == 0u && b % 5u == 0u) { a /= 5u; b /= 5u; }
    if (a % 23u == 0u && b % 23u == 0u) { a /= 23u; b /= 23u; }
    if (a % 29u == 0u && b % 29u == 0u) { a /= 29u; b /= 29u; }
}

template <int L>
__device__ __forceinline__ void mul_small_into(uint32_t (&x)[L], uint32_t m) {
    uint32_t c = 0u;
#pragma unroll
    for (int j = 0; j < L; ++j) {
        const uint64_t t = (uint64_t)x[j] * m + c;
        x[j] = (uint32_t)t;
        c = (uint32_t)(t >> 32);
    }
}

template <bool HEAD>
__global__ void k_leaves(uint32_t *P, uint32_t *Q, uint32_t *R, uint32_t rows) {
    for (uint32_t i2 = blockIdx.x * blockDim.x + threadIdx.x; i2 < rows; i2 += gridDim.x * blockDim.x) {
        const uint32_t i = HEAD ? i2 * 17u + 16u : i2 + (i2 >> 4);
        uint32_t p1 = 6u * i + 1u, p2 = 2u * i + 1u, p3 = 6u * i + 5u;
        uint32_t q1 = i + 1u, q2 = i + 1u, q3 = i + 1u;
        uint32_t q4 = 640320u >> 6, q5 = 40020u >> 2;
        const uint32_t q6 = 426880u >> 7;
        const uint64_t r1 = 545140134ull * i + 13591409ull;
        if (p1 % 5u == 0u && q1 % 5u == 0u) { p1 /= 5u; q1 /= 5u; }
        if (p1 % 5u == 0u && q2 % 5u == 0u) { p1 /= 5u; q2 /= 5u; }
        if (p1 % 5u == 0u && q3 % 5u == 0u) { p1 /= 5u; q3 /= 5u; }
        reduce_pair(p1, q4);
        reduce_pair(p1, q5);
        reduce_pair(p2, q4);
        reduce_pair(p2, q5);
        reduce_pair(p3, q4);
        reduce_pair(p3, q5);
        uint32_t pp[3] = {p1, 0u, 0u};
        mul_small_into<3>(pp, p2);
        mul_small_into<3>(pp, p3);
        uint32_t qq[4] = {q1, 0u, 0u, 0u};
        mul_small_into<4>(qq, q2);
        mul_small_into<4>(qq, q3);
        mul_small_into<4>(qq, q4);
        mul_small_into<4>(qq, q5);
        mul_small_into<4>(qq, q6);
        uint32_t rr[6] = {(uint32_t)r1, (uint32_t)(r1 >> 32), 0u, 0u, 0u, 0u};
        mul_small_into<6>(rr, q1);
        mul_small_into<6>(rr, q2);
        mul_small_into<6>(rr, q3);
        mul_small_into<6>(rr, q4);
        mul_small_into<6>(rr, q5);
#pragma unroll
        for (int k = 0; k < 3; ++k) P[(uint64_t)i2 * 3 + k] = pp[k];
#pragma unroll
        for (int k = 0; k < 4; ++k) Q[(uint64_t)i2 * 4 + k] = qq[k];
#pragma unroll
        for (int k = 0; k < 6; ++k) R[(uint64_t)i2 * 6 + k] = rr[k];
    }
}

// ---------------------------------------------------------------------------
// Stage profiler (pi_bs_gpu.cu:133-242): one event pair per op, synchronised.
// ---------------------------------------------------------------------------
struct Profiler {
    std::vector<StageEntry> entries;
    bool on = false;
};

template <typename Fn>
static cudaError_t stage(Profiler *pr, const char *kind, const char *label, uint32_t n1, uint32_t batch,
                         uint32_t lhs, uint32_t rhs, bool uses_ntt, Fn &&fn) {
    if (pr == nullptr || !pr->on) return fn();
    cudaStream_t st = current_stream();
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, st);
    cudaError_t err = fn();
    if (err == cudaSuccess) err = cudaEventRecord(b, st);
    if (err == cudaSuccess) err = cudaEventSynchronize(b);
    float ms = 0.f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, a, b);
    if (err == cudaSuccess && pr->entries.size() < 2048) {
        StageEntry e;
        e.kind = kind;
        e.label = label;
        e.n1 = n1;
        e.batch = batch;
        e.lhs = lhs;
        e.rhs = rhs;
        e.ms = ms;
        e.uses_ntt = uses_ntt;
        pr->entries.push_back(e);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return err;
}

#define TRY(x)                                   \
    do {                                         \
        cudaError_t _e = (x);                    \
        if (_e != cudaSuccess) return _e;        \
    } while (0)

static cudaError_t p_mul(BatchMPContext *ctx, Profiler *pr, BatchMPArray A, BatchMPArray B, BatchMPArray C,
                         const char *label, uint32_t n1) {
    return stage(pr, "mul", label, n1, A.batch_size, A.length, B.length,
                 (size_t)A.length + B.length > (size_t)BATCH_MUL_NAIVE_L_MAX,
                 [&]() { return mul_tuned(ctx, A, B, C); });
}
// ---------------------------------------------------------------------------
// The splitting tree's length schedule.  Every level of the tree ends in
// compact(): a device scan whose result the host reads back (a stream
// synchronisation) to size the next level's rows, as in the reference.  The
// lengths depend only on the tree size, so the first run for a size records
// them (RECORD); later runs take them from the record and only launch the
// scans, writing into a device array that is compared with the record once
// the tree is done (REPLAY).  With no host synchronisation left inside it,
// the tree can be captured into a CUDA graph (tree_start).
// ---------------------------------------------------------------------------
cudaError_t limb_length_to_device(const uint32_t *A, uint32_t N, uint32_t L, uint32_t stride, uint32_t *d_out);
cudaError_t limb_length_prepare();

enum TreeMode { kTreeDirect = 0, kTreeRecord = 1, kTreeReplay = 2 };
struct TreeLens {
    TreeMode mode = kTreeDirect;
    std::vector<uint32_t> *lens = nullptr;   // the record (written in RECORD, read in REPLAY)
    uint32_t *d_check = nullptr;             // REPLAY: the scans' results, one word per compact
    size_t cursor = 0;
    bool overflow = false;                   // REPLAY met more compacts than recorded
};
static thread_local TreeLens t_tree;

static cudaError_t p_compact(BatchMPContext *ctx, Profiler *pr, BatchMPArray &A, const char *label, uint32_t n1) {
    TreeLens &t = t_tree;
    if (t.mode == kTreeReplay) {
        if (t.cursor >= t.lens->size()) {
            t.overflow = true;
            return cudaErrorInvalidValue;
        }
        const cudaError_t err = limb_length_to_device(A.data, A.batch_size, A.length, A.stride, t.d_check + t.cursor);
        A.length = (*t.lens)[t.cursor++];
        return err;
    }
    const cudaError_t err =
        stage(pr, "compact", label, n1, A.batch_size, A.length, 0, false, [&]() { return A.compact(ctx); });
    if (err == cudaSuccess && t.mode == kTreeRecord) t.lens->push_back(A.length);
    return err;
}
static cudaError_t p_shift_addsub(BatchMPContext *ctx, Profiler *pr, BatchMPArray A, BatchMPArray B,
                                  BatchMPArray C, uint32_t shift, bool sub, uint32_t n1) {
    return stage(pr, sub ? "sub" : "add", sub ? "R*Q<<15n-P*R" : "R*Q<<15n+P*R", n1, A.batch_size, A.length,
                 B.length, false, [&]() {
                     return sub ? batch_mp_shift_sub(ctx, A, B, shift, C) : batch_mp_shift_add(ctx, A, B, shift, C);
                 });
}
static cudaError_t p_exactdiv(BatchMPContext *ctx, Profiler *pr, BatchMPArray A, const char *label, uint32_t d,
                              uint32_t n1) {
    return stage(pr, "exactdiv", label, n1, A.batch_size, A.length, 0, false,
                 [&]() { return batch_mp_exactdiv_small(ctx, A, d); });
}
static cudaError_t p_add(BatchMPContext *ctx, Profiler *pr, BatchMPArray A, BatchMPArray B, BatchMPArray C,
                         const char *label, uint32_t dg) {
    return stage(pr, "add", label, dg, A.batch_size, A.length, B.length, false,
                 [&]() { return batch_mp_add(ctx, A, B, C); });
}
static cudaError_t p_sub(BatchMPContext *ctx, Profiler *pr, BatchMPArray A, BatchMPArray B, BatchMPArray C,
                         const char *label, uint32_t dg) {
    return stage(pr, "sub", label, dg, A.batch_size, A.length, B.length, false,
                 [&]() { return batch_mp_sub(ctx, A, B, C); });
}
static cudaError_t p_add_small(BatchMPContext *ctx, Profiler *pr, BatchMPArray A, uint32_t v, BatchMPArray C,
                               const char *label, uint32_t dg) {
    return stage(pr, "add", label, dg, A.batch_size, A.length, 1, false,
                 [&]() { return batch_mp_add_small(ctx, A, v, C); });
}
static cudaError_t p_mul_small(BatchMPContext *ctx, Profiler *pr, BatchMPArray A, uint32_t v, BatchMPArray C,
                               const char *label, uint32_t dg) {
    return stage(pr, "mul_small", label, dg, A.batch_size, A.length, 1, false,
                 [&]() { return batch_mp_mul_small(ctx, A, v, C); });
}
static cudaError_t p_shift(BatchMPContext *ctx, Profiler *pr, BatchMPArray A, BatchMPArray B, int32_t s,
                           const char *label, uint32_t dg) {
    return stage(pr, "shift", label, dg, A.batch_size, A.length, 0, false,
                 [&]() { return batch_mp_shift_bits(ctx, A, B, s); });
}

// Device buffer from the stream's scratch arena.
struct Buf {
    uint32_t *p = nullptr;
    Buf() = default;
    Buf(const Buf &) = delete;
    Buf &operator=(const Buf &) = delete;
    ~Buf() { reset(); }
    void reset() {
        scratch_free(p);
        p = nullptr;
    }
    cudaError_t alloc(size_t words) {
        reset();
        if (words == 0) words = 1;
        return scratch_alloc((void **)&p, words * 4);
    }
    void swap(Buf &o) { std::swap(p, o.p); }
    uint32_t *release() {   // give up ownership without freeing
        uint32_t *q = p;
        p = nullptr;
        return q;
    }
};

static const uint32_t kDivLo = 830297u;       // pi_bs_gpu.cu:147
static const uint32_t kDivHi = 156590819u;    // pi_bs_gpu.cu:148

// One merge level as the reference issues it (pi_bs_gpu.cu:625-723): four
// products, the shifted addition or subtraction, three compactions.
static cudaError_t plain_level(BatchMPContext *ctx, Profiler *pr, uint32_t n, uint32_t n1, uint32_t half,
                               uint32_t ignore, bool subtract, const BatchMPArray &P, const BatchMPArray &Q,
                               const BatchMPArray &R, Buf &pn, BatchMPArray &Pn, Buf &qn, BatchMPArray &Qn, Buf &rn,
                               BatchMPArray &Rn) {
    Buf r1b, r2b;
    BatchMPArray P_even{P.data, P.length, half - ignore, P.stride * 2};
    BatchMPArray P_odd{P.data + P.stride, P.length, half - ignore, P.stride * 2};
    Pn = BatchMPArray{nullptr, P.length * 2u, half - ignore, P.length * 2u};
    if (P_odd.batch_size > 0u) {
        TRY(pn.alloc((size_t)Pn.batch_size * Pn.stride));
        Pn.data = pn.p;
        TRY(p_mul(ctx, pr, P_even, P_odd, Pn, "P", n1));
        TRY(p_compact(ctx, pr, Pn, "P", n1));
    } else {
        pn.reset();
        Pn = BatchMPArray{nullptr, 0, 0, 0};
    }
    BatchMPArray Q_even{Q.data, Q.length, half, Q.stride * 2};
    BatchMPArray Q_odd{Q.data + Q.stride, Q.length, half, Q.stride * 2};
    Qn = BatchMPArray{nullptr, Q.length * 2u, half, Q.length * 2u};
    TRY(qn.alloc((size_t)half * Qn.stride));
    Qn.data = qn.p;
    TRY(p_mul(ctx, pr, Q_even, Q_odd, Qn, "Q", n1));
    TRY(p_compact(ctx, pr, Qn, "Q", n1));
    BatchMPArray R_even{R.data, R.length, half, R.stride * 2};
    BatchMPArray R_odd{R.data + R.stride, R.length, half, R.stride * 2};
    BatchMPArray R1{nullptr, R.length + Q.length, half, R.length + Q.length};
    TRY(r1b.alloc((size_t)half * R1.stride));
    R1.data = r1b.p;
    TRY(p_mul(ctx, pr, R_even, Q_odd, R1, "R*Q", n1));
    const uint32_t shift = 15u * ((n / n1) + ((n / n1) >> 4));
    BatchMPArray R2{nullptr, R.length + P.length, half, R.length + P.length};
    TRY(r2b.alloc((size_t)half * R2.stride));
    R2.data = r2b.p;
    P_even.batch_size = half;
    TRY(p_mul(ctx, pr, P_even, R_odd, R2, "P*R", n1));
    const uint32_t r1_shifted = R1.length + (shift >> 5) + ((shift & 31u) != 0u ? 1u : 0u);
    const uint32_t rlen = std::max(r1_shifted, R2.length) + (subtract ? 0u : 1u);
    Rn = BatchMPArray{nullptr, rlen, half, rlen};
    TRY(rn.alloc((size_t)half * rlen));
    Rn.data = rn.p;
    TRY(p_shift_addsub(ctx, pr, R1, R2, Rn, shift, subtract, n1));
    TRY(p_compact(ctx, pr, Rn, "R", n1));
    return cudaSuccess;
}

// ---------------------------------------------------------------------------
// One merge level with shared forward transforms (the tuned form of
// pi_bs_gpu.cu:625-723): Q_o serves Q' = Q_e Q_o and R1 = R_e Q_o, P_e
// serves P' = P_e P_o and R2 = P_e R_o, so the level's four products take
// six forward transforms instead of eight (four inverse either way): the
// six operands' column passes, then one row kernel for the four products
// (spectrum_level_rows), then each product's inverse column passes and
// CRT; R' = (R1 << s) +- R2 as in the plain level.  All products run at the
// largest one's transform shape; used when that costs less than the plain
// level (summing R' in the transform domain would need room for R1 << s,
// about 6 % longer than R1, which sits just below a power of two at every
// level and would double the transforms).  At the root P' is not formed
// (as in the plain level): five forward and three inverse transforms.  The
// integers are those of the plain level.  *done = false (nothing issued)
// when the level does not qualify.
// ---------------------------------------------------------------------------
static cudaError_t tuned_level(BatchMPContext *ctx, Profiler *pr, uint32_t n, uint32_t n1, uint32_t half,
                               uint32_t ignore, bool subtract, const BatchMPArray &P, const BatchMPArray &Q,
                               const BatchMPArray &R, Buf &pn, BatchMPArray &Pn, Buf &qn, BatchMPArray &Qn, Buf &rn,
                               BatchMPArray &Rn, bool *done) {
    *done = false;
    const uint32_t lp = P.length, lq = Q.length, lr = R.length;
    const uint32_t pb = half - ignore;   // rows of P' (0 at the root: P' is not needed there)
    // One shape serves the level: the largest product's.  A product whose
    // own shape is smaller runs at it too (exact either way: the shape only
    // has to cover the coefficients), which pays when the shared forward
    // transforms save more than the larger inverse costs.  Cost model:
    // residues transformed, M * K per row transform; the plain level runs
    // three transforms per product at each product's own shape.
    const uint64_t needs[4] = {2ull * lq - 1u, (uint64_t)lr + lq - 1u, (uint64_t)lp + lr - 1u, 2ull * lp - 1u};
    const uint32_t rows_of[4] = {half, half, half, pb};
    uint64_t most = 0;
    for (int i = 0; i < 4; ++i)
        if (rows_of[i]) most = std::max(most, needs[i]);
    const SpectrumShape S = spectrum_shape(most);
    if (S.M == 0) return cudaSuccess;
    auto cap = [](SpectrumShape s, uint64_t need) { return s.M ? (uint64_t)s.M << s.log_k : need; };
    uint64_t plain_cost = 0;
    for (int i = 0; i < 4; ++i) plain_cost += 3ull * rows_of[i] * cap(spectrum_shape(needs[i]), needs[i]);
    // forward: P_e, Q_e, Q_o, R_e, R_o (half rows each) and P_o (pb rows);
    // inverse: Q', R1, R2 (half rows each) and P' (pb rows)
    const uint64_t tuned_cost = (8ull * half + 2ull * pb) * cap(S, most);
    if (tuned_cost > plain_cost) return cudaSuccess;
    *done = true;
    const NTTPrecomputedTables &tab = context_tables(ctx);
    const uint64_t words = spectrum_words(S, half);
    const BatchMPArray P_even{P.data, lp, half, P.stride * 2}, P_odd{P.data + P.stride, lp, pb, P.stride * 2};
    const BatchMPArray Q_even{Q.data, lq, half, Q.stride * 2}, Q_odd{Q.data + Q.stride, lq, half, Q.stride * 2};
    const BatchMPArray R_even{R.data, lr, half, R.stride * 2}, R_odd{R.data + R.stride, lr, half, R.stride * 2};
    Buf fpe, fpo, fqe, fqo, fre, fro, flags, r1b, r2b;
    const uint32_t shift = 15u * ((n / n1) + ((n / n1) >> 4));
    const uint32_t r1_shifted = lr + lq + (shift >> 5) + ((shift & 31u) != 0u ? 1u : 0u);
    const uint32_t rlen = std::max(r1_shifted, lr + lp) + (subtract ? 0u : 1u);
    TRY(flags.alloc(spectrum_flag_words(
        half, std::max(std::max(std::max(lr + lq, 2u * lq), std::max(lr + lp, 2u * lp)), rlen))));
    // column passes of the six operands, two per launch: P_e and P_o share
    // the pb rows they both have (P_e's last row follows alone when P has an
    // odd row count; P_o's row there is left unset and its product unused)
    TRY(stage(pr, "fwd", "P,Q,R columns", n1, half, lp, lq, true, [&]() {
        TRY(fpe.alloc(words));
        if (pb) TRY(fpo.alloc(words));
        TRY(fqo.alloc(words));
        TRY(fqe.alloc(words));
        TRY(fre.alloc(words));
        TRY(fro.alloc(words));
        if (pb)
            spectrum_forward(tab, S, pb, P_even.data, P_even.stride, lp, fpe.p, P_odd.data, P_odd.stride, lp,
                             fpo.p, false);
        if (pb < half)
            spectrum_forward(tab, S, 1u, P_even.data + (size_t)pb * P_even.stride, P_even.stride, lp,
                             fpe.p + spectrum_words(S, pb), nullptr, 0, 0, nullptr, false);
        spectrum_forward(tab, S, half, Q_odd.data, Q_odd.stride, lq, fqo.p, Q_even.data, Q_even.stride, lq, fqe.p,
                         false);
        spectrum_forward(tab, S, half, R_even.data, R_even.stride, lr, fre.p, R_odd.data, R_odd.stride, lr, fro.p,
                         false);
        // the four products' row passes in one kernel (three without P')
        spectrum_level_rows(tab, S, half, fpe.p, pb ? fpo.p : nullptr, fro.p, fqo.p, fqe.p, fre.p);
        fpe.reset();
        fqo.reset();
        return cudaGetLastError();
    }));
    auto finish = [&](const char *label, uint32_t rows, Buf &f, uint32_t *C, uint32_t Lc, uint32_t la,
                      uint32_t lb) {
        return stage(pr, "mul", label, n1, rows, la, lb, true, [&]() {
            spectrum_inverse(tab, S, rows, 1, nullptr, nullptr, f.p, C, Lc, Lc, flags.p, false);
            f.reset();
            return cudaGetLastError();
        });
    };
    if (pb) {
        Pn = BatchMPArray{nullptr, 2u * lp, pb, 2u * lp};
        TRY(pn.alloc((size_t)pb * Pn.stride));
        Pn.data = pn.p;
        TRY(finish("P", pb, fpo, Pn.data, Pn.length, lp, lp));
        TRY(p_compact(ctx, pr, Pn, "P", n1));
    } else {
        pn.reset();
        Pn = BatchMPArray{nullptr, 0, 0, 0};
    }
    Qn = BatchMPArray{nullptr, 2u * lq, half, 2u * lq};
    TRY(qn.alloc((size_t)half * Qn.stride));
    Qn.data = qn.p;
    TRY(finish("Q", half, fqe, Qn.data, Qn.length, lq, lq));
    TRY(p_compact(ctx, pr, Qn, "Q", n1));
    const BatchMPArray R1{nullptr, lr + lq, half, lr + lq}, R2{nullptr, lr + lp, half, lr + lp};
    TRY(r1b.alloc((size_t)half * R1.stride));
    TRY(finish("R*Q", half, fre, r1b.p, R1.length, lr, lq));
    Rn = BatchMPArray{nullptr, rlen, half, rlen};
    TRY(rn.alloc((size_t)half * rlen));
    Rn.data = rn.p;
    if (!subtract) {
        // R' = (R1 << s) + R2 straight out of R2's CRT and carry pass: R1's
        // shifted limbs join the carry chain, R2 is never stored and no
        // separate addition pass runs (same integers as the plain level)
        const SpectrumAddend add{r1b.p, R1.stride, R1.length, shift, lr + lp - 1u};
        TRY(stage(pr, "mul", "P*R+(R*Q<<15n)", n1, half, lp, lr, true, [&]() {
            spectrum_inverse(tab, S, half, 1, nullptr, nullptr, fro.p, Rn.data, rlen, rlen, flags.p, false, &add);
            fro.reset();
            return cudaGetLastError();
        }));
        return p_compact(ctx, pr, Rn, "R", n1);
    }
    TRY(r2b.alloc((size_t)half * R2.stride));
    TRY(finish("P*R", half, fro, r2b.p, R2.length, lp, lr));
    TRY(p_shift_addsub(ctx, pr, BatchMPArray{r1b.p, R1.length, half, R1.stride},
                       BatchMPArray{r2b.p, R2.length, half, R2.stride}, Rn, shift, subtract, n1));
    return p_compact(ctx, pr, Rn, "R", n1);
}

// ---------------------------------------------------------------------------
// Binary splitting of 17N terms (pi_bs_gpu.cu:504-792).
// Q and R (batch 1) are returned in qbuf/rbuf with their compacted lengths.
// tuned: levels whose four products share one transform shape of at least
// 8192 points run as tuned_level (same integers).
// ---------------------------------------------------------------------------
static cudaError_t binary_split(BatchMPContext *ctx, Profiler *pr, uint32_t N, Buf &qbuf, BatchMPArray &Q,
                                Buf &rbuf, BatchMPArray &R, bool tuned) {
    if (N == 0u || (N & (N - 1u)) != 0u) return cudaErrorInvalidValue;
    cudaStream_t st = current_stream();
    const uint32_t n = N * 16u;
    Buf p0, q0, r0, pb, qb, rb, pn, qn, rn, r1b, r2b;
    TRY(p0.alloc((size_t)N * 3));
    TRY(q0.alloc((size_t)N * 4));
    TRY(r0.alloc((size_t)N * 6));
    TRY(pb.alloc((size_t)n * 3));
    TRY(qb.alloc((size_t)n * 4));
    TRY(rb.alloc((size_t)n * 6));
    TRY(stage(pr, "leaf", "construct_leaf", N * 17u, N, 3, 0, false, [&]() {
        k_leaves<true><<<grid_for(N, 128, 65535), 128, 0, st>>>(p0.p, q0.p, r0.p, N);
        count_launch();
        return cudaGetLastError();
    }));
    TRY(stage(pr, "leaf", "construct_leaf", N * 17u, n, 3, 0, false, [&]() {
        k_leaves<false><<<grid_for(n, 128, 65535), 128, 0, st>>>(pb.p, qb.p, rb.p, n);
        count_launch();
        return cudaGetLastError();
    }));
    const BatchMPArray P0{p0.p, 3, N, 3}, Q0{q0.p, 4, N, 4}, R0{r0.p, 6, N, 6};
    BatchMPArray P{pb.p, 3, n, 3};
    Q = BatchMPArray{qb.p, 4, n, 4};
    R = BatchMPArray{rb.p, 6, n, 6};

    for (uint32_t n1 = n; n1 > 1u; n1 >>= 1) {
        const bool subtract = (n1 == n) || (n1 == (n >> 4));
        const uint32_t ignore = (n1 <= N) ? 1u : 0u;
        const uint32_t half = n1 / 2u;
        BatchMPArray Pn, Qn, Rn;
        bool done = false;
        if (tuned) TRY(tuned_level(ctx, pr, n, n1, half, ignore, subtract, P, Q, R, pn, Pn, qn, Qn, rn, Rn, &done));
        if (!done) TRY(plain_level(ctx, pr, n, n1, half, ignore, subtract, P, Q, R, pn, Pn, qn, Qn, rn, Rn));
        pb.swap(pn);
        qb.swap(qn);
        rb.swap(rn);
        P = Pn;
        Q = Qn;
        R = Rn;
        pn.reset();
        qn.reset();
        rn.reset();
        if (n1 == (n >> 3)) {
            // merge the head term of every 17-term block (pi_bs_gpu.cu:725-784)
            BatchMPArray Pm{nullptr, P.length + P0.length, half, P.length + P0.length};
            TRY(pn.alloc((size_t)half * Pm.stride));
            Pm.data = pn.p;
            TRY(p_mul(ctx, pr, P, P0, Pm, "P", n1));
            TRY(p_compact(ctx, pr, Pm, "P", n1));
            BatchMPArray Qm{nullptr, Q.length + Q0.length, half, Q.length + Q0.length};
            TRY(qn.alloc((size_t)half * Qm.stride));
            Qm.data = qn.p;
            TRY(p_mul(ctx, pr, Q, Q0, Qm, "Q", n1));
            TRY(p_compact(ctx, pr, Qm, "Q", n1));
            BatchMPArray M1{nullptr, R.length + Q0.length, half, R.length + Q0.length};
            TRY(r1b.alloc((size_t)half * M1.stride));
            M1.data = r1b.p;
            TRY(p_mul(ctx, pr, R, Q0, M1, "R*Q", n1));
            BatchMPArray M2{nullptr, P.length + R0.length, half, P.length + R0.length};
            TRY(r2b.alloc((size_t)half * M2.stride));
            M2.data = r2b.p;
            TRY(p_mul(ctx, pr, P, R0, M2, "P*R", n1));
            const uint32_t ml = std::max(M1.length + 1u, M2.length) + 1u;
            BatchMPArray Rm{nullptr, ml, half, ml};
            TRY(rn.alloc((size_t)half * ml));
            Rm.data = rn.p;
            TRY(p_shift_addsub(ctx, pr, M1, M2, Rm, 15u, false, n1));
            TRY(p_compact(ctx, pr, Rm, "R", n1));
            TRY(p_exactdiv(ctx, pr, Pm, "P", kDivLo, n1));
            TRY(p_exactdiv(ctx, pr, Pm, "P", kDivHi, n1));
            TRY(p_compact(ctx, pr, Pm, "P", n1));
            TRY(p_exactdiv(ctx, pr, Qm, "Q", kDivLo, n1));
            TRY(p_exactdiv(ctx, pr, Qm, "Q", kDivHi, n1));
            TRY(p_compact(ctx, pr, Qm, "Q", n1));
            TRY(p_exactdiv(ctx, pr, Rm, "R", kDivLo, n1));
            TRY(p_exactdiv(ctx, pr, Rm, "R", kDivHi, n1));
            TRY(p_compact(ctx, pr, Rm, "R", n1));
            pb.swap(pn);
            qb.swap(qn);
            rb.swap(rn);
            P = Pm;
            Q = Qm;
            R = Rm;
            r1b.reset();
            r2b.reset();
            pn.reset();
            qn.reset();
            rn.reset();
        }
    }
    qbuf.swap(qb);
    rbuf.swap(rb);
    return cudaSuccess;
}

// ---------------------------------------------------------------------------
// The splitting tree as a CUDA graph.
//
// Per (context, tree size, form): the first run records the length schedule
// (and the tree's peak of scratch bytes); the second captures the tree with
// the recorded lengths (no host synchronisation inside) into a graph, its
// temporaries carved from a private device block so that the graph's
// addresses stay valid; every later run launches that graph on the
// library's tree stream (ordered after and before the caller's stream by
// events) and checks the lengths the device computed against the schedule
// with one copy.  A disagreement (never expected: the computation is
// deterministic) runs the tree directly and records again, so the result is
// always the exact one.  Q and R then live in the private block until the
// next run of the same graph.  Not used while the stage profiler or the
// kernel timers are on (both time individual launches), when the block
// would not leave 8 GB of the device free, or with GPUPI_TREE_GRAPH=0.
// ---------------------------------------------------------------------------
namespace {
struct TreeGraph {
    const BatchMPContext *ctx = nullptr;
    int dev = -1;
    uint32_t N = 0;
    bool tuned = false;
    int state = 0;   // 0 nothing, 1 schedule recorded, 2 graph captured, 3 graph not possible
    std::vector<uint32_t> lens;
    size_t peak = 0;
    void *pool = nullptr;
    size_t pool_cap = 0;
    uint32_t *d_check = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t *q = nullptr, *r = nullptr;
    uint32_t lq = 0, lr = 0;
    int64_t launches = 0;
    const void *ws = nullptr;
    size_t ws_size = 0;
};
std::mutex g_tree_mu;
std::vector<TreeGraph> g_trees;
TreeGraphStats g_tree_stats{};

void tree_release(TreeGraph &g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.pool) {
        scratch_private_drop(g.pool);
        cudaFree(g.pool);
    }
    if (g.d_check) cudaFree(g.d_check);
    g.exec = nullptr;
    g.pool = nullptr;
    g.d_check = nullptr;
    g.q = g.r = nullptr;
}

cudaStream_t tree_stream(int dev) {
    static cudaStream_t s[64] = {};
    if (dev < 0 || dev >= 64) return nullptr;
    if (!s[dev] && cudaStreamCreateWithFlags(&s[dev], cudaStreamNonBlocking) != cudaSuccess) s[dev] = nullptr;
    return s[dev];
}

// Two events per device: the caller's stream's work before the graph, and
// the graph's end.
cudaEvent_t *tree_events(int dev) {
    static cudaEvent_t evs[64][2] = {};
    cudaEvent_t *ev = evs[dev & 63];
    if (!ev[0]) {
        cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
    }
    return ev;
}

bool tree_graphs_enabled() {
    const char *e = getenv("GPUPI_TREE_GRAPH");
    return !(e && e[0] == '0');
}
}  // namespace

TreeGraphStats tree_graph_stats() {
    std::lock_guard<std::mutex> l(g_tree_mu);
    return g_tree_stats;
}

void tree_graph_perturb() {
    std::lock_guard<std::mutex> l(g_tree_mu);
    for (TreeGraph &g : g_trees)
        if (!g.lens.empty() && g.lens[0] > 1u) g.lens[0] -= 1u;
}

// A second context per caller context for the work that runs beside the
// tree's graph (the sqrt(10005) iteration): the graph's products use the
// caller context's workspace, so the side work needs its own.
static std::mutex g_side_mu;
static std::vector<std::pair<const BatchMPContext *, BatchMPContext *>> g_sides;

static BatchMPContext *side_context(const BatchMPContext *ctx) {
    std::lock_guard<std::mutex> l(g_side_mu);
    for (auto &e : g_sides)
        if (e.first == ctx) return e.second;
    BatchMPContext *side = batch_mp_init();
    if (!side) return nullptr;
    // the side work's products below the shared-transform sizes: no
    // workspace growth (a synchronising allocation) while the graph runs
    if (batch_mp_ensure_workspace(side, batch_mul_ntt_workspace_size(1u, 8192u, 8192u)) != cudaSuccess) {
        batch_mp_destroy(side);
        return nullptr;
    }
    g_sides.emplace_back(ctx, side);
    return side;
}

void pi_forget_context(const BatchMPContext *ctx) {
    BatchMPContext *side = nullptr;
    {
        std::lock_guard<std::mutex> l(g_side_mu);
        for (auto it = g_sides.begin(); it != g_sides.end(); ++it)
            if (it->first == ctx) {
                side = it->second;
                g_sides.erase(it);
                break;
            }
    }
    if (side) batch_mp_destroy(side);
    std::lock_guard<std::mutex> l(g_tree_mu);
    for (auto it = g_trees.begin(); it != g_trees.end();) {
        if (it->ctx == ctx) {
            int cur = 0;
            cudaGetDevice(&cur);
            if (it->dev != cur) cudaSetDevice(it->dev);
            cudaDeviceSynchronize();
            tree_release(*it);
            if (it->dev != cur) cudaSetDevice(cur);
            it = g_trees.erase(it);
        } else {
            ++it;
        }
    }
}

// Captures the tree into g (state 1 -> 2).  Returns cudaSuccess with
// *usable false when a graph is not possible here (a capture-specific
// failure: the tree then runs directly), or the error of the tree itself.
static cudaError_t tree_capture(BatchMPContext *ctx, TreeGraph &g, bool *usable) {
    *usable = false;
    const size_t cap = g.peak + g.peak / 4 + ((size_t)64 << 20);
    // the block comes on top of the stream's arena: only with room to spare
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || cap + ((size_t)8 << 30) > free_b) {
        cudaGetLastError();
        return cudaSuccess;
    }
    if (cudaMalloc(&g.pool, cap) != cudaSuccess ||
        cudaMalloc((void **)&g.d_check, std::max<size_t>(1, g.lens.size()) * 4) != cudaSuccess) {
        cudaGetLastError();
        tree_release(g);
        return cudaSuccess;
    }
    g.pool_cap = cap;
    cudaStream_t st = current_stream(), ts = tree_stream(g.dev);
    if (!ts) {
        tree_release(g);
        return cudaSuccess;
    }
    const uint64_t l0 = launch_counter();
    t_tree = TreeLens{};
    t_tree.mode = kTreeReplay;
    t_tree.lens = &g.lens;
    t_tree.d_check = g.d_check;
    set_current_stream(ts);
    if (limb_length_prepare() != cudaSuccess) {   // the tree stream's length-scan words, before capturing
        set_current_stream(st);
        t_tree = TreeLens{};
        tree_release(g);
        return cudaSuccess;
    }
    scratch_private_begin(g.pool, cap);
    cudaGraph_t graph = nullptr;
    Buf q, r;
    BatchMPArray Q, R;
    cudaError_t err = cudaStreamBeginCapture(ts, cudaStreamCaptureModeThreadLocal);
    const bool began = err == cudaSuccess;
    if (began) err = binary_split(ctx, nullptr, g.N, q, Q, r, R, g.tuned);
    const cudaError_t cerr = began ? cudaStreamEndCapture(ts, &graph) : err;
    const bool fits = scratch_private_end();
    set_current_stream(st);
    const bool complete = !t_tree.overflow && t_tree.cursor == g.lens.size();
    t_tree = TreeLens{};
    const int64_t recorded = (int64_t)(launch_counter() - l0);
    add_launches(-recorded);   // captured, not run: counted at each launch of the graph
    g.launches = 0;
    if (began && err == cudaSuccess && cerr == cudaSuccess && fits && complete && graph &&
        cudaGraphInstantiate(&g.exec, graph, 0) == cudaSuccess) {
        cudaGraphDestroy(graph);
        g.q = q.release();
        g.r = r.release();
        g.lq = Q.length;
        g.lr = R.length;
        g.ws = context_workspace(ctx);
        g.ws_size = batch_mp_workspace_size(ctx);
        g.launches = recorded;
        g.state = 2;
        *usable = true;
        return cudaSuccess;
    }
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    q.reset();
    r.reset();
    tree_release(g);
    // an error of the tree itself (not of capturing it) is the caller's
    if (began && err != cudaSuccess && fits && cerr == cudaSuccess) return err;
    return cudaSuccess;
}

// A tree whose graph was launched and not yet joined: the graph runs on the
// tree stream while the caller's stream is free for independent work.  The
// tree's lock is held until the join.
struct TreeJoin {
    std::unique_lock<std::mutex> lock;
    TreeGraph *g = nullptr;   // null: the tree has already run (directly)
    BatchMPContext *ctx = nullptr;
    Profiler *pr = nullptr;
    uint32_t N = 0;
    bool tuned = false;
};

// Starts the tree: a captured graph is launched on the tree stream after
// the caller's stream's work and left running (tj.g set; tree_join orders
// the caller's stream after it and checks the lengths); otherwise the tree
// runs directly, recording or capturing its graph on the way.
static cudaError_t tree_start(BatchMPContext *ctx, Profiler *pr, uint32_t N, Buf &qbuf, BatchMPArray &Q,
                              Buf &rbuf, BatchMPArray &R, bool tuned, TreeJoin &tj) {
    tj = TreeJoin{};
    if (!tree_graphs_enabled() || (pr && pr->on) || kernel_timer_enabled())
        return binary_split(ctx, pr, N, qbuf, Q, rbuf, R, tuned);
    int dev = 0;
    cudaGetDevice(&dev);
    std::unique_lock<std::mutex> lock(g_tree_mu);
    TreeGraph *g = nullptr;
    for (TreeGraph &x : g_trees)
        if (x.ctx == ctx && x.dev == dev && x.N == N && x.tuned == tuned) g = &x;
    if (!g) {
        g_trees.push_back(TreeGraph{});
        g = &g_trees.back();
        g->ctx = ctx;
        g->dev = dev;
        g->N = N;
        g->tuned = tuned;
    }
    if (g->state == 3) {
        lock.unlock();
        return binary_split(ctx, pr, N, qbuf, Q, rbuf, R, tuned);
    }
    if (g->state == 2 && (g->ws != context_workspace(ctx) || g->ws_size != batch_mp_workspace_size(ctx))) {
        tree_release(*g);   // the graph's products used another workspace
        g->state = 1;
    }
    if (g->state == 0) {
        std::vector<uint32_t> lens;
        t_tree = TreeLens{};
        t_tree.mode = kTreeRecord;
        t_tree.lens = &lens;
        scratch_window_begin();
        const cudaError_t err = binary_split(ctx, pr, N, qbuf, Q, rbuf, R, tuned);
        const size_t peak = scratch_window_peak();
        t_tree = TreeLens{};
        if (err != cudaSuccess) return err;
        g->lens.swap(lens);
        g->peak = peak;
        g->state = 1;
        ++g_tree_stats.recorded;
        return cudaSuccess;
    }
    if (g->state == 1) {
        bool usable = false;
        const cudaError_t err = tree_capture(ctx, *g, &usable);
        if (err != cudaSuccess) return err;
        if (!usable) {
            g->state = 3;
            ++g_tree_stats.disabled;
            lock.unlock();
            return binary_split(ctx, pr, N, qbuf, Q, rbuf, R, tuned);
        }
        ++g_tree_stats.captured;
    }
    // launch the graph after the caller's stream's work
    cudaStream_t st = current_stream(), ts = tree_stream(dev);
    cudaEvent_t *ev = tree_events(dev);
    cudaError_t err = cudaEventRecord(ev[0], st);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(ts, ev[0], 0);
    if (err == cudaSuccess) err = cudaGraphLaunch(g->exec, ts);
    if (err == cudaSuccess) err = cudaEventRecord(ev[1], ts);
    if (err != cudaSuccess) return err;
    add_launches(g->launches);
    tj.lock = std::move(lock);
    tj.g = g;
    tj.ctx = ctx;
    tj.pr = pr;
    tj.N = N;
    tj.tuned = tuned;
    return cudaSuccess;
}

// Orders the caller's stream after a launched graph and checks the lengths
// the device found against the schedule the graph used (a disagreement,
// never expected, runs the tree directly and records it again).
static cudaError_t tree_join(TreeJoin &tj, Buf &qbuf, BatchMPArray &Q, Buf &rbuf, BatchMPArray &R) {
    TreeGraph *g = tj.g;
    if (!g) return cudaSuccess;
    tj.g = nullptr;
    cudaStream_t st = current_stream();
    cudaError_t err = cudaStreamWaitEvent(st, tree_events(g->dev)[1], 0);
    if (err != cudaSuccess) return err;
    std::vector<uint32_t> seen(g->lens.size());
    if (!seen.empty()) {
        err = cudaMemcpyAsync(seen.data(), g->d_check, seen.size() * 4, cudaMemcpyDeviceToHost, st);
        if (err == cudaSuccess) err = cudaStreamSynchronize(st);
        if (err != cudaSuccess) return err;
        note_d2h(seen.size() * 4);
    }
    if (seen != g->lens) {
        ++g_tree_stats.fallbacks;
        tree_release(*g);
        g->lens.clear();
        g->state = 0;
        tj.lock.unlock();
        return binary_split(tj.ctx, tj.pr, tj.N, qbuf, Q, rbuf, R, tj.tuned);
    }
    ++g_tree_stats.replayed;
    qbuf.reset();
    rbuf.reset();
    Q = BatchMPArray{g->q, g->lq, 1, g->lq};
    R = BatchMPArray{g->r, g->lr, 1, g->lr};
    tj.lock.unlock();
    return cudaSuccess;
}

// ---------------------------------------------------------------------------
// sqrt(10005) Pell iteration (pi_bs_gpu.cu:1346-1522): (p, q) <- (p^2 +
// 10005 q^2, 2pq) from (4001, 40) while 7.5 * 2^k < digits.
// ---------------------------------------------------------------------------
// One Pell step in the tuned form: the same P' = P^2 + 10005 Q^2 and
// Q' = 2 P Q from shared transforms.  P and Q are transformed once, and so
// is 10005 Q (one small multiply), and P' is the spectral sum
// P P + (10005 Q) Q: three forward and two inverse transforms instead of
// four and three, and no separate 10005 x, addition or intermediate
// compaction passes.  Both results are compacted, as in the plain step, so
// the lengths (and every later operation) are the plain step's.
// *done = false (nothing issued) below the shared-transform sizes.
static cudaError_t sqrt_step_tuned(BatchMPContext *ctx, Profiler *pr, uint32_t sd, const BatchMPArray &P,
                                   const BatchMPArray &Q, Buf &np, BatchMPArray &NP, Buf &nq, BatchMPArray &NQ,
                                   bool *done) {
    *done = false;
    const uint32_t lp = P.length, lq = Q.length;
    const uint32_t npl = std::max(2u * lp, 2u * lq + 1u) + 1u;   // P^2 + 10005 Q^2 < 2^(32 (npl - 1) + 1)
    const SpectrumShape S = spectrum_shape(std::max<uint64_t>(npl - 1u, (uint64_t)lp + lq - 1u));
    const uint32_t la[2] = {lp, lq + 1u}, lb[2] = {lp, lq};
    if (S.M == 0 || !spectrum_sum_fits(la, lb, 2)) return cudaSuccess;
    *done = true;
    const NTTPrecomputedTables &tab = context_tables(ctx);
    const uint64_t words = spectrum_words(S, 1u);
    Buf q5, fp, fq, fq5, flags;
    TRY(q5.alloc(lq + 1u));
    const BatchMPArray Q5{q5.p, lq + 1u, 1, lq + 1u};
    TRY(p_mul_small(ctx, pr, Q, 10005u, Q5, "10005*Q", sd));
    TRY(flags.alloc(spectrum_flag_words(1u, std::max(npl, lp + lq))));
    NP = BatchMPArray{nullptr, npl, 1, npl};
    TRY(np.alloc(npl));
    NP.data = np.p;
    BatchMPArray PQ{nullptr, lp + lq, 1, lp + lq};
    Buf pq;
    TRY(pq.alloc(PQ.stride));
    PQ.data = pq.p;
    TRY(stage(pr, "mul", "P*P+10005*Q*Q, P*Q", sd, 1, lp, lq, true, [&]() {
        TRY(fp.alloc(words));
        TRY(fq.alloc(words));
        TRY(fq5.alloc(words));
        spectrum_forward(tab, S, 1, P.data, P.stride, lp, fp.p, Q.data, Q.stride, lq, fq.p);
        spectrum_forward(tab, S, 1, Q5.data, Q5.stride, Q5.length, fq5.p, nullptr, 0, 0, nullptr);
        const uint32_t *x2[2] = {fp.p, fq5.p}, *y2[2] = {fp.p, fq.p};
        spectrum_inverse(tab, S, 1, 2, x2, y2, fq5.p, NP.data, NP.stride, NP.length, flags.p);
        const uint32_t *x1[1] = {fp.p}, *y1[1] = {fq.p};
        spectrum_inverse(tab, S, 1, 1, x1, y1, fp.p, PQ.data, PQ.stride, PQ.length, flags.p);
        return cudaGetLastError();
    }));
    TRY(p_compact(ctx, pr, NP, "P", sd));
    NQ = BatchMPArray{nullptr, PQ.length + 1u, 1, PQ.length + 1u};
    TRY(nq.alloc(NQ.stride));
    NQ.data = nq.p;
    TRY(p_shift(ctx, pr, PQ, NQ, 1, "2*P*Q", sd));
    return p_compact(ctx, pr, NQ, "Q", sd);
}

static cudaError_t sqrt_10005(BatchMPContext *ctx, Profiler *pr, int target, Buf &pbuf, BatchMPArray &P,
                              Buf &qbuf, BatchMPArray &Q, bool tuned) {
    cudaStream_t st = current_stream();
    TRY(pbuf.alloc(1));
    TRY(qbuf.alloc(1));
    const uint32_t p15 = 4001u, q15 = 40u;
    TRY(cudaMemcpyAsync(pbuf.p, &p15, 4, cudaMemcpyHostToDevice, st));
    TRY(cudaMemcpyAsync(qbuf.p, &q15, 4, cudaMemcpyHostToDevice, st));
    note_h2d(8);
    TRY(cudaStreamSynchronize(st));
    P = BatchMPArray{pbuf.p, 1, 1, 1};
    Q = BatchMPArray{qbuf.p, 1, 1, 1};
    double valid = 7.5;
    while (valid < (double)target) {
        valid *= 2;
        const uint32_t sd = (uint32_t)valid;
        Buf pq, nq, pp, qq, qq5, np;
        if (tuned) {
            BatchMPArray NP, NQ;
            bool done = false;
            TRY(sqrt_step_tuned(ctx, pr, sd, P, Q, np, NP, nq, NQ, &done));
            if (done) {
                pbuf.swap(np);
                qbuf.swap(nq);
                P = NP;
                Q = NQ;
                continue;
            }
        }
        BatchMPArray PQ{nullptr, P.length + Q.length, 1, P.length + Q.length};
        TRY(pq.alloc(PQ.stride));
        PQ.data = pq.p;
        TRY(p_mul(ctx, pr, P, Q, PQ, "P*Q", sd));
        TRY(p_compact(ctx, pr, PQ, "P*Q", sd));
        BatchMPArray NQ{nullptr, PQ.length + 1u, 1, PQ.length + 1u};
        TRY(nq.alloc(NQ.stride));
        NQ.data = nq.p;
        TRY(p_shift(ctx, pr, PQ, NQ, 1, "2*P*Q", sd));
        TRY(p_compact(ctx, pr, NQ, "Q", sd));
        BatchMPArray PP{nullptr, P.length * 2u, 1, P.length * 2u};
        TRY(pp.alloc(PP.stride));
        PP.data = pp.p;
        TRY(p_mul(ctx, pr, P, P, PP, "P*P", sd));
        TRY(p_compact(ctx, pr, PP, "P*P", sd));
        BatchMPArray QQ{nullptr, Q.length * 2u, 1, Q.length * 2u};
        TRY(qq.alloc(QQ.stride));
        QQ.data = qq.p;
        TRY(p_mul(ctx, pr, Q, Q, QQ, "Q*Q", sd));
        TRY(p_compact(ctx, pr, QQ, "Q*Q", sd));
        BatchMPArray Q5{nullptr, QQ.length + 1u, 1, QQ.length + 1u};
        TRY(qq5.alloc(Q5.stride));
        Q5.data = qq5.p;
        TRY(p_mul_small(ctx, pr, QQ, 10005u, Q5, "10005*Q*Q", sd));
        TRY(p_compact(ctx, pr, Q5, "10005*Q*Q", sd));
        const uint32_t npl = std::max(PP.length, Q5.length) + 1u;
        BatchMPArray NP{nullptr, npl, 1, npl};
        TRY(np.alloc(npl));
        NP.data = np.p;
        TRY(p_add(ctx, pr, PP, Q5, NP, "P*P+10005*Q*Q", sd));
        TRY(p_compact(ctx, pr, NP, "P", sd));
        pbuf.swap(np);
        qbuf.swap(nq);
        P = NP;
        Q = NQ;
    }
    return cudaSuccess;
}

// ---------------------------------------------------------------------------
// Exact host division for the inverse base case: (q, r) = divmod(2^e, v).
// Knuth, TAOCP vol. 2, 4.3.1 Algorithm D on 32-bit limbs.
// ---------------------------------------------------------------------------
static void divmod_pow2(uint32_t e, std::vector<uint32_t> v, std::vector<uint32_t> &q, std::vector<uint32_t> &r) {
    while (!v.empty() && v.back() == 0u) v.pop_back();
    const size_t n = v.size();
    std::vector<uint32_t> u(e / 32u + 2u, 0u);
    u[e / 32u] = 1u << (e % 32u);
    while (u.size() > 1 && u.back() == 0u) u.pop_back();
    if (n == 0) {
        q.clear();
        r.clear();
        return;
    }
    if (u.size() < n) {
        q.assign(1, 0u);
        r = u;
        return;
    }
    const size_t m = u.size() - n;
    q.assign(m + 1, 0u);
    if (n == 1) {
        uint64_t rem = 0;
        for (size_t j = u.size(); j-- > 0;) {
            const uint64_t cur = (rem << 32) | u[j];
            q[j] = (uint32_t)(cur / v[0]);
            rem = cur % v[0];
        }
        r.assign(1, (uint32_t)rem);
        while (q.size() > 1 && q.back() == 0u) q.pop_back();
        return;
    }
    const int s = __builtin_clz(v[n - 1]);
    std::vector<uint32_t> vn(n), un(u.size() + 1, 0u);
    for (size_t i = n - 1; i > 0; --i) vn[i] = (v[i] << s) | (s ? (uint32_t)((uint64_t)v[i - 1] >> (32 - s)) : 0u);
    vn[0] = v[0] << s;
    un[u.size()] = s ? (uint32_t)((uint64_t)u[u.size() - 1] >> (32 - s)) : 0u;
    for (size_t i = u.size() - 1; i > 0; --i) un[i] = (u[i] << s) | (s ? (uint32_t)((uint64_t)u[i - 1] >> (32 - s)) : 0u);
    un[0] = u[0] << s;
    for (size_t j = m + 1; j-- > 0;) {
        const uint64_t num = ((uint64_t)un[j + n] << 32) | un[j + n - 1];
        uint64_t qhat = num / vn[n - 1];
        uint64_t rhat = num % vn[n - 1];
        while (qhat >= (1ull << 32) || qhat * vn[n - 2] > ((rhat << 32) | un[j + n - 2])) {
            --qhat;
            rhat += vn[n - 1];
            if (rhat >= (1ull << 32)) break;
        }
        int64_t borrow = 0;
        uint64_t carry = 0;
        for (size_t i = 0; i < n; ++i) {
            const uint64_t prod = qhat * vn[i] + carry;
            carry = prod >> 32;
            const int64_t t = (int64_t)un[i + j] - (int64_t)(uint32_t)prod + borrow;
            un[i + j] = (uint32_t)t;
            borrow = t >> 32;
        }
        const int64_t t = (int64_t)un[j + n] - (int64_t)carry + borrow;
        un[j + n] = (uint32_t)t;
        if (t < 0) {
            --qhat;
            uint64_t c = 0;
            for (size_t i = 0; i < n; ++i) {
                const uint64_t sum = (uint64_t)un[i + j] + vn[i] + c;
                un[i + j] = (uint32_t)sum;
                c = sum >> 32;
            }
            un[j + n] += (uint32_t)c;
        }
        q[j] = (uint32_t)qhat;
    }
    r.assign(n, 0u);
    for (size_t i = 0; i < n; ++i)
        r[i] = (un[i] >> s) | (s ? (uint32_t)((uint64_t)un[i + 1] << (32 - s)) : 0u);
    while (q.size() > 1 && q.back() == 0u) q.pop_back();
    while (r.size() > 1 && r.back() == 0u) r.pop_back();
}

static BatchMPArray subview(const BatchMPArray &a, uint32_t start, uint32_t length) {
    // make_subview, pi_bs_gpu.cu:1095-1110
    if (start > a.length) start = a.length;
    const uint32_t maxl = a.length - start;
    if (length > maxl) length = maxl;
    const uint32_t stride = (a.stride >= start) ? (a.stride - start) : 0u;
    return BatchMPArray{a.data + start, length, a.batch_size, stride};
}

static cudaError_t shift_right_large(BatchMPContext *ctx, Profiler *pr, BatchMPArray A, uint64_t bits,
                                     BatchMPArray B, const char *label, uint32_t dg) {
    // pi_bs_gpu.cu:1068-1093
    const uint64_t limb_shift = bits / 32u;
    if (limb_shift >= A.length) return cudaErrorInvalidValue;
    const uint32_t ls = (uint32_t)limb_shift;
    BatchMPArray pre{A.data + ls, A.length - ls, A.batch_size, A.stride - ls};
    return p_shift(ctx, pr, pre, B, -(int32_t)(bits % 32u), label, dg);
}

// ---------------------------------------------------------------------------
// Recursive inverse y ~ 2^L / x (pi_bs_gpu.cu:1145-1344).
// y_out is allocated with x.length limbs; see the reference's python spec.
// ---------------------------------------------------------------------------
static const uint64_t kInverseCpuLimit = 32 * 1024;   // pi_bs_gpu.cu:1143

// The tuned form's Newton step shares y's forward transform between x2 y
// and res1m y (five transforms instead of six) when both products fit one
// shape at less cost than their own two: returns that shape, else M = 0.
static SpectrumShape newton_shared_shape(uint32_t lx2, uint32_t lres, uint32_t ly) {
    const uint64_t n1 = (uint64_t)lx2 + ly - 1u, n2 = (uint64_t)lres + ly - 1u;
    const SpectrumShape s1 = spectrum_shape(n1), s2 = spectrum_shape(n2), S = spectrum_shape(std::max(n1, n2));
    const uint32_t la[1] = {std::max(lx2, lres)}, lb[1] = {ly};
    if (s1.M == 0 || s2.M == 0 || S.M == 0 || !spectrum_sum_fits(la, lb, 1)) return SpectrumShape{0, 0};
    auto cap = [](SpectrumShape s) { return (uint64_t)s.M << s.log_k; };
    if (5u * cap(S) >= 3u * (cap(s1) + cap(s2))) return SpectrumShape{0, 0};
    return S;
}

static cudaError_t recursive_inverse(BatchMPContext *ctx, Profiler *pr, BatchMPArray x, uint64_t L, Buf &ybuf,
                                     BatchMPArray &y_out, uint32_t digits, bool tuned) {
    cudaStream_t st = current_stream();
    std::vector<uint64_t> levels{L};
    while (levels.back() > kInverseCpuLimit) {
        const uint64_t m = ((levels.back() - 2u) / 4u) & ~31ull;
        levels.push_back(levels.back() - m * 2u);
    }
    const size_t L_res = (L + 31) / 32 + 2;
    const size_t L_res2 = (L + 31) / 32 + 1;
    const size_t L_y2 = x.length + 1;
    TRY(ybuf.alloc(x.length));
    y_out = BatchMPArray{ybuf.p, x.length, 1, x.length};
    TRY(cudaMemsetAsync(ybuf.p, 0, (size_t)x.length * 4, st));
    Buf ws;
    TRY(ws.alloc(L_res + L_res2 + L_y2));
    uint32_t *res_base = ws.p;
    uint32_t *res2_base = ws.p + L_res;
    uint32_t *y2_base = res2_base + L_res2;
    TRY(cudaMemsetAsync(res_base, 0, L_res * 4, st));

    BatchMPArray res;
    {
        const uint64_t L0 = levels.back();
        const uint32_t start = (uint32_t)((L - L0) >> 6);
        BatchMPArray x0 = subview(x, start, x.length - start);
        BatchMPArray y0 = subview(y_out, start, y_out.length - start);
        res = BatchMPArray{res_base + start * 2u, x0.length + 1u, 1, x0.length + 1u};
        std::vector<uint32_t> hx(x0.length);
        if (x0.length)
            TRY(cudaMemcpyAsync(hx.data(), x0.data, (size_t)x0.length * 4, cudaMemcpyDeviceToHost, st));
        note_d2h((size_t)x0.length * 4);
        TRY(cudaStreamSynchronize(st));
        std::vector<uint32_t> hq, hr;
        divmod_pow2((uint32_t)L0, hx, hq, hr);
        // store_mpz_to_device writes the whole stride (pi_bs_gpu.cu:1121-1141)
        if (hq.size() > y0.stride || hr.size() > res.stride) return cudaErrorInvalidValue;
        hq.resize(y0.stride, 0u);
        hr.resize(res.stride, 0u);
        TRY(cudaMemcpyAsync(y0.data, hq.data(), (size_t)y0.stride * 4, cudaMemcpyHostToDevice, st));
        TRY(cudaMemcpyAsync(res.data, hr.data(), (size_t)res.stride * 4, cudaMemcpyHostToDevice, st));
        note_h2d((size_t)(y0.stride + res.stride) * 4);
        TRY(cudaStreamSynchronize(st));
    }
    TRY(res.compact(ctx));

    for (int i = (int)levels.size() - 1; i > 0; --i) {
        const uint64_t L1 = levels[i], L2 = levels[i - 1];
        const uint64_t m = (L2 - L1) >> 1;
        const uint32_t dg = (uint32_t)(L2 >> 5);
        BatchMPArray x2 = subview(x, (uint32_t)((L - L2) >> 6), (uint32_t)(m >> 5));
        BatchMPArray y1 = subview(y_out, (uint32_t)((L - L1) >> 6), y_out.length - (uint32_t)((L - L1) >> 6));
        BatchMPArray x2y1{res2_base, x2.length + y1.length, 1, x2.length + y1.length};
        BatchMPArray res1m{res.data - (uint32_t)(m >> 5), res.length + (uint32_t)(m >> 5) + 1u, 1,
                           res.length + (uint32_t)(m >> 5) + 1u};
        const SpectrumShape S =
            tuned ? newton_shared_shape(x2.length, res1m.length, y1.length) : SpectrumShape{0, 0};
        Buf fy, fz, flags;
        if (S.M) {
            const NTTPrecomputedTables &tab = context_tables(ctx);
            TRY(fy.alloc(spectrum_words(S, 1u)));
            TRY(fz.alloc(spectrum_words(S, 1u)));
            TRY(flags.alloc(spectrum_flag_words(1u, std::max(x2y1.length, res1m.length + y1.length))));
            TRY(stage(pr, "mul", "x2*y", dg, 1, x2.length, y1.length, true, [&]() {
                spectrum_forward(tab, S, 1, x2.data, x2.stride, x2.length, fz.p, y1.data, y1.stride, y1.length,
                                 fy.p);
                const uint32_t *xs[1] = {fz.p}, *ys[1] = {fy.p};
                spectrum_inverse(tab, S, 1, 1, xs, ys, fz.p, x2y1.data, x2y1.stride, x2y1.length, flags.p);
                return cudaGetLastError();
            }));
        } else {
            TRY(p_mul(ctx, pr, x2, y1, x2y1, "x2*y", dg));
        }
        TRY(p_sub(ctx, pr, res1m, x2y1, res1m, "res1_m", dg));
        uint32_t top = 0u;
        TRY(cudaMemcpyAsync(&top, res1m.data + res1m.length - 1, 4, cudaMemcpyDeviceToHost, st));
        note_d2h(4);
        TRY(cudaStreamSynchronize(st));
        const bool neg = top >= 0x80000000u;
        if (neg) {
            TRY(p_sub(ctx, pr, BatchMPArray{res1m.data, 0, 1, 0}, res1m, res1m, "res1_m_neg", dg));
        }
        BatchMPArray res2{res2_base, res1m.length + y1.length, 1, res1m.length + y1.length};
        if (S.M) {
            const NTTPrecomputedTables &tab = context_tables(ctx);
            TRY(stage(pr, "mul", "res2*y", dg, 1, res1m.length, y1.length, true, [&]() {
                spectrum_forward(tab, S, 1, res1m.data, res1m.stride, res1m.length, fz.p, nullptr, 0, 0, nullptr);
                const uint32_t *xs[1] = {fz.p}, *ys[1] = {fy.p};
                spectrum_inverse(tab, S, 1, 1, xs, ys, fz.p, res2.data, res2.stride, res2.length, flags.p);
                return cudaGetLastError();
            }));
            fy.reset();
            fz.reset();
        } else {
            TRY(p_mul(ctx, pr, res1m, y1, res2, "res2*y", dg));
        }
        const uint32_t y2len = res2.length - (uint32_t)((L2 - m * 2) >> 5);
        BatchMPArray y2{y2_base, y2len, 1, y2len};
        TRY(shift_right_large(ctx, pr, res2, L2 - m * 2u, y2, "y2", dg));
        if (neg) TRY(p_add_small(ctx, pr, y2, 1u, y2, "y2_inc", dg));
        BatchMPArray ynew = subview(y_out, (uint32_t)((L - L2) >> 6), y_out.length - (uint32_t)((L - L2) >> 6));
        if (!neg)
            TRY(p_add(ctx, pr, ynew, y2, ynew, "(y<<m)+y2", dg));
        else
            TRY(p_sub(ctx, pr, ynew, y2, ynew, "(y<<m)-y2", dg));
        if (L2 != L) {
            BatchMPArray xn = subview(x, (uint32_t)((L - L2) >> 6), x.length - (uint32_t)((L - L2) >> 6));
            res = BatchMPArray{res1m.data - (uint32_t)(m >> 5), res1m.length + (uint32_t)(m >> 5), 1,
                               res1m.length + (uint32_t)(m >> 5)};
            BatchMPArray y2x{res2_base, y2.length + xn.length, 1, y2.length + xn.length};
            TRY(p_mul(ctx, pr, y2, xn, y2x, "y2*x", dg));
            if (!neg)
                TRY(p_sub(ctx, pr, res, y2x, res, "(res<<m)-y2x", dg));
            else
                TRY(p_sub(ctx, pr, y2x, res, res, "y2x-(res<<m)", dg));
            TRY(res.compact(ctx));
        }
    }
    return cudaSuccess;
}

// ---------------------------------------------------------------------------
// pi_fractional (pi_bs_gpu.cu:1524-1685)
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Checkpoint of the splitting tree's result (Q and R of 17N terms, batch 1);
// the file format is checkpoint_file.h's.
// ---------------------------------------------------------------------------
// Lengths outside what a tree of size N can produce are rejected: Q and R
// hold at most 8 limbs per term (the 1e9-digit tree's hold about 3.5), and R
// must reach past the limbs that pi_fractional shifts away (15 * 17N - 8
// bits).
static bool ckpt_load(const char *path, uint32_t N, Buf &qb, BatchMPArray &Q, Buf &rb, BatchMPArray &R) {
    std::vector<uint32_t> q, r;
    const uint64_t max_limbs = 8ull * 17ull * N + 64ull;
    if (!ckpt_read(path, N, q, r, max_limbs)) return false;
    const uint32_t lq = (uint32_t)q.size(), lr = (uint32_t)r.size();
    const uint64_t rlimbs = (15ull * N * 17ull - 8ull) / 32ull;
    if ((uint64_t)lr <= rlimbs + 1ull) return false;
    cudaStream_t st = current_stream();
    if (qb.alloc(lq) != cudaSuccess || rb.alloc(lr) != cudaSuccess) return false;
    Q = BatchMPArray{qb.p, lq, 1, lq};
    R = BatchMPArray{rb.p, lr, 1, lr};
    const bool ok = cudaMemcpyAsync(Q.data, q.data(), (size_t)lq * 4, cudaMemcpyHostToDevice, st) == cudaSuccess &&
                    cudaMemcpyAsync(R.data, r.data(), (size_t)lr * 4, cudaMemcpyHostToDevice, st) == cudaSuccess &&
                    cudaStreamSynchronize(st) == cudaSuccess;
    note_h2d(((size_t)lq + lr) * 4);
    return ok;
}

static cudaError_t ckpt_save(const char *path, uint32_t N, const BatchMPArray &Q, const BatchMPArray &R) {
    cudaStream_t st = current_stream();
    std::vector<uint32_t> q(Q.length), r(R.length);
    TRY(cudaMemcpyAsync(q.data(), Q.data, (size_t)Q.length * 4, cudaMemcpyDeviceToHost, st));
    TRY(cudaMemcpyAsync(r.data(), R.data, (size_t)R.length * 4, cudaMemcpyDeviceToHost, st));
    TRY(cudaStreamSynchronize(st));
    note_d2h(((size_t)Q.length + R.length) * 4);
    return ckpt_write(path, N, q, r) ? cudaSuccess : cudaErrorInvalidValue;
}

static cudaError_t pi_fractional(BatchMPContext *ctx, Profiler *pr, int target, Buf &retbuf, BatchMPArray &RET,
                                 bool tuned, const char *ckpt, int *ckpt_state) {
    cudaStream_t st = current_stream();
    uint32_t N = 1;
    while (N * 17 * 14.3 < target) N *= 2;
    const int prec = (int)(((long)(target * 3.322) + 31) / 32 + 1);
    Buf qbs, rbs;
    BatchMPArray Qbs, Rbs;
    Buf p15b, q15b;
    BatchMPArray P15, Q15;
    bool have_sqrt = false;
    if (ckpt && ckpt_load(ckpt, N, qbs, Qbs, rbs, Rbs)) {
        *ckpt_state = 1;
    } else {
        TreeJoin tj;
        TRY(tree_start(ctx, pr, N, qbs, Qbs, rbs, Rbs, tuned, tj));
        if (tj.g && tuned) {
            // the tree's graph runs on its own stream; sqrt(10005), which
            // does not depend on it, runs meanwhile on this one (the same
            // operations and integers, the side context's workspace)
            BatchMPContext *side = side_context(ctx);
            if (side) {
                const cudaError_t e = sqrt_10005(side, pr, target, p15b, P15, q15b, Q15, tuned);
                if (e != cudaSuccess) {
                    tree_join(tj, qbs, Qbs, rbs, Rbs);
                    return e;
                }
                have_sqrt = true;
            }
        }
        TRY(tree_join(tj, qbs, Qbs, rbs, Rbs));
        if (ckpt) {
            // a file that cannot be written (unwritable directory, full
            // disk) does not fail the computation: state 3 reports it
            *ckpt_state = ckpt_save(ckpt, N, Qbs, Rbs) == cudaSuccess ? 2 : 3;
            cudaGetLastError();
        }
    }
    const long rts = 15l * N * 17 - 8;
    const int rbits = (int)(rts % 32), rlimbs = (int)(rts / 32);
    BatchMPArray Rpre{Rbs.data + rlimbs, Rbs.length - rlimbs, 1, Rbs.length - rlimbs};
    Buf rsb;
    TRY(rsb.alloc(Rpre.length + 1u));
    BatchMPArray Rs{rsb.p, Rpre.length + 1u, 1, Rpre.length + 1u};
    TRY(p_shift(ctx, pr, Rpre, Rs, -rbits, "R_shift", (uint32_t)target));
    rbs.reset();
    TRY(Rs.compact(ctx));
    long extra = std::max(0l, std::min((long)Qbs.length, (long)Rs.length) - prec);
    BatchMPArray Qt{Qbs.data + extra, Qbs.length - (uint32_t)extra, 1, Qbs.length - (uint32_t)extra};
    BatchMPArray Rt{Rs.data + extra, Rs.length - (uint32_t)extra, 1, Rs.length - (uint32_t)extra};
    if (!have_sqrt) TRY(sqrt_10005(ctx, pr, target, p15b, P15, q15b, Q15, tuned));
    Buf pfb, qfb;
    BatchMPArray Pf{nullptr, P15.length + Qt.length, 1, P15.length + Qt.length};
    BatchMPArray Qf{nullptr, Q15.length + Rt.length, 1, Q15.length + Rt.length};
    TRY(pfb.alloc(Pf.stride));
    TRY(qfb.alloc(Qf.stride));
    Pf.data = pfb.p;
    Qf.data = qfb.p;
    TRY(p_mul(ctx, pr, P15, Qt, Pf, "P15*Q", (uint32_t)target));
    TRY(p_mul(ctx, pr, Rt, Q15, Qf, "R*Q15", (uint32_t)target));
    TRY(p_compact(ctx, pr, Pf, "P", (uint32_t)target));
    TRY(p_compact(ctx, pr, Qf, "Q", (uint32_t)target));
    qbs.reset();
    rsb.reset();
    p15b.reset();
    q15b.reset();
    extra = std::max(0l, std::min((long)Pf.length, (long)Qf.length) - prec);
    BatchMPArray Ptf = subview(Pf, (uint32_t)extra, Pf.length - (uint32_t)extra);
    BatchMPArray Qtf = subview(Qf, (uint32_t)extra, Qf.length - (uint32_t)extra);
    TRY(Qtf.compact(ctx));
    uint32_t qbits = 0u;
    if (Qtf.length > 0u) {
        uint32_t topl = 0u;
        TRY(cudaMemcpyAsync(&topl, Qtf.data + Qtf.length - 1, 4, cudaMemcpyDeviceToHost, st));
        note_d2h(4);
        TRY(cudaStreamSynchronize(st));
        qbits = (Qtf.length - 1u) * 32u + (topl ? 32u - (uint32_t)__builtin_clz(topl) : 0u);
    }
    const uint64_t inv_bits = (uint64_t)qbits * 2u - 1u;
    Buf invb;
    BatchMPArray inv;
    TRY(recursive_inverse(ctx, pr, Qtf, inv_bits, invb, inv, (uint32_t)target, tuned));
    qfb.reset();
    Buf rpb;
    BatchMPArray RP{nullptr, Ptf.length + inv.length, 1, Ptf.length + inv.length};
    TRY(rpb.alloc(RP.stride));
    RP.data = rpb.p;
    TRY(p_mul(ctx, pr, Ptf, inv, RP, "P*invQ", (uint32_t)target));
    TRY(p_compact(ctx, pr, RP, "P*invQ", (uint32_t)target));
    pfb.reset();
    invb.reset();
    const uint32_t retlen = RP.length - (uint32_t)(inv_bits / 32u) + (uint32_t)prec;
    TRY(retbuf.alloc(retlen));
    RET = BatchMPArray{retbuf.p, retlen, 1, retlen};
    const uint64_t fshift = inv_bits - (uint64_t)prec * 32u;
    TRY(shift_right_large(ctx, pr, RP, fshift, RET, "RET_shift", (uint32_t)target));
    TRY(p_compact(ctx, pr, RET, "RET", (uint32_t)target));
    return cudaSuccess;
}

}  // namespace gpupi

// ---------------------------------------------------------------------------
// Public driver
// ---------------------------------------------------------------------------
namespace gpupi {

uint32_t round_up_decimal_digits(uint32_t requested, uint32_t *leaf_out) {
    // pi_bs_gpu.cu:924-939
    if (requested == 0u) {
        *leaf_out = 0u;
        return 0u;
    }
    uint32_t digits = requested, levels = 0u;
    while (digits >= 32u * 18u) {
        digits >>= 1;
        ++levels;
    }
    if ((digits << levels) < requested) ++digits;
    *leaf_out = digits;
    return digits << levels;
}

constexpr uint32_t kMaxDigits = 1290000000u;   // digits * 3.322 + 31 < 2^32

// Digits [0, total) of d_digits to sink in chunks: the copy of chunk i + 1
// into one pinned buffer runs while the sink consumes chunk i from the other.
static cudaError_t stream_digits(const char *d_digits, size_t total, const PiRequest &req, float *host_ms) {
    const auto t0 = std::chrono::steady_clock::now();
    const size_t chunk = std::max<size_t>(req.sink_chunk, 4096u);
    char *h[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaStream_t cs = nullptr;
    cudaError_t err = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    for (int i = 0; i < 2 && err == cudaSuccess; ++i) {
        err = cudaHostAlloc((void **)&h[i], std::min(chunk, std::max<size_t>(total, 1u)), cudaHostAllocDefault);
        if (err == cudaSuccess) err = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
    }
    auto issue = [&](size_t k) {
        const size_t off = k * chunk, n = std::min(chunk, total - off);
        cudaError_t e = cudaMemcpyAsync(h[k & 1], d_digits + off, n, cudaMemcpyDeviceToHost, cs);
        note_d2h(n);
        if (e == cudaSuccess) e = cudaEventRecord(ev[k & 1], cs);
        return e;
    };
    const size_t chunks = (total + chunk - 1) / chunk;
    if (err == cudaSuccess && chunks) err = issue(0);
    for (size_t k = 0; k < chunks && err == cudaSuccess; ++k) {
        if (k + 1 < chunks) err = issue(k + 1);   // its buffer's previous chunk was consumed at k - 1
        if (err == cudaSuccess) err = cudaEventSynchronize(ev[k & 1]);
        const size_t n = std::min(chunk, total - k * chunk);
        if (err == cudaSuccess && !req.sink(h[k & 1], n, req.sink_user)) break;
    }
    if (cs) {
        cudaStreamSynchronize(cs);
        cudaStreamDestroy(cs);
    }
    for (int i = 0; i < 2; ++i) {
        if (h[i]) cudaFreeHost(h[i]);
        if (ev[i]) cudaEventDestroy(ev[i]);
    }
    *host_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return err;
}

// Host copies of the digits while they are converted: the conversion runs
// in parts (convert_decimal_in_parts) and each part's digits go to the
// caller's buffer on a copy stream once the part is done.  A part's copy is
// issued when the next part has been issued, so that a copy into pageable
// memory (which returns only when done) never keeps the GPU waiting.
struct DigitCopies {
    cudaStream_t st = nullptr, copy = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    const char *src = nullptr;
    char *dst = nullptr;
    size_t want = 0, pend_off = 0, pend_n = 0;
    int parts = 0;
    bool pending = false;
    cudaError_t err = cudaSuccess;

    cudaError_t open(cudaStream_t s) {
        st = s;
        cudaError_t e = cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking);
        for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
        return e;
    }
    void issue_pending() {
        if (!pending || err != cudaSuccess) return;
        pending = false;
        if (pend_off >= want) return;
        const size_t n = std::min(pend_n, want - pend_off);
        err = cudaStreamWaitEvent(copy, ev[(parts - 1) & 1], 0);
        if (err == cudaSuccess) err = cudaMemcpyAsync(dst + pend_off, src + pend_off, n, cudaMemcpyDeviceToHost, copy);
        note_d2h(n);
    }
    static void ready(size_t off, size_t n, void *user) {
        DigitCopies &d = *static_cast<DigitCopies *>(user);
        if (d.err != cudaSuccess) return;
        d.err = cudaEventRecord(d.ev[d.parts & 1], d.st);   // this part's digits are issued before it
        d.issue_pending();                                   // the previous part's copy
        ++d.parts;
        d.pend_off = off;
        d.pend_n = n;
        d.pending = true;
    }
    void drain() {   // wait for the copies issued so far (error paths)
        if (copy) cudaStreamSynchronize(copy);
    }
    cudaError_t finish() {   // the last part's copy, then wait for all
        issue_pending();
        if (copy) {
            const cudaError_t e = cudaStreamSynchronize(copy);
            if (err == cudaSuccess) err = e;
        }
        return err;
    }
    ~DigitCopies() {
        if (copy) {
            cudaStreamSynchronize(copy);
            cudaStreamDestroy(copy);
        }
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
    }
};

// Parts of the conversion (2^3) when at least this many digits go to the host.
constexpr uint32_t kCopyPartsMinDigits = 1u << 24;
constexpr uint32_t kLogCopyParts = 3;

uint32_t prec_limbs_for_digits(uint32_t digits) {
    const uint32_t bits = (uint32_t)((double)digits * 3.322) + 31u;   // pi_bs_gpu.cu:941-944
    return bits / 32u + 1u;
}

cudaError_t pi_run(const PiRequest &req, PiOutput &out) {
    out = PiOutput{};
    const uint32_t requested = req.digits;
    uint32_t leaf = 0u;
    const uint32_t convert = round_up_decimal_digits(requested, &leaf);
    // round_up_decimal_digits leaves the reference's global leaf size (477)
    // untouched when nothing is requested (pi_bs_gpu.cu:155, 924-928)
    if (leaf == 0u) leaf = 477u;
    const uint32_t prec = prec_limbs_for_digits(requested);
    out.target_digits = requested;
    out.convert_digits = convert;
    if (requested > 0u && convert == 0u) return cudaErrorInvalidValue;
    // The working precision in bits (digits * 3.322 + 31, pi_bs_gpu.cu:941-944)
    // is a 32-bit count.  Up to 1.011e9 digits the splitting tree has 2^22 x
    // 17 terms and its products stay below the reference's 2^28-limb NTT
    // ceiling; above that the tree doubles and its top products (about 5.5e8
    // limbs) need this library's 20-coset transforms.
    if (requested > kMaxDigits) return cudaErrorInvalidValue;
    BatchMPContext *ctx = req.ctx;
    bool own_ctx = false;
    if (!ctx) {
        ctx = batch_mp_init();
        own_ctx = true;
        if (!ctx) return cudaErrorMemoryAllocation;
    }
    cudaStream_t st = current_stream();
    {
        // keep freed blocks in the stream-ordered pool across synchronisations
        int dev = 0;
        cudaMemPool_t pool;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    Profiler prof;
    prof.on = req.profile_stages;
    const uint32_t levels = convert ? (uint32_t)__builtin_ctz(convert / leaf) : 0u;
    // The timed region starts here, before any allocation, as the
    // reference's does (its workspace and buffers are allocated inside it).
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaError_t err = cudaEventRecord(e0, st);
    // Size the multiply workspace once for the largest product (P * invQ, two
    // operands of about prec_limbs limbs) so that no level regrows it, and
    // the scratch arena for every level's temporaries (high-water marks of
    // 16 B per digit for the plain form and up to 32 B per digit for the
    // tuned form's spectra, at 3e8 digits; the margin absorbs fragmentation,
    // and a request that still misses spills to the pool).
    if (err == cudaSuccess)
        err = batch_mp_ensure_workspace(ctx, batch_mul_ntt_workspace_size(1u, prec + 8u, prec + 8u));
    if (err == cudaSuccess)
        scratch_reserve((size_t)requested * (req.plain ? 21u : 40u) + ((size_t)64 << 20));
    Buf retb;
    BatchMPArray RET{};
    ConvertDecimalPowerTable powers{};
    char *d_digits = nullptr;
    if (err == cudaSuccess)
        err = pi_fractional(ctx, &prof, (int)requested, retb, RET, !req.plain, req.checkpoint, &out.checkpoint);
    // RET into the caller's buffer on a side stream, overlapping the decimal
    // conversion (which only reads RET)
    cudaStream_t side = nullptr;
    cudaEvent_t ret_ready = nullptr;
    if (err == cudaSuccess && !req.device_only && req.host_ret && RET.length) {
        const size_t n = std::min<size_t>(req.host_ret_cap, RET.length);
        err = cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking);
        if (err == cudaSuccess) err = cudaEventCreateWithFlags(&ret_ready, cudaEventDisableTiming);
        if (err == cudaSuccess) err = cudaEventRecord(ret_ready, st);
        if (err == cudaSuccess) err = cudaStreamWaitEvent(side, ret_ready, 0);
        if (err == cudaSuccess && n) {
            err = cudaMemcpyAsync(req.host_ret, RET.data, n * 4, cudaMemcpyDeviceToHost, side);
            note_d2h(n * 4);
        }
    }
    if (err == cudaSuccess) {
        err = stage(&prof, "decimal_powers", "precompute_5pow", levels == 0u ? leaf : (leaf << levels), 1u, levels,
                    leaf, false, [&]() { return convert_decimal_precompute_powers(ctx, &powers, leaf, levels); });
    }
    // digits for the host: copied part by part while the rest converts
    const uint32_t want = req.device_only ? 0u : std::min(requested, req.copy_digits);
    char *dst = req.host_digits;
    if (want > 0u && !dst) {
        out.digits.resize(want);
        dst = &out.digits[0];
    }
    const bool in_parts = want >= kCopyPartsMinDigits && !req.profile_stages;
    DigitCopies copies;
    if (err == cudaSuccess && requested > 0u) {
        err = scratch_alloc((void **)&d_digits, convert);
        if (err == cudaSuccess && in_parts) {
            err = copies.open(st);
            copies.src = d_digits;
            copies.dst = dst;
            copies.want = want;
        }
        if (err == cudaSuccess) {
            BatchMPArray frac = subview(RET, 0u, std::min<uint32_t>(prec, RET.length));
            err = stage(&prof, "decimal_convert", "equal_split", convert, frac.batch_size, frac.length, leaf, false,
                        [&]() {
                            if (in_parts)
                                return convert_decimal_in_parts(ctx, frac, prec * 32u, convert, leaf, &powers,
                                                                d_digits, kLogCopyParts, DigitCopies::ready, &copies);
                            return convert_decimal_equal_split(ctx, frac, prec * 32u, convert, leaf, &powers,
                                                               d_digits);
                        });
        }
    }
    if (err == cudaSuccess) err = cudaEventRecord(e1, st);
    if (err == cudaSuccess) err = cudaEventSynchronize(e1);
    if (err == cudaSuccess) err = cudaEventElapsedTime(&out.elapsed_ms, e0, e1);
    out.ret_len = RET.length;
    out.workspace_bytes = batch_mp_workspace_size(ctx);
    if (err == cudaSuccess && !req.device_only) {
        if (!req.host_ret) out.ret.resize(RET.length);
        if (RET.length && !req.host_ret) {
            err = cudaMemcpyAsync(out.ret.data(), RET.data, (size_t)RET.length * 4, cudaMemcpyDeviceToHost, st);
            note_d2h((size_t)RET.length * 4);
        }
        if (err == cudaSuccess && want > 0u && in_parts) err = copies.finish();
        if (err == cudaSuccess && want > 0u && !in_parts) {
            err = cudaMemcpyAsync(dst, d_digits, want, cudaMemcpyDeviceToHost, st);
            note_d2h(want);
        }
        if (err == cudaSuccess && req.copy_digits < requested && requested > 0u) {
            // tail for the --benchmark preview
            const uint32_t tail = std::min<uint32_t>(requested, 64u);
            out.tail.resize(tail);
            err = cudaMemcpyAsync(&out.tail[0], d_digits + (requested - tail), tail, cudaMemcpyDeviceToHost, st);
        }
        if (err == cudaSuccess) err = cudaStreamSynchronize(st);
        if (err == cudaSuccess && req.sink && requested > 0u)
            err = stream_digits(d_digits, requested, req, &out.output_ms);
    }
    if (side) {
        const cudaError_t serr = cudaStreamSynchronize(side);
        if (err == cudaSuccess) err = serr;
        cudaStreamDestroy(side);
    }
    if (ret_ready) cudaEventDestroy(ret_ready);
    out.stages = prof.entries;
    copies.drain();
    scratch_free(d_digits);
    convert_decimal_release_powers(&powers);
    retb.reset();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamSynchronize(st);
    if (own_ctx) batch_mp_destroy(ctx);
    return err;
}

}  // namespace gpupi
