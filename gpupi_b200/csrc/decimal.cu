// Binary -> decimal conversion (gpupi convert_decimal.cu, batch_decimal_naive.cu).
//
// Leaf (batch_decimal_naive.cu:16-217): a fraction X / 2^(32L) yields its
// truncated decimal digits 9 at a time: X *= 10^9, the limb that overflows
// the top is the next 9-digit chunk.  Here a row is first placed at the top of
// a fixed-size register array (MAXL limbs, zeros below), so every index is a
// compile-time constant; one thread converts one row.  Rows longer than 64
// limbs use one warp per row, where each x10^9 round is a binary-carry add of
// lo(a_j*10^9) and hi(a_(j-1)*10^9) resolved with ballots.
//
// Divide and conquer (convert_decimal.cu:198-474), per level on every row:
//   high child = top child_bits of X
//   low child  = top child_bits of (X mod 2^(B-d)) * 5^d      (d = child digits)
// with 5^d broadcast to all rows (stride 0) so its transform is computed once.
// The reference's digit semantics (truncating fixed-point splits, 34 margin
// bits) are reproduced exactly; output is natural order.
#include "common.cuh"
#include "batch_arith.h"
#include "batch_decimal_naive.h"
#include "batch_shift.h"
#include "convert_decimal.h"
#include "pi_engine.h"

#include <math.h>
#include <new>
#include <vector>

namespace gpupi {

constexpr uint32_t kTen9 = 1000000000u;

// out(pos) for the digit of place 10^-k (k = 1..L_dec):
//   LSD-first layout (API): pos = L_dec - k;  natural layout: pos = k - 1.
//
// One thread per row; the CTA's 128 rows write their digits through shared
// memory, eight 9-digit rounds (72 places) at a time: the CTA then stores
// each row's 72-place run with consecutive threads on consecutive bytes,
// instead of every thread storing single bytes one row apart (one sector
// per lane per store).  The whole CTA runs every round (barriers); rows past
// N compute nothing and store nothing.
constexpr int kDecRows = 128;
constexpr int kDecRounds = 8;
constexpr int kDecSpan = 9 * kDecRounds;   // places per flush

template <int MAXL, bool NATURAL>
__global__ void __launch_bounds__(kDecRows) k_decimal_thread(const uint32_t *__restrict__ A,
                                                             char *__restrict__ B, uint32_t N,
                                                             uint32_t L, uint64_t sA, uint32_t L_dec,
                                                             uint64_t sB) {
    __shared__ char stage[kDecRows][kDecSpan + 1];
    const uint32_t t = threadIdx.x;
    for (uint64_t row0 = (uint64_t)blockIdx.x * kDecRows; row0 < N; row0 += (uint64_t)gridDim.x * kDecRows) {
        const uint64_t row = row0 + t;
        const bool valid = row < N;
        const uint32_t rows = (N - row0 < (uint64_t)kDecRows) ? (uint32_t)(N - row0) : (uint32_t)kDecRows;
        uint32_t x[MAXL];
        const uint32_t *ar = A + row * sA;
        const uint32_t pad = MAXL - L;
#pragma unroll
        for (int i = 0; i < MAXL; ++i) x[i] = (valid && (uint32_t)i >= pad) ? ar[i - pad] : 0u;
        for (uint32_t start = 0; start < L_dec; start += kDecSpan) {
            const uint32_t span = min((uint32_t)kDecSpan, L_dec - start);
            for (uint32_t r = 0; r * 9u < span; ++r) {
                uint32_t carry = 0u;
#pragma unroll
                for (int i = 0; i < MAXL; ++i) {
                    const uint64_t v = (uint64_t)x[i] * kTen9 + carry;
                    x[i] = (uint32_t)v;
                    carry = (uint32_t)(v >> 32);
                }
                // carry = the next 9 digits (places start + 9r + 1 .. + 9)
                const uint32_t cnt = min(9u, span - r * 9u);
                uint32_t v = carry;
                for (uint32_t m = 9; m > cnt; --m) v /= 10u;   // drop places beyond L_dec
                for (uint32_t m = cnt; m >= 1; --m) {
                    stage[t][r * 9u + m - 1u] = (char)('0' + v % 10u);
                    v /= 10u;
                }
            }
            __syncthreads();
            // places start + 1 .. start + span of rows row0 .. row0 + rows - 1;
            // w / span as (w * ceil(2^32 / span)) >> 32, exact for w < 2^14
            const uint64_t magic = (0x100000000ull + span - 1u) / span;
            for (uint32_t w = t; w < rows * span; w += kDecRows) {
                const uint32_t rr = (uint32_t)(((uint64_t)w * magic) >> 32);
                const uint32_t j = w - rr * span;
                const uint32_t k = start + j + 1u;   // place 10^-k
                B[(row0 + rr) * sB + (NATURAL ? (k - 1u) : (L_dec - k))] = stage[rr][j];
            }
            __syncthreads();
        }
    }
}

// Warp per row, L <= 32*G limbs.
template <int G, bool NATURAL>
__global__ void __launch_bounds__(128) k_decimal_warp(const uint32_t *__restrict__ A,
                                                      char *__restrict__ B, uint32_t N, uint32_t L,
                                                      uint64_t sA, uint32_t L_dec, uint64_t sB) {
    const uint32_t lane = lane_id();
    const uint32_t wpc = blockDim.x >> 5;
    for (uint32_t row = blockIdx.x * wpc + (threadIdx.x >> 5); row < N; row += gridDim.x * wpc) {
        const uint32_t *ar = A + row * sA;
        const uint32_t pad = 32u * G - L;
        uint32_t x[G];
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const uint32_t i = g * 32u + lane;
            x[g] = (i >= pad) ? ar[i - pad] : 0u;
        }
        char *out = B + row * sB;
        for (uint32_t start = 0; start < L_dec; start += 9u) {
            uint32_t cin = 0u;
            uint32_t prev_hi = 0u;   // hi(x[lane-1 of flattened]*1e9) for lane 0 of group g
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const uint64_t t = (uint64_t)x[g] * kTen9;
                const uint32_t lo = (uint32_t)t;
                const uint32_t hi = (uint32_t)(t >> 32);
                uint32_t y = __shfl_up_sync(0xffffffffu, hi, 1);
                if (lane == 0) y = prev_hi;
                prev_hi = __shfl_sync(0xffffffffu, hi, 31);
                bool gg, pp;
                const uint32_t s = raw_limb<false>(lo, y, gg, pp);
                const uint32_t gm = __ballot_sync(0xffffffffu, gg);
                const uint32_t pm = __ballot_sync(0xffffffffu, pp);
                const GroupCarry gc = resolve_group(gm, pm, cin);
                cin = gc.carry_out;
                x[g] = s + ((gc.carry_in_mask >> lane) & 1u);
            }
            const uint32_t chunk = prev_hi + cin;   // overflow out of the top limb
            const uint32_t cnt = min(9u, L_dec - start);
            if (lane < cnt) {
                // lane m-1 writes place start+m
                const uint32_t m = lane + 1u;
                uint32_t v = chunk;
                for (uint32_t e = 9; e > m; --e) v /= 10u;
                const uint32_t k = start + m;
                out[NATURAL ? (k - 1u) : (L_dec - k)] = (char)('0' + v % 10u);
            }
        }
    }
}

template <bool NATURAL>
void decimal_rows(const uint32_t *A, char *B, uint32_t N, uint32_t L, uint64_t sA, uint32_t L_dec,
                  uint64_t sB) {
    if (N == 0u || L == 0u || L_dec == 0u) return;
    cudaStream_t st = current_stream();
    KernelTimed kt("decimal_leaf", 4.0 * N * L + (double)N * L_dec);
    const unsigned gt = grid_for(N, 128, kNumSMs * 32);
    const unsigned gw = grid_for(N, 4, kNumSMs * 32);
    if (L <= 8u) k_decimal_thread<8, NATURAL><<<gt, 128, 0, st>>>(A, B, N, L, sA, L_dec, sB);
    else if (L <= 16u) k_decimal_thread<16, NATURAL><<<gt, 128, 0, st>>>(A, B, N, L, sA, L_dec, sB);
    else if (L <= 32u) k_decimal_thread<32, NATURAL><<<gt, 128, 0, st>>>(A, B, N, L, sA, L_dec, sB);
    else if (L <= 64u) k_decimal_thread<64, NATURAL><<<gt, 128, 0, st>>>(A, B, N, L, sA, L_dec, sB);
    else if (L <= 256u) k_decimal_warp<8, NATURAL><<<gw, 128, 0, st>>>(A, B, N, L, sA, L_dec, sB);
    else if (L <= 1024u) k_decimal_warp<32, NATURAL><<<gw, 128, 0, st>>>(A, B, N, L, sA, L_dec, sB);
    else k_decimal_warp<64, NATURAL><<<gw, 128, 0, st>>>(A, B, N, L, sA, L_dec, sB);
    count_launch();
}

// dst row (2*row + off) limb j = bits [shift + 32j, shift + 32j + 32) of src row.
__global__ void k_extract_shifted(const uint32_t *__restrict__ src, uint64_t s_stride, uint32_t s_len,
                                  uint32_t *__restrict__ dst, uint64_t d_stride, uint32_t d_len,
                                  uint32_t rows, uint32_t shift, uint32_t off) {
    const uint64_t total = (uint64_t)rows * d_len;
    const uint32_t w = shift >> 5, b = shift & 31u;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t row = (uint32_t)(t / d_len);
        const uint32_t j = (uint32_t)(t - (uint64_t)row * d_len);
        const uint32_t *s = src + row * s_stride;
        const uint32_t i = j + w;
        uint32_t v = 0u;
        if (i < s_len) {
            v = s[i] >> b;
            if (b != 0u && i + 1u < s_len) v |= s[i + 1u] << (32u - b);
        }
        dst[(uint64_t)(2u * row + off) * d_stride + j] = v;
    }
}

// dst limb j = src limb j for j < d_len, top limb masked to `top_mask`.
__global__ void k_extract_low(const uint32_t *__restrict__ src, uint64_t s_stride,
                              uint32_t *__restrict__ dst, uint64_t d_stride, uint32_t d_len,
                              uint32_t rows, uint32_t top_mask) {
    const uint64_t total = (uint64_t)rows * d_len;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t row = (uint32_t)(t / d_len);
        const uint32_t j = (uint32_t)(t - (uint64_t)row * d_len);
        uint32_t v = src[row * s_stride + j];
        if (j + 1u == d_len) v &= top_mask;
        dst[row * d_stride + j] = v;
    }
}

static void extract_shifted(const BatchMPArray &src, uint32_t *dst, uint32_t d_stride,
                            uint32_t d_len, uint32_t rows, uint32_t shift, uint32_t off) {
    if (d_len == 0u || rows == 0u) return;
    const uint64_t total = (uint64_t)rows * d_len;
    KernelTimed kt("decimal_extract", 8.0 * (double)total);
    k_extract_shifted<<<grid_for(total, 256, kNumSMs * 32), 256, 0, current_stream()>>>(
        src.data, src.stride, src.length, dst, d_stride, d_len, rows, shift, off);
    count_launch();
}

static void extract_low(const BatchMPArray &src, uint32_t *dst, uint32_t d_stride, uint32_t d_len,
                        uint32_t rows, uint32_t valid_bits) {
    if (d_len == 0u || rows == 0u) return;
    uint32_t mask = 0xffffffffu;
    if (valid_bits & 31u) mask = (1u << (valid_bits & 31u)) - 1u;
    const uint64_t total = (uint64_t)rows * d_len;
    KernelTimed kt("decimal_extract", 8.0 * (double)total);
    k_extract_low<<<grid_for(total, 256, kNumSMs * 32), 256, 0, current_stream()>>>(
        src.data, src.stride, dst, d_stride, d_len, rows, mask);
    count_launch();
}

constexpr double kLog2_10 = 3.32192809488736234787;   // convert_decimal.cu:15
constexpr uint32_t kMarginBits = 34u;                 // convert_decimal.cu:16

static uint32_t bits_for_digits(uint32_t digits) {
    return (uint32_t)(ceil((double)digits * kLog2_10) + (double)kMarginBits);
}

static uint32_t levels_for_shape(uint32_t total, uint32_t leaf) {
    if (leaf == 0u || total == 0u || total % leaf != 0u) return UINT32_MAX;
    uint32_t ratio = total / leaf, levels = 0u;
    while (ratio > 1u && (ratio & 1u) == 0u) {
        ratio >>= 1;
        ++levels;
    }
    return ratio == 1u ? levels : UINT32_MAX;
}

// 5^e as little-endian limbs (host).
static std::vector<uint32_t> pow5(uint32_t e) {
    std::vector<uint32_t> v(1, 1u);
    for (uint32_t i = 0; i < e; ++i) {
        uint64_t c = 0;
        for (auto &w : v) {
            const uint64_t t = (uint64_t)w * 5u + c;
            w = (uint32_t)t;
            c = t >> 32;
        }
        if (c) v.push_back((uint32_t)c);
    }
    return v;
}

// Scratch buffer from the stream's arena (no synchronisation on free).
struct DevBuf {
    uint32_t *p = nullptr;
    ~DevBuf() { scratch_free(p); }
    cudaError_t alloc(size_t words) {
        scratch_free(p);
        p = nullptr;
        return words ? scratch_alloc((void **)&p, words * 4) : cudaSuccess;
    }
};

// One row of the power table, from the stream's arena.
BatchMPArray power_array(uint32_t length) {
    BatchMPArray a{nullptr, length, 1u, length};
    if (length && scratch_alloc((void **)&a.data, (size_t)length * 4) != cudaSuccess) a = BatchMPArray{};
    return a;
}
void power_release(BatchMPArray &a) {
    scratch_free(a.data);
    a = BatchMPArray{};
}

}  // namespace gpupi

using namespace gpupi;

void batch_decimal_naive(const uint32_t *A, char *B, uint32_t N, int L_limb, uint32_t stride_A,
                         int L_dec, uint32_t stride_B) {
    if (N == 0u || L_limb <= 0 || L_dec <= 0 || L_limb > BATCH_DECIMAL_NAIVE_L_LIMB_MAX) return;
    decimal_rows<false>(A, B, N, (uint32_t)L_limb, stride_A, (uint32_t)L_dec, stride_B);
}

cudaError_t convert_decimal_precompute_powers(BatchMPContext *ctx, ConvertDecimalPowerTable *table,
                                              uint32_t leaf_digits, uint32_t levels) {
    if (ctx == nullptr || table == nullptr || leaf_digits == 0u) return cudaErrorInvalidValue;
    table->powers = nullptr;
    table->levels = 0u;
    table->leaf_digits = leaf_digits;
    if (levels == 0u) return cudaSuccess;
    BatchMPArray *powers = new (std::nothrow) BatchMPArray[levels];
    if (powers == nullptr) return cudaErrorMemoryAllocation;
    for (uint32_t i = 0; i < levels; ++i) powers[i] = BatchMPArray{};
    auto fail = [&](uint32_t made, cudaError_t e) {
        for (uint32_t i = 0; i < made; ++i) power_release(powers[i]);
        delete[] powers;
        return e;
    };
    const std::vector<uint32_t> base = pow5(leaf_digits);
    powers[0] = power_array((uint32_t)base.size());
    if (powers[0].data == nullptr) return fail(0, cudaErrorMemoryAllocation);
    cudaError_t err = cudaMemcpyAsync(powers[0].data, base.data(), base.size() * 4,
                                      cudaMemcpyHostToDevice, current_stream());
    note_h2d(base.size() * 4);
    if (err == cudaSuccess) err = cudaStreamSynchronize(current_stream());
    if (err != cudaSuccess) return fail(1, err);
    for (uint32_t l = 1; l < levels; ++l) {
        BatchMPArray next = power_array(powers[l - 1].length * 2u);
        if (next.data == nullptr) return fail(l, cudaErrorMemoryAllocation);
        err = mul_tuned(ctx, powers[l - 1], powers[l - 1], next);
        if (err == cudaSuccess) err = next.compact(ctx);
        if (err != cudaSuccess) {
            power_release(next);
            return fail(l, err);
        }
        powers[l] = next;
    }
    table->powers = powers;
    table->levels = levels;
    return cudaSuccess;
}

void convert_decimal_release_powers(ConvertDecimalPowerTable *table) {
    if (table == nullptr) return;
    if (table->powers != nullptr) {
        for (uint32_t i = 0; i < table->levels; ++i) power_release(table->powers[i]);
        delete[] table->powers;
    }
    table->powers = nullptr;
    table->levels = 0u;
}

namespace gpupi {

// Level sizes of one conversion (convert_decimal.cu:285-330): digits, bits
// and limbs of a row at each level.
struct ConvertPlan {
    uint32_t levels;
    std::vector<uint32_t> digs, bits, limbs;
};

static ConvertPlan convert_plan(uint32_t levels, uint32_t total_digits, uint32_t input_bits, uint32_t input_len) {
    ConvertPlan p{levels, std::vector<uint32_t>(levels + 1), std::vector<uint32_t>(levels + 1),
                  std::vector<uint32_t>(levels + 1)};
    p.digs[0] = total_digits;
    p.bits[0] = input_bits;
    p.limbs[0] = input_len;
    for (uint32_t l = 1; l <= levels; ++l) {
        p.digs[l] = p.digs[l - 1] >> 1;
        p.bits[l] = bits_for_digits(p.digs[l]);
        p.limbs[l] = (p.bits[l] + 31u) / 32u;
    }
    return p;
}

// Buffers of levels [l0, l1) for `rows0` rows at level l0: two row sets
// (ping / pong), the mantissas and the products.
struct LevelBufs {
    DevBuf ping, pong, mant, prod;
    cudaError_t alloc(const ConvertPlan &p, const ConvertDecimalPowerTable *table, uint32_t l0, uint32_t l1,
                      size_t rows0) {
        size_t rows_words = 0, max_mant = 0, max_prod = 0;
        for (uint32_t l = l0; l < l1; ++l) {
            const size_t rows = rows0 << (l - l0);
            rows_words = std::max(rows_words, rows * 2 * p.limbs[l + 1]);
            const uint32_t mant_len = (p.bits[l] - p.digs[l + 1] + 31u) / 32u;
            max_mant = std::max(max_mant, rows * mant_len);
            max_prod = std::max(max_prod, rows * (mant_len + table->powers[p.levels - 1 - l].length));
        }
        cudaError_t err = ping.alloc(rows_words);
        if (err == cudaSuccess) err = pong.alloc(rows_words);
        if (err == cudaSuccess) err = mant.alloc(max_mant);
        if (err == cudaSuccess) err = prod.alloc(max_prod);
        return err;
    }
};

// Levels [l0, l1) on every row of `current` (convert_decimal.cu:331-430):
// row r becomes rows 2r (high child) and 2r + 1 (low child).  Rows are
// independent, so any contiguous range of a level's rows can run alone.
static cudaError_t convert_levels(BatchMPContext *ctx, BatchMPArray &current, const ConvertPlan &p,
                                  const ConvertDecimalPowerTable *table, uint32_t l0, uint32_t l1, LevelBufs &b) {
    DevBuf *bufs[2] = {&b.ping, &b.pong};
    for (uint32_t l = l0; l < l1; ++l) {
        const uint32_t d = p.digs[l + 1];
        const uint32_t cb = p.bits[l + 1];
        const uint32_t B = p.bits[l];
        if (current.length < p.limbs[l]) return cudaErrorInvalidValue;
        if (B <= d || B < cb) return cudaErrorInvalidValue;
        const uint32_t rows = current.batch_size;
        const uint32_t nl = p.limbs[l + 1];
        uint32_t *next = bufs[(l - l0) & 1]->p;
        // every child limb is written by the two extractions below
        extract_shifted(current, next, nl, nl, rows, B - cb, 0u);
        const uint32_t mant_bits = B - d;
        const uint32_t mant_len = (mant_bits + 31u) / 32u;
        extract_low(current, b.mant.p, mant_len, mant_len, rows, mant_bits);
        const BatchMPArray &pw = table->powers[p.levels - 1 - l];
        BatchMPArray mA{b.mant.p, mant_len, rows, mant_len};
        BatchMPArray pB{pw.data, pw.length, rows, 0u};
        BatchMPArray pC{b.prod.p, mant_len + pw.length, rows, mant_len + pw.length};
        const cudaError_t err = mul_tuned(ctx, mA, pB, pC);
        if (err != cudaSuccess) return err;
        extract_shifted(pC, next, nl, nl, rows, mant_bits - cb, 1u);
        current = BatchMPArray{next, nl, rows * 2u, nl};
    }
    return cudaSuccess;
}

// Leaf rows -> digits (convert_decimal.cu:431-474): align each row's
// leaf_bits at the top of its limbs, then 9 digits per x 10^9 step.
static cudaError_t convert_leaves(const BatchMPArray &current, uint32_t leaf_bits, uint32_t leaf_digits,
                                  char *output_digits) {
    const uint32_t align = current.length * 32u - leaf_bits;
    DevBuf aligned;
    cudaError_t err = aligned.alloc((size_t)current.batch_size * current.length);
    if (err != cudaSuccess) return err;
    batch_shift_bits(current.data, aligned.p, current.batch_size, current.length, current.length,
                     current.stride, current.length, (int32_t)align);
    decimal_rows<true>(aligned.p, output_digits, current.batch_size, current.length, current.length,
                       leaf_digits, leaf_digits);
    return cudaGetLastError();
}

static cudaError_t convert_check(BatchMPContext *ctx, const BatchMPArray &input, uint32_t total_digits,
                                 uint32_t leaf_digits, const ConvertDecimalPowerTable *table, char *output_digits,
                                 uint32_t *levels) {
    if (ctx == nullptr || output_digits == nullptr || input.batch_size != 1u || input.data == nullptr)
        return cudaErrorInvalidValue;
    *levels = levels_for_shape(total_digits, leaf_digits);
    if (*levels == UINT32_MAX || table == nullptr || table->leaf_digits != leaf_digits ||
        table->levels != *levels)
        return cudaErrorInvalidValue;
    return cudaSuccess;
}

// The conversion with its digits in 2^log_chunks parts: all levels but the
// last kTailLevels on the whole fraction, then those levels and the leaves
// for each contiguous range of rows (one part of the digits) after the
// other; ready(offset, count, user) is called (on the host, in digit order)
// once each part's digits are issued on the current stream, so that the
// caller can copy them out while the next parts convert.  Splitting only the
// last levels keeps the extra launches few and each part's work (about
// four levels of one part of the rows) longer than its digits' copy.  The
// digits are those of convert_decimal_equal_split.
constexpr uint32_t kTailLevels = 4;

cudaError_t convert_decimal_in_parts(BatchMPContext *ctx, BatchMPArray input, uint32_t input_bits,
                                     uint32_t total_digits, uint32_t leaf_digits,
                                     const ConvertDecimalPowerTable *table, char *output_digits,
                                     uint32_t log_chunks, void (*ready)(size_t, size_t, void *), void *user) {
    uint32_t levels = 0;
    cudaError_t err = convert_check(ctx, input, total_digits, leaf_digits, table, output_digits, &levels);
    if (err != cudaSuccess) return err;
    const uint32_t s = levels > kTailLevels ? levels - kTailLevels : 0u;   // first split level
    const uint32_t lp = std::min(log_chunks, s);                            // 2^lp parts of 2^(s - lp) rows
    if (levels == 0u || lp == 0u) {
        err = convert_decimal_equal_split(ctx, input, input_bits, total_digits, leaf_digits, table, output_digits);
        if (err == cudaSuccess && ready) ready(0, total_digits, user);
        return err;
    }
    const ConvertPlan p = convert_plan(levels, total_digits, input_bits, input.length);
    BatchMPArray top = input;
    LevelBufs tb;
    err = tb.alloc(p, table, 0u, s, 1u);
    if (err == cudaSuccess) err = convert_levels(ctx, top, p, table, 0u, s, tb);
    if (err != cudaSuccess) return err;
    const uint32_t rows = 1u << (s - lp);
    const size_t part_digits = (size_t)leaf_digits << (levels - lp);
    LevelBufs cb;
    err = cb.alloc(p, table, s, levels, rows);
    for (uint32_t c = 0; c < (1u << lp) && err == cudaSuccess; ++c) {
        BatchMPArray cur{top.data + (size_t)c * rows * top.stride, top.length, rows, top.stride};
        err = convert_levels(ctx, cur, p, table, s, levels, cb);
        if (err == cudaSuccess) err = convert_leaves(cur, p.bits[levels], leaf_digits, output_digits + c * part_digits);
        if (err == cudaSuccess && ready) ready(c * part_digits, part_digits, user);
    }
    return err;
}

}  // namespace gpupi

cudaError_t convert_decimal_equal_split(BatchMPContext *ctx, BatchMPArray input, uint32_t input_bits,
                                        uint32_t total_digits, uint32_t leaf_digits,
                                        const ConvertDecimalPowerTable *table, char *output_digits) {
    uint32_t levels = 0;
    cudaError_t err = convert_check(ctx, input, total_digits, leaf_digits, table, output_digits, &levels);
    if (err != cudaSuccess) return err;
    cudaStream_t st = current_stream();
    BatchMPArray current = input;
    uint32_t leaf_bits = 0;
    if (levels == 0u) {
        const uint32_t need = bits_for_digits(total_digits);
        const uint32_t nl = (need + 31u) / 32u;
        if (input_bits < need) return cudaErrorInvalidValue;
        DevBuf one;
        err = one.alloc(nl);
        if (err != cudaSuccess) return err;
        cudaMemsetAsync(one.p, 0, (size_t)nl * 4, st);
        // single row: dst row index 2*0+0 = 0
        extract_shifted(input, one.p, nl, nl, 1u, input_bits - need, 0u);
        current = BatchMPArray{one.p, nl, 1u, nl};
        err = convert_leaves(current, need, leaf_digits, output_digits);
        if (err == cudaSuccess) err = cudaStreamSynchronize(st);
        return err;
    }
    const ConvertPlan p = convert_plan(levels, total_digits, input_bits, input.length);
    LevelBufs b;
    err = b.alloc(p, table, 0u, levels, 1u);
    if (err == cudaSuccess) err = convert_levels(ctx, current, p, table, 0u, levels, b);
    leaf_bits = p.bits[levels];
    if (err == cudaSuccess) err = convert_leaves(current, leaf_bits, leaf_digits, output_digits);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
    return err;
}
