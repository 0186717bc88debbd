// Ragged batched multiplication: N independent products with per-product
// lengths, one call (no counterpart in the reference, whose batches share one
// L_a / L_b; gpupi's callers with uneven pairs issue one call per pair).
//
// Products are bucketed on the host:
//   * L_a = 0 or L_b = 0: the L_a + L_b output limbs are zeroed;
//   * products the tune table gives to the CUDA-core schoolbook: one
//     k_school_cols launch reading every product's offsets and lengths from a
//     descriptor array; those it gives to the tensor-core schoolbook: one
//     k_mul_tc launch over their descriptors;
//   * otherwise by transform size 2^ceil(log2(L_a + L_b - 1)): each bucket's
//     operands are gathered into zero-padded rows (longer operand first: the
//     product commutes), multiplied as one uniform batch (mul_tuned), and
//     the L_a + L_b limbs of each row scattered to the product's output.
//     Zeros above an operand leave the low L_a + L_b limbs of the product
//     unchanged.
// Device scratch comes from the stream's scratch arena.
#include "common.cuh"
#include "batch_arith.h"

#include <algorithm>
#include <map>
#include <vector>

namespace gpupi {

void school_mul_ragged(const uint32_t *A, const uint32_t *B, uint32_t *C, uint32_t N, const RaggedRow *rows,
                       uint64_t limb_products);
cudaError_t tc_mul_ragged(const uint32_t *A, const uint32_t *B, uint32_t *C, uint32_t n, const RaggedRow *rows,
                          uint32_t maxQ, uint32_t maxN, uint64_t limbs_moved);
void tc_shape(uint32_t La, uint32_t Lb, uint32_t *Q, uint32_t *N);
int mul_kind(uint32_t La, uint32_t Lb, bool public_api);
cudaError_t mul_tuned(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, BatchMPArray C);

namespace {

// dst row r (stride limbs) = src[off_r .. off_r + len_r) zero-padded; which
// selects the A (0) or B (1) side of the descriptor.
__global__ void __launch_bounds__(256) k_gather_rows(uint32_t *__restrict__ dst, uint64_t stride,
                                                     const uint32_t *__restrict__ src,
                                                     const RaggedRow *__restrict__ rows, uint32_t n, int which) {
    for (uint32_t r = blockIdx.x; r < n; r += gridDim.x) {
        const RaggedRow d = rows[r];
        const uint64_t off = which ? d.offB : d.offA;
        const uint32_t len = which ? d.Lb : d.La;
        uint32_t *out = dst + r * stride;
        for (uint64_t i = threadIdx.x; i < stride; i += blockDim.x) out[i] = (i < len) ? src[off + i] : 0u;
    }
}

// C[offC_r .. + La_r + Lb_r) = the low limbs of padded product row r.
__global__ void __launch_bounds__(256) k_scatter_rows(uint32_t *__restrict__ C, const uint32_t *__restrict__ src,
                                                      uint64_t stride, const RaggedRow *__restrict__ rows,
                                                      uint32_t n) {
    for (uint32_t r = blockIdx.x; r < n; r += gridDim.x) {
        const RaggedRow d = rows[r];
        const uint32_t *in = src + r * stride;
        const uint64_t len = (uint64_t)d.La + d.Lb;
        for (uint64_t i = threadIdx.x; i < len; i += blockDim.x) C[d.offC + i] = in[i];
    }
}

__global__ void __launch_bounds__(256) k_zero_rows(uint32_t *__restrict__ C, const RaggedRow *__restrict__ rows,
                                                   uint32_t n) {
    for (uint32_t r = blockIdx.x; r < n; r += gridDim.x) {
        const RaggedRow d = rows[r];
        const uint64_t len = (uint64_t)d.La + d.Lb;
        for (uint64_t i = threadIdx.x; i < len; i += blockDim.x) C[d.offC + i] = 0u;
    }
}

int ceil_log2_u64(uint64_t x) {
    int k = 0;
    while ((1ull << k) < x) ++k;
    return k;
}

unsigned grid_rows(uint32_t n) { return (unsigned)std::max<uint32_t>(1u, std::min<uint32_t>(n, kNumSMs * 16)); }

// One NTT bucket: rows with La >= Lb come first (sources A, B), rows with
// La < Lb follow with their operands exchanged (sources B, A).
cudaError_t ntt_bucket(BatchMPContext *ctx, const std::vector<RaggedRow> &rows, const uint32_t *A,
                       const uint32_t *B, uint32_t *C, cudaStream_t st) {
    std::vector<RaggedRow> ord;
    ord.reserve(rows.size());
    for (const RaggedRow &d : rows)
        if (d.La >= d.Lb) ord.push_back(d);
    const uint32_t nk = (uint32_t)ord.size();
    for (RaggedRow d : rows)
        if (d.La < d.Lb) {
            std::swap(d.La, d.Lb);
            std::swap(d.offA, d.offB);
            ord.push_back(d);
        }
    const uint32_t n = (uint32_t)ord.size(), ns = n - nk;
    uint32_t ma = 0, mb = 0;
    for (const RaggedRow &d : ord) {
        ma = std::max(ma, d.La);
        mb = std::max(mb, d.Lb);
    }
    const uint64_t lc = (uint64_t)ma + mb;
    uint32_t *pa = nullptr, *pb = nullptr, *pc = nullptr;
    RaggedRow *dr = nullptr;
    cudaError_t err = scratch_alloc((void **)&pa, (size_t)n * ma * 4);
    if (err == cudaSuccess) err = scratch_alloc((void **)&pb, (size_t)n * mb * 4);
    if (err == cudaSuccess) err = scratch_alloc((void **)&pc, (size_t)n * lc * 4);
    if (err == cudaSuccess) err = scratch_alloc((void **)&dr, (size_t)n * sizeof(RaggedRow));
    if (err == cudaSuccess) {
        err = cudaMemcpyAsync(dr, ord.data(), (size_t)n * sizeof(RaggedRow), cudaMemcpyHostToDevice, st);
        note_h2d((size_t)n * sizeof(RaggedRow));
    }
    if (err == cudaSuccess && nk) {
        k_gather_rows<<<grid_rows(nk), 256, 0, st>>>(pa, ma, A, dr, nk, 0);
        k_gather_rows<<<grid_rows(nk), 256, 0, st>>>(pb, mb, B, dr, nk, 1);
        count_launch();
        count_launch();
    }
    if (err == cudaSuccess && ns) {
        k_gather_rows<<<grid_rows(ns), 256, 0, st>>>(pa + (size_t)nk * ma, ma, B, dr + nk, ns, 0);
        k_gather_rows<<<grid_rows(ns), 256, 0, st>>>(pb + (size_t)nk * mb, mb, A, dr + nk, ns, 1);
        count_launch();
        count_launch();
    }
    if (err == cudaSuccess) {
        const BatchMPArray a{pa, ma, n, ma}, b{pb, mb, n, mb}, c{pc, (uint32_t)lc, n, (uint32_t)lc};
        err = mul_tuned(ctx, a, b, c);
    }
    if (err == cudaSuccess) {
        k_scatter_rows<<<grid_rows(n), 256, 0, st>>>(C, pc, lc, dr, n);
        count_launch();
        err = cudaGetLastError();
    }
    scratch_free(pa);
    scratch_free(pb);
    scratch_free(pc);
    scratch_free(dr);
    return err;
}

}  // namespace

cudaError_t mul_ragged(BatchMPContext *ctx, uint32_t N, const uint32_t *A, const uint64_t *offA, const uint32_t *La,
                       const uint32_t *B, const uint64_t *offB, const uint32_t *Lb, uint32_t *C,
                       const uint64_t *offC) {
    if (N == 0u) return cudaSuccess;
    if (!ctx || !A || !B || !C || !offA || !La || !offB || !Lb || !offC) return cudaErrorInvalidValue;
    cudaStream_t st = current_stream();
    std::vector<RaggedRow> zero, school, tensor;
    std::map<int, std::vector<RaggedRow>> ntt;   // by log2 of the transform size
    uint64_t school_work = 0, tc_limbs = 0;
    uint32_t tcQ = 0, tcN = 0;
    for (uint32_t i = 0; i < N; ++i) {
        const RaggedRow d{offA[i], offB[i], offC[i], La[i], Lb[i]};
        const uint64_t Lc = (uint64_t)d.La + d.Lb;
        if (Lc > (20ull << 25) || std::min(d.La, d.Lb) > (1u << 28)) return cudaErrorInvalidValue;
        if (d.La == 0u || d.Lb == 0u) {
            zero.push_back(d);
        } else if (const int kind = mul_kind(d.La, d.Lb, false); kind == 0) {
            school.push_back(d);
            school_work += (uint64_t)d.La * d.Lb;
        } else if (kind == 1) {
            tensor.push_back(d);
            uint32_t q = 0, n = 0;
            tc_shape(d.La, d.Lb, &q, &n);
            tcQ = std::max(tcQ, q);
            tcN = std::max(tcN, n);
            tc_limbs += 2ull * Lc;
        } else {
            ntt[ceil_log2_u64(Lc - 1)].push_back(d);
        }
    }
    cudaError_t err = cudaSuccess;
    if (!zero.empty() || !school.empty() || !tensor.empty()) {
        std::vector<RaggedRow> both(zero);
        both.insert(both.end(), school.begin(), school.end());
        both.insert(both.end(), tensor.begin(), tensor.end());
        RaggedRow *dr = nullptr;
        err = scratch_alloc((void **)&dr, both.size() * sizeof(RaggedRow));
        if (err == cudaSuccess) {
            err = cudaMemcpyAsync(dr, both.data(), both.size() * sizeof(RaggedRow), cudaMemcpyHostToDevice, st);
            note_h2d(both.size() * sizeof(RaggedRow));
        }
        if (err == cudaSuccess && !zero.empty()) {
            k_zero_rows<<<grid_rows((uint32_t)zero.size()), 256, 0, st>>>(C, dr, (uint32_t)zero.size());
            count_launch();
        }
        if (err == cudaSuccess && !school.empty())
            school_mul_ragged(A, B, C, (uint32_t)school.size(), dr + zero.size(), school_work);
        if (err == cudaSuccess && !tensor.empty())
            err = tc_mul_ragged(A, B, C, (uint32_t)tensor.size(), dr + zero.size() + school.size(), tcQ, tcN,
                                tc_limbs);
        if (err == cudaSuccess) err = cudaGetLastError();
        scratch_free(dr);
    }
    for (auto &kv : ntt) {
        if (err != cudaSuccess) break;
        err = ntt_bucket(ctx, kv.second, A, B, C, st);
    }
    return err;
}

}  // namespace gpupi
