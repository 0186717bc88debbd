// Test infrastructure (checker only): runs one benchmark configuration
// through gpupi's public batched API and writes the raw result to stdout, so
// that the same workload can be pinned against the reference build.
//
// It is written against the reference's headers (batch_arith.h:8-152,
// convert_decimal.h:7-41), so the same source links against the reference's
// own objects (oracle/_ref/ref_configs_ref, built by oracle/build_ref.py) and
// against libgpupi_b200.so.  Inputs come from a splitmix64 stream (the seed
// is part of the configuration), identical to oracle/ref_inputs.py.
//
//   ref_configs c2              4096 products, lengths 2^e + r (e in 3..11)
//                               per operand, each through batch_mp_mul with
//                               N = 1 (the reference has no ragged batch):
//                               products concatenated, limbs LE
//   ref_configs c3 <log2 L>     one L x L-limb product (batch_mp_mul, N = 1)
//   ref_configs c4              a 2^25-limb fraction (2^30 bits) to
//                               308 << 20 = 322,961,408 digits
//                               (convert_decimal_precompute_powers +
//                               convert_decimal_equal_split)
//
// The elapsed device time of the call goes to stderr as "elapsed_ms=...".
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "batch_arith.h"
#include "convert_decimal.h"

static uint64_t splitmix64(uint64_t &state) {
    uint64_t z = (state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// n limbs: output k of the stream gives limbs 2k (low half) and 2k+1 (high).
static std::vector<uint32_t> limbs(uint64_t &state, size_t n) {
    std::vector<uint32_t> v(n);
    for (size_t i = 0; i < n; i += 2) {
        const uint64_t z = splitmix64(state);
        v[i] = (uint32_t)z;
        if (i + 1 < n) v[i + 1] = (uint32_t)(z >> 32);
    }
    return v;
}

#define CHECK(x)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (x);                                                                 \
        if (e_ != cudaSuccess) {                                                              \
            fprintf(stderr, "%s:%d: %s -> %s\n", __FILE__, __LINE__, #x, cudaGetErrorString(e_)); \
            exit(2);                                                                          \
        }                                                                                     \
    } while (0)

static void write_all(const void *p, size_t n) {
    const char *c = (const char *)p;
    while (n) {
        size_t w = fwrite(c, 1, n, stdout);
        if (w == 0) exit(3);
        c += w;
        n -= w;
    }
}

static BatchMPArray upload(const std::vector<uint32_t> &h) {
    BatchMPArray a = batch_mp_array_create(1u, (uint32_t)h.size());
    if (!a.data) exit(4);
    CHECK(cudaMemcpy(a.data, h.data(), h.size() * 4, cudaMemcpyHostToDevice));
    return a;
}

struct Timer {
    cudaEvent_t a, b;
    Timer() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a);
    }
    void stop() {
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        fprintf(stderr, "elapsed_ms=%.3f\n", ms);
    }
};

static int run_c2(BatchMPContext *ctx) {
    const int n = 4096;
    uint64_t st = 0xC2;
    std::vector<uint32_t> La(n), Lb(n);
    for (int i = 0; i < n; ++i) {
        const uint64_t z = splitmix64(st);
        const uint32_t ea = 3u + (uint32_t)(z % 9u), eb = 3u + (uint32_t)((z >> 8) % 9u);
        La[i] = (1u << ea) + (uint32_t)((z >> 16) & ((1u << ea) - 1u));
        Lb[i] = (1u << eb) + (uint32_t)((z >> 40) & ((1u << eb) - 1u));
    }
    size_t ta = 0, tb = 0;
    for (int i = 0; i < n; ++i) ta += La[i], tb += Lb[i];
    std::vector<uint32_t> A = limbs(st, ta), B = limbs(st, tb);
    BatchMPArray dA = upload(A), dB = upload(B);
    BatchMPArray dC = batch_mp_array_create(1u, (uint32_t)(ta + tb));
    if (!dC.data) return 4;
    Timer t;
    size_t oa = 0, ob = 0, oc = 0;
    for (int i = 0; i < n; ++i) {
        BatchMPArray a{dA.data + oa, La[i], 1u, La[i]};
        BatchMPArray b{dB.data + ob, Lb[i], 1u, Lb[i]};
        BatchMPArray c{dC.data + oc, La[i] + Lb[i], 1u, La[i] + Lb[i]};
        CHECK(batch_mp_mul(ctx, a, b, c));
        oa += La[i];
        ob += Lb[i];
        oc += La[i] + Lb[i];
    }
    t.stop();
    std::vector<uint32_t> C(ta + tb);
    CHECK(cudaMemcpy(C.data(), dC.data, C.size() * 4, cudaMemcpyDeviceToHost));
    write_all(C.data(), C.size() * 4);
    batch_mp_array_release(dA);
    batch_mp_array_release(dB);
    batch_mp_array_release(dC);
    return 0;
}

static int run_c3(BatchMPContext *ctx, int log2L) {
    const uint32_t L = 1u << log2L;
    uint64_t st = 0xC3;
    std::vector<uint32_t> A = limbs(st, L), B = limbs(st, L);
    BatchMPArray dA = upload(A), dB = upload(B);
    A.clear();
    A.shrink_to_fit();
    B.clear();
    B.shrink_to_fit();
    BatchMPArray dC = batch_mp_array_create(1u, 2u * L);
    if (!dC.data) return 4;
    Timer t;
    CHECK(batch_mp_mul(ctx, dA, dB, dC));
    t.stop();
    batch_mp_array_release(dA);
    batch_mp_array_release(dB);
    std::vector<uint32_t> C((size_t)2 * L);
    CHECK(cudaMemcpy(C.data(), dC.data, C.size() * 4, cudaMemcpyDeviceToHost));
    write_all(C.data(), C.size() * 4);
    batch_mp_array_release(dC);
    return 0;
}

static int run_c4(BatchMPContext *ctx) {
    const uint32_t L = 1u << 25, leaf = 308u, levels = 20u;
    const uint32_t total = leaf << levels;
    uint64_t st = 0xC4;
    std::vector<uint32_t> X = limbs(st, L);
    BatchMPArray dX = upload(X);
    char *d_out = nullptr;
    CHECK(cudaMalloc(&d_out, total));
    ConvertDecimalPowerTable table{};
    CHECK(convert_decimal_precompute_powers(ctx, &table, leaf, levels));
    Timer t;
    CHECK(convert_decimal_equal_split(ctx, dX, 32u * L, total, leaf, &table, d_out));
    t.stop();
    std::vector<char> out(total);
    CHECK(cudaMemcpy(out.data(), d_out, total, cudaMemcpyDeviceToHost));
    write_all(out.data(), total);
    convert_decimal_release_powers(&table);
    cudaFree(d_out);
    batch_mp_array_release(dX);
    return 0;
}

int main(int argc, char **argv) {
    if (argc < 2) {
        fprintf(stderr, "usage: %s c2 | c3 <log2 L> | c4\n", argv[0]);
        return 1;
    }
    BatchMPContext *ctx = batch_mp_init();
    if (!ctx) return 5;
    int rc = 1;
    if (!strcmp(argv[1], "c2")) rc = run_c2(ctx);
    else if (!strcmp(argv[1], "c3") && argc > 2) rc = run_c3(ctx, atoi(argv[2]));
    else if (!strcmp(argv[1], "c4")) rc = run_c4(ctx);
    fflush(stdout);
    batch_mp_destroy(ctx);
    return rc;
}
