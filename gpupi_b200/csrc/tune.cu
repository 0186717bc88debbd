// Autotuner and its persisted table (replaces the reference's fixed
// constants: the schoolbook / NTT crossover BATCH_MUL_NAIVE_L_MAX,
// batch_arith.cu:181, and the NTT size rule of get_N_max and the schedule
// tables, batch_mul_ntt.cu:1781-1915).
//
// The table decides, per length bucket,
//   * which kernel computes a product of L_a + L_b limbs: the CUDA-core
//     schoolbook (mul_naive.cu), the tensor-core schoolbook (mul_tc.cu) or the
//     NTT (mul_ntt.cu);
//   * the NTT's transform shape for a product needing `need` = L_a + L_b - 1
//     points: K = 2^log_k points times M cosets, M K >= need (one transform
//     of the next power of two, or several cosets of a smaller one).
// The result is the exact product whatever the table says; only the time
// changes.  Without a table the built-in rule applies (schoolbook up to the
// crossover set by gpupi_set_mul_crossover, 448 limbs, then the NTT at the
// next power of two).
//
// File format (text, one entry per line, '#' starts a comment):
//   mul <max_sum> school|tc|ntt        products with L_a + L_b <= max_sum
//                                      (and above the previous entry)
//   ntt <min_need> <max_need> <log_k> <M>   transforms for min_need <= need <= max_need
// The table is read at context creation from $GPUPI_TUNE_TABLE, else from
// tune_table.txt beside libgpupi_b200.so; gpupi_autotune() measures the
// candidates on the current GPU (CUDA events, best of several runs, each
// candidate's product checked against the reference candidate's, word for
// word) and writes the file.
#include "common.cuh"
#include "batch_arith.h"
#include "batch_mul_ntt.h"

#include <dlfcn.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

namespace gpupi {

void school_mul(const uint32_t *A, const uint32_t *B, uint32_t *C, uint32_t N, uint32_t La, uint32_t Lb,
                uint64_t sA, uint64_t sB, uint64_t sC);
bool school_thread_fits(uint32_t La, uint32_t Lb);
bool tc_fits(uint32_t La, uint32_t Lb);
cudaError_t tc_mul(const uint32_t *A, const uint32_t *B, uint32_t *C, uint32_t N, uint32_t La, uint32_t Lb,
                   uint64_t sA, uint64_t sB, uint64_t sC);
cudaError_t mul_ntt_direct(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, BatchMPArray C);
uint32_t school_max();

enum MulKind { kSchool = 0, kTensor = 1, kNtt = 2 };

namespace {

struct MulEntry {
    uint32_t max_sum;
    int kind;
};
struct NttEntry {
    uint64_t min_need, max_need;
    int log_k, M;
};
struct Table {
    std::mutex mu;
    bool loaded = false;
    std::string source;
    std::vector<MulEntry> mul;
    std::vector<NttEntry> ntt;
    // a shape forced by the tuner while it measures (log_k 0: none)
    int force_log_k = 0, force_M = 0;
};
Table &table() {
    static Table t;
    return t;
}

const char *kind_name(int k) { return k == kSchool ? "school" : k == kTensor ? "tc" : "ntt"; }

int parse_kind(const char *s) {
    if (!strcmp(s, "school")) return kSchool;
    if (!strcmp(s, "tc")) return kTensor;
    if (!strcmp(s, "ntt")) return kNtt;
    return -1;
}

bool shape_ok(uint64_t need, int log_k, int M) {
    if (log_k < 1 || log_k > 25 || M < 1 || M > 20) return false;
    if (M > 1 && log_k <= 12) return false;   // cosets need the column passes
    return (uint64_t)M << log_k >= need;
}

// Parse `text`; returns the number of entries, or -(line number) of the
// first malformed line.  On success the table is replaced.
int parse_table(const std::string &text, const std::string &source) {
    std::vector<MulEntry> mul;
    std::vector<NttEntry> ntt;
    size_t pos = 0;
    int line = 0;
    while (pos <= text.size()) {
        size_t end = text.find('\n', pos);
        if (end == std::string::npos) end = text.size();
        std::string l = text.substr(pos, end - pos);
        pos = end + 1;
        ++line;
        const size_t hash = l.find('#');
        if (hash != std::string::npos) l.resize(hash);
        char word[16] = {0}, kind[16] = {0};
        unsigned long long a = 0, a2 = 0;
        int b = 0, c = 0;
        if (sscanf(l.c_str(), " %15s", word) != 1) continue;   // blank
        if (!strcmp(word, "mul")) {
            if (sscanf(l.c_str(), " mul %llu %15s", &a, kind) != 2 || parse_kind(kind) < 0 || a == 0 ||
                a > 0xffffffffull)
                return -line;
            mul.push_back(MulEntry{(uint32_t)a, parse_kind(kind)});
        } else if (!strcmp(word, "ntt")) {
            if (sscanf(l.c_str(), " ntt %llu %llu %d %d", &a, &a2, &b, &c) != 4 || a > a2 || !shape_ok(a2, b, c))
                return -line;
            ntt.push_back(NttEntry{a, a2, b, c});
        } else {
            return -line;
        }
        if (end == text.size()) break;
    }
    std::sort(mul.begin(), mul.end(), [](const MulEntry &x, const MulEntry &y) { return x.max_sum < y.max_sum; });
    std::sort(ntt.begin(), ntt.end(), [](const NttEntry &x, const NttEntry &y) { return x.max_need < y.max_need; });
    Table &t = table();
    std::lock_guard<std::mutex> g(t.mu);
    t.mul = std::move(mul);
    t.ntt = std::move(ntt);
    t.loaded = true;
    t.source = source;
    return (int)(t.mul.size() + t.ntt.size());
}

bool read_file(const std::string &path, std::string &out) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return false;
    char buf[4096];
    size_t n;
    out.clear();
    while ((n = fread(buf, 1, sizeof buf, f)) > 0) out.append(buf, n);
    fclose(f);
    return true;
}

std::string default_table_path() {
    const char *env = getenv("GPUPI_TUNE_TABLE");
    if (env && *env) return env;
    Dl_info info{};
    if (dladdr((void *)&default_table_path, &info) && info.dli_fname) {
        std::string p(info.dli_fname);
        const size_t slash = p.find_last_of('/');
        return (slash == std::string::npos ? std::string(".") : p.substr(0, slash)) + "/tune_table.txt";
    }
    return "tune_table.txt";
}

}  // namespace

// Kernel for a product of La x Lb limbs.  public_api: gpupi's batch_mp_mul
// contract (no product above 1024 limbs avoids the NTT, none at or below
// it uses the NTT's workspace).
int mul_kind(uint32_t La, uint32_t Lb, bool public_api) {
    const uint64_t L = (uint64_t)La + Lb;
    if (La == 0u || Lb == 0u || school_thread_fits(La, Lb)) return kSchool;
    int k = -1;
    {
        Table &t = table();
        std::lock_guard<std::mutex> g(t.mu);
        if (t.loaded) {
            k = kNtt;
            for (const MulEntry &e : t.mul)
                if (L <= e.max_sum) {
                    k = e.kind;
                    break;
                }
        }
    }
    if (k < 0) k = (L <= school_max() && L <= 1024u) ? kSchool : kNtt;
    if (public_api) {
        if (L > 1024u) return kNtt;
        if (k == kNtt) return kSchool;
    }
    if (k == kTensor && !tc_fits(La, Lb)) k = (L <= 1024u) ? kSchool : kNtt;
    if (k == kSchool && L > 1024u) k = kNtt;
    return k;
}

// NTT shape for `need` points from the table (or the tuner's forced
// shape); false: use the built-in rule.
bool ntt_shape_override(uint64_t need, int *log_k, int *M) {
    Table &t = table();
    std::lock_guard<std::mutex> g(t.mu);
    if (t.force_log_k > 0 && shape_ok(need, t.force_log_k, t.force_M)) {
        *log_k = t.force_log_k;
        *M = t.force_M;
        return true;
    }
    if (!t.loaded) return false;
    for (const NttEntry &e : t.ntt)
        if (need >= e.min_need && need <= e.max_need) {
            if (!shape_ok(need, e.log_k, e.M)) return false;
            *log_k = e.log_k;
            *M = e.M;
            return true;
        }
    return false;
}

void tune_load_default() {
    Table &t = table();
    {
        std::lock_guard<std::mutex> g(t.mu);
        if (t.loaded || !t.source.empty()) return;
        t.source = "(built-in rule)";
    }
    std::string text;
    const std::string path = default_table_path();
    if (read_file(path, text)) parse_table(text, path);
}

int tune_load(const char *path) {
    std::string text;
    if (!path || !read_file(path, text)) return -1000000;
    return parse_table(text, path);
}

int tune_load_text(const char *text) { return text ? parse_table(text, "(text)") : -1000000; }

void tune_reset() {
    Table &t = table();
    std::lock_guard<std::mutex> g(t.mu);
    t.mul.clear();
    t.ntt.clear();
    t.loaded = false;
    t.source = "(built-in rule)";
    t.force_log_k = t.force_M = 0;
}

std::string tune_describe() {
    Table &t = table();
    std::lock_guard<std::mutex> g(t.mu);
    std::string s = "# source: " + (t.source.empty() ? std::string("(built-in rule)") : t.source) + "\n";
    char line[128];
    for (const MulEntry &e : t.mul) {
        snprintf(line, sizeof line, "mul %u %s\n", e.max_sum, kind_name(e.kind));
        s += line;
    }
    for (const NttEntry &e : t.ntt) {
        snprintf(line, sizeof line, "ntt %llu %llu %d %d\n", (unsigned long long)e.min_need,
                 (unsigned long long)e.max_need, e.log_k, e.M);
        s += line;
    }
    return s;
}

// ---------------------------------------------------------------------------
// Measurement
// ---------------------------------------------------------------------------
namespace {

__global__ void k_fill_random(uint32_t *p, uint64_t n, uint64_t seed) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        p[i] = (uint32_t)(z ^ (z >> 31));
    }
}

__global__ void k_count_diff(const uint32_t *a, const uint32_t *b, uint64_t n, unsigned long long *out) {
    unsigned long long c = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        c += (a[i] != b[i]);
    if (c) atomicAdd(out, c);
}

struct Bench {
    BatchMPContext *ctx;
    cudaStream_t st;
    uint32_t *A = nullptr, *B = nullptr, *C = nullptr, *R = nullptr;
    unsigned long long *diff = nullptr;
    size_t cap = 0;   // limbs per buffer
};

// Runs kind k on N products of La x Lb (packed rows); returns ms (best of
// `reps` after one warm-up) or a negative value on failure.
float run_kind(Bench &b, int k, uint32_t N, uint32_t La, uint32_t Lb, int reps) {
    const BatchMPArray a{b.A, La, N, La}, bb{b.B, Lb, N, Lb}, c{b.C, La + Lb, N, La + Lb};
    auto once = [&]() -> cudaError_t {
        if (k == kSchool) {
            school_mul(b.A, b.B, b.C, N, La, Lb, La, Lb, La + Lb);
            return cudaGetLastError();
        }
        if (k == kTensor) return tc_mul(b.A, b.B, b.C, N, La, Lb, La, Lb, La + Lb);
        return mul_ntt_direct(b.ctx, a, bb, c);
    };
    if (once() != cudaSuccess || cudaStreamSynchronize(b.st) != cudaSuccess) return -1.f;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int r = 0; r < reps; ++r) {
        cudaEventRecord(e0, b.st);
        if (once() != cudaSuccess) best = -1.f;
        cudaEventRecord(e1, b.st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (best > 0.f) best = std::min(best, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

// Word-for-word comparison of C with the reference result R.
bool same_result(Bench &b, uint64_t words) {
    cudaMemsetAsync(b.diff, 0, sizeof(unsigned long long), b.st);
    k_count_diff<<<grid_for(words, 256, kNumSMs * 8), 256, 0, b.st>>>(b.C, b.R, words, b.diff);
    unsigned long long h = 1;
    if (cudaMemcpyAsync(&h, b.diff, sizeof h, cudaMemcpyDeviceToHost, b.st) != cudaSuccess) return false;
    cudaStreamSynchronize(b.st);
    return h == 0;
}

}  // namespace

// Measures every candidate and writes the table to `path` (then loads it).
// budget_limbs: total limbs of the operands of one measured batch.
cudaError_t autotune(BatchMPContext *ctx, const char *path, uint64_t budget_limbs, std::string *report) {
    if (!ctx || !path) return cudaErrorInvalidValue;
    if (budget_limbs < (1ull << 16)) budget_limbs = 1ull << 16;
    Bench b;
    b.ctx = ctx;
    b.st = current_stream();
    // the largest batch: budget_limbs of operands, as many of product
    b.cap = (size_t)budget_limbs + (1u << 26);
    cudaError_t err = cudaMalloc(&b.A, b.cap * 4);
    if (err == cudaSuccess) err = cudaMalloc(&b.B, b.cap * 4);
    if (err == cudaSuccess) err = cudaMalloc(&b.C, 2 * b.cap * 4);
    if (err == cudaSuccess) err = cudaMalloc(&b.R, 2 * b.cap * 4);
    if (err == cudaSuccess) err = cudaMalloc(&b.diff, sizeof(unsigned long long));
    auto release = [&]() {
        cudaFree(b.A);
        cudaFree(b.B);
        cudaFree(b.C);
        cudaFree(b.R);
        cudaFree(b.diff);
    };
    if (err != cudaSuccess) {
        release();
        return err;
    }
    k_fill_random<<<kNumSMs * 8, 256, 0, b.st>>>(b.A, b.cap, 11);
    k_fill_random<<<kNumSMs * 8, 256, 0, b.st>>>(b.B, b.cap, 12);
    tune_reset();   // measure the kernels, not a previous table
    std::string out = "# gpupi_b200 tune table: measured by gpupi_autotune on ";
    {
        int dev = 0;
        cudaDeviceProp prop{};
        cudaGetDevice(&dev);
        cudaGetDeviceProperties(&prop, dev);
        out += prop.name;
        out += " (" + std::to_string(prop.multiProcessorCount) + " SMs)\n";
    }
    out += "# balanced products (L_a = L_b), batches of about " + std::to_string(budget_limbs) +
           " operand limbs; times in ms (best of 3)\n";
    std::string log;
    char line[256];
    // 1. product kernel per length bucket (L_a + L_b up to 8192)
    static const uint32_t sums[] = {40,   48,   64,   96,   128,  192,  256,  320,  384,  448,  512,  640,
                                    768,  896,  1024, 1536, 2048, 3072, 4096, 6144, 8192};
    for (uint32_t L : sums) {
        const uint32_t La = L / 2, Lb = L - La;
        const uint32_t N = (uint32_t)std::max<uint64_t>(1, budget_limbs / L);
        float t[3] = {-1.f, -1.f, -1.f};
        // reference result: the NTT
        t[kNtt] = run_kind(b, kNtt, N, La, Lb, 3);
        if (t[kNtt] < 0.f) {
            release();
            return cudaErrorUnknown;
        }
        cudaMemcpyAsync(b.R, b.C, (size_t)N * L * 4, cudaMemcpyDeviceToDevice, b.st);
        if (L <= 1024u) {
            t[kSchool] = run_kind(b, kSchool, N, La, Lb, 3);
            if (t[kSchool] > 0.f && !same_result(b, (uint64_t)N * L)) t[kSchool] = -2.f;
        }
        if (tc_fits(La, Lb)) {
            t[kTensor] = run_kind(b, kTensor, N, La, Lb, 3);
            if (t[kTensor] > 0.f && !same_result(b, (uint64_t)N * L)) t[kTensor] = -2.f;
        }
        int best = kNtt;
        for (int k = 0; k < 3; ++k)
            if (t[k] > 0.f && t[k] < t[best]) best = k;
        snprintf(line, sizeof line, "mul %u %s   # N=%u school=%.4f tc=%.4f ntt=%.4f\n", L, kind_name(best), N,
                 t[kSchool], t[kTensor], t[kNtt]);
        out += line;
    }
    // 2. NTT shape per need bucket: quarters of each octave (2^k, 2^(k+1)]
    for (int k = 13; k < 25; ++k) {
        for (int qtr = 1; qtr <= 4; ++qtr) {
            const uint64_t need = (1ull << k) + ((uint64_t)qtr << (k - 2));   // top of the bucket
            const uint32_t L = (uint32_t)need + 1u;
            const uint32_t La = L / 2, Lb = L - La;
            const uint32_t N = (uint32_t)std::max<uint64_t>(1, budget_limbs / L);
            struct Cand {
                int log_k, M;
                float ms;
            };
            std::vector<Cand> cands;
            for (int lk = k + 1; lk >= std::max(13, k - 2); --lk) {
                const int M = (int)((need + (1ull << lk) - 1) >> lk);
                if (shape_ok(need, lk, M)) cands.push_back(Cand{lk, M, -1.f});
            }
            for (size_t i = 0; i < cands.size(); ++i) {
                {
                    Table &t = table();
                    std::lock_guard<std::mutex> g(t.mu);
                    t.force_log_k = cands[i].log_k;
                    t.force_M = cands[i].M;
                }
                cands[i].ms = run_kind(b, kNtt, N, La, Lb, 3);
                if (i == 0)
                    cudaMemcpyAsync(b.R, b.C, (size_t)N * L * 4, cudaMemcpyDeviceToDevice, b.st);
                else if (cands[i].ms > 0.f && !same_result(b, (uint64_t)N * L))
                    cands[i].ms = -2.f;
            }
            {
                Table &t = table();
                std::lock_guard<std::mutex> g(t.mu);
                t.force_log_k = t.force_M = 0;
            }
            size_t best = 0;
            for (size_t i = 1; i < cands.size(); ++i)
                if (cands[i].ms > 0.f && (cands[best].ms < 0.f || cands[i].ms < cands[best].ms)) best = i;
            const uint64_t lo = (1ull << k) + ((uint64_t)(qtr - 1) << (k - 2)) + 1u;
            snprintf(line, sizeof line, "ntt %llu %llu %d %d   #", (unsigned long long)lo, (unsigned long long)need,
                     cands[best].log_k, cands[best].M);
            out += line;
            for (const Cand &c : cands) {
                snprintf(line, sizeof line, " K=2^%d,M=%d:%.4f", c.log_k, c.M, c.ms);
                out += line;
            }
            snprintf(line, sizeof line, " (N=%u)\n", N);
            out += line;
        }
    }
    release();
    FILE *f = fopen(path, "wb");
    if (!f) return cudaErrorInvalidValue;
    const bool ok = fwrite(out.data(), 1, out.size(), f) == out.size();
    if (fclose(f) != 0 || !ok) return cudaErrorInvalidValue;
    if (report) *report = out;
    return parse_table(out, path) > 0 ? cudaSuccess : cudaErrorUnknown;
}

}  // namespace gpupi
