// pi_bs_gpu command line (gpupi pi_bs_gpu.cu:2073-2437, main_fractional).
//
//   pi_bs_gpu <digits> [--benchmark|--profile-stages|--full-print] [--plain] [--output FILE]
//             [--checkpoint FILE]
//
// Same arguments, stdout/stderr lines and exit codes as the reference; the
// computation is gpupi_b200's pipeline (pi_engine.cu), by default in its
// tuned form (forward transforms shared within each merge level of the
// splitting tree); --plain (an addition) runs the reference's op sequence,
// which --profile-stages also uses so that its stage list is the
// reference's.  Both print the same RET and digits.  --output FILE
// (an addition; default or --benchmark mode) writes "3<digits>\n" to FILE
// instead of stdout.  Digits are streamed out after the timed region: each
// chunk's device-to-host copy overlaps the write of the chunk before.
// --checkpoint FILE (an addition) loads the splitting tree's result from
// FILE when it is valid for this digit count and otherwise writes it there.
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "pi_engine.h"

namespace {

constexpr uint32_t kValidationMod = 1000000007u;            // pi_bs_gpu.cu:149
constexpr uint64_t kLimbBaseMod = (1ull << 32) % kValidationMod;

bool parse_int_arg(const char *text, int *value) {
    if (!text || !value) return false;
    char *end = nullptr;
    const long v = strtol(text, &end, 10);
    if (end == text || *end != '\0') return false;
    *value = (int)v;
    return true;
}

uint32_t mod_hash(const uint32_t *limbs, uint32_t n) {           // pi_bs_gpu.cu:852-858
    uint64_t v = 0;
    for (int i = (int)n - 1; i >= 0; --i) v = (v * kLimbBaseMod + limbs[i]) % kValidationMod;
    return (uint32_t)v;
}

uint32_t decimal_hash(const char *d, uint32_t n) {               // pi_bs_gpu.cu:860-866
    uint64_t v = 3u;
    for (uint32_t i = 0; i < n; ++i) v = (v * 10u + (uint32_t)(d[i] - '0')) % kValidationMod;
    return (uint32_t)v;
}

void hex_preview(const char *label, const uint32_t *limbs, uint32_t length) {   // :868-896
    const uint32_t hash = mod_hash(limbs, length);
    if (length == 0) {
        printf("%s = 0 hash = %u\n", label, hash);
        return;
    }
    const uint32_t first = std::min(length, 2u), last = std::min(length, 2u);
    printf("%s = ", label);
    for (uint32_t i = 0; i < last; ++i) {
        const uint32_t idx = length - 1 - i;
        if (i == 0) printf("%x", limbs[idx]);
        else printf("%08x", limbs[idx]);
    }
    if (length > first + last) printf("...");
    for (uint32_t i = first; i > 0; --i) {
        const uint32_t idx = i - 1;
        if (length <= first + last && idx >= length - last) continue;
        printf("%08x", limbs[idx]);
    }
    printf(" hash = %u\n", hash);
}

void usage(const char *prog) {
    fprintf(stderr, "Usage: %s <target_digits> [--benchmark|--profile-stages|--full-print] [--plain] [--output FILE] "
            "[--checkpoint FILE]\n",
            prog);
}

}  // namespace

int main(int argc, char **argv) {
    // Load every kernel when the CUDA context is created instead of at its
    // first launch: the library's NTT module holds one kernel per prime,
    // radix and direction, and loading it lazily would put ~17 ms of module
    // loading inside the timed pipeline (an explicit setting is kept).
    setenv("CUDA_MODULE_LOADING", "EAGER", 0);
    int target = 0;
    if (argc < 2 || !parse_int_arg(argv[1], &target) || target < 0) {
        usage(argv[0]);
        return 1;
    }
    const uint32_t requested = (uint32_t)target;
    bool benchmark = false, profile = false, full = false, plain = false;
    const char *out_path = nullptr, *ckpt_path = nullptr;
    int modes = 0;
    for (int i = 2; i < argc; ++i) {
        if (strcmp(argv[i], "--benchmark") == 0) benchmark = true, ++modes;
        else if (strcmp(argv[i], "--profile-stages") == 0) profile = true, ++modes;
        else if (strcmp(argv[i], "--full-print") == 0) full = true, ++modes;
        else if (strcmp(argv[i], "--plain") == 0 && !plain) plain = true;
        else if (strcmp(argv[i], "--output") == 0 && !out_path && i + 1 < argc) out_path = argv[++i];
        else if (strcmp(argv[i], "--checkpoint") == 0 && !ckpt_path && i + 1 < argc) ckpt_path = argv[++i];
        else modes = 2;
    }
    if (modes > 1 || (out_path && (profile || full))) {
        usage(argv[0]);
        return 1;
    }
    FILE *out_file = nullptr;
    if (out_path) {
        out_file = fopen(out_path, "wb");
        if (!out_file) {
            fprintf(stderr, "cannot open %s\n", out_path);
            return 1;
        }
    }
    gpupi::PiRequest req;
    req.digits = requested;
    // --profile-stages lists the reference's stages: it runs the plain form
    req.plain = plain || profile;
    req.profile_stages = profile;
    req.checkpoint = ckpt_path;
    if (benchmark) req.copy_digits = std::min<uint32_t>(requested, 63u);
    else if (profile) req.copy_digits = std::min<uint32_t>(requested, 4096u);
    else if (full) req.copy_digits = requested;
    else req.copy_digits = 0u;   // streamed
    gpupi::PiOutput out;
    // Streamed digits (after the timed region).  In the default mode the first
    // chunk first prints the result line to stderr and "3" to stdout, the
    // order in which the reference prints them; --output sends "3<digits>" to
    // the file instead.
    struct Sink {
        FILE *f;
        const gpupi::PiOutput *out;
        uint32_t requested;
        bool announce;
        bool started;
    } sink{out_file ? out_file : stdout, &out, requested, !out_file && !benchmark, false};
    if (requested > 0u && (out_file || (!benchmark && !profile && !full))) {
        req.sink = [](const char *data, size_t n, void *user) {
            Sink *k = static_cast<Sink *>(user);
            if (!k->started) {
                if (k->announce)
                    fprintf(stderr, "target_digits=%u convert_digits=%u RET_len=%u elapsed_ms=%.3f\n", k->requested,
                            k->out->convert_digits, k->out->ret_len, k->out->elapsed_ms);
                fputc('3', k->f);
                k->started = true;
            }
            return fwrite(data, 1, n, k->f) == n;
        };
        req.sink_user = &sink;
    }
    const cudaError_t err = gpupi::pi_run(req, out);
    if (err != cudaSuccess) {
        fprintf(stderr, "pi_fractional failed: %s\n", cudaGetErrorString(err));
        if (out_file) fclose(out_file);
        return 1;
    }
    if (ckpt_path)
        fprintf(stderr, "checkpoint=%s %s\n", ckpt_path,
                out.checkpoint == 1 ? "loaded" : out.checkpoint == 2 ? "written" : "not-written");
    if (out_file) {
        if (!sink.started) fputc('3', out_file);
        fputc('\n', out_file);
        const bool ok = fclose(out_file) == 0;
        fprintf(stderr, "output=%s bytes=%llu output_ms=%.3f\n", out_path, (unsigned long long)requested + 2ull,
                out.output_ms);
        if (!ok) return 1;
    }
    const int ws_mb = (int)(out.workspace_bytes / (1024 * 1024));
    if (benchmark) {
        printf("target_digits=%u convert_digits=%u RET_len=%u elapsed_ms=%.3f workspace_max=%dMB\n", requested,
               out.convert_digits, out.ret_len, out.elapsed_ms, ws_mb);
        hex_preview("RET", out.ret.data(), out.ret_len);
        if (requested > 0u) {
            const uint32_t suffix = std::min<uint32_t>(requested, 64u);
            std::string tail = out.tail.empty() ? out.digits.substr(out.digits.size() - suffix) : out.tail;
            printf("DEC = 3%s...%.*s\n", out.digits.c_str(), (int)suffix, tail.c_str());
        } else {
            printf("DEC = 3\n");
        }
        return 0;
    }
    if (profile) {
        float leaf = 0, mul = 0, mul_small = 0, shift = 0, add = 0, sub = 0, compact = 0, exactdiv = 0,
              dpow = 0, dconv = 0, ntt = 0;
        for (size_t i = 0; i < out.stages.size(); ++i) {
            const gpupi::StageEntry &e = out.stages[i];
            if (!strcmp(e.kind, "leaf")) leaf += e.ms;
            else if (!strcmp(e.kind, "mul")) {
                mul += e.ms;
                if (e.uses_ntt) ntt += e.ms;
            } else if (!strcmp(e.kind, "mul_small")) mul_small += e.ms;
            else if (!strcmp(e.kind, "shift")) shift += e.ms;
            else if (!strcmp(e.kind, "add")) add += e.ms;
            else if (!strcmp(e.kind, "sub")) sub += e.ms;
            else if (!strcmp(e.kind, "compact")) compact += e.ms;
            else if (!strcmp(e.kind, "exactdiv")) exactdiv += e.ms;
            else if (!strcmp(e.kind, "decimal_powers")) dpow += e.ms;
            else if (!strcmp(e.kind, "decimal_convert")) dconv += e.ms;
            printf("stage[%03d] kind=%9s label=%18s digits=%8u batch=%8u lhs_len=%9u rhs_len=%9u kernel_ms=%6.3f "
                   "uses_ntt=%d\n",
                   (int)i, e.kind, e.label, e.n1, e.batch, e.lhs, e.rhs, e.ms, e.uses_ntt ? 1 : 0);
        }
        printf("leaf_total_ms=%.3f mul_total_ms=%.3f mul_small_total_ms=%.3f shift_total_ms=%.3f add_total_ms=%.3f "
               "sub_total_ms=%.3f compact_total_ms=%.3f exactdiv_total_ms=%.3f decimal_powers_total_ms=%.3f "
               "decimal_convert_total_ms=%.3f ntt_total_ms=%.3f\n",
               leaf, mul, mul_small, shift, add, sub, compact, exactdiv, dpow, dconv, ntt);
        const float acc = leaf + mul + mul_small + shift + add + sub + compact + exactdiv + dpow + dconv;
        printf("target_digits=%u convert_digits=%u RET_len=%u elapsed_ms=%.3f accounted_ms=%.3f workspace_max=%dMB\n",
               requested, out.convert_digits, out.ret_len, out.elapsed_ms, acc, ws_mb);
        hex_preview("RET", out.ret.data(), out.ret_len);
        if (requested > 0u)
            printf("DEC_preview_hash = %u\n", decimal_hash(out.digits.data(), (uint32_t)out.digits.size()));
        return 0;
    }
    if (!sink.started || !sink.announce)
        fprintf(stderr, "target_digits=%u convert_digits=%u RET_len=%u elapsed_ms=%.3f\n", requested,
                out.convert_digits, out.ret_len, out.elapsed_ms);
    if (full) {
        printf("RET = ");
        if (out.ret_len == 0) {
            printf("0\n");
        } else {
            for (int i = (int)out.ret_len - 1; i >= 0; --i) {
                if (i == (int)out.ret_len - 1) printf("%x", out.ret[i]);
                else printf("%08x", out.ret[i]);
            }
            printf("\n");
        }
        if (requested == 0u) {
            printf("DEC = 3\n");
        } else {
            printf("DEC = 3");
            fwrite(out.digits.data(), 1, requested, stdout);
            printf("\n");
        }
    } else if (out_file) {
        return 0;
    } else if (!sink.started) {
        fputc('3', stdout);
    }
    fputc('\n', stdout);
    return 0;
}
