// Internal interface of the pi pipeline driver (pi_engine.cu).
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

#include "batch_arith.h"
#include "batch_mul_ntt.h"

struct ConvertDecimalPowerTable;

namespace gpupi {

struct StageEntry {
    const char *kind;
    const char *label;
    uint32_t n1, batch, lhs, rhs;
    float ms;
    bool uses_ntt;
};

struct PiRequest {
    uint32_t digits = 0;            // requested decimal digits after the point
    bool profile_stages = false;    // time every op (serialises the run)
    uint32_t copy_digits = 0;       // how many leading digits to copy to the host
    BatchMPContext *ctx = nullptr;  // reuse a context (keeps its workspace); null = private
    bool device_only = false;       // leave RET and the digits on the device (no host copies)
    char *host_digits = nullptr;    // caller buffer (>= copy_digits bytes, may be pinned) for the digits
    uint32_t *host_ret = nullptr;   // caller buffer for RET (copied while the digits are converted)
    size_t host_ret_cap = 0;        // its capacity in limbs
    bool plain = false;             // the reference's op sequence; default: shared forward transforms (same results)
    // Streamed digit output: after the timed region the requested digits are
    // handed to sink in order, in chunks of at most sink_chunk bytes; each
    // chunk's device-to-host copy (two pinned buffers, one copy stream)
    // overlaps the sink call of the chunk before.  A false return stops.
    bool (*sink)(const char *data, size_t n, void *user) = nullptr;
    void *sink_user = nullptr;
    size_t sink_chunk = (size_t)64 << 20;
    // Checkpoint file of the splitting tree's result: loaded (and the tree
    // skipped) when it holds a valid result for this digit count's tree,
    // else written after the tree.  Null: none.
    const char *checkpoint = nullptr;
};

struct PiOutput {
    uint32_t target_digits = 0;
    uint32_t convert_digits = 0;
    uint32_t ret_len = 0;
    float elapsed_ms = 0.f;
    float output_ms = 0.f;          // host time of the streamed output (sink set)
    int checkpoint = 0;             // 1: tree loaded from the checkpoint, 2: tree computed and saved
    size_t workspace_bytes = 0;
    std::vector<uint32_t> ret;      // RET limbs (little endian)
    std::string digits;             // first copy_digits digits (unless PiRequest::host_digits)
    std::string tail;               // last 64 requested digits when not all were copied
    std::vector<StageEntry> stages;
};

cudaError_t pi_run(const PiRequest &req, PiOutput &out);
uint32_t round_up_decimal_digits(uint32_t requested, uint32_t *leaf_out);
uint32_t prec_limbs_for_digits(uint32_t digits);

// convert_decimal_equal_split in 2^log_chunks parts, each part's digits
// announced to ready(offset, count, user) as soon as they are issued on the
// current stream (decimal.cu).
cudaError_t convert_decimal_in_parts(BatchMPContext *ctx, BatchMPArray input, uint32_t input_bits,
                                     uint32_t total_digits, uint32_t leaf_digits,
                                     const ConvertDecimalPowerTable *table, char *output_digits,
                                     uint32_t log_chunks, void (*ready)(size_t, size_t, void *), void *user);

cudaError_t mul_ntt_direct(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, BatchMPArray C);
// batch_mp_mul with this library's schoolbook/NTT crossover (school_max()).
cudaError_t mul_tuned(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, BatchMPArray C);
const NTTPrecomputedTables &context_tables(const BatchMPContext *ctx);
const void *context_workspace(const BatchMPContext *ctx);
void pi_forget_context(const BatchMPContext *ctx);
// The splitting tree as a CUDA graph: counts of runs that recorded the
// length schedule, captured the graph, replayed it, fell back after the
// device's lengths disagreed with the schedule, and of sizes where no graph
// was possible; perturb alters every recorded schedule (tests of the
// fallback).
struct TreeGraphStats {
    uint64_t recorded, captured, replayed, fallbacks, disabled;
};
TreeGraphStats tree_graph_stats();
void tree_graph_perturb();
void set_school_max(uint32_t v);
uint32_t school_max();

}  // namespace gpupi
