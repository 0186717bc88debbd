/* C ABI of gpupi_b200 (libgpupi_b200.so).
 *
 * Plain pointers and sizes only.  Every pointer named d_* is device memory;
 * h_* is host memory.  Functions return a cudaError_t value as int (0 =
 * success, 1 = cudaErrorInvalidValue for malformed arguments, 2 = allocation
 * failure).  Work is queued on the library's current stream
 * (gpupi_set_stream), the legacy default stream unless changed.
 *
 * Each batched entry point mirrors one gpupi function; the reference
 * declaration it replaces is cited beside it.  A batch item i of an operand X
 * lives at d_X + i*stride_X (stride 0 broadcasts item 0), exactly like
 * gpupi's BatchMPArray (batch_arith.h:10-22).
 */
#ifndef GPUPI_C_H
#define GPUPI_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gpupi_ctx gpupi_ctx; /* wraps BatchMPContext */

/* Library identification and launch accounting. */
const char *gpupi_version(void);
uint64_t gpupi_launch_count(void);
int gpupi_set_stream(void *cuda_stream);
int gpupi_device_sync(void);

/* batch_mp_init / batch_mp_destroy / batch_mp_workspace_size /
 * batch_mp_ensure_workspace (batch_arith.h:35-43) */
gpupi_ctx *gpupi_ctx_create(void);
void gpupi_ctx_destroy(gpupi_ctx *ctx);
size_t gpupi_ctx_workspace_size(const gpupi_ctx *ctx);
int gpupi_ctx_ensure_workspace(gpupi_ctx *ctx, size_t bytes);

/* batch_mp_mul (batch_arith.h:48-53): C = A * B, L_c must be L_a + L_b. */
int gpupi_mp_mul(gpupi_ctx *ctx, uint32_t N, const uint32_t *d_A, uint32_t L_a, uint32_t stride_A,
                 const uint32_t *d_B, uint32_t L_b, uint32_t stride_B, uint32_t *d_C, uint32_t L_c,
                 uint32_t stride_C);
/* batch_mp_add / batch_mp_sub (batch_arith.h:75-80, 115-120) */
int gpupi_mp_add(gpupi_ctx *ctx, uint32_t N, const uint32_t *d_A, uint32_t L_a, uint32_t stride_A,
                 const uint32_t *d_B, uint32_t L_b, uint32_t stride_B, uint32_t *d_C, uint32_t L_c,
                 uint32_t stride_C);
int gpupi_mp_sub(gpupi_ctx *ctx, uint32_t N, const uint32_t *d_A, uint32_t L_a, uint32_t stride_A,
                 const uint32_t *d_B, uint32_t L_b, uint32_t stride_B, uint32_t *d_C, uint32_t L_c,
                 uint32_t stride_C);
/* batch_mp_shift_add / batch_mp_shift_sub (batch_arith.h:94-111) */
int gpupi_mp_shift_add(gpupi_ctx *ctx, uint32_t N, const uint32_t *d_A, uint32_t L_a, uint32_t stride_A,
                       const uint32_t *d_B, uint32_t L_b, uint32_t stride_B, uint32_t shift, uint32_t *d_C,
                       uint32_t L_c, uint32_t stride_C);
int gpupi_mp_shift_sub(gpupi_ctx *ctx, uint32_t N, const uint32_t *d_A, uint32_t L_a, uint32_t stride_A,
                       const uint32_t *d_B, uint32_t L_b, uint32_t stride_B, uint32_t shift, uint32_t *d_C,
                       uint32_t L_c, uint32_t stride_C);
/* batch_mp_add_small / sub_small / mul_small (batch_arith.h:57-62, 84-89, 124-129) */
int gpupi_mp_add_small(gpupi_ctx *ctx, uint32_t N, const uint32_t *d_A, uint32_t L_a, uint32_t stride_A,
                       uint32_t b, uint32_t *d_C, uint32_t L_c, uint32_t stride_C);
int gpupi_mp_sub_small(gpupi_ctx *ctx, uint32_t N, const uint32_t *d_A, uint32_t L_a, uint32_t stride_A,
                       uint32_t b, uint32_t *d_C, uint32_t L_c, uint32_t stride_C);
int gpupi_mp_mul_small(gpupi_ctx *ctx, uint32_t N, const uint32_t *d_A, uint32_t L_a, uint32_t stride_A,
                       uint32_t b, uint32_t *d_C, uint32_t L_c, uint32_t stride_C);
/* batch_mp_exactdiv_small (batch_arith.h:67-71): in place, b odd, L_a <= 128 */
int gpupi_mp_exactdiv_small(gpupi_ctx *ctx, uint32_t N, uint32_t *d_A, uint32_t L_a, uint32_t stride_A,
                            uint32_t b);
/* batch_mp_shift_bits (batch_arith.h:132-137) */
int gpupi_mp_shift_bits(gpupi_ctx *ctx, uint32_t N, const uint32_t *d_A, uint32_t L_a, uint32_t stride_A,
                        uint32_t *d_B, uint32_t L_b, uint32_t stride_B, int32_t shift_bits);
/* batch_mp_bitlength_max / batch_mp_limblength_max (batch_arith.h:140-151) */
int gpupi_mp_bitlength_max(gpupi_ctx *ctx, uint32_t N, const uint32_t *d_A, uint32_t L_a, uint32_t stride_A,
                           uint32_t *h_result);
int gpupi_mp_limblength_max(gpupi_ctx *ctx, uint32_t N, const uint32_t *d_A, uint32_t L_a, uint32_t stride_A,
                            uint32_t *h_result);

/* batch_mul_naive (batch_mul_naive.h:16-25) and batch_mul_ntt
 * (batch_mul_ntt.h:24-40) called directly, bypassing the crossover. */
int gpupi_mul_naive(uint32_t N, const uint32_t *d_A, uint32_t L_a, uint32_t stride_A, const uint32_t *d_B,
                    uint32_t L_b, uint32_t stride_B, uint32_t *d_C, uint32_t stride_C);
int gpupi_mul_ntt(gpupi_ctx *ctx, uint32_t N, const uint32_t *d_A, uint32_t L_a, uint32_t stride_A,
                  const uint32_t *d_B, uint32_t L_b, uint32_t stride_B, uint32_t *d_C, uint32_t stride_C);

/* batch_mul_naive's operation (batch_mul_naive.h:16-25) on the tensor cores:
 * C = A * B for N pairs by split-integer int8 MMAs (tcgen05, INT32
 * accumulators; each 32-bit limb as four byte digits, exact).  Bit-identical
 * to gpupi_mul_naive.  min(L_a, L_b) <= 2048 and L_a + L_b <= 8192, both
 * nonzero; otherwise returns 1 (cudaErrorInvalidValue). */
int gpupi_mul_tc(uint32_t N, const uint32_t *d_A, uint32_t L_a, uint32_t stride_A, const uint32_t *d_B,
                 uint32_t L_b, uint32_t stride_B, uint32_t *d_C, uint32_t stride_C);
/* Reads and clears the tensor-core kernels' device error word: 1 when a
 * bounded wait for MMA completion ran out (the products are then
 * incomplete), 0 otherwise.  Synchronises with the device. */
int gpupi_tc_error(void);
/* Failure-detection self-test of the tensor-core kernel (no counterpart in
 * the reference): one small product whose CTA first waits on a barrier that
 * never completes.  The bounded wait runs out, the kernel records it
 * (*seen = 2), waits for its own MMAs, frees its tensor memory and returns;
 * an ordinary product right after it then leaves *after = 0 (the GPU and the
 * context stay usable).  No GPU fault is involved. */
int gpupi_tc_selftest_timeout(uint32_t *seen, uint32_t *after);

/* The splitting tree as a CUDA graph (no counterpart in the reference,
 * whose tree synchronises with the host at every compact()): for each
 * context, tree size and form, the first gpupi_pi_compute records the
 * length schedule, the second captures the tree into a graph, later ones
 * launch it and check the device's lengths against the schedule with one
 * copy (a mismatch runs the tree directly; results are always the exact
 * ones).  out5 = {schedules recorded, graphs captured, graph runs,
 * fallbacks after a mismatch, sizes where a graph was not possible}.
 * gpupi_tree_graph_perturb alters every recorded schedule so that the next
 * graph run exercises the fallback (testing).  GPUPI_TREE_GRAPH=0 in the
 * environment runs the tree directly. */
int gpupi_tree_graph_stats(uint64_t *out5);
int gpupi_tree_graph_perturb(void);

/* Error-path testing (no counterpart in the reference, whose allocations
 * are partly unchecked, pi_bs_gpu.cu:1199-1203): the nth following device
 * allocation whose category is in kind_mask fails once with
 * cudaErrorMemoryAllocation (returned as 2), on the host, without touching
 * the GPU.  Categories: 1 scratch arena, 2 context workspace growth,
 * 4 batch_mp_array_create.  nth = 0 disarms.  gpupi_scratch_live_bytes:
 * bytes of the scratch arenas currently handed out (0 when no call is in
 * progress and nothing leaked). */
int gpupi_fail_alloc(uint32_t kind_mask, uint32_t nth);
uint64_t gpupi_scratch_live_bytes(void);

/* Integer-pipe peaks of the current GPU (no counterpart in the reference):
 * warp instructions per second of 32-bit multiply-adds (IMAD, the
 * FMA-heavy pipe) and of three-input logic (LOP3, the ALU pipe), from
 * eight independent chains per thread on every SM, timed with CUDA events.
 * The ceiling the NTT and schoolbook kernels are measured against. */
int gpupi_int_peak(double *imad_winst_per_s, double *alu_winst_per_s);

/* Tune table (replaces the reference's compile-time BATCH_MUL_NAIVE_L_MAX,
 * batch_arith.cu:181, get_N_max and the NTT schedule tables,
 * batch_mul_ntt.cu:1781-1915): per length bucket, the product kernel
 * (CUDA-core schoolbook, tensor-core schoolbook or NTT) and the NTT's
 * transform shape (K points x M cosets).  Text lines
 *     mul <max_sum> school|tc|ntt
 *     ntt <min_need> <max_need> <log_k> <M>
 * ('#' comments).  Read at context creation from $GPUPI_TUNE_TABLE, else
 * tune_table.txt beside the library.  Results are bit-identical whatever the
 * table says.  load / load_text return the number of entries, or
 * -(line number) of the first malformed line (the table is then unchanged);
 * reset returns to the built-in rule; describe writes the table in effect.
 * gpupi_mul_kind: the kernel a product would use (0 schoolbook, 1 tensor
 * cores, 2 NTT; public_api = gpupi's batch_mp_mul rule).  gpupi_autotune
 * measures every candidate on the current GPU (batches of about
 * budget_limbs operand limbs), checks each candidate's product word for
 * word, writes the table to path and loads it. */
int gpupi_tune_load(const char *path);
int gpupi_tune_load_text(const char *text);
int gpupi_tune_reset(void);
size_t gpupi_tune_describe(char *buf, size_t cap);
int gpupi_mul_kind(uint32_t L_a, uint32_t L_b, int public_api);
/* Transform shape (2^log_k points x M cosets) of an NTT product of L_a x L_b
 * limbs under the table in effect (host only). */
int gpupi_ntt_shape(uint32_t L_a, uint32_t L_b, int *log_k, int *M);
int gpupi_autotune(gpupi_ctx *ctx, const char *path, uint64_t budget_limbs);

/* Ragged batch (no counterpart in the reference, whose batches share one
 * L_a / L_b): product i = A[offA[i] .. + L_a[i]) * B[offB[i] .. + L_b[i]) into
 * C[offC[i] .. + L_a[i] + L_b[i]).  d_A, d_B, d_C are device pointers; the
 * offset and length arrays are host arrays of N entries.  Products are bucketed
 * (schoolbook in one launch, NTT per transform size) so N uneven products cost
 * a few launches instead of N calls.  L_a[i] + L_b[i] <= 20 * 2^25, min(L_a[i], L_b[i]) <= 2^28. */
int gpupi_mp_mul_ragged(gpupi_ctx *ctx, uint32_t N, const uint32_t *d_A, const uint64_t *offA, const uint32_t *L_a,
                        const uint32_t *d_B, const uint64_t *offB, const uint32_t *L_b, uint32_t *d_C,
                        const uint64_t *offC);

/* batch_decimal_naive (batch_decimal_naive.h:23-31): LSD-first ASCII digits */
int gpupi_decimal_naive(uint32_t N, const uint32_t *d_A, uint32_t L_limb, uint32_t stride_A, char *d_out,
                        uint32_t L_dec, uint32_t stride_out);
/* convert_decimal_precompute_powers + convert_decimal_equal_split
 * (convert_decimal.h:16-41) in one call; d_out gets total_digits digits in
 * natural order. */
int gpupi_convert_decimal(gpupi_ctx *ctx, const uint32_t *d_X, uint32_t L_x, uint32_t input_bits,
                          uint32_t total_digits, uint32_t leaf_digits, char *d_out);

/* Whole pi_bs_gpu pipeline (pi_bs_gpu.cu:2073-2431, main_fractional).
 * h_ret (capacity ret_cap limbs) receives RET, h_digits (capacity digits_cap)
 * the first min(digits, digits_cap) decimal digits after "3."; both are
 * copied straight from the device (RET while the digits are still being
 * converted), so pinned memory makes those copies fastest.  Either
 * may be null.  info[0..7] receives: convert_digits, RET length, elapsed ms
 * on the device (float bits), workspace MB, number of profiled stages, leaf
 * digits, 0, 0.  flags bit 0 = profile every stage, bit 1 = keep RET and the
 * digits on the device (no host copies), bit 2 = plain form: the
 * reference's op sequence, one batched product per op (the default, tuned
 * form shares forward transforms within each merge level of the splitting
 * tree; both give the same RET and digits). */
int gpupi_pi_compute(gpupi_ctx *ctx, uint32_t digits, uint32_t flags, uint32_t *h_ret, size_t ret_cap,
                     char *h_digits, size_t digits_cap, uint32_t *info);

/* C = A B, or A B + D E when D is not null, through shared-transform
 * spectra: each operand's forward transform is computed once and the sum
 * costs one inverse transform (the building block of the tuned form of the
 * splitting tree).  N rows, each operand and C packed (stride = length);
 * Lc >= La + Lb (and >= Ld + Le + 1).  cudaErrorInvalidValue when the
 * product is below 8192 transform points, above 20 * 2^25, or when
 * min(La, Lb) + min(Ld, Le) limbs of 32-bit products would exceed the
 * three-prime CRT capacity.  No counterpart in the reference. */
int gpupi_mp_mul_spectra(gpupi_ctx *ctx, uint32_t N, const uint32_t *A, uint32_t La, const uint32_t *B,
                         uint32_t Lb, const uint32_t *D, uint32_t Ld, const uint32_t *E, uint32_t Le, uint32_t *C,
                         uint32_t Lc);

/* gpupi_pi_compute with a checkpoint file of the splitting tree's result
 * (Q and R, about 1 GB at 1e9 digits): when the file holds a valid result for
 * this digit count's tree (header, tree size and checksum match) it is loaded
 * and the tree is skipped, else the tree runs and the file is written
 * (through a temporary name, synced to the disk and renamed when complete).
 * info[7] = 1 loaded, 2 written, 3 not written (the file could not be
 * written; the computation still completes and returns 0).  No counterpart
 * in the reference. */
int gpupi_pi_compute_checkpointed(gpupi_ctx *ctx, uint32_t digits, uint32_t flags, const char *checkpoint,
                                  uint32_t *h_ret, size_t ret_cap, char *h_digits, size_t digits_cap,
                                  uint32_t *info);

/* Streamed digits: the same computation as gpupi_pi_compute, then the
 * first `digits` decimal digits after "3." handed to sink in order, in chunks
 * of at most `chunk` bytes (0: 64 MiB).  Each chunk's device-to-host copy
 * overlaps the sink call for the chunk before (two pinned buffers); a nonzero
 * return from sink stops the output.  info as for gpupi_pi_compute, with
 * info[6] = host milliseconds of the output (float bits).  flags bit 2 =
 * plain form.  No counterpart in the reference, whose CLI copies all digits
 * and then writes them. */
typedef int (*gpupi_digit_sink)(const char *data, size_t n, void *user);
int gpupi_pi_stream(gpupi_ctx *ctx, uint32_t digits, uint32_t flags, gpupi_digit_sink sink, void *user,
                    size_t chunk, uint32_t *info);

/* Per-kernel timing: CUDA events around each launch on the current stream,
 * with the launch's algorithmic HBM bytes.  The report has one line per
 * kernel family: "name launches total_ms total_bytes", then one line per
 * pair of consecutive families: "gap:prev>next count device_ms host_ms",
 * the device time between the end of one timed launch and the start of
 * the next, and the host time between recording the two. */
int gpupi_timer_enable(int on);
int gpupi_timer_reset(void);
size_t gpupi_timer_report(char *buf, size_t cap);

/* Cumulative host->device and device->host bytes copied by the library. */
int gpupi_transfer_bytes(uint64_t *h2d, uint64_t *d2h);

/* Scratch arena used for the library's temporaries (pipeline levels,
 * conversion buffers): device bytes held in arena blocks, the high-water mark
 * of live scratch bytes, and how many requests were ever served outside the
 * blocks (each such spill regrows the arena once its live bytes return to
 * zero; a repeated workload then adds none).  No counterpart in the
 * reference, which allocates per call. */
int gpupi_scratch_stats(uint64_t *block_bytes, uint64_t *high_water, uint64_t *spills);

/* Allocation-free batched addition: C = A + B exactly like gpupi_mp_add, but
 * without a context and without allocating.  It has no counterpart in the
 * reference.  It is for callers that cannot allocate device memory when they
 * need an add (all memory already handed to another allocator, or loops that
 * must not call cudaMalloc/cudaFree because those can synchronise the device).
 * The carry flags of long rows live in a fixed 256 KiB array inside the
 * library: N * ceil(L_c / 4096) must stay <= 65536 when rows take the
 * multi-tile path (fewer than 9472 rows of more than 4096 limbs), otherwise
 * the call returns 1 (cudaErrorInvalidValue) and does nothing.  The first
 * call on each device looks the array up (with that device current); make
 * that first call before starting any stream capture.  Calls share the
 * array: two calls whose kernels overlap on the GPU race. */
int gpupi_mp_add_noalloc(uint32_t N, const uint32_t *d_A, uint32_t L_a, uint32_t stride_A, const uint32_t *d_B,
                         uint32_t L_b, uint32_t stride_B, uint32_t *d_C, uint32_t L_c, uint32_t stride_C);

/* Multiply crossover: largest L_a + L_b computed by schoolbook (<= 1024). */
int gpupi_set_mul_crossover(uint32_t max_school_len);

/* BBP spot check of pi's hex digits, independent of the binary-splitting
 * pipeline (the north-star C5 check; no counterpart in the reference).
 * fractions[i] = floor(2^64 * frac(16^positions[i] * pi)) up to an error of
 * at most 8 * (positions[i] + 17) units (integer fixed point, host arrays),
 * so hex digits positions[i] + 1, ... of pi can be compared with RET where
 * that bound cannot flip them.  positions[i] <= 2^30. */
int gpupi_bbp_fractions(const uint64_t *positions, uint32_t count, uint64_t *fractions);

#ifdef __cplusplus
}
#endif

#endif
