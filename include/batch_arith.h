// Batched multi-precision API (drop-in for gpupi batch_arith.h:8-152).
//
// A BatchMPArray is a view of N unsigned integers stored as little-endian
// 32-bit limbs in device memory: item i occupies data[i*stride .. i*stride+length).
// stride == 0 broadcasts a single row to every item.  Every entry point returns
// cudaErrorInvalidValue for malformed views (length > stride with stride != 0,
// mismatched batch sizes, null data with batch_size != 0) and otherwise the
// launch status.  Work is issued on the library's current stream (the legacy
// default stream unless gpupi_set_stream() changed it), so calls are ordered.
#pragma once

#include <stddef.h>
#include <stdint.h>

#include <cuda_runtime.h>

struct BatchMPContext;

struct BatchMPArray {
    uint32_t *data;
    uint32_t length;
    uint32_t batch_size;
    uint32_t stride;

    // Shrink length to the largest used limb count over the batch
    // (gpupi batch_arith.cu:415-424).  Synchronises with the device.
    cudaError_t compact(BatchMPContext *ctx);
};

// Device allocation of batch_size rows of `stride` limbs (stride 0 -> length).
// On failure data == nullptr.  (gpupi batch_arith.h:24-28)
BatchMPArray batch_mp_array_create(uint32_t batch_size, uint32_t length, uint32_t stride = 0);

// Frees storage returned by batch_mp_array_create.  (batch_arith.h:31)
void batch_mp_array_release(BatchMPArray array);

// Context: NTT twiddle tables plus one grow-only scratch workspace.
// (batch_arith.h:35-43)
BatchMPContext *batch_mp_init();
void batch_mp_destroy(BatchMPContext *ctx);
size_t batch_mp_workspace_size(const BatchMPContext *ctx);
cudaError_t batch_mp_ensure_workspace(BatchMPContext *ctx, size_t required_bytes);

// C = A * B exactly; requires C.length == A.length + B.length.  (batch_arith.h:48-53)
cudaError_t batch_mp_mul(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, BatchMPArray C);

// C = A * B (single host limb), truncated / zero-extended to C.length.  (:57-62)
cudaError_t batch_mp_mul_small(BatchMPContext *ctx, BatchMPArray A, uint32_t B, BatchMPArray C);

// A /= B in place, exact, modulo 2^(32*A.length); B odd, A.length <= 128.  (:67-71)
cudaError_t batch_mp_exactdiv_small(BatchMPContext *ctx, BatchMPArray A, uint32_t B);

// C = A + B truncated / zero-extended to C.length; C may alias A or B.  (:75-80)
cudaError_t batch_mp_add(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, BatchMPArray C);

// C = A + B (single host limb).  (:84-89)
cudaError_t batch_mp_add_small(BatchMPContext *ctx, BatchMPArray A, uint32_t B, BatchMPArray C);

// C = (A << shift) + B; C must not alias A or B.  (:94-100)
cudaError_t batch_mp_shift_add(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, uint32_t shift,
                               BatchMPArray C);

// C = (A << shift) - B modulo 2^(32*C.length); no aliasing.  (:105-111)
cudaError_t batch_mp_shift_sub(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, uint32_t shift,
                               BatchMPArray C);

// C = A - B modulo 2^(32*C.length).  (:115-120)
cudaError_t batch_mp_sub(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, BatchMPArray C);

// C = A - B (single host limb) modulo 2^(32*C.length).  (:124-129)
cudaError_t batch_mp_sub_small(BatchMPContext *ctx, BatchMPArray A, uint32_t B, BatchMPArray C);

// B = A shifted by a signed bit count (positive = left), truncated to B.length.  (:132-137)
cudaError_t batch_mp_shift_bits(BatchMPContext *ctx, BatchMPArray A, BatchMPArray B, int32_t shift_bits);

// Largest bit length / used limb count over the batch (host result).  (:140-151)
cudaError_t batch_mp_bitlength_max(BatchMPContext *ctx, BatchMPArray A, uint32_t *result);
cudaError_t batch_mp_limblength_max(BatchMPContext *ctx, BatchMPArray A, uint32_t *result);
