// B = A shifted by a signed bit count (positive: left), truncated or
// zero-extended to L_out (drop-in for gpupi batch_shift.h:5-47).
// A and B must not overlap.
#pragma once
#include <stdint.h>

void batch_shift_bits(const uint32_t *A, uint32_t *B, uint32_t N, uint32_t L_in, uint32_t L_out,
                      uint32_t stride_in, uint32_t stride_out, int32_t shift_bits);

inline void batch_shift_left(const uint32_t *A, uint32_t *B, uint32_t N, uint32_t L_in,
                             uint32_t L_out, uint32_t stride_in, uint32_t stride_out,
                             uint32_t shift_bits) {
    batch_shift_bits(A, B, N, L_in, L_out, stride_in, stride_out, (int32_t)shift_bits);
}

inline void batch_shift_right(const uint32_t *A, uint32_t *B, uint32_t N, uint32_t L_in,
                              uint32_t L_out, uint32_t stride_in, uint32_t stride_out,
                              uint32_t shift_bits) {
    batch_shift_bits(A, B, N, L_in, L_out, stride_in, stride_out, -(int32_t)shift_bits);
}
