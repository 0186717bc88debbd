// C = (A << shift) + B, truncated or zero-extended to L_c; C must not alias
// A or B (drop-in for gpupi batch_shift_add.h:6-43).
#pragma once
#include <stddef.h>
#include <stdint.h>

void batch_shift_add_simple(const uint32_t *A, const uint32_t *B, uint32_t *C, uint32_t *workspace,
                            uint32_t shift, uint32_t N, uint32_t L_a, uint32_t L_b, uint32_t L_c,
                            uint32_t stride_A, uint32_t stride_B, uint32_t stride_C);
size_t batch_shift_add_simple_workspace_size(uint32_t N, uint32_t L_a, uint32_t L_b, uint32_t L_c,
                                             uint32_t shift);
