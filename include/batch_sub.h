// Raw batched subtraction, C = A - B modulo 2^(32*L_c)
// (drop-in for gpupi batch_sub.h:6-36).  Aliasing rules as batch_add_simple.
#pragma once
#include <stddef.h>
#include <stdint.h>

void batch_sub_simple(uint32_t *A, uint32_t *B, uint32_t *C, uint32_t *workspace, uint32_t N,
                      uint32_t L_a, uint32_t L_b, uint32_t L_c, uint32_t stride_A,
                      uint32_t stride_B, uint32_t stride_C);
size_t batch_sub_simple_workspace_size(uint32_t N, uint32_t L_a, uint32_t L_b, uint32_t L_c);
