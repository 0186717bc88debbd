// C = A - B mod 2^(32*L_c) for a single host limb B
// (drop-in for gpupi batch_sub_small.h:6-33).
#pragma once
#include <stddef.h>
#include <stdint.h>

void batch_sub_small(const uint32_t *A, uint32_t B, uint32_t *C, uint32_t *workspace, uint32_t N,
                     uint32_t L_a, uint32_t L_c, uint32_t stride_A, uint32_t stride_C);
size_t batch_sub_small_workspace_size(uint32_t N, uint32_t L_a, uint32_t L_c);
