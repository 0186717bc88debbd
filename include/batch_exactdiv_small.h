// In-place exact division of N integers by one odd host limb, modulo
// 2^(32*L) (drop-in for gpupi batch_exactdiv_small.h:5-16).  L <= 128.
#pragma once
#include <stdint.h>

void batch_exactdiv_small(uint32_t *A, uint32_t B, uint32_t N, uint32_t L, uint32_t stride_A);
