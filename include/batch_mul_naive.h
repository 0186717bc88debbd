// Batched schoolbook product ret = A * B over L_a + L_b limbs
// (drop-in for gpupi batch_mul_naive.h:5-25).  Requires L_a + L_b <=
// BATCH_MUL_NAIVE_L_MAX; batch_mp_mul picks this path only below its
// measured crossover.
#pragma once
#include <stdint.h>

const int BATCH_MUL_NAIVE_L_MAX = 1024;

void batch_mul_naive(uint32_t *A, uint32_t *B, uint32_t *ret, int N, int L_a, int L_b,
                     int stride_A, int stride_B, int stride_ret);
