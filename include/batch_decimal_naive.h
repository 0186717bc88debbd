// Fixed-point fraction X / 2^(32*L_limb) -> L_dec truncated decimal digits per
// row, written least significant first as ASCII (the first byte is the
// 10^-L_dec place) (drop-in for gpupi batch_decimal_naive.h:5-31).
#pragma once
#include <stdint.h>

constexpr int BATCH_DECIMAL_NAIVE_L_LIMB_MAX = 2047;

void batch_decimal_naive(const uint32_t *A, char *B, uint32_t N, int L_limb, uint32_t stride_A,
                         int L_dec, uint32_t stride_B);
