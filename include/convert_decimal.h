// Divide-and-conquer binary -> decimal conversion of one fixed-point fraction
// (drop-in for gpupi convert_decimal.h:7-41).
#pragma once
#include <stdint.h>
#include "batch_arith.h"

struct ConvertDecimalPowerTable {
    BatchMPArray *powers;   // powers[l] = 5^(leaf_digits << l), one row each
    uint32_t levels;
    uint32_t leaf_digits;
};

cudaError_t convert_decimal_precompute_powers(BatchMPContext *ctx, ConvertDecimalPowerTable *table,
                                              uint32_t leaf_digits, uint32_t levels);
void convert_decimal_release_powers(ConvertDecimalPowerTable *table);

// X / 2^input_bits -> total_digits digits in natural order (output_digits[0]
// is the 10^-1 place).  total_digits == leaf_digits << levels.
cudaError_t convert_decimal_equal_split(BatchMPContext *ctx, BatchMPArray input, uint32_t input_bits,
                                        uint32_t total_digits, uint32_t leaf_digits,
                                        const ConvertDecimalPowerTable *table, char *output_digits);
