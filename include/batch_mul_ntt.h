// Batched exact product by number-theoretic transform
// (drop-in for gpupi batch_mul_ntt.h:5-40).
//
// The three table pointers are device buffers of the reference's sizes
// (65536, 65536 and 33 uint3 entries).  This library stores in them the
// twiddle and coset tables of its own three-prime transform, one prime per
// uint3 component; callers treat them as opaque.
#pragma once
#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime.h>

struct NTTPrecomputedTables {
    uint3 *roots_table_lv1;  // 65536 entries
    uint3 *roots_table_lv2;  // 65536 entries
    uint3 *inv2n_table;      // 33 entries
};

void init_ntt_precomputed_tables(NTTPrecomputedTables *tables);

// ret = A * B for N pairs; ret rows have L_a + L_b limbs.  workspace must hold
// batch_mul_ntt_workspace_size(N, L_a, L_b) bytes.  Product length up to 20 * 2^25 limbs
// (the reference stops at 2^28) with min(L_a, L_b) < 4.18e8 (CRT capacity).
void batch_mul_ntt(uint32_t *A, uint32_t *B, uint32_t *ret, uint32_t *workspace,
                   NTTPrecomputedTables tables, uint32_t N, uint32_t L_a, uint32_t L_b,
                   uint32_t stride_A, uint32_t stride_B, uint32_t stride_ret);
size_t batch_mul_ntt_workspace_size(uint32_t N, uint32_t L_a, uint32_t L_b);
