// Raw batched addition (drop-in for gpupi batch_add.h:6-40).
// C = A + B over max(L_a, L_b) + 1 limbs, truncated or zero-extended to L_c.
// Rows are at X + i*stride_X.  C may alias A or B when the aliased operand has
// the same length and stride as C.  workspace: device scratch of at least
// batch_add_simple_workspace_size() bytes (may be null when that is 0).
#pragma once
#include <stddef.h>
#include <stdint.h>

void batch_add_simple(uint32_t *A, uint32_t *B, uint32_t *C, uint32_t *workspace, uint32_t N,
                      uint32_t L_a, uint32_t L_b, uint32_t L_c, uint32_t stride_A,
                      uint32_t stride_B, uint32_t stride_C);
size_t batch_add_simple_workspace_size(uint32_t N, uint32_t L_a, uint32_t L_b, uint32_t L_c);
