// Largest bit length / used limb count over a batch
// (drop-in for gpupi batch_bitlength.h:6-35).  Synchronous: returns the value
// on the host.
#pragma once
#include <stddef.h>
#include <stdint.h>

uint32_t batch_bitlength_max(const uint32_t *A, uint32_t *workspace, uint32_t N, uint32_t L,
                             uint32_t stride_A);
uint32_t batch_limblength_max(const uint32_t *A, uint32_t *workspace, uint32_t N, uint32_t L,
                              uint32_t stride_A);
size_t batch_bitlength_workspace_size(uint32_t N, uint32_t L);
