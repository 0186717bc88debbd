// Products that share forward transforms (mul_ntt.cu).
//
// A spectrum is the complete forward transform of N rows at one shape
// (N * M * 3 * K residues).  Operands transformed once serve every product
// they take part in, and a sum of products costs one inverse transform:
//   spectrum_forward(X) ; spectrum_forward(Y) ; ...
//   spectrum_inverse(sum_t X_t Y_t) -> limbs.
// The result is the exact integer sum, provided spectrum_sum_fits() holds
// for the operand lengths and the shape covers the output's L_c - 1
// coefficients (spectrum_shape(L_c - 1)).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "batch_mul_ntt.h"

namespace gpupi {

struct SpectrumShape {
    int log_k;   // K = 2^log_k points per coset
    int M;       // cosets; 0 = no shared-transform path for this size
};

// Shape for outputs of up to ncoef coefficients; M = 0 below 8192 points
// (one fused kernel per product) and above 20 * 2^25 points.
SpectrumShape spectrum_shape(uint64_t ncoef);
uint64_t spectrum_words(SpectrumShape s, uint32_t N);        // N * M * 3 * K
uint64_t spectrum_flag_words(uint32_t N, uint32_t Lc);       // carry flags of spectrum_inverse
// CRT capacity: sum_t min(La_t, Lb_t) (2^32 - 1)^2 < p0 p1 p2.
bool spectrum_sum_fits(const uint32_t *La, const uint32_t *Lb, int terms);

// FX (and FY when Y is not null) = forward transforms of N rows of X (Y);
// rows at X + i * sX, Lx limbs (zero above).
// rows = false: the column passes only (for spectrum_level_rows).
void spectrum_forward(const NTTPrecomputedTables &tables, SpectrumShape s, uint32_t N, const uint32_t *X,
                      uint64_t sX, uint32_t Lx, uint32_t *FX, const uint32_t *Y, uint64_t sY, uint32_t Ly,
                      uint32_t *FY, bool rows = true);
// An addend folded into the CRT and carry pass: C = product + (D << shift)
// (D rows at D + i * sD, Ld limbs); the product has ncoef coefficients and
// C's Lc limbs must hold the sum.  It replaces a separate shifted-addition
// pass (and the product's own buffer).
struct SpectrumAddend {
    const uint32_t *D;
    uint64_t sD;
    uint32_t Ld;
    uint32_t shift;
    uint32_t ncoef;
};

// C rows (stride sC, Lc limbs) = sum over terms (<= 2) of X_t Y_t (plus the
// addend when add is not null).  Fout receives the intermediate residues and
// may be one of the X_t / Y_t; flags: spectrum_flag_words(N, Lc) words.
// rows = false: Fout already holds the product after its inverse row pass
// (spectrum_level_rows); X and Y are not read.
void spectrum_inverse(const NTTPrecomputedTables &tables, SpectrumShape s, uint32_t N, int terms,
                      const uint32_t *const *X, const uint32_t *const *Y, uint32_t *Fout, uint32_t *C, uint64_t sC,
                      uint32_t Lc, uint32_t *flags, bool rows = true, const SpectrumAddend *add = nullptr);

// One merge level's row products from six column-transformed operands
// (spectrum_forward with rows = false): P' = P_e P_o into Fpo, R2 = P_e R_o
// into Fro, Q' = Q_e Q_o into Fqe, R1 = R_e Q_o into Fre, each after its
// inverse row pass; N rows of shape s.  Fpo null: no P' (five operands).
void spectrum_level_rows(const NTTPrecomputedTables &tables, SpectrumShape s, uint32_t N, uint32_t *Fpe,
                         uint32_t *Fpo, uint32_t *Fro, uint32_t *Fqo, uint32_t *Fqe, uint32_t *Fre);

}  // namespace gpupi
