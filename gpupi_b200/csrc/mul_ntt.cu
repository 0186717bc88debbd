// Batched exact multiplication by three-prime NTT (gpupi batch_mul_ntt.cu;
// API batch_mul_ntt.h:24-40).
//
// Shape.  A product of L_c = L_a + L_b limbs is a cyclic convolution of
// M * K points, K = 2^k <= 2^25, M <= 20, M * K >= L_a + L_b - 1.  M = 1 for
// products up to 2^25 points.  Longer products are split into M cosets:
// with c_i = g^(iK) (g a generator, i < M) the residues
// C_i = A B mod (x^K - c_i) are K-point cyclic convolutions of the twisted
// inputs (A mod (x^K - c_i))(g^i x), and the M blocks of K coefficients of
// C = A B follow from C_i = sum_b C_b c_i^b by the inverse Vandermonde
// matrix of the nodes c_i.
//
// Workspace: F[vrow][q][K] residues (vrow = row * M + coset), one such array
// for A (FA) and one for B (FB; none when B is A, one row when B is
// broadcast), then the CRT tile flags.
//
// Passes (four-step decomposition K = R1 [* R2] * C, C = 4096):
//   k_cols_r<first>   load limbs (fold + twist for cosets), R1-point DIF
//                     down each column of a 4096-residue tile, twist by
//                     w_K^(col * bitrev(pos)), store
//   k_cols_r          same on each segment for R2 (sizes above 2^21)
//   k_rows_r          C-point DIF of the A and B segments, pointwise product
//                     * K^-1, C-point inverse DIT, store
//   k_cols_r<inv>     untwist + inverse DIT on columns, mirror order
//   k_combine<M>      (M > 1) untwist the cosets, inverse Vandermonde
//   k_crt             Garner CRT to 96-bit coefficients, carry into limbs
//                     (+ carry_fixup_kernel when a row spans several tiles)
// Small products (K <= 4096) are one k_rows_r (or k_rows_small) launch and
// k_crt.  Every CTA handles one prime, fixed at compile time inside the CTA;
// the prime is the slowest grid index, so an SM works on one prime's tables
// and code at a time.
#include "ntt_core.cuh"
#include "carry_tile.cuh"
#include "batch_mul_ntt.h"
#include "spectrum.h"

#include <stdio.h>
#include <stdlib.h>
#include <vector>

namespace gpupi {
namespace ntt {

static const uint32_t kP[kPrimes] = {Prime<0>::p, Prime<1>::p, Prime<2>::p};
static const uint32_t kGen[kPrimes] = {Prime<0>::g, Prime<1>::g, Prime<2>::g};

struct NttParams {
    Tables tab;
};

// ---------------------------------------------------------------------------
// Host modular helpers (table construction, coset matrices)
// ---------------------------------------------------------------------------
static uint32_t h_mul(uint32_t a, uint32_t b, uint32_t p) { return (uint32_t)((uint64_t)a * b % p); }
static uint32_t h_pow(uint32_t a, uint64_t e, uint32_t p) {
    uint32_t r = 1u % p;
    a %= p;
    while (e) {
        if (e & 1u) r = h_mul(r, a, p);
        a = h_mul(a, a, p);
        e >>= 1;
    }
    return r;
}
static uint32_t h_inv(uint32_t a, uint32_t p) { return h_pow(a, p - 2u, p); }
static uint32_t h_mont(uint32_t x, uint32_t p) { return (uint32_t)(((uint64_t)x << 32) % p); }

static NttParams make_params(const NTTPrecomputedTables &t) {
    NttParams P{};
    const uint32_t *lv1 = reinterpret_cast<const uint32_t *>(t.roots_table_lv1);
    const uint32_t *lv2 = reinterpret_cast<const uint32_t *>(t.roots_table_lv2);
    P.tab.root_lo = reinterpret_cast<const uint2 *>(lv1);
    P.tab.root_hi = reinterpret_cast<const uint2 *>(lv1 + kRootLoWords);
    P.tab.level = reinterpret_cast<const uint2 *>(lv1 + kLevelOffset);
    P.tab.coset_lo = lv2;
    P.tab.coset_hi = lv2 + kCosetWords;
    P.tab.inv2n = reinterpret_cast<const uint32_t *>(t.inv2n_table);
    return P;
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
constexpr int kThreads = 256;
constexpr int kTile = 4096;                    // residues per register-stage CTA tile
constexpr int kTilePad = kTile + kTile / 32;   // padded shared-memory words

// Grid index -> (prime, index within that prime's third of the grid).
__device__ __forceinline__ int grid_prime(uint64_t &b) {
    const uint32_t per = gridDim.x / kPrimes;
    const int q = (int)(blockIdx.x / per);
    b = blockIdx.x - (uint32_t)q * per;
    return q;
}

struct ColsArgs {
    const uint32_t *X;   // limbs (first forward pass only)
    uint64_t sX;
    uint32_t Lx;
    uint32_t nb;         // K-limb blocks of X folded into each coset (first pass)
    uint32_t *F;         // workspace of this operand: F[vrow][q][K]
    int log_k, log_s;
    int M;               // cosets per row
    // second operand of a paired forward pass (same shape, same tile)
    const uint32_t *X2;
    uint64_t sX2;
    uint32_t Lx2;
    uint32_t nb2;
    uint32_t *F2;
};

// Offset of element j from element 0 in a LO = 0 stage with 2^B-point groups
// (LOG_R >= 4): j = g 2^B + v sits at pos_0 + v + g 2^(LOG_R - 4 + B), bits
// disjoint from those of pos_0.
__host__ __device__ constexpr uint32_t stage_delta(int j, int B, int log_r) {
    return ((uint32_t)j & ((1u << B) - 1u)) + (((uint32_t)j >> B) << (log_r - 4 + B));
}

// Twist the 16 residues of stage S (the LO = 0 stage: last forward, first
// inverse) by w_S^(col * bitrev(pos)) or its inverse, E = colsh * bitrev(pos)
// with colsh = col << shift; with PAIR the same factors twist y as well.
// For LOG_R >= 4 the column is the same for all 16 residues and
// bitrev(pos_j) = bitrev(pos_0) + sum over the set bits i of j of
// bitrev(delta_(2^i)), so the 16 factors are the subset products of w^(E_0)
// and four D_i = w^(colsh bitrev(delta_(2^i))): five table lookups and
// fifteen products instead of sixteen scattered lookup pairs.
template <class S, int LOG_R, int Q, bool PAIR>
__device__ __forceinline__ void twist16(uint32_t (&x)[16], uint32_t (&y)[16], uint32_t t, uint32_t c0, int shift,
                                        const uint2 *lo, const uint2 *hi) {
    if constexpr (LOG_R >= 4) {
        constexpr int B = S::kB;
        static_assert(S::kLO == 0, "twist stage");
        uint32_t pos0, c;
        S::elem(t, 0, pos0, c);
        const uint32_t colsh = (c0 + c) << shift;
        uint32_t F[16];
        F[0] = root_m<Q>(lo, hi, colsh * bitrev(pos0, LOG_R));
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const uint32_t D = root_m<Q>(lo, hi, colsh * crev(stage_delta(1 << i, B, LOG_R), LOG_R));
#pragma unroll
            for (int k = 0; k < (1 << i); ++k) F[(1 << i) + k] = mont<Q>(F[k], D);   // lazy, < 2p
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            x[j] = norm<Q>(mont<Q>(x[j], F[j]));
            if (PAIR) y[j] = norm<Q>(mont<Q>(y[j], F[j]));
        }
    } else {
        // short columns: the 16 residues span several columns
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            uint32_t pos, c;
            S::elem(t, j, pos, c);
            const uint32_t E = ((c0 + c) << shift) * bitrev(pos, LOG_R);
            x[j] = mul_root<Q>(x[j], lo, hi, E);
            if (PAIR) y[j] = mul_root<Q>(y[j], lo, hi, E);
        }
    }
}

// The 16 first-pass residues of one operand (limbs, folded into coset
// `coset` and twisted by g^(coset i) when the row is split into cosets).
template <class First, int LOG_R, int Q>
__device__ __forceinline__ void load_limbs(const ColsArgs &a, uint32_t (&x)[16], const uint32_t *xr, uint32_t Lx,
                                           uint32_t nb, uint64_t K, int log_cols, uint32_t c0, uint32_t t,
                                           int coset, uint32_t cm, const uint32_t *clo, const uint32_t *chi) {
    if (a.M == 1) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            uint32_t pos, c;
            First::elem(t, j, pos, c);
            const uint64_t i = ((uint64_t)pos << log_cols) + c0 + c;
            x[j] = (i < Lx) ? reduce_limb<Q>(__ldg(xr + i)) : 0u;
        }
        return;
    }
    // X mod (x^K - c): Horner over the K-limb blocks, top block first, the
    // 16 loads of a block issued together
#pragma unroll
    for (int j = 0; j < 16; ++j) x[j] = 0u;
    for (int blk = (int)nb - 1; blk >= 0; --blk) {
        uint32_t v[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            uint32_t pos, c;
            First::elem(t, j, pos, c);
            const uint64_t i = ((uint64_t)pos << log_cols) + c0 + c + (uint64_t)blk * K;
            v[j] = (i < Lx) ? __ldg(xr + i) : 0u;
        }
#pragma unroll
        for (int j = 0; j < 16; ++j)
            x[j] = add_n<Q>(coset ? norm<Q>(mont<Q>(x[j], cm)) : x[j], reduce_limb<Q>(v[j]));
    }
    if (coset) {
        // twist by g^(coset i).  For LOG_R >= 4 the 16 residues of a thread sit
        // at i_0 + v 2^(LO + log_cols) (one group), so the factors are
        // g^(coset i_0) D^v with D = g^(coset 2^(LO + log_cols)), the same for
        // the whole CTA: two lookup pairs and fifteen products.
        if constexpr (LOG_R >= 4) {
            static_assert(First::kB == 4, "one group per thread");
            uint32_t pos, c;
            First::elem(t, 0, pos, c);
            const uint32_t i0 = (uint32_t)(((uint64_t)pos << log_cols) + c0 + c);
            uint32_t f = mul_coset<Q, 0>(PrimeC<Q>::r1, clo, chi, (uint32_t)coset * i0);
            const uint32_t d = mul_coset<Q, 0>(PrimeC<Q>::r1, clo, chi, (uint32_t)coset << (First::kLO + log_cols));
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                x[j] = norm<Q>(mont<Q>(x[j], f));
                f = mont<Q>(f, d);   // lazy, < 2p
            }
        } else {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                uint32_t pos, c;
                First::elem(t, j, pos, c);
                const uint32_t i = (uint32_t)(((uint64_t)pos << log_cols) + c0 + c);
                x[j] = mul_coset<Q, 0>(x[j], clo, chi, (uint32_t)coset * i);
            }
        }
    }
}

// Column pass: R = 2^LOG_R (<= 512) points per column, TC = 4096 / R columns
// per CTA; segment of S = 2^log_s points viewed as [R][S/R].  PAIR: the
// forward pass of A and B together (same tile, shared twiddles and twists).
template <int LOG_R, bool FROM_LIMBS, bool INVERSE, bool PAIR, int Q>
__device__ __forceinline__ void cols_body(const NttParams &P, const ColsArgs &a, uint64_t b, uint32_t *Sm,
                                          uint32_t *Sm2, uint2 *tw) {
    constexpr int LOG_TC = 12 - LOG_R;
    constexpr int NS = StagePlan<LOG_R>::n;
    using First = typename ExecStage<LOG_R, LOG_TC, INVERSE, 0>::S;
    using Last = typename ExecStage<LOG_R, LOG_TC, INVERSE, NS - 1>::S;
    const int log_cols = a.log_s - LOG_R;
    const uint32_t ctiles = 1u << (log_cols - LOG_TC);
    const uint32_t nseg = 1u << (a.log_k - a.log_s);
    uint32_t ct, seg;
    uint64_t vrow;
    if constexpr (FROM_LIMBS) {
        // virtual row fastest: the cosets of one tile run back to back and
        // share its limbs in L2 (the first pass covers the whole transform)
        const uint64_t vrows = (gridDim.x / kPrimes) / ctiles;
        vrow = b % vrows;
        ct = (uint32_t)(b / vrows);
        seg = 0u;
    } else {
        ct = (uint32_t)(b % ctiles);
        b /= ctiles;
        seg = (uint32_t)(b % nseg);
        vrow = b / nseg;
    }
    const int dir = INVERSE ? 1 : 0;
    const uint64_t K = 1ull << a.log_k;
    const uint2 *twhi = root_hi_ptr(P.tab, dir, Q);
    const uint2 *twlo = root_lo_ptr(P.tab, dir, Q);
    const uint2 *lev = level_ptr(P.tab, dir, Q);
    for (uint32_t e = threadIdx.x; e < (1u << LOG_R) - 1u; e += kThreads) tw[e] = __ldg(lev + e);
    const uint64_t off = vrow * 3 * K + (uint64_t)Q * K + ((uint64_t)seg << a.log_s);
    uint32_t *F = a.F + off;
    uint32_t *F2 = PAIR ? a.F2 + off : nullptr;
    const uint32_t c0 = ct << LOG_TC;
    const int twist_shift = kMaxLog - a.log_s;
    const uint32_t t = threadIdx.x;
    uint32_t x[16], y[16];
    if constexpr (FROM_LIMBS) {
        const uint64_t row = vrow / (uint32_t)a.M;
        const int coset = (int)(vrow - row * (uint32_t)a.M);
        const uint32_t *clo = coset_lo_ptr(P.tab, 0, Q);
        const uint32_t *chi = coset_hi_ptr(P.tab, 0, Q);
        // coset node c = g^(coset K), Montgomery form
        const uint32_t cm = (a.M > 1) ? mul_coset<Q, 0>(PrimeC<Q>::r1, clo, chi, (uint32_t)coset << a.log_k) : 0u;
        load_limbs<First, LOG_R, Q>(a, x, a.X + row * a.sX, a.Lx, a.nb, K, log_cols, c0, t, coset, cm, clo, chi);
        if constexpr (PAIR)
            load_limbs<First, LOG_R, Q>(a, y, a.X2 + row * a.sX2, a.Lx2, a.nb2, K, log_cols, c0, t, coset, cm, clo,
                                        chi);
    } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            uint32_t pos, c;
            First::elem(t, j, pos, c);
            const uint64_t i = ((uint64_t)pos << log_cols) + c0 + c;
            x[j] = F[i];
            if constexpr (PAIR) y[j] = F2[i];
        }
        if constexpr (INVERSE) twist16<First, LOG_R, Q, PAIR>(x, y, t, c0, twist_shift, twlo, twhi);
    }
    __syncthreads();   // twiddle table ready
    run_stages_pair<LOG_R, LOG_TC, INVERSE, Q, 0, PAIR>(x, y, Sm, Sm2, t, tw);
    if constexpr (!INVERSE) twist16<Last, LOG_R, Q, PAIR>(x, y, t, c0, twist_shift, twlo, twhi);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        uint32_t pos, c;
        Last::elem(t, j, pos, c);
        const uint64_t i = ((uint64_t)pos << log_cols) + c0 + c;
        F[i] = x[j];
        if constexpr (PAIR) F2[i] = y[j];
    }
}

template <int LOG_R, bool PAIR>
constexpr size_t cols_smem_bytes() {   // one or two padded tiles + the twiddle levels
    return (size_t)(PAIR ? 2 : 1) * kTilePad * 4u + (size_t)((1 << LOG_R) - 1) * 8u;
}

// Four CTAs per SM for every pass (64 registers): the paired passes hold two
// operands' residues, and for the first of them a few words spill, but the
// extra resident warps hide more of the limb and tile latency (first pass of
// a 2^24 x 2^24-limb product 0.589 -> 0.541 ms against three CTAs per SM).
template <int LOG_R, bool FROM_LIMBS, bool INVERSE, bool PAIR>
__global__ void __launch_bounds__(kThreads, 4) k_cols_r(NttParams P, ColsArgs a) {
    extern __shared__ uint4 cols_smem[];
    uint32_t *Sm = reinterpret_cast<uint32_t *>(cols_smem);
    uint32_t *Sm2 = PAIR ? Sm + kTilePad : Sm;
    uint2 *tw = reinterpret_cast<uint2 *>(Sm + (PAIR ? 2 : 1) * kTilePad);
    uint64_t b;
    const int q = grid_prime(b);
    if (q == 0)
        cols_body<LOG_R, FROM_LIMBS, INVERSE, PAIR, 0>(P, a, b, Sm, Sm2, tw);
    else if (q == 1)
        cols_body<LOG_R, FROM_LIMBS, INVERSE, PAIR, 1>(P, a, b, Sm, Sm2, tw);
    else
        cols_body<LOG_R, FROM_LIMBS, INVERSE, PAIR, 2>(P, a, b, Sm, Sm2, tw);
}

struct RowsArgs {
    const uint32_t *A;   // limbs (FROM_LIMBS)
    uint64_t sA;
    uint32_t La;
    const uint32_t *B;
    uint64_t sB;
    uint32_t Lb;
    uint32_t *FA;
    const uint32_t *FB;
    int log_k;
    int M;               // cosets per row
    int b_bcast;         // B row 0 serves every row
    int square;          // B is A
};

// Fused row pass on C = 2^LOG_C points (T = C/16 threads): forward stages of
// A then B (A stays in registers while B reuses the shared tile), pointwise
// product * scale, inverse stages.  The last forward and the first inverse
// stage share one thread mapping, so the product never leaves registers.
// The forward twiddle levels are replaced by the inverse ones in the same
// shared buffer once the forward stages are done.
template <int LOG_C, bool FROM_LIMBS, int Q>
__device__ __forceinline__ void rows_body(const NttParams &P, const RowsArgs &a, uint64_t b, uint32_t *Sm,
                                          uint2 *tw) {
    constexpr int C = 1 << LOG_C;
    constexpr int T = C / 16;
    constexpr int NS = StagePlan<LOG_C>::n;
    using First = typename ExecStage<LOG_C, 0, false, 0>::S;
    using Out = typename ExecStage<LOG_C, 0, true, NS - 1>::S;
    const uint32_t nseg = 1u << (a.log_k - LOG_C);
    const uint32_t seg = (uint32_t)(b % nseg);
    const uint64_t vrow = b / nseg;
    const uint64_t brow = a.b_bcast ? (vrow % (uint32_t)a.M) : vrow;
    const uint64_t K = 1ull << a.log_k;
    const uint32_t scale = __ldg(P.tab.inv2n + a.log_k * kPrimes + Q);
    const uint2 *levf = level_ptr(P.tab, 0, Q);
    const uint2 *levi = level_ptr(P.tab, 1, Q);
    for (uint32_t e = threadIdx.x; e < C - 1; e += T) tw[e] = __ldg(levf + e);
    const uint64_t offA = vrow * 3 * K + (uint64_t)Q * K + ((uint64_t)seg << LOG_C);
    const uint64_t offB = brow * 3 * K + (uint64_t)Q * K + ((uint64_t)seg << LOG_C);
    const uint32_t t = threadIdx.x;
    uint32_t xa[16], xb[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        uint32_t pos, c;
        First::elem(t, j, pos, c);
        if (FROM_LIMBS) {
            xa[j] = (pos < a.La) ? reduce_limb<Q>(__ldg(a.A + vrow * a.sA + pos)) : 0u;
            xb[j] = (!a.square && pos < a.Lb) ? reduce_limb<Q>(__ldg(a.B + brow * a.sB + pos)) : 0u;
        } else {
            xa[j] = a.FA[offA + pos];
            xb[j] = a.square ? 0u : a.FB[offB + pos];
        }
    }
    __syncthreads();
    // A then B through one copy of the forward stages (a loop, not two
    // copies: smaller code for the instruction cache); B waits in xb and
    // trades places with the transformed A between the passes.  A and B one
    // after the other: a second tile would cost a CTA per SM.
#pragma unroll 1
    for (int op = 0; op < (a.square ? 1 : 2); ++op) {
        if (op) {
            // the tile is free again: every thread has passed the last stage's loads
            __syncthreads();
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const uint32_t v = xa[j];
                xa[j] = xb[j];
                xb[j] = v;
            }
        }
        run_stages<LOG_C, 0, false, Q, 0>(xa, Sm, t, tw);
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const uint32_t y = a.square ? xa[j] : xb[j];
        xa[j] = norm<Q>(mont<Q>(mont<Q>(xa[j], y), scale));   // x y K^-1
    }
    __syncthreads();   // forward twiddles and tile no longer read
    for (uint32_t e = threadIdx.x; e < C - 1; e += T) tw[e] = __ldg(levi + e);
    __syncthreads();
    run_stages<LOG_C, 0, true, Q, 0>(xa, Sm, t, tw);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        uint32_t pos, c;
        Out::elem(t, j, pos, c);
        a.FA[offA + pos] = xa[j];
    }
}

template <int LOG_C>
constexpr size_t rows_smem_bytes() {   // the padded tile + the twiddle levels
    return (size_t)((1 << LOG_C) + (1 << LOG_C) / 32) * 4u + (size_t)((1 << LOG_C) - 1) * 8u;
}

template <int LOG_C, bool FROM_LIMBS>
__global__ void __launch_bounds__((1 << LOG_C) / 16, LOG_C == 12 ? 4 : 1) k_rows_r(NttParams P, RowsArgs a) {
    extern __shared__ uint4 rows_smem[];
    constexpr int C = 1 << LOG_C;
    uint32_t *Sm = reinterpret_cast<uint32_t *>(rows_smem);
    uint2 *tw = reinterpret_cast<uint2 *>(Sm + C + C / 32);
    uint64_t b;
    const int q = grid_prime(b);
    if (q == 0)
        rows_body<LOG_C, FROM_LIMBS, 0>(P, a, b, Sm, tw);
    else if (q == 1)
        rows_body<LOG_C, FROM_LIMBS, 1>(P, a, b, Sm, tw);
    else
        rows_body<LOG_C, FROM_LIMBS, 2>(P, a, b, Sm, tw);
}

// Whole product of K <= 2^8 points per CTA (one prime, one row), radix-2
// levels in shared memory.
constexpr int kSmallLog = 8;

template <int Q>
__device__ __forceinline__ void rows_small_body(const NttParams &P, const RowsArgs &a, uint64_t row,
                                                uint32_t *SA, uint32_t *SB, uint2 *twf, uint2 *twi) {
    const int log_k = a.log_k;
    const uint32_t K = 1u << log_k;
    const uint64_t brow = a.b_bcast ? 0u : row;
    const uint32_t scale = __ldg(P.tab.inv2n + log_k * kPrimes + Q);
    const uint2 *levf = level_ptr(P.tab, 0, Q) + (K / 2 - 1u);   // top level: w_K^e, e < K/2
    const uint2 *levi = level_ptr(P.tab, 1, Q) + (K / 2 - 1u);
    for (uint32_t e = threadIdx.x; e < K / 2; e += blockDim.x) {
        twf[e] = __ldg(levf + e);
        twi[e] = __ldg(levi + e);
    }
    for (uint32_t i = threadIdx.x; i < K; i += blockDim.x) {
        SA[i] = (i < a.La) ? reduce_limb<Q>(__ldg(a.A + row * a.sA + i)) : 0u;
        SB[i] = (!a.square && i < a.Lb) ? reduce_limb<Q>(__ldg(a.B + brow * a.sB + i)) : 0u;
    }
    __syncthreads();
    tile_transform<Q, false>(SA, log_k, 0, twf);
    if (!a.square) tile_transform<Q, false>(SB, log_k, 0, twf);
    for (uint32_t i = threadIdx.x; i < K; i += blockDim.x) {
        const uint32_t x = SA[i];
        const uint32_t y = a.square ? x : SB[i];
        SA[i] = norm<Q>(mont<Q>(mont<Q>(x, y), scale));
    }
    __syncthreads();
    tile_transform<Q, true>(SA, log_k, 0, twi);
    for (uint32_t i = threadIdx.x; i < K; i += blockDim.x) a.FA[row * 3 * K + (uint64_t)Q * K + i] = SA[i];
}

__global__ void __launch_bounds__(128) k_rows_small(NttParams P, RowsArgs a) {
    __shared__ uint32_t SA[1 << kSmallLog], SB[1 << kSmallLog];
    __shared__ uint2 twf[1 << (kSmallLog - 1)], twi[1 << (kSmallLog - 1)];
    uint64_t row;
    const int q = grid_prime(row);
    if (q == 0)
        rows_small_body<0>(P, a, row, SA, SB, twf, twi);
    else if (q == 1)
        rows_small_body<1>(P, a, row, SA, SB, twf, twi);
    else
        rows_small_body<2>(P, a, row, SA, SB, twf, twi);
}

// ---------------------------------------------------------------------------
// Split row passes for products that share forward transforms.
//
// k_rows_fwd finishes the forward transform of one or two operands whose
// column passes are done; the last stage's registers (thread t holds
// positions 16t .. 16t + 15) go through the shared tile to the first
// stage's order (thread t holds t + 256 j), so the spectrum is stored with
// coalesced 128-byte warp accesses.  k_rows_inv loads T pairs of spectra in
// that order, forms sum_t X_t Y_t K^-1 (mod p), moves the result back to
// the last stage's order through the tile and runs the inverse stages,
// leaving the segment in the order the inverse column passes expect, as the
// fused k_rows_r does.  So a transform computed once serves every product
// it takes part in, and a sum of products costs one inverse transform.
// ---------------------------------------------------------------------------
constexpr int kSplitLogC = 12;
using SplitLast = ExecStage<kSplitLogC, 0, false, StagePlan<kSplitLogC>::n - 1>::S;
static_assert(SplitLast::kLO == 0 && SplitLast::kB == 4, "last row stage holds 16 consecutive positions");

struct RowsFwdArgs {
    uint32_t *F0;   // spectra [vrow][q][K], column passes done
    uint32_t *F1;   // second operand of the same shape, or null
    int log_k;
};

template <int Q>
__device__ __forceinline__ void rows_fwd_body(const RowsFwdArgs &a, uint64_t b, uint32_t *Sm, uint2 *tw) {
    constexpr int C = 1 << kSplitLogC;
    constexpr int T = C / 16;
    using First = typename ExecStage<kSplitLogC, 0, false, 0>::S;
    const uint32_t nseg = 1u << (a.log_k - kSplitLogC);
    const uint64_t K = 1ull << a.log_k;
    const uint64_t off = (b / nseg) * 3 * K + (uint64_t)Q * K + ((uint64_t)(b % nseg) << kSplitLogC);
    const uint32_t t = threadIdx.x;
    for (int op = 0; op < (a.F1 ? 2 : 1); ++op) {
        uint32_t *F = (op == 0 ? a.F0 : a.F1) + off;
        uint32_t x[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            uint32_t pos, c;
            First::elem(t, j, pos, c);
            x[j] = F[pos];
        }
        __syncthreads();   // twiddles loaded; the previous operand has left the tile
        run_stages<kSplitLogC, 0, false, Q, 0>(x, Sm, t, tw);
        SplitLast::store(Sm, x, t);   // every thread passed the last stage's tile loads
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            uint32_t pos, c;
            First::elem(t, j, pos, c);
            F[pos] = Sm[First::addr(pos, c)];
        }
        __syncthreads();
    }
    (void)T;
}

__global__ void __launch_bounds__((1 << kSplitLogC) / 16, 4) k_rows_fwd(NttParams P, RowsFwdArgs a) {
    extern __shared__ uint4 rows_smem[];
    constexpr int C = 1 << kSplitLogC;
    uint32_t *Sm = reinterpret_cast<uint32_t *>(rows_smem);
    uint2 *tw = reinterpret_cast<uint2 *>(Sm + C + C / 32);
    uint64_t b;
    const int q = grid_prime(b);
    const uint2 *lev = level_ptr(P.tab, 0, q);
    for (uint32_t e = threadIdx.x; e < C - 1; e += C / 16) tw[e] = __ldg(lev + e);
    if (q == 0)
        rows_fwd_body<0>(a, b, Sm, tw);
    else if (q == 1)
        rows_fwd_body<1>(a, b, Sm, tw);
    else
        rows_fwd_body<2>(a, b, Sm, tw);
}

constexpr int kMaxTerms = 2;
struct RowsInvArgs {
    const uint32_t *X[kMaxTerms];
    const uint32_t *Y[kMaxTerms];
    uint32_t *Fout;   // may be one of the X or Y (each CTA reads its segment before writing it)
    int terms;
    int log_k;
};

template <int TERMS, int Q>
__device__ __forceinline__ void rows_inv_body(const NttParams &P, const RowsInvArgs &a, uint64_t b, uint32_t *Sm,
                                              uint2 *tw) {
    using Out = typename ExecStage<kSplitLogC, 0, true, StagePlan<kSplitLogC>::n - 1>::S;
    const uint32_t nseg = 1u << (a.log_k - kSplitLogC);
    const uint64_t K = 1ull << a.log_k;
    const uint64_t off = (b / nseg) * 3 * K + (uint64_t)Q * K + ((uint64_t)(b % nseg) << kSplitLogC);
    const uint32_t t = threadIdx.x;
    const uint32_t scale = __ldg(P.tab.inv2n + a.log_k * kPrimes + Q);
    using First = typename ExecStage<kSplitLogC, 0, false, 0>::S;
    uint32_t x[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) x[j] = 0u;
#pragma unroll
    for (int term = 0; term < TERMS; ++term) {
        const uint32_t *X = a.X[term] + off, *Y = a.Y[term] + off;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            uint32_t pos, c;
            First::elem(t, j, pos, c);
            x[j] = add_n<Q>(x[j], norm<Q>(mont<Q>(__ldg(X + pos), __ldg(Y + pos))));
        }
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) x[j] = norm<Q>(mont<Q>(x[j], scale));   // sum K^-1
    First::store(Sm, x, t);
    __syncthreads();   // tile written, inverse twiddles loaded
    SplitLast::load(Sm, x, t);
    __syncthreads();
    run_stages<kSplitLogC, 0, true, Q, 0>(x, Sm, t, tw);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        uint32_t pos, c;
        Out::elem(t, j, pos, c);
        a.Fout[off + pos] = x[j];
    }
}

template <int TERMS>
__global__ void __launch_bounds__((1 << kSplitLogC) / 16, 4) k_rows_inv(NttParams P, RowsInvArgs a) {
    extern __shared__ uint4 rows_smem[];
    constexpr int C = 1 << kSplitLogC;
    uint32_t *Sm = reinterpret_cast<uint32_t *>(rows_smem);
    uint2 *tw = reinterpret_cast<uint2 *>(Sm + C + C / 32);
    uint64_t b;
    const int q = grid_prime(b);
    const uint2 *lev = level_ptr(P.tab, 1, q);
    for (uint32_t e = threadIdx.x; e < C - 1; e += C / 16) tw[e] = __ldg(lev + e);
    // two segments per CTA (their count is even: K >= 8192) share the
    // twiddle table load
    for (uint64_t s = 2 * b; s < 2 * b + 2; ++s) {
        if (q == 0)
            rows_inv_body<TERMS, 0>(P, a, s, Sm, tw);
        else if (q == 1)
            rows_inv_body<TERMS, 1>(P, a, s, Sm, tw);
        else
            rows_inv_body<TERMS, 2>(P, a, s, Sm, tw);
        __syncthreads();   // the tile is free for the next segment
    }
}

// One merge level's four row products in one pass (the tuned form's level):
// from the column-transformed segments of P_e, P_o, R_o, Q_o, Q_e, R_e the
// CTA forms P' = P_e P_o, R2 = P_e R_o, Q' = Q_e Q_o, R1 = R_e Q_o (each
// x K^-1) and runs their inverse row stages, writing them over P_o, R_o, Q_e
// and R_e: six forward and four inverse row transforms, the kept operand
// (P_e, then Q_o) and one product in registers, no spectrum stored.  With
// Fpo null (the tree's root) P' is not formed: five and three.
struct RowsLevelArgs {
    uint32_t *Fpe, *Fpo, *Fro, *Fqo, *Fqe, *Fre;
    int log_k;
};

template <int Q>
__device__ __forceinline__ void rows_level_body(const NttParams &P, const RowsLevelArgs &a, uint64_t b,
                                                uint32_t *Sm, uint2 *tw) {
    constexpr int C = 1 << kSplitLogC;
    constexpr int T = C / 16;
    using First = typename ExecStage<kSplitLogC, 0, false, 0>::S;
    using Out = typename ExecStage<kSplitLogC, 0, true, StagePlan<kSplitLogC>::n - 1>::S;
    const uint32_t nseg = 1u << (a.log_k - kSplitLogC);
    const uint64_t K = 1ull << a.log_k;
    const uint64_t off = (b / nseg) * 3 * K + (uint64_t)Q * K + ((uint64_t)(b % nseg) << kSplitLogC);
    const uint32_t t = threadIdx.x;
    const uint32_t scale = __ldg(P.tab.inv2n + a.log_k * kPrimes + Q);
    const uint2 *levf = level_ptr(P.tab, 0, Q);
    const uint2 *levi = level_ptr(P.tab, 1, Q);
    auto load = [&](const uint32_t *F, uint32_t (&x)[16]) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            uint32_t pos, c;
            First::elem(t, j, pos, c);
            x[j] = __ldg(F + off + pos);
        }
    };
    auto store = [&](uint32_t *F, const uint32_t (&x)[16]) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            uint32_t pos, c;
            Out::elem(t, j, pos, c);
            F[off + pos] = x[j];
        }
    };
    auto table = [&](const uint2 *lev) {
        __syncthreads();   // the previous stages have left the tile and the table
        for (uint32_t e = t; e < C - 1; e += T) tw[e] = __ldg(lev + e);
        __syncthreads();
    };
    // The six operand segments (16 KiB each, contiguous, 16-byte aligned) go
    // to L2 by bulk prefetch (the copy engine, no registers or shared memory)
    // as the CTA starts, so the later loads, issued between transforms, find
    // them in L2 instead of waiting on HBM.
    if (t < 6u) {
        const uint32_t *F = t == 0u ? a.Fpe : t == 1u ? a.Fpo : t == 2u ? a.Fro : t == 3u ? a.Fqo
                                                                      : t == 4u ? a.Fqe : a.Fre;
        if (F)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(F + off), "r"((uint32_t)C * 4u)
                         : "memory");
    }
    // One copy of the forward and one of the inverse stages per prime, run
    // in loops (the ten transforms written out would not fit the instruction
    // cache).  Per half: the kept operand F_keep, then F0 (its product with
    // F_keep waits in F0's own segment: word j of thread t at j * T + t,
    // coalesced; every thread has loaded F0 before the next barrier and reads
    // back only its own words; the segment is rewritten by the product's
    // inverse anyway, and keeping the product out of shared memory leaves
    // room for a fourth CTA per SM), then F1 (its product stays in registers);
    // the inverse of F_keep F1 goes to F1, that of the held product to F0.
    // F0 null (the tree's root, uniform over the grid): no P' product.
    uint32_t k[16], x[16];
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
        const uint32_t *Fk = h ? a.Fqo : a.Fpe;
        uint32_t *F0 = h ? a.Fqe : a.Fpo;
        uint32_t *F1 = h ? a.Fre : a.Fro;
        uint32_t *held = F0 ? F0 + off : nullptr;
        table(levf);
#pragma unroll 1
        for (int step = 0; step < 3; ++step) {
            const uint32_t *src = step == 0 ? Fk : (step == 1 ? F0 : F1);
            if (!src) continue;
            if (step) __syncthreads();   // the previous transform has left the tile
            load(src, x);
            run_stages<kSplitLogC, 0, false, Q, 0>(x, Sm, t, tw);
            if (step == 0) {
#pragma unroll
                for (int j = 0; j < 16; ++j) k[j] = x[j];
            } else if (step == 1) {
#pragma unroll
                for (int j = 0; j < 16; ++j) held[j * T + t] = norm<Q>(mont<Q>(mont<Q>(k[j], x[j]), scale));
            } else {
#pragma unroll
                for (int j = 0; j < 16; ++j) x[j] = norm<Q>(mont<Q>(mont<Q>(k[j], x[j]), scale));
            }
        }
        table(levi);
#pragma unroll 1
        for (int step = 0; step < 2; ++step) {
            if (step == 1) {
                if (!held) break;
                __syncthreads();
#pragma unroll
                for (int j = 0; j < 16; ++j) x[j] = held[j * T + t];
            }
            run_stages<kSplitLogC, 0, true, Q, 0>(x, Sm, t, tw);
            store(step ? F0 : F1, x);
        }
    }
}

// the padded tile and the twiddle levels
constexpr size_t rows_level_smem_bytes() { return rows_smem_bytes<kSplitLogC>(); }

__global__ void __launch_bounds__((1 << kSplitLogC) / 16, 4) k_rows_level(NttParams P, RowsLevelArgs a) {
    extern __shared__ uint4 rows_smem[];
    constexpr int C = 1 << kSplitLogC;
    uint32_t *Sm = reinterpret_cast<uint32_t *>(rows_smem);
    uint2 *tw = reinterpret_cast<uint2 *>(Sm + C + C / 32);
    uint64_t b;
    const int q = grid_prime(b);
    if (q == 0)
        rows_level_body<0>(P, a, b, Sm, tw);
    else if (q == 1)
        rows_level_body<1>(P, a, b, Sm, tw);
    else
        rows_level_body<2>(P, a, b, Sm, tw);
}

// Coset recombination.  Row r holds z_i[j] = C_i[j] g^(ij) for cosets i < M;
// C_i[j] = sum_b C_b[j] c_i^b, so C_b[j] = sum_i Vinv[b][i] C_i[j].  The M
// outputs of position j overwrite the M inputs of position j.
struct CombineArgs {
    uint32_t *F;
    int log_k;
    uint32_t vinv[kPrimes][kMaxCosets][kMaxCosets];   // Montgomery form, [q][b][i]
};

template <int M, int Q>
__device__ __forceinline__ void combine_body(const NttParams &P, const CombineArgs &a, uint64_t row, uint32_t j) {
    const uint64_t K = 1ull << a.log_k;
    uint32_t *F0 = a.F + row * M * 3 * K + (uint64_t)Q * K + j;
    const uint32_t *clo = coset_lo_ptr(P.tab, 1, Q);
    const uint32_t *chi = coset_hi_ptr(P.tab, 1, Q);
    uint32_t u[M];
    u[0] = F0[0];
#pragma unroll
    for (int i = 1; i < M; ++i) u[i] = mul_coset<Q, 1>(F0[(uint64_t)i * 3 * K], clo, chi, (uint32_t)i * j);
#pragma unroll
    for (int b = 0; b < M; ++b) {
        uint32_t acc = 0u;
#pragma unroll
        for (int i = 0; i < M; ++i) acc = add_n<Q>(acc, norm<Q>(mont<Q>(u[i], a.vinv[Q][b][i])));
        F0[(uint64_t)b * 3 * K] = acc;
    }
}

template <int M>
__global__ void __launch_bounds__(kThreads) k_combine(NttParams P, CombineArgs a) {
    uint64_t rest;
    const int q = grid_prime(rest);
    const uint32_t jblocks = (1u << a.log_k) / kThreads;
    const uint64_t row = rest / jblocks;
    const uint32_t j = (uint32_t)(rest - row * jblocks) * kThreads + threadIdx.x;
    if (q == 0)
        combine_body<M, 0>(P, a, row, j);
    else if (q == 1)
        combine_body<M, 1>(P, a, row, j);
    else
        combine_body<M, 2>(P, a, row, j);
}

// Garner: residues (r0, r1, r2) -> coefficient < p0 p1 p2 as 3 limbs.
//   t1 = (r1 - r0) / p0 mod p1,  t2 = ((r2 - r0) / p0 - t1) / p1 mod p2,
//   x  = r0 + p0 t1 + p0 p1 t2.
constexpr uint32_t kI01 = cinv(Prime<0>::p, Prime<1>::p);
constexpr uint32_t kI02 = cinv(Prime<0>::p, Prime<2>::p);
constexpr uint32_t kI12 = cinv(Prime<1>::p, Prime<2>::p);
constexpr uint32_t kI01q = shoup_of(kI01, Prime<1>::p);
constexpr uint32_t kI02q = shoup_of(kI02, Prime<2>::p);
constexpr uint32_t kI12q = shoup_of(kI12, Prime<2>::p);
constexpr uint64_t kP0P1 = (uint64_t)Prime<0>::p * Prime<1>::p;

__device__ __forceinline__ void garner(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t (&out)[3]) {
    const uint32_t t1 = norm<1>(shoup<1>(sub_n<1>(r1, r0), kI01, kI01q));   // r0 < p0 < p1
    const uint32_t u = norm<2>(shoup<2>(sub_n<2>(r2, r0), kI02, kI02q));
    const uint32_t t2 = norm<2>(shoup<2>(sub_n<2>(u, t1), kI12, kI12q));    // t1 < p1 < p2
    const unsigned __int128 x = (unsigned __int128)kP0P1 * t2 + (uint64_t)Prime<0>::p * t1 + r0;
    out[0] = (uint32_t)x;
    out[1] = (uint32_t)(x >> 32);
    out[2] = (uint32_t)(x >> 64);
}

constexpr int kCrtV = 4;
constexpr uint32_t kCrtSpan = kThreads * kCrtV;   // 1024 limbs per tile

struct CrtArgs {
    const uint32_t *F;
    int log_k;
    int M;
    uint32_t *C;
    uint64_t sC;
    uint32_t Lc;
    uint32_t tiles;
    uint32_t *flags;
    uint32_t ncoef;      // coefficients of the product (L_a + L_b - 1)
    // optional addend: C = product + (D << dshift), D rows at D + row * sD,
    // Ld limbs; C's L_c limbs must hold the sum
    const uint32_t *D;
    uint64_t sD;
    uint32_t Ld;
    uint32_t dshift;
};

// Adds limbs base .. base + kCrtV - 1 of (D << dshift) to the chunk sum S
// (carries run into S's three top words, which stay far from overflowing).
__device__ __forceinline__ void crt_add_shifted(const CrtArgs &a, const uint32_t *Dr, int64_t base,
                                                uint32_t (&S)[kCrtV + 3]) {
    const int64_t sw = a.dshift >> 5;
    const uint32_t sb = a.dshift & 31u;
    uint64_t cy = 0;
#pragma unroll
    for (int v = 0; v < kCrtV + 3; ++v) {
        uint32_t d = 0u;
        if (v < kCrtV) {
            const int64_t i = base + v - sw;   // source limb of the low part
            const uint32_t lo = (i >= 0 && i < (int64_t)a.Ld) ? Dr[i] : 0u;
            const uint32_t hi = (sb && i - 1 >= 0 && i - 1 < (int64_t)a.Ld) ? Dr[i - 1] : 0u;
            d = sb ? ((lo << sb) | (hi >> (32u - sb))) : lo;
        }
        const uint64_t t = (uint64_t)S[v] + d + cy;
        S[v] = (uint32_t)t;
        cy = t >> 32;
    }
}

// Coefficient n of a row lives in block b = n / K at F0[(b * 3 + q) * K + n mod K];
// there are ncoef = L_c - 1 <= M K of them (the top limb only receives carries).
__device__ __forceinline__ void crt_chunk(const uint32_t *F0, int log_k, uint32_t ncoef, int64_t base,
                                          uint32_t (&S)[kCrtV + 3]) {
    uint32_t c[kCrtV][3];
    const uint64_t K = 1ull << log_k;
    if (base >= 0 && base + kCrtV <= (int64_t)ncoef && K >= (uint64_t)kCrtV) {
        // the chunk lies in one block: one 128-bit load per prime (K and base are multiples of 4)
        const uint64_t off = (((uint64_t)base >> log_k) * 3) * K + ((uint64_t)base & (K - 1));
        const uint4 r0 = *reinterpret_cast<const uint4 *>(F0 + off);
        const uint4 r1 = *reinterpret_cast<const uint4 *>(F0 + off + K);
        const uint4 r2 = *reinterpret_cast<const uint4 *>(F0 + off + 2 * K);
        garner(r0.x, r1.x, r2.x, c[0]);
        garner(r0.y, r1.y, r2.y, c[1]);
        garner(r0.z, r1.z, r2.z, c[2]);
        garner(r0.w, r1.w, r2.w, c[3]);
        chunk_sum3<kCrtV>(c, S);
        return;
    }
#pragma unroll
    for (int v = 0; v < kCrtV; ++v) {
        const int64_t i = base + v;
        if (i >= 0 && i < (int64_t)ncoef) {
            const uint64_t off = (((uint64_t)i >> log_k) * 3) * K + ((uint64_t)i & (K - 1));
            garner(F0[off], F0[off + K], F0[off + 2 * K], c[v]);
        } else {
            c[v][0] = c[v][1] = c[v][2] = 0u;
        }
    }
    chunk_sum3<kCrtV>(c, S);
}

__global__ void __launch_bounds__(kThreads) k_crt(CrtArgs a) {
    __shared__ uint32_t sg[kThreads / 32], sp[kThreads / 32], spre[kThreads / 32];
    __shared__ uint32_t spill[kThreads / 32][3];
    const uint32_t tile = blockIdx.x;
    const uint64_t row = tile / a.tiles;
    const uint32_t t = tile - (uint32_t)row * a.tiles;
    const uint64_t K = 1ull << a.log_k;
    const uint32_t *F0 = a.F + row * (uint64_t)a.M * 3 * K;
    const int64_t base = (int64_t)t * kCrtSpan + threadIdx.x * kCrtV;
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    uint32_t S[kCrtV + 3];
    const uint32_t *Dr = a.D ? a.D + row * a.sD : nullptr;
    crt_chunk(F0, a.log_k, a.ncoef, base, S);
    if (Dr) crt_add_shifted(a, Dr, base, S);
    // words of the previous chunk's sum that land in this chunk: from the
    // previous lane, from the previous warp's last lane, and for the tile's
    // first thread from the last chunk of the previous tile (recomputed)
    uint32_t H[3];
    H[0] = __shfl_up_sync(0xffffffffu, S[kCrtV], 1);
    H[1] = __shfl_up_sync(0xffffffffu, S[kCrtV + 1], 1);
    H[2] = __shfl_up_sync(0xffffffffu, S[kCrtV + 2], 1);
    if (lane == 31) {
        spill[warp][0] = S[kCrtV];
        spill[warp][1] = S[kCrtV + 1];
        spill[warp][2] = S[kCrtV + 2];
    }
    if (threadIdx.x == 0) {
        uint32_t Sp[kCrtV + 3];
        crt_chunk(F0, a.log_k, a.ncoef, base - kCrtV, Sp);
        if (Dr) crt_add_shifted(a, Dr, base - kCrtV, Sp);
        H[0] = Sp[kCrtV];
        H[1] = Sp[kCrtV + 1];
        H[2] = Sp[kCrtV + 2];
    }
    __syncthreads();
    if (lane == 0 && warp > 0) {
        H[0] = spill[warp - 1][0];
        H[1] = spill[warp - 1][1];
        H[2] = spill[warp - 1][2];
    }
    uint32_t X[kCrtV];
    const uint32_t g = chunk_add_spill<kCrtV>(S, H, X);
    bool p = true;
#pragma unroll
    for (int v = 0; v < kCrtV; ++v) p = p && (X[v] == 0xffffffffu) && (base + v < (int64_t)a.Lc);
    const BlockCarry bc = block_resolve<kThreads / 32>(g != 0u, p, sg, sp);
    chunk_increment<kCrtV>(X, bc.cin);
    uint32_t *out = a.C + row * a.sC;
#pragma unroll
    for (int v = 0; v < kCrtV; ++v)
        if (base + v < (int64_t)a.Lc) out[base + v] = X[v];
    if (a.tiles > 1u) {
        uint32_t local = kCrtV;
#pragma unroll
        for (int v = kCrtV - 1; v >= 0; --v)
            if (X[v] != 0xffffffffu || base + v >= (int64_t)a.Lc) local = v;
        const uint32_t pre = block_prefix<kThreads / 32, kCrtV>(local, spre);
        if (threadIdx.x == 0) a.flags[tile] = bc.G | (bc.P << 1) | (pre << 2);
    }
}

// ---------------------------------------------------------------------------
// Host orchestration
// ---------------------------------------------------------------------------
static int ceil_log2(uint64_t x) {
    int k = 0;
    while ((1ull << k) < x) ++k;
    return k;
}

struct Shape {
    int log_k;   // K = 2^log_k points per coset
    int M;       // cosets
};

// Smallest shape with M * K >= L_a + L_b - 1: one power-of-two transform up to
// 2^25 points, above that M cosets of 2^25 points.
}  // namespace ntt
bool ntt_shape_override(uint64_t need, int *log_k, int *M);   // tune.cu
namespace ntt {

static Shape shape_for(uint32_t La, uint32_t Lb);

// The product's transform shape: the tune table's, else the built-in rule
// (shape_for).  Used by the plain product and its workspace size; the
// tuned splitting tree's spectra keep the built-in rule.
static Shape shape_tuned(uint32_t La, uint32_t Lb) {
    int lk = 0, M = 0;
    if (ntt_shape_override((uint64_t)La + Lb - 1u, &lk, &M)) return Shape{lk, M};
    return shape_for(La, Lb);
}

static Shape shape_for(uint32_t La, uint32_t Lb) {
    const uint64_t need = (uint64_t)La + Lb - 1u;
    if (need <= (1ull << kMaxLog)) {
        const int k = ceil_log2(need < 2 ? 2 : need);
        return {k < 1 ? 1 : k, 1};
    }
    const uint64_t K = 1ull << kMaxLog;
    return {kMaxLog, (int)((need + K - 1) / K)};
}

// Paired passes exist for R >= 32 only (shorter columns twist per residue
// and would spill with two operands).
constexpr int kPairMinLogR = 5;
// Column lengths up to 1024 run as one pass (tiles of 4096 / R columns; for
// R = 1024 a row segment is half a 32-byte sector, whose other half the
// neighbouring tile reads at the same time from L2).  Longer columns are
// split in two passes: single passes of 2048 / 4096 points measured slower
// (K = 2^23: 0.82 against 0.72 ms) with their 4095-entry twiddle tables per
// CTA and 4- / 8-byte row segments; K = 2^22 runs 0.36 ms in one 1024-point
// pass against 0.41 ms in two.
constexpr int kOnePassMaxLog = 10;

template <int LOG_R, bool FL, bool INV, bool PAIR>
static void cols_launch(unsigned blocks, const NttParams &P, const ColsArgs &a, cudaStream_t st) {
    constexpr size_t smem = cols_smem_bytes<LOG_R, PAIR>();
    static bool attr = false;
    if (!attr) {
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(k_cols_r<LOG_R, FL, INV, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        attr = true;
    }
    k_cols_r<LOG_R, FL, INV, PAIR><<<blocks, kThreads, smem, st>>>(P, a);
}

template <bool FL, bool INV, bool PAIR>
static void cols_r_dispatch(int log_r, unsigned blocks, const NttParams &P, const ColsArgs &a, cudaStream_t st) {
    if constexpr (!PAIR) {
        switch (log_r) {
            case 1: cols_launch<1, FL, INV, false>(blocks, P, a, st); return;
            case 2: cols_launch<2, FL, INV, false>(blocks, P, a, st); return;
            case 3: cols_launch<3, FL, INV, false>(blocks, P, a, st); return;
            case 4: cols_launch<4, FL, INV, false>(blocks, P, a, st); return;
            default: break;
        }
    }
    switch (log_r) {
        case 5: cols_launch<5, FL, INV, PAIR>(blocks, P, a, st); break;
        case 6: cols_launch<6, FL, INV, PAIR>(blocks, P, a, st); break;
        case 7: cols_launch<7, FL, INV, PAIR>(blocks, P, a, st); break;
        case 8: cols_launch<8, FL, INV, PAIR>(blocks, P, a, st); break;
        case 9: cols_launch<9, FL, INV, PAIR>(blocks, P, a, st); break;
        default: cols_launch<10, FL, INV, PAIR>(blocks, P, a, st); break;
    }
}

// One column pass over vrows virtual rows (pair: operands A and B together).
static void launch_cols_r(bool from_limbs, bool inverse, bool pair, int log_r, const NttParams &P,
                          const ColsArgs &a, uint64_t vrows, cudaStream_t st) {
    const uint64_t ctiles = 1ull << (a.log_s - 12);
    const uint64_t nseg = 1ull << (a.log_k - a.log_s);
    const unsigned blocks = (unsigned)(vrows * kPrimes * nseg * ctiles);
    // algorithmic bytes: 4 B per residue read and written (3 primes per
    // point); the first pass reads the limbs instead (once per coset)
    const double K = (double)(1ull << a.log_k);
    const double limbs = (double)a.Lx + (pair ? (double)a.Lx2 : 0.0);
    const double ops = pair ? 2.0 : 1.0;
    const double bytes = from_limbs ? (4.0 * limbs * (double)vrows / a.M + 12.0 * K * (double)vrows * ops)
                                    : 24.0 * K * (double)vrows * ops;
    KernelTimed kt(from_limbs ? "ntt_cols_fwd_first" : (inverse ? "ntt_cols_inv" : "ntt_cols_fwd"), bytes);
    if (from_limbs) {
        if (pair)
            cols_r_dispatch<true, false, true>(log_r, blocks, P, a, st);
        else
            cols_r_dispatch<true, false, false>(log_r, blocks, P, a, st);
    } else if (!inverse) {
        if (pair)
            cols_r_dispatch<false, false, true>(log_r, blocks, P, a, st);
        else
            cols_r_dispatch<false, false, false>(log_r, blocks, P, a, st);
    } else {
        cols_r_dispatch<false, true, false>(log_r, blocks, P, a, st);
    }
    count_launch();
}

template <int LOG_C, bool FL>
static void rows_launch(unsigned blocks, const NttParams &P, const RowsArgs &r, cudaStream_t st) {
    constexpr size_t smem = rows_smem_bytes<LOG_C>();
    static bool attr = false;
    if (!attr) {
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(k_rows_r<LOG_C, FL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    k_rows_r<LOG_C, FL><<<blocks, (1 << LOG_C) / 16, smem, st>>>(P, r);
}

template <bool FL>
static void rows_r_dispatch(int log_c, unsigned blocks, const NttParams &P, const RowsArgs &r, cudaStream_t st) {
    switch (log_c) {
        case 9: rows_launch<9, FL>(blocks, P, r, st); break;
        case 10: rows_launch<10, FL>(blocks, P, r, st); break;
        case 11: rows_launch<11, FL>(blocks, P, r, st); break;
        default: rows_launch<12, FL>(blocks, P, r, st); break;
    }
}

// Inverse of the Vandermonde matrix V[i][b] = c_i^b (c_i = g^(i 2^log_k)) mod
// p_q, Montgomery form, out[q][b][i].
static void coset_matrix(int M, int log_k, uint32_t (&out)[kPrimes][kMaxCosets][kMaxCosets]) {
    for (int q = 0; q < kPrimes; ++q) {
        const uint32_t p = kP[q];
        uint32_t V[kMaxCosets][2 * kMaxCosets] = {};
        for (int i = 0; i < M; ++i) {
            const uint32_t c = h_pow(kGen[q], (uint64_t)i << log_k, p);
            uint32_t x = 1u;
            for (int b = 0; b < M; ++b) {
                V[i][b] = x;
                x = h_mul(x, c, p);
            }
            V[i][M + i] = 1u;
        }
        for (int col = 0; col < M; ++col) {   // Gauss-Jordan; the nodes are distinct
            int piv = col;
            while (V[piv][col] == 0u) ++piv;
            if (piv != col)
                for (int k = 0; k < 2 * M; ++k) {
                    const uint32_t tmp = V[piv][k];
                    V[piv][k] = V[col][k];
                    V[col][k] = tmp;
                }
            const uint32_t inv = h_inv(V[col][col], p);
            for (int k = 0; k < 2 * M; ++k) V[col][k] = h_mul(V[col][k], inv, p);
            for (int r = 0; r < M; ++r) {
                if (r == col || V[r][col] == 0u) continue;
                const uint32_t f = V[r][col];
                for (int k = 0; k < 2 * M; ++k)
                    V[r][k] = (uint32_t)((V[r][k] + (uint64_t)(p - h_mul(f, V[col][k], p))) % p);
            }
        }
        for (int b = 0; b < kMaxCosets; ++b)
            for (int i = 0; i < kMaxCosets; ++i)
                out[q][b][i] = (b < M && i < M) ? h_mont(V[b][M + i], p) : 0u;
    }
}

// Column passes below the 4096-point rows: one for up to 2^10 points,
// else two; returns their count.
static int column_passes(int log_k, int (&passes)[2]) {
    const int rest = log_k - 12;
    if (rest <= kOnePassMaxLog) {
        passes[0] = rest;
        return 1;
    }
    passes[0] = (rest + 1) / 2;
    passes[1] = rest / 2;
    return 2;
}

// Every coefficient, at most min(L_a, L_b) (2^32 - 1)^2, is below p0 p1 p2
// (min(L_a, L_b) < 4.18e8).
static bool crt_fits(uint64_t min_len) {
    unsigned __int128 cap = 1;
    for (int q = 0; q < kPrimes; ++q) cap *= kP[q];
    return (unsigned __int128)min_len * 0xffffffffull * 0xffffffffull < cap;
}

static void launch_combine(int M, const NttParams &P, const CombineArgs &c, uint32_t N, cudaStream_t st) {
    const uint64_t K = 1ull << c.log_k;
    const unsigned blocks = (unsigned)((uint64_t)N * kPrimes * (K / kThreads));
    KernelTimed kt("ntt_coset_combine", 24.0 * (double)K * M * N);
    switch (M) {
        case 2: k_combine<2><<<blocks, kThreads, 0, st>>>(P, c); break;
        case 3: k_combine<3><<<blocks, kThreads, 0, st>>>(P, c); break;
        case 4: k_combine<4><<<blocks, kThreads, 0, st>>>(P, c); break;
        case 5: k_combine<5><<<blocks, kThreads, 0, st>>>(P, c); break;
        case 6: k_combine<6><<<blocks, kThreads, 0, st>>>(P, c); break;
        case 7: k_combine<7><<<blocks, kThreads, 0, st>>>(P, c); break;
        case 8: k_combine<8><<<blocks, kThreads, 0, st>>>(P, c); break;
        case 9: k_combine<9><<<blocks, kThreads, 0, st>>>(P, c); break;
        case 10: k_combine<10><<<blocks, kThreads, 0, st>>>(P, c); break;
        case 11: k_combine<11><<<blocks, kThreads, 0, st>>>(P, c); break;
        case 12: k_combine<12><<<blocks, kThreads, 0, st>>>(P, c); break;
        case 13: k_combine<13><<<blocks, kThreads, 0, st>>>(P, c); break;
        case 14: k_combine<14><<<blocks, kThreads, 0, st>>>(P, c); break;
        case 15: k_combine<15><<<blocks, kThreads, 0, st>>>(P, c); break;
        case 16: k_combine<16><<<blocks, kThreads, 0, st>>>(P, c); break;
        case 17: k_combine<17><<<blocks, kThreads, 0, st>>>(P, c); break;
        case 18: k_combine<18><<<blocks, kThreads, 0, st>>>(P, c); break;
        case 19: k_combine<19><<<blocks, kThreads, 0, st>>>(P, c); break;
        default: k_combine<20><<<blocks, kThreads, 0, st>>>(P, c); break;
    }
    count_launch();
}

size_t workspace_bytes(uint32_t N, uint32_t La, uint32_t Lb) {
    if (N == 0u || La == 0u || Lb == 0u) return 0;
    const Shape s = shape_tuned(La, Lb);
    const uint64_t K = 1ull << s.log_k;
    const uint64_t Lc = (uint64_t)La + Lb;
    const uint64_t tiles = (Lc + kCrtSpan - 1) / kCrtSpan;
    return (size_t)(2ull * N * s.M * 3 * K * 4 + N * tiles * 4 + 256);
}

static void mul(const NttParams &P, const uint32_t *A, const uint32_t *B, uint32_t *C, uint32_t *ws,
                uint32_t N, uint32_t La, uint32_t Lb, uint64_t sA, uint64_t sB, uint64_t sC) {
    cudaStream_t st = current_stream();
    const uint32_t Lc = La + Lb;
    if (N == 0u || Lc == 0u) return;
    if (La == 0u || Lb == 0u) {
        cudaMemset2DAsync(C, sC * 4, 0, (size_t)Lc * 4, N, st);
        return;
    }
    const Shape s = shape_tuned(La, Lb);
    if (s.M > kMaxCosets) {
        fprintf(stderr, "gpupi_b200: product of %u limbs exceeds the 20 * 2^25-point limit\n", Lc);
        return;
    }
    if (!crt_fits(La < Lb ? La : Lb)) {
        fprintf(stderr, "gpupi_b200: min(L_a, L_b) = %u exceeds the three-prime CRT capacity\n", La < Lb ? La : Lb);
        return;
    }
    const int log_k = s.log_k, M = s.M;
    const uint64_t K = 1ull << log_k;
    const uint64_t VR = (uint64_t)N * M;   // virtual rows (row, coset)
    const bool square = (A == B && La == Lb && sA == sB);
    const bool bcast = (!square && sB == 0u && N > 1u);
    uint32_t *FA = ws;
    uint32_t *FB = square ? FA : ws + VR * 3 * K;
    const uint64_t tiles = ((uint64_t)Lc + kCrtSpan - 1) / kCrtSpan;
    uint32_t *flags = ws + 2ull * VR * 3 * K;

    if (log_k <= 12) {
        RowsArgs r{A, sA, La, B, sB, Lb, FA, FB, log_k, 1, bcast ? 1 : 0, square ? 1 : 0};
        KernelTimed kt("ntt_local", 4.0 * N * ((double)La + (square ? 0 : Lb)) + 12.0 * K * N);
        if (log_k >= 9)
            rows_r_dispatch<true>(log_k, (unsigned)(N * kPrimes), P, r, st);
        else
            k_rows_small<<<(unsigned)(N * kPrimes), 128, 0, st>>>(P, r);
        count_launch();
    } else {
        const int log_c = 12;
        int passes[2];
        const int npass = column_passes(log_k, passes);
        // forward column passes: A and B together (one launch per pass) unless
        // B is A or a broadcast row
        const bool pair = !square && !bcast && passes[0] >= kPairMinLogR && (npass == 1 || passes[1] >= kPairMinLogR);
        for (int op = 0; op < (pair || square ? 1 : 2); ++op) {
            const uint32_t *X = op == 0 ? A : B;
            const uint64_t sX = op == 0 ? sA : sB;
            const uint32_t Lx = op == 0 ? La : Lb;
            uint32_t *F = op == 0 ? FA : FB;
            const uint64_t vrows = (op == 1 && bcast) ? (uint64_t)M : VR;
            const uint32_t nb = (uint32_t)((Lx + K - 1) / K);
            const uint32_t nb2 = (uint32_t)((Lb + K - 1) / K);
            int log_s = log_k;
            for (int ps = 0; ps < npass; ++ps) {
                ColsArgs a{X, sX, Lx, nb, F, log_k, log_s, M, pair ? B : nullptr, sB, Lb, nb2, pair ? FB : nullptr};
                launch_cols_r(ps == 0, false, pair, passes[ps], P, a, vrows, st);
                log_s -= passes[ps];
            }
        }
        RowsArgs r{A, sA, La, B, sB, Lb, FA, FB, log_k, M, bcast ? 1 : 0, square ? 1 : 0};
        const uint64_t blocks = VR * kPrimes * (K >> log_c);
        {
            KernelTimed kt("ntt_rows_fused", 12.0 * (double)K * ((square ? 2.0 : 3.0) * (double)VR));
            rows_r_dispatch<false>(log_c, (unsigned)blocks, P, r, st);
            count_launch();
        }
        // inverse column passes, innermost first
        int log_s = log_c;
        for (int ps = npass - 1; ps >= 0; --ps) {
            log_s += passes[ps];
            ColsArgs a{nullptr, 0, 0, 0, FA, log_k, log_s, M, nullptr, 0, 0, 0, nullptr};
            launch_cols_r(false, true, false, passes[ps], P, a, VR, st);
        }
        if (M > 1) {
            CombineArgs c{};
            c.F = FA;
            c.log_k = log_k;
            coset_matrix(M, log_k, c.vinv);
            launch_combine(M, P, c, N, st);
        }
    }
    CrtArgs c{FA, log_k, M, C, sC, Lc, (uint32_t)tiles, flags, Lc - 1u, nullptr, 0, 0, 0};
    KernelTimed kt("ntt_crt_carry", 12.0 * (double)Lc * N + 4.0 * (double)Lc * N);
    k_crt<<<(unsigned)(N * tiles), kThreads, 0, st>>>(c);
    count_launch();
    if (tiles > 1) launch_carry_fixup(false, C, sC, N, Lc, (uint32_t)tiles, kCrtSpan, flags, st);
}

// ---------------------------------------------------------------------------
// Shared-transform products: spectrum_forward computes the forward transform
// of one operand (or two of the same shape) into caller buffers;
// spectrum_inverse turns a sum of products of such spectra into limbs.
// ---------------------------------------------------------------------------
static void rows_split_attr() {
    static bool done = false;
    if (!done) {
        constexpr int smem = (int)rows_smem_bytes<kSplitLogC>();
        cudaFuncSetAttribute(k_rows_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        cudaFuncSetAttribute(k_rows_inv<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        cudaFuncSetAttribute(k_rows_inv<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        cudaFuncSetAttribute(k_rows_level, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)rows_level_smem_bytes());
        done = true;
    }
}

static void spectrum_forward(const NttParams &P, Shape s, uint32_t N, const uint32_t *X, uint64_t sX, uint32_t Lx,
                             uint32_t *FX, const uint32_t *Y, uint64_t sY, uint32_t Ly, uint32_t *FY,
                             cudaStream_t st, bool rows) {
    const int log_k = s.log_k, M = s.M;
    const uint64_t K = 1ull << log_k;
    const uint64_t VR = (uint64_t)N * M;
    int passes[2];
    const int npass = column_passes(log_k, passes);
    const bool pair = Y && passes[0] >= kPairMinLogR && (npass == 1 || passes[1] >= kPairMinLogR);
    for (int op = 0; op < ((pair || !Y) ? 1 : 2); ++op) {
        const uint32_t *Z = op == 0 ? X : Y;
        const uint64_t sZ = op == 0 ? sX : sY;
        const uint32_t Lz = op == 0 ? Lx : Ly;
        uint32_t *F = op == 0 ? FX : FY;
        const uint32_t nb = (uint32_t)((Lz + K - 1) / K);
        const uint32_t nb2 = (uint32_t)((Ly + K - 1) / K);
        int log_s = log_k;
        for (int ps = 0; ps < npass; ++ps) {
            ColsArgs a{Z, sZ, Lz, nb, F, log_k, log_s, M, pair ? Y : nullptr, sY, Ly, nb2, pair ? FY : nullptr};
            launch_cols_r(ps == 0, false, pair, passes[ps], P, a, VR, st);
            log_s -= passes[ps];
        }
    }
    if (!rows) return;
    rows_split_attr();
    RowsFwdArgs r{FX, Y ? FY : nullptr, log_k};
    const unsigned blocks = (unsigned)(VR * kPrimes * (K >> kSplitLogC));
    KernelTimed kt("ntt_rows_fwd", 8.0 * (double)K * (double)VR * (Y ? 2.0 : 1.0) * kPrimes);
    k_rows_fwd<<<blocks, (1 << kSplitLogC) / 16, rows_smem_bytes<kSplitLogC>(), st>>>(P, r);
    count_launch();
}

static void spectrum_inverse(const NttParams &P, Shape s, uint32_t N, int terms, const uint32_t *const *X,
                             const uint32_t *const *Y, uint32_t *Fout, uint32_t *C, uint64_t sC, uint32_t Lc,
                             uint32_t *flags, cudaStream_t st, bool rows, const SpectrumAddend *add) {
    const int log_k = s.log_k, M = s.M;
    const uint64_t K = 1ull << log_k;
    const uint64_t VR = (uint64_t)N * M;
    rows_split_attr();
    if (rows) {
    RowsInvArgs r{};
    for (int i = 0; i < terms; ++i) {
        r.X[i] = X[i];
        r.Y[i] = Y[i];
    }
    r.Fout = Fout;
    r.terms = terms;
    r.log_k = log_k;
    const unsigned blocks = (unsigned)(VR * kPrimes * (K >> kSplitLogC) / 2);   // two segments per CTA
    {
        KernelTimed kt("ntt_rows_inv", 4.0 * (double)K * (double)VR * kPrimes * (2.0 * terms + 1.0));
        if (terms == 1)
            k_rows_inv<1><<<blocks, (1 << kSplitLogC) / 16, rows_smem_bytes<kSplitLogC>(), st>>>(P, r);
        else
            k_rows_inv<2><<<blocks, (1 << kSplitLogC) / 16, rows_smem_bytes<kSplitLogC>(), st>>>(P, r);
        count_launch();
    }
    }
    int passes[2];
    const int npass = column_passes(log_k, passes);
    int log_s = kSplitLogC;
    for (int ps = npass - 1; ps >= 0; --ps) {
        log_s += passes[ps];
        ColsArgs a{nullptr, 0, 0, 0, Fout, log_k, log_s, M, nullptr, 0, 0, 0, nullptr};
        launch_cols_r(false, true, false, passes[ps], P, a, VR, st);
    }
    if (M > 1) {
        CombineArgs c{};
        c.F = Fout;
        c.log_k = log_k;
        coset_matrix(M, log_k, c.vinv);
        launch_combine(M, P, c, N, st);
    }
    const uint64_t tiles = ((uint64_t)Lc + kCrtSpan - 1) / kCrtSpan;
    CrtArgs c{Fout, log_k, M, C, sC, Lc, (uint32_t)tiles, flags, Lc - 1u, nullptr, 0, 0, 0};
    if (add) {
        c.ncoef = add->ncoef;
        c.D = add->D;
        c.sD = add->sD;
        c.Ld = add->Ld;
        c.dshift = add->shift;
    }
    KernelTimed kt("ntt_crt_carry", 12.0 * (double)c.ncoef * N + 4.0 * (double)Lc * N +
                                        (add ? 4.0 * (double)add->Ld * N : 0.0));
    k_crt<<<(unsigned)(N * tiles), kThreads, 0, st>>>(c);
    count_launch();
    if (tiles > 1) launch_carry_fixup(false, C, sC, N, Lc, (uint32_t)tiles, kCrtSpan, flags, st);
}

void build_tables(std::vector<uint32_t> &lv1, std::vector<uint32_t> &lv2, std::vector<uint32_t> &inv2n) {
    lv1.assign(65536u * 3u, 0u);
    lv2.assign(65536u * 3u, 0u);
    inv2n.assign(33u * 3u, 0u);
    for (int q = 0; q < kPrimes; ++q) {
        const uint32_t p = kP[q];
        const uint32_t g = kGen[q];
        const uint32_t w = h_pow(g, (p - 1u) >> kMaxLog, p);   // primitive 2^25-th root
        for (int dir = 0; dir < 2; ++dir) {
            const uint32_t base = dir ? h_inv(w, p) : w;
            uint32_t x = 1u;
            for (uint32_t e = 0; e < kLoSize; ++e) {
                const size_t o = ((size_t)(dir * kPrimes + q) * kLoSize + e) * 2u;
                lv1[o] = x;
                lv1[o + 1] = shoup_of(x, p);
                x = h_mul(x, base, p);
            }
            const uint32_t step = h_pow(base, kLoSize, p);
            x = 1u;
            for (uint32_t e = 0; e < kHiSize; ++e) {
                const size_t o = kRootLoWords + ((size_t)(dir * kPrimes + q) * kHiSize + e) * 2u;
                lv1[o] = x;
                lv1[o + 1] = shoup_of(x, p);
                x = h_mul(x, step, p);
            }
            for (int lh = 0; lh < kLevelLogMax; ++lh) {
                const uint32_t root = h_pow(base, 1ull << (kMaxLog - 1 - lh), p);   // w_(2h), h = 2^lh
                x = 1u;
                for (uint32_t m = 0; m < (1u << lh); ++m) {
                    const size_t o =
                        kLevelOffset + ((size_t)(dir * kPrimes + q) * kLevelSize + (1u << lh) - 1u + m) * 2u;
                    lv1[o] = x;
                    lv1[o + 1] = shoup_of(x, p);
                    x = h_mul(x, root, p);
                }
            }
            const uint32_t gb = dir ? h_inv(g, p) : g;
            x = 1u;
            for (uint32_t e = 0; e < kCosetSize; ++e) {
                lv2[(size_t)(dir * kPrimes + q) * kCosetSize + e] = h_mont(x, p);
                x = h_mul(x, gb, p);
            }
            const uint32_t gstep = h_pow(gb, kCosetSize, p);
            x = 1u;
            for (uint32_t e = 0; e < kCosetSize; ++e) {
                lv2[kCosetWords + (size_t)(dir * kPrimes + q) * kCosetSize + e] = h_mont(x, p);
                x = h_mul(x, gstep, p);
            }
        }
        const uint32_t r2 = h_mont(h_mont(1u, p), p);   // R^2 mod p
        for (int k = 0; k <= 32; ++k) {
            const uint32_t kinv = h_inv(h_pow(2u, (uint64_t)k, p), p);
            inv2n[(size_t)k * kPrimes + q] = h_mul(kinv, r2, p);
        }
    }
}

}  // namespace ntt
}  // namespace gpupi

void init_ntt_precomputed_tables(NTTPrecomputedTables *tables) {
    std::vector<uint32_t> lv1, lv2, inv2n;
    gpupi::ntt::build_tables(lv1, lv2, inv2n);
    cudaMemcpy(tables->roots_table_lv1, lv1.data(), lv1.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(tables->roots_table_lv2, lv2.data(), lv2.size() * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(tables->inv2n_table, inv2n.data(), inv2n.size() * 4, cudaMemcpyHostToDevice);
}

void batch_mul_ntt(uint32_t *A, uint32_t *B, uint32_t *ret, uint32_t *workspace,
                   NTTPrecomputedTables tables, uint32_t N, uint32_t L_a, uint32_t L_b,
                   uint32_t stride_A, uint32_t stride_B, uint32_t stride_ret) {
    const gpupi::ntt::NttParams P = gpupi::ntt::make_params(tables);
    gpupi::ntt::mul(P, A, B, ret, workspace, N, L_a, L_b, stride_A, stride_B, stride_ret);
}

size_t batch_mul_ntt_workspace_size(uint32_t N, uint32_t L_a, uint32_t L_b) {
    return gpupi::ntt::workspace_bytes(N, L_a, L_b);
}

namespace gpupi {

// Transform shape a product of La x Lb limbs gets (tune table or built-in rule).
void ntt_shape_of(uint32_t La, uint32_t Lb, int *log_k, int *M) {
    const ntt::Shape s = ntt::shape_tuned(La, Lb);
    *log_k = s.log_k;
    *M = s.M;
}

SpectrumShape spectrum_shape(uint64_t ncoef) {
    if (ncoef < 2u || ncoef > ((uint64_t)ntt::kMaxCosets << ntt::kMaxLog)) return SpectrumShape{0, 0};
    const ntt::Shape s = ntt::shape_for((uint32_t)ncoef, 1u);
    if (s.log_k <= ntt::kSplitLogC) return SpectrumShape{0, 0};
    return SpectrumShape{s.log_k, s.M};
}

uint64_t spectrum_words(SpectrumShape s, uint32_t N) { return (uint64_t)N * s.M * ntt::kPrimes << s.log_k; }

uint64_t spectrum_flag_words(uint32_t N, uint32_t Lc) {
    return (uint64_t)N * (((uint64_t)Lc + ntt::kCrtSpan - 1) / ntt::kCrtSpan);
}

bool spectrum_sum_fits(const uint32_t *La, const uint32_t *Lb, int terms) {
    // every coefficient of sum_t A_t B_t is below sum_t min(La_t, Lb_t) (2^32 - 1)^2,
    // which must stay below p0 p1 p2 for the CRT to be exact
    unsigned __int128 bound = 0;
    for (int t = 0; t < terms; ++t) {
        const uint64_t m = La[t] < Lb[t] ? La[t] : Lb[t];
        bound += (unsigned __int128)m * 0xffffffffull * 0xffffffffull;
    }
    unsigned __int128 cap = 1;
    for (int q = 0; q < ntt::kPrimes; ++q) cap *= ntt::kP[q];
    return bound < cap;
}

void spectrum_forward(const NTTPrecomputedTables &tables, SpectrumShape s, uint32_t N, const uint32_t *X,
                      uint64_t sX, uint32_t Lx, uint32_t *FX, const uint32_t *Y, uint64_t sY, uint32_t Ly,
                      uint32_t *FY, bool rows) {
    const ntt::NttParams P = ntt::make_params(tables);
    ntt::spectrum_forward(P, ntt::Shape{s.log_k, s.M}, N, X, sX, Lx, FX, Y, sY, Ly, FY, current_stream(), rows);
}

void spectrum_inverse(const NTTPrecomputedTables &tables, SpectrumShape s, uint32_t N, int terms,
                      const uint32_t *const *X, const uint32_t *const *Y, uint32_t *Fout, uint32_t *C, uint64_t sC,
                      uint32_t Lc, uint32_t *flags, bool rows, const SpectrumAddend *add) {
    const ntt::NttParams P = ntt::make_params(tables);
    ntt::spectrum_inverse(P, ntt::Shape{s.log_k, s.M}, N, terms, X, Y, Fout, C, sC, Lc, flags, current_stream(),
                          rows, add);
}

void spectrum_level_rows(const NTTPrecomputedTables &tables, SpectrumShape s, uint32_t N, uint32_t *Fpe,
                         uint32_t *Fpo, uint32_t *Fro, uint32_t *Fqo, uint32_t *Fqe, uint32_t *Fre) {
    const ntt::NttParams P = ntt::make_params(tables);
    cudaStream_t st = current_stream();
    ntt::rows_split_attr();
    const uint64_t VR = (uint64_t)N * s.M;
    const unsigned blocks = (unsigned)(VR * ntt::kPrimes * ((1ull << s.log_k) >> ntt::kSplitLogC));
    ntt::RowsLevelArgs a{Fpe, Fpo, Fro, Fqo, Fqe, Fre, s.log_k};
    // six residues read and four written per point, or five and three
    KernelTimed kt("ntt_rows_level", (Fpo ? 40.0 : 32.0) * (double)(1ull << s.log_k) * (double)VR * ntt::kPrimes);
    ntt::k_rows_level<<<blocks, (1 << ntt::kSplitLogC) / 16, ntt::rows_level_smem_bytes(), st>>>(P, a);
    count_launch();
}

}  // namespace gpupi
