// Batched exact multiplication by three-prime NTT (gpupi batch_mul_ntt.cu;
// API batch_mul_ntt.h:24-40).
//
// Per product row, per prime q, the workspace holds a transform of K = 2^k
// points (K >= L_a + L_b - 1, so the cyclic convolution has no wrap).
// Layout: F[row][q][K] (u32, plain residues).  A and B each get one such
// array (FA, FB); B is transformed once when it is broadcast (stride 0) and
// not at all when B is A (squaring).
//
// Pass structure (four-step decomposition K = R1 * [R2 *] C, C <= 4096):
//   k_cols<limbs,fwd>   load limbs, reduce mod p, R1-point DIF down each
//                       column of a [R1][TC] shared tile, twist by w_K^(c*k1),
//                       store                               (strided, coalesced in c)
//   k_cols<ws,fwd>      same on each segment for R2 (3-pass sizes only)
//   k_rows              C-point DIF of the A and B segments, pointwise
//                       product * K^-1, C-point inverse DIT, store   (contiguous)
//   k_cols<ws,inv>      untwist + inverse DIT on columns, mirror order
//   k_crt               Garner CRT to 96-bit coefficients, carry to limbs
//                       (+ carry_fixup_kernel when a row spans several tiles)
// Small products (K <= 4096) are one k_rows<from limbs> launch + k_crt.
// Products longer than 2^27 limbs (up to 2^28) use two cosets of 2^27
// points (see coef_residue), the third prime's 2-adicity being 27.
//
// The shared-memory butterflies are radix-2 levels separated by
// __syncthreads; every DIF level needs one Montgomery product per pair.
#include "ntt_core.cuh"
#include "carry_tile.cuh"
#include "batch_mul_ntt.h"

#include <stdio.h>
#include <stdlib.h>
#include <vector>

namespace gpupi {
namespace ntt {

static const uint32_t kP[kPrimes] = {3221225473u, 3489660929u, 3892314113u};
static const uint32_t kGen[kPrimes] = {5u, 3u, 3u};   // primitive roots

struct NttParams {
    PrimeConsts pr[kPrimes];
    CrtConsts crt;
    Tables tab;
    // two-coset split of a 2^28-point product: c1 = beta^(2^27) and
    // (c1 - 1)^-1, both Montgomery form, per prime
    uint32_t coset_c[kPrimes];
    uint32_t coset_cm1_inv[kPrimes];
};

// ---------------------------------------------------------------------------
// Host modular helpers (table construction)
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
static uint32_t h_inv_2_32(uint32_t p) {
    uint32_t x = p;
    for (int i = 0; i < 5; ++i) x *= 2u - p * x;
    return x;
}

static NttParams make_params(const NTTPrecomputedTables &t) {
    NttParams P{};
    for (int q = 0; q < kPrimes; ++q) {
        P.pr[q].p = kP[q];
        P.pr[q].pinv = h_inv_2_32(kP[q]);
    }
    P.crt.p0_inv_mod_p1_m = h_mont(h_inv(kP[0] % kP[1], kP[1]), kP[1]);
    P.crt.p0_inv_mod_p2_m = h_mont(h_inv(kP[0] % kP[2], kP[2]), kP[2]);
    P.crt.p1_inv_mod_p2_m = h_mont(h_inv(kP[1] % kP[2], kP[2]), kP[2]);
    P.crt.p0p1 = (uint64_t)kP[0] * kP[1];
    const uint32_t *lv1 = reinterpret_cast<const uint32_t *>(t.roots_table_lv1);
    const uint32_t *lv2 = reinterpret_cast<const uint32_t *>(t.roots_table_lv2);
    P.tab.tw_lo = lv1;
    P.tab.tw_hi = lv2;
    P.tab.beta_lo = lv2 + 2 * kPrimes * kHiSize;
    P.tab.beta_hi = P.tab.beta_lo + 2 * kPrimes * kLoSize;
    P.tab.inv2n = reinterpret_cast<const uint32_t *>(t.inv2n_table);
    for (int q = 0; q < kPrimes; ++q) {
        const uint32_t c1 = h_pow(kGen[q], 1ull << kMaxLog, kP[q]);
        P.coset_c[q] = h_mont(c1, kP[q]);
        const uint32_t cm1 = (c1 == 0u) ? kP[q] - 1u : c1 - 1u;   // c1 - 1 mod p without 32-bit overflow
        P.coset_cm1_inv[q] = h_mont(h_inv(cm1, kP[q]), kP[q]);
    }
    return P;
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
constexpr int kThreads = 256;

// Per-prime constants chosen by value (indexing the kernel-parameter arrays
// with a run-time prime index would force a local-memory copy).
__device__ __forceinline__ PrimeConsts prime_of(const NttParams &P, int q) {
    return q == 0 ? P.pr[0] : (q == 1 ? P.pr[1] : P.pr[2]);
}
__device__ __forceinline__ uint32_t sel3(const uint32_t (&v)[kPrimes], int q) {
    return q == 0 ? v[0] : (q == 1 ? v[1] : v[2]);
}

struct ColsArgs {
    const uint32_t *X;   // limbs (first forward pass only)
    uint64_t sX;
    uint32_t Lx;
    uint32_t *F;         // workspace of this operand: F[vrow][q][K]
    int log_k, log_s, log_r, log_tc;
    int coset_bits;      // 1: vrow = 2*row + coset (2^28-point products)
};

template <bool FROM_LIMBS, bool INVERSE>
__global__ void __launch_bounds__(kThreads) k_cols(NttParams P, ColsArgs a) {
    extern __shared__ uint32_t smem[];
    const uint32_t R = 1u << a.log_r;
    const uint32_t TC = 1u << a.log_tc;
    uint32_t *T = smem;
    uint32_t *tw = smem + R * TC;
    const int log_cols = a.log_s - a.log_r;
    const uint32_t ctiles = 1u << (log_cols - a.log_tc);
    const uint32_t nseg = 1u << (a.log_k - a.log_s);
    uint64_t b = blockIdx.x;
    const int q = (int)(b % kPrimes);
    b /= kPrimes;
    const uint32_t ct = (uint32_t)(b % ctiles);
    b /= ctiles;
    const uint32_t seg = (uint32_t)(b % nseg);
    const uint64_t vrow = b / nseg;
    const PrimeConsts pc = prime_of(P, q);
    const uint32_t p = pc.p, pinv = pc.pinv;
    const int dir = INVERSE ? 1 : 0;
    const uint64_t K = 1ull << a.log_k;
    const uint32_t *twhi = tw_hi_ptr(P.tab, dir, q);
    const uint32_t *twlo = tw_lo_ptr(P.tab, dir, q);
    for (uint32_t e = threadIdx.x; e < R / 2; e += blockDim.x) tw[e] = __ldg(twhi + (e << (13 - a.log_r)));
    uint32_t *F = a.F + vrow * 3 * K + (uint64_t)q * K + ((uint64_t)seg << a.log_s);
    const uint32_t c0 = ct << a.log_tc;
    const int twist_shift = kMaxLog - a.log_s;
    for (uint32_t idx = threadIdx.x; idx < R * TC; idx += blockDim.x) {
        const uint32_t r = idx >> a.log_tc;
        const uint32_t c = idx & (TC - 1u);
        const uint64_t i = ((uint64_t)r << log_cols) + c0 + c;
        uint32_t v;
        if (FROM_LIMBS) {
            const uint64_t row = vrow >> a.coset_bits;
            const uint32_t *xr = a.X + row * a.sX;
            v = (i < a.Lx) ? reduce_limb(xr[i], p) : 0u;
            if (a.coset_bits) {
                // a mod (x^K - c_j) = a_low + c_j * a_high, then scale by beta_j^i
                const uint64_t i2 = i + K;
                const uint32_t hi = (i2 < a.Lx) ? reduce_limb(xr[i2], p) : 0u;
                if ((vrow & 1u) == 0u) {
                    v = add_mod(v, hi, p);
                } else {
                    v = add_mod(v, mont_mul(hi, sel3(P.coset_c, q), p, pinv), p);
                    v = mont_mul(v, root_pow(beta_lo_ptr(P.tab, 0, q), beta_hi_ptr(P.tab, 0, q), (uint32_t)i, p, pinv),
                                 p, pinv);
                }
            }
        } else {
            v = F[i];
        }
        if (INVERSE) {
            const uint32_t E = ((c0 + c) * bitrev(r, a.log_r)) << twist_shift;
            v = mont_mul(v, root_pow(twlo, twhi, E, p, pinv), p, pinv);
        }
        T[idx] = v;
    }
    __syncthreads();
    tile_transform<INVERSE>(T, a.log_r, a.log_tc, tw, p, pinv);
    for (uint32_t idx = threadIdx.x; idx < R * TC; idx += blockDim.x) {
        const uint32_t r = idx >> a.log_tc;
        const uint32_t c = idx & (TC - 1u);
        const uint64_t i = ((uint64_t)r << log_cols) + c0 + c;
        uint32_t v = T[idx];
        if (!INVERSE) {
            const uint32_t E = ((c0 + c) * bitrev(r, a.log_r)) << twist_shift;
            v = mont_mul(v, root_pow(twlo, twhi, E, p, pinv), p, pinv);
        }
        F[i] = v;
    }
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
    int log_k, log_c;
    int b_bcast;         // B row 0 serves every row
    int square;          // B is A
    int coset_bits;      // virtual rows are (row, coset) pairs
};

template <bool FROM_LIMBS>
__global__ void __launch_bounds__(kThreads) k_rows(NttParams P, RowsArgs a) {
    extern __shared__ uint32_t smem[];
    const uint32_t C = 1u << a.log_c;
    uint32_t *SA = smem;
    uint32_t *SB = smem + C;
    uint32_t *twf = smem + 2 * C;
    uint32_t *twi = twf + C / 2;
    uint64_t b = blockIdx.x;
    const int q = (int)(b % kPrimes);
    b /= kPrimes;
    const uint32_t nseg = 1u << (a.log_k - a.log_c);
    const uint32_t seg = (uint32_t)(b % nseg);
    const uint64_t vrow = b / nseg;
    const uint64_t brow = a.b_bcast ? (vrow & ((1u << a.coset_bits) - 1u)) : vrow;
    const PrimeConsts pc = prime_of(P, q);
    const uint32_t p = pc.p, pinv = pc.pinv;
    const uint64_t K = 1ull << a.log_k;
    const uint32_t scale = __ldg(P.tab.inv2n + a.log_k * kPrimes + q);
    const uint32_t *thf = tw_hi_ptr(P.tab, 0, q);
    const uint32_t *thi = tw_hi_ptr(P.tab, 1, q);
    for (uint32_t e = threadIdx.x; e < C / 2; e += blockDim.x) {
        twf[e] = __ldg(thf + (e << (13 - a.log_c)));
        twi[e] = __ldg(thi + (e << (13 - a.log_c)));
    }
    const uint64_t offA = vrow * 3 * K + (uint64_t)q * K + ((uint64_t)seg << a.log_c);
    const uint64_t offB = brow * 3 * K + (uint64_t)q * K + ((uint64_t)seg << a.log_c);
    for (uint32_t i = threadIdx.x; i < C; i += blockDim.x) {
        if (FROM_LIMBS) {
            SA[i] = (i < a.La) ? reduce_limb(a.A[vrow * a.sA + i], p) : 0u;
            if (!a.square) SB[i] = (i < a.Lb) ? reduce_limb(a.B[brow * a.sB + i], p) : 0u;
        } else {
            SA[i] = a.FA[offA + i];
            if (!a.square) SB[i] = a.FB[offB + i];
        }
    }
    __syncthreads();
    tile_transform<false>(SA, a.log_c, 0, twf, p, pinv);
    if (!a.square) tile_transform<false>(SB, a.log_c, 0, twf, p, pinv);
    for (uint32_t i = threadIdx.x; i < C; i += blockDim.x) {
        const uint32_t x = SA[i];
        const uint32_t y = a.square ? x : SB[i];
        SA[i] = mont_mul(mont_mul(x, y, p, pinv), scale, p, pinv);
    }
    __syncthreads();
    tile_transform<true>(SA, a.log_c, 0, twi, p, pinv);
    for (uint32_t i = threadIdx.x; i < C; i += blockDim.x) a.FA[offA + i] = SA[i];
}

// ---------------------------------------------------------------------------
// Register-stage kernels (ntt_core.cuh: Stage / run_stages).  Same arithmetic
// as k_cols / k_rows, with 16 residues per thread and shared memory touched
// only between stages of up to four radix-2 levels.
// ---------------------------------------------------------------------------
constexpr int kTile = 4096;                    // elements per register-stage CTA tile
constexpr int kTilePad = kTile + kTile / 32;   // padded shared-memory words

__device__ __forceinline__ uint32_t load_operand(const NttParams &P, const ColsArgs &a, const uint32_t *F,
                                                 uint64_t vrow, uint64_t i, uint64_t K, int q, uint32_t p,
                                                 uint32_t pinv) {
    (void)F;
    const uint64_t row = vrow >> a.coset_bits;
    const uint32_t *xr = a.X + row * a.sX;
    uint32_t v = (i < a.Lx) ? reduce_limb(xr[i], p) : 0u;
    if (a.coset_bits) {
        // a mod (x^K - c_j) = a_low + c_j * a_high, then scale by beta_j^i
        const uint64_t i2 = i + K;
        const uint32_t hi = (i2 < a.Lx) ? reduce_limb(xr[i2], p) : 0u;
        if ((vrow & 1u) == 0u) {
            v = add_mod(v, hi, p);
        } else {
            v = add_mod(v, mont_mul(hi, sel3(P.coset_c, q), p, pinv), p);
            v = mont_mul(v, root_pow(beta_lo_ptr(P.tab, 0, q), beta_hi_ptr(P.tab, 0, q), (uint32_t)i, p, pinv), p,
                         pinv);
        }
    }
    return v;
}

// Column pass: R = 2^LOG_R (<= 512) points per column, TC = 4096 / R columns.
template <int LOG_R, bool FROM_LIMBS, bool INVERSE>
__global__ void __launch_bounds__(kThreads) k_cols_r(NttParams P, ColsArgs a) {
    constexpr int LOG_TC = 12 - LOG_R;
    constexpr int NS = StagePlan<LOG_R>::n;
    using First = typename ExecStage<LOG_R, LOG_TC, INVERSE, 0>::S;
    using Last = typename ExecStage<LOG_R, LOG_TC, INVERSE, NS - 1>::S;
    __shared__ uint32_t Sm[kTilePad];
    __shared__ uint32_t tw[(1 << LOG_R) / 2 > 0 ? (1 << LOG_R) / 2 : 1];
    const int log_cols = a.log_s - LOG_R;
    const uint32_t ctiles = 1u << (log_cols - LOG_TC);
    const uint32_t nseg = 1u << (a.log_k - a.log_s);
    uint64_t b = blockIdx.x;
    const int q = (int)(b % kPrimes);
    b /= kPrimes;
    const uint32_t ct = (uint32_t)(b % ctiles);
    b /= ctiles;
    const uint32_t seg = (uint32_t)(b % nseg);
    const uint64_t vrow = b / nseg;
    const PrimeConsts pc = prime_of(P, q);
    const uint32_t p = pc.p, pinv = pc.pinv;
    const int dir = INVERSE ? 1 : 0;
    const uint64_t K = 1ull << a.log_k;
    const uint32_t *twhi = tw_hi_ptr(P.tab, dir, q);
    const uint32_t *twlo = tw_lo_ptr(P.tab, dir, q);
    for (uint32_t e = threadIdx.x; e < (1u << LOG_R) / 2; e += kThreads) tw[e] = __ldg(twhi + (e << (13 - LOG_R)));
    uint32_t *F = a.F + vrow * 3 * K + (uint64_t)q * K + ((uint64_t)seg << a.log_s);
    const uint32_t c0 = ct << LOG_TC;
    const int twist_shift = kMaxLog - a.log_s;
    const uint32_t t = threadIdx.x;
    uint32_t x[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        uint32_t pos, c;
        First::elem(t, j, pos, c);
        const uint64_t i = ((uint64_t)pos << log_cols) + c0 + c;
        uint32_t v = FROM_LIMBS ? load_operand(P, a, F, vrow, i, K, q, p, pinv) : F[i];
        if (INVERSE) {
            const uint32_t E = ((c0 + c) * bitrev(pos, LOG_R)) << twist_shift;
            v = mont_mul(v, root_pow(twlo, twhi, E, p, pinv), p, pinv);
        }
        x[j] = v;
    }
    __syncthreads();   // twiddle table ready
    run_stages<LOG_R, LOG_TC, INVERSE, 0>(x, Sm, t, tw, p, pinv);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        uint32_t pos, c;
        Last::elem(t, j, pos, c);
        const uint64_t i = ((uint64_t)pos << log_cols) + c0 + c;
        uint32_t v = x[j];
        if (!INVERSE) {
            const uint32_t E = ((c0 + c) * bitrev(pos, LOG_R)) << twist_shift;
            v = mont_mul(v, root_pow(twlo, twhi, E, p, pinv), p, pinv);
        }
        F[i] = v;
    }
}

// Fused row pass on C = 2^LOG_C points (T = C/16 threads): forward stages of
// A then B (A stays in registers while B reuses the shared tile), pointwise
// product * scale, inverse stages.  The last forward and the first inverse
// stage share one thread mapping, so the product never leaves registers.
template <int LOG_C, bool FROM_LIMBS>
__global__ void __launch_bounds__(kThreads) k_rows_r(NttParams P, RowsArgs a) {
    constexpr int C = 1 << LOG_C;
    constexpr int NS = StagePlan<LOG_C>::n;
    using First = typename ExecStage<LOG_C, 0, false, 0>::S;
    using Mid = typename ExecStage<LOG_C, 0, false, NS - 1>::S;
    using Out = typename ExecStage<LOG_C, 0, true, NS - 1>::S;
    __shared__ uint32_t Sm[C + C / 32];
    __shared__ uint32_t twf[C / 2], twi[C / 2];
    uint64_t b = blockIdx.x;
    const int q = (int)(b % kPrimes);
    b /= kPrimes;
    const uint32_t nseg = 1u << (a.log_k - LOG_C);
    const uint32_t seg = (uint32_t)(b % nseg);
    const uint64_t vrow = b / nseg;
    const uint64_t brow = a.b_bcast ? (vrow & ((1u << a.coset_bits) - 1u)) : vrow;
    const PrimeConsts pc = prime_of(P, q);
    const uint32_t p = pc.p, pinv = pc.pinv;
    const uint64_t K = 1ull << a.log_k;
    const uint32_t scale = __ldg(P.tab.inv2n + a.log_k * kPrimes + q);
    const uint32_t *thf = tw_hi_ptr(P.tab, 0, q);
    const uint32_t *thi = tw_hi_ptr(P.tab, 1, q);
    for (uint32_t e = threadIdx.x; e < C / 2; e += blockDim.x) {
        twf[e] = __ldg(thf + (e << (13 - LOG_C)));
        twi[e] = __ldg(thi + (e << (13 - LOG_C)));
    }
    const uint64_t offA = vrow * 3 * K + (uint64_t)q * K + ((uint64_t)seg << LOG_C);
    const uint64_t offB = brow * 3 * K + (uint64_t)q * K + ((uint64_t)seg << LOG_C);
    const uint32_t t = threadIdx.x;
    uint32_t xa[16], xb[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        uint32_t pos, c;
        First::elem(t, j, pos, c);
        if (FROM_LIMBS) {
            xa[j] = (pos < a.La) ? reduce_limb(a.A[vrow * a.sA + pos], p) : 0u;
            xb[j] = (!a.square && pos < a.Lb) ? reduce_limb(a.B[brow * a.sB + pos], p) : 0u;
        } else {
            xa[j] = a.FA[offA + pos];
            xb[j] = a.square ? 0u : a.FB[offB + pos];
        }
    }
    __syncthreads();
    run_stages<LOG_C, 0, false, 0>(xa, Sm, t, twf, p, pinv);
    if (!a.square) {
        // the tile is free again: every thread has passed the last stage's loads
        __syncthreads();
        run_stages<LOG_C, 0, false, 0>(xb, Sm, t, twf, p, pinv);
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const uint32_t y = a.square ? xa[j] : xb[j];
        xa[j] = mont_mul(mont_mul(xa[j], y, p, pinv), scale, p, pinv);
    }
    __syncthreads();
    run_stages<LOG_C, 0, true, 0>(xa, Sm, t, twi, p, pinv);
    (void)sizeof(Mid);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        uint32_t pos, c;
        Out::elem(t, j, pos, c);
        a.FA[offA + pos] = xa[j];
    }
}

__device__ __forceinline__ void garner(const NttParams &P, uint32_t r0, uint32_t r1, uint32_t r2,
                                       uint32_t (&out)[3]) {
    const uint32_t p1 = P.pr[1].p, q1 = P.pr[1].pinv;
    const uint32_t p2 = P.pr[2].p, q2 = P.pr[2].pinv;
    const uint32_t t1 = mont_mul(sub_mod(r1, r0, p1), P.crt.p0_inv_mod_p1_m, p1, q1);
    const uint32_t u = mont_mul(sub_mod(r2, r0, p2), P.crt.p0_inv_mod_p2_m, p2, q2);
    const uint32_t t2 = mont_mul(sub_mod(u, t1, p2), P.crt.p1_inv_mod_p2_m, p2, q2);
    const unsigned __int128 x =
        (unsigned __int128)P.crt.p0p1 * t2 + (uint64_t)P.pr[0].p * t1 + r0;
    out[0] = (uint32_t)x;
    out[1] = (uint32_t)(x >> 32);
    out[2] = (uint32_t)(x >> 64);
}

constexpr int kCrtV = 4;
constexpr uint32_t kCrtSpan = kThreads * kCrtV;   // 1024 limbs per tile

struct CrtArgs {
    const uint32_t *F;
    int log_k;
    uint32_t *C;
    uint64_t sC;
    uint32_t Lc;
    uint32_t tiles;
    uint32_t *flags;
};

// Residue mod p_q of convolution coefficient n.  Without cosets it is read
// directly.  With two cosets (K = transform length, product length <= 2K) the
// row holds r0 = C mod (x^K - 1) and beta^i * r1, r1 = C mod (x^K - c1):
// C_high = (r1 - r0) / (c1 - 1), C_low = r0 - C_high.
template <bool COSET>
__device__ __forceinline__ uint32_t coef_residue(const NttParams &P, const uint32_t *F0, uint64_t K, int q,
                                                 uint64_t n) {
    if (!COSET) return F0[(uint64_t)q * K + n];
    const PrimeConsts pc = prime_of(P, q);
    const uint32_t p = pc.p, pinv = pc.pinv;
    const uint64_t i = n & (K - 1);
    const uint32_t r0 = F0[(uint64_t)q * K + i];
    const uint32_t s1 = F0[3 * K + (uint64_t)q * K + i];
    const uint32_t r1 =
        mont_mul(s1, root_pow(beta_lo_ptr(P.tab, 1, q), beta_hi_ptr(P.tab, 1, q), (uint32_t)i, p, pinv), p, pinv);
    const uint32_t hi = mont_mul(sub_mod(r1, r0, p), sel3(P.coset_cm1_inv, q), p, pinv);
    return (n >= K) ? hi : sub_mod(r0, hi, p);
}

template <bool COSET>
__device__ __forceinline__ void crt_chunk(const NttParams &P, const uint32_t *F0, uint64_t K,
                                          uint32_t Lc, int64_t base, uint32_t (&S)[kCrtV + 3]) {
    uint32_t c[kCrtV][3];
    const uint64_t span = COSET ? 2 * K : K;
    if (!COSET && base >= 0 && (uint64_t)base + kCrtV <= K && base + kCrtV <= (int64_t)Lc) {
        // whole chunk inside the row: one 128-bit load per prime (K and base are multiples of 4)
        const uint4 r0 = *reinterpret_cast<const uint4 *>(F0 + base);
        const uint4 r1 = *reinterpret_cast<const uint4 *>(F0 + K + base);
        const uint4 r2 = *reinterpret_cast<const uint4 *>(F0 + 2 * K + base);
        garner(P, r0.x, r1.x, r2.x, c[0]);
        garner(P, r0.y, r1.y, r2.y, c[1]);
        garner(P, r0.z, r1.z, r2.z, c[2]);
        garner(P, r0.w, r1.w, r2.w, c[3]);
        chunk_sum3<kCrtV>(c, S);
        return;
    }
#pragma unroll
    for (int v = 0; v < kCrtV; ++v) {
        const int64_t i = base + v;
        if (i >= 0 && (uint64_t)i < span && i < (int64_t)Lc) {
            garner(P, coef_residue<COSET>(P, F0, K, 0, i), coef_residue<COSET>(P, F0, K, 1, i),
                   coef_residue<COSET>(P, F0, K, 2, i), c[v]);
        } else {
            c[v][0] = c[v][1] = c[v][2] = 0u;
        }
    }
    chunk_sum3<kCrtV>(c, S);
}

template <bool COSET>
__global__ void __launch_bounds__(kThreads) k_crt(NttParams P, CrtArgs a) {
    __shared__ uint32_t sg[kThreads / 32], sp[kThreads / 32], spre[kThreads / 32];
    const uint32_t tile = blockIdx.x;
    const uint64_t row = tile / a.tiles;
    const uint32_t t = tile - (uint32_t)row * a.tiles;
    const uint64_t K = 1ull << a.log_k;
    const uint32_t *F0 = a.F + row * (COSET ? 6 : 3) * K;
    const int64_t base = (int64_t)t * kCrtSpan + threadIdx.x * kCrtV;
    uint32_t S[kCrtV + 3];
    crt_chunk<COSET>(P, F0, K, a.Lc, base, S);
    uint32_t H[3];
    H[0] = __shfl_up_sync(0xffffffffu, S[kCrtV], 1);
    H[1] = __shfl_up_sync(0xffffffffu, S[kCrtV + 1], 1);
    H[2] = __shfl_up_sync(0xffffffffu, S[kCrtV + 2], 1);
    if (lane_id() == 0) {
        uint32_t Sp[kCrtV + 3];
        crt_chunk<COSET>(P, F0, K, a.Lc, base - kCrtV, Sp);
        H[0] = Sp[kCrtV];
        H[1] = Sp[kCrtV + 1];
        H[2] = Sp[kCrtV + 2];
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

static int transform_log(uint32_t La, uint32_t Lb) {
    const uint64_t need = (uint64_t)La + Lb - 1u;
    int k = ceil_log2(need < 2 ? 2 : need);
    return k < 1 ? 1 : k;
}

template <class Kern>
static void set_smem(Kern kern, size_t bytes) {
    if (bytes > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

static void launch_cols(bool from_limbs, bool inverse, const NttParams &P, const ColsArgs &a,
                        uint64_t vrows, cudaStream_t st) {
    const uint64_t ctiles = 1ull << (a.log_s - a.log_r - a.log_tc);
    const uint64_t nseg = 1ull << (a.log_k - a.log_s);
    const uint64_t blocks = vrows * kPrimes * nseg * ctiles;
    const size_t smem = ((size_t(1) << (a.log_r + a.log_tc)) + (size_t(1) << (a.log_r - 1))) * 4;
    // algorithmic bytes: 12 B per coefficient (3 primes x 4 B) read and written;
    // the first pass reads each limb once instead
    const double K = (double)(1ull << a.log_k);
    const double bytes = from_limbs ? (4.0 * a.Lx * (double)(vrows >> a.coset_bits) + 12.0 * K * (double)vrows)
                                    : 24.0 * K * (double)vrows;
    KernelTimed kt(from_limbs ? "ntt_cols_fwd_first" : (inverse ? "ntt_cols_inv" : "ntt_cols_fwd"), bytes);
    if (from_limbs) {
        set_smem(k_cols<true, false>, smem);
        k_cols<true, false><<<(unsigned)blocks, kThreads, smem, st>>>(P, a);
    } else if (!inverse) {
        set_smem(k_cols<false, false>, smem);
        k_cols<false, false><<<(unsigned)blocks, kThreads, smem, st>>>(P, a);
    } else {
        set_smem(k_cols<false, true>, smem);
        k_cols<false, true><<<(unsigned)blocks, kThreads, smem, st>>>(P, a);
    }
    count_launch();
}

static bool use_radix2() {
    static const bool v = [] {
        const char *e = getenv("GPUPI_NTT_RADIX2");
        return e && e[0] == '1';
    }();
    return v;
}

template <bool FL, bool INV>
static void cols_r_dispatch(int log_r, unsigned blocks, const NttParams &P, const ColsArgs &a, cudaStream_t st) {
    switch (log_r) {
        case 1: k_cols_r<1, FL, INV><<<blocks, kThreads, 0, st>>>(P, a); break;
        case 2: k_cols_r<2, FL, INV><<<blocks, kThreads, 0, st>>>(P, a); break;
        case 3: k_cols_r<3, FL, INV><<<blocks, kThreads, 0, st>>>(P, a); break;
        case 4: k_cols_r<4, FL, INV><<<blocks, kThreads, 0, st>>>(P, a); break;
        case 5: k_cols_r<5, FL, INV><<<blocks, kThreads, 0, st>>>(P, a); break;
        case 6: k_cols_r<6, FL, INV><<<blocks, kThreads, 0, st>>>(P, a); break;
        case 7: k_cols_r<7, FL, INV><<<blocks, kThreads, 0, st>>>(P, a); break;
        case 8: k_cols_r<8, FL, INV><<<blocks, kThreads, 0, st>>>(P, a); break;
        default: k_cols_r<9, FL, INV><<<blocks, kThreads, 0, st>>>(P, a); break;
    }
}

static void launch_cols_r(bool from_limbs, bool inverse, const NttParams &P, const ColsArgs &a, uint64_t vrows,
                          cudaStream_t st) {
    const uint64_t ctiles = 1ull << (a.log_s - a.log_r - (12 - a.log_r));
    const uint64_t nseg = 1ull << (a.log_k - a.log_s);
    const unsigned blocks = (unsigned)(vrows * kPrimes * nseg * ctiles);
    const double K = (double)(1ull << a.log_k);
    const double bytes = from_limbs ? (4.0 * a.Lx * (double)(vrows >> a.coset_bits) + 12.0 * K * (double)vrows)
                                    : 24.0 * K * (double)vrows;
    KernelTimed kt(from_limbs ? "ntt_cols_fwd_first" : (inverse ? "ntt_cols_inv" : "ntt_cols_fwd"), bytes);
    if (from_limbs)
        cols_r_dispatch<true, false>(a.log_r, blocks, P, a, st);
    else if (!inverse)
        cols_r_dispatch<false, false>(a.log_r, blocks, P, a, st);
    else
        cols_r_dispatch<false, true>(a.log_r, blocks, P, a, st);
    count_launch();
}

template <bool FL>
static void rows_r_dispatch(int log_c, unsigned blocks, const NttParams &P, const RowsArgs &r, cudaStream_t st) {
    switch (log_c) {
        case 9: k_rows_r<9, FL><<<blocks, 32, 0, st>>>(P, r); break;
        case 10: k_rows_r<10, FL><<<blocks, 64, 0, st>>>(P, r); break;
        case 11: k_rows_r<11, FL><<<blocks, 128, 0, st>>>(P, r); break;
        default: k_rows_r<12, FL><<<blocks, 256, 0, st>>>(P, r); break;
    }
}

static int tc_for(int log_r, int log_cols) {
    int log_tc = 12 - log_r;
    if (log_tc < 4) log_tc = 4;
    if (log_tc > log_cols) log_tc = log_cols;
    return log_tc;
}

size_t workspace_bytes(uint32_t N, uint32_t La, uint32_t Lb) {
    if (N == 0u || La == 0u || Lb == 0u) return 0;
    const int log_k = transform_log(La, Lb);
    const uint64_t K = 1ull << log_k;
    const uint64_t Lc = (uint64_t)La + Lb;
    const uint64_t tiles = (Lc + kCrtSpan - 1) / kCrtSpan;
    return (size_t)(2ull * N * 3 * K * 4 + N * tiles * 4 + 256);
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
    const int log_total = transform_log(La, Lb);
    if (log_total > kMaxLog + 1) {
        fprintf(stderr, "gpupi_b200: product of %u limbs exceeds the 2^28-point limit\n", Lc);
        return;
    }
    // Above 2^27 points the product is split into two cosets of 2^27 points.
    const int cb = (log_total > kMaxLog) ? 1 : 0;
    const int log_k = log_total - cb;
    const uint64_t K = 1ull << log_k;
    const uint64_t VR = (uint64_t)N << cb;   // virtual rows (row, coset)
    const bool square = (A == B && La == Lb && sA == sB);
    const bool bcast = (!square && sB == 0u && N > 1u);
    uint32_t *FA = ws;
    uint32_t *FB = square ? FA : ws + VR * 3 * K;
    const uint64_t tiles = ((uint64_t)Lc + kCrtSpan - 1) / kCrtSpan;
    uint32_t *flags = ws + 2ull * VR * 3 * K;

    if (log_k <= 12) {
        RowsArgs r{A, sA, La, B, sB, Lb, FA, FB, log_k, log_k, bcast ? 1 : 0, square ? 1 : 0, 0};
        KernelTimed kt("ntt_local", 4.0 * N * ((double)La + (square ? 0 : Lb)) + 12.0 * K * N);
        if (log_k >= 9 && !use_radix2()) {
            rows_r_dispatch<true>(log_k, (unsigned)(N * kPrimes), P, r, st);
        } else {
            const size_t smem = (size_t)3 * K * 4;
            set_smem(k_rows<true>, smem);
            k_rows<true><<<(unsigned)(N * kPrimes), kThreads, smem, st>>>(P, r);
        }
        count_launch();
    } else {
        const int log_c = 12;
        const int rest = log_k - log_c;
        const bool r2 = use_radix2();
        int passes[2];
        int npass;
        if (rest <= (r2 ? 10 : 9)) {
            passes[0] = rest;
            npass = 1;
        } else {
            passes[0] = (rest + 1) / 2;
            passes[1] = rest / 2;
            npass = 2;
        }
        // forward column passes for A and (unless squaring) B
        for (int op = 0; op < (square ? 1 : 2); ++op) {
            const uint32_t *X = op == 0 ? A : B;
            const uint64_t sX = op == 0 ? sA : sB;
            const uint32_t Lx = op == 0 ? La : Lb;
            uint32_t *F = op == 0 ? FA : FB;
            const uint64_t vrows = (op == 1 && bcast) ? (1ull << cb) : VR;
            int log_s = log_k;
            for (int ps = 0; ps < npass; ++ps) {
                ColsArgs a{X, sX, Lx, F, log_k, log_s, passes[ps], 0, cb};
                if (r2) {
                    a.log_tc = tc_for(passes[ps], log_s - passes[ps]);
                    launch_cols(ps == 0, false, P, a, vrows, st);
                } else {
                    a.log_tc = 12 - passes[ps];
                    launch_cols_r(ps == 0, false, P, a, vrows, st);
                }
                log_s -= passes[ps];
            }
        }
        RowsArgs r{A, sA, La, B, sB, Lb, FA, FB, log_k, log_c, bcast ? 1 : 0, square ? 1 : 0, cb};
        const uint64_t blocks = VR * kPrimes * (K >> log_c);
        {
            KernelTimed kt("ntt_rows_fused", 12.0 * (double)K * ((square ? 2.0 : 3.0) * (double)VR));
            if (r2) {
                const size_t smem = (size_t)3 * (1u << log_c) * 4;
                set_smem(k_rows<false>, smem);
                k_rows<false><<<(unsigned)blocks, kThreads, smem, st>>>(P, r);
            } else {
                rows_r_dispatch<false>(log_c, (unsigned)blocks, P, r, st);
            }
            count_launch();
        }
        // inverse column passes, innermost first
        int log_s = log_c;
        for (int ps = npass - 1; ps >= 0; --ps) {
            log_s += passes[ps];
            ColsArgs a{nullptr, 0, 0, FA, log_k, log_s, passes[ps], 0, 0};
            if (r2) {
                a.log_tc = tc_for(passes[ps], log_s - passes[ps]);
                launch_cols(false, true, P, a, VR, st);
            } else {
                a.log_tc = 12 - passes[ps];
                launch_cols_r(false, true, P, a, VR, st);
            }
        }
    }
    CrtArgs c{FA, log_k, C, sC, Lc, (uint32_t)tiles, flags};
    KernelTimed kt("ntt_crt_carry", 12.0 * (double)Lc * N + 4.0 * (double)Lc * N);
    if (cb)
        k_crt<true><<<(unsigned)(N * tiles), kThreads, 0, st>>>(P, c);
    else
        k_crt<false><<<(unsigned)(N * tiles), kThreads, 0, st>>>(P, c);
    count_launch();
    if (tiles > 1) launch_carry_fixup(false, C, sC, N, Lc, (uint32_t)tiles, kCrtSpan, flags, st);
}

void build_tables(std::vector<uint32_t> &lv1, std::vector<uint32_t> &lv2, std::vector<uint32_t> &inv2n) {
    lv1.assign(65536u * 3u, 0u);
    lv2.assign(65536u * 3u, 0u);
    inv2n.assign(33u * 3u, 0u);
    for (int q = 0; q < kPrimes; ++q) {
        const uint32_t p = kP[q];
        const uint32_t w = h_pow(kGen[q], (p - 1u) >> kMaxLog, p);
        const uint32_t beta = kGen[q];
        for (int dir = 0; dir < 2; ++dir) {
            const uint32_t base = dir ? h_inv(w, p) : w;
            const uint32_t bb = dir ? h_inv(beta, p) : beta;
            uint32_t x = 1u;
            for (uint32_t e = 0; e < kLoSize; ++e) {
                lv1[(size_t)(dir * kPrimes + q) * kLoSize + e] = h_mont(x, p);
                x = h_mul(x, base, p);
            }
            const uint32_t step = h_pow(base, kLoSize, p);
            x = 1u;
            for (uint32_t e = 0; e < kHiSize; ++e) {
                lv2[(size_t)(dir * kPrimes + q) * kHiSize + e] = h_mont(x, p);
                x = h_mul(x, step, p);
            }
            const size_t blo = 2u * kPrimes * kHiSize;
            const size_t bhi = blo + 2u * kPrimes * kLoSize;
            x = 1u;
            for (uint32_t e = 0; e < kLoSize; ++e) {
                lv2[blo + (size_t)(dir * kPrimes + q) * kLoSize + e] = h_mont(x, p);
                x = h_mul(x, bb, p);
            }
            const uint32_t bstep = h_pow(bb, kLoSize, p);
            x = 1u;
            for (uint32_t e = 0; e < kHiSize; ++e) {
                lv2[bhi + (size_t)(dir * kPrimes + q) * kHiSize + e] = h_mont(x, p);
                x = h_mul(x, bstep, p);
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
