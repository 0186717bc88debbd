// Three-prime number-theoretic transform building blocks (sm_100a).
//
// An exact product of 32-bit-limb integers is computed as a cyclic
// convolution modulo three primes p0 < p1 < p2 (all just below 2^32, product
// ~2^95.1) and recombined by Garner's CRT.  A convolution coefficient is at
// most min(L_a, L_b) * (2^32-1)^2 < 2^92 for products up to 2^29 limbs, so
// the CRT value is the exact coefficient.
//
//   p0 = 3 * 2^30 + 1   (2-adicity 30)
//   p1 = 13 * 2^28 + 1  (2-adicity 28)
//   p2 = 29 * 2^27 + 1  (2-adicity 27)
//
// Direct transforms are limited to 2^27 points (p2's 2-adicity); products of
// length up to 2^28 are split into the residues mod x^K - 1 and mod
// x^K - beta^K (two cosets of 2^27 points each).
//
// Arithmetic is Montgomery with R = 2^32 on 32-bit words.  Data stays in plain
// form; twiddles are stored in Montgomery form, so mont(x, w_M) = x*w.
#pragma once

#include "common.cuh"

namespace gpupi {
namespace ntt {

constexpr int kPrimes = 3;
constexpr int kMaxLog = 27;          // largest direct transform
constexpr int kLoBits = 14;          // two-level twiddle split: 2^27 = 2^14 * 2^13
constexpr uint32_t kLoSize = 1u << kLoBits;
constexpr uint32_t kHiSize = 1u << (kMaxLog - kLoBits);   // 8192

struct PrimeConsts {
    uint32_t p;
    uint32_t pinv;   // p^-1 mod 2^32
};

// Table layout inside NTTPrecomputedTables (raw u32 views of the uint3 buffers):
//   lv1: [dir][prime][kLoSize]  TW_LO[e]   = w^e            (w = primitive 2^27-th root; dir 1 = w^-1)
//   lv2: [dir][prime][kHiSize]  TW_HI[e]   = w^(e * 2^14)   (= 8192-th roots)
//        then [dir][prime][kLoSize] BETA_LO[e] = beta^e, [dir][prime][kHiSize] BETA_HI[e] = beta^(e*2^14)
//   inv2n: [k][prime]           K^-1 * R^2 mod p  (K = 2^k), folds the 1/K of the
//                                inverse and the R^-1 of the pointwise product
//   Everything in Montgomery form.
struct Tables {
    const uint32_t *tw_lo;     // lv1
    const uint32_t *tw_hi;     // lv2
    const uint32_t *beta_lo;   // lv2 + 2*3*kHiSize
    const uint32_t *beta_hi;   // beta_lo + 2*3*kLoSize
    const uint32_t *inv2n;     // 33*3
};

__device__ __forceinline__ const uint32_t *tw_lo_ptr(const Tables &t, int dir, int q) {
    return t.tw_lo + ((size_t)dir * kPrimes + q) * kLoSize;
}
__device__ __forceinline__ const uint32_t *tw_hi_ptr(const Tables &t, int dir, int q) {
    return t.tw_hi + ((size_t)dir * kPrimes + q) * kHiSize;
}
__device__ __forceinline__ const uint32_t *beta_lo_ptr(const Tables &t, int dir, int q) {
    return t.beta_lo + ((size_t)dir * kPrimes + q) * kLoSize;
}
__device__ __forceinline__ const uint32_t *beta_hi_ptr(const Tables &t, int dir, int q) {
    return t.beta_hi + ((size_t)dir * kPrimes + q) * kHiSize;
}

__device__ __forceinline__ uint32_t mont_mul(uint32_t a, uint32_t b, uint32_t p, uint32_t pinv) {
    // a*b < p*2^32 required (a < 2^32, b < p).  Result in [0, p).
    const uint64_t t = (uint64_t)a * b;
    const uint32_t tlo = (uint32_t)t;
    const uint32_t thi = (uint32_t)(t >> 32);
    const uint32_t m = tlo * pinv;
    const uint32_t mh = __umulhi(m, p);
    const uint32_t r = thi - mh;
    return (thi < mh) ? r + p : r;
}

__device__ __forceinline__ uint32_t add_mod(uint32_t a, uint32_t b, uint32_t p) {
    const uint32_t s = a + b;
    const uint32_t t = s - p;
    return (s < a || s >= p) ? t : s;
}

__device__ __forceinline__ uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t p) {
    const uint32_t d = a - b;
    return (a < b) ? d + p : d;
}

__device__ __forceinline__ uint32_t reduce_limb(uint32_t a, uint32_t p) {
    return (a >= p) ? a - p : a;   // a < 2^32 < 2p
}

// w^E for E < 2^27 (w the table's root), Montgomery form.
__device__ __forceinline__ uint32_t root_pow(const uint32_t *lo, const uint32_t *hi, uint32_t E,
                                             uint32_t p, uint32_t pinv) {
    return mont_mul(__ldg(lo + (E & (kLoSize - 1))), __ldg(hi + (E >> kLoBits)), p, pinv);
}

__device__ __forceinline__ uint32_t bitrev(uint32_t x, int bits) {
    return bits ? (__brev(x) >> (32 - bits)) : 0u;
}

// In-place radix-2 transform of every column of a shared-memory tile
// T[R][TC] (row-major, R = 2^log_r points per column, TC = 2^log_tc columns).
// Forward: decimation in frequency, natural order in, bit-reversed order out.
// Inverse: decimation in time, bit-reversed in, natural out (unscaled).
// tw[e] = (w_R)^e or (w_R)^-e for e < R/2, Montgomery form, in shared memory.
template <bool INVERSE>
__device__ __forceinline__ void tile_transform(uint32_t *T, int log_r, int log_tc,
                                               const uint32_t *tw, uint32_t p, uint32_t pinv) {
    const uint32_t nb = 1u << (log_r - 1 + log_tc);
    const uint32_t tcmask = (1u << log_tc) - 1u;
    for (int step = 0; step < log_r; ++step) {
        const int lh = INVERSE ? step : (log_r - 1 - step);
        const uint32_t h = 1u << lh;
        const int twshift = log_r - 1 - lh;
        for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) {
            const uint32_t c = b & tcmask;
            const uint32_t j = b >> log_tc;
            const uint32_t pos = j & (h - 1u);
            const uint32_t r0 = ((j >> lh) << (lh + 1)) + pos;
            const uint32_t i0 = (r0 << log_tc) + c;
            const uint32_t i1 = i0 + (h << log_tc);
            const uint32_t x = T[i0];
            const uint32_t y = T[i1];
            const uint32_t w = tw[pos << twshift];
            if (!INVERSE) {
                T[i0] = add_mod(x, y, p);
                T[i1] = mont_mul(sub_mod(x, y, p), w, p, pinv);
            } else {
                const uint32_t t = mont_mul(y, w, p, pinv);
                T[i0] = add_mod(x, t, p);
                T[i1] = sub_mod(x, t, p);
            }
        }
        __syncthreads();
    }
}

// Garner: (r0, r1, r2) residues -> 96-bit value (3 limbs).
struct CrtConsts {
    uint32_t p0_inv_mod_p1_m;   // (p0^-1 mod p1) in Montgomery form mod p1
    uint32_t p0_inv_mod_p2_m;
    uint32_t p1_inv_mod_p2_m;
    uint64_t p0p1;
};


// ---------------------------------------------------------------------------
// Register-resident radix-2^B stages (all shapes compile-time).
//
// A CTA of T threads owns a tile of TC = 2^LOG_TC interleaved transforms of
// R = 2^LOG_R points each, R * TC = 16 * T: element (position r, transform c)
// lives at tile index r * TC + c.  In a stage each thread holds 16 elements =
// 16 / 2^B groups of 2^B points; a group is {base + s*v : v < 2^B} with
// s = 2^LO, and the stage performs the B radix-2 levels with half-spans
// s*2^(B-1) .. s (forward, decimation in frequency) or s .. s*2^(B-1)
// (inverse, decimation in time).  The arithmetic is exactly that of
// tile_transform; only the grouping of levels changes, so results are
// identical.  Group id q = t + g*T; transform c = q mod TC; the remaining bits
// give (low, high) with base = high * s * 2^B + low.
//
// Forward stages cover the levels top-down in chunks of 4 (LOG_R = 12:
// [8..11], [4..7], [0..3]; 9: [5..8], [1..4], [0]); inverse stages walk the
// same chunks bottom-up, so the last forward and first inverse stage share a
// thread mapping.
// ---------------------------------------------------------------------------
template <int LOG_R, int K>
struct StageInfo {
    static constexpr int top = LOG_R - 4 * K;
    static constexpr int B = top >= 4 ? 4 : top;
    static constexpr int LO = top - B;
};

template <int LOG_R>
struct StagePlan {
    static constexpr int n = (LOG_R + 3) / 4;
};

template <int LOG_R, int LOG_TC, int LO, int B>
struct Stage {
    static constexpr uint32_t T = 1u << (LOG_R + LOG_TC - 4);
    __device__ static __forceinline__ void elem(uint32_t t, int j, uint32_t &pos, uint32_t &c) {
        const int g = j >> B;
        const uint32_t v = (uint32_t)j & ((1u << B) - 1u);
        const uint32_t q = t + (uint32_t)g * T;
        c = q & ((1u << LOG_TC) - 1u);
        const uint32_t rem = q >> LOG_TC;
        const uint32_t low = rem & ((1u << LO) - 1u);
        const uint32_t high = rem >> LO;
        pos = (high << (LO + B)) + low + (v << LO);
    }
    __device__ static __forceinline__ uint32_t addr(uint32_t pos, uint32_t c) {
        const uint32_t i = (pos << LOG_TC) + c;
        return i + (i >> 5);   // one pad word per 32 avoids bank conflicts
    }
    __device__ static __forceinline__ void store(uint32_t *S, const uint32_t (&x)[16], uint32_t t) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            uint32_t pos, c;
            elem(t, j, pos, c);
            S[addr(pos, c)] = x[j];
        }
    }
    __device__ static __forceinline__ void load(const uint32_t *S, uint32_t (&x)[16], uint32_t t) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            uint32_t pos, c;
            elem(t, j, pos, c);
            x[j] = S[addr(pos, c)];
        }
    }
    // tw[e] = w_R^(+/-e), e < R/2
    template <bool INV>
    __device__ static __forceinline__ void levels(uint32_t (&x)[16], uint32_t t, const uint32_t *tw, uint32_t p,
                                                  uint32_t pinv) {
#pragma unroll
        for (int step = 0; step < B; ++step) {
            const int lm = INV ? step : (B - 1 - step);
            const int mm = 1 << lm;
            const int lh = LO + lm;
            const int shift = LOG_R - 1 - lh;
            const uint32_t hmask = (1u << lh) - 1u;
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                if (j & mm) continue;   // partner j + mm stays inside the 2^B group
                uint32_t pos, c;
                elem(t, j, pos, c);
                const uint32_t w = tw[(pos & hmask) << shift];
                const uint32_t a = x[j];
                const uint32_t b = x[j + mm];
                if (!INV) {
                    x[j] = add_mod(a, b, p);
                    x[j + mm] = mont_mul(sub_mod(a, b, p), w, p, pinv);
                } else {
                    const uint32_t u = mont_mul(b, w, p, pinv);
                    x[j] = add_mod(a, u, p);
                    x[j + mm] = sub_mod(a, u, p);
                }
            }
        }
    }
};

// Stage number K of the execution order (forward: top-down, inverse: bottom-up).
template <int LOG_R, int LOG_TC, bool INV, int K>
struct ExecStage {
    static constexpr int idx = INV ? (StagePlan<LOG_R>::n - 1 - K) : K;
    using I = StageInfo<LOG_R, idx>;
    using S = Stage<LOG_R, LOG_TC, I::LO, I::B>;
};

// Runs execution stages K .. n-1 on x; S is the shared tile (stage hand-off).
template <int LOG_R, int LOG_TC, bool INV, int K>
__device__ __forceinline__ void run_stages(uint32_t (&x)[16], uint32_t *Sm, uint32_t t, const uint32_t *tw,
                                           uint32_t p, uint32_t pinv) {
    constexpr int n = StagePlan<LOG_R>::n;
    if constexpr (K < n) {
        using Cur = typename ExecStage<LOG_R, LOG_TC, INV, K>::S;
        if constexpr (K > 0) {
            using Prev = typename ExecStage<LOG_R, LOG_TC, INV, K - 1>::S;
            Prev::store(Sm, x, t);
            __syncthreads();
            Cur::load(Sm, x, t);
            __syncthreads();
        }
        Cur::template levels<INV>(x, t, tw, p, pinv);
        run_stages<LOG_R, LOG_TC, INV, K + 1>(x, Sm, t, tw, p, pinv);
    }
}

}  // namespace ntt
}  // namespace gpupi
