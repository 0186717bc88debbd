// Three-prime number-theoretic transform building blocks (sm_100a).
//
// An exact product of 32-bit-limb integers is a cyclic convolution computed
// modulo three primes below 2^31 and recombined by Garner's CRT:
//
//   p0 = 27 * 2^26 + 1 = 1811939329   (2-adicity 26, generator 13)
//   p1 = 15 * 2^27 + 1 = 2013265921   (2-adicity 27, generator 31)
//   p2 = 63 * 2^25 + 1 = 2113929217   (2-adicity 25, generator 5)
//
// p0 p1 p2 > 2^92.6 and a convolution coefficient is at most
// min(L_a, L_b) * (2^32 - 1)^2, so every product with min(L_a, L_b) < 2^28
// is recovered exactly.  Transforms have at most 2^25 points (p2's
// 2-adicity); longer products are split into cosets (mul_ntt.cu).
//
// Residues are kept in [0, p).  Since 2p < 2^32 a sum or difference needs
// one unsigned min to reduce (x - p wraps above x exactly when x < p), and a
// product by a table constant w uses Shoup's method with w' = floor(w 2^32/p):
// q = hi(x w'), r = x w - q p lies in [0, 2p) for every 32-bit x.  Products
// of two variables use Montgomery reduction with R = 2^32.
#pragma once

#include "common.cuh"

namespace gpupi {
namespace ntt {

constexpr int kPrimes = 3;
constexpr int kMaxLog = 25;          // largest transform: 2^25 points
constexpr int kLoBits = 13;          // root tables: w^e = LO[e mod 2^13] * HI[e >> 13]
constexpr uint32_t kLoSize = 1u << kLoBits;
constexpr uint32_t kHiSize = 1u << (kMaxLog - kLoBits);   // 4096
constexpr int kCosetLoBits = 14;     // coset tables: g^e for e < 2^28
constexpr uint32_t kCosetSize = 1u << kCosetLoBits;
constexpr int kMaxCosets = 20;   // products up to 20 * 2^25 limbs
static_assert((uint64_t)kMaxCosets << 25 <= 3ull << 28, "coset exponents below 3 * 2^28");

constexpr uint32_t inv_2_32(uint32_t p) {
    uint32_t x = p;   // Newton iteration for p^-1 mod 2^32
    for (int i = 0; i < 5; ++i) x *= 2u - p * x;
    return x;
}
constexpr uint32_t cmul(uint32_t a, uint32_t b, uint32_t p) { return (uint32_t)((uint64_t)a * b % p); }
constexpr uint32_t cpow(uint32_t a, uint64_t e, uint32_t p) {
    uint32_t r = 1u;
    while (e) {
        if (e & 1u) r = cmul(r, a, p);
        a = cmul(a, a, p);
        e >>= 1;
    }
    return r;
}
constexpr uint32_t cinv(uint32_t a, uint32_t p) { return cpow(a % p, p - 2u, p); }
constexpr uint32_t shoup_of(uint32_t w, uint32_t p) { return (uint32_t)(((uint64_t)w << 32) / p); }

template <int Q>
struct Prime;
template <>
struct Prime<0> {
    static constexpr uint32_t p = 1811939329u, g = 13u;
};
template <>
struct Prime<1> {
    static constexpr uint32_t p = 2013265921u, g = 31u;
};
template <>
struct Prime<2> {
    static constexpr uint32_t p = 2113929217u, g = 5u;
};
// b^e mod p (host and compile time)
constexpr uint32_t cpow(uint64_t b, uint64_t e, uint64_t p) {
    uint64_t r = 1u % p;
    b %= p;
    while (e) {
        if (e & 1u) r = r * b % p;
        b = b * b % p;
        e >>= 1;
    }
    return (uint32_t)r;
}

template <int Q>
struct PrimeC {
    static constexpr uint32_t p = Prime<Q>::p;
    static constexpr uint32_t pinv = inv_2_32(p);
    static constexpr uint32_t r1 = (uint32_t)((1ull << 32) % p);   // R mod p: Montgomery form of 1
    // Montgomery forms of g^(+-k 2^28), k = 1, 2: coset exponents reach 20 * 2^25
    static constexpr uint32_t g28 = (uint32_t)(((uint64_t)cpow(Prime<Q>::g, 1ull << 28, p) << 32) % p);
    static constexpr uint32_t g29 = (uint32_t)(((uint64_t)cpow(Prime<Q>::g, 1ull << 29, p) << 32) % p);
    static constexpr uint32_t g28inv =
        (uint32_t)(((uint64_t)cpow(Prime<Q>::g, (p - 1ull) - ((1ull << 28) % (p - 1ull)), p) << 32) % p);
    static constexpr uint32_t g29inv =
        (uint32_t)(((uint64_t)cpow(Prime<Q>::g, (p - 1ull) - ((1ull << 29) % (p - 1ull)), p) << 32) % p);
};
static_assert((uint64_t)cpow(13, 1ull << 28, 1811939329u) * cpow(13, 1811939328ull - (1ull << 28), 1811939329u) %
                      1811939329u == 1u, "g^(2^28) g^(-2^28) = 1");
static_assert(PrimeC<0>::p * PrimeC<0>::pinv == 1u, "p0 inverse");
static_assert(PrimeC<1>::p * PrimeC<1>::pinv == 1u, "p1 inverse");
static_assert(PrimeC<2>::p * PrimeC<2>::pinv == 1u, "p2 inverse");

// x in [0, 2p) -> [0, p)
template <int Q>
__device__ __forceinline__ uint32_t norm(uint32_t x) {
    return min(x, x - Prime<Q>::p);
}
template <int Q>
__device__ __forceinline__ uint32_t add_n(uint32_t a, uint32_t b) {
    return norm<Q>(a + b);
}
template <int Q>
__device__ __forceinline__ uint32_t sub_n(uint32_t a, uint32_t b) {
    return norm<Q>(a - b + Prime<Q>::p);
}
// x < 2^32 (< 3p) -> [0, p)
template <int Q>
__device__ __forceinline__ uint32_t reduce_limb(uint32_t x) {
    return norm<Q>(min(x, x - Prime<Q>::p));
}
// x * w mod p in [0, 2p), w < p with wq = floor(w 2^32 / p), any 32-bit x
template <int Q>
__device__ __forceinline__ uint32_t shoup(uint32_t x, uint32_t w, uint32_t wq) {
    const uint32_t q = __umulhi(x, wq);
    return x * w - q * Prime<Q>::p;
}
// a * b / 2^32 mod p in (0, 2p); requires a * b < 2^32 * p
template <int Q>
__device__ __forceinline__ uint32_t mont(uint32_t a, uint32_t b) {
    const uint64_t t = (uint64_t)a * b;
    const uint32_t m = (uint32_t)t * PrimeC<Q>::pinv;
    return (uint32_t)(t >> 32) - __umulhi(m, Prime<Q>::p) + Prime<Q>::p;
}

// Table layout inside NTTPrecomputedTables (raw u32 views of the uint3 buffers).
//   lv1: ROOT_LO[dir][q][2^13]  uint2 {w^e, shoup}        w = primitive 2^25-th root,
//        ROOT_HI[dir][q][2^12]  uint2 {w^(e 2^13), shoup}  dir 1 holds w^-1
//        LEVEL[dir][q][4095]    uint2 {w_(2h)^m, shoup} at (h - 1) + m for
//                               h = 2^lh, m < h, lh < 12: the twiddles of
//                               radix-2 level lh, contiguous per level
//   lv2: COSET_LO[dir][q][2^14] g^e, COSET_HI[dir][q][2^14] g^(e 2^14), Montgomery
//        form, dir 1 holds g^-1 (coset twists beta_i^j = g^(i j), i j < 20 2^25:
//        the bits above 2^28 through PrimeC::g28 / g29 and inverses)
//   inv2n: [k][q]  2^-k * R^2 mod p (scale of the pointwise product)
constexpr int kLevelLogMax = 12;
constexpr uint32_t kLevelSize = (1u << kLevelLogMax) - 1u;        // 4095
constexpr size_t kRootLoWords = 2u * kPrimes * kLoSize * 2u;     // 98304
constexpr size_t kRootHiWords = 2u * kPrimes * kHiSize * 2u;     // 49152
constexpr size_t kLevelOffset = kRootLoWords + kRootHiWords;     // 147456
constexpr size_t kLevelWords = 2u * kPrimes * kLevelSize * 2u;   // 49140
constexpr size_t kCosetWords = 2u * kPrimes * kCosetSize;        // per level: 98304
static_assert(kLevelOffset + kLevelWords <= 65536u * 3u, "lv1 capacity");
static_assert(2u * kCosetWords <= 65536u * 3u, "lv2 capacity");

struct Tables {
    const uint2 *root_lo;       // [dir][q][kLoSize]
    const uint2 *root_hi;       // [dir][q][kHiSize]
    const uint2 *level;         // [dir][q][kLevelSize]
    const uint32_t *coset_lo;   // [dir][q][kCosetSize]
    const uint32_t *coset_hi;   // [dir][q][kCosetSize]
    const uint32_t *inv2n;      // [33][q]
};

__device__ __forceinline__ const uint2 *root_lo_ptr(const Tables &t, int dir, int q) {
    return t.root_lo + ((size_t)dir * kPrimes + q) * kLoSize;
}
__device__ __forceinline__ const uint2 *root_hi_ptr(const Tables &t, int dir, int q) {
    return t.root_hi + ((size_t)dir * kPrimes + q) * kHiSize;
}
__device__ __forceinline__ const uint2 *level_ptr(const Tables &t, int dir, int q) {
    return t.level + ((size_t)dir * kPrimes + q) * kLevelSize;
}
__device__ __forceinline__ const uint32_t *coset_lo_ptr(const Tables &t, int dir, int q) {
    return t.coset_lo + ((size_t)dir * kPrimes + q) * kCosetSize;
}
__device__ __forceinline__ const uint32_t *coset_hi_ptr(const Tables &t, int dir, int q) {
    return t.coset_hi + ((size_t)dir * kPrimes + q) * kCosetSize;
}

// x * w^E for E < 2^25 (w the root table's root), result in [0, p)
template <int Q>
__device__ __forceinline__ uint32_t mul_root(uint32_t x, const uint2 *lo, const uint2 *hi, uint32_t E) {
    const uint2 a = __ldg(lo + (E & (kLoSize - 1u)));
    const uint2 b = __ldg(hi + (E >> kLoBits));
    return norm<Q>(shoup<Q>(shoup<Q>(x, a.x, a.y), b.x, b.y));
}
// R * w^E (Montgomery form of w^E) for E < 2^25, result in [0, p)
template <int Q>
__device__ __forceinline__ uint32_t root_m(const uint2 *lo, const uint2 *hi, uint32_t E) {
    return mul_root<Q>(PrimeC<Q>::r1, lo, hi, E);
}
// x * g^E (DIR 0) or x * g^-E (DIR 1, lo / hi the dir-1 tables) for
// E < 3 * 2^28, result in [0, p); the tables cover E < 2^28, the top bits
// are one more product.
template <int Q, int DIR>
__device__ __forceinline__ uint32_t mul_coset(uint32_t x, const uint32_t *lo, const uint32_t *hi, uint32_t E) {
    const uint32_t top = E >> 28;
    if (top) {
        const uint32_t f = DIR ? (top == 1u ? PrimeC<Q>::g28inv : PrimeC<Q>::g29inv)
                               : (top == 1u ? PrimeC<Q>::g28 : PrimeC<Q>::g29);
        x = norm<Q>(mont<Q>(x, f));
        E &= (1u << 28) - 1u;
    }
    const uint32_t a = __ldg(lo + (E & (kCosetSize - 1u)));
    const uint32_t b = __ldg(hi + (E >> kCosetLoBits));
    return norm<Q>(mont<Q>(mont<Q>(x, a), b));
}

__device__ __forceinline__ uint32_t bitrev(uint32_t x, int bits) {
    return bits ? (__brev(x) >> (32 - bits)) : 0u;
}
__host__ __device__ constexpr uint32_t crev(uint32_t x, int bits) {
    uint32_t r = 0u;
    for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
}

// In-place radix-2 transform of every column of a shared-memory tile
// T[R][TC] (row-major, R = 2^log_r points per column, TC = 2^log_tc columns);
// used for transforms too small for the register-stage kernels.
// Forward: decimation in frequency, natural order in, bit-reversed order out.
// Inverse: decimation in time, bit-reversed in, natural out (unscaled).
// tw[e] = (w_R)^(+-e) for e < R/2 with its Shoup companion (the LEVEL table
// of level log_r - 1).
template <int Q, bool INVERSE>
__device__ __forceinline__ void tile_transform(uint32_t *T, int log_r, int log_tc, const uint2 *tw) {
    constexpr uint32_t P = Prime<Q>::p;
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
            const uint2 w = tw[pos << twshift];
            if (!INVERSE) {
                T[i0] = add_n<Q>(x, y);
                T[i1] = norm<Q>(shoup<Q>(x - y + P, w.x, w.y));
            } else {
                const uint32_t t = norm<Q>(shoup<Q>(y, w.x, w.y));
                T[i0] = add_n<Q>(x, t);
                T[i1] = sub_n<Q>(x, t);
            }
        }
        __syncthreads();
    }
}

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
    static constexpr int kB = B, kLO = LO;
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
    // tw = the LEVEL table (levels 0 .. LOG_R - 1).
    // In a level of half-span h = s*2^lm the butterfly of group element v uses
    // w_(2h)^(low + s*(v mod 2^lm)): only 2^lm distinct twiddles per group,
    // loaded once each from the contiguous table of that level, so the lanes
    // of a warp read consecutive entries or one broadcast entry.  The
    // half-span-1 level (LO = 0, lm = 0) has twiddle 1 and needs no product.
    template <bool INV, int Q>
    __device__ static __forceinline__ void bfly(uint32_t (&x)[16], int j, int mm, uint2 w, bool trivial) {
        constexpr uint32_t P = Prime<Q>::p;
        const uint32_t a = x[j];
        const uint32_t b = x[j + mm];
        if (!INV) {
            x[j] = add_n<Q>(a, b);
            x[j + mm] = trivial ? sub_n<Q>(a, b) : norm<Q>(shoup<Q>(a - b + P, w.x, w.y));
        } else {
            const uint32_t y = trivial ? b : norm<Q>(shoup<Q>(b, w.x, w.y));
            x[j] = add_n<Q>(a, y);
            x[j + mm] = sub_n<Q>(a, y);
        }
    }
    template <bool INV, int Q>
    __device__ static __forceinline__ void levels(uint32_t (&x)[16], uint32_t t, const uint2 *tw) {
        levels_pair<INV, Q, false>(x, x, t, tw);
    }
    // Two independent transforms of the same shape (PAIR): every twiddle is
    // loaded once and serves both.
    template <bool INV, int Q, bool PAIR>
    __device__ static __forceinline__ void levels_pair(uint32_t (&x)[16], uint32_t (&y)[16], uint32_t t,
                                                       const uint2 *tw) {
        constexpr int G = 16 >> B;
#pragma unroll
        for (int step = 0; step < B; ++step) {
            const int lm = INV ? step : (B - 1 - step);
            const int mm = 1 << lm;
            const int lh = LO + lm;
            const uint32_t lbase = (1u << lh) - 1u;
            const bool trivial = (lh == 0);
#pragma unroll
            for (int g = 0; g < G; ++g) {
                uint32_t pos0, c0;
                elem(t, g << B, pos0, c0);                  // v = 0 of this group
                const uint32_t low = pos0 & ((1u << LO) - 1u);
#pragma unroll
                for (int u = 0; u < mm; ++u) {
                    const uint2 w = trivial ? make_uint2(1u, 0u) : tw[lbase + low + ((uint32_t)u << LO)];
#pragma unroll
                    for (int v = u; v < (1 << B); v += 2 * mm) {
                        bfly<INV, Q>(x, (g << B) + v, mm, w, trivial);
                        if (PAIR) bfly<INV, Q>(y, (g << B) + v, mm, w, trivial);
                    }
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

// Runs execution stages K .. n-1 on x (and, with PAIR, in lockstep on y);
// Sx / Sy are the shared tiles of the stage hand-offs.
template <int LOG_R, int LOG_TC, bool INV, int Q, int K, bool PAIR>
__device__ __forceinline__ void run_stages_pair(uint32_t (&x)[16], uint32_t (&y)[16], uint32_t *Sx, uint32_t *Sy,
                                                uint32_t t, const uint2 *tw) {
    constexpr int n = StagePlan<LOG_R>::n;
    if constexpr (K < n) {
        using Cur = typename ExecStage<LOG_R, LOG_TC, INV, K>::S;
        if constexpr (K > 0) {
            using Prev = typename ExecStage<LOG_R, LOG_TC, INV, K - 1>::S;
            Prev::store(Sx, x, t);
            if (PAIR) Prev::store(Sy, y, t);
            __syncthreads();
            Cur::load(Sx, x, t);
            if (PAIR) Cur::load(Sy, y, t);
            __syncthreads();
        }
        Cur::template levels_pair<INV, Q, PAIR>(x, y, t, tw);
        run_stages_pair<LOG_R, LOG_TC, INV, Q, K + 1, PAIR>(x, y, Sx, Sy, t, tw);
    }
}

template <int LOG_R, int LOG_TC, bool INV, int Q, int K>
__device__ __forceinline__ void run_stages(uint32_t (&x)[16], uint32_t *Sm, uint32_t t, const uint2 *tw) {
    run_stages_pair<LOG_R, LOG_TC, INV, Q, K, false>(x, x, Sm, Sm, t, tw);
}

}  // namespace ntt
}  // namespace gpupi
