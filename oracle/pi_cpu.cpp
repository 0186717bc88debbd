// Host C++17 restatement of gpupi's pi_bs_gpu pipeline with GMP integers,
// multi-threaded (std::thread) over the rows of every batched step.
//
// TEST INFRASTRUCTURE and CPU BASELINE only: it follows oracle/pi_ref.py step
// for step (the same compact()-derived lengths, truncations, modular widths
// and sign probe of the recursive inverse, the same truncating equal-split
// conversion), so its RET and digits equal the GPU pipeline's bit for bit.
// Nothing in the product links it.  References are file:line in gpupi.
//
//   pi_cpu <digits> [threads]
// prints the lines of `pi_bs_gpu <digits> --benchmark` (elapsed_ms is host
// wall time of the whole pipeline) plus the thread count.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <string>
#include <thread>
#include <vector>

#include "gmp.h"

namespace {

struct Z {
    mpz_t v;
    Z() { mpz_init(v); }
    explicit Z(unsigned long x) { mpz_init(v); mpz_set_ui(v, x); }
    Z(const Z &o) { mpz_init(v); mpz_set(v, o.v); }
    Z(Z &&o) noexcept { mpz_init(v); mpz_swap(v, o.v); }
    Z &operator=(Z &&o) noexcept { mpz_swap(v, o.v); return *this; }
    Z &operator=(const Z &o) { mpz_set(v, o.v); return *this; }
    ~Z() { mpz_clear(v); }
};

unsigned g_threads = 1;

// Runs f(i) for i < n on g_threads threads (dynamic assignment).
void parallel_for(size_t n, const std::function<void(size_t)> &f) {
    const unsigned T = (unsigned)std::min<size_t>(g_threads, n);
    if (T <= 1) {
        for (size_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < T; ++t)
        pool.emplace_back([&] {
            for (size_t i; (i = next.fetch_add(1)) < n;) f(i);
        });
    for (auto &th : pool) th.join();
}

uint32_t nlimbs(const mpz_t x) {   // compact() limb count (0 for 0)
    if (mpz_sgn(x) == 0) return 0;
    return (uint32_t)((mpz_sizeinbase(x, 2) + 31) / 32);
}
size_t nbits(const mpz_t x) { return mpz_sgn(x) == 0 ? 0 : mpz_sizeinbase(x, 2); }
void mod_limbs(mpz_t r, const mpz_t x, uint64_t len) { mpz_fdiv_r_2exp(r, x, 32 * len); }
void shr(mpz_t r, const mpz_t x, uint64_t bits) { mpz_fdiv_q_2exp(r, x, bits); }
void shl(mpz_t r, const mpz_t x, uint64_t bits) { mpz_mul_2exp(r, x, bits); }

// ---------------------------------------------------------------------------
// Leaves (pi_bs_gpu.cu:17-131)
// ---------------------------------------------------------------------------
void reduce_pair(uint64_t &a, uint64_t &b) {   // pi_bs_gpu.cu:17-34
    for (uint64_t d : {3ull, 5ull, 23ull, 29ull})
        if (a % d == 0 && b % d == 0) {
            a /= d;
            b /= d;
        }
}

void leaf_term(uint64_t i, Z &P, Z &Q, Z &R) {   // construct_leaf_17 body, :48-95
    uint64_t p1 = 6 * i + 1, p2 = 2 * i + 1, p3 = 6 * i + 5;
    uint64_t q1 = i + 1, q2 = i + 1, q3 = i + 1;
    uint64_t q4 = 640320 >> 6, q5 = 40020 >> 2, q6 = 426880 >> 7;
    const uint64_t r1 = 545140134ull * i + 13591409ull;
    for (uint64_t *q : {&q1, &q2, &q3})
        if (p1 % 5 == 0 && *q % 5 == 0) {
            p1 /= 5;
            *q /= 5;
        }
    reduce_pair(p1, q4);
    reduce_pair(p1, q5);
    reduce_pair(p2, q4);
    reduce_pair(p2, q5);
    reduce_pair(p3, q4);
    reduce_pair(p3, q5);
    mpz_set_ui(P.v, p1);
    mpz_mul_ui(P.v, P.v, p2);
    mpz_mul_ui(P.v, P.v, p3);
    mpz_set_ui(Q.v, q1);
    for (uint64_t f : {q2, q3, q4, q5, q6}) mpz_mul_ui(Q.v, Q.v, f);
    mpz_set_ui(R.v, r1);
    for (uint64_t f : {q1, q2, q3, q4, q5}) mpz_mul_ui(R.v, R.v, f);
}

uint64_t leaf_index(uint64_t i2, bool head) { return head ? i2 * 17 + 16 : i2 + (i2 >> 4); }   // :40-45

// ---------------------------------------------------------------------------
// Binary splitting (pi_bs_gpu.cu:504-792)
// ---------------------------------------------------------------------------
void binary_split(uint64_t N, Z &Qout, Z &Rout) {
    const uint64_t n = 16 * N;
    std::vector<Z> P0(N), Q0(N), R0(N), P(n), Q(n), R(n);
    parallel_for(N, [&](size_t j) { leaf_term(leaf_index(j, true), P0[j], Q0[j], R0[j]); });
    parallel_for(n, [&](size_t j) { leaf_term(leaf_index(j, false), P[j], Q[j], R[j]); });
    for (uint64_t n1 = n; n1 > 1; n1 >>= 1) {
        const bool subtract = (n1 == n || n1 == (n >> 4));
        const uint64_t ignore_last_p = (n1 <= N) ? 1 : 0;
        const uint64_t half = n1 / 2;
        const uint64_t shift = 15 * ((n / n1) + ((n / n1) >> 4));
        std::vector<Z> nP(half - ignore_last_p), nQ(half), nR(half), nRB(half);
        // four independent products per output row: P, Q, R_e Q_o, P_e R_o
        parallel_for(4 * half, [&](size_t t) {
            const size_t k = t >> 2;
            switch (t & 3) {
                case 0:
                    if (k < half - ignore_last_p) mpz_mul(nP[k].v, P[2 * k].v, P[2 * k + 1].v);
                    break;
                case 1: mpz_mul(nQ[k].v, Q[2 * k].v, Q[2 * k + 1].v); break;
                case 2:
                    mpz_mul(nR[k].v, R[2 * k].v, Q[2 * k + 1].v);
                    shl(nR[k].v, nR[k].v, shift);
                    break;
                default: mpz_mul(nRB[k].v, P[2 * k].v, R[2 * k + 1].v); break;
            }
        });
        parallel_for(half, [&](size_t k) {
            if (subtract)
                mpz_sub(nR[k].v, nR[k].v, nRB[k].v);
            else
                mpz_add(nR[k].v, nR[k].v, nRB[k].v);
            if (mpz_sgn(nR[k].v) < 0) {
                fprintf(stderr, "pi_cpu: shift_sub result would wrap\n");
                std::abort();
            }
        });
        P = std::move(nP);
        Q = std::move(nQ);
        R = std::move(nR);
        if (n1 == (n >> 3)) {   // head merge, pi_bs_gpu.cu:725-784
            std::vector<Z> mP(half), mQ(half), mR(half), mRB(half);
            parallel_for(4 * half, [&](size_t t) {
                const size_t k = t >> 2;
                switch (t & 3) {
                    case 0: mpz_mul(mP[k].v, P[k].v, P0[k].v); break;
                    case 1: mpz_mul(mQ[k].v, Q[k].v, Q0[k].v); break;
                    case 2:
                        mpz_mul(mR[k].v, R[k].v, Q0[k].v);
                        shl(mR[k].v, mR[k].v, 15);
                        break;
                    default: mpz_mul(mRB[k].v, P[k].v, R0[k].v); break;
                }
            });
            parallel_for(3 * half, [&](size_t t) {
                const size_t k = t / 3;
                Z &z = (t % 3 == 0) ? mP[k] : ((t % 3 == 1) ? mQ[k] : mR[k]);
                if (t % 3 == 2) mpz_add(z.v, z.v, mRB[k].v);
                mpz_divexact_ui(z.v, z.v, 830297ul);      // BLOCK_DIV_LO, :147
                mpz_divexact_ui(z.v, z.v, 156590819ul);   // BLOCK_DIV_HI, :148
            });
            P = std::move(mP);
            Q = std::move(mQ);
            R = std::move(mR);
        }
    }
    Qout = std::move(Q[0]);
    Rout = std::move(R[0]);
}

// sqrt(10005) Pell iteration (pi_bs_gpu.cu:1346-1522)
void sqrt_10005(uint64_t target_digits, Z &p, Z &q) {
    mpz_set_ui(p.v, 4001);
    mpz_set_ui(q.v, 40);
    double valid = 7.5;
    while (valid < (double)target_digits) {
        valid *= 2;
        Z pp, qq, pq;
        std::thread a([&] { mpz_mul(pp.v, p.v, p.v); });
        std::thread b([&] {
            mpz_mul(qq.v, q.v, q.v);
            mpz_mul_ui(qq.v, qq.v, 10005);
        });
        mpz_mul(pq.v, p.v, q.v);
        a.join();
        b.join();
        mpz_add(p.v, pp.v, qq.v);
        shl(q.v, pq.v, 1);
    }
}

// ---------------------------------------------------------------------------
// Recursive inverse (pi_bs_gpu.cu:1145-1344)
// ---------------------------------------------------------------------------
std::vector<uint64_t> inverse_levels(uint64_t L) {   // :1187-1192
    std::vector<uint64_t> lv{L};
    while (lv.back() > 32 * 1024) {
        const uint64_t m = ((lv.back() - 2) / 4) & ~31ull;
        lv.push_back(lv.back() - 2 * m);
    }
    return lv;
}

void recursive_inverse(const mpz_t x, uint64_t x_len, uint64_t L, Z &y) {
    const std::vector<uint64_t> levels = inverse_levels(L);
    const uint64_t y_len = x_len;
    const uint64_t L0 = levels.back();
    const uint64_t start = (L - L0) >> 6;
    Z x0, num, res, t, v, res2, y2, xn, y2x;
    shr(x0.v, x, 32 * start);
    mpz_set_ui(num.v, 1);
    shl(num.v, num.v, L0);
    mpz_fdiv_qr(y.v, res.v, num.v, x0.v);   // GMP base case, :1237-1253
    uint64_t res_len = nlimbs(res.v);
    for (size_t i = levels.size() - 1; i > 0; --i) {
        const uint64_t L1 = levels[i], L2 = levels[i - 1];
        const uint64_t m = (L2 - L1) >> 1;
        const uint64_t off2 = (L - L2) >> 6, off1 = (L - L1) >> 6;
        const uint64_t x2_len = std::min<uint64_t>(m >> 5, x_len - off2);
        Z x2, x2y1;
        shr(x2.v, x, 32 * off2);
        mod_limbs(x2.v, x2.v, x2_len);
        const uint64_t y1_len = y_len - off1;
        mpz_mul(x2y1.v, x2.v, y.v);
        const uint64_t r1m_len = res_len + (m >> 5) + 1;
        shl(t.v, res.v, m);
        mpz_sub(t.v, t.v, x2y1.v);
        mod_limbs(v.v, t.v, r1m_len);
        Z top;
        shr(top.v, v.v, 32 * (r1m_len - 1));
        const bool neg = mpz_cmp_ui(top.v, 0x80000000ul) >= 0;
        if (neg) {
            mpz_neg(t.v, v.v);
            mod_limbs(v.v, t.v, r1m_len);
        }
        mpz_mul(res2.v, v.v, y.v);
        const uint64_t res2_len = r1m_len + y1_len;
        const uint64_t sh = L2 - 2 * m;
        const uint64_t y2_len = res2_len - (sh >> 5);
        shr(y2.v, res2.v, sh);
        mod_limbs(y2.v, y2.v, y2_len);
        if (neg) {
            mpz_add_ui(y2.v, y2.v, 1);
            mod_limbs(y2.v, y2.v, y2_len);
        }
        const uint64_t ynew_len = y_len - off2;
        shl(t.v, y.v, m);
        if (neg)
            mpz_sub(t.v, t.v, y2.v);
        else
            mpz_add(t.v, t.v, y2.v);
        mod_limbs(y.v, t.v, ynew_len);
        if (L2 != L) {
            shr(xn.v, x, 32 * off2);
            const uint64_t res_full_len = r1m_len + (m >> 5);
            Z resv;
            shl(resv.v, v.v, m);
            mpz_mul(y2x.v, y2.v, xn.v);
            if (neg)
                mpz_sub(t.v, y2x.v, resv.v);
            else
                mpz_sub(t.v, resv.v, y2x.v);
            mod_limbs(res.v, t.v, res_full_len);
            res_len = nlimbs(res.v);
        }
    }
}

// pi_fractional (pi_bs_gpu.cu:1524-1685)
uint64_t series_blocks(uint64_t d) {
    uint64_t N = 1;
    while ((double)N * 17 * 14.3 < (double)d) N *= 2;
    return N;
}
uint64_t prec_limbs_for(uint64_t d) { return ((uint64_t)(d * 3.322) + 31) / 32 + 1; }

void pi_fractional(uint64_t target, Z &ret) {
    const uint64_t N = series_blocks(target);
    const uint64_t prec = prec_limbs_for(target);
    Z Q, R, Rs, Qt, Rt, P15, Q15, Pf, Qf, Pt, Qtt, inv;
    binary_split(N, Q, R);
    shr(Rs.v, R.v, 15 * N * 17 - 8);
    uint64_t extra = std::max<int64_t>(0, (int64_t)std::min(nlimbs(Q.v), nlimbs(Rs.v)) - (int64_t)prec);
    shr(Qt.v, Q.v, 32 * extra);
    shr(Rt.v, Rs.v, 32 * extra);
    sqrt_10005(target, P15, Q15);
    std::thread a([&] { mpz_mul(Pf.v, P15.v, Qt.v); });
    mpz_mul(Qf.v, Rt.v, Q15.v);
    a.join();
    extra = std::max<int64_t>(0, (int64_t)std::min(nlimbs(Pf.v), nlimbs(Qf.v)) - (int64_t)prec);
    shr(Pt.v, Pf.v, 32 * extra);
    shr(Qtt.v, Qf.v, 32 * extra);
    const uint64_t L = 2 * nbits(Qtt.v) - 1;
    recursive_inverse(Qtt.v, nlimbs(Qtt.v), L, inv);
    mpz_mul(ret.v, Pt.v, inv.v);
    shr(ret.v, ret.v, L - 32 * prec);
}

// ---------------------------------------------------------------------------
// Decimal conversion (convert_decimal.cu:285-474, batch_decimal_naive.cu)
// ---------------------------------------------------------------------------
void round_up_decimal_digits(uint64_t requested, uint64_t &leaf, uint64_t &conv) {   // :924-939
    if (requested == 0) {
        leaf = conv = 0;
        return;
    }
    uint64_t digits = requested, levels = 0;
    while (digits >= 32 * 18) {
        digits >>= 1;
        ++levels;
    }
    if ((digits << levels) < requested) ++digits;
    leaf = digits;
    conv = digits << levels;
}

uint64_t bits_for_digits(uint64_t d) {   // convert_decimal.cu:36-39
    return (uint64_t)std::ceil((double)d * 3.32192809488736234787) + 34;
}

std::string convert_decimal(const mpz_t value, uint64_t value_len, uint64_t input_bits, uint64_t total,
                            uint64_t leaf) {
    uint64_t ratio = total / leaf, levels = 0;
    while ((2ull << levels) <= ratio) ++levels;
    std::vector<uint64_t> bits(levels + 1), digs(levels + 1), limbs(levels + 1);
    bits[0] = input_bits;
    digs[0] = total;
    limbs[0] = value_len;
    for (uint64_t lv = 1; lv <= levels; ++lv) {
        digs[lv] = digs[lv - 1] >> 1;
        bits[lv] = bits_for_digits(digs[lv]);
        limbs[lv] = (bits[lv] + 31) / 32;
    }
    std::vector<Z> cur(1);
    uint64_t cur_len, leaf_bits;
    if (levels == 0) {
        const uint64_t need = bits_for_digits(total);
        const uint64_t nl = (need + 31) / 32;
        shr(cur[0].v, value, input_bits - need);
        mod_limbs(cur[0].v, cur[0].v, nl);
        cur_len = nl;
        leaf_bits = need;
    } else {
        mpz_set(cur[0].v, value);
        cur_len = value_len;
        for (uint64_t lv = 0; lv < levels; ++lv) {
            const uint64_t d = digs[lv + 1], cb = bits[lv + 1], nl = limbs[lv + 1], B = bits[lv];
            const uint64_t mant_bits = B - d;
            Z power;
            mpz_ui_pow_ui(power.v, 5, d);
            std::vector<Z> nxt(2 * cur.size());
            parallel_for(cur.size(), [&](size_t k) {
                Z x, mant;
                mod_limbs(x.v, cur[k].v, cur_len);
                shr(nxt[2 * k].v, x.v, B - cb);
                mod_limbs(nxt[2 * k].v, nxt[2 * k].v, nl);
                mpz_fdiv_r_2exp(mant.v, x.v, mant_bits);
                mpz_mul(mant.v, mant.v, power.v);
                shr(nxt[2 * k + 1].v, mant.v, mant_bits - cb);
                mod_limbs(nxt[2 * k + 1].v, nxt[2 * k + 1].v, nl);
            });
            cur = std::move(nxt);
            cur_len = nl;
        }
        leaf_bits = bits[levels];
    }
    const uint64_t align = cur_len * 32 - leaf_bits;
    std::string out(cur.size() * leaf, '0');
    parallel_for(cur.size(), [&](size_t k) {
        Z x, ten;
        shl(x.v, cur[k].v, align);
        mod_limbs(x.v, x.v, cur_len);
        mpz_ui_pow_ui(ten.v, 10, leaf);
        mpz_mul(x.v, x.v, ten.v);
        shr(x.v, x.v, 32 * cur_len);   // truncated digits, batch_decimal_naive.cu:16-176
        char *s = mpz_get_str(nullptr, 10, x.v);
        const size_t len = strlen(s);
        const size_t take = std::min<size_t>(len, leaf);
        memcpy(&out[k * leaf + (leaf - take)], s + (len - take), take);
        free(s);
    });
    return out;
}

// Output helpers (pi_bs_gpu.cu:852-896)
std::vector<uint32_t> limbs_of(const mpz_t x) {
    std::vector<uint32_t> v(nlimbs(x));
    size_t cnt = 0;
    if (!v.empty()) mpz_export(v.data(), &cnt, -1, 4, 0, 0, x);
    return v;
}
uint32_t mod_hash(const std::vector<uint32_t> &l) {
    const uint64_t M = 1000000007ull, base = (1ull << 32) % M;
    uint64_t v = 0;
    for (size_t i = l.size(); i-- > 0;) v = (v * base + l[i]) % M;
    return (uint32_t)v;
}
void print_preview(const std::vector<uint32_t> &l) {
    printf("RET = ");
    const size_t n = l.size();
    for (size_t i = 0; i < std::min<size_t>(n, 2); ++i) printf(i == 0 ? "%x" : "%08x", l[n - 1 - i]);
    if (n > 4) printf("...");
    for (size_t i = std::min<size_t>(n, 2); i > 0; --i) {
        const size_t idx = i - 1;
        if (n <= 4 && idx >= n - std::min<size_t>(n, 2)) continue;
        printf("%08x", l[idx]);
    }
    printf(" hash = %u\n", mod_hash(l));
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2) {
        fprintf(stderr, "usage: %s <digits> [threads]\n", argv[0]);
        return 1;
    }
    const uint64_t digits = strtoull(argv[1], nullptr, 10);
    g_threads = argc > 2 ? (unsigned)atoi(argv[2]) : std::max(1u, std::thread::hardware_concurrency());
    const auto t0 = std::chrono::steady_clock::now();
    Z ret;
    pi_fractional(digits, ret);
    uint64_t leaf = 0, conv = 0;
    round_up_decimal_digits(digits, leaf, conv);
    const uint64_t prec = prec_limbs_for(digits);
    std::string dec;
    if (digits > 0) {
        Z frac;
        const uint64_t frac_len = std::min<uint64_t>(prec, nlimbs(ret.v));
        mod_limbs(frac.v, ret.v, frac_len);
        dec = convert_decimal(frac.v, frac_len, prec * 32, conv, leaf);
    }
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    const std::vector<uint32_t> l = limbs_of(ret.v);
    printf("target_digits=%llu convert_digits=%llu RET_len=%zu elapsed_ms=%.3f threads=%u\n",
           (unsigned long long)digits, (unsigned long long)conv, l.size(), ms, g_threads);
    print_preview(l);
    const size_t head = std::min<size_t>(63, digits), tail = std::min<size_t>(64, digits);
    if (digits > 0) printf("DEC = 3%s...%s\n", dec.substr(0, head).c_str(), dec.substr(digits - tail, tail).c_str());
    // compute_decimal_hash (pi_bs_gpu.cu:860-866) over "3" and every requested digit
    uint64_t h = 3;
    for (uint64_t i = 0; i < digits; ++i) h = (h * 10 + (uint64_t)(dec[i] - '0')) % 1000000007ull;
    printf("DEC_hash = %llu\n", (unsigned long long)h);
    return 0;
}
