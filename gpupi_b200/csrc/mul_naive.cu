// Batched schoolbook multiplication (gpupi batch_mul_naive.cu:8-273).
//
// Two shapes:
//   * k_school_thread<MA, MB>: one thread per product for operands of at most
//     MA x MB limbs (the bottom levels of the splitting tree: 3..16-limb rows
//     in batches of millions).  Register arrays, fully unrolled MACs.
//   * k_school_seg<G>: G = 8, 16 or 32 lanes per product for
//     L_a + L_b <= 4 G (up to 128), carries resolved with one ballot pair.
//   * k_school_cols: one CTA per product, 64-256 threads x 4 consecutive output
//     columns.  Each column sum sum_i a_i b_(k-i) is accumulated exactly in a
//     3-word register with mad.lo.cc / madc.hi.cc / addc (3 instructions per
//     32x32 product), then the 96-bit column sums are carried into limbs with
//     the same chunk/ballot carry as the NTT's CRT stage.  L_a + L_b <= 1024.
// Both are IMAD-bound; algorithmic work = L_a * L_b 32x32->64 products.
#include "common.cuh"
#include "carry_tile.cuh"
#include "batch_mul_naive.h"

namespace gpupi {

template <int MA, int MB>
__global__ void __launch_bounds__(128) k_school_thread(const uint32_t *__restrict__ A,
                                                       const uint32_t *__restrict__ B,
                                                       uint32_t *__restrict__ C, uint32_t N,
                                                       uint32_t La, uint32_t Lb, uint64_t sA,
                                                       uint64_t sB, uint64_t sC) {
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < N;
         row += gridDim.x * blockDim.x) {
        uint32_t a[MA], b[MB], o[MA + MB];
        const uint32_t *ar = A + row * sA;
        const uint32_t *br = B + row * sB;
#pragma unroll
        for (int i = 0; i < MA; ++i) a[i] = (i < (int)La) ? ar[i] : 0u;
#pragma unroll
        for (int j = 0; j < MB; ++j) b[j] = (j < (int)Lb) ? br[j] : 0u;
#pragma unroll
        for (int k = 0; k < MA + MB; ++k) o[k] = 0u;
#pragma unroll
        for (int i = 0; i < MA; ++i) {
            uint32_t carry = 0u;
#pragma unroll
            for (int j = 0; j < MB; ++j) {
                const uint64_t t = (uint64_t)a[i] * b[j] + o[i + j] + carry;
                o[i + j] = (uint32_t)t;
                carry = (uint32_t)(t >> 32);
            }
            o[i + MB] = carry;
        }
        uint32_t *cr = C + row * sC;
        const uint32_t Lc = La + Lb;
#pragma unroll
        for (int k = 0; k < MA + MB; ++k)
            if (k < (int)Lc) cr[k] = o[k];
    }
}

__device__ __forceinline__ void mac3(uint32_t &c0, uint32_t &c1, uint32_t &c2, uint32_t a, uint32_t b) {
    asm("mad.lo.cc.u32 %0, %3, %4, %0;\n\t"
        "madc.hi.cc.u32 %1, %3, %4, %1;\n\t"
        "addc.u32 %2, %2, 0;"
        : "+r"(c0), "+r"(c1), "+r"(c2)
        : "r"(a), "r"(b));
}

constexpr int kSchoolV = 4;
constexpr int kSchoolMaxL = 256 * kSchoolV;   // 1024 output limbs

// G lanes per product (G = 8, 16, 32; L_a + L_b <= 4 G): lane l of a group
// owns output columns 4l .. 4l+3, carries between the group's lanes are
// resolved with one ballot pair.  32 / G products per warp, so short
// products (the lower levels of the splitting tree) keep most lanes busy.
constexpr int kSegWarps = 8;   // warps per CTA

template <int G>
__global__ void __launch_bounds__(32 * kSegWarps) k_school_seg(const uint32_t *__restrict__ A,
                                                               const uint32_t *__restrict__ B,
                                                               uint32_t *__restrict__ C, uint32_t N,
                                                               uint32_t La, uint32_t Lb, uint64_t sA,
                                                               uint64_t sB, uint64_t sC) {
    constexpr int PW = 32 / G;                    // products per warp
    constexpr int NP = kSegWarps * PW;            // products per CTA
    // row pitches: 4G + 1 words for A (the groups' broadcast reads of a_i hit
    // different banks), 4G + 13 for B (the groups' windows start in
    // different banks modulo 4)
    __shared__ uint32_t sa[NP][4 * G + 1];
    __shared__ uint32_t sb[NP][4 * G + 13];
    const uint32_t lane = lane_id();
    const uint32_t w = threadIdx.x >> 5;
    const uint32_t grp = lane / G, gl = lane % G;   // group in the warp, lane in the group
    const uint32_t slot = w * PW + grp;
    const uint32_t kPad = La + 4;
    const uint32_t Lc = La + Lb;
    const uint32_t gmask = (G == 32) ? 0xffffffffu : ((1u << G) - 1u);
    // the whole warp runs every iteration (ballots), rows past N compute zeros
    for (uint64_t base = ((uint64_t)blockIdx.x * kSegWarps + w) * PW; base < N;
         base += (uint64_t)gridDim.x * NP) {
        const uint64_t row = base + grp;
        const bool valid = row < N;
        const uint32_t *ar = A + row * sA;
        const uint32_t *br = B + row * sB;
        for (uint32_t i = gl; i < La; i += G) sa[slot][i] = valid ? ar[i] : 0u;
        for (uint32_t j = gl; j < kPad + Lb + 8; j += G)
            sb[slot][j] = (valid && j >= kPad && j - kPad < Lb) ? br[j - kPad] : 0u;
        __syncwarp();
        const uint32_t k0 = gl * kSchoolV;
        uint32_t c[kSchoolV][3];
#pragma unroll
        for (int v = 0; v < kSchoolV; ++v) c[v][0] = c[v][1] = c[v][2] = 0u;
        if (k0 < Lc) {
            const int ilo = max(0, (int)k0 + 1 - (int)Lb);
            const int ihi = min((int)La - 1, (int)k0 + kSchoolV - 1);
            // window bw[v] = b_(k0 + v - i), slid down one word per step of i:
            // one shared-memory load per four products
            const uint32_t *bcol = &sb[slot][kPad + k0];
            uint32_t bw[kSchoolV];
#pragma unroll
            for (int v = 0; v < kSchoolV; ++v) bw[v] = bcol[v - ilo];
            for (int i = ilo; i <= ihi; ++i) {
                const uint32_t ai = sa[slot][i];
#pragma unroll
                for (int v = 0; v < kSchoolV; ++v) mac3(c[v][0], c[v][1], c[v][2], ai, bw[v]);
#pragma unroll
                for (int v = kSchoolV - 1; v > 0; --v) bw[v] = bw[v - 1];
                bw[0] = bcol[-i - 1];
            }
        }
        uint32_t S[kSchoolV + 3];
        chunk_sum3<kSchoolV>(c, S);
        uint32_t H[3];
        H[0] = __shfl_up_sync(0xffffffffu, S[kSchoolV], 1);
        H[1] = __shfl_up_sync(0xffffffffu, S[kSchoolV + 1], 1);
        H[2] = __shfl_up_sync(0xffffffffu, S[kSchoolV + 2], 1);
        if (gl == 0) H[0] = H[1] = H[2] = 0u;
        uint32_t X[kSchoolV];
        const uint32_t g = chunk_add_spill<kSchoolV>(S, H, X);
        bool pp = true;
#pragma unroll
        for (int v = 0; v < kSchoolV; ++v) pp = pp && (X[v] == 0xffffffffu);
        const uint32_t gb = (__ballot_sync(0xffffffffu, g != 0u) >> (grp * G)) & gmask;
        const uint32_t pb = (__ballot_sync(0xffffffffu, pp) >> (grp * G)) & gmask;
        const GroupCarry gc = resolve_group_n(gb, pb, 0u, G);
        chunk_increment<kSchoolV>(X, (gc.carry_in_mask >> gl) & 1u);
        if (valid) {
            uint32_t *cr = C + row * sC;
#pragma unroll
            for (int v = 0; v < kSchoolV; ++v)
                if (k0 + v < Lc) cr[k0 + v] = X[v];
        }
        __syncwarp();
    }
}

template <int G>
static void launch_seg(const uint32_t *A, const uint32_t *B, uint32_t *C, uint32_t N, uint32_t La, uint32_t Lb,
                       uint64_t sA, uint64_t sB, uint64_t sC, cudaStream_t st) {
    constexpr int NP = kSegWarps * (32 / G);
    k_school_seg<G><<<grid_for(N, NP, kNumSMs * 32), 32 * kSegWarps, 0, st>>>(A, B, C, N, La, Lb, sA, sB, sC);
    count_launch();
}

// RAGGED: per-product descriptors (rows) give each product's offsets and
// lengths; otherwise La_u, Lb_u and the strides apply to every row.
template <int kSchoolThreads, bool RAGGED>
__global__ void __launch_bounds__(kSchoolThreads) k_school_cols(const uint32_t *__restrict__ A,
                                                                const uint32_t *__restrict__ B,
                                                                uint32_t *__restrict__ C, uint32_t N,
                                                                uint32_t La_u, uint32_t Lb_u, uint64_t sA,
                                                                uint64_t sB, uint64_t sC,
                                                                const RaggedRow *__restrict__ rows) {
    // a[0..La), bpad[j + kPad] = b_j (zero outside [0, Lb))
    __shared__ uint32_t sa[kSchoolMaxL];
    __shared__ uint32_t sb[kSchoolMaxL + kSchoolMaxL + 8];
    __shared__ uint32_t sg[kSchoolThreads / 32], sp[kSchoolThreads / 32];
    for (uint32_t row = blockIdx.x; row < N; row += gridDim.x) {
        const RaggedRow d = RAGGED ? rows[row] : RaggedRow{row * sA, row * sB, row * sC, La_u, Lb_u};
        const uint32_t La = d.La, Lb = d.Lb;
        const uint32_t kPad = La + 4;
        const uint32_t Lc = La + Lb;
        const uint32_t *ar = A + d.offA;
        const uint32_t *br = B + d.offB;
        for (uint32_t i = threadIdx.x; i < La; i += blockDim.x) sa[i] = ar[i];
        for (uint32_t j = threadIdx.x; j < kPad + Lb + 8; j += blockDim.x)
            sb[j] = (j >= kPad && j - kPad < Lb) ? br[j - kPad] : 0u;
        __syncthreads();
        const uint32_t k0 = threadIdx.x * kSchoolV;
        uint32_t c[kSchoolV][3];
#pragma unroll
        for (int v = 0; v < kSchoolV; ++v) c[v][0] = c[v][1] = c[v][2] = 0u;
        if (k0 < Lc) {
            // terms a_i * b_(k-i) for k in [k0, k0+4): i in [max(0, k0+1-Lb), min(La-1, k0+3)]
            const int ilo = max(0, (int)k0 + 1 - (int)Lb);
            const int ihi = min((int)La - 1, (int)k0 + kSchoolV - 1);
            for (int i = ilo; i <= ihi; ++i) {
                const uint32_t ai = sa[i];
                const uint32_t *bw = sb + kPad + k0 - i;   // bw[v] = b_(k0+v-i)
#pragma unroll
                for (int v = 0; v < kSchoolV; ++v) mac3(c[v][0], c[v][1], c[v][2], ai, bw[v]);
            }
        }
        uint32_t S[kSchoolV + 3];
        chunk_sum3<kSchoolV>(c, S);
        uint32_t H[3];
        H[0] = __shfl_up_sync(0xffffffffu, S[kSchoolV], 1);
        H[1] = __shfl_up_sync(0xffffffffu, S[kSchoolV + 1], 1);
        H[2] = __shfl_up_sync(0xffffffffu, S[kSchoolV + 2], 1);
        __shared__ uint32_t spill[kSchoolThreads / 32][3];
        if (lane_id() == 31) {
            spill[threadIdx.x >> 5][0] = S[kSchoolV];
            spill[threadIdx.x >> 5][1] = S[kSchoolV + 1];
            spill[threadIdx.x >> 5][2] = S[kSchoolV + 2];
        }
        __syncthreads();
        if (lane_id() == 0) {
            const int w = threadIdx.x >> 5;
            H[0] = w ? spill[w - 1][0] : 0u;
            H[1] = w ? spill[w - 1][1] : 0u;
            H[2] = w ? spill[w - 1][2] : 0u;
        }
        uint32_t X[kSchoolV];
        const uint32_t g = chunk_add_spill<kSchoolV>(S, H, X);
        bool p = true;
#pragma unroll
        for (int v = 0; v < kSchoolV; ++v) p = p && (X[v] == 0xffffffffu);
        const BlockCarry bc = block_resolve<kSchoolThreads / 32>(g != 0u, p, sg, sp);
        chunk_increment<kSchoolV>(X, bc.cin);
        uint32_t *cr = C + d.offC;
#pragma unroll
        for (int v = 0; v < kSchoolV; ++v)
            if (k0 + v < Lc) cr[k0 + v] = X[v];
        __syncthreads();
    }
}

// Thread-per-product size classes.
template <int MA, int MB>
static void launch_thread(const uint32_t *A, const uint32_t *B, uint32_t *C, uint32_t N, uint32_t La,
                          uint32_t Lb, uint64_t sA, uint64_t sB, uint64_t sC, cudaStream_t st) {
    k_school_thread<MA, MB><<<grid_for(N, 128, kNumSMs * 32), 128, 0, st>>>(A, B, C, N, La, Lb, sA, sB, sC);
    count_launch();
}

bool school_thread_fits(uint32_t La, uint32_t Lb) {
    return (La <= 16u && Lb <= 16u);
}

void school_mul(const uint32_t *A, const uint32_t *B, uint32_t *C, uint32_t N, uint32_t La,
                uint32_t Lb, uint64_t sA, uint64_t sB, uint64_t sC) {
    cudaStream_t st = current_stream();
    if (N == 0u || La + Lb == 0u) return;
    if (La == 0u || Lb == 0u) {
        cudaMemset2DAsync(C, sC * 4, 0, (size_t)(La + Lb) * 4, N, st);
        return;
    }
    KernelTimed kt("schoolbook", 4.0 * N * (2.0 * (La + Lb)));
    // keep the longer operand as A for the register kernels
    if (La < Lb) {
        std::swap(A, B);
        std::swap(La, Lb);
        std::swap(sA, sB);
    }
    if (La <= 4u && Lb <= 4u) {
        launch_thread<4, 4>(A, B, C, N, La, Lb, sA, sB, sC, st);
    } else if (La <= 8u && Lb <= 8u) {
        launch_thread<8, 8>(A, B, C, N, La, Lb, sA, sB, sC, st);
    } else if (La <= 16u && Lb <= 8u) {
        launch_thread<16, 8>(A, B, C, N, La, Lb, sA, sB, sC, st);
    } else if (La <= 16u && Lb <= 16u) {
        launch_thread<16, 16>(A, B, C, N, La, Lb, sA, sB, sC, st);
    } else if (La + Lb <= 32u) {
        launch_seg<8>(A, B, C, N, La, Lb, sA, sB, sC, st);
    } else if (La + Lb <= 64u) {
        launch_seg<16>(A, B, C, N, La, Lb, sA, sB, sC, st);
    } else if (La + Lb <= 128u) {
        launch_seg<32>(A, B, C, N, La, Lb, sA, sB, sC, st);
    } else {
        // one CTA per product, 4 output columns per thread
        const uint32_t g = grid_for(N, 1, kNumSMs * 16);
        if (La + Lb <= 256u)
            k_school_cols<64, false><<<g, 64, 0, st>>>(A, B, C, N, La, Lb, sA, sB, sC, nullptr);
        else if (La + Lb <= 512u)
            k_school_cols<128, false><<<g, 128, 0, st>>>(A, B, C, N, La, Lb, sA, sB, sC, nullptr);
        else
            k_school_cols<256, false><<<g, 256, 0, st>>>(A, B, C, N, La, Lb, sA, sB, sC, nullptr);
        count_launch();
    }
}

// Ragged batch: rows[i] gives the operands' offsets and lengths (L_a >= L_b,
// L_a + L_b <= 1024) and the output offset of product i (L_a + L_b limbs).
void school_mul_ragged(const uint32_t *A, const uint32_t *B, uint32_t *C, uint32_t N, const RaggedRow *rows,
                       uint64_t limb_products) {
    if (N == 0u) return;
    cudaStream_t st = current_stream();
    KernelTimed kt("schoolbook", 8.0 * (double)limb_products);
    k_school_cols<256, true><<<grid_for(N, 1, kNumSMs * 16), 256, 0, st>>>(A, B, C, N, 0u, 0u, 0u, 0u, 0u, rows);
    count_launch();
}

}  // namespace gpupi

void batch_mul_naive(uint32_t *A, uint32_t *B, uint32_t *ret, int N, int L_a, int L_b, int stride_A,
                     int stride_B, int stride_ret) {
    if (N <= 0 || L_a < 0 || L_b < 0 || L_a + L_b > BATCH_MUL_NAIVE_L_MAX) return;
    gpupi::school_mul(A, B, ret, (uint32_t)N, (uint32_t)L_a, (uint32_t)L_b, (uint32_t)stride_A,
                      (uint32_t)stride_B, (uint32_t)stride_ret);
}
