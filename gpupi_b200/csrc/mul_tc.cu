// Schoolbook products on the tensor cores: split-integer int8 MMAs
// (tcgen05.mma kind::i8, INT32 accumulators in tensor memory), beside the
// CUDA-core schoolbook of mul_naive.cu (gpupi batch_mul_naive.cu:146-273,
// whose warp-per-product IMAD kernels this replaces where it is faster).
//
// Each 32-bit limb is four byte digits, so A * B = sum_k c_k 2^(8k) with
// c_k = sum_i a_i b_(k-i) over the byte digits of the shorter operand A (n_a
// bytes) and the longer B (n_b bytes).  One CTA computes all c_k of a
// product as a 128 x N matrix D in tensor memory,
//
//     D[s][u] = c_(128u + s),   s < 128, u < N = ceil((n_a + n_b) / 128),
//
// accumulated by Q x 4 MMAs of M = 128, K = 32 bytes, Q = ceil-ish(n_a/128)+1:
// for chunk q and step m (K index t < 32, taken in reverse within a step)
//
//     A_qm[s][t] = a_(128q - 32m + s - 31 + t)          (a Toeplitz band of a)
//     B_qm[u][t] = b_(128(u - q) + 32m + 31 - t)        (b in 128-byte blocks)
//
// so that every pair (i, j) with i + j = 128u + s meets exactly once.  Both
// operands are K-major, no swizzle (core matrices of 8 rows x 16 bytes):
//   * A from one shared-memory array P of 16-byte rows, P[r] = a[r-15 .. r]:
//     row s of A_qm is P[x - 16] (bytes t < 16) and P[x] (t >= 16) with
//     x = 128q - 32m + s, i.e. start = &P[x0 - 16], SBO = 128 (8 rows),
//     LBO = 256 (16 rows).  P costs 16 bytes of shared memory per byte of a.
//   * B from eight planes of 16-byte rows, plane j row u' = the 16 bytes
//     b[128u' + 16(7-j) .. +16) in reverse order; B_qm's K halves are planes
//     6 - 2m and 7 - 2m at row u - q (start shifted by -16q, LBO = plane size).
// Exactness: every c_k is a sum of at most n_a products of two bytes, each
// <= 255^2, so c_k <= 8192 * 65025 < 2^31 for n_a <= 8192 (A <= 2048 limbs):
// the signed 32-bit accumulators never overflow (static_assert below).
// Epilogue: D is read back with tcgen05.ld into shared memory, limb L of
// the product is S_L = c_4L + c_(4L+1) 2^8 + c_(4L+2) 2^16 + c_(4L+3) 2^24
// (< 2^56), and limb_L = lo(S_L) + hi(S_(L-1)) + carry, the binary carries
// resolved with ballots across the CTA, pass after pass of 512 limbs.
//
// Limits: min(L_a, L_b) <= 2048, L_a + L_b <= 8192 (N <= 256 columns).
// Waits on the MMA completion barrier are bounded; a wait that runs out sets
// the library's device error word (tc_error()) and the CTA stops.
#include "common.cuh"
#include "carry_tile.cuh"

namespace gpupi {
namespace tc {

constexpr int kThreads = 128;   // four warps: one per tensor-memory lane quadrant
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kMaxShort = 2048u;   // limbs of the shorter operand
constexpr uint32_t kMaxSum = 8192u;     // L_a + L_b
static_assert(4ull * kMaxShort * 255ull * 255ull < (1ull << 31), "int32 accumulators must not overflow");

struct Shape {
    uint32_t na, nb;   // bytes of A (shorter operand) and B
    uint32_t Q;        // reduction chunks of 128 bytes
    uint32_t N;        // output blocks of 128 bytes (MMA N, multiple of 16)
};

__host__ __device__ inline Shape shape_of(uint32_t La, uint32_t Lb) {
    Shape s;
    s.na = 4u * La;
    s.nb = 4u * Lb;
    s.Q = (s.na + 126u) / 128u + 1u;
    const uint32_t u = (s.na + s.nb + 127u) / 128u;
    s.N = (u + 15u) & ~15u;
    return s;
}

// Shared-memory layout for the largest shape of a launch (byte offsets).
struct Layout {
    uint32_t abuf;    // a's bytes at [128, 128 + n_a), zero around: 128Q + 160 bytes
    uint32_t p;       // P rows r in [-112, 128Q) (16 bytes each); later the c_k (4 bytes each)
    uint32_t planes;  // 8 planes of N + Q - 1 rows
    uint32_t total;
};

__host__ __device__ inline uint32_t up128(uint32_t x) { return (x + 127u) & ~127u; }

// Rows per plane: N + Q - 1, rounded up to an odd count so that the eight
// planes' rows u' fall in eight different 16-byte bank groups (the fill
// writes one row of all eight planes per eight lanes).
__host__ __device__ inline uint32_t plane_rows(uint32_t Q, uint32_t N) { return (N + Q - 1u) | 1u; }

__host__ __device__ inline Layout layout_of(uint32_t maxQ, uint32_t maxN) {
    Layout l;
    l.abuf = 0u;
    const uint32_t abytes = up128(128u * maxQ + 160u);
    l.p = abytes;
    const uint32_t psz = 16u * (128u * maxQ + 112u), csz = 4u * 128u * maxN;
    l.planes = l.p + up128(psz > csz ? psz : csz);
    l.total = l.planes + 8u * 16u * plane_rows(maxQ, maxN);
    return l;
}

__device__ uint32_t g_tc_error;   // nonzero after a bounded wait ran out

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor of tcgen05: start address, leading (K)
// and stride (M/N) byte offsets in 16-byte units, version 1, no swizzle.
__device__ __forceinline__ uint64_t desc_of(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: D s32 (bits 4-5 = 2), A and B unsigned 8-bit
// (format 0), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__device__ __forceinline__ uint32_t idesc_u8(uint32_t N) {
    return (2u << 4) | ((N >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma_u8(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    const uint32_t z = 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t"
        "}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    return ok != 0u;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

constexpr uint32_t kWaitLimit = 1u << 22;   // polls of the completion barrier
constexpr uint32_t kProbeLimit = 1u << 12;  // polls of the self-test's never-completing barrier

// S_L = c_4L + c_(4L+1) 2^8 + c_(4L+2) 2^16 + c_(4L+3) 2^24 (0 beyond the product)
__device__ __forceinline__ uint64_t limb_sum(const uint32_t *cs, uint32_t L, uint32_t Lc) {
    if (L >= Lc) return 0ull;
    const uint4 c = *reinterpret_cast<const uint4 *>(cs + 4u * L);
    return (uint64_t)c.x + ((uint64_t)c.y << 8) + ((uint64_t)c.z << 16) + ((uint64_t)c.w << 24);
}

template <bool RAGGED>
__global__ void __launch_bounds__(kThreads, 8)
    k_mul_tc(const uint32_t *__restrict__ A, const uint32_t *__restrict__ B, uint32_t *__restrict__ C, uint32_t nrows,
             uint32_t La_u, uint32_t Lb_u, uint64_t sA, uint64_t sB, uint64_t sC,
             const RaggedRow *__restrict__ rows, uint32_t tmem_cols, uint32_t maxQ, uint32_t maxN,
             uint32_t probe_timeout) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ __align__(8) uint64_t mbar_never;   // no arrival ever: the timeout self-test waits on it
    __shared__ uint32_t tmem_slot;
    __shared__ uint32_t sg[kWarps], sp[kWarps];
    const uint32_t tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
    const Layout lay = layout_of(maxQ, maxN);
    uint32_t *abuf = reinterpret_cast<uint32_t *>(smem + lay.abuf);
    uint8_t *P = smem + lay.p;
    uint32_t *cs = reinterpret_cast<uint32_t *>(smem + lay.p);
    uint8_t *planes = smem + lay.planes;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"(tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&mbar)));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&mbar_never)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;
    const uint32_t mbar_a = smem_addr(&mbar);
    uint32_t phase = 0u;
    bool failed = false;

    for (uint32_t row = blockIdx.x; row < nrows && !failed; row += gridDim.x) {
        const RaggedRow d = RAGGED ? rows[row] : RaggedRow{row * sA, row * sB, row * sC, La_u, Lb_u};
        const bool swap = d.La > d.Lb;
        const uint32_t *ap = swap ? B + d.offB : A + d.offA;
        const uint32_t *bp = swap ? A + d.offA : B + d.offB;
        const uint32_t La = swap ? d.Lb : d.La, Lb = swap ? d.La : d.Lb;
        const uint32_t Lc = La + Lb;
        const Shape sh = shape_of(La, Lb);
        const uint32_t prow_n = 128u * sh.Q + 112u;    // rows of P
        const uint32_t brow_n = sh.N + sh.Q - 1u;      // rows of each plane
        const uint32_t plane_bytes = 16u * plane_rows(sh.Q, sh.N);

        // 1. a's limbs at byte 128 of abuf (limb w - 32 in word w), zeros around
        const uint32_t abw = (128u * sh.Q + 160u) / 4u;
        for (uint32_t w = tid; w < abw; w += kThreads) abuf[w] = (w >= 32u && w - 32u < La) ? ap[w - 32u] : 0u;
        // 2. the planes of b: plane j row rr holds b[128u' + 16(7-j) .. +16)
        //    reversed, u' = rr - (Q - 1); zero outside b.  Eight consecutive
        //    threads read one 128-byte block of b (coalesced) and write row
        //    rr of the eight planes.
        for (uint32_t idx = tid; idx < 8u * brow_n; idx += kThreads) {
            const uint32_t j = idx & 7u, rr = idx >> 3;
            const int up = (int)rr - (int)(sh.Q - 1u);
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (up >= 0) {
                const uint32_t l0 = 32u * (uint32_t)up + 4u * (7u - j);   // first limb of the piece
                uint32_t w[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) w[e] = (l0 + e < Lb) ? bp[l0 + e] : 0u;
                v = make_uint4(__byte_perm(w[3], 0u, 0x0123), __byte_perm(w[2], 0u, 0x0123),
                               __byte_perm(w[1], 0u, 0x0123), __byte_perm(w[0], 0u, 0x0123));
            }
            *reinterpret_cast<uint4 *>(planes + j * plane_bytes + 16u * rr) = v;
        }
        __syncthreads();
        // 3. P: stored row rr is P[rr - 112] = a[rr - 127 .. rr - 112], i.e.
        //    abuf bytes rr + 1 .. rr + 16
        for (uint32_t rr = tid; rr < prow_n; rr += kThreads) {
            const uint32_t b0 = rr + 1u, i0 = b0 >> 2, sh8 = 8u * (b0 & 3u);
            uint32_t w[5];
#pragma unroll
            for (int e = 0; e < 5; ++e) w[e] = abuf[i0 + e];
            uint4 v;
            v.x = __funnelshift_r(w[0], w[1], sh8);
            v.y = __funnelshift_r(w[1], w[2], sh8);
            v.z = __funnelshift_r(w[2], w[3], sh8);
            v.w = __funnelshift_r(w[3], w[4], sh8);
            *reinterpret_cast<uint4 *>(P + 16u * rr) = v;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        fence_before();
        __syncthreads();

        // 4. one thread issues the Q x 4 MMAs and commits them to the barrier
        if (tid == 0) {
            fence_after();
            const uint32_t idesc = idesc_u8(sh.N);
            const uint32_t p0 = smem_addr(P), b0 = smem_addr(planes);
            for (uint32_t q = 0; q < sh.Q; ++q) {
#pragma unroll
                for (uint32_t m = 0; m < 4u; ++m) {
                    const uint32_t prow = 128u * q - 32u * m + 96u;   // stored row of P[x0 - 16], x0 = 128q - 32m
                    const uint64_t adesc = desc_of(p0 + 16u * prow, 256u, 128u);
                    const uint32_t j0 = 6u - 2u * m;
                    const uint64_t bdesc = desc_of(b0 + j0 * plane_bytes + 16u * (sh.Q - 1u - q), plane_bytes, 128u);
                    mma_u8(tmem, adesc, bdesc, idesc, (q | m) != 0u);
                }
            }
            mma_commit(mbar_a);
        }
        // 5. bounded wait for the MMAs.  The timeout self-test first waits on
        //    a barrier nothing arrives on, records that the wait ran out
        //    (error word 2), then waits, bounded again, for its own MMAs so
        //    that tensor memory is idle before it is released.
        uint32_t polls = 0u;
        if (probe_timeout) {
            while (!mbar_try_wait(smem_addr(&mbar_never), 0u) && ++polls < kProbeLimit) {
            }
            if (polls >= kProbeLimit && tid == 0) atomicExch(&g_tc_error, 2u);
            failed = true;
            polls = 0u;
        }
        while (!mbar_try_wait(mbar_a, phase)) {
            if (++polls >= kWaitLimit) {
                if (tid == 0) atomicExch(&g_tc_error, 1u);
                failed = true;
                break;
            }
        }
        phase ^= 1u;
        if (__syncthreads_or(failed)) {
            failed = true;
            break;
        }
        fence_after();
        // 6. D -> shared memory: cs[128u + s] = c_(128u + s) (the MMAs no
        //    longer read P, whose space this reuses); warp w reads lanes
        //    32w .. 32w + 31 of tensor memory
        {
            const uint32_t s = 32u * warp + lane;
            for (uint32_t g = 0; g < sh.N / 16u; ++g) {
                uint32_t r[16];
                tmem_ld16(tmem + ((32u * warp) << 16) + 16u * g, r);
#pragma unroll
                for (int e = 0; e < 16; ++e) cs[128u * (16u * g + e) + s] = r[e];
            }
        }
        fence_before();
        __syncthreads();
        // 7. limbs with carries, 4 limbs per thread per pass
        uint32_t pass_cin = 0u;
        uint32_t *out = C + d.offC;
        const uint32_t lt = (1u << lane) - 1u, wmask = (1u << warp) - 1u;
        for (uint32_t base = 0; base < Lc; base += 4u * kThreads) {
            const uint32_t L0 = base + 4u * tid;
            uint64_t prev = (L0 > 0u) ? limb_sum(cs, L0 - 1u, Lc) : 0ull;
            uint32_t X[4], cy = 0u;
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const uint64_t S = limb_sum(cs, L0 + v, Lc);
                const uint64_t t = (uint64_t)(uint32_t)S + (prev >> 32) + cy;
                X[v] = (uint32_t)t;
                cy = (uint32_t)(t >> 32);
                prev = S;
            }
            const bool p = (X[0] & X[1] & X[2] & X[3]) == 0xffffffffu;
            const BlockCarry bc = block_resolve<kWarps>(cy != 0u, p, sg, sp);
            const uint32_t pm = __ballot_sync(0xffffffffu, p);
            uint32_t wp = 0u;
#pragma unroll
            for (int k = 0; k < kWarps; ++k) wp |= sp[k] << k;
            const bool prev_all = ((pm & lt) == lt) && ((wp & wmask) == wmask);
            chunk_increment<4>(X, bc.cin | (prev_all ? pass_cin : 0u));
#pragma unroll
            for (int v = 0; v < 4; ++v)
                if (L0 + v < Lc) out[L0 + v] = X[v];
            pass_cin = bc.G | (bc.P & pass_cin);
            __syncthreads();
        }
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
}

}  // namespace tc

bool tc_fits(uint32_t La, uint32_t Lb) {
    return La > 0u && Lb > 0u && std::min(La, Lb) <= tc::kMaxShort && La + Lb <= tc::kMaxSum;
}

namespace {
uint32_t tmem_cols_for(uint32_t N) {
    uint32_t c = 32u;
    while (c < N) c <<= 1;
    return c;
}

template <bool RAGGED>
cudaError_t launch_tc(const uint32_t *A, const uint32_t *B, uint32_t *C, uint32_t n, uint32_t La, uint32_t Lb,
                      uint64_t sA, uint64_t sB, uint64_t sC, const RaggedRow *rows, uint32_t maxQ, uint32_t maxN,
                      cudaStream_t st, uint32_t probe = 0u) {
    const tc::Layout lay = tc::layout_of(maxQ, maxN);
    const uint32_t cols = tmem_cols_for(maxN);
    // opt in to the dynamic shared memory this shape needs (once per size
    // increase); the static part (barrier, carry flags) comes on top
    static size_t configured[2] = {0, 0};
    const size_t smem = lay.total;
    cudaError_t err = cudaSuccess;
    if (configured[RAGGED] < smem) {
        cudaFuncAttributes fa{};
        err = cudaFuncGetAttributes(&fa, tc::k_mul_tc<RAGGED>);
        if (err != cudaSuccess) return err;
        int dev = 0, optin = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (smem + fa.sharedSizeBytes > (size_t)optin) return cudaErrorInvalidValue;
        err = cudaFuncSetAttribute(tc::k_mul_tc<RAGGED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err != cudaSuccess) return err;
        configured[RAGGED] = smem;
    }
    // Resident CTAs per SM, the grid of this persistent kernel: the least of
    // what threads, registers (allocated per warp in units of 256),
    // shared memory (plus the 1 KiB the driver reserves per CTA) and
    // tensor memory (512 columns per SM) allow.  More CTAs than that would
    // only wait in tcgen05.alloc for a resident one to finish.
    static int occ_cache[2][6] = {};   // by RAGGED and log2(cols / 32)
    int lc = 0;
    while ((32u << lc) < cols) ++lc;
    int &occ = occ_cache[RAGGED][lc];
    static size_t occ_smem[2][6] = {};
    if (occ == 0 || occ_smem[RAGGED][lc] != smem) {
        cudaFuncAttributes fa{};
        err = cudaFuncGetAttributes(&fa, tc::k_mul_tc<RAGGED>);
        if (err != cudaSuccess) return err;
        int dev = 0, smem_sm = 0, regs_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
        const int warps = tc::kThreads / 32;
        const int regs_cta = warps * ((fa.numRegs * 32 + 255) / 256) * 256;
        const size_t smem_cta = smem + fa.sharedSizeBytes + 1024u;
        int o = 2048 / tc::kThreads;
        o = std::min(o, regs_sm / std::max(regs_cta, 1));
        o = std::min(o, (int)((size_t)smem_sm / smem_cta));
        o = std::min(o, (int)(512u / cols));
        occ = std::max(o, 1);
        occ_smem[RAGGED][lc] = smem;
    }
    const unsigned grid = (unsigned)std::min<uint64_t>(n, (uint64_t)kNumSMs * occ);
    tc::k_mul_tc<RAGGED><<<grid, tc::kThreads, smem, st>>>(A, B, C, n, La, Lb, sA, sB, sC, rows, cols, maxQ, maxN,
                                                           probe);
    count_launch();
    return cudaGetLastError();
}
}  // namespace

// Uniform batch: N products of La x Lb limbs (strides in limbs, 0 broadcasts).
cudaError_t tc_mul(const uint32_t *A, const uint32_t *B, uint32_t *C, uint32_t N, uint32_t La, uint32_t Lb,
                   uint64_t sA, uint64_t sB, uint64_t sC) {
    if (N == 0u) return cudaSuccess;
    if (!tc_fits(La, Lb)) return cudaErrorInvalidValue;
    const tc::Shape sh = tc::shape_of(std::min(La, Lb), std::max(La, Lb));
    KernelTimed kt("schoolbook_tc", 4.0 * N * (2.0 * (La + Lb)));
    return launch_tc<false>(A, B, C, N, La, Lb, sA, sB, sC, nullptr, sh.Q, sh.N, current_stream());
}

// Ragged batch (descriptors on the device); maxQ / maxN from the host's rows.
cudaError_t tc_mul_ragged(const uint32_t *A, const uint32_t *B, uint32_t *C, uint32_t n, const RaggedRow *rows,
                          uint32_t maxQ, uint32_t maxN, uint64_t limbs_moved) {
    if (n == 0u) return cudaSuccess;
    KernelTimed kt("schoolbook_tc", 4.0 * (double)limbs_moved);
    return launch_tc<true>(A, B, C, n, 0u, 0u, 0u, 0u, 0u, rows, maxQ, maxN, current_stream());
}

void tc_shape(uint32_t La, uint32_t Lb, uint32_t *Q, uint32_t *N) {
    const tc::Shape sh = tc::shape_of(std::min(La, Lb), std::max(La, Lb));
    *Q = sh.Q;
    *N = sh.N;
}

uint32_t tc_error();

// Timeout self-test: one 64 x 64-limb product whose CTA first waits on a
// barrier that never completes.  Returns the error word that call left (2:
// the bounded wait ran out and the kernel returned; the GPU stays usable)
// and, in *after, the error word of an ordinary product right after it (0).
cudaError_t tc_selftest_timeout(uint32_t *seen, uint32_t *after) {
    uint32_t *buf = nullptr;
    cudaError_t err = scratch_alloc((void **)&buf, 4u * 256u);
    if (err != cudaSuccess) return err;
    cudaStream_t st = current_stream();
    cudaMemsetAsync(buf, 0x5a, 4u * 256u, st);
    const tc::Shape sh = tc::shape_of(64u, 64u);
    tc_error();
    err = launch_tc<false>(buf, buf + 64, buf + 128, 1u, 64u, 64u, 64u, 64u, 128u, nullptr, sh.Q, sh.N, st, 1u);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
    if (err == cudaSuccess) *seen = tc_error();
    if (err == cudaSuccess) err = launch_tc<false>(buf, buf + 64, buf + 128, 1u, 64u, 64u, 64u, 64u, 128u, nullptr,
                                                   sh.Q, sh.N, st, 0u);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
    if (err == cudaSuccess) *after = tc_error();
    scratch_free(buf);
    return err;
}

// Reads and clears the device error word (1: a completion wait ran out).
uint32_t tc_error() {
    uint32_t v = 0u, z = 0u;
    if (cudaMemcpyFromSymbol(&v, tc::g_tc_error, sizeof v) != cudaSuccess) return 0xffffffffu;
    if (v) cudaMemcpyToSymbol(tc::g_tc_error, &z, sizeof z);
    return v;
}

}  // namespace gpupi
