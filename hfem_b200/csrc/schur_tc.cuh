// Static condensation on the 5th-generation tensor cores (sm_100a tcgen05,
// kind::tf32, FP32 accumulation in tensor memory): the mixed-precision form
// of the two element GEMMs of schur_primal_matrix (elementschur.cpp:98-220),
//   DinvF = D^-1 F            (n x nb)
//   H     = H - K DinvF       (nb x nb)
// with D^-1 from the FP64 element LU.  One CTA per element at a time
// (persistent over elements), 512 threads:
//   * all threads stage the FP64 operands into shared memory as FP32 in the
//     canonical K-major, no-swizzle UMMA layout (8-row x 16-byte core
//     matrices; row r of k-chunk c at byte 16 (c * ROWS + r));
//   * one thread issues tcgen05.mma (M = 128, N = nb rounded to 16, k-step 8)
//     and commits to an mbarrier;
//   * every warp reads its 32 TMEM lanes back with tcgen05.ld for the
//     epilogues: DinvF goes to global memory (FP64, for the solution update)
//     and into shared memory as the B operand of the second GEMM; the Schur
//     update is applied to H in FP64.
// The Schur update's two 128-row tiles of K have their own A buffers, TMEM
// accumulators and barriers: the second tile is staged while the first
// tile's MMAs run, and its MMAs run while the first tile's epilogue reads
// and writes H.
// Every mbarrier wait is bounded; on expiry the kernel records an error,
// waits (bounded) for its MMAs, frees its tensor memory and returns.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace hfem {

struct SchurTcArgs {
    int ne;
    const double* Dinv;   // ne x (n x n), column-major
    const double* F;      // ne x (n x nb)
    const double* K;      // ne x (nb x n)
    double* H;            // ne x (nb x nb), H -= K D^-1 F in place
    double* DinvF;        // ne x (n x nb), written
    int* err;             // set to 1 when an MMA completion wait expires
};

template <int N, int NB>
struct TcCfg {
    static constexpr int KP = (N + 7) / 8 * 8;        // K padded to the tf32 k-step
    static constexpr int NBP = (NB + 15) / 16 * 16;   // MMA N (multiple of 16 for M = 128, <= 256)
    static constexpr int MT2 = (NB + 127) / 128;      // M tiles of the Schur update
    static constexpr int KC = KP / 4;                 // 16-byte k-chunks
    static constexpr uint32_t LBO_A = 128 * 16;       // bytes between k-chunks of an A tile
    static constexpr uint32_t LBO_B = NBP * 16;       // bytes between k-chunks of B
    static constexpr int A_BYTES = 128 * KP * 4;
    static constexpr int B_BYTES = NBP * KP * 4;
    static constexpr int NA = MT2 > 1 ? 2 : 1;        // A buffers (one per row tile of K)
    static constexpr int SMEM = NA * A_BYTES + B_BYTES + 1024;
    // accumulators: one per A buffer, ACC columns apart; the allocation is a
    // power of two of at least 32 columns
    static constexpr uint32_t ACC = NBP <= 32 ? 32 : (NBP <= 64 ? 64 : (NBP <= 128 ? 128 : 256));
    static constexpr uint32_t TMEM_COLS = NA * ACC < 32 ? 32 : NA * ACC;
    static_assert(N <= 128, "D must fit one 128-row MMA tile");
    static_assert(MT2 <= 2, "K must fit two 128-row MMA tiles");
    static_assert(NBP <= 256, "nb must fit one MMA N");
};

constexpr int TC_THREADS = 512;
constexpr int TC_GROUPS = TC_THREADS / 128;      // warp groups sharing the 128 TMEM lanes
constexpr long long TC_WAIT_LIMIT = 1ll << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: K-major, no swizzle, Blackwell version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: kind::tf32, F32 accumulator, A and B K-major.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int Nn) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(Nn >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(phase)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
    for (long long i = 0; i < TC_WAIT_LIMIT; i++)
        if (mbar_try(bar, phase)) return true;
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld8_nowait(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// A tile (128 rows x KP) from a column-major FP64 matrix: row r of the tile is
// global row r0 + r (valid while < rows), column k < KDIM; 4 chunks per thread
// have their 16 loads in flight together.
template <int KDIM, int ROWS>
__device__ __forceinline__ void stage_rows(float4* dst, const double* __restrict__ src, int ld, int r0, int rows,
                                           int tid) {
    constexpr int KC = (KDIM + 7) / 8 * 2;
    constexpr int TOT = KC * ROWS;
    constexpr int U = 4;
    for (int t0 = tid; t0 < TOT; t0 += TC_THREADS * U) {
        double v[U][4];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int t = t0 + u * TC_THREADS;
            const int kc = t / ROWS, m = t - kc * ROWS, k0 = 4 * kc, rg = r0 + m;
            const bool ok = t < TOT && rg < rows;
#pragma unroll
            for (int q = 0; q < 4; q++) v[u][q] = (ok && k0 + q < KDIM) ? src[rg + (size_t)ld * (k0 + q)] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int t = t0 + u * TC_THREADS;
            if (t < TOT) dst[t] = make_float4((float)v[u][0], (float)v[u][1], (float)v[u][2], (float)v[u][3]);
        }
    }
}

// B operand (NBP rows x KP) = transpose of a column-major FP64 KDIM x NCOL
// matrix: tile row nn is column nn, read as 16-byte pairs along k.
template <int KDIM, int NCOL, int NBP>
__device__ __forceinline__ void stage_cols(float4* dst, const double* __restrict__ src, int tid) {
    constexpr int KC = (KDIM + 7) / 8 * 2;
    constexpr int TOT = KC * NBP;
    constexpr int U = 4;
    for (int t0 = tid; t0 < TOT; t0 += TC_THREADS * U) {
        double2 v[U][2];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int t = t0 + u * TC_THREADS;
            const int kc = t / NBP, nn = t - kc * NBP, k0 = 4 * kc;
            const bool ok = t < TOT && nn < NCOL;
            const double2* col = reinterpret_cast<const double2*>(src + (size_t)KDIM * nn + k0);
            v[u][0] = (ok && k0 < KDIM) ? col[0] : make_double2(0.0, 0.0);
            v[u][1] = (ok && k0 + 2 < KDIM) ? col[1] : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int t = t0 + u * TC_THREADS;
            if (t < TOT) dst[t] = make_float4((float)v[u][0].x, (float)v[u][0].y, (float)v[u][1].x, (float)v[u][1].y);
        }
    }
}

template <int N, int NB>
__global__ void __launch_bounds__(TC_THREADS, 1) schur_tc_kernel(SchurTcArgs A) {
    using C = TcCfg<N, NB>;
    extern __shared__ __align__(16) unsigned char tc_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(tc_raw) + 1023) &
                                                           ~static_cast<uintptr_t>(1023));
    float4* sA[2] = {reinterpret_cast<float4*>(base),                       // [kc][128 rows]
                     reinterpret_cast<float4*>(base + (C::NA - 1) * C::A_BYTES)};
    float4* sB = reinterpret_cast<float4*>(base + C::NA * C::A_BYTES);      // [kc][NBP rows]
    float* sBf = reinterpret_cast<float*>(sB);
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ uint32_t tslot;
    __shared__ int s_bad;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wq = warp & 3, grp = warp >> 2;
    const int row = 32 * wq + lane;                               // accumulator row = TMEM lane
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tslot)),
                     "r"(C::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[1])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_bad = 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tslot;
    const uint32_t acc[2] = {tmem, tmem + C::ACC};
    const uint32_t lane_off = (uint32_t)(32 * wq) << 16;
    const uint32_t abase[2] = {smem_u32(sA[0]), smem_u32(sA[1])}, bbase = smem_u32(sB);
    const uint32_t barp[2] = {smem_u32(&bar[0]), smem_u32(&bar[1])};
    constexpr uint32_t IDESC = idesc_tf32(128, C::NBP);
    uint32_t phase[2] = {0, 0};
    int pend[2] = {0, 0};                                         // thread 0: commits whose wait expired
    uint32_t pend_phase[2] = {0, 0};

    auto issue = [&](int a, int t) {                              // thread 0: A buffer a x B -> accumulator t
        tc_fence_after();
#pragma unroll 1
        for (int s = 0; s < C::KP / 8; s++)
            tc_mma(acc[t], umma_desc(abase[a] + 2 * s * C::LBO_A, C::LBO_A, 128),
                   umma_desc(bbase + 2 * s * C::LBO_B, C::LBO_B, 128), IDESC, s > 0 ? 1u : 0u);
        tc_commit(barp[t]);
    };
    auto wait = [&](int t) {
        if (!mbar_wait(barp[t], phase[t])) {
            s_bad = 1;
            if (tid == 0) pend[t] = 1, pend_phase[t] = phase[t];
        }
        phase[t] ^= 1;
        tc_fence_after();
    };

    for (int e = blockIdx.x; e < A.ne; e += gridDim.x) {
        const double* Di = A.Dinv + (size_t)e * N * N;
        const double* Fe = A.F + (size_t)e * N * NB;
        const double* Ke = A.K + (size_t)e * NB * N;
        double* He = A.H + (size_t)e * NB * NB;
        double* DFe = A.DinvF + (size_t)e * N * NB;
        // ---- stage A = D^-1 (row m, k) and B = F^T (row nn, k) as FP32
        stage_rows<N, 128>(sA[0], Di, N, 0, N, tid);
        stage_cols<N, NB, C::NBP>(sB, Fe, tid);
        proxy_fence();
        __syncthreads();
        // ---- GEMM 1: accumulator 0 = D^-1 F
        if (tid == 0) issue(0, 0);
        wait(0);
        // ---- epilogue 1: DinvF to global (FP64) and to sB as B = DinvF^T (row nn, k)
        for (int cb = grp; cb < C::NBP / 8; cb += TC_GROUPS) {
            uint32_t r[8];
            tmem_ld8(acc[0] + lane_off + 8 * cb, r);
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const int nn = 8 * cb + j;
                const float v = __uint_as_float(r[j]);
                const bool valid = row < N && nn < NB;
                if (valid) DFe[row + N * nn] = (double)v;
                if (row < C::KP) sBf[((row >> 2) * C::NBP + nn) * 4 + (row & 3)] = valid ? v : 0.f;
            }
        }
        tc_fence_before();
        // ---- GEMM 2: the row tiles of K, each in its own A buffer and accumulator
        __syncthreads();                  // sA[0] free (GEMM 1 done), accumulator 0 read
        stage_rows<N, 128>(sA[0], Ke, NB, 0, NB, tid);
        proxy_fence();
        __syncthreads();
        if (s_bad) break;
        if (tid == 0) issue(0, 0);
        if constexpr (C::MT2 > 1) {
            stage_rows<N, 128>(sA[1], Ke, NB, 128, NB, tid);      // while tile 0's MMAs run
            proxy_fence();
            __syncthreads();
            if (tid == 0) issue(1, 1);
        }
#pragma unroll 1
        for (int mt = 0; mt < C::MT2; mt++) {
            const int t = mt;                                     // row tile mt: A buffer and accumulator mt
            wait(t);
            const int rg = 128 * mt + row;
            for (int cb = grp; cb < C::NBP / 8; cb += 2 * TC_GROUPS) {
                const bool two = cb + TC_GROUPS < C::NBP / 8;
                double h[16];
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const int nn = 8 * (j < 8 ? cb : cb + TC_GROUPS) + (j & 7);
                    h[j] = (rg < NB && nn < NB && (j < 8 || two)) ? He[rg + (size_t)NB * nn] : 0.0;
                }
                uint32_t r0[8], r1[8];
                tmem_ld8_nowait(acc[t] + lane_off + 8 * cb, r0);
                if (two) tmem_ld8_nowait(acc[t] + lane_off + 8 * (cb + TC_GROUPS), r1);
                tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const int nn = 8 * (j < 8 ? cb : cb + TC_GROUPS) + (j & 7);
                    const uint32_t bits = j < 8 ? r0[j] : r1[j & 7];
                    if (rg < NB && nn < NB && (j < 8 || two)) He[rg + (size_t)NB * nn] = h[j] - (double)__uint_as_float(bits);
                }
            }
        }
        tc_fence_before();
        __syncthreads();                  // accumulators read, sA / sB free for the next element
        if (s_bad) break;
    }
    __syncthreads();
    if (s_bad && tid == 0) {
        atomicExch(A.err, 1);
        // let any MMA still in flight finish before the tensor memory is released
        for (int t = 0; t < 2; t++)
            if (pend[t]) mbar_wait(barp[t], pend_phase[t]);
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(C::TMEM_COLS));
    }
}

}  // namespace hfem
