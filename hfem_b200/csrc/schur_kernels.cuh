// Static condensation on sm_100a, FP64 (restating elementschur.cpp:6-329):
//   1. inverse_blocked_kernel (inverse_blocked.cuh): D^-1 and D^-1 Ru by blocked
//      Gauss-Jordan with partial pivoting;
//   2. batched_dgemm: D^-1 F and H - K (D^-1 F) on the FP64 tensor cores
//      (mma.sync m8n8k4 f64), one CTA per 40-row stripe of one element;
//   3. batched_dgemv: Rh - K (D^-1 Ru).
#pragma once
#include <cuda_runtime.h>

namespace hfem {

// ------------------------------------------------------------ FP64 mma GEMM
// D(8x8) += A(8x4, row) * B(4x8, col); lane l holds A(l/4, l%4), B(l%4, l/4),
// C(l/4, 2(l%4)) and C(l/4, 2(l%4)+1).
__device__ __forceinline__ void dmma8x8x4(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// C_e = beta C_e + alpha A_e B_e for e in [0, batch), column-major, batch strides
// sA, sB, sC.  CTA: NW warps, tile BM = 8*MT rows x BN = 8*WN*NW columns; warp w
// owns n-tiles [w*WN, (w+1)*WN) of all MT m-tiles.  K staged 20 deep; shared
// leading dimensions (A: 8*MT padded to 4 mod 16 doubles, B: 20) make the
// fragment loads bank-conflict free.  Grid: ceil(M/BM) * ceil(N/BN) * batch CTAs,
// element-major (the tiles of one element run together and share it in L2).
template <int MT, int WN, int NW, int BK_ = 20, int STAGES_ = 2>
struct GemmCfg {
    static constexpr int BM = 8 * MT, BN = 8 * WN * NW, BK = BK_, STAGES = STAGES_;
    static_assert(BK % 4 == 0 && STAGES >= 2, "k stages of whole DMMA steps, at least double buffered");
    static constexpr int LDA = ((BM + 11) / 16) * 16 + 4;     // >= BM, == 4 (mod 16)
    static constexpr int LDB = (BK % 16 == 4 || BK % 16 == 12) ? BK : BK + 4;   // == 4 or 12 (mod 16)
    static constexpr int THREADS = 32 * NW;
    static constexpr int ASZ = LDA * BK, BSZ = LDB * BN;
    static constexpr size_t SMEM = sizeof(double) * (size_t)STAGES * (ASZ + BSZ);
};

// 8-byte asynchronous global->shared copy; with valid == false nothing is read
// (src-size 0) and the shared word is zero-filled.  gmem must always be a valid
// global address (callers pass the operand's base when the element is outside).
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem), "r"(n));
}
// 16-byte variant (both addresses 16-byte aligned); zero-fills when !valid.
__device__ __forceinline__ void cp_async16z(double* smem, const double* gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N)); }

template <int MT, int WN, int NW, int BK_ = 20, int STAGES_ = 2>
__global__ void __launch_bounds__(32 * NW) batched_dgemm_kernel(int M, int N, int K, double alpha,
                                                                const double* __restrict__ A, int lda, long long sA,
                                                                const double* __restrict__ B, int ldb, long long sB,
                                                                double beta, double* __restrict__ C, int ldc,
                                                                long long sC) {
    using G = GemmCfg<MT, WN, NW, BK_, STAGES_>;
    extern __shared__ __align__(16) double gsm[];
    const int tilesM = (M + G::BM - 1) / G::BM, tilesN = (N + G::BN - 1) / G::BN;
    const int e = blockIdx.x / (tilesM * tilesN), tile = blockIdx.x % (tilesM * tilesN);
    const int m0 = (tile % tilesM) * G::BM, n0 = (tile / tilesM) * G::BN;
    const double* Ae = A + (size_t)e * sA;
    const double* Be = B + (size_t)e * sB;
    double* Ce = C + (size_t)e * sC;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gr = lane >> 2, gc = lane & 3;

    auto stage_a = [&](int st) { return gsm + st * (G::ASZ + G::BSZ); };
    auto stage_b = [&](int st) { return gsm + st * (G::ASZ + G::BSZ) + G::ASZ; };
    // pairs of doubles per copy when every column of A and B starts 16-byte
    // aligned and the copied extents (M rows of A, K rows of B) are even
    const bool pairs = ((M | K | lda | ldb) & 1) == 0 && ((reinterpret_cast<size_t>(Ae) | reinterpret_cast<size_t>(Be)) & 15) == 0;
    auto load = [&](int st, int k0) {
        double* As = stage_a(st);
        double* Bs = stage_b(st);
        if (pairs) {
            for (int t = tid; t < (G::BM / 2) * G::BK; t += G::THREADS) {
                const int m = 2 * (t % (G::BM / 2)), k = t / (G::BM / 2);
                const bool ok = (m0 + m < M) && (k0 + k < K);
                cp_async16z(&As[m + G::LDA * k], Ae + (ok ? (m0 + m) + (size_t)lda * (k0 + k) : 0), ok);
            }
            for (int t = tid; t < (G::BK / 2) * G::BN; t += G::THREADS) {
                const int k = 2 * (t % (G::BK / 2)), n = t / (G::BK / 2);
                const bool ok = (n0 + n < N) && (k0 + k < K);
                cp_async16z(&Bs[k + G::LDB * n], Be + (ok ? (k0 + k) + (size_t)ldb * (n0 + n) : 0), ok);
            }
        } else {
            for (int t = tid; t < G::BM * G::BK; t += G::THREADS) {
                const int m = t % G::BM, k = t / G::BM;
                const bool ok = (m0 + m < M) && (k0 + k < K);
                cp_async8(&As[m + G::LDA * k], Ae + (ok ? (m0 + m) + (size_t)lda * (k0 + k) : 0), ok);
            }
            for (int t = tid; t < G::BK * G::BN; t += G::THREADS) {
                const int k = t % G::BK, n = t / G::BK;
                const bool ok = (n0 + n < N) && (k0 + k < K);
                cp_async8(&Bs[k + G::LDB * n], Be + (ok ? (k0 + k) + (size_t)ldb * (n0 + n) : 0), ok);
            }
        }
    };

    // the accumulators start from beta C (loaded while the first stage is in
    // flight) and take alpha A B, so the epilogue only stores
    load(0, 0);
    cp_async_commit();
    double acc[MT][WN][2];
#pragma unroll
    for (int a = 0; a < MT; a++)
#pragma unroll
        for (int b = 0; b < WN; b++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int m = m0 + 8 * a + gr, n = n0 + 8 * (warp * WN + b) + 2 * gc + h;
                acc[a][b][h] = (beta != 0.0 && m < M && n < N) ? beta * Ce[m + (size_t)ldc * n] : 0.0;
            }
    const int nk = (K + G::BK - 1) / G::BK;
    // STAGES - 1 k stages in flight; one commit group per stage (empty past K)
#pragma unroll
    for (int st = 1; st < G::STAGES - 1; st++) {
        if (st < nk) load(st, st * G::BK);
        cp_async_commit();
    }
    for (int kt = 0; kt < nk; kt++) {
        cp_async_wait<G::STAGES - 2>();
        __syncthreads();
        // every thread is past stage kt - 1: its slot takes stage kt + STAGES - 1
        {
            const int nx = kt + G::STAGES - 1;
            if (nx < nk) load(nx % G::STAGES, nx * G::BK);
            cp_async_commit();
        }
        const double* As = stage_a(kt % G::STAGES);
        const double* Bs = stage_b(kt % G::STAGES);
#pragma unroll
        for (int ks = 0; ks < G::BK; ks += 4) {
            double af[MT], bf[WN];
#pragma unroll
            for (int a = 0; a < MT; a++) af[a] = alpha * As[(8 * a + gr) + G::LDA * (ks + gc)];
#pragma unroll
            for (int b = 0; b < WN; b++) bf[b] = Bs[(ks + gc) + G::LDB * (8 * (warp * WN + b) + gr)];
#pragma unroll
            for (int a = 0; a < MT; a++)
#pragma unroll
                for (int b = 0; b < WN; b++) dmma8x8x4(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
        }
    }
#pragma unroll
    for (int a = 0; a < MT; a++)
#pragma unroll
        for (int b = 0; b < WN; b++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int m = m0 + 8 * a + gr, n = n0 + 8 * (warp * WN + b) + 2 * gc + h;
                if (m < M && n < N) Ce[m + (size_t)ldc * n] = acc[a][b][h];
            }
}

// y_e = y_e + alpha A_e x_e   (A_e: M x K column-major)
__global__ void batched_dgemv_kernel(int batch, int M, int K, double alpha, const double* __restrict__ A,
                                     long long sA, const double* __restrict__ x, long long sx, double* __restrict__ y,
                                     long long sy) {
    const long long total = (long long)batch * M;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int e = (int)(t / M), r = (int)(t % M);
        const double* Ae = A + (size_t)e * sA;
        const double* xe = x + (size_t)e * sx;
        double s = 0.0;
        for (int k = 0; k < K; k++) s += Ae[r + (size_t)M * k] * xe[k];
        y[(size_t)e * sy + r] += alpha * s;
    }
}

}  // namespace hfem
