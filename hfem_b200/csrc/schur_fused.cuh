// Static condensation, FP64, both products in one kernel (elementschur.cpp:6-329):
//   X = D^-1 F  (n x nb, written out as DinvF)  and  H <- H - K X,
// on the FP64 tensor cores (mma.sync m8n8k4 f64).  One CTA per (element, strip
// of BN columns of F / DinvF / H): the strip of X never leaves shared memory
// between the two products.  A operands (D^-1, then K in row chunks) stream
// through a 2-stage cp.async ring in k tiles of 20; the B operand (the F strip,
// then the X strip) sits in shared memory whole.  Warp w owns m-tiles w, w+NW,
// ... of every job and all BN/8 n-tiles.  H's accumulators start from H.
// DinvF may be F itself: a CTA has its whole F strip in shared memory before it
// writes the X strip over it, and strips are disjoint.
#pragma once
#include <cuda_runtime.h>
#include "schur_kernels.cuh"

namespace hfem {

template <int N, int NB, int BN, int NW>
struct FusedCfg {
    static constexpr int BK = 20;
    static constexpr int MT = (N + 7) / 8;                 // m-tiles per job (rows of D^-1, or a chunk of K)
    static constexpr int BM = 8 * MT;
    static constexpr int NTN = BN / 8;                     // n-tiles
    static constexpr int KT = (N + BK - 1) / BK;           // k tiles
    static constexpr int KP = KT * BK;                     // padded k extent (rows of the B strip)
    static constexpr int LDA = ((BM + 11) / 16) * 16 + 4;  // == 4 (mod 16)
    static constexpr int LDB = ((KP + 11) / 16) * 16 + 4;  // == 4 (mod 16)
    static constexpr int MPW = (MT + NW - 1) / NW;         // m-tiles per warp
    static constexpr int CHUNKS = (NB + BM - 1) / BM;      // row chunks of K / H
    static constexpr int STRIPS = (NB + BN - 1) / BN;
    static constexpr int THREADS = 32 * NW;
    static constexpr size_t SMEM = sizeof(double) * ((size_t)LDB * BN + 2 * (size_t)LDA * BK);
    static_assert(BN % 8 == 0 && N % 2 == 0 && NB % 2 == 0, "tile and 16-byte copy granularity");
};

template <int N, int NB, int BN, int NW>
__global__ void __launch_bounds__(32 * NW) schur_fused_kernel(int ne, const double* __restrict__ Dinv,
                                                              const double* F,
                                                              const double* __restrict__ K, double* __restrict__ H,
                                                              double* DinvF) {
    using C = FusedCfg<N, NB, BN, NW>;
    extern __shared__ __align__(16) double fsm[];
    double* Bs = fsm;                                  // LDB x BN: the F strip, then the X strip
    double* As = fsm + (size_t)C::LDB * BN;            // 2 stages of LDA x BK
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gr = lane >> 2, gc = lane & 3;
    const int e = blockIdx.x / C::STRIPS, c0 = (blockIdx.x % C::STRIPS) * BN;
    if (e >= ne) return;
    const double* De = Dinv + (size_t)e * N * N;
    const double* Fe = F + (size_t)e * N * NB;
    const double* Ke = K + (size_t)e * NB * N;
    double* He = H + (size_t)e * NB * NB;
    double* Xe = DinvF + (size_t)e * N * NB;

    // the F strip (rows >= N and columns past NB zero)
    for (int t = tid; t < (C::KP / 2) * BN; t += C::THREADS) {
        const int k = 2 * (t % (C::KP / 2)), col = t / (C::KP / 2);
        const bool ok = k < N && c0 + col < NB;
        cp_async16z(&Bs[k + C::LDB * col], Fe + (ok ? k + (size_t)N * (c0 + col) : 0), ok);
    }
    cp_async_commit();

    // A tile loader: rows [m0, m0 + BM) of A (lda rows, m_end valid), k columns [k0, k0 + BK)
    auto load_a = [&](int st, const double* A, int lda, int m0, int m_end, int k0) {
        double* as = As + (size_t)st * C::LDA * C::BK;
        for (int t = tid; t < (C::BM / 2) * C::BK; t += C::THREADS) {
            const int m = 2 * (t % (C::BM / 2)), k = t / (C::BM / 2);
            const bool ok = m0 + m < m_end && k0 + k < N;
            cp_async16z(&as[m + C::LDA * k], A + (ok ? (m0 + m) + (size_t)lda * (k0 + k) : 0), ok);
        }
    };

    double acc[C::MPW][C::NTN][2];
    // one product: acc (+)= alpha A[m0.., :] Bs, k tiles through the ring
    auto run = [&](const double* A, int lda, int m0, int m_end, double alpha) {
        load_a(0, A, lda, m0, m_end, 0);
        cp_async_commit();
        for (int kt = 0; kt < C::KT; kt++) {
            cp_async_wait<0>();
            __syncthreads();
            if (kt + 1 < C::KT) load_a((kt + 1) & 1, A, lda, m0, m_end, (kt + 1) * C::BK);
            cp_async_commit();
            const double* as = As + (size_t)(kt & 1) * C::LDA * C::BK;
#pragma unroll
            for (int ks = 0; ks < C::BK; ks += 4) {
                double bf[C::NTN];
#pragma unroll
                for (int b = 0; b < C::NTN; b++) bf[b] = Bs[(kt * C::BK + ks + gc) + C::LDB * (8 * b + gr)];
#pragma unroll
                for (int a = 0; a < C::MPW; a++) {
                    const int mt = warp + NW * a;
                    if (mt < C::MT) {
                        const double af = alpha * as[(8 * mt + gr) + C::LDA * (ks + gc)];
#pragma unroll
                        for (int b = 0; b < C::NTN; b++) dmma8x8x4(acc[a][b][0], acc[a][b][1], af, bf[b]);
                    }
                }
            }
        }
        __syncthreads();   // every warp is done with the ring and with Bs
    };

    // ---- X = D^-1 F_strip
#pragma unroll
    for (int a = 0; a < C::MPW; a++)
#pragma unroll
        for (int b = 0; b < C::NTN; b++) acc[a][b][0] = acc[a][b][1] = 0.0;
    run(De, N, 0, N, 1.0);
    // X to global and into Bs (the B operand of the second product)
#pragma unroll
    for (int a = 0; a < C::MPW; a++) {
        const int mt = warp + NW * a;
#pragma unroll
        for (int b = 0; b < C::NTN; b++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int row = 8 * mt + gr, col = 8 * b + 2 * gc + h;
                if (mt < C::MT && row < N) {
                    Bs[row + C::LDB * col] = acc[a][b][h];
                    if (c0 + col < NB) Xe[row + (size_t)N * (c0 + col)] = acc[a][b][h];
                }
            }
    }
    __syncthreads();

    // ---- H_strip -= K X, in row chunks of BM
    for (int ch = 0; ch < C::CHUNKS; ch++) {
        const int m0 = ch * C::BM;
#pragma unroll
        for (int a = 0; a < C::MPW; a++)
#pragma unroll
            for (int b = 0; b < C::NTN; b++)
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int mt = warp + NW * a;
                    const int row = m0 + 8 * mt + gr, col = c0 + 8 * b + 2 * gc + h;
                    acc[a][b][h] = (mt < C::MT && row < NB && col < NB) ? He[row + (size_t)NB * col] : 0.0;
                }
        run(Ke, NB, m0, NB, -1.0);
#pragma unroll
        for (int a = 0; a < C::MPW; a++) {
            const int mt = warp + NW * a;
#pragma unroll
            for (int b = 0; b < C::NTN; b++)
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int row = m0 + 8 * mt + gr, col = c0 + 8 * b + 2 * gc + h;
                    if (mt < C::MT && row < NB && col < NB) He[row + (size_t)NB * col] = acc[a][b][h];
                }
        }
    }
}

}  // namespace hfem
