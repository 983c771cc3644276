// Element LU step of the static condensation (elementschur.cpp:6-329): D^-1 and
// D^-1 Ru by blocked Gauss-Jordan elimination with partial pivoting, the
// trailing updates on the FP64 tensor cores (mma.sync m8n8k4 f64).
//
// [D | Ru] sits in shared memory (one CTA per element).  Columns are eliminated
// in panels of 8:
//   1. warp 0 holds the panel (all rows x 8 columns) in registers and runs the
//      8 Gauss-Jordan steps on it alone -- pivot search by warp shuffles (first
//      row of maximal |.| among rows not yet pivoted), the in-place form that
//      leaves in column k the transformation column of step k;
//   2. the pivot rows' entries outside the panel are moved into a buffer B
//      (8 x columns) and zeroed in place;
//   3. every other column c takes the whole panel at once,
//      A(:, c) += W B(:, c), W = the panel's columns -- with T the product of
//      the panel's 8 elementary steps, column j of W is T e_{p_j}, so this is
//      T applied to A(:, c) (a rank-8 update, one 8x8 output tile per DMMA pair).
// No rows are swapped.  After the last panel the in-place result X satisfies
// D^-1(k, p_m) = X(p_k, m) and (D^-1 Ru)(k) = X(p_k, Ru column), p_k the row
// pivoted at step k.  A zero pivot reports 1 + step in info[e].  D^-1 replaces
// D; D^-1 Ru goes to RuOut (which may be Ru itself).
#pragma once
#include <cuda_runtime.h>
#include "schur_kernels.cuh"

namespace hfem {

// 16-byte asynchronous global->shared copy (both addresses 16-byte aligned).
__device__ __forceinline__ void cp_async16(double* smem, const double* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem));
}

template <int N>
struct InvBlk {
    static_assert(N % 2 == 0, "16-byte column copies need an even order");
    static constexpr int NP = ((N + 7) / 8) * 8;     // rows and matrix columns, padded to tiles
    static constexpr int RUC = NP;                   // column of Ru
    static constexpr int NCP = NP + 8;               // columns incl. the Ru tile
    static constexpr int LDA = NP + 2;               // 2*LDA = 4 (mod 16): conflict-free C fragments
    static constexpr int LDB = 12;                   // B(k, c) at k + LDB c
    static constexpr int R4 = (NP + 31) / 32;        // panel rows per lane of warp 0
    static constexpr int MT = NP / 8, NTL = NCP / 8; // row / column tiles
    static constexpr int THREADS = NP <= 24 ? 64 : (NP <= 64 ? 128 : 256);
    static constexpr size_t SMEM = sizeof(double) * ((size_t)LDA * NCP + (size_t)LDB * NCP);
};

// Gauss-Jordan steps kb .. kb+bn-1 on the panel columns kb..kb+7, by warp 0
// alone; returns 1 + step on a zero pivot, else 0.  `used` (per lane) marks the
// lane's rows that have pivoted.
template <int N>
__device__ __forceinline__ int inv_panel(double* __restrict__ A, int* __restrict__ piv, int kb, unsigned& used,
                                         int lane) {
    using C = InvBlk<N>;
    constexpr int NP = C::NP, LDA = C::LDA, R4 = C::R4;
    const int bn = min(8, N - kb);
    // panel columns kb..kb+7 of rows lane + 32 r; the column being
    // eliminated is always pv[.][0]: every step shifts the panel left by
    // one and appends the step's transformation column at pv[.][7]
    double pv[R4][8];
#pragma unroll
    for (int r = 0; r < R4; r++) {
        const int row = lane + 32 * r;
#pragma unroll
        for (int c = 0; c < 8; c++) pv[r][c] = (row < NP) ? A[row + LDA * (kb + c)] : 0.0;
    }
    int bad = 0;
#pragma unroll 1
    for (int j = 0; j < bn; j++) {
        // pivot: first row of maximal |.| among rows not yet pivoted.  Lane
        // candidates are compared across the warp as (high word, low word)
        // of the non-negative magnitude, then by row.
        double v = -1.0;
        int vi = NP;
#pragma unroll
        for (int r = 0; r < R4; r++) {
            const int row = lane + 32 * r;
            if (row < N && !((used >> r) & 1u)) {
                const double a = fabs(pv[r][0]);
                if (a > v) { v = a; vi = row; }
            }
        }
        const unsigned hi = v > 0.0 ? (unsigned)__double2hiint(v) : 0u;
        const unsigned lo = v > 0.0 ? (unsigned)__double2loint(v) : 0u;
        const unsigned mh = __reduce_max_sync(0xffffffffu, hi);
        const unsigned ml = __reduce_max_sync(0xffffffffu, hi == mh ? lo : 0u);
        if (mh == 0u && ml == 0u) {
            bad = kb + j + 1;
            break;
        }
        const int p = (int)__reduce_min_sync(0xffffffffu, (hi == mh && lo == ml) ? (unsigned)vi : 0xffffffffu);
        const int owner = p & 31, slot = p >> 5;
        double sp[8];
#pragma unroll
        for (int c = 0; c < 8; c++) {
            double x = pv[0][c];
#pragma unroll
            for (int r = 1; r < R4; r++)
                if (slot == r) x = pv[r][c];
            sp[c] = __shfl_sync(0xffffffffu, x, owner);
        }
        const double inv = 1.0 / sp[0];
#pragma unroll
        for (int c = 1; c < 8; c++) sp[c] *= inv;
#pragma unroll
        for (int r = 0; r < R4; r++) {
            const double f = pv[r][0];
#pragma unroll
            for (int c = 0; c < 7; c++) pv[r][c] = fma(-f, sp[c + 1], pv[r][c + 1]);
            pv[r][7] = -f * inv;
            if (lane + 32 * r == p) {
#pragma unroll
                for (int c = 0; c < 7; c++) pv[r][c] = sp[c + 1];
                pv[r][7] = inv;
                used |= 1u << r;
            }
        }
        if (lane == 0) piv[kb + j] = p;
    }
    // after bn shifts, position q holds panel column (q + bn) mod 8: the
    // transformation column of step j at kb + j, zero padding columns after
#pragma unroll
    for (int r = 0; r < R4; r++) {
        const int row = lane + 32 * r;
        if (row < NP)
#pragma unroll
            for (int q = 0; q < 8; q++) A[row + LDA * (kb + ((q + bn) & 7))] = pv[r][q];
    }
    return bad;
}

// One 8x8 tile of the rank-8 update A(:, c) += W B(:, c), W = A(:, kb..kb+7).
template <int N>
__device__ __forceinline__ void inv_tile(double* __restrict__ A, const double* __restrict__ B, int mt, int nt, int kb,
                                         int bn, int gr, int gc) {
    constexpr int LDA = InvBlk<N>::LDA, LDB = InvBlk<N>::LDB;
    double* cp = A + 8 * mt + gr + LDA * (8 * nt + 2 * gc);
    double c0 = cp[0], c1 = cp[LDA];
    const double* wp = A + 8 * mt + gr + LDA * (kb + gc);
    const double* bp = B + gc + LDB * (8 * nt + gr);
    dmma8x8x4(c0, c1, wp[0], bp[0]);
    if (bn > 4) dmma8x8x4(c0, c1, wp[4 * LDA], bp[4]);
    cp[0] = c0;
    cp[LDA] = c1;
}

template <int N>
__global__ void __launch_bounds__(InvBlk<N>::THREADS, 2)
    inverse_blocked_kernel(int ne, double* __restrict__ D, const double* Ru, double* RuOut, int* __restrict__ info) {
    using C = InvBlk<N>;
    constexpr int NP = C::NP, LDA = C::LDA, LDB = C::LDB, NW = C::THREADS / 32;
    extern __shared__ __align__(16) unsigned char inv_raw[];
    double* A = reinterpret_cast<double*>(inv_raw);   // LDA x NCP
    double* B = A + (size_t)LDA * C::NCP;             // LDB x NCP
    __shared__ int piv[NP];
    __shared__ int s_bad;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gr = lane >> 2, gc = lane & 3;
    for (int e = blockIdx.x; e < ne; e += gridDim.x) {
        double* De = D + (size_t)e * N * N;
        // D by 16-byte asynchronous copies, all in flight at once (N is even, so
        // every column starts 16-byte aligned in global and shared memory)
        for (int t = tid; t < (N / 2) * N; t += C::THREADS) {
            const int i2 = t % (N / 2), j = t / (N / 2);
            cp_async16(A + 2 * i2 + LDA * j, De + 2 * i2 + (size_t)N * j);
        }
        cp_async_commit();
        for (int t = tid; t < NP * C::NCP; t += C::THREADS) {
            const int i = t % NP, j = t / NP;
            if (i < N && j < N) continue;
            A[i + LDA * j] = (i < N && j == C::RUC) ? Ru[(size_t)e * N + i] : 0.0;
        }
        if (tid == 0) s_bad = 0;
        unsigned used = 0;   // warp 0: bit r set once row lane + 32 r has pivoted
        cp_async_wait<0>();
        __syncthreads();
        if (warp == 0) {
            const int bad = inv_panel<N>(A, piv, 0, used, lane);
            if (lane == 0 && bad) s_bad = bad;
        }
        __syncthreads();
        // Look-ahead: block kb's update reaches the next panel's columns first;
        // then warp 0 factors that panel while the other warps update the rest.
        for (int kb = 0; kb < N && !s_bad; kb += 8) {
            const int bn = min(8, N - kb);
            // pivot rows outside the panel -> B, zeroed in place
            for (int t = tid; t < 8 * C::NCP; t += C::THREADS) {
                const int j = t & 7, c = t >> 3;
                double v = 0.0;
                if (j < bn && (c < kb || c >= kb + 8)) {
                    double* a = A + piv[kb + j] + LDA * c;
                    v = *a;
                    *a = 0.0;
                }
                B[j + LDB * c] = v;
            }
            __syncthreads();
            const int ptile = kb >> 3;
            const bool more = kb + 8 < N;
            const int ntile = more ? ptile + 1 : -1;
            if (more) {
                for (int mt = warp; mt < C::MT; mt += NW) inv_tile<N>(A, B, mt, ntile, kb, bn, gr, gc);
                __syncthreads();
            }
            if (warp == 0) {
                if (more) {
                    const int bad = inv_panel<N>(A, piv, kb + 8, used, lane);
                    if (lane == 0 && bad) s_bad = bad;
                }
            } else {
                // the other warps: pairs of row tiles x column tiles, each warp a
                // contiguous run of them, so the panel fragments of its row pair
                // stay in registers across the run and every B fragment feeds
                // both row tiles
                constexpr int PR = (C::MT + 1) / 2, ITEMS = PR * C::NTL, UW = NW - 1;
                constexpr int RUN = (ITEMS + UW - 1) / UW;
                const int t0 = (warp - 1) * RUN, t1 = min(ITEMS, t0 + RUN);
                int cur = -1;
                double w[2][2];
                for (int t = t0; t < t1; t++) {
                    const int pr = t / C::NTL, nt = t % C::NTL;
                    if (pr != cur) {
                        cur = pr;
#pragma unroll
                        for (int u = 0; u < 2; u++) {
                            const int mt = 2 * pr + u;
                            const double* wp = A + 8 * mt + gr + LDA * (kb + gc);
                            w[u][0] = mt < C::MT ? wp[0] : 0.0;
                            w[u][1] = (mt < C::MT && bn > 4) ? wp[4 * LDA] : 0.0;
                        }
                    }
                    if (nt == ptile || nt == ntile) continue;
                    const double* bp = B + gc + LDB * (8 * nt + gr);
                    const double b0 = bp[0], b1 = bp[4];
#pragma unroll
                    for (int u = 0; u < 2; u++) {
                        const int mt = 2 * pr + u;
                        if (mt >= C::MT) continue;
                        double* cp = A + 8 * mt + gr + LDA * (8 * nt + 2 * gc);
                        double c0 = cp[0], c1 = cp[LDA];
                        dmma8x8x4(c0, c1, w[u][0], b0);
                        if (bn > 4) dmma8x8x4(c0, c1, w[u][1], b1);
                        cp[0] = c0;
                        cp[LDA] = c1;
                    }
                }
            }
            __syncthreads();
        }
        if (s_bad) {
            if (tid == 0) info[e] = s_bad;
            __syncthreads();
            continue;
        }
        for (int t = tid; t < N * N; t += C::THREADS) {
            const int k = t % N, m = t / N;
            De[k + (size_t)N * piv[m]] = A[piv[k] + LDA * m];
        }
        for (int k = tid; k < N; k += C::THREADS) RuOut[(size_t)e * N + k] = A[piv[k] + LDA * C::RUC];
        if (tid == 0) info[e] = 0;
        __syncthreads();
    }
}

}  // namespace hfem
