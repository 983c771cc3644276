// Block ILU(0) preconditioner on the face-block system (sm_100a), in a given
// row order (kernel/computeBILU0.m:1-46, kernel/applyBILU0.m:1-48).
//
// Mg has Hg's block-CSR pattern and holds, after the factorisation, the unit
// lower factor's blocks L_ik (neighbours k earlier in the order), the upper
// factor's blocks U_ik (neighbours later) and the inverted diagonal blocks
// U_ii^-1.  The factorisation is computed row by row ("IKJ" form): row i takes
// the updates of its earlier neighbours k in increasing order -- the same
// sequence of block updates the reference's right-looking loop applies to
// row i -- so rows whose earlier neighbours are all final can be factored
// concurrently.  The host groups rows into such levels, and the factorisation
// and the triangular solves of the apply walk them level by level: in one CTA
// when the levels are short (the scheduled forms at the end of this file),
// else one launch per level (one CTA per row).
#pragma once
#include <cuda_runtime.h>

namespace hfem {

constexpr int BILU_THREADS = 128;

// C = A B for bsz x bsz column-major blocks in shared memory (all threads).
__device__ __forceinline__ void smem_blk_mul(int b, const double* A, const double* B, double* C) {
    for (int t = threadIdx.x; t < b * b; t += blockDim.x) {
        const int r = t % b, c = t / b;
        double s = 0.0;
        for (int k = 0; k < b; k++) s += A[r + b * k] * B[k + b * c];
        C[t] = s;
    }
}

// In-place inverse of a bsz x bsz block in shared memory, Gauss-Jordan with
// partial pivoting; returns 1 + k on a zero pivot (all threads agree).
__device__ int smem_blk_inv(int b, double* a, double* col, int* piv, int* s_p) {
    for (int k = 0; k < b; k++) {
        if (threadIdx.x == 0) {
            int p = k;
            double best = fabs(a[k + b * k]);
            for (int r = k + 1; r < b; r++) {
                const double v = fabs(a[r + b * k]);
                if (v > best) { best = v; p = r; }
            }
            *s_p = p;
            piv[k] = p;
        }
        __syncthreads();
        const int p = *s_p;
        if (a[p + b * k] == 0.0) return k + 1;
        if (p != k)
            for (int c = threadIdx.x; c < b; c += blockDim.x) {
                const double t = a[k + b * c];
                a[k + b * c] = a[p + b * c];
                a[p + b * c] = t;
            }
        __syncthreads();
        const double dinv = 1.0 / a[k + b * k];
        for (int r = threadIdx.x; r < b; r += blockDim.x) col[r] = (r == k) ? 0.0 : a[r + b * k];
        __syncthreads();
        for (int c = threadIdx.x; c < b; c += blockDim.x) a[k + b * c] = (c == k ? 1.0 : a[k + b * c]) * dinv;
        __syncthreads();
        for (int t = threadIdx.x; t < b * b; t += blockDim.x) {
            const int r = t % b, c = t / b;
            if (r != k) a[r + b * c] = (c == k ? 0.0 : a[r + b * c]) - col[r] * a[k + b * c];
        }
        __syncthreads();
    }
    for (int k = b - 1; k >= 0; k--) {
        const int p = piv[k];
        if (p != k)
            for (int r = threadIdx.x; r < b; r += blockDim.x) {
                const double t = a[r + b * k];
                a[r + b * k] = a[r + b * p];
                a[r + b * p] = t;
            }
        __syncthreads();
    }
    return 0;
}

struct BiluArgs {
    int bsz;
    const int* rowstart;
    const int* colidx;
    const int* u2o;
    const int* rows;        // rows of this level
    int nrows;              // rows in this level
    const int* fptr;        // per row: earlier neighbours' positions, sorted by order (fptr[i]..fptr[i+1])
    const int* fpos;
    double* Mg;
    int* info;              // per row: 1 + pivot on a singular diagonal block
};

// Factor the rows of one level (one CTA per row).
__global__ void __launch_bounds__(BILU_THREADS) bilu0_factor_kernel(BiluArgs A) {
    extern __shared__ __align__(16) unsigned char bl_raw[];
    const int b = A.bsz;
    const size_t b2 = (size_t)b * b;
    double* L = reinterpret_cast<double*>(bl_raw);   // b2
    double* T = L + b2;                               // b2
    double* col = T + b2;                             // b
    int* piv = reinterpret_cast<int*>(col + b);       // b
    __shared__ int s_p;
    for (int w = blockIdx.x; w < A.nrows; w += gridDim.x) {
        const int i = A.rows[w];
        const int r0 = A.rowstart[i], r1 = A.rowstart[i + 1];
        for (int f = A.fptr[i]; f < A.fptr[i + 1]; f++) {
            const int p = A.fpos[f];
            const int k = A.colidx[p];
            const int ok = A.u2o[k];
            // L_ik = M_ik U_kk^-1
            __syncthreads();
            for (int t = threadIdx.x; t < (int)b2; t += blockDim.x) T[t] = A.Mg[(size_t)p * b2 + t];
            __syncthreads();
            smem_blk_mul(b, T, A.Mg + (size_t)A.rowstart[k] * b2, L);
            __syncthreads();
            for (int t = threadIdx.x; t < (int)b2; t += blockDim.x) A.Mg[(size_t)p * b2 + t] = L[t];
            // M_il -= L_ik U_kl for every neighbour l of i later than k that is also a neighbour of k
            for (int q = r0; q < r1; q++) {
                const int l = A.colidx[q];
                if (A.u2o[l] <= ok) continue;
                int m = -1;
                for (int s = A.rowstart[k] + 1; s < A.rowstart[k + 1]; s++)
                    if (A.colidx[s] == l) m = s;
                if (m < 0) continue;
                __syncthreads();
                smem_blk_mul(b, L, A.Mg + (size_t)m * b2, T);
                __syncthreads();
                for (int t = threadIdx.x; t < (int)b2; t += blockDim.x) A.Mg[(size_t)q * b2 + t] -= T[t];
            }
        }
        __syncthreads();
        for (int t = threadIdx.x; t < (int)b2; t += blockDim.x) T[t] = A.Mg[(size_t)r0 * b2 + t];
        __syncthreads();
        const int bad = smem_blk_inv(b, T, col, piv, &s_p);
        __syncthreads();
        if (bad) {
            if (threadIdx.x == 0) A.info[i] = bad;
            continue;
        }
        for (int t = threadIdx.x; t < (int)b2; t += blockDim.x) A.Mg[(size_t)r0 * b2 + t] = T[t];
        if (threadIdx.x == 0) A.info[i] = 0;
    }
}

struct BiluSolveArgs {
    int bsz;
    const int* rowstart;
    const int* colidx;
    const int* u2o;
    const int* rows;
    int nrows;
    const void* Mg;         // factors, double or float (FP32 factors in mixed precision)
    const double* x;        // right-hand side (lower solve)
    double* y;              // lower: y = L^-1 x; upper: in y, out v
    double* v;
};

// Lower solve of one level: y_i = x_i - sum_{k earlier} L_ik y_k (one CTA per row).
// MT is the factors' type; vectors and sums are FP64.
template <class MT>
__global__ void __launch_bounds__(64) bilu0_lower_kernel(BiluSolveArgs A) {
    const MT* Mg = static_cast<const MT*>(A.Mg);
    const int b = A.bsz;
    const size_t b2 = (size_t)b * b;
    for (int w = blockIdx.x; w < A.nrows; w += gridDim.x) {
        const int i = A.rows[w], oi = A.u2o[i];
        for (int r = threadIdx.x; r < b; r += blockDim.x) {
            double t = A.x[(size_t)i * b + r];
            for (int p = A.rowstart[i] + 1; p < A.rowstart[i + 1]; p++) {
                const int k = A.colidx[p];
                if (A.u2o[k] >= oi) continue;
                const MT* L = Mg + (size_t)p * b2;
                const double* yk = A.y + (size_t)k * b;
                double s = 0.0;
                for (int c = 0; c < b; c++) s += (double)L[r + b * c] * yk[c];
                t -= s;
            }
            A.y[(size_t)i * b + r] = t;
        }
    }
}

// Upper solve of one level: v_i = U_ii^-1 (y_i - sum_{k later} U_ik v_k).
template <class MT>
__global__ void __launch_bounds__(64) bilu0_upper_kernel(BiluSolveArgs A) {
    __shared__ double t[64];
    const MT* Mg = static_cast<const MT*>(A.Mg);
    const int b = A.bsz;
    const size_t b2 = (size_t)b * b;
    for (int w = blockIdx.x; w < A.nrows; w += gridDim.x) {
        const int i = A.rows[w], oi = A.u2o[i];
        __syncthreads();
        for (int r = threadIdx.x; r < b; r += blockDim.x) {
            double s = A.y[(size_t)i * b + r];
            for (int p = A.rowstart[i] + 1; p < A.rowstart[i + 1]; p++) {
                const int k = A.colidx[p];
                if (A.u2o[k] <= oi) continue;
                const MT* U = Mg + (size_t)p * b2;
                const double* vk = A.v + (size_t)k * b;
                double d = 0.0;
                for (int c = 0; c < b; c++) d += (double)U[r + b * c] * vk[c];
                s -= d;
            }
            t[r] = s;
        }
        __syncthreads();
        const MT* Dinv = Mg + (size_t)A.rowstart[i] * b2;
        for (int r = threadIdx.x; r < b; r += blockDim.x) {
            double s = 0.0;
            for (int c = 0; c < b; c++) s += (double)Dinv[r + b * c] * t[c];
            A.v[(size_t)i * b + r] = s;
        }
    }
}

// Both triangular solves in one CTA of 1024 threads, level after level with a
// CTA barrier in between: for orderings whose levels hold few rows (MDF gives
// long dependency chains) this replaces two launches per level by one launch.
// Each warp takes one row of the level at a time; lanes own the row's entries.
template <class MT>
__global__ void __launch_bounds__(1024) bilu0_apply_cta_kernel(BiluSolveArgs A, const int* __restrict__ lvl_lo,
                                                               int nlo, const int* __restrict__ rows_lo,
                                                               const int* __restrict__ lvl_up, int nup,
                                                               const int* __restrict__ rows_up) {
    __shared__ double t[32][64];
    const MT* Mg = static_cast<const MT*>(A.Mg);
    const int b = A.bsz;
    const size_t b2 = (size_t)b * b;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int l = 0; l < nlo; l++) {
        for (int q = lvl_lo[l] + w; q < lvl_lo[l + 1]; q += nw) {
            const int i = rows_lo[q], oi = A.u2o[i];
            for (int r = lane; r < b; r += 32) {
                double s = A.x[(size_t)i * b + r];
                for (int p = A.rowstart[i] + 1; p < A.rowstart[i + 1]; p++) {
                    const int k = A.colidx[p];
                    if (A.u2o[k] >= oi) continue;
                    const MT* L = Mg + (size_t)p * b2;
                    const double* yk = A.y + (size_t)k * b;
                    double d = 0.0;
                    for (int c = 0; c < b; c++) d += (double)L[r + b * c] * yk[c];
                    s -= d;
                }
                A.y[(size_t)i * b + r] = s;
            }
        }
        __syncthreads();
    }
    for (int l = 0; l < nup; l++) {
        for (int q = lvl_up[l] + w; q < lvl_up[l + 1]; q += nw) {
            const int i = rows_up[q], oi = A.u2o[i];
            for (int r = lane; r < b; r += 32) {
                double s = A.y[(size_t)i * b + r];
                for (int p = A.rowstart[i] + 1; p < A.rowstart[i + 1]; p++) {
                    const int k = A.colidx[p];
                    if (A.u2o[k] <= oi) continue;
                    const MT* U = Mg + (size_t)p * b2;
                    const double* vk = A.v + (size_t)k * b;
                    double d = 0.0;
                    for (int c = 0; c < b; c++) d += (double)U[r + b * c] * vk[c];
                    s -= d;
                }
                t[w][r] = s;
            }
            __syncwarp();
            const MT* Dinv = Mg + (size_t)A.rowstart[i] * b2;
            for (int r = lane; r < b; r += 32) {
                double s = 0.0;
                for (int c = 0; c < b; c++) s += (double)Dinv[r + b * c] * t[w][c];
                A.v[(size_t)i * b + r] = s;
            }
            __syncwarp();
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Scheduled forms for block sizes up to 32, for orderings whose levels hold
// few rows.  One CTA walks the levels with a CTA barrier between them; warp w
// owns slots w, w + nw, ... of the level order (a slot is a row's place in
// it), lane r owning row r of the row's blocks.  The host flattens every
// index chain into one fixed-stride record per slot, and each warp requests
// what does not depend on earlier levels -- its next row's record, and the
// blocks that are final before that row's level starts -- by asynchronous
// copies as soon as its previous row is done, typically levels ahead; after
// a row's level barrier only what the previous levels produced is fetched.
//
// Every array these kernels write (the factors, y, v) is written by this one
// CTA, so the L1-cached copies below see its own writes after a barrier.
constexpr int BILU_ROWMAX = 7;   // blocks per row: 2 nfe - 1 for triangles (5) and tetrahedra (7)

// Per-slot records, fixed stride so one asynchronous copy fetches a slot's
// whole description (ints):
//   factorisation (BILU_FREC): [0] row i, [1] rowstart[i], [2] blocks in the
//     row, [3] records n_r, [4] U blocks n_u; [8 + 2t, 9 + 2t] record t, t < 32:
//     per earlier neighbour k in order {M_ik's block in the row, updates n},
//     then n x {M_il's block in the row, 0}; [72 + t] U block t, t < 32: the
//     positions of U_kk^-1 and the U_kl in the order the records use them;
//   solves (BILU_SREC): [0] row i, [1] entries n_e (at most BILU_ROWMAX - 1),
//     [2] position of U_ii^-1 (upper solve), [3] the row's slot; [4 + 2j,
//     5 + 2j] entry j: {position of L_ik or U_ik, k}; [16 + j] k's slot.
// Slots: a row's result (y_i in the lower solve, v_i in the upper) is also
// kept in a shared-memory slot from its level to the last level that reads
// it; the host assigns the slots (an interval colouring of those live
// ranges), so that a level reads its neighbours' results from shared memory.
constexpr int BILU_FREC = 128, BILU_SREC = 32;

struct BiluSched {
    int nlo, nup;               // levels of the lower (and factorisation) order and of the upper order
    const int* lvl_lo;          // level l: slots lvl_lo[l] .. lvl_lo[l+1] of the lower order
    const int* lvl_up;
    const int* frec;            // per slot of the lower order
    const int* lrec;            // per slot of the lower order
    const int* urec;            // per slot of the upper order
    int nslot_lo, nslot_up;     // slots of each solve (0: results read from global memory)
};

// 4- or 8-byte asynchronous global->shared copy, cached in L1.
template <class T>
__device__ __forceinline__ void bl_cp_async(T* smem, const T* gmem) {
    static_assert(sizeof(T) == 4 || sizeof(T) == 8, "element copies of 4 or 8 bytes");
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(sa), "l"(gmem), "n"(sizeof(T)) : "memory");
}
__device__ __forceinline__ void bl_cp_async16(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void bl_cp_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
template <class T>
__device__ __forceinline__ void bl_warp_copy(T* s, const T* g, int n, int lane) {
    for (int t = lane; t < n; t += 32) bl_cp_async(s + t, g + t);
}
// a slot's record into the warp's record area (issued ahead; waited for by the next copy round)
__device__ __forceinline__ void bl_fetch_record(int* rc, const int* rec, int stride, int lane) {
    __syncwarp();
    if (4 * lane < stride) bl_cp_async16(rc + 4 * lane, rec + 4 * lane);
}

template <int B>
struct BiluFacCfg {
    static constexpr int B2 = B * B;
    static constexpr int UBUF = B <= 20 ? 8 : 4;                       // U blocks staged per round
    static constexpr size_t BLK_BYTES = (((size_t)(BILU_ROWMAX + UBUF) * B2 * sizeof(double) + 15) / 16) * 16;
    static constexpr size_t WARP_BYTES = BLK_BYTES + 2 * BILU_FREC * 4;  // blocks, two records
    static constexpr int NW0 = (int)((200 * 1024) / WARP_BYTES);
    static constexpr int NW = NW0 > 8 ? 8 : NW0;                       // warps of the CTA
    static constexpr size_t SMEM = WARP_BYTES * NW;
};

// The factorisation of every level in one CTA: row i, held in shared memory,
// takes for each earlier neighbour k in order L_ik = M_ik U_kk^-1 and
// M_il -= L_ik U_kl, then inverts its diagonal block by Gauss-Jordan with
// partial pivoting in registers, and is written back.  The inverse is the one
// smem_blk_inv computes (same pivots: the first position of largest magnitude;
// same operations), with the lanes of a row keeping it and tracking the
// position the row swaps give it, so a swap costs no data movement.  The block
// products sum in the order of smem_blk_mul.  For B <= 16 the two half-warps
// split every row's columns, halving each lane's products and eliminations.
template <int B>
__global__ void __launch_bounds__(256, 1) bilu0_factor_sched_kernel(BiluSched S, double* Mg, int* info) {
    static_assert(B <= 32, "one lane per block row");
    using C = BiluFacCfg<B>;
    constexpr int B2 = C::B2, UBUF = C::UBUF;
    constexpr unsigned FULL = 0xffffffffu;
    extern __shared__ __align__(16) unsigned char bf_raw[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    // for B <= 16 each half-warp holds half of every block row's columns:
    // lane h * 16 + r owns row r, columns h * CH .. h * CH + CH - 1
    constexpr int H = B <= 16 ? 2 : 1, LW = 32 / H, CH = (B + H - 1) / H;
    const int h = lane / LW, rl = lane % LW, cb = h * CH;
    const bool act = rl < B;
    const int r = act ? rl : 0;   // lanes of rows >= B repeat row 0 and store nothing
    double* rowbuf = reinterpret_cast<double*>(bf_raw + (size_t)w * C::WARP_BYTES);
    double* ubuf = rowbuf + (size_t)BILU_ROWMAX * B2;
    int* rcb = reinterpret_cast<int*>(bf_raw + (size_t)w * C::WARP_BYTES + C::BLK_BYTES);   // 2 x BILU_FREC
    int* rc = rcb;   // the record of the warp's current row
    // stage U blocks ub .. ub + UBUF - 1 of the row's list
    auto stage = [&](int ub, int nu) {
        __syncwarp();
        const int n = min(UBUF, nu - ub);
        for (int j = 0; j < n; j++) bl_warp_copy(ubuf + (size_t)j * B2, Mg + (size_t)rc[72 + ub + j] * B2, B2, lane);
        bl_cp_wait_all();
        __syncwarp();
    };
    // the row's own blocks were requested by advance (below); stage(0) waits for them
    auto factor_row = [&]() {
        const int i = rc[0], r0 = rc[1], nrb = rc[2], nrec = rc[3], nu = rc[4];
        int uc = 0, rb = 0;
        stage(0, nu);
        for (int j = 0; j < nrec;) {
            const int pl = rc[8 + 2 * j], nupd = rc[9 + 2 * j];
            j++;
            if (uc - rb == UBUF) stage(rb = uc, nu);
            const double* Ukk = ubuf + (size_t)(uc - rb) * B2;
            uc++;
            double* Mik = rowbuf + (size_t)pl * B2;
            // L_ik = M_ik U_kk^-1: the lane's columns of row r (the whole row of
            // M_ik, which the other half-warp may have just updated, is read)
            double m[B], lv[CH];
            __syncwarp();
#pragma unroll
            for (int q = 0; q < B; q++) m[q] = Mik[r + B * q];
#pragma unroll
            for (int cc = 0; cc < CH; cc++) {
                const int c = min(cb + cc, B - 1);
                double t = 0.0;
#pragma unroll
                for (int q = 0; q < B; q++) t = fma(m[q], Ukk[q + B * c], t);
                lv[cc] = t;
            }
            __syncwarp();
            if (act)
#pragma unroll
                for (int cc = 0; cc < CH; cc++)
                    if (cb + cc < B) Mik[r + B * (cb + cc)] = lv[cc];
            __syncwarp();
            // M_il -= L_ik U_kl with the whole row r of L_ik
#pragma unroll
            for (int q = 0; q < B; q++) m[q] = Mik[r + B * q];
            for (int u = 0; u < nupd; u++) {
                const int ql = rc[8 + 2 * j];
                j++;
                if (uc - rb == UBUF) stage(rb = uc, nu);
                const double* Ukl = ubuf + (size_t)(uc - rb) * B2;
                uc++;
                double* Mil = rowbuf + (size_t)ql * B2;
#pragma unroll
                for (int cc = 0; cc < CH; cc++) {
                    const int c = min(cb + cc, B - 1);
                    double t = 0.0;
#pragma unroll
                    for (int q = 0; q < B; q++) t = fma(m[q], Ukl[q + B * c], t);
                    if (act && cb + cc < B) Mil[r + B * c] -= t;
                }
            }
        }
        // the diagonal block (first in the row), inverted in place: the lanes
        // of row r hold the row now at position pos (row swaps move positions only)
        double a[CH];
        int piv[B];
        __syncwarp();
#pragma unroll
        for (int cc = 0; cc < CH; cc++) a[cc] = cb + cc < B ? rowbuf[r + B * (cb + cc)] : 0.0;
        int pos = rl, bad = 0;
#pragma unroll
        for (int k = 0; k < B; k++) {
            const int hk = k / CH, kc = k % CH;   // the half and slot holding column k
            // pivot: the first position >= k of largest magnitude in column k,
            // compared across the warp as (high word, low word) of |a|, then position
            const bool cand = h == hk && pos >= k && pos < B;
            const double mg = cand ? fabs(a[kc]) : 0.0;
            const unsigned hi = mg > 0.0 ? (unsigned)__double2hiint(mg) : 0u;
            const unsigned lo = mg > 0.0 ? (unsigned)__double2loint(mg) : 0u;
            const unsigned mh = __reduce_max_sync(FULL, cand ? hi : 0u);
            const unsigned ml = __reduce_max_sync(FULL, (cand && hi == mh) ? lo : 0u);
            if (mh == 0u && ml == 0u) {
                bad = k + 1;
                break;
            }
            const unsigned key =
                __reduce_min_sync(FULL, (cand && hi == mh && lo == ml) ? (unsigned)(pos * 32 + lane) : 0xffffffffu);
            const int pp = (int)(key >> 5), lp = (int)(key & 31u), lr = lp % LW;
            piv[k] = pp;
            if (pos == k) pos = pp;
            else if (rl == lr) pos = k;
            const double dinv = 1.0 / __shfl_sync(FULL, a[kc], lp);
            if (rl == lr)
#pragma unroll
                for (int cc = 0; cc < CH; cc++) a[cc] = (cb + cc == k ? 1.0 : a[cc]) * dinv;
            const double col = __shfl_sync(FULL, a[kc], hk * LW + rl);
#pragma unroll
            for (int cc = 0; cc < CH; cc++) {
                const double pc = __shfl_sync(FULL, a[cc], h * LW + lr);
                if (rl != lr) a[cc] = (cb + cc == k ? 0.0 : a[cc]) - col * pc;
            }
        }
        if (!bad) {
            // undo the column order of the pivots: swap columns k and piv[k], last first
#pragma unroll
            for (int k = B - 1; k >= 0; k--) {
                const int p = piv[k];
                const int hk = k / CH, kc = k % CH, hp = p / CH, pc = p % CH;
                if (p != k && hk == hp) {
                    if (h == hk) {
                        const double ak = a[kc];
#pragma unroll
                        for (int cc = 0; cc < CH; cc++)
                            if (cc == pc) {
                                a[kc] = a[cc];
                                a[cc] = ak;
                            }
                    }
                } else if (p != k) {
                    double xp = 0.0;
#pragma unroll
                    for (int cc = 0; cc < CH; cc++)
                        if (cc == pc) xp = a[cc];
                    const double vk = __shfl_sync(FULL, a[kc], hk * LW + rl);
                    const double vp = __shfl_sync(FULL, xp, hp * LW + rl);
                    if (h == hk) a[kc] = vp;
                    if (h == hp)
#pragma unroll
                        for (int cc = 0; cc < CH; cc++)
                            if (cc == pc) a[cc] = vk;
                }
            }
            __syncwarp();
            if (act)
#pragma unroll
                for (int cc = 0; cc < CH; cc++)
                    if (cb + cc < B) rowbuf[pos + B * (cb + cc)] = a[cc];
        }
        __syncwarp();
        for (int t = lane; t < nrb * B2; t += 32) Mg[(size_t)r0 * B2 + t] = rowbuf[t];
        if (lane == 0) info[i] = bad;
    };
    // warp w owns slots w, w + nw, ... of the level order; the record of its
    // jr-th row lives in record buffer jr mod 2.  A row's own blocks change
    // only while it is factored, so they are requested as soon as the warp's
    // previous row is done (after the barrier that ends its level), typically
    // levels before the row's own level starts.
    const int nrow = S.nlo > 0 ? S.lvl_lo[S.nlo] : 0;
    int s = w, jr = 0;
    auto advance = [&]() {   // row jr (slot s): its blocks, then the record of the warp's next row
        __syncwarp();
        if (s < nrow) {
            bl_cp_wait_all();
            __syncwarp();
            rc = rcb + (jr & 1) * BILU_FREC;
            bl_warp_copy(rowbuf, Mg + (size_t)rc[1] * B2, rc[2] * B2, lane);
        }
        if (s + nw < nrow)
            bl_fetch_record(rcb + ((jr + 1) & 1) * BILU_FREC, S.frec + (size_t)(s + nw) * BILU_FREC, BILU_FREC, lane);
    };
    if (s < nrow) bl_fetch_record(rcb, S.frec + (size_t)s * BILU_FREC, BILU_FREC, lane);
    advance();
    bool pend = false;
    for (int l = 0; l < S.nlo; l++) {
        for (const int se = S.lvl_lo[l + 1]; s < se;) {
            if (pend) advance();
            factor_row();
            s += nw;
            jr++;
            pend = true;
        }
        __syncthreads();
        if (pend) {
            advance();
            pend = false;
        }
    }
    bl_cp_wait_all();
}

template <int B, class MT>
struct BiluSolCfg {
    static constexpr int B2 = B * B;
    static constexpr size_t BLK_BYTES = ((BILU_ROWMAX * B2 * sizeof(MT) + 15) / 16) * 16;
    static constexpr size_t WARP_BYTES = BLK_BYTES + 3 * BILU_SREC * 4;   // blocks, three records
    static constexpr size_t BUDGET = 200 * 1024;                          // shared memory of the CTA
    // warps for a slot table of nslot rows (0: too large for shared memory)
    static int warps(int nslot) {
        const size_t tab = (size_t)nslot * B * sizeof(double);
        if (tab + WARP_BYTES > BUDGET) return 0;
        const size_t n = (BUDGET - tab) / WARP_BYTES;
        return n > 16 ? 16 : (int)n;
    }
    static size_t smem(int nw, int nslot) { return WARP_BYTES * nw + (size_t)nslot * B * sizeof(double); }
};

__device__ __forceinline__ void bl_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bl_cp_wait_but_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Both triangular solves in one CTA, v = U^-1 L^-1 x, software-pipelined
// over each warp's rows: warp w owns slots w, w + nw, ... of the level order,
// and after the barrier that ends a level in which it finished a row it
// requests the blocks and right-hand side entry of its next row (typically
// several levels later) and the record of the row after that, so a row's own
// data has arrived by the time its level starts and only the neighbours'
// results (previous levels') are read after the barrier.  For
// B <= 16 the two half-warps take alternate entries and add their partial
// sums by one shuffle; the upper solve's product with U_ii^-1 takes the row's
// sums from the lanes that hold them.
template <int B, class MT>
__global__ void __launch_bounds__(512, 1) bilu0_solve_sched_kernel(BiluSched S, const MT* __restrict__ Mg,
                                                                   const double* __restrict__ x, double* y,
                                                                   double* v) {
    static_assert(B <= 32, "one lane per block row");
    using C = BiluSolCfg<B, MT>;
    constexpr int B2 = C::B2, H = B <= 16 ? 2 : 1, LW = 32 / H;
    constexpr unsigned FULL = 0xffffffffu;
    extern __shared__ __align__(16) unsigned char bs_raw[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int g = lane / LW, r = lane % LW;
    const int rr = r < B ? r : 0;
    MT* blk = reinterpret_cast<MT*>(bs_raw + (size_t)w * C::WARP_BYTES);
    int* rcb = reinterpret_cast<int*>(bs_raw + (size_t)w * C::WARP_BYTES + C::BLK_BYTES);   // 3 x BILU_SREC
    double* tab = reinterpret_cast<double*>(bs_raw + (size_t)nw * C::WARP_BYTES);           // slot table
    // the row of record rc: its blocks (U_ii^-1 after them for the upper
    // solve) by asynchronous copies, and its right-hand side entry
    auto issue_row = [&](const int* rc, const double* b, bool upper) {
        const int i = rc[0], ne = rc[1];
        for (int j = 0; j < ne; j++) bl_warp_copy(blk + (size_t)j * B2, Mg + (size_t)rc[4 + 2 * j] * B2, B2, lane);
        if (upper) bl_warp_copy(blk + (size_t)ne * B2, Mg + (size_t)rc[2] * B2, B2, lane);
        return b[(size_t)i * B + rr];
    };
    // sum_j (block j row r) . vec_kj over the row's entries, whole row in every
    // lane; vec_kj from k's slot when the solve has slots
    auto rowsum = [&](const int* rc, const double* vec, bool slots) {
        const int ne = rc[1];
        auto src = [&](int j) { return slots ? tab + (size_t)rc[16 + j] * B : vec + (size_t)rc[5 + 2 * j] * B; };
        double t = 0.0;
        if (g < ne) {
            double va[B], vb[B];
            const bool two = g + H < ne;
            const double* ka = src(g);
            const double* kb = src(two ? g + H : g);
#pragma unroll
            for (int c = 0; c < B; c++) va[c] = ka[c];
#pragma unroll
            for (int c = 0; c < B; c++) vb[c] = kb[c];
            const MT* ba = blk + (size_t)g * B2 + rr;
            double d = 0.0;
#pragma unroll
            for (int c = 0; c < B; c++) d = fma((double)ba[B * c], va[c], d);
            t = d;
            if (two) {
                const MT* bb = blk + (size_t)(g + H) * B2 + rr;
                d = 0.0;
#pragma unroll
                for (int c = 0; c < B; c++) d = fma((double)bb[B * c], vb[c], d);
                t += d;
            }
            for (int j = g + 2 * H; j < ne; j += H) {
                const MT* bj = blk + (size_t)j * B2 + rr;
                const double* kj = src(j);
                d = 0.0;
#pragma unroll
                for (int c = 0; c < B; c++) d = fma((double)bj[B * c], kj[c], d);
                t += d;
            }
        }
        if (H == 2) t += __shfl_xor_sync(FULL, t, 16);
        return t;
    };
    // one triangular solve over its levels; out_i = rhs_i - sum (lower) or
    // U_ii^-1 (rhs_i - sum) (upper)
    auto sweep = [&](int nlev, const int* lvl, const int* rec, const double* b, const double* vec, double* out,
                     bool upper, bool slots) {
        const int nrow = nlev > 0 ? lvl[nlev] : 0;
        // this warp's rows: slots w, w + nw, w + 2 nw, ... of the level order
        // (about nw / (rows per level) levels apart); the record of the warp's
        // j-th row lives in record buffer j mod 2
        int s = w, j = 0;
        double rhs = 0.0;
        // prologue: the records of the first two rows, the blocks of the first
        if (s < nrow) bl_fetch_record(rcb, rec + (size_t)s * BILU_SREC, BILU_SREC, lane);
        bl_cp_wait_all();
        __syncwarp();
        if (s < nrow) rhs = issue_row(rcb, b, upper);
        bl_cp_commit();
        if (s + nw < nrow) bl_fetch_record(rcb + BILU_SREC, rec + (size_t)(s + nw) * BILU_SREC, BILU_SREC, lane);
        bl_cp_commit();
        // request the warp's next row (slot s, its j-th): its blocks (its record
        // arrived while the previous row waited), then the record of the row after it
        auto advance = [&]() {
            __syncwarp();
            if (s < nrow) {
                bl_cp_wait_all();
                __syncwarp();
                rhs = issue_row(rcb + (j & 1) * BILU_SREC, b, upper);
            }
            bl_cp_commit();
            if (s + nw < nrow)
                bl_fetch_record(rcb + ((j + 1) & 1) * BILU_SREC, rec + (size_t)(s + nw) * BILU_SREC, BILU_SREC, lane);
            bl_cp_commit();
        };
        // a warp that finished a row requests its next one after the barrier,
        // off the path of the level that row ended
        bool pend = false;
        for (int l = 0; l < nlev; l++) {
            for (const int se = lvl[l + 1]; s < se;) {
                if (pend) advance();
                const int* rc = rcb + (j & 1) * BILU_SREC;
                bl_cp_wait_but_one();   // this row's blocks (the next row's record may still be in flight)
                __syncwarp();
                const double t = rowsum(rc, vec, slots);
                double o = rhs - t;
                if (upper) {
                    const MT* Dinv = blk + (size_t)rc[1] * B2 + rr;
                    double u = 0.0;
#pragma unroll
                    for (int c = 0; c < B; c++) u = fma((double)Dinv[B * c], __shfl_sync(FULL, o, c), u);
                    o = u;
                }
                if (g == 0 && r < B) {
                    out[(size_t)rc[0] * B + r] = o;
                    if (slots) tab[(size_t)rc[3] * B + r] = o;
                }
                s += nw;
                j++;
                pend = true;
            }
            __syncthreads();
            if (pend) {
                advance();
                pend = false;
            }
        }
        bl_cp_wait_all();
    };
    sweep(S.nlo, S.lvl_lo, S.lrec, x, y, y, false, S.nslot_lo > 0);
    __syncthreads();   // the slot table changes hands
    sweep(S.nup, S.lvl_up, S.urec, y, v, v, true, S.nslot_up > 0);
}

}  // namespace hfem
