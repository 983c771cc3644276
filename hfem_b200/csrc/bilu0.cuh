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
// concurrently.  The host groups rows into such levels; one launch per level
// (one CTA per row), and the triangular solves of the apply run level by
// level the same way.
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

}  // namespace hfem
