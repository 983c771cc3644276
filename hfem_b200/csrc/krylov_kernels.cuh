// Face-block linear algebra for the condensed HDG system on sm_100a:
// block-CSR matvec fused with the block-Jacobi apply, batched inverses of the
// diagonal blocks, and deterministic dot products for GMRES.
//
// Specifications (the reference ships these only as closed archives):
//   kernel/matvec.m:1-12         y_i = sum_k Hg_k x_{col(k)}
//   kernel/mkBlockJacobi.m:1-16  M_i^-1 = inv(Hg_ii), the first block of row i
//   kernel/gmres_bilu0.m:17-105  left-preconditioned restarted GMRES, MGS
#pragma once
#include <cuda_runtime.h>

namespace hfem {

constexpr int DOT_CTAS = 296;       // 2 x 148 SMs
constexpr int DOT_THREADS = 256;

// Inverse of each row's diagonal block by Gauss-Jordan with partial pivoting.
// One CTA per block row; bsz <= 64.  info[i] = 1 + k on a zero pivot.
__global__ void bj_inverse_kernel(int nrows, int bsz, const int* __restrict__ rowstart, const double* __restrict__ Hg,
                                  double* __restrict__ Minv, int* __restrict__ info) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* a = reinterpret_cast<double*>(smem_raw);   // bsz x bsz
    double* col = a + bsz * bsz;
    int* piv = reinterpret_cast<int*>(col + bsz);
    __shared__ int s_p;
    const int tid = threadIdx.x;
    for (int i = blockIdx.x; i < nrows; i += gridDim.x) {
        __syncthreads();
        const double* blk = Hg + (size_t)rowstart[i] * bsz * bsz;
        for (int t = tid; t < bsz * bsz; t += blockDim.x) a[t] = blk[t];
        __syncthreads();
        int bad = 0;
        for (int k = 0; k < bsz; k++) {
            if (tid == 0) {
                int p = k;
                double best = fabs(a[k + bsz * k]);
                for (int r = k + 1; r < bsz; r++) {
                    const double v = fabs(a[r + bsz * k]);
                    if (v > best) { best = v; p = r; }
                }
                s_p = p;
                piv[k] = p;
            }
            __syncthreads();
            const int p = s_p;
            if (a[p + bsz * k] == 0.0) { bad = k + 1; break; }
            if (p != k)
                for (int c = tid; c < bsz; c += blockDim.x) {
                    const double t = a[k + bsz * c];
                    a[k + bsz * c] = a[p + bsz * c];
                    a[p + bsz * c] = t;
                }
            __syncthreads();
            const double dinv = 1.0 / a[k + bsz * k];
            for (int r = tid; r < bsz; r += blockDim.x) col[r] = (r == k) ? 0.0 : a[r + bsz * k];
            __syncthreads();
            for (int c = tid; c < bsz; c += blockDim.x) a[k + bsz * c] = (c == k ? 1.0 : a[k + bsz * c]) * dinv;
            __syncthreads();
            for (int t = tid; t < bsz * bsz; t += blockDim.x) {
                const int r = t % bsz, c = t / bsz;
                if (r != k) a[r + bsz * c] = (c == k ? 0.0 : a[r + bsz * c]) - col[r] * a[k + bsz * c];
            }
            __syncthreads();
        }
        if (bad) {
            if (tid == 0) info[i] = bad;
            continue;
        }
        for (int k = bsz - 1; k >= 0; k--) {
            const int p = piv[k];
            if (p != k)
                for (int r = tid; r < bsz; r += blockDim.x) {
                    const double t = a[r + bsz * k];
                    a[r + bsz * k] = a[r + bsz * p];
                    a[r + bsz * p] = t;
                }
            __syncthreads();
        }
        double* out = Minv + (size_t)i * bsz * bsz;
        for (int t = tid; t < bsz * bsz; t += blockDim.x) out[t] = a[t];
        if (tid == 0) info[i] = 0;
    }
}

// z = M^-1 (Hg x) for every block row (M^-1 == NULL: z = Hg x).
// One CTA of 64 threads per block row, rows r = threadIdx.x < bsz.
template <typename MT>
__global__ void bsr_matvec_bj_kernel(int nrows, int bsz, const int* __restrict__ rowstart, const int* __restrict__ colidx,
                                     const double* __restrict__ Hg, const MT* __restrict__ Minv,
                                     const double* __restrict__ x, double* __restrict__ z) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* y = reinterpret_cast<double*>(smem_raw);
    const int r = threadIdx.x;
    for (int i = blockIdx.x; i < nrows; i += gridDim.x) {
        double s = 0.0;
        if (r < bsz) {
            for (int k = rowstart[i]; k < rowstart[i + 1]; k++) {
                const double* blk = Hg + (size_t)k * bsz * bsz;
                const double* xj = x + (size_t)colidx[k] * bsz;
                for (int c = 0; c < bsz; c++) s += blk[r + bsz * c] * __ldg(&xj[c]);
            }
        }
        if (!Minv) {
            if (r < bsz) z[(size_t)i * bsz + r] = s;
            continue;
        }
        __syncthreads();
        if (r < bsz) y[r] = s;
        __syncthreads();
        if (r < bsz) {
            const MT* m = Minv + (size_t)i * bsz * bsz;
            double t = 0.0;
            for (int c = 0; c < bsz; c++) t += (double)m[r + bsz * c] * y[c];
            z[(size_t)i * bsz + r] = t;
        }
    }
}

// z = M^-1 b (block-diagonal apply; MT = float: the FP32 preconditioner of the mixed mode).
template <typename MT>
__global__ void bj_apply_kernel(int nrows, int bsz, const MT* __restrict__ Minv, const double* __restrict__ b,
                                double* __restrict__ z) {
    const long long total = (long long)nrows * bsz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / bsz), r = (int)(t % bsz);
        const MT* m = Minv + (size_t)i * bsz * bsz;
        const double* bi = b + (size_t)i * bsz;
        double s = 0.0;
        for (int c = 0; c < bsz; c++) s += (double)m[r + bsz * c] * bi[c];
        z[t] = s;
    }
}

// FP32 copy of the block-Jacobi inverses (the mixed mode's preconditioner).
__global__ void to_float_kernel(long long n, const double* __restrict__ a, float* __restrict__ b) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

// Deterministic dot product: fixed grid of DOT_CTAS partial sums, then one CTA.
__global__ void dot_partial_kernel(long long n, const double* __restrict__ a, const double* __restrict__ b,
                                   double* __restrict__ part) {
    __shared__ double red[DOT_THREADS / 32];
    double s = 0.0;
    for (long long i = blockIdx.x * (long long)DOT_THREADS + threadIdx.x; i < n; i += (long long)DOT_CTAS * DOT_THREADS)
        s += a[i] * b[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < DOT_THREADS / 32; w++) t += red[w];
        part[blockIdx.x] = t;
    }
}

// out = sum(part); if sq, out = sqrt(out).  Also stores to out2 (may be NULL).
__global__ void dot_final_kernel(const double* __restrict__ part, double* out, int sq) {
    __shared__ double red[DOT_CTAS];
    for (int i = threadIdx.x; i < DOT_CTAS; i += blockDim.x) red[i] = part[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < DOT_CTAS; i++) t += red[i];
        *out = sq ? sqrt(t) : t;
    }
}

// y -= (*h) * x    (MGS projection with the coefficient read on the device)
__global__ void axpy_dev_kernel(long long n, const double* __restrict__ h, const double* __restrict__ x,
                                double* __restrict__ y) {
    const double a = *h;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] -= a * x[i];
}

// y = x / (*nrm) when *nrm != 0   (Arnoldi normalisation; y may alias x)
__global__ void scale_dev_kernel(long long n, const double* __restrict__ nrm, const double* x, double* y) {
    const double d = *nrm;
    if (d == 0.0) return;
    const double inv = 1.0 / d;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = x[i] * inv;
}

// r = b - r ; used for the initial residual
__global__ void sub_from_kernel(long long n, const double* __restrict__ b, double* __restrict__ r) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        r[i] = b[i] - r[i];
}

// x += V y  (y on the device, k columns of stride n)
__global__ void combine_kernel(long long n, int k, const double* __restrict__ V, const double* __restrict__ y,
                               double* __restrict__ x) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < k; j++) s += V[(size_t)j * n + i] * y[j];
        x[i] += s;
    }
}

}  // namespace hfem
