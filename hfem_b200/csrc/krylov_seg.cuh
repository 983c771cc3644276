// Krylov kernels for several independent systems packed into one vector
// (sm_100a): each problem's trace unknowns form one contiguous segment, and
// every reduction is per segment, so one launch advances the GMRES of every
// problem while each keeps its own Arnoldi basis, Hessenberg matrix and
// convergence test (the per-problem algorithm of kernel/gmres_bilu0.m:17-105).
//
// A segment is cut into pieces of at most SEG_PIECE entries, one CTA each
// (the host picks the piece length so that there are a few CTAs per SM).
// Reductions are deterministic: a CTA reduces its piece in a fixed tree, and
// the last CTA of a segment to finish (counted with an atomic ticket, the
// threadfence-reduction pattern; nothing waits) sums the segment's piece
// partials in piece order and resets the ticket.
#pragma once
#include <cuda_runtime.h>

namespace hfem {

constexpr int SEG_PIECE = 8192;
constexpr int SEG_THREADS = 256;

struct SegPieces {
    int npieces;
    const long long* pstart;   // npieces + 1 entry offsets
    const int* pseg;           // segment of each piece
    const int* seg_p0;         // first piece of each segment (nseg + 1)
    int* ticket;               // per segment, zero between launches
    double* part;              // per piece partial sums
    const unsigned char* act;  // per segment: 0 = skip
};

__device__ __forceinline__ double seg_block_sum(double s, double* red) {
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < SEG_THREADS / 32; w++) t += red[w];
    return t;   // valid in thread 0
}

// Finish a per-segment reduction: thread 0 of every CTA holds its piece sum.
__device__ __forceinline__ void seg_finish(const SegPieces& P, int piece, int seg, double s, double* out, int sq,
                                           double* red) {
    __shared__ int last;
    if (threadIdx.x == 0) {
        P.part[piece] = s;
        __threadfence();
        const int need = P.seg_p0[seg + 1] - P.seg_p0[seg];
        last = (atomicAdd(&P.ticket[seg], 1) == need - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int p0 = P.seg_p0[seg], p1 = P.seg_p0[seg + 1];
    double t = 0.0;
    for (int k = p0 + threadIdx.x; k < p1; k += SEG_THREADS) t += __ldcg(&P.part[k]);
    t = seg_block_sum(t, red);
    if (threadIdx.x == 0) {
        out[seg] = sq ? sqrt(t) : t;
        P.ticket[seg] = 0;
    }
}

// One modified Gram-Schmidt step fused with the next projection:
//   w -= hprev[seg] * vprev       (skipped when hprev == NULL)
//   out[seg] = <b, w>             (sqrt when sq; b may alias w for the norm)
__global__ void __launch_bounds__(SEG_THREADS) seg_axpy_dot_kernel(SegPieces P, const double* __restrict__ hprev,
                                                                   const double* __restrict__ vprev, double* w,
                                                                   const double* b, double* __restrict__ out,
                                                                   int sq) {
    __shared__ double red[SEG_THREADS / 32];
    const int piece = blockIdx.x;
    const int seg = P.pseg[piece];
    if (P.act && !P.act[seg]) return;
    const long long i0 = P.pstart[piece], i1 = P.pstart[piece + 1];
    double s = 0.0;
    if (hprev) {
        const double a = hprev[seg];
        for (long long i = i0 + threadIdx.x; i < i1; i += SEG_THREADS) {
            const double v = w[i] - a * vprev[i];
            w[i] = v;
            s += b[i] * v;
        }
    } else {
        for (long long i = i0 + threadIdx.x; i < i1; i += SEG_THREADS) s += b[i] * w[i];
    }
    s = seg_block_sum(s, red);
    seg_finish(P, piece, seg, s, out, sq, red);
}

// Classical Gram-Schmidt projections, all at once:
//   out[i * nseg + seg] = <V_i, w>  for i < k   (V_i: column i of stride n)
// Each CTA keeps its piece of w in registers (SEG_PIECE / SEG_THREADS per
// thread), reduces the k piece partials in a fixed tree into part[i * npieces +
// piece], and the last CTA of the segment sums them in piece order.
__global__ void __launch_bounds__(SEG_THREADS) seg_multidot_kernel(SegPieces P, long long n, int k, int nseg,
                                                                   const double* __restrict__ V,
                                                                   const double* __restrict__ w,
                                                                   double* __restrict__ partk,
                                                                   double* __restrict__ out) {
    constexpr int R = SEG_PIECE / SEG_THREADS;
    __shared__ double red[SEG_THREADS / 32];
    __shared__ int last;
    const int piece = blockIdx.x;
    const int seg = P.pseg[piece];
    if (P.act && !P.act[seg]) return;
    const long long i0 = P.pstart[piece], i1 = P.pstart[piece + 1];
    double wr[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
        const long long idx = i0 + threadIdx.x + (long long)SEG_THREADS * r;
        wr[r] = idx < i1 ? w[idx] : 0.0;
    }
    for (int i = 0; i < k; i++) {
        const double* vi = V + (size_t)i * n;
        double s = 0.0;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const long long idx = i0 + threadIdx.x + (long long)SEG_THREADS * r;
            if (idx < i1) s += vi[idx] * wr[r];
        }
        s = seg_block_sum(s, red);
        if (threadIdx.x == 0) partk[(size_t)i * P.npieces + piece] = s;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        const int need = P.seg_p0[seg + 1] - P.seg_p0[seg];
        last = (atomicAdd(&P.ticket[seg], 1) == need - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int p0 = P.seg_p0[seg], p1 = P.seg_p0[seg + 1];
    for (int i = 0; i < k; i++) {
        double t = 0.0;
        for (int q = p0 + threadIdx.x; q < p1; q += SEG_THREADS) t += __ldcg(&partk[(size_t)i * P.npieces + q]);
        t = seg_block_sum(t, red);
        if (threadIdx.x == 0) out[(size_t)i * nseg + seg] = t;
    }
    if (threadIdx.x == 0) P.ticket[seg] = 0;
}

// w -= sum_{i<k} h[i * nseg + seg] V_i, and with nrm != NULL also
// nrm[seg] = |w| after the update (per-segment reduction as above).
__global__ void __launch_bounds__(SEG_THREADS) seg_update_kernel(SegPieces P, long long n, int k, int nseg,
                                                                 const double* __restrict__ V,
                                                                 const double* __restrict__ h, double* w,
                                                                 double* __restrict__ nrm) {
    __shared__ double red[SEG_THREADS / 32];
    __shared__ double hs[64];
    const int piece = blockIdx.x;
    const int seg = P.pseg[piece];
    if (P.act && !P.act[seg]) return;
    for (int i = threadIdx.x; i < k; i += SEG_THREADS) hs[i] = h[(size_t)i * nseg + seg];
    __syncthreads();
    const long long i0 = P.pstart[piece], i1 = P.pstart[piece + 1];
    double s = 0.0;
    for (long long idx = i0 + threadIdx.x; idx < i1; idx += SEG_THREADS) {
        double a = 0.0;
        for (int i = 0; i < k; i++) a += hs[i] * V[(size_t)i * n + idx];
        const double v = w[idx] - a;
        w[idx] = v;
        s += v * v;
    }
    if (!nrm) return;
    s = seg_block_sum(s, red);
    seg_finish(P, piece, seg, s, nrm, 1, red);
}

// y = x / nrm[seg] where nrm[seg] != 0 (y may alias x).
__global__ void __launch_bounds__(SEG_THREADS) seg_scale_kernel(SegPieces P, const double* __restrict__ nrm,
                                                                const double* x, double* y) {
    const int piece = blockIdx.x;
    const int seg = P.pseg[piece];
    if (P.act && !P.act[seg]) return;
    const double d = nrm[seg];
    if (d == 0.0) return;
    const double inv = 1.0 / d;
    for (long long i = P.pstart[piece] + threadIdx.x; i < P.pstart[piece + 1]; i += SEG_THREADS) y[i] = x[i] * inv;
}

// x += sum_{j<kseg[seg]} V_j y[seg * ldy + j]   (columns of stride n)
__global__ void __launch_bounds__(SEG_THREADS) seg_combine_kernel(SegPieces P, long long n, const int* __restrict__ kseg,
                                                                  int ldy, const double* __restrict__ V,
                                                                  const double* __restrict__ y,
                                                                  double* __restrict__ x) {
    const int piece = blockIdx.x;
    const int seg = P.pseg[piece];
    if (P.act && !P.act[seg]) return;
    const int k = kseg[seg];
    const double* ys = y + (size_t)seg * ldy;
    for (long long i = P.pstart[piece] + threadIdx.x; i < P.pstart[piece + 1]; i += SEG_THREADS) {
        double s = 0.0;
        for (int j = 0; j < k; j++) s += V[(size_t)j * n + i] * ys[j];
        x[i] += s;
    }
}

// r = b - r on active segments
__global__ void __launch_bounds__(SEG_THREADS) seg_sub_from_kernel(SegPieces P, const double* __restrict__ b,
                                                                   double* __restrict__ r) {
    const int piece = blockIdx.x;
    const int seg = P.pseg[piece];
    if (P.act && !P.act[seg]) return;
    for (long long i = P.pstart[piece] + threadIdx.x; i < P.pstart[piece + 1]; i += SEG_THREADS) r[i] = b[i] - r[i];
}

// z = M^-1 (Hg x) with one warp per block row.  A row's blocks are contiguous
// in Hg, so the row is one column-major BSZ x (nblk * BSZ) matrix; the warp's
// lanes form G = 32 / BSZ column groups of BSZ rows (R = 2 rows per lane when
// BSZ > 32), and the groups' partial sums are added in group order.  Rows of
// inactive segments (act[rseg[i]] == 0) are skipped.
template <int BSZ, typename MT>
__global__ void __launch_bounds__(256) bsr_matvec_warp_kernel(int nrows, const int* __restrict__ rowstart,
                                                              const int* __restrict__ colidx,
                                                              const double* __restrict__ Hg,
                                                              const MT* __restrict__ Minv,
                                                              const double* __restrict__ x, double* __restrict__ z,
                                                              const int* __restrict__ rseg,
                                                              const unsigned char* __restrict__ act) {
    constexpr int G = BSZ <= 32 ? 32 / BSZ : 1;
    constexpr int R = (BSZ + 31) / 32;
    constexpr int LDY = R * 32;
    // even block sizes up to 32: a lane reads two rows of a column as one
    // 16-byte load, BSZ / 2 lanes per column and G2 columns at a time (2D p=2:
    // 0.91 -> 0.66 ms per 62 products; for BSZ = 50 the 25 busy lanes of this
    // form were slower than two 8-byte loads per lane)
    constexpr bool PAIRS = BSZ % 2 == 0 && BSZ <= 32;
    constexpr int L2 = PAIRS ? BSZ / 2 : 1;
    constexpr int G2 = PAIRS ? 32 / L2 : 1;
    constexpr int GY = PAIRS ? G2 : G;
    __shared__ double ys[8][GY][LDY];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int g = BSZ <= 32 ? lane / BSZ : 0;
    const int r0 = BSZ <= 32 ? lane % BSZ : lane;
    const bool on = g < G;
    const int nwarps = gridDim.x * 8;
    for (int i = blockIdx.x * 8 + wib; i < nrows; i += nwarps) {
        if (act && !act[rseg[i]]) continue;
        const int k0 = rowstart[i], k1 = rowstart[i + 1];
        const int ncol = (k1 - k0) * BSZ;
        const double* A = Hg + (size_t)k0 * BSZ * BSZ;
        double acc[R];
#pragma unroll
        for (int t = 0; t < R; t++) acc[t] = 0.0;
        if constexpr (PAIRS) {
            const int g2 = lane / L2, q = lane - g2 * L2;
            if (g2 < G2) {
                double a0 = 0.0, a1 = 0.0;
#pragma unroll 4
                for (int cc = g2; cc < ncol; cc += G2) {
                    const int kb = cc / BSZ, c = cc - kb * BSZ;
                    const double xv = __ldg(&x[(size_t)colidx[k0 + kb] * BSZ + c]);
                    const double2 av = __ldg(reinterpret_cast<const double2*>(A + (size_t)cc * BSZ) + q);
                    a0 += av.x * xv;
                    a1 += av.y * xv;
                }
                ys[wib][g2][2 * q] = a0;
                ys[wib][g2][2 * q + 1] = a1;
            }
        } else if (on) {
#pragma unroll 4
            for (int cc = g; cc < ncol; cc += G) {
                const int kb = cc / BSZ, c = cc - kb * BSZ;
                const double xv = __ldg(&x[(size_t)colidx[k0 + kb] * BSZ + c]);
#pragma unroll
                for (int t = 0; t < R; t++) {
                    const int r = r0 + 32 * t;
                    if (r < BSZ) acc[t] += __ldg(&A[(size_t)cc * BSZ + r]) * xv;
                }
            }
#pragma unroll
            for (int t = 0; t < R; t++) {
                const int r = r0 + 32 * t;
                if (r < BSZ) ys[wib][g][r] = acc[t];
            }
        }
        __syncwarp();
        double y[R];
#pragma unroll
        for (int t = 0; t < R; t++) {
            const int r = lane + 32 * t;
            double s = 0.0;
            if (r < BSZ)
#pragma unroll
                for (int gg = 0; gg < GY; gg++) s += ys[wib][gg][r];
            y[t] = s;
        }
        __syncwarp();
        if (!Minv) {
#pragma unroll
            for (int t = 0; t < R; t++) {
                const int r = lane + 32 * t;
                if (r < BSZ) z[(size_t)i * BSZ + r] = y[t];
            }
            continue;
        }
#pragma unroll
        for (int t = 0; t < R; t++) {
            const int r = lane + 32 * t;
            if (r < BSZ) ys[wib][0][r] = y[t];
        }
        __syncwarp();
        const MT* m = Minv + (size_t)i * BSZ * BSZ;
#pragma unroll
        for (int t = 0; t < R; t++) {
            const int r = lane + 32 * t;
            if (r < BSZ) {
                double s = 0.0;
#pragma unroll 4
                for (int c = 0; c < BSZ; c++) s += (double)__ldg(&m[(size_t)c * BSZ + r]) * ys[wib][0][c];
                z[(size_t)i * BSZ + r] = s;
            }
        }
        __syncwarp();
    }
}


// ---- GMRES bookkeeping on the device (one thread per problem), so that the
// host enqueues Arnoldi steps without reading every Hessenberg column back.
// Per problem p: H ((restart + 1) x restart, column-major), Givens cosines and
// sines (restart), g (restart + 1), the rhs norm nrmb, state (2 running,
// 1 converged, 0 iteration limit, -1 breakdown), iterations, the cycle's step
// count jc, and act (the segment mask every segment kernel reads).
struct GmState {
    int P, restart, maxit;
    double tol;
    double *H, *cs, *sn, *g, *nrmb;
    int *state, *its, *jc;
    unsigned char* act;
    double* hist;               // problem 0's relative residual per iteration (hist_len entries) or NULL
    int hist_len;
};

__global__ void gm_init_kernel(GmState S, const double* __restrict__ nrm) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= S.P) return;
    S.nrmb[p] = nrm[p] == 0.0 ? 1.0 : nrm[p];
    S.state[p] = 2;
    S.its[p] = 0;
}

// the mask of the problems still running
__global__ void gm_running_kernel(GmState S) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < S.P) S.act[p] = S.state[p] == 2;
}

// start of a restart cycle: beta = |r| per problem (nrm)
__global__ void gm_cycle_kernel(GmState S, const double* __restrict__ nrm) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= S.P) return;
    S.jc[p] = 0;
    unsigned char a = 0;
    if (S.state[p] == 2) {
        if (nrm[p] / S.nrmb[p] <= S.tol) {
            S.state[p] = 1;
        } else {
            a = 1;
            double* gp = S.g + (size_t)(S.restart + 1) * p;
            gp[0] = nrm[p];
            for (int i = 1; i <= S.restart; i++) gp[i] = 0.0;
        }
    }
    S.act[p] = a;
}

// Arnoldi step j: the new Hessenberg column (h, plus h2 for the second CGS
// projection), the previous rotations applied, the new rotation, the residual
// estimate and the stopping test (kernel/gmres_bilu0.m:17-105)
__global__ void gm_givens_kernel(GmState S, int j, const double* __restrict__ h, const double* __restrict__ h2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= S.P || !S.act[p]) return;
    const int R = S.restart, P = S.P;
    double* hc = S.H + (size_t)(R + 1) * R * p + (size_t)(R + 1) * j;
    double* cp = S.cs + (size_t)R * p;
    double* sp = S.sn + (size_t)R * p;
    double* gp = S.g + (size_t)(R + 1) * p;
    for (int i = 0; i <= j + 1; i++) hc[i] = h[(size_t)i * P + p] + ((h2 && i <= j) ? h2[(size_t)i * P + p] : 0.0);
    const double nn = h[(size_t)(j + 1) * P + p];
    for (int i = 0; i < j; i++) {
        const double a = hc[i], b = hc[i + 1];
        hc[i] = cp[i] * a + sp[i] * b;
        hc[i + 1] = -sp[i] * a + cp[i] * b;
    }
    const double a = hc[j], b = hc[j + 1];
    const double rr = sqrt(a * a + b * b);
    cp[j] = a / rr;
    sp[j] = b / rr;
    hc[j] = rr;
    hc[j + 1] = 0.0;
    gp[j + 1] = -sp[j] * gp[j];
    gp[j] = cp[j] * gp[j];
    const int it = ++S.its[p];
    S.jc[p] = j + 1;
    const double res = fabs(gp[j + 1]);
    if (p == 0 && S.hist && it - 1 < S.hist_len) S.hist[it - 1] = res / S.nrmb[0];
    int stop = 2;
    if (res / S.nrmb[p] <= S.tol) stop = 1;
    else if (it >= S.maxit) stop = 0;
    else if (nn == 0.0) stop = -1;
    if (stop != 2) {
        S.state[p] = stop;
        S.act[p] = 0;
    }
}

// end of a cycle: y = H^-1 g by back substitution for every problem that took
// steps, its step count and mask for the combination x += V y
__global__ void gm_solve_kernel(GmState S, double* __restrict__ y, int* __restrict__ kseg) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= S.P) return;
    const int R = S.restart, J = S.jc[p];
    S.act[p] = J > 0;
    kseg[p] = J;
    const double* hp = S.H + (size_t)(R + 1) * R * p;
    const double* gp = S.g + (size_t)(R + 1) * p;
    double* yp = y + (size_t)R * p;
    for (int i = J - 1; i >= 0; i--) {
        double s = gp[i];
        for (int k = i + 1; k < J; k++) s -= hp[i + (R + 1) * k] * yp[k];
        yp[i] = s / hp[i + (R + 1) * i];
    }
}

}  // namespace hfem
