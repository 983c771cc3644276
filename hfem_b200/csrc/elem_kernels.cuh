// Shared pieces of the HDG element kernels for sm_100a: element shapes and
// arguments, geometry and q-equation matrices, the Cholesky helpers, the
// face-block scatter, the residual norm, q recovery and the solution update.
// The element assembly itself is element_kernel (elem_kernel.cuh).
//
// Structure of the element blocks (restating elementassembly.cpp faceint
// 717-1321): every face contribution to the element equations is the
// trace-equation entry lifted to the element node that carries the face dof,
//   D = D_vol + P K,   F = F_vol + P H,   Ru = Ru_vol + P Rh,
// where P (npv x ndf) is the incidence perm[fdof] = node.
#pragma once
#include <cuda_runtime.h>
#include "ns_flux.cuh"

namespace hfem {

template <int ND_, int NPV_, int NPF_, int NGV_, int NGF_>
struct Shape {
    static constexpr int ND = ND_, NPV = NPV_, NPF = NPF_, NGV = NGV_, NGF = NGF_;
    static constexpr int NFE = ND + 1, NCU = ND + 2, NC = NCU * (ND + 1), NCH = NCU;
    static constexpr int NDF = NPF * NFE, ND1 = ND + 1, N = NPV * NCU, NB = NCH * NDF, BSZ = NCH * NPF;
    static constexpr int NA = NGF * NFE;          // face points of one element
    static constexpr int NQ = NGV * ND1;          // (volume point, derivative) pairs
    static constexpr int MAXINC = ND;             // faces meeting at a node
};

struct Tables {                 // master element tables, reference layouts
    const double *shapvt, *shapvg, *svsv, *shapft, *shapfg, *sfsf;
    const int* perm;            // nfe x npf
};

struct ElemArgs {
    Tables T;
    const double* dgnodes;      // ne x nd x npv
    const int* elcon;           // ne x ndf
    const double *udg, *uh, *sh;
    double param[6];
    int tdep;
    double fc_u, fc_q;
    int ne;
    double *D, *F, *K, *H, *Ru, *Rh, *Ro, *ru2;
    double* ws;                 // gridDim.x workspace slots of EK<S>::WS doubles (element_kernel)
    // several problems in one mesh (NULL = the uniform values above): element ->
    // problem, and per problem [gamma, eps, Re, Pr, Mach, tau, tdep, fc_u]
    const int* eprob;
    const double* pparam;
    // boundary faces (NULL bf = none): bf[e * nfe + face] < 0 is boundary -(ib + 1),
    // condition bcm[ib] (fbou.cpp types 1, 2, 5, 6, 7) with state bcs[ib * nch + c]
    const int* bf;
    const int* bcm;
    const double* bcs;
    int inviscid;               // 1: Euler flux (app.appname 0)
    int* err = nullptr;         // set to 2 when a bulk-copy wait expires (NULL: not recorded)
    int conv_stab = 0;          // app.convStabMethod: 0 constant tau, 1 Lax-Friedrichs, 2 Roe
    int visc_model = 0;         // app.viscosityModel: 0 constant, 1 Sutherland's law
    int e_begin = 0;            // element range [e_begin, ne) of this launch
};

constexpr int NT = 256;         // threads per CTA for element kernels

// --------------------------------------------------------------- helpers
__device__ __forceinline__ double block_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += red[i];
    return s;                   // valid on thread 0
}

// Geometry at volume and face points (elementassembly.cpp:11-237).
template <class S>
__device__ void geometry(const Tables& T, const double* x, double* jac, double* Xx, double* jacf, double* nl) {
    constexpr int ND = S::ND, NPV = S::NPV, NGV = S::NGV, NGF = S::NGF, NPF = S::NPF, NA = S::NA;
    for (int g = threadIdx.x; g < NGV + NA; g += blockDim.x) {
        if (g < NGV) {
            double J[ND][ND];
#pragma unroll
            for (int d = 0; d < ND; d++)
#pragma unroll
                for (int i = 0; i < ND; i++) {
                    double s = 0.0;
                    for (int a = 0; a < NPV; a++) s += T.shapvt[g + NGV * (a + NPV * (i + 1))] * x[a + NPV * d];
                    J[d][i] = s;
                }
            double adj[ND][ND], det;
            if constexpr (ND == 2) {
                det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
                adj[0][0] = J[1][1]; adj[0][1] = -J[0][1];
                adj[1][0] = -J[1][0]; adj[1][1] = J[0][0];
            } else {
                adj[0][0] = J[1][1] * J[2][2] - J[1][2] * J[2][1];
                adj[0][1] = J[0][2] * J[2][1] - J[0][1] * J[2][2];
                adj[0][2] = J[0][1] * J[1][2] - J[0][2] * J[1][1];
                adj[1][0] = J[1][2] * J[2][0] - J[1][0] * J[2][2];
                adj[1][1] = J[0][0] * J[2][2] - J[0][2] * J[2][0];
                adj[1][2] = J[0][2] * J[1][0] - J[0][0] * J[1][2];
                adj[2][0] = J[1][0] * J[2][1] - J[1][1] * J[2][0];
                adj[2][1] = J[0][1] * J[2][0] - J[0][0] * J[2][1];
                adj[2][2] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
                det = J[0][0] * adj[0][0] + J[0][1] * adj[1][0] + J[0][2] * adj[2][0];
            }
            jac[g] = det;
#pragma unroll
            for (int d = 0; d < ND; d++)
#pragma unroll
                for (int i = 0; i < ND; i++) Xx[g + NGV * (d + ND * i)] = adj[i][d];
        } else {
            const int gg = g - NGV, fc = gg / NGF, q = gg % NGF;
            double Tt[ND][ND - 1];
#pragma unroll
            for (int d = 0; d < ND; d++)
#pragma unroll
                for (int r = 0; r < ND - 1; r++) {
                    double s = 0.0;
                    for (int m = 0; m < NPF; m++)
                        s += T.shapft[q + NGF * (m + NPF * (r + 1))] * x[T.perm[fc * NPF + m] + NPV * d];
                    Tt[d][r] = s;
                }
            double nv[ND];
            if constexpr (ND == 2) {
                nv[0] = Tt[1][0];
                nv[1] = -Tt[0][0];
            } else {
                nv[0] = Tt[1][0] * Tt[2][1] - Tt[2][0] * Tt[1][1];
                nv[1] = Tt[2][0] * Tt[0][1] - Tt[0][0] * Tt[2][1];
                nv[2] = Tt[0][0] * Tt[1][1] - Tt[1][0] * Tt[0][1];
            }
            double j = 0.0;
#pragma unroll
            for (int d = 0; d < ND; d++) j += nv[d] * nv[d];
            j = sqrt(j);
            jacf[gg] = j;
#pragma unroll
            for (int d = 0; d < ND; d++) nl[gg + NA * d] = nv[d] / j;
        }
    }
}

// q-equation matrices (elementassembly.cpp:1323-1412): M (npv^2), C (npv^2 nd), E (npv ndf nd).
template <class S>
__device__ void qmatrices(const Tables& T, double fc_q, const double* jac, const double* Xx, const double* jacf,
                          const double* nl, double* M, double* C, double* E) {
    constexpr int ND = S::ND, NPV = S::NPV, NGV = S::NGV, NGF = S::NGF, NPF = S::NPF, NA = S::NA, NDF = S::NDF;
    constexpr int NPV2 = NPV * NPV, NPF2 = NPF * NPF;
    for (int t = threadIdx.x; t < NPV2 * (ND + 1); t += blockDim.x) {
        const int r = t % NPV2, d = t / NPV2;
        if (d == 0) {
            double s = 0.0;
            for (int g = 0; g < NGV; g++) s += T.svsv[r + NPV2 * g] * jac[g];
            M[r] = fc_q * s;
        } else {
            double c = 0.0;
            for (int i = 0; i < ND; i++)
                for (int g = 0; g < NGV; g++)
                    c += T.svsv[r + NPV2 * (g + NGV * (i + 1))] * Xx[g + NGV * ((d - 1) + ND * i)];
            C[r + NPV2 * (d - 1)] = c;
        }
    }
    for (int t = threadIdx.x; t < NPV * NDF * ND; t += blockDim.x) E[t] = 0.0;
    __syncthreads();
    for (int t = threadIdx.x; t < ND * NDF * NPF; t += blockDim.x) {
        const int k = t % NPF, j = (t / NPF) % NPF, fc = (t / NPF2) % S::NFE, d = t / (NPF2 * S::NFE);
        double s = 0.0;
        for (int g = 0; g < NGF; g++)
            s += T.sfsf[(k + NPF * j) + NPF2 * g] * nl[g + NGF * fc + NA * d] * jacf[g + NGF * fc];
        E[T.perm[fc * NPF + k] + NPV * ((fc * NPF + j) + NDF * d)] = s;
    }
}

// Lower Cholesky of M (npv x npv) in place, one warp; rdg (if given) receives
// the reciprocals of the diagonal.
template <int NPV>
__device__ void cholesky_warp(double* a, double* rdg = nullptr) {
    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    for (int j = 0; j < NPV; j++) {
        if (lane == 0) {
            double s = a[j + NPV * j];
            for (int k = 0; k < j; k++) s -= a[j + NPV * k] * a[j + NPV * k];
            a[j + NPV * j] = sqrt(s);
            if (rdg) rdg[j] = 1.0 / a[j + NPV * j];
        }
        __syncwarp();
        const double djj = a[j + NPV * j];
        for (int i = j + 1 + lane; i < NPV; i += 32) {
            double t = a[i + NPV * j];
            for (int k = 0; k < j; k++) t -= a[i + NPV * k] * a[j + NPV * k];
            a[i + NPV * j] = t / djj;
        }
        __syncwarp();
    }
}

template <int NPV>
__device__ __forceinline__ void chol_solve_col(const double* l, double* x) {
    for (int i = 0; i < NPV; i++) {
        double t = x[i];
        for (int k = 0; k < i; k++) t -= l[i + NPV * k] * x[k];
        x[i] = t / l[i + NPV * i];
    }
    for (int i = NPV - 1; i >= 0; i--) {
        double t = x[i];
        for (int k = i + 1; k < NPV; k++) t -= l[k + NPV * i] * x[k];
        x[i] = t / l[i + NPV * i];
    }
}

// --------------------------------------------------------------- scatter
// Owner-gather into the face-block system (globalassembly.cpp:40-89): every
// Hg entry sums its (at most two) element contributions in ascending element
// order, exactly the order of the reference's serial element loop.
struct ScatterArgs {
    int nblk, nf, npf, nch, nfe, nb;
    const int* blk_src;        // nblk x 2 x 3: (element, a, b) or -1
    const int* face_src;       // nf x 2 x 2: (element, a) or -1
    const int* elcon;          // ne x ndf
    const int* rowface;        // nblk: row face i of block k
    const int* colface;        // nblk: column face j of block k
    const double *H, *Rh, *Ro;
    double *Hg, *Rg, *Rr;
};

// Scatter of the condensed blocks into Hg (mapElement2LinearSystem,
// globalassembly.cpp:40-89) as an owner-gather, one warp per Hg block, face shape known
// at compile time: the warp first resolves, for each (at most two)
// contributing element, the offsets of the block's rows and columns inside
// that element's H (elcon gives the permutation of the face nodes), then
// streams the block's entries in Hg order (rows fastest, coalesced stores).
template <int NPF, int NCH, int NFE>
__global__ void __launch_bounds__(256) scatter_H_block_kernel(ScatterArgs A) {
    constexpr int BSZ = NPF * NCH, NDF = NPF * NFE, NB = NDF * NCH;
    constexpr int WARPS = 8;
    __shared__ long long s_col[WARPS][2][NPF];
    __shared__ int s_row[WARPS][2][NPF];
    __shared__ long long s_base[WARPS][2];
    __shared__ int s_n[WARPS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = blockIdx.x * WARPS + w; k < A.nblk; k += gridDim.x * WARPS) {
        const int i = A.rowface[k], j = A.colface[k];
        if (lane == 0) {
            int n = 0;
            for (int c = 0; c < 2; c++) {
                const int e = A.blk_src[(k * 2 + c) * 3 + 0];
                if (e < 0) break;
                s_base[w][c] = (long long)e * NB * NB;
                n++;
            }
            s_n[w] = n;
        }
        for (int t = lane; t < 2 * 2 * NPF; t += 32) {
            const int c = t / (2 * NPF), r = t % (2 * NPF), m = r % NPF, isc = r / NPF;
            const int e = A.blk_src[(k * 2 + c) * 3 + 0];
            if (e < 0) continue;
            const int a = A.blk_src[(k * 2 + c) * 3 + 1], b = A.blk_src[(k * 2 + c) * 3 + 2];
            if (!isc) {
                const int ind = A.elcon[(size_t)e * NDF + a * NPF + m] - i * NPF;
                s_row[w][c][m] = a * BSZ + ind * NCH;
            } else {
                const int jnd = A.elcon[(size_t)e * NDF + b * NPF + m] - j * NPF;
                s_col[w][c][m] = (long long)NB * (b * BSZ + jnd * NCH);
            }
        }
        __syncwarp();
        const int n = s_n[w];
        double* out = A.Hg + (size_t)k * BSZ * BSZ;
        for (int t = lane; t < BSZ * BSZ; t += 32) {
            const int colpos = t / BSZ, rowpos = t - colpos * BSZ;
            const int m1 = colpos / NCH, n1 = colpos - m1 * NCH, m2 = rowpos / NCH, n2 = rowpos - m2 * NCH;
            double s = 0.0;
            for (int c = 0; c < n; c++)
                s += A.H[s_base[w][c] + s_row[w][c][m2] + n2 + s_col[w][c][m1] + (long long)NB * n1];
            out[t] = s;
        }
        __syncwarp();
    }
}

__global__ void scatter_R_kernel(ScatterArgs A) {
    const int bsz = A.npf * A.nch, ndf = A.npf * A.nfe;
    const int total = A.nf * bsz;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const int i = t / bsz, w = t % bsz, m1 = w / A.nch, n1 = w % A.nch;
        double s = 0.0, so = 0.0;
        for (int c = 0; c < 2; c++) {
            const int e = A.face_src[(i * 2 + c) * 2 + 0];
            if (e < 0) break;
            const int a = A.face_src[(i * 2 + c) * 2 + 1];
            const int ind = A.elcon[(size_t)e * ndf + a * A.npf + m1] - i * A.npf;
            const size_t idx = (size_t)e * A.nb + a * bsz + ind * A.nch + n1;
            s += A.Rh[idx];
            if (A.Ro) so += A.Ro[idx];
        }
        if (A.Rg) A.Rg[t] = s;
        if (A.Rr) A.Rr[t] = so;
    }
}

// Partial sums of ru2 and Rr^2 per CTA (fixed grid-stride order).
__global__ void rnorm_partial_kernel(int ne, const double* __restrict__ ru2, long long nr,
                                     const double* __restrict__ rr, double* __restrict__ part) {
    __shared__ double red[32];
    double s = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ne; i += stride) s += ru2[i];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nr; i += stride) s += rr[i] * rr[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
        part[blockIdx.x] = t;
    }
}

// out = sqrt(sum of the n partial sums), in order.
__global__ void rnorm_final_kernel(int n, const double* __restrict__ part, double* out) {
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < n; i++) t += part[i];
        *out = sqrt(t);
    }
}

// ------------------------------------------------------ q recovery / update
struct QArgs {
    Tables T;
    const double* dgnodes;
    const int* elcon;
    double* udg;                // u read, q written
    const double *uh, *sh;
    double fc_q;
    int ne;
    // optional update before the q solve: u += alpha (DinvRu - DinvF duh_e)
    const double *DinvRu, *DinvF, *duh;
    double alpha;
    const int* eprob;           // per-problem step lengths (NULL: alpha for all)
    const double* palpha;
};

template <class S>
struct QSmem {
    double x[S::NPV * S::ND];
    double jac[S::NGV], Xx[S::NGV * S::ND * S::ND];
    double jacf[S::NA], nl[S::NA * S::ND];
    double M[S::NPV * S::NPV];
    double C[S::NPV * S::NPV * S::ND];
    double E[S::NPV * S::NDF * S::ND];
    double u[S::NPV * S::NCU];
    double uhe[S::NDF * S::NCH];
    double de[S::NB];
    double q[S::NPV * S::NCU * S::ND];
};

// getQ (elementassembly.cpp:1414-1479), optionally preceded by getU (solutionupdate.cpp:6-68).
template <class S>
__global__ void __launch_bounds__(NT) getq_kernel(QArgs A) {
    constexpr int ND = S::ND, NPV = S::NPV, NCU = S::NCU, NC = S::NC, NCH = S::NCH, NDF = S::NDF, N = S::N, NB = S::NB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    QSmem<S>& sm = *reinterpret_cast<QSmem<S>*>(smem_raw);
    const int tid = threadIdx.x;
    for (int e = blockIdx.x; e < A.ne; e += gridDim.x) {
        __syncthreads();
        double* ue = A.udg + (size_t)e * NPV * NC;
        for (int t = tid; t < NPV * ND; t += NT) sm.x[t] = A.dgnodes[(size_t)e * NPV * ND + t];
        for (int t = tid; t < NDF * NCH; t += NT) {
            const int fn = t / NCH, c = t % NCH;
            const int gd = A.elcon[(size_t)e * NDF + fn];
            sm.uhe[fn + NDF * c] = A.uh[(size_t)gd * NCH + c];
            if (A.DinvF) sm.de[fn * NCH + c] = A.duh[(size_t)gd * NCH + c];
        }
        __syncthreads();
        const double alpha = A.palpha ? A.palpha[A.eprob[e]] : A.alpha;
        for (int t = tid; t < N; t += NT) {
            double v = ue[t];
            if (A.DinvF) {
                const double* df = A.DinvF + (size_t)e * N * NB;
                double s = 0.0;
                for (int c = 0; c < NB; c++) s += df[t + (size_t)N * c] * sm.de[c];
                v += -alpha * s;
                v += alpha * A.DinvRu[(size_t)e * N + t];
                ue[t] = v;
            }
            sm.u[t] = v;
        }
        geometry<S>(A.T, sm.x, sm.jac, sm.Xx, sm.jacf, sm.nl);
        __syncthreads();
        qmatrices<S>(A.T, A.fc_q, sm.jac, sm.Xx, sm.jacf, sm.nl, sm.M, sm.C, sm.E);
        __syncthreads();
        const double* she = A.sh + (size_t)e * NPV * NC;
        for (int t = tid; t < NPV * NCU * ND; t += NT) {
            const int i = t % NPV, c = (t / NPV) % NCU, d = t / (NPV * NCU);
            double s = 0.0;
            for (int a = 0; a < NPV; a++) s += sm.M[i + NPV * a] * she[a + NPV * (NCU * (1 + d) + c)];
            for (int a = 0; a < NPV; a++) s += sm.C[i + NPV * (a + NPV * d)] * sm.u[a + NPV * c];
            for (int fn = 0; fn < NDF; fn++) s -= sm.E[i + NPV * (fn + NDF * d)] * sm.uhe[fn + NDF * c];
            sm.q[t] = s;
        }
        __syncthreads();
        cholesky_warp<NPV>(sm.M);
        __syncthreads();
        for (int t = tid; t < NCU * ND; t += NT) chol_solve_col<NPV>(sm.M, &sm.q[NPV * t]);
        __syncthreads();
        for (int t = tid; t < NPV * NCU * ND; t += NT) {
            const int i = t % NPV, c = (t / NPV) % NCU, d = t / (NPV * NCU);
            ue[i + NPV * (NCU * (1 + d) + c)] = sm.q[t];
        }
    }
}

__global__ void axpy_kernel(long long n, double alpha, const double* x, double* y) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] += alpha * x[i];
}

// y += alpha[prob[i / per]] x  (per-problem step lengths on the trace unknowns)
__global__ void axpy_prob_kernel(long long n, int per, const int* __restrict__ prob, const double* __restrict__ alpha,
                                 const double* x, double* y) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] += alpha[prob[i / per]] * x[i];
}

}  // namespace hfem
