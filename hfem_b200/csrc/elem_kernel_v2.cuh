// Element assembly on the FP64 tensor cores (sm_100a, mma.sync m8n8k4 f64).
//
// Same outputs and phases as element_kernel up to the pointwise fluxes; every
// contraction after that is a small GEMM whose B operand is generated on the
// fly into shared memory (restating elementassembly.cpp elementint 307-572 and
// faceint 717-1321):
//   K_fc = shapfg (npf x ngf) * T_k,  T_k(q; j,m,a) = [a on fc] phi_kk(a)(q) fhn_u(q; j,m)
//                                               + sum_d fhn_u(q; j, q_dm) (phi M^-1 C_d)(q; a)
//   H_fc = shapfg * T_h,  T_h(q; j,m,f2) = [f2 on fc] phi_f2(q) fhn_uh(q; j,m)
//                                        - sum_d fhn_u(q; j, q_dm) (phi M^-1 E_d)(q; f2)
//   D_vol = shapvg (npv x ngv(nd+1)) * W,  W(g,r; j,a,k) = wrl(g,r; j,k) phi_a(g)
//                                               + sum_d wrl(g,r; j, q_dk) (phi M^-1 C_d)(g; a)
//   F_vol = shapvg * W_f,  W_f(g,r; j,k,f2) = sum_d wrl(g,r; j, q_dk) (-phi M^-1 E_d)(g; f2)
// followed by the lifted trace terms D = D_vol + P K, F = F_vol + P H.  The
// face mass product uses shapfgdotshapfc = shapfg .* shapfc (its definition,
// mkmasterelement.m:113-115) in factored form.
#pragma once
#include <cuda_runtime.h>
#include "elem_kernels.cuh"
#include "schur_kernels.cuh"

namespace hfem {

template <class S>
struct V2 {
    static constexpr int MTV = (S::NPV + 7) / 8;              // m-tiles of shapvg
    static constexpr int MTF = (S::NPF + 7) / 8;              // m-tiles of shapfg
    static constexpr int KV = ((S::NQ + 3) / 4) * 4;          // padded k of volume GEMMs
    static constexpr int KF = ((S::NGF + 3) / 4) * 4;         // padded k of face GEMMs
    static constexpr int LDAV = ((8 * MTV + 11) / 16) * 16 + 4;
    static constexpr int LDAF = ((8 * MTF + 11) / 16) * 16 + 4;
    static constexpr int LDBV = ((KV + 11) / 16) * 16 + 4;    // >= KV, == 4 (mod 16)
    static constexpr int LDBF = ((KF + 11) / 16) * 16 + 4;
    static constexpr int NTWV = 1, NTWF = 5;                  // n-tiles per warp (8 warps)
    static constexpr int CWV = 8 * NTWV * (NT / 32);          // chunk width, volume jobs
    static constexpr int CWF = 8 * NTWF * (NT / 32);          // chunk width, face jobs
    static constexpr int QSZ = S::NPV * S::NPV * (1 + S::ND) + S::NPV * S::NDF * S::ND + S::NGV * S::NC +
                               S::NA * (S::NC + S::NCH);
    static constexpr int BSZV = LDBV * CWV, BSZF = LDBF * CWF;
    static constexpr int UN = (QSZ > BSZV ? (QSZ > BSZF ? QSZ : BSZF) : (BSZV > BSZF ? BSZV : BSZF));
};

template <class S>
struct ElemSmemV2 {
    double x[S::NPV * S::ND];
    double u[S::NPV * S::NC];
    double uhe[S::NDF * S::NCH];
    double shu[S::NPV * S::NCU];
    double jac[S::NGV], Xx[S::NGV * S::ND * S::ND];
    double jacf[S::NA], nl[S::NA * S::ND];
    double wrk[S::NQ * S::NCU];
    double fn[S::NA * S::NCH];
    double Av[V2<S>::LDAV * V2<S>::KV];   // shapvg, zero padded: Av[i + LDAV*q]
    double Af[V2<S>::LDAF * V2<S>::KF];   // shapfg, zero padded: Af[ip + LDAF*q]
    double sfc[S::NGF * S::NPF];          // face basis values shapfc(kk, q) = shapft[q + NGF*kk]
    double red[NT / 32];
    double un[V2<S>::UN];                 // q-phase matrices, then the generated B chunks
    int perm[S::NDF];
    int inc_n[S::NPV];
    int inc_f[S::NPV * S::MAXINC];
    int pos[S::NFE * S::NPV];             // position of element node a on face fc, or -1
};

// acc(MT x NTW tiles) += A(8MT x 4KST, smem col-major lda) * B(4KST x 8 NTW*warps, smem col-major ldb)
template <int MT, int NTW, int KST>
__device__ __forceinline__ void chunk_mma(const double* As, int lda, const double* Bs, int ldb,
                                          double (&acc)[MT][NTW][2]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gr = lane >> 2, gc = lane & 3;
#pragma unroll 4
    for (int ks = 0; ks < KST; ks++) {
        double af[MT], bf[NTW];
#pragma unroll
        for (int a = 0; a < MT; a++) af[a] = As[(8 * a + gr) + lda * (4 * ks + gc)];
#pragma unroll
        for (int b = 0; b < NTW; b++) bf[b] = Bs[(4 * ks + gc) + ldb * (8 * (warp * NTW + b) + gr)];
#pragma unroll
        for (int a = 0; a < MT; a++)
#pragma unroll
            for (int b = 0; b < NTW; b++) dmma8x8x4(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
    }
}

template <class S>
__global__ void __launch_bounds__(NT, 2) element_kernel_v2(ElemArgs A) {
    constexpr int ND = S::ND, NPV = S::NPV, NPF = S::NPF, NGV = S::NGV, NGF = S::NGF, NFE = S::NFE;
    constexpr int NCU = S::NCU, NC = S::NC, NCH = S::NCH, NDF = S::NDF, ND1 = S::ND1, N = S::N, NB = S::NB;
    constexpr int NA = S::NA, NQ = S::NQ;
    using C2 = V2<S>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ElemSmemV2<S>& sm = *reinterpret_cast<ElemSmemV2<S>*>(smem_raw);
    const Tables& T = A.T;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gr = lane >> 2, gc = lane & 3;

    double* ws = A.ws + (size_t)blockIdx.x * S::WS;
    double* wrl = ws;
    double* sMiC = wrl + S::W_WRL;
    double* sMiE = sMiC + S::W_SMIC;
    double* sMiCf = sMiE + S::W_SMIE;
    double* sMiEf = sMiCf + S::W_SMICF;
    double* fnu = sMiEf + S::W_SMIEF;
    double* fnuh = fnu + S::W_FNU;

    // q-phase views into the union
    double* M = sm.un;
    double* Cm = M + NPV * NPV;
    double* Em = Cm + NPV * NPV * ND;
    double* ug = Em + NPV * NDF * ND;
    double* ugf = ug + NGV * NC;
    double* uhg = ugf + NA * NC;
    double* Bs = sm.un;

    for (int t = tid; t < C2::LDAV * C2::KV; t += NT) {
        const int i = t % C2::LDAV, q = t / C2::LDAV;
        sm.Av[t] = (i < NPV && q < NQ) ? T.shapvg[i + NPV * q] : 0.0;
    }
    for (int t = tid; t < C2::LDAF * C2::KF; t += NT) {
        const int i = t % C2::LDAF, q = t / C2::LDAF;
        sm.Af[t] = (i < NPF && q < NGF) ? T.shapfg[i + NPF * q] : 0.0;
    }
    for (int t = tid; t < NGF * NPF; t += NT) sm.sfc[t] = T.shapft[t];
    for (int t = tid; t < NDF; t += NT) sm.perm[t] = T.perm[t];
    __syncthreads();
    for (int i = tid; i < NPV; i += NT) {
        int c = 0;
        for (int f = 0; f < NDF; f++)
            if (sm.perm[f] == i && c < S::MAXINC) sm.inc_f[i * S::MAXINC + c++] = f;
        sm.inc_n[i] = c;
        for (int fc = 0; fc < NFE; fc++) {
            int p = -1;
            for (int kk = 0; kk < NPF; kk++)
                if (sm.perm[fc * NPF + kk] == i) p = kk;
            sm.pos[fc * NPV + i] = p;
        }
    }

    for (int e = blockIdx.x; e < A.ne; e += gridDim.x) {
        __syncthreads();
        const double* xg = A.dgnodes + (size_t)e * NPV * ND;
        const double* ugl = A.udg + (size_t)e * NPV * NC;
        const double* shg = A.sh + (size_t)e * NPV * NC;
        for (int t = tid; t < NPV * ND; t += NT) sm.x[t] = xg[t];
        for (int t = tid; t < NPV * NC; t += NT) sm.u[t] = ugl[t];
        for (int t = tid; t < NPV * NCU; t += NT) sm.shu[t] = shg[t];
        for (int t = tid; t < NDF * NCH; t += NT) {
            const int fn = t / NCH, c = t % NCH;
            sm.uhe[fn + NDF * c] = A.uh[(size_t)A.elcon[(size_t)e * NDF + fn] * NCH + c];
        }
        __syncthreads();
        geometry<S>(T, sm.x, sm.jac, sm.Xx, sm.jacf, sm.nl);
        __syncthreads();
        qmatrices<S>(T, A.fc_q, sm.jac, sm.Xx, sm.jacf, sm.nl, M, Cm, Em);
        for (int t = tid; t < NGV * NC; t += NT) {
            const int g = t % NGV, c = t / NGV;
            double s = 0.0;
            for (int a = 0; a < NPV; a++) s += T.shapvt[g + NGV * a] * sm.u[a + NPV * c];
            ug[t] = s;
        }
        for (int t = tid; t < NA * (NC + NCH); t += NT) {
            const int gg = t % NA, c = t / NA, fc = gg / NGF, q = gg % NGF;
            double s = 0.0;
            if (c < NC) {
                for (int m = 0; m < NPF; m++) s += sm.sfc[q + NGF * m] * sm.u[sm.perm[fc * NPF + m] + NPV * c];
                ugf[gg + NA * c] = s;
            } else {
                for (int m = 0; m < NPF; m++) s += sm.sfc[q + NGF * m] * sm.uhe[fc * NPF + m + NDF * (c - NC)];
                uhg[gg + NA * (c - NC)] = s;
            }
        }
        __syncthreads();
        cholesky_warp<NPV>(M);
        __syncthreads();
        for (int t = tid; t < NPV * ND + NDF * ND; t += NT) {
            double* col = (t < NPV * ND) ? &Cm[NPV * t] : &Em[NPV * (t - NPV * ND)];
            chol_solve_col<NPV>(M, col);
        }
        __syncthreads();
        for (int t = tid; t < NGV * NPV * ND; t += NT) {
            const int g = t % NGV, ad = t / NGV;
            double s = 0.0;
            for (int b = 0; b < NPV; b++) s += T.shapvt[g + NGV * b] * Cm[b + NPV * ad];
            sMiC[t] = s;
        }
        for (int t = tid; t < NGV * NDF * ND; t += NT) {
            const int g = t % NGV, fd = t / NGV;
            double s = 0.0;
            for (int b = 0; b < NPV; b++) s += T.shapvt[g + NGV * b] * Em[b + NPV * fd];
            sMiE[t] = -s;
        }
        for (int t = tid; t < NA * NPV * ND; t += NT) {
            const int gg = t % NA, ad = t / NA, fc = gg / NGF, q = gg % NGF;
            double s = 0.0;
            for (int m = 0; m < NPF; m++) s += sm.sfc[q + NGF * m] * Cm[sm.perm[fc * NPF + m] + NPV * ad];
            sMiCf[t] = s;
        }
        for (int t = tid; t < NA * NDF * ND; t += NT) {
            const int gg = t % NA, fd = t / NA, fc = gg / NGF, q = gg % NGF;
            double s = 0.0;
            for (int m = 0; m < NPF; m++) s += sm.sfc[q + NGF * m] * Em[sm.perm[fc * NPF + m] + NPV * fd];
            sMiEf[t] = s;
        }
        // pointwise fluxes: one work item per (point, differentiated variable k);
        // a one-derivative dual pass gives f and df/dw_k at that point.
        for (int t = tid; t < (NGV + NA) * NC; t += NT) {
            using DD = Dual<1>;
            const int p = t % (NGV + NA), k = t / (NGV + NA);
            const bool vol = p < NGV;
            const int g = vol ? p : p - NGV;
            DD w[NC], f[ND * NCU];
#pragma unroll
            for (int c = 0; c < NC; c++) {
                const double val = vol ? ug[g + NGV * c] : ((c < NCU) ? uhg[g + NA * c] : ugf[g + NA * c]);
                w[c].v = val;
                w[c].d[0] = (c == k) ? 1.0 : 0.0;
            }
            ns_flux_dual<ND>(A.param, w, f);
            if (vol) {
                const double jg = sm.jac[g];
#pragma unroll
                for (int j = 0; j < NCU; j++) {
                    if (k == 0) {
                        double s = 0.0;
                        if (A.tdep) {
                            double tt = 0.0;
                            for (int a = 0; a < NPV; a++) tt += T.shapvt[g + NGV * a] * sm.shu[a + NPV * j];
                            s = tt - ug[g + NGV * j] * A.fc_u;
                        }
                        sm.wrk[g + NGV * (0 + ND1 * j)] = s * jg;
#pragma unroll
                        for (int m = 0; m < ND; m++) {
                            double fx = 0.0;
#pragma unroll
                            for (int d = 0; d < ND; d++) fx += f[d * NCU + j].v * sm.Xx[g + NGV * (d + ND * m)];
                            sm.wrk[g + NGV * ((m + 1) + ND1 * j)] = fx;
                        }
                    }
                    const double su = (A.tdep && k == j) ? -A.fc_u : 0.0;
                    wrl[g + NGV * (0 + ND1 * (j + NCU * k))] = -su * jg;
#pragma unroll
                    for (int m = 0; m < ND; m++) {
                        double tt = 0.0;
#pragma unroll
                        for (int d = 0; d < ND; d++) tt += f[d * NCU + j].d[0] * sm.Xx[g + NGV * (d + ND * m)];
                        wrl[g + NGV * ((m + 1) + ND1 * (j + NCU * k))] = -tt;
                    }
                }
            } else {
                // fhat = F(uh, q).n + tau (u - uh)   (fhatDriver.cpp:54-236), times jacf
                const double tau = A.param[5];
                const double jf = sm.jacf[g];
#pragma unroll
                for (int j = 0; j < NCU; j++) {
                    if (k == 0) {
                        double tt = tau * (ugf[g + NA * j] - uhg[g + NA * j]);
#pragma unroll
                        for (int d = 0; d < ND; d++) tt += f[d * NCU + j].v * sm.nl[g + NA * d];
                        sm.fn[g + NA * j] = tt * jf;
                    }
                    double dn = 0.0;
#pragma unroll
                    for (int d = 0; d < ND; d++) dn += f[d * NCU + j].d[0] * sm.nl[g + NA * d];
                    if (k < NCU) {
                        fnuh[g + NA * (j + NCH * k)] = (dn - (k == j ? tau : 0.0)) * jf;
                        fnu[g + NA * (j + NCH * k)] = (k == j ? tau : 0.0) * jf;
                    } else {
                        fnu[g + NA * (j + NCH * k)] = dn * jf;
                    }
                }
            }
        }
        __syncthreads();

        double* Ke = A.K + (size_t)e * NB * N;
        double* He = A.H + (size_t)e * NB * NB;
        double* Rhe = A.Rh + (size_t)e * NB;
        double* Roe = A.Ro + (size_t)e * NB;
        for (int t = tid; t < NB; t += NT) {
            const int j = t % NCH, fdof = t / NCH, fc = fdof / NPF, ip = fdof % NPF;
            double s = 0.0;
            for (int q = 0; q < NGF; q++) s += sm.Af[ip + C2::LDAF * q] * sm.fn[q + NGF * fc + NA * j];
            Rhe[t] = -s;
            Roe[t] = -s;
        }
        // ---- K and H, face by face: columns (j, m, a) and (j, m, f2), chunks of CWF
        constexpr int NCOLK = NCH * NCU * NPV, NCOLH = NCH * NCU * NDF;
        for (int job = 0; job < NFE * 2; job++) {
            const int fc = job % NFE;
            const bool isH = job >= NFE;
            const int ncol = isH ? NCOLH : NCOLK;
            for (int c0 = 0; c0 < ncol; c0 += C2::CWF) {
                __syncthreads();
                for (int t = tid; t < C2::KF * C2::CWF; t += NT) {
                    const int q = t % C2::KF, cl = t / C2::KF, c = c0 + cl;
                    double v = 0.0;
                    if (q < NGF && c < ncol) {
                        const int gg = q + NGF * fc;
                        const int j = c % NCH, m = (c / NCH) % NCU, z = c / (NCH * NCU);
                        double s = 0.0;
#pragma unroll
                        for (int d = 0; d < ND; d++)
                            s += fnu[gg + NA * (j + NCH * (NCU * (1 + d) + m))] *
                                 (isH ? sMiEf[gg + NA * (z + NDF * d)] : sMiCf[gg + NA * (z + NPV * d)]);
                        if (isH) {
                            v = -s;
                            if (z / NPF == fc) v += sm.sfc[q + NGF * (z % NPF)] * fnuh[gg + NA * (j + NCH * m)];
                        } else {
                            v = s;
                            const int p = sm.pos[fc * NPV + z];
                            if (p >= 0) v += sm.sfc[q + NGF * p] * fnu[gg + NA * (j + NCH * m)];
                        }
                    }
                    Bs[q + C2::LDBF * cl] = v;
                }
                __syncthreads();
                double acc[C2::MTF][C2::NTWF][2];
#pragma unroll
                for (int a = 0; a < C2::MTF; a++)
#pragma unroll
                    for (int b = 0; b < C2::NTWF; b++) acc[a][b][0] = acc[a][b][1] = 0.0;
                chunk_mma<C2::MTF, C2::NTWF, C2::KF / 4>(sm.Af, C2::LDAF, Bs, C2::LDBF, acc);
#pragma unroll
                for (int a = 0; a < C2::MTF; a++)
#pragma unroll
                    for (int b = 0; b < C2::NTWF; b++)
#pragma unroll
                        for (int h = 0; h < 2; h++) {
                            const int ip = 8 * a + gr, c = c0 + 8 * (warp * C2::NTWF + b) + 2 * gc + h;
                            if (ip < NPF && c < ncol) {
                                const int j = c % NCH, m = (c / NCH) % NCU, z = c / (NCH * NCU);
                                const int row = j + NCH * (fc * NPF + ip);
                                if (isH) He[row + (size_t)NB * (m + NCH * z)] = acc[a][b][h];
                                else Ke[row + (size_t)NB * (z + NPV * m)] = acc[a][b][h];
                            }
                        }
            }
        }
        __syncthreads();
        // ---- D and F: volume GEMMs, then the lifted trace rows of K and H
        double* De = A.D + (size_t)e * N * N;
        double* Fe = A.F + (size_t)e * N * NB;
        constexpr int NCOLD = NCU * NPV * NCU, NCOLF = NCU * NCU * NDF;
        for (int job = 0; job < 2; job++) {
            const bool isF = job == 1;
            const int ncol = isF ? NCOLF : NCOLD;
            for (int c0 = 0; c0 < ncol; c0 += C2::CWV) {
                __syncthreads();
                for (int t = tid; t < C2::KV * C2::CWV; t += NT) {
                    const int q = t % C2::KV, cl = t / C2::KV, c = c0 + cl;
                    double v = 0.0;
                    if (q < NQ && c < ncol) {
                        const int g = q % NGV, r = q / NGV;
                        if (!isF) {                 // column (j, a, k)
                            const int j = c % NCU, a = (c / NCU) % NPV, k = c / (NCU * NPV);
                            v = wrl[g + NGV * (r + ND1 * (j + NCU * k))] * T.shapvt[g + NGV * a];
#pragma unroll
                            for (int d = 0; d < ND; d++)
                                v += wrl[g + NGV * (r + ND1 * (j + NCU * (NCU * (1 + d) + k)))] * sMiC[g + NGV * (a + NPV * d)];
                        } else {                    // column (j, k, f2)
                            const int j = c % NCU, k = (c / NCU) % NCU, f2 = c / (NCU * NCU);
#pragma unroll
                            for (int d = 0; d < ND; d++)
                                v += wrl[g + NGV * (r + ND1 * (j + NCU * (NCU * (1 + d) + k)))] * sMiE[g + NGV * (f2 + NDF * d)];
                        }
                    }
                    Bs[q + C2::LDBV * cl] = v;
                }
                __syncthreads();
                double acc[C2::MTV][C2::NTWV][2];
#pragma unroll
                for (int a = 0; a < C2::MTV; a++) acc[a][0][0] = acc[a][0][1] = 0.0;
                chunk_mma<C2::MTV, C2::NTWV, C2::KV / 4>(sm.Av, C2::LDAV, Bs, C2::LDBV, acc);
#pragma unroll
                for (int a = 0; a < C2::MTV; a++)
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const int i = 8 * a + gr, c = c0 + 8 * warp + 2 * gc + h;
                        if (i < NPV && c < ncol) {
                            double s = acc[a][0][h];
                            const int j = c % NCU;
                            if (!isF) {
                                const int kcol = c / NCU;       // a + NPV*k
                                for (int c2 = 0; c2 < sm.inc_n[i]; c2++)
                                    s += Ke[j + NCH * sm.inc_f[i * S::MAXINC + c2] + (size_t)NB * kcol];
                                De[i + NPV * c] = s;
                            } else {
                                const int hcol = c / NCU;       // k + NCH*f2
                                for (int c2 = 0; c2 < sm.inc_n[i]; c2++)
                                    s += He[j + NCH * sm.inc_f[i * S::MAXINC + c2] + (size_t)NB * hcol];
                                Fe[i + NPV * c] = s;
                            }
                        }
                    }
            }
        }
        double ru2 = 0.0;
        for (int t = tid; t < N; t += NT) {
            const int i = t % NPV, j = t / NPV;
            double s = 0.0;
            for (int q = 0; q < NQ; q++) s += sm.Av[i + C2::LDAV * q] * sm.wrk[q + NQ * j];
            for (int c2 = 0; c2 < sm.inc_n[i]; c2++) s += Rhe[j + NCH * sm.inc_f[i * S::MAXINC + c2]];
            A.Ru[(size_t)e * N + t] = s;
            ru2 += s * s;
        }
        const double tot = block_sum(ru2, sm.red);
        if (tid == 0) A.ru2[e] = tot;
    }
}

}  // namespace hfem
