// Element assembly on the FP64 tensor cores (sm_100a, mma.sync m8n8k4 f64).
//
// One CTA owns one element at a time (persistent grid, 2 CTAs per SM).  Every
// contraction after the pointwise fluxes is a GEMM with rows over (test node,
// equation, variable) and a B operand resident in shared memory (restating
// elementassembly.cpp elementint 307-572 and faceint 717-1321):
//   K_fc[(ip,j,m), a]  = sum_{q,d'} shapfg(ip,q) fhn(q; j, (d',m)) Phi_fc[(q,d'), a],
//        Phi_fc[(q,0),a] = [a on fc] phi_pos(a)(q),  Phi_fc[(q,d+1),a] = (phi M^-1 C_d)(q; a)
//   H_fc[(ip,j,m), f2] = sum_{q,d'} shapfg(ip,q) fhn'(q; j, (d',m)) Psi_fc[(q,d'), f2],
//        d' = 0 uses fhn_uh and Psi_fc[(q,0),f2] = [f2 on fc] phi_f2(q); d' > 0 uses
//        fhn_u(q; j, q_dm) and Psi_fc = -(phi M^-1 E_d)(q; f2)
//   Y(i,g,j,c) = sum_r shapvg(i,(g,r)) wrl((g,r), j, c)       (the derivative index r)
//   D_vol[(i,j,k), a]  = sum_{g,d'} Y(i,g,j,(d',k)) Phi[(g,d'), a],  Phi = [phi_a(g); (phi M^-1 C_d)(g;a)]
//   F_vol[(i,j,k), f2] = sum_{g,d} Y(i,g,j,(d+1,k)) (-phi M^-1 E_d)(g; f2)
// The B operands are formed in shared memory from M^-1 C and M^-1 E, which
// stay in shared memory after the local Cholesky solves: their rows d' > 0 are
// the products shapvt (M^-1 C | M^-1 E) and, per face, shapfc (M^-1 C | M^-1 E)
// at the face's nodes, small GEMMs on the same FP64 tensor cores.  Of the lifted trace
// terms, D += P K is added here by reductions in L2 (face after face, so each
// sum has a fixed order), and F += P H of interior faces by the condensation
// kernels when they load F (lift.cuh), where H is read anyway; boundary faces,
// whose trace rows take the boundary flux while their element rows keep fhat,
// are lifted here in full.  The face mass product uses shapfgdotshapfc = shapfg .* shapfc (its
// definition, mkmasterelement.m:113-115) in factored form.
#pragma once
#include <cuda_runtime.h>
#include <type_traits>
#include "elem_kernels.cuh"
#include "schur_kernels.cuh"
#include "tf32x3.cuh"
#include "bulk_copy.cuh"

namespace hfem {

// Tiles of the row-major element GEMMs (K/H per face, D/F volume) and the
// shared-memory and workspace budgets of one CTA.
template <class S>
struct EK {
    static constexpr int NKP = ((S::NPV + 7) / 8) * 8;             // K columns (a), padded
    static constexpr int NHP = ((S::NDF + 7) / 8) * 8;             // H columns (f2), padded
    static constexpr int NTK = NKP / 8, NTH = NHP / 8;             // n-tiles
    static constexpr int KFD = ((S::NGF * (S::ND + 1) + 3) / 4) * 4;  // face k = (q, d')
    static constexpr int KV3 = ((S::NGV * (S::ND + 1) + 3) / 4) * 4;  // volume k = (g, d')
    static constexpr int KQ3 = ((S::NGV * S::ND + 3) / 4) * 4;        // volume k = (g, d)
    static constexpr int LDBK = ((KFD + 11) / 16) * 16 + 4;        // == 4 (mod 16): conflict-free B fragments
    static constexpr int LDBD = ((KV3 + 11) / 16) * 16 + 4;
    static constexpr int BKH = LDBK * (NKP + NHP);                 // one face's B operand
    static constexpr int BDF = LDBD * (NKP + NHP);                 // the volume B operand
    static constexpr int MTV = (S::NPV + 7) / 8;
    static constexpr int MTF = (S::NPF + 7) / 8;
    static constexpr int KV = ((S::NQ + 3) / 4) * 4;               // padded k of shapvg
    static constexpr int KF = ((S::NGF + 3) / 4) * 4;              // padded k of shapfg
    static constexpr int LDAV = S::NPV | 1;                        // odd: lanes along q hit distinct banks
    static constexpr int LDAF = ((8 * MTF + 11) / 16) * 16 + 4;
    // one face's flux-Jacobian slices: [q + NGF (j + NCH c)], c < NC for fhn_u / fb_u,
    // then NGF NCH NCU entries for fhn_uh / fb_uh
    static constexpr int FSL = S::NGF * S::NCH * (S::NC + S::NCU);
    static constexpr int FSLP = (FSL + 1) / 2 * 2;                 // per-face stride: 16-byte copies
    // shared-memory union: M^-1 C and M^-1 E, then either the q/flux phase
    // scratch or the B operand of the GEMM being run
    static constexpr int CME = S::NPV * S::NPV * S::ND + S::NPV * S::NDF * S::ND;
    // the q / flux phase region: M, point states, then u, uhe and the source,
    // u and the source at even offsets (16-byte bulk copies land there)
    static constexpr int O_UG = S::NPV * S::NPV;
    static constexpr int O_UGF = O_UG + S::NGV * S::NC;
    static constexpr int O_UHG = O_UGF + S::NA * S::NC;
    static constexpr int O_U = (O_UHG + S::NA * S::NCH + 1) / 2 * 2;
    static constexpr int O_UHE = O_U + S::NPV * S::NC;
    static constexpr int O_SHU = (O_UHE + S::NDF * S::NCH + 1) / 2 * 2;
    static constexpr int QPH = O_SHU + S::NPV * S::NCU;
    static constexpr int GPH = BDF > BKH + FSLP ? BDF : BKH + FSLP;
    static constexpr int UN = CME + (QPH > GPH ? QPH : GPH);
    // global workspace per CTA slot (doubles): wrl, the interior and boundary
    // face slices, the boundary flux values, Y
    static constexpr int W_WRL = S::NQ * S::NCU * S::NC;
    static constexpr int W_FSL = S::NFE * FSLP;
    static constexpr int W_FNB = S::NA * S::NCH;
    static constexpr int W_Y = S::NPV * S::NGV * S::NCU * S::NC;
    static constexpr int WS = W_WRL + 2 * W_FSL + W_FNB + W_Y;
    static_assert(CME % 2 == 0 && BKH % 2 == 0 && W_WRL % 2 == 0 && WS % 2 == 0 && W_FSL % 2 == 0,
                  "16-byte alignment of the staged face slices");
    static_assert(O_U % 2 == 0 && O_SHU % 2 == 0, "16-byte alignment of the bulk-copied element inputs");
};

// Cholesky solves L L' x = b for one column held in registers, in the axpy
// (column) form: after x_j is final every later entry takes its update, so each
// step has up to npv - 1 independent FMAs; rdg holds 1 / L(j, j).
template <int NPV>
__device__ __forceinline__ void chol_solve_col_axpy(const double* lm, const double* rdg, double* col) {
    const volatile double* l = lm;
    double x[NPV];
#pragma unroll
    for (int i = 0; i < NPV; i++) x[i] = col[i];
#pragma unroll
    for (int j = 0; j < NPV; j++) {
        x[j] *= rdg[j];
#pragma unroll
        for (int i = j + 1; i < NPV; i++) x[i] = fma(-l[i + NPV * j], x[j], x[i]);
    }
#pragma unroll
    for (int j = NPV - 1; j >= 0; j--) {
        x[j] *= rdg[j];
#pragma unroll
        for (int i = 0; i < j; i++) x[i] = fma(-l[j + NPV * i], x[j], x[i]);
    }
#pragma unroll
    for (int i = 0; i < NPV; i++) col[i] = x[i];
}

// Basis-by-(M^-1 C | M^-1 E) products on the FP64 tensor cores, one n-tile per
// warp at a time:
//   OUT(r, n) = sum_kk A(r, kk) CE(row(kk), n),  r < MR, kk < KD, n < NPV ND + NDF ND
// with A(r, kk) = a[r + lda kk], CE the column-major npv x (npv nd + ndf nd)
// block [M^-1 C | M^-1 E] and row(kk) = rmap[kk] (a face's nodes) or kk.
// st(r, n, v) receives every valid entry.
template <int MR, int KD, int NPV, int NCOL, int NW, class Store>
__device__ __forceinline__ void basis_ce_gemm(const double* a, int lda, const int* rmap, const double* CE, Store st) {
    constexpr int MT = (MR + 7) / 8, KS = (KD + 3) / 4, NNT = (NCOL + 7) / 8;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, gr = lane >> 2, gc = lane & 3;
    double af[MT][KS];
    int brow[KS];
#pragma unroll
    for (int ks = 0; ks < KS; ks++) {
        const int kk = 4 * ks + gc;
        brow[ks] = kk < KD ? (rmap ? rmap[kk] : kk) : -1;
#pragma unroll
        for (int mt = 0; mt < MT; mt++) {
            const int r = 8 * mt + gr;
            af[mt][ks] = (r < MR && kk < KD) ? a[r + lda * kk] : 0.0;
        }
    }
    // the warp's n-tiles unrolled, so their DMMA chains overlap
#pragma unroll
    for (int it = 0; it < (NNT + NW - 1) / NW; it++) {
        const int nt = warp + it * NW;
        if (nt >= NNT) break;
        const int n = 8 * nt + gr;
        double acc[MT][2];
#pragma unroll
        for (int mt = 0; mt < MT; mt++) acc[mt][0] = acc[mt][1] = 0.0;
#pragma unroll
        for (int ks = 0; ks < KS; ks++) {
            const double bv = (brow[ks] >= 0 && n < NCOL) ? CE[brow[ks] + NPV * n] : 0.0;
#pragma unroll
            for (int mt = 0; mt < MT; mt++) dmma8x8x4(acc[mt][0], acc[mt][1], af[mt][ks], bv);
        }
#pragma unroll
        for (int mt = 0; mt < MT; mt++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int r = 8 * mt + gr, nn = 8 * nt + 2 * gc + h;
                if (r < MR && nn < NCOL) st(r, nn, acc[mt][h]);
            }
    }
}

template <class S>
struct ElemSmem {
    double x[S::NPV * S::ND];
    double jac[S::NGV], Xx[S::NGV * S::ND * S::ND];
    double jacf[S::NA], nl[S::NA * S::ND];
    double wrk[S::NQ * S::NCU];
    double fn[S::NA * S::NCH];
    double rh[S::NB];                      // Rh with fhat on every face (the element equations' lift)
    double Av[EK<S>::LDAV * EK<S>::KV];    // shapvg, zero padded: Av[i + LDAV*q]
    double Af[EK<S>::LDAF * EK<S>::KF];    // shapfg, zero padded: Af[ip + LDAF*q]
    double sfc[S::NGF * S::NPF];           // face basis values shapfc(kk, q) = shapft[q + NGF*kk]
    double red[NT / 32];
    double rdg[S::NPV];                    // 1 / L(j, j) of the Cholesky factor of M
    uint64_t bar_in, bar_sl;               // bulk-copy barriers: element inputs, face slices
    alignas(16) double un[EK<S>::UN];
    int perm[S::NDF];
    int inc_n[S::NPV];
    int inc_f[S::NPV * S::MAXINC];
    int pos[S::NFE * S::NPV];              // position of element node a on face fc, or -1
};

// TF: the contractions in 3xTF32 (precision modes 1, 3); GEN: the Lax-Friedrichs
// / Roe stabilization tensors and Sutherland's law compiled in (the default
// instantiation holds the constant-tau, constant-viscosity physics only).
template <class S, bool TF = false, bool GEN = false>
__global__ void __launch_bounds__(NT, 2) element_kernel(ElemArgs A) {
    constexpr int ND = S::ND, NPV = S::NPV, NPF = S::NPF, NGV = S::NGV, NGF = S::NGF, NFE = S::NFE;
    constexpr int NCU = S::NCU, NC = S::NC, NCH = S::NCH, NDF = S::NDF, ND1 = S::ND1, N = S::N, NB = S::NB;
    constexpr int NA = S::NA, NQ = S::NQ;
    using G = EK<S>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ElemSmem<S>& sm = *reinterpret_cast<ElemSmem<S>*>(smem_raw);
    const Tables& T = A.T;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gr = lane >> 2, gc = lane & 3;

    double* ws = A.ws + (size_t)blockIdx.x * G::WS;
    double* wrl = ws;                              // [g + NGV (r + ND1 (j + NCU c))]
    double* fsl = wrl + G::W_WRL;                  // per face: fhat Jacobian slices
    double* fslb = fsl + G::W_FSL;                 // per face: boundary-flux Jacobian slices
    double* fnb = fslb + G::W_FSL;                 // boundary flux [g' + NA j]
    double* Ys = fnb + G::W_FNB;                   // Y(i,g,j,c) at [g + NGV (c + NC (i + NPV j))]

    // shared union: M^-1 C, M^-1 E, then the phase region
    double* Cm = sm.un;                            // [b + NPV (a + NPV d)]
    double* Em = Cm + NPV * NPV * ND;              // [b + NPV (f + NDF d)]
    double* ph = sm.un + G::CME;
    double* M = ph;                                // q / flux phase
    double* ug = ph + G::O_UG;
    double* ugf = ph + G::O_UGF;
    double* uhg = ph + G::O_UHG;
    double* u = ph + G::O_U;
    double* uhe = ph + G::O_UHE;
    double* shu = ph + G::O_SHU;
    double* Bs = ph;                               // GEMM phases

    for (int t = tid; t < G::LDAV * G::KV; t += NT) {
        const int i = t % G::LDAV, q = t / G::LDAV;
        sm.Av[t] = (i < NPV && q < NQ) ? T.shapvg[i + NPV * q] : 0.0;
    }
    for (int t = tid; t < G::LDAF * G::KF; t += NT) {
        const int i = t % G::LDAF, q = t / G::LDAF;
        sm.Af[t] = (i < NPF && q < NGF) ? T.shapfg[i + NPF * q] : 0.0;
    }
    for (int t = tid; t < NGF * NPF; t += NT) sm.sfc[t] = T.shapft[t];
    for (int t = tid; t < NDF; t += NT) sm.perm[t] = T.perm[t];
    if (tid == 0) {
        bulk_bar_init(&sm.bar_in);
        bulk_bar_init(&sm.bar_sl);
    }
    uint32_t ph_in = 0, ph_sl = 0;                 // barrier phases (the same in every thread)
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

    for (int e = A.e_begin + blockIdx.x; e < A.ne; e += gridDim.x) {
        bulk_proxy_fence();
        __syncthreads();
        const double* xg = A.dgnodes + (size_t)e * NPV * ND;
        const double* ugl = A.udg + (size_t)e * NPV * NC;
        const double* shg = A.sh + (size_t)e * NPV * NC;
        // the element's contiguous inputs (coordinates, u with q, source) by the
        // TMA engine's bulk copies while the threads gather uh through elcon;
        // plain loads when a caller's array is not 16-byte aligned
        const bool bulk = bulk_aligned(xg) && bulk_aligned(ugl) && bulk_aligned(shg);
        if (bulk) {
            if (tid == 0) {
                constexpr uint32_t BX = NPV * ND * 8, BU = NPV * NC * 8, BS = NPV * NCU * 8;
                static_assert(BX % 16 == 0 && BU % 16 == 0 && BS % 16 == 0, "bulk copies move 16-byte multiples");
                bulk_bar_expect(&sm.bar_in, BX + BU + BS);
                bulk_load(sm.x, xg, BX, &sm.bar_in);
                bulk_load(u, ugl, BU, &sm.bar_in);
                bulk_load(shu, shg, BS, &sm.bar_in);
            }
        } else {
            for (int t = tid; t < NPV * ND; t += NT) sm.x[t] = xg[t];
            for (int t = tid; t < NPV * NC; t += NT) u[t] = ugl[t];
            for (int t = tid; t < NPV * NCU; t += NT) shu[t] = shg[t];
        }
        for (int t = tid; t < NDF * NCH; t += NT) {
            const int fdof = t / NCH, c = t % NCH;
            uhe[fdof + NDF * c] = A.uh[(size_t)A.elcon[(size_t)e * NDF + fdof] * NCH + c];
        }
        if (bulk) {
            if (!bulk_bar_wait(&sm.bar_in, ph_in) && tid == 0 && A.err) atomicExch(A.err, 2);
            ph_in ^= 1u;
        }
        __syncthreads();
        geometry<S>(T, sm.x, sm.jac, sm.Xx, sm.jacf, sm.nl);
        __syncthreads();
        qmatrices<S>(T, A.fc_q, sm.jac, sm.Xx, sm.jacf, sm.nl, M, Cm, Em);
        __syncthreads();
        const double* P = A.pparam ? A.pparam + 8 * A.eprob[e] : A.param;
        const int tdep = A.pparam ? (int)P[6] : A.tdep;
        const double fc_u = A.pparam ? P[7] : A.fc_u;
        const int* bfe = A.bf ? A.bf + (size_t)e * NFE : nullptr;
        // warp 0 factors M while the other warps evaluate the states at the points
        // and the pointwise fluxes, which do not depend on M
        if (warp == 0) {
            cholesky_warp<NPV>(M, sm.rdg);
        } else {
            constexpr int NT1 = NT - 32;
            const int tid1 = tid - 32;
            for (int t = tid1; t < NGV * NC; t += NT1) {
                const int g = t % NGV, c = t / NGV;
                double s = 0.0;
                for (int a = 0; a < NPV; a++) s += T.shapvt[g + NGV * a] * u[a + NPV * c];
                ug[t] = s;
            }
            for (int t = tid1; t < NA * (NC + NCH); t += NT1) {
                const int gg = t % NA, c = t / NA, fc = gg / NGF, q = gg % NGF;
                double s = 0.0;
                if (c < NC) {
                    for (int m = 0; m < NPF; m++) s += sm.sfc[q + NGF * m] * u[sm.perm[fc * NPF + m] + NPV * c];
                    ugf[gg + NA * c] = s;
                } else {
                    for (int m = 0; m < NPF; m++) s += sm.sfc[q + NGF * m] * uhe[fc * NPF + m + NDF * (c - NC)];
                    uhg[gg + NA * (c - NC)] = s;
                }
            }
            asm volatile("bar.sync 1, %0;" ::"r"(NT1) : "memory");
            // pointwise fluxes: one work item per (point, differentiated variable k);
            // a one-derivative dual pass gives f and df/dw_k at that point.
            for (int t = tid1; t < (NGV + NA) * NC; t += NT1) {
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
                ns_flux_dual<ND, 1, GEN>(P, w, f, !A.inviscid, A.visc_model);
                if (vol) {
                    const double jg = sm.jac[g];
#pragma unroll
                    for (int j = 0; j < NCU; j++) {
                        if (k == 0) {
                            double s = 0.0;
                            if (tdep) {
                                double tt = 0.0;
                                for (int a = 0; a < NPV; a++) tt += T.shapvt[g + NGV * a] * shu[a + NPV * j];
                                s = tt - ug[g + NGV * j] * fc_u;
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
                        const double su = (tdep && k == j) ? -fc_u : 0.0;
                        wrl[g + NGV * (0 + ND1 * (j + NCU * k))] = -su * jg;
#pragma unroll
                        for (int m = 0; m < ND; m++) {
                            double tt = 0.0;
#pragma unroll
                            for (int d = 0; d < ND; d++) tt += f[d * NCU + j].d[0] * sm.Xx[g + NGV * (d + ND * m)];
                            wrl[g + NGV * ((m + 1) + ND1 * (j + NCU * k))] = -tt;
                        }
                    }
                } else if (!GEN || A.conv_stab == 0) {
                    // fhat = F(uh, q).n + tau (u - uh)   (fhatDriver.cpp:54-236), times jacf
                    const double tau = P[5];
                    const double jf = sm.jacf[g];
                    const int fc = g / NGF, q = g % NGF;
                    double* sl = fsl + fc * G::FSLP;
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
                            sl[NGF * NCH * NC + q + NGF * (j + NCH * k)] = (dn - (k == j ? tau : 0.0)) * jf;
                            sl[q + NGF * (j + NCH * k)] = (k == j ? tau : 0.0) * jf;
                        } else {
                            sl[q + NGF * (j + NCH * k)] = dn * jf;
                        }
                    }
                } else {
                    // fhat = F(uh, q).n + tau(uh) (u - uh) with the Lax-Friedrichs or
                    // Roe tensor (ns_stab_point): the uh-derivative of the
                    // stabilization term along this item's variable and column k of tau
                    const double jf = sm.jacf[g];
                    const int fc = g / NGF, q = g % NGF;
                    double* sl = fsl + fc * G::FSLP;
                    double nlq[ND], uhv[NCU], uv[NCU], sv[NCU], sd[NCU], tcol[NCU];
#pragma unroll
                    for (int d = 0; d < ND; d++) nlq[d] = sm.nl[g + NA * d];
#pragma unroll
                    for (int m = 0; m < NCU; m++) {
                        uhv[m] = w[m].v;
                        uv[m] = ugf[g + NA * m];
                    }
                    ns_stab_point<ND>(A.conv_stab, P, nlq, uhv, uv, k, sv, sd, tcol);
#pragma unroll
                    for (int j = 0; j < NCU; j++) {
                        if (k == 0) {
                            double tt = sv[j];
#pragma unroll
                            for (int d = 0; d < ND; d++) tt += f[d * NCU + j].v * sm.nl[g + NA * d];
                            sm.fn[g + NA * j] = tt * jf;
                        }
                        double dn = 0.0;
#pragma unroll
                        for (int d = 0; d < ND; d++) dn += f[d * NCU + j].d[0] * sm.nl[g + NA * d];
                        if (k < NCU) {
                            sl[NGF * NCH * NC + q + NGF * (j + NCH * k)] = (dn + sd[j]) * jf;
                            sl[q + NGF * (j + NCH * k)] = tcol[j] * jf;
                        } else {
                            sl[q + NGF * (j + NCH * k)] = dn * jf;
                        }
                    }
                }
            }
            // boundary faces: fb and its Jacobians at their points (one item per point and variable)
            if (bfe) {
                for (int t = tid1; t < NFE * NGF * (NC + NCH); t += NT1) {
                    const int fc = t / (NGF * (NC + NCH)), r = t % (NGF * (NC + NCH));
                    if (bfe[fc] >= 0) continue;
                    using DD = Dual<1>;
                    const int q = r % NGF, k = r / NGF, gg = q + NGF * fc;
                    DD w[NC], uhd[NCH], fb[NCH];
#pragma unroll
                    for (int c = 0; c < NC; c++) {
                        w[c].v = ugf[gg + NA * c];
                        w[c].d[0] = (c == k) ? 1.0 : 0.0;
                    }
#pragma unroll
                    for (int c = 0; c < NCH; c++) {
                        uhd[c].v = uhg[gg + NA * c];
                        uhd[c].d[0] = (NC + c == k) ? 1.0 : 0.0;
                    }
                    double nlq[ND];
#pragma unroll
                    for (int d = 0; d < ND; d++) nlq[d] = sm.nl[gg + NA * d];
                    const int ib = -bfe[fc] - 1;
                    if (!ns_fbou_dual<ND, 1, GEN>(A.bcm[ib], P, A.bcs + (size_t)ib * NCH, nlq, w, uhd, fb,
                                                  !A.inviscid, A.conv_stab, A.visc_model)) {
                        for (int j = 0; j < NCH; j++) fb[j] = dc<1>(0.0);
                    }
                    const double jf = sm.jacf[gg];
                    double* sl = fslb + fc * G::FSLP;
#pragma unroll
                    for (int j = 0; j < NCH; j++) {
                        if (k == 0) fnb[gg + NA * j] = fb[j].v * jf;
                        if (k < NC) sl[q + NGF * (j + NCH * k)] = fb[j].d[0] * jf;
                        else sl[NGF * NCH * NC + q + NGF * (j + NCH * (k - NC))] = fb[j].d[0] * jf;
                    }
                }
            }
        }
        __syncthreads();
        // M^-1 C and M^-1 E in place, one column per thread
        for (int t = tid; t < NPV * ND + NDF * ND; t += NT) chol_solve_col_axpy<NPV>(M, sm.rdg, &Cm[NPV * t]);
        __syncthreads();

        double* Ke = A.K + (size_t)e * NB * N;
        double* De = A.D + (size_t)e * N * N;
        double* Fe = A.F + (size_t)e * N * NB;
        double* He = A.H + (size_t)e * NB * NB;
        double* Rhe = A.Rh + (size_t)e * NB;
        double* Roe = A.Ro + (size_t)e * NB;
        for (int t = tid; t < NB; t += NT) {
            const int j = t % NCH, fdof = t / NCH, fc = fdof / NPF, ip = fdof % NPF;
            double s = 0.0;
            for (int q = 0; q < NGF; q++) s += sm.Af[ip + G::LDAF * q] * sm.fn[q + NGF * fc + NA * j];
            sm.rh[t] = -s;
            Rhe[t] = -s;
            Roe[t] = -s;
        }
        // Y, point index fastest: Ys[g + NGV (c + NC (i + NPV j))], c = NCU d' + k.
        // One thread per (g, j, c) with g fastest: its wrl words are read once and
        // the stores of a warp are runs of consecutive words.
        // The next item's wrl words are requested before this item's products, so
        // their latency overlaps them.
        {
            constexpr int NY = NGV * NCU * NC;
            auto wload = [&](int t, double* w) {
                const int g = t % NGV, j = (t / NGV) % NCU, c = t / (NGV * NCU);
#pragma unroll
                for (int r = 0; r < ND1; r++) w[r] = t < NY ? wrl[g + NGV * (r + ND1 * (j + NCU * c))] : 0.0;
            };
            double w[ND1], wn[ND1];
            wload(tid, w);
            for (int t = tid; t < NY; t += NT) {
                wload(t + NT, wn);
                const int g = t % NGV, j = (t / NGV) % NCU, c = t / (NGV * NCU);
#pragma unroll 4
                for (int i = 0; i < NPV; i++) {
                    double y = 0.0;
#pragma unroll
                    for (int r = 0; r < ND1; r++) y += sm.Av[i + G::LDAV * (g + NGV * r)] * w[r];
                    bput<TF>(&Ys[g + NGV * (c + NC * (i + NPV * j))], y);
                }
#pragma unroll
                for (int r = 0; r < ND1; r++) w[r] = wn[r];
            }
        }
        // volume B operands: Phi (KV3 x NKP) and Psi (KQ3 x NHP), ld LDBD.  The
        // rows d' > 0 are shapvt (M^-1 C | M^-1 E) on the tensor cores; the d' = 0
        // rows of Phi (the basis values) and the zero padding are written directly.
        {
            double* Phi = Bs;
            double* Psi = Bs + G::LDBD * G::NKP;
            for (int t = tid; t < G::KV3 * G::NKP; t += NT) {
                const int k = t % G::KV3, a = t / G::KV3;
                if (a < NPV && k >= NGV && k < NGV * ND1) continue;
                bput<TF>(&Phi[k + G::LDBD * a], (a < NPV && k < NGV) ? T.shapvt[k + NGV * a] : 0.0);
            }
            for (int t = tid; t < G::KV3 * G::NHP; t += NT) {
                const int k = t % G::KV3, f2 = t / G::KV3;
                if (f2 < NDF && k < NGV * ND) continue;
                bput<TF>(&Psi[k + G::LDBD * f2], 0.0);
            }
            basis_ce_gemm<NGV, NPV, NPV, NPV * ND + NDF * ND, NT / 32>(
                T.shapvt, NGV, nullptr, Cm, [&](int g, int n, double v) {
                    if (n < NPV * ND) {
                        const int a = n % NPV, d = n / NPV;
                        bput<TF>(&Phi[(g + NGV * (d + 1)) + G::LDBD * a], v);
                    } else {
                        const int f2 = (n - NPV * ND) % NDF, d = (n - NPV * ND) / NDF;
                        bput<TF>(&Psi[(g + NGV * d) + G::LDBD * f2], -v);
                    }
                });
        }
        __syncthreads();
        // ---- D_vol = Y' Phi and F_vol = Y'_q Psi (right after Y is written, while it is in L2)
        {
            const double* Phi = Bs;
            const double* Psi = Bs + G::LDBD * G::NKP;
            // m-tiles in pairs: every B fragment read from shared memory feeds two
            // DMMAs (shared-memory bandwidth is the busiest unit of this kernel)
            constexpr int MTD = (NPV * NCU * NCU + 7) / 8;
            // with NGV a multiple of 4 the F part's A values are the D part's
            // shifted by NGV/4 k-steps (the q derivatives d' = d + 1)
            constexpr bool SHIFT = NGV % 4 == 0 && G::KV3 == NGV * ND1;
            if constexpr (!TF) {
            for (int mp = warp; 2 * mp < MTD; mp += NT / 32) {
                int rr[2];
                bool rv[2];
                const double* yrow[2];
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    rr[u] = 8 * (2 * mp + u) + gr;
                    rv[u] = rr[u] < NPV * NCU * NCU;
                    const int i = rr[u] % NPV, j = (rr[u] / NPV) % NCU, k = rr[u] / (NPV * NCU);
                    yrow[u] = Ys + NGV * (k + NC * (i + NPV * j));
                }
                // the A values of both m-tiles for every k-step are loaded before the
                // first DMMA, so their latencies overlap
                double av[2][G::KV3 / 4];
#pragma unroll
                for (int u = 0; u < 2; u++)
#pragma unroll
                    for (int ks = 0; ks < G::KV3 / 4; ks++) {
                        const int kk = 4 * ks + gc, g = kk % NGV, dp = kk / NGV;
                        av[u][ks] = (rv[u] && kk < NGV * ND1) ? yrow[u][g + NGV * NCU * dp] : 0.0;
                    }
                double acc[2][G::NTK][2];
#pragma unroll
                for (int u = 0; u < 2; u++)
#pragma unroll
                    for (int b = 0; b < G::NTK; b++) acc[u][b][0] = acc[u][b][1] = 0.0;
#pragma unroll
                for (int ks = 0; ks < G::KV3 / 4; ks++) {
                    const int kk = 4 * ks + gc;
#pragma unroll
                    for (int b = 0; b < G::NTK; b++) {
                        const double bv = Phi[kk + G::LDBD * (8 * b + gr)];
                        dmma8x8x4(acc[0][b][0], acc[0][b][1], av[0][ks], bv);
                        dmma8x8x4(acc[1][b][0], acc[1][b][1], av[1][ks], bv);
                    }
                }
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    if (!rv[u]) continue;
                    const int i = rr[u] % NPV, j = (rr[u] / NPV) % NCU, k = rr[u] / (NPV * NCU);
#pragma unroll
                    for (int b = 0; b < G::NTK; b++)
#pragma unroll
                        for (int h = 0; h < 2; h++) {
                            const int a = 8 * b + 2 * gc + h;
                            if (a < NPV) De[i + NPV * (j + NCU * (a + NPV * k))] = acc[u][b][h];
                        }
                }
                double aq[2][G::KQ3 / 4];
#pragma unroll
                for (int u = 0; u < 2; u++)
#pragma unroll
                    for (int ks = 0; ks < G::KQ3 / 4; ks++) {
                        if constexpr (SHIFT) {
                            aq[u][ks] = av[u][ks + NGV / 4];
                        } else {
                            const int kk = 4 * ks + gc, g = kk % NGV, d = kk / NGV;
                            aq[u][ks] = (rv[u] && kk < NGV * ND) ? yrow[u][g + NGV * NCU * (d + 1)] : 0.0;
                        }
                    }
                double accf[2][G::NTH][2];
#pragma unroll
                for (int u = 0; u < 2; u++)
#pragma unroll
                    for (int b = 0; b < G::NTH; b++) accf[u][b][0] = accf[u][b][1] = 0.0;
#pragma unroll
                for (int ks = 0; ks < G::KQ3 / 4; ks++) {
                    const int kk = 4 * ks + gc;
#pragma unroll
                    for (int b = 0; b < G::NTH; b++) {
                        const double bv = Psi[kk + G::LDBD * (8 * b + gr)];
                        dmma8x8x4(accf[0][b][0], accf[0][b][1], aq[0][ks], bv);
                        dmma8x8x4(accf[1][b][0], accf[1][b][1], aq[1][ks], bv);
                    }
                }
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    if (!rv[u]) continue;
                    const int i = rr[u] % NPV, j = (rr[u] / NPV) % NCU, k = rr[u] / (NPV * NCU);
#pragma unroll
                    for (int b = 0; b < G::NTH; b++)
#pragma unroll
                        for (int h = 0; h < 2; h++) {
                            const int f2 = 8 * b + 2 * gc + h;
                            if (f2 < NDF) Fe[i + NPV * (j + NCU * (k + NCH * f2))] = accf[u][b][h];
                        }
                }
            }
            } else {
            // 3xTF32: the same m-tile pairs as one m16 tile, k-steps of 8
            const uint2* Phi2 = reinterpret_cast<const uint2*>(Phi);
            const uint2* Psi2 = reinterpret_cast<const uint2*>(Psi);
            constexpr int KS = G::KV3 / 4, KSQ = G::KQ3 / 4;
            for (int mp = warp; 2 * mp < MTD; mp += NT / 32) {
                int rr[2];
                bool rv[2];
                const uint2* yrow[2];
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    rr[u] = 8 * (2 * mp + u) + gr;
                    rv[u] = rr[u] < NPV * NCU * NCU;
                    const int i = rr[u] % NPV, j = (rr[u] / NPV) % NCU, k = rr[u] / (NPV * NCU);
                    yrow[u] = reinterpret_cast<const uint2*>(Ys) + NGV * (k + NC * (i + NPV * j));
                }
                uint32_t ah[2][KS], al[2][KS];
#pragma unroll
                for (int u = 0; u < 2; u++)
#pragma unroll
                    for (int ks = 0; ks < KS; ks++) {
                        const int kk = 4 * ks + gc, g = kk % NGV, dp = kk / NGV;
                        const uint2 y = (rv[u] && kk < NGV * ND1) ? yrow[u][g + NGV * NCU * dp] : make_uint2(0u, 0u);
                        ah[u][ks] = y.x;
                        al[u][ks] = y.y;
                    }
                {
                    float acc[G::NTK][4];
#pragma unroll
                    for (int b = 0; b < G::NTK; b++) acc[b][0] = acc[b][1] = acc[b][2] = acc[b][3] = 0.f;
#pragma unroll
                    for (int s8 = 0; s8 < (KS + 1) / 2; s8++) {
                        const int k0 = 2 * s8, k1 = 2 * s8 + 1;
                        const uint32_t fh[4] = {ah[0][k0], ah[1][k0], k1 < KS ? ah[0][k1 < KS ? k1 : 0] : 0u,
                                                k1 < KS ? ah[1][k1 < KS ? k1 : 0] : 0u};
                        const uint32_t fl[4] = {al[0][k0], al[1][k0], k1 < KS ? al[0][k1 < KS ? k1 : 0] : 0u,
                                                k1 < KS ? al[1][k1 < KS ? k1 : 0] : 0u};
#pragma unroll
                        for (int b = 0; b < G::NTK; b++) {
                            const uint2 b0 = Phi2[(8 * s8 + gc) + G::LDBD * (8 * b + gr)];
                            const uint2 b1 = k1 < KS ? Phi2[(8 * s8 + 4 + gc) + G::LDBD * (8 * b + gr)] : make_uint2(0u, 0u);
                            mma_3xtf32(acc[b], fh, fl, b0, b1);
                        }
                    }
#pragma unroll
                    for (int u = 0; u < 2; u++) {
                        if (!rv[u]) continue;
                        const int i = rr[u] % NPV, j = (rr[u] / NPV) % NCU, k = rr[u] / (NPV * NCU);
#pragma unroll
                        for (int b = 0; b < G::NTK; b++)
#pragma unroll
                            for (int h = 0; h < 2; h++) {
                                const int a = 8 * b + 2 * gc + h;
                                if (a < NPV) De[i + NPV * (j + NCU * (a + NPV * k))] = (double)acc[b][2 * u + h];
                            }
                    }
                }
                uint32_t qh[2][KSQ], ql[2][KSQ];
#pragma unroll
                for (int u = 0; u < 2; u++)
#pragma unroll
                    for (int ks = 0; ks < KSQ; ks++) {
                        if constexpr (SHIFT) {
                            qh[u][ks] = ah[u][ks + NGV / 4];
                            ql[u][ks] = al[u][ks + NGV / 4];
                        } else {
                            const int kk = 4 * ks + gc, g = kk % NGV, d = kk / NGV;
                            const uint2 y =
                                (rv[u] && kk < NGV * ND) ? yrow[u][g + NGV * NCU * (d + 1)] : make_uint2(0u, 0u);
                            qh[u][ks] = y.x;
                            ql[u][ks] = y.y;
                        }
                    }
                float accf[G::NTH][4];
#pragma unroll
                for (int b = 0; b < G::NTH; b++) accf[b][0] = accf[b][1] = accf[b][2] = accf[b][3] = 0.f;
#pragma unroll
                for (int s8 = 0; s8 < (KSQ + 1) / 2; s8++) {
                    const int k0 = 2 * s8, k1 = 2 * s8 + 1;
                    const uint32_t fh[4] = {qh[0][k0], qh[1][k0], k1 < KSQ ? qh[0][k1 < KSQ ? k1 : 0] : 0u,
                                            k1 < KSQ ? qh[1][k1 < KSQ ? k1 : 0] : 0u};
                    const uint32_t fl[4] = {ql[0][k0], ql[1][k0], k1 < KSQ ? ql[0][k1 < KSQ ? k1 : 0] : 0u,
                                            k1 < KSQ ? ql[1][k1 < KSQ ? k1 : 0] : 0u};
#pragma unroll
                    for (int b = 0; b < G::NTH; b++) {
                        const uint2 b0 = Psi2[(8 * s8 + gc) + G::LDBD * (8 * b + gr)];
                        const uint2 b1 = k1 < KSQ ? Psi2[(8 * s8 + 4 + gc) + G::LDBD * (8 * b + gr)] : make_uint2(0u, 0u);
                        mma_3xtf32(accf[b], fh, fl, b0, b1);
                    }
                }
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    if (!rv[u]) continue;
                    const int i = rr[u] % NPV, j = (rr[u] / NPV) % NCU, k = rr[u] / (NPV * NCU);
#pragma unroll
                    for (int b = 0; b < G::NTH; b++)
#pragma unroll
                        for (int h = 0; h < 2; h++) {
                            const int f2 = 8 * b + 2 * gc + h;
                            if (f2 < NDF) Fe[i + NPV * (j + NCU * (k + NCH * f2))] = (double)accf[b][2 * u + h];
                        }
                }
            }
            }
        }
        // ---- Ru = Ru_vol + P Rh (fhat on every face) and ||Ru||^2
        double ru2 = 0.0;
        for (int t = tid; t < N; t += NT) {
            const int i = t % NPV, j = t / NPV;
            double s = 0.0;
            for (int q = 0; q < NQ; q++) s += sm.Av[i + G::LDAV * q] * sm.wrk[q + NQ * j];
            for (int c2 = 0; c2 < sm.inc_n[i]; c2++) s += sm.rh[j + NCH * sm.inc_f[i * S::MAXINC + c2]];
            A.Ru[(size_t)e * N + t] = s;
            ru2 += s * s;
        }
        const double tot = block_sum(ru2, sm.red);
        if (tid == 0) A.ru2[e] = tot;

        // ---- K and H face by face: rows (ip, j, m), k = (q, d'), generated A = shapfg(ip,q) x fhn.
        // store: the rows are the face's trace equations (K, H); liftD / liftF:
        // they are added to the element equations of the face's nodes
        // (D += P K, F += P H) by reductions in L2, face after face
        auto face_rows = [&](int fc, const double* slices, bool store, bool liftD, bool liftF) {
            bulk_proxy_fence();
            __syncthreads();
            double* BK = Bs;                              // KFD x NKP  (ld LDBK)
            double* BH = Bs + G::LDBK * G::NKP;           // KFD x NHP  (ld LDBK)
            double* sfu = Bs + G::BKH;                    // the face's slices
            double* sfuh = sfu + NGF * NCH * NC;
            // the slices arrive by one bulk copy (TMA engine) while B is built
            if (tid == 0) {
                bulk_bar_expect(&sm.bar_sl, G::FSLP * 8);
                bulk_load(sfu, slices, G::FSLP * 8, &sm.bar_sl);
            }
            // d' = 0 rows (the face basis at the face's nodes) directly (the zero
            // padding is written once per element, before the first face); rows
            // d' > 0 = shapfc (M^-1 C | M^-1 E)(face nodes) on the tensor cores
            for (int t = tid; t < NGF * (NPV + NDF); t += NT) {
                const int q = t % NGF, c = t / NGF;
                if (c < NPV) {
                    const int p = sm.pos[fc * NPV + c];
                    bput<TF>(&BK[q + G::LDBK * c], (p >= 0) ? sm.sfc[q + NGF * p] : 0.0);
                } else {
                    const int f2 = c - NPV;
                    bput<TF>(&BH[q + G::LDBK * f2], (f2 / NPF == fc) ? sm.sfc[q + NGF * (f2 % NPF)] : 0.0);
                }
            }
            basis_ce_gemm<NGF, NPF, NPV, NPV * ND + NDF * ND, NT / 32>(
                sm.sfc, NGF, sm.perm + fc * NPF, Cm, [&](int q, int n, double v) {
                    if (n < NPV * ND) {
                        const int a = n % NPV, d = n / NPV;
                        bput<TF>(&BK[(q + NGF * (d + 1)) + G::LDBK * a], v);
                    } else {
                        const int f2 = (n - NPV * ND) % NDF, d = (n - NPV * ND) / NDF;
                        bput<TF>(&BH[(q + NGF * (d + 1)) + G::LDBK * f2], -v);
                    }
                });
            if (!bulk_bar_wait(&sm.bar_sl, ph_sl) && tid == 0 && A.err) atomicExch(A.err, 2);
            ph_sl ^= 1u;
            __syncthreads();
            constexpr int MTK = (NPF * NCH * NCU + 7) / 8;
            constexpr int KH0 = (NGF + 3) / 4;            // k-steps holding d' = 0 rows
            // the d' = 0 rows of BH are zero outside the face's own columns
            // fc NPF .. fc NPF + NPF - 1: those n-tiles are skipped there
            const int blo = (fc * NPF) / 8, bhi = (fc * NPF + NPF - 1) / 8;
            if constexpr (!TF) {
            // m-tiles in pairs, as in the volume GEMM: one B fragment, two DMMAs
            for (int mp = warp; 2 * mp < MTK; mp += NT / 32) {
                int jj[2], ipp[2], mm[2], inode[2];
                bool rv[2];
                double aK[2][G::KFD / 4], aH0[2][KH0];
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    const int r = 8 * (2 * mp + u) + gr;
                    rv[u] = r < NPF * NCH * NCU;
                    // j fastest: the 8 rows of a tile are 8 consecutive words of a K/H column
                    jj[u] = r % NCH, ipp[u] = (r / NCH) % NPF, mm[u] = r / (NPF * NCH);
                    inode[u] = sm.perm[fc * NPF + ipp[u]];
#pragma unroll
                    for (int ks = 0; ks < G::KFD / 4; ks++) {
                        const int k = 4 * ks + gc, q = k % NGF, dp = k / NGF;
                        double vK = 0.0, vH = 0.0;
                        if (rv[u] && k < NGF * ND1) {
                            const double sf = sm.Af[ipp[u] + G::LDAF * q];
                            if (dp == 0) {
                                vK = sf * sfu[q + NGF * (jj[u] + NCH * mm[u])];
                                vH = sf * sfuh[q + NGF * (jj[u] + NCH * mm[u])];
                            } else {
                                vK = sf * sfu[q + NGF * (jj[u] + NCH * (NCU * dp + mm[u]))];
                                vH = vK;
                            }
                        }
                        aK[u][ks] = vK;
                        if (ks < KH0) aH0[u][ks] = vH;
                    }
                }
                double acc[2][G::NTK][2];
#pragma unroll
                for (int u = 0; u < 2; u++)
#pragma unroll
                    for (int b = 0; b < G::NTK; b++) acc[u][b][0] = acc[u][b][1] = 0.0;
#pragma unroll
                for (int ks = 0; ks < G::KFD / 4; ks++)
#pragma unroll
                    for (int b = 0; b < G::NTK; b++) {
                        const double bv = BK[(4 * ks + gc) + G::LDBK * (8 * b + gr)];
                        dmma8x8x4(acc[0][b][0], acc[0][b][1], aK[0][ks], bv);
                        dmma8x8x4(acc[1][b][0], acc[1][b][1], aK[1][ks], bv);
                    }
#pragma unroll
                for (int u = 0; u < 2; u++)
#pragma unroll
                    for (int b = 0; b < G::NTK; b++)
#pragma unroll
                        for (int h = 0; h < 2; h++) {
                            const int a = 8 * b + 2 * gc + h;
                            if (rv[u] && a < NPV) {
                                const int j = jj[u], ip = ipp[u], m = mm[u];
                                if (store) Ke[j + NCH * (fc * NPF + ip) + (size_t)NB * (a + NPV * m)] = acc[u][b][h];
                                if (liftD) atomicAdd(&De[inode[u] + NPV * (j + NCU * (a + NPV * m))], acc[u][b][h]);
                            }
                        }
                // H in two column halves: half the accumulators live at a time
                auto hpart = [&](auto b0c, auto nbc) {
                    constexpr int B0 = decltype(b0c)::value, NBN = decltype(nbc)::value;
                    double acch[2][NBN][2];
#pragma unroll
                    for (int u = 0; u < 2; u++)
#pragma unroll
                        for (int b = 0; b < NBN; b++) acch[u][b][0] = acch[u][b][1] = 0.0;
#pragma unroll
                    for (int ks = 0; ks < G::KFD / 4; ks++)
#pragma unroll
                        for (int bb = 0; bb < NBN; bb++) {
                            const int b = B0 + bb;
                            if (4 * ks + 3 < NGF && (b < blo || b > bhi)) continue;
                            const double bv = BH[(4 * ks + gc) + G::LDBK * (8 * b + gr)];
                            dmma8x8x4(acch[0][bb][0], acch[0][bb][1], ks < KH0 ? aH0[0][ks < KH0 ? ks : 0] : aK[0][ks], bv);
                            dmma8x8x4(acch[1][bb][0], acch[1][bb][1], ks < KH0 ? aH0[1][ks < KH0 ? ks : 0] : aK[1][ks], bv);
                        }
#pragma unroll
                    for (int u = 0; u < 2; u++)
#pragma unroll
                        for (int bb = 0; bb < NBN; bb++)
#pragma unroll
                            for (int h = 0; h < 2; h++) {
                                const int f2 = 8 * (B0 + bb) + 2 * gc + h;
                                if (rv[u] && f2 < NDF) {
                                    const int j = jj[u], ip = ipp[u], m = mm[u];
                                    if (store) He[j + NCH * (fc * NPF + ip) + (size_t)NB * (m + NCH * f2)] = acch[u][bb][h];
                                    if (liftF) atomicAdd(&Fe[inode[u] + NPV * (j + NCU * (m + NCH * f2))], acch[u][bb][h]);
                                }
                            }
                };
                constexpr int NTH1 = (G::NTH + 1) / 2;
                hpart(std::integral_constant<int, 0>{}, std::integral_constant<int, NTH1>{});
                if constexpr (G::NTH - NTH1 > 0)
                    hpart(std::integral_constant<int, NTH1>{}, std::integral_constant<int, G::NTH - NTH1>{});
            }
            } else {
            // 3xTF32: the m-tile pair as one m16 tile, k-steps of 8
            const uint2* BK2 = reinterpret_cast<const uint2*>(BK);
            const uint2* BH2 = reinterpret_cast<const uint2*>(BH);
            constexpr int KS = G::KFD / 4;
            for (int mp = warp; 2 * mp < MTK; mp += NT / 32) {
                int jj[2], ipp[2], mm[2], inode[2];
                bool rv[2];
                uint32_t kh[2][KS], kl[2][KS], hh[2][KH0], hl[2][KH0];
#pragma unroll
                for (int u = 0; u < 2; u++) {
                    const int r = 8 * (2 * mp + u) + gr;
                    rv[u] = r < NPF * NCH * NCU;
                    jj[u] = r % NCH, ipp[u] = (r / NCH) % NPF, mm[u] = r / (NPF * NCH);
                    inode[u] = sm.perm[fc * NPF + ipp[u]];
#pragma unroll
                    for (int ks = 0; ks < KS; ks++) {
                        const int k = 4 * ks + gc, q = k % NGF, dp = k / NGF;
                        double vK = 0.0, vH = 0.0;
                        if (rv[u] && k < NGF * ND1) {
                            const double sf = sm.Af[ipp[u] + G::LDAF * q];
                            if (dp == 0) {
                                vK = sf * sfu[q + NGF * (jj[u] + NCH * mm[u])];
                                vH = sf * sfuh[q + NGF * (jj[u] + NCH * mm[u])];
                            } else {
                                vK = sf * sfu[q + NGF * (jj[u] + NCH * (NCU * dp + mm[u]))];
                                vH = vK;
                            }
                        }
                        const uint2 sk = tf32_split(vK);
                        kh[u][ks] = sk.x;
                        kl[u][ks] = sk.y;
                        if (ks < KH0) {
                            const uint2 sh = tf32_split(vH);
                            hh[u][ks < KH0 ? ks : 0] = sh.x;
                            hl[u][ks < KH0 ? ks : 0] = sh.y;
                        }
                    }
                }
                {
                    float acc[G::NTK][4];
#pragma unroll
                    for (int b = 0; b < G::NTK; b++) acc[b][0] = acc[b][1] = acc[b][2] = acc[b][3] = 0.f;
#pragma unroll
                    for (int s8 = 0; s8 < (KS + 1) / 2; s8++) {
                        const int k0 = 2 * s8, k1 = 2 * s8 + 1, k1c = k1 < KS ? k1 : 0;
                        const uint32_t fh[4] = {kh[0][k0], kh[1][k0], k1 < KS ? kh[0][k1c] : 0u, k1 < KS ? kh[1][k1c] : 0u};
                        const uint32_t fl[4] = {kl[0][k0], kl[1][k0], k1 < KS ? kl[0][k1c] : 0u, k1 < KS ? kl[1][k1c] : 0u};
#pragma unroll
                        for (int b = 0; b < G::NTK; b++) {
                            const uint2 b0 = BK2[(8 * s8 + gc) + G::LDBK * (8 * b + gr)];
                            const uint2 b1 = k1 < KS ? BK2[(8 * s8 + 4 + gc) + G::LDBK * (8 * b + gr)] : make_uint2(0u, 0u);
                            mma_3xtf32(acc[b], fh, fl, b0, b1);
                        }
                    }
#pragma unroll
                    for (int u = 0; u < 2; u++)
#pragma unroll
                        for (int b = 0; b < G::NTK; b++)
#pragma unroll
                            for (int h = 0; h < 2; h++) {
                                const int a = 8 * b + 2 * gc + h;
                                if (rv[u] && a < NPV) {
                                    const int j = jj[u], ip = ipp[u], m = mm[u];
                                    const double v = (double)acc[b][2 * u + h];
                                    if (store) Ke[j + NCH * (fc * NPF + ip) + (size_t)NB * (a + NPV * m)] = v;
                                    if (liftD) atomicAdd(&De[inode[u] + NPV * (j + NCU * (a + NPV * m))], v);
                                }
                            }
                }
                float acch[G::NTH][4];
#pragma unroll
                for (int b = 0; b < G::NTH; b++) acch[b][0] = acch[b][1] = acch[b][2] = acch[b][3] = 0.f;
#pragma unroll
                for (int s8 = 0; s8 < (KS + 1) / 2; s8++) {
                    const int k0 = 2 * s8, k1 = 2 * s8 + 1, k1c = k1 < KS ? k1 : 0;
                    // entries of k4-step ks: the d' = 0 values for ks < KH0, else K's
                    auto eh = [&](int u, int ks) { return ks < KH0 ? hh[u][ks < KH0 ? ks : 0] : kh[u][ks]; };
                    auto el = [&](int u, int ks) { return ks < KH0 ? hl[u][ks < KH0 ? ks : 0] : kl[u][ks]; };
                    const uint32_t fh[4] = {eh(0, k0), eh(1, k0), k1 < KS ? eh(0, k1c) : 0u, k1 < KS ? eh(1, k1c) : 0u};
                    const uint32_t fl[4] = {el(0, k0), el(1, k0), k1 < KS ? el(0, k1c) : 0u, k1 < KS ? el(1, k1c) : 0u};
#pragma unroll
                    for (int b = 0; b < G::NTH; b++) {
                        if (4 * k1 + 3 < NGF && (b < blo || b > bhi)) continue;
                        const uint2 b0 = BH2[(8 * s8 + gc) + G::LDBK * (8 * b + gr)];
                        const uint2 b1 = k1 < KS ? BH2[(8 * s8 + 4 + gc) + G::LDBK * (8 * b + gr)] : make_uint2(0u, 0u);
                        mma_3xtf32(acch[b], fh, fl, b0, b1);
                    }
                }
#pragma unroll
                for (int u = 0; u < 2; u++)
#pragma unroll
                    for (int b = 0; b < G::NTH; b++)
#pragma unroll
                        for (int h = 0; h < 2; h++) {
                            const int f2 = 8 * b + 2 * gc + h;
                            if (rv[u] && f2 < NDF) {
                                const int j = jj[u], ip = ipp[u], m = mm[u];
                                const double v = (double)acch[b][2 * u + h];
                                if (store) He[j + NCH * (fc * NPF + ip) + (size_t)NB * (m + NCH * f2)] = v;
                                if (liftF) atomicAdd(&Fe[inode[u] + NPV * (j + NCU * (m + NCH * f2))], v);
                            }
                        }
            }
            }
        };
        // zero padding of the face B operands (rows past NGF ND1, columns past
        // npv and ndf), the same for every face
        {
            double* BK = Bs;
            double* BH = Bs + G::LDBK * G::NKP;
            for (int t = tid; t < G::KFD * G::NKP; t += NT) {
                const int k = t % G::KFD, a = t / G::KFD;
                if (k >= NGF * ND1 || a >= NPV) bput<TF>(&BK[k + G::LDBK * a], 0.0);
            }
            for (int t = tid; t < G::KFD * G::NHP; t += NT) {
                const int k = t % G::KFD, f2 = t / G::KFD;
                if (k >= NGF * ND1 || f2 >= NDF) bput<TF>(&BH[k + G::LDBK * f2], 0.0);
            }
        }
        for (int fc = 0; fc < NFE; fc++) {
            const bool bnd = bfe && bfe[fc] < 0;
            // interior faces: the trace rows, lifted into D; boundary faces: fhat
            // rows lifted into D and F
            face_rows(fc, fsl + fc * G::FSLP, !bnd, true, bnd);
            if (bnd) {
                // the boundary face's trace equations take the boundary flux
                // (faceint 1075-1246)
                for (int t = tid; t < NPF * NCH; t += NT) {
                    const int j = t % NCH, ip = t / NCH;
                    double s = 0.0;
                    for (int q = 0; q < NGF; q++) s += sm.Af[ip + G::LDAF * q] * fnb[q + NGF * fc + NA * j];
                    Rhe[j + NCH * (fc * NPF + ip)] = -s;
                    Roe[j + NCH * (fc * NPF + ip)] = -s;
                }
                face_rows(fc, fslb + fc * G::FSLP, true, false, false);
            }
        }
    }
}

}  // namespace hfem
