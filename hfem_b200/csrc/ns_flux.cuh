// Compressible Navier-Stokes flux F(u, q) and its Jacobian dF/d(u, q) at one
// point, for the HDG element kernels (sm_100a).
//
// Restates application/FM/nsNew/flux_ns2dNEW.c:22-74 / flux_ns3dNEW.c (the
// reference's symbolically generated flux, constant viscosity mu = 1 from
// FM/getViscosity.c:5-12):
//   f_rho^d = m_d
//   f_mi^d  = m_i v_d + p delta_id + tau_id
//   f_E^d   = (E + p) v_d + sum_i tau_id v_i
//             + gamma/(Re Pr) (q_E^d/rho - E q_rho^d/rho^2 - sum_i v_i dv_i/dx_d)
// with dv_i/dx_d = (q_mi^d - v_i q_rho^d)/rho and
// tau_ij = (1/Re)(dv_i/dx_j + dv_j/dx_i - 2/3 delta_ij div v).
// Variables: w = [rho, m_1..m_nd, E, q_1 (ncu comps), .., q_nd].
//
// The Jacobian is exact forward-mode differentiation (dual numbers).
#pragma once

namespace hfem {

template <int N>
struct Dual {
    double v;
    double d[N];
};

template <int N>
__device__ __forceinline__ Dual<N> dc(double v) {
    Dual<N> r;
    r.v = v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = 0.0;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(double s, const Dual<N>& a) {
    Dual<N> r;
    r.v = s * a.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = s * a.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    const double ib = 1.0 / b.v;
    r.v = a.v * ib;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}

// f[d*ncu + c] for one point; w has ND+2 + (ND+2)*ND entries, each carrying M
// partial derivatives (M = nc for the full Jacobian, 1 for one column of it).
template <int ND, int M>
__device__ __forceinline__ void ns_flux_dual(const double* __restrict__ param, const Dual<M>* w, Dual<M>* f) {
    constexpr int NCU = ND + 2;
    constexpr int NC = M;
    using D = Dual<M>;
    const double gam = param[0], Re = param[2], Pr = param[3];
    const double iRe = 1.0 / Re;
    const D& rho = w[0];
    const D& E = w[ND + 1];
    D v[ND];
    D ke = dc<NC>(0.0);
#pragma unroll
    for (int i = 0; i < ND; i++) {
        v[i] = w[1 + i] / rho;
        ke = ke + v[i] * w[1 + i];
    }
    const D p = (gam - 1.0) * (E - 0.5 * ke);
    D dv[ND][ND];
#pragma unroll
    for (int d = 0; d < ND; d++)
#pragma unroll
        for (int i = 0; i < ND; i++) dv[i][d] = (w[NCU * (1 + d) + 1 + i] - v[i] * w[NCU * (1 + d)]) / rho;
    D div = dv[0][0];
#pragma unroll
    for (int i = 1; i < ND; i++) div = div + dv[i][i];
    const double kappa = gam / (Re * Pr);
#pragma unroll
    for (int d = 0; d < ND; d++) {
        f[d * NCU + 0] = w[1 + d];
        D fe = (E + p) * v[d];
        D vdv = dc<NC>(0.0);
#pragma unroll
        for (int i = 0; i < ND; i++) {
            D t = dv[i][d] + dv[d][i];
            if (i == d) t = t - (2.0 / 3.0) * div;
            t = iRe * t;                                   // tau_id
            D fm = w[1 + i] * v[d] + t;
            if (i == d) fm = fm + p;
            f[d * NCU + 1 + i] = fm;
            fe = fe + t * v[i];
            vdv = vdv + v[i] * dv[i][d];
        }
        const D heat = w[NCU * (1 + d) + ND + 1] / rho - E * w[NCU * (1 + d)] / (rho * rho) - vdv;
        f[d * NCU + ND + 1] = fe + kappa * heat;
    }
}

// Boundary flux fb(u, q, uh) of the NS boundary conditions at one point
// (application/FM/fbou.cpp on a fixed mesh), in dual numbers so that one pass
// per differentiated variable gives fb and its derivative:
//   2 no-slip adiabatic wall: rho - rho_hat, -m_hat, and for energy the
//     interior trace flux F(uh, q).n + tau (E - E_hat);
//   5 Dirichlet: tau (ui - uh);   6 extrapolation: u - uh;
//   7 slip wall: rho - rho_hat, m - (m.n) n - m_hat, E - E_hat.
// w holds (u, q) (NC entries), uh the trace state (NCH); returns false for a
// type without a restatement.
template <int ND, int M>
__device__ __forceinline__ bool ns_fbou_dual(int bn, const double* __restrict__ param, const double* ui,
                                             const double* nl, const Dual<M>* w, const Dual<M>* uh, Dual<M>* fb) {
    constexpr int NCU = ND + 2, NC = NCU * (ND + 1);
    const double tau = param[5];
    if (bn == 2) {
        fb[0] = w[0] - uh[0];
#pragma unroll
        for (int j = 0; j < ND; j++) fb[1 + j] = dc<M>(0.0) - uh[1 + j];
        Dual<M> wf[NC], f[ND * NCU];
#pragma unroll
        for (int k = 0; k < NCU; k++) wf[k] = uh[k];
#pragma unroll
        for (int k = NCU; k < NC; k++) wf[k] = w[k];
        ns_flux_dual<ND, M>(param, wf, f);
        Dual<M> t = tau * (w[ND + 1] - uh[ND + 1]);
#pragma unroll
        for (int d = 0; d < ND; d++) t = t + nl[d] * f[d * NCU + ND + 1];
        fb[ND + 1] = t;
        return true;
    }
    if (bn == 5) {
#pragma unroll
        for (int j = 0; j < NCU; j++) fb[j] = tau * (dc<M>(ui[j]) - uh[j]);
        return true;
    }
    if (bn == 6) {
#pragma unroll
        for (int j = 0; j < NCU; j++) fb[j] = w[j] - uh[j];
        return true;
    }
    if (bn == 7) {
        fb[0] = w[0] - uh[0];
        Dual<M> un = dc<M>(0.0);
#pragma unroll
        for (int i = 0; i < ND; i++) un = un + nl[i] * w[1 + i];
#pragma unroll
        for (int j = 0; j < ND; j++) fb[1 + j] = w[1 + j] - nl[j] * un - uh[1 + j];
        fb[ND + 1] = w[ND + 1] - uh[ND + 1];
        return true;
    }
    return false;
}

}  // namespace hfem
