// Compressible Navier-Stokes flux F(u, q) and its Jacobian dF/d(u, q) at one
// point, for the HDG element kernels (sm_100a).
//
// Restates application/FM/nsNew/flux_ns2dNEW.c:22-74 / flux_ns3dNEW.c (the
// reference's symbolically generated flux, viscosity mu(u) from
// FM/getViscosity.c):
//   f_rho^d = m_d
//   f_mi^d  = m_i v_d + p delta_id + tau_id
//   f_E^d   = (E + p) v_d + sum_i tau_id v_i
//             + mu gamma/(Re Pr) (q_E^d/rho - E q_rho^d/rho^2 - sum_i v_i dv_i/dx_d)
// with dv_i/dx_d = (q_mi^d - v_i q_rho^d)/rho and
// tau_ij = (mu/Re)(dv_i/dx_j + dv_j/dx_i - 2/3 delta_ij div v).
// The trace flux's stabilization tensor (ns_stab_apply) and the boundary
// fluxes (ns_fbou_dual) follow.
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

template <int N>
__device__ __forceinline__ Dual<N> datan(const Dual<N>& a) {
    Dual<N> r;
    r.v = atan(a.v);
    const double h = 1.0 / (1.0 + a.v * a.v);
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * h;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> dpow15(const Dual<N>& a) {       // a^(3/2)
    Dual<N> r;
    r.v = pow(a.v, 1.5);
    const double h = 1.5 * sqrt(a.v);
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * h;
    return r;
}

// Sutherland's law (application/FM/getViscosity.c, sutherlandLaw2d 25-146 and
// sutherlandLaw3d 275-...; app.viscosityModel 1), regularised at zero: with the
// temperature T = (rE - |m|^2/(2 rho)) / (rho gamma (gamma - 1) Mach^2) and
// a = (S + T0) T^(3/2) / (S + T0 T), S = 111, T0 = 300,
//   mu = c + a (atan(b a)/pi + 1/2),  b = 100, c = 1/2 - atan(b)/pi.
template <int ND, int M>
__device__ __forceinline__ Dual<M> ns_sutherland(const double* __restrict__ param, const Dual<M>* w) {
    using D = Dual<M>;
    const double gam = param[0], mach = param[4], S = 111.0, T0 = 300.0, b = 100.0, pi = 3.141592653589793;
    D ke = dc<M>(0.0);
#pragma unroll
    for (int i = 0; i < ND; i++) ke = ke + w[1 + i] * w[1 + i];
    const D T = (w[ND + 1] - 0.5 * (ke / w[0])) / ((gam * (gam - 1.0) * mach * mach) * w[0]);
    const D a = (S + T0) * (dpow15(T) / (dc<M>(S) + T0 * T));
    return dc<M>(0.5 - atan(b) / pi) + a * ((1.0 / pi) * datan(b * a) + dc<M>(0.5));
}

// f[d*ncu + c] for one point; w has ND+2 + (ND+2)*ND entries, each carrying M
// partial derivatives (M = nc for the full Jacobian, 1 for one column of it).
// viscous == false: the Euler flux (flux_euler2dNEW.c / flux_euler3dNEW.c), the
// same expression without the stress and heat terms.  visc_model: 0 mu = 1,
// 1 Sutherland's law (ns_sutherland); GEN false compiles the constant-viscosity
// flux alone.
template <int ND, int M, bool GEN = false>
__device__ __forceinline__ void ns_flux_dual(const double* __restrict__ param, const Dual<M>* w, Dual<M>* f,
                                             bool viscous = true, int visc_model = 0) {
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
    const bool vm = GEN && viscous && visc_model != 0;
    D mu = dc<NC>(1.0);
    if constexpr (GEN) {
        if (vm) mu = ns_sutherland<ND, M>(param, w);
    }
#pragma unroll
    for (int d = 0; d < ND; d++) {
        f[d * NCU + 0] = w[1 + d];
        D fe = (E + p) * v[d];
        D vdv = dc<NC>(0.0);
#pragma unroll
        for (int i = 0; i < ND; i++) {
            D t = dv[i][d] + dv[d][i];
            if (i == d) t = t - (2.0 / 3.0) * div;
            t = viscous ? iRe * (vm ? mu * t : t) : dc<NC>(0.0);   // tau_id
            D fm = w[1 + i] * v[d] + t;
            if (i == d) fm = fm + p;
            f[d * NCU + 1 + i] = fm;
            fe = fe + t * v[i];
            vdv = vdv + v[i] * dv[i][d];
        }
        const D heat = w[NCU * (1 + d) + ND + 1] / rho - E * w[NCU * (1 + d)] / (rho * rho) - vdv;
        f[d * NCU + ND + 1] = viscous ? fe + kappa * (vm ? mu * heat : heat) : fe;
    }
}

template <int N>
__device__ __forceinline__ Dual<N> dsqrt(const Dual<N>& a) {
    Dual<N> r;
    r.v = sqrt(a.v);
    const double h = 0.5 / r.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * h;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> dabs(const Dual<N>& a) {
    return a.v < 0.0 ? (-1.0) * a : a;
}

// Free-stream far field (application/FM/fbou.cpp:126-218):
//   fb = (A_n + |A_n|)(u - uh) - (A_n - |A_n|)(ui - uh)
// with the Euler normal-flux Jacobian A_n at uh and |A_n| = R |Lambda| R^-1 in the
// closed form of application/FM/getan.c (eigenvalues un + c, un - c, un; with
// eps > 0 the eigenvalues below eps c are smoothed as there).  Column k of
// either matrix is lam3 e_k + cc1_k [1, v, h] + cc2_k [0, n, un]; the matrices
// are applied column by column without being stored.
template <int ND, int M>
__device__ __forceinline__ void ns_farfield_dual(const double* __restrict__ param, const double* ui, const double* nl,
                                                 const Dual<M>* w, const Dual<M>* uh, Dual<M>* fb) {
    constexpr int NCU = ND + 2;
    using D = Dual<M>;
    const double gam = param[0], eps = param[1], g1 = gam - 1.0;
    const D r = uh[0];
    D uv[ND], af = dc<M>(0.0), un = dc<M>(0.0);
#pragma unroll
    for (int i = 0; i < ND; i++) {
        uv[i] = uh[1 + i] / r;
        af = af + 0.5 * (uv[i] * uv[i]);
        un = un + nl[i] * uv[i];
    }
    const D E = uh[ND + 1] / r;
    const D p = g1 * (uh[ND + 1] - r * af);
    const D h = E + p / r;
    const D c2 = gam * (p / r);
    const D c = dsqrt(c2);
    D la[3] = {un + c, un - c, un}, lb[3];
#pragma unroll
    for (int m = 0; m < 3; m++) {
        lb[m] = dabs(la[m]);
        if (eps > 0.0 && lb[m].v < eps * c.v) lb[m] = 0.5 * (lb[m] * lb[m] / (eps * c) + eps * c);
    }
    const D s1a = 0.5 * (la[0] + la[1]), s2a = 0.5 * (la[0] - la[1]);
    const D s1b = 0.5 * (lb[0] + lb[1]), s2b = 0.5 * (lb[0] - lb[1]);
#pragma unroll
    for (int j = 0; j < NCU; j++) fb[j] = dc<M>(0.0);
#pragma unroll
    for (int k = 0; k < NCU; k++) {
        const D a = (k == 0) ? af : (k == ND + 1 ? dc<M>(1.0) : dc<M>(0.0) - uv[k > 0 ? k - 1 : 0]);
        const D b = (k == 0) ? dc<M>(0.0) - un : (k == ND + 1 ? dc<M>(0.0) : dc<M>(nl[k > 0 ? k - 1 : 0]));
        const D c1a = g1 * ((s1a - la[2]) * a / c2) + s2a * b / c, c2a = g1 * (s2a * a / c) + (s1a - la[2]) * b;
        const D c1b = g1 * ((s1b - lb[2]) * a / c2) + s2b * b / c, c2b = g1 * (s2b * a / c) + (s1b - lb[2]) * b;
        const D du = w[k] - uh[k], di = dc<M>(ui[k]) - uh[k];
#pragma unroll
        for (int j = 0; j < NCU; j++) {
            const D v1 = (j == 0) ? dc<M>(1.0) : (j == ND + 1 ? h : uv[j > 0 ? j - 1 : 0]);
            const D v2 = (j == 0) ? dc<M>(0.0) : (j == ND + 1 ? un : dc<M>(nl[j > 0 ? j - 1 : 0]));
            D Aa = c1a * v1 + c2a * v2, Ab = c1b * v1 + c2b * v2;
            if (j == k) {
                Aa = Aa + la[2];
                Ab = Ab + lb[2];
            }
            fb[j] = fb[j] + (Aa + Ab) * du - (Aa - Ab) * di;
        }
    }
}

// out = tau(uh) v, the convective stabilization tensor of the trace flux
// (application/FM/stabilizationTensor.cpp, getConvectiveStabilizationTensor
// 3439-3456; app.convStabMethod):
//   0 constant: param[5] v (getConstantStabilizationTensor, 9-29);
//   1 Lax-Friedrichs: lam v, lam = |un| + c at uh (3D, 221-425); the 2D routine
//     (31-218) evaluates lam at the fixed state (rho, rho u, rho v, rho E) =
//     (1, 0.9994, 0.0349, 1.7858e4) and has a zero Jacobian: restated as it is;
//   2 Roe (440-1716): |A_n(uh)| v, eigenvalues un + c, un - c, un through the
//     smooth absolute value r(x) = 2 (x (atan(b x)/pi + 1/2) - atan(b)/pi +
//     1/2) - x, b = 10, and, with eps = param[1] > 0, r < eps c replaced by
//     (r^2/(eps c) + eps c)/2; columns lam3 e_k + cc1_k [1, v, h] + cc2_k [0, n, un].
template <int ND, int M>
__device__ __forceinline__ void ns_stab_apply(int method, const double* __restrict__ param, const double* nl,
                                              const Dual<M>* uh, const Dual<M>* v, Dual<M>* out) {
    constexpr int NCU = ND + 2;
    using D = Dual<M>;
    if (method == 0) {
#pragma unroll
        for (int j = 0; j < NCU; j++) out[j] = param[5] * v[j];
        return;
    }
    const double gam = param[0], g1 = gam - 1.0, eps = param[1];
    if (method == 1) {
        D lam;
        if constexpr (ND == 2) {
            const double r = 1.0, ru = 0.9994, rv = 0.0349, rE = 1.7858e+04;
            const double uv = ru / r, vv = rv / r, af = 0.5 * (uv * uv + vv * vv), p = g1 * (rE - r * af);
            const double c = sqrt(gam * p / r), un = uv * nl[0] + vv * nl[1];
            lam = dc<M>(un >= 0 ? un + c : -un + c);
        } else {
            const D r = uh[0];
            D af = dc<M>(0.0), un = dc<M>(0.0);
#pragma unroll
            for (int i = 0; i < ND; i++) {
                const D vi = uh[1 + i] / r;
                af = af + 0.5 * (vi * vi);
                un = un + nl[i] * vi;
            }
            const D p = g1 * (uh[ND + 1] - r * af);
            const D c = dsqrt(gam * (p / r));
            lam = un.v >= 0 ? un + c : c - un;
        }
#pragma unroll
        for (int j = 0; j < NCU; j++) out[j] = lam * v[j];
        return;
    }
    const double b = 10.0, pi = 3.141592653589793;
    const D r = uh[0];
    D uv[ND], af = dc<M>(0.0), un = dc<M>(0.0);
#pragma unroll
    for (int i = 0; i < ND; i++) {
        uv[i] = uh[1 + i] / r;
        af = af + 0.5 * (uv[i] * uv[i]);
        un = un + nl[i] * uv[i];
    }
    const D E = uh[ND + 1] / r;
    const D p = g1 * (uh[ND + 1] - r * af);
    const D h = E + p / r;
    const D c2 = gam * (p / r);
    const D c = dsqrt(c2);
    D rl[3] = {un + c, un - c, un};
#pragma unroll
    for (int m = 0; m < 3; m++) {
        const D x = rl[m];
        rl[m] = 2.0 * (x * ((1.0 / pi) * datan(b * x) + dc<M>(0.5)) + dc<M>(0.5 - atan(b) / pi)) - x;
        if (eps > 0.0 && rl[m].v < eps * c.v) rl[m] = 0.5 * (rl[m] * rl[m] / (eps * c) + eps * c);
    }
    const D s1 = 0.5 * (rl[0] + rl[1]), s2 = 0.5 * (rl[0] - rl[1]), l3 = rl[2];
#pragma unroll
    for (int j = 0; j < NCU; j++) out[j] = dc<M>(0.0);
#pragma unroll
    for (int k = 0; k < NCU; k++) {
        const D a = (k == 0) ? af : (k == ND + 1 ? dc<M>(1.0) : dc<M>(0.0) - uv[k > 0 ? k - 1 : 0]);
        const D bb = (k == 0) ? dc<M>(0.0) - un : (k == ND + 1 ? dc<M>(0.0) : dc<M>(nl[k > 0 ? k - 1 : 0]));
        const D cc1 = g1 * ((s1 - l3) * a / c2) + s2 * bb / c;
        const D cc2 = g1 * (s2 * a / c) + (s1 - l3) * bb;
#pragma unroll
        for (int j = 0; j < NCU; j++) {
            const D v1 = (j == 0) ? dc<M>(1.0) : (j == ND + 1 ? h : uv[j > 0 ? j - 1 : 0]);
            const D v2 = (j == 0) ? dc<M>(0.0) : (j == ND + 1 ? un : dc<M>(nl[j > 0 ? j - 1 : 0]));
            D m = cc1 * v1 + cc2 * v2;
            if (j == k) m = m + l3;
            out[j] = out[j] + m * v[k];
        }
    }
}

// The stabilization term of fhat at one face point for the element kernel's
// flux pass: sv = tau(uh)(u - uh), sd = its derivative along uh_k (k < ncu;
// 0 otherwise), tcol = column k of tau (k < ncu).
template <int ND>
__device__ __forceinline__ void ns_stab_point(int method, const double* __restrict__ param, const double* nl,
                                           const double* uh, const double* u, int k, double* sv, double* sd,
                                           double* tcol) {
    constexpr int NCU = ND + 2;
    using DD = Dual<1>;
    DD uhd[NCU], dv[NCU], st[NCU];
#pragma unroll
    for (int m = 0; m < NCU; m++) {
        uhd[m].v = uh[m];
        uhd[m].d[0] = (m == k) ? 1.0 : 0.0;
        dv[m] = dc<1>(u[m]) - uhd[m];
    }
    ns_stab_apply<ND, 1>(method, param, nl, uhd, dv, st);
#pragma unroll
    for (int j = 0; j < NCU; j++) {
        sv[j] = st[j].v;
        sd[j] = st[j].d[0];
    }
    if (k < NCU) {
#pragma unroll
        for (int m = 0; m < NCU; m++) {
            uhd[m] = dc<1>(uh[m]);
            dv[m] = dc<1>(m == k ? 1.0 : 0.0);
        }
        ns_stab_apply<ND, 1>(method, param, nl, uhd, dv, st);
#pragma unroll
        for (int j = 0; j < NCU; j++) tcol[j] = st[j].v;
    }
}

// Boundary flux fb(u, q, uh) of the NS boundary conditions at one point
// (application/FM/fbou.cpp on a fixed mesh), in dual numbers so that one pass
// per differentiated variable gives fb and its derivative:
//   1 free-stream far field (ns_farfield_dual);
//   2 no-slip adiabatic wall: rho - rho_hat, -m_hat, and for energy the
//     interior trace flux F(uh, q).n + [tau(uh) (u - uh)]_E (ns_stab_apply);
//   5 Dirichlet: tau (ui - uh);   6 extrapolation: u - uh;
//   7 slip wall: rho - rho_hat, m - (m.n) n - m_hat, E - E_hat.
// w holds (u, q) (NC entries), uh the trace state (NCH); returns false for a
// type without a restatement.
template <int ND, int M, bool GEN = false>
__device__ __forceinline__ bool ns_fbou_dual(int bn, const double* __restrict__ param, const double* ui,
                                             const double* nl, const Dual<M>* w, const Dual<M>* uh, Dual<M>* fb,
                                             bool viscous = true, int conv_stab = 0, int visc_model = 0) {
    constexpr int NCU = ND + 2, NC = NCU * (ND + 1);
    const double tau = param[5];
    if (bn == 1) {
        ns_farfield_dual<ND, M>(param, ui, nl, w, uh, fb);
        return true;
    }
    if (bn == 2) {
        fb[0] = w[0] - uh[0];
#pragma unroll
        for (int j = 0; j < ND; j++) fb[1 + j] = dc<M>(0.0) - uh[1 + j];
        Dual<M> wf[NC], f[ND * NCU];
#pragma unroll
        for (int k = 0; k < NCU; k++) wf[k] = uh[k];
#pragma unroll
        for (int k = NCU; k < NC; k++) wf[k] = w[k];
        ns_flux_dual<ND, M, GEN>(param, wf, f, viscous, visc_model);
        Dual<M> t;
        if (!GEN || conv_stab == 0) {
            t = tau * (w[ND + 1] - uh[ND + 1]);
        } else {
            Dual<M> du[NCU], st[NCU];
#pragma unroll
            for (int k = 0; k < NCU; k++) du[k] = w[k] - uh[k];
            ns_stab_apply<ND, M>(conv_stab, param, nl, uh, du, st);
            t = st[ND + 1];
        }
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
