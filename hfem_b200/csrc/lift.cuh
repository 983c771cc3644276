// Interior-face lift of the trace rows into the element rows (faceint,
// elementassembly.cpp:903-924).
//
// The face terms of the element equations are the trace-equation entries moved
// to the element node that carries the face dof, so
//   D = D_vol + P K,   F = F_vol + P H,
// with P the node <- face-dof incidence given by perm.  The element kernel
// writes D (lifted), F_vol and the trace rows K, H; lift_inplace_kernel adds
// P H to F between the element kernel and the condensation, one coalesced pass
// instead of reductions in L2 from the element kernel.  Boundary faces are
// lifted by the element kernel itself (their trace rows take the boundary flux
// while their element rows keep fhat), so the lift here skips them.
//
// Row r = i + npv j of D (or F) with column c receives, for every interior face
// dof fdof of node i in increasing order (the order of the reference's face
// loop), src[j + nch fdof + nb c] of the element's K (or H).
#pragma once
#include <cuda_runtime.h>

namespace hfem {

constexpr int LIFT_MAXNPV = 32;   // nodes per element (20 for the tetrahedron p = 3)
constexpr int LIFT_MAXINC = 3;    // faces meeting at a node (nd)

struct LiftArgs {
    const double* src = nullptr;  // K (for D) or H (for F): per element nb x cols; NULL: no lift
    const int* perm = nullptr;    // npf x nfe, device
    const int* bf = nullptr;      // ne x nfe, < 0 on boundary faces; NULL: no boundary faces
    int npv = 0, npf = 0, nfe = 0, nch = 0, cols = 0;
};

struct LiftTable {
    int n[LIFT_MAXNPV];                     // face dofs of node i
    int f[LIFT_MAXNPV * LIFT_MAXINC];       // ... ascending
};

// Fills the node -> face-dof table from perm (one CTA; the caller syncs).
__device__ __forceinline__ void lift_table(const LiftArgs& L, LiftTable& t) {
    if (!L.src) return;
    for (int i = threadIdx.x; i < L.npv; i += blockDim.x) {
        int c = 0;
        for (int f = 0; f < L.npf * L.nfe; f++)
            if (L.perm[f] == i && c < LIFT_MAXINC) t.f[i * LIFT_MAXINC + c++] = f;
        t.n[i] = c;
    }
}

// v plus the lifted trace entries of row `row` of element e, one column; hs is
// that column of the element's src (K or H), already in shared memory.
__device__ __forceinline__ double lift_add_col(const LiftArgs& L, const LiftTable& t, int e, int row,
                                              const double* hs, double v) {
    const int i = row % L.npv, j = row / L.npv;
    const int cnt = t.n[i];
    for (int q = 0; q < cnt; q++) {
        const int fdof = t.f[i * LIFT_MAXINC + q];
        if (L.bf && L.bf[(size_t)e * L.nfe + fdof / L.npf] < 0) continue;
        v += hs[j + L.nch * fdof];
    }
    return v;
}

// T += P src in place for every element (rows x cols per element, column-major):
// the lift on its own, ahead of a condensation kernel that reads T whole.  One
// warp per column: the column of src (nb values) is read coalesced into shared
// memory, then the warp's lanes update the column of T from it.
constexpr int LIFT_WARPS = 8;
constexpr int LIFT_MAXNB = 200;                  // trace dofs per element (tetrahedron p = 3)

__global__ void __launch_bounds__(32 * LIFT_WARPS) lift_inplace_kernel(int ne, int rows, LiftArgs L,
                                                                       double* __restrict__ T) {
    __shared__ LiftTable tab;
    __shared__ double hs[LIFT_WARPS][LIFT_MAXNB];
    lift_table(L, tab);
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nb = L.nch * L.npf * L.nfe;
    const long long ncol = (long long)ne * L.cols;
    for (long long col = (long long)blockIdx.x * LIFT_WARPS + w; col < ncol; col += (long long)gridDim.x * LIFT_WARPS) {
        const int e = (int)(col / L.cols), c = (int)(col - (long long)e * L.cols);
        const double* src = L.src + (size_t)e * nb * L.cols + (size_t)nb * c;
        for (int r = lane; r < nb; r += 32) hs[w][r] = src[r];
        __syncwarp();
        double* t = T + (size_t)e * rows * L.cols + (size_t)rows * c;
        for (int r = lane; r < rows; r += 32) t[r] = lift_add_col(L, tab, e, r, hs[w], t[r]);
        __syncwarp();
    }
}

}  // namespace hfem
