// Restatements of the four routines the reference ships only as closed
// archives (gmres/*.a, preprocessing/dmdserlib.a) -- TEST INFRASTRUCTURE ONLY.
//
// They are compiled into oracle/_ref/hfem_ref together with the reference's own
// sources so that its serial driver links.  None of the archives is read or
// linked.  The algorithms follow the readable MATLAB specifications:
//   dmdserial             face-to-face block CSR with the diagonal block first
//                         (kernel/computeBILU0.m:15-17, kernel/mkBlockJacobi.m:10)
//   computeOrdering       identity (reorderMethod 0), else minimum discarded
//                         fill (kernel/computeMDFordering.m:1-150) for BILU0
//   computePreconditioner 0: block ILU(0) in that order (kernel/computeBILU0.m);
//                         2: block Jacobi, inverse of each row's diagonal block
//                         (kernel/mkBlockJacobi.m:1-16); -1 = none
//   gmres                 restarted GMRES with left preconditioning and MGS
//                         (kernel/gmres_bilu0.m:17-105), via oracle_gmres
//
// This file is included into the harness translation unit after the reference
// headers, so the reference's struct definitions are visible here.
#include <algorithm>
#include <set>
#include <vector>

extern "C" {
int oracle_bj_inverse(int nrows, int bsz, const int* rowstart, const double* Hg, double* Minv);
int oracle_gmres(int nrows, int bsz, const int* rowstart, const int* colidx, const double* Hg,
                 const double* Minv, const double* b, double* x, int restart, double tol, int maxit,
                 int* iters, double* hist, int hist_len);
int oracle_mdf_ordering(int nrows, int bsz, const int* rowstart, const int* colidx, const double* Hg,
                        int* o2u, int* u2o);
int oracle_bilu0_factor(int nrows, int bsz, const int* rowstart, const int* colidx, const double* Hg,
                        const int* o2u, const int* u2o, double* Mg);
int oracle_gmres_bilu0(int nrows, int bsz, const int* rowstart, const int* colidx, const double* Hg,
                       const double* Mg, const int* o2u, const int* u2o, const double* b, double* x, int restart,
                       double tol, int maxit, int* iters, double* hist, int hist_len);
}

// GMRES residual histories and the assembly residual seen by each linear solve.
static std::vector<double> g_gmres_hist;
static std::vector<int> g_gmres_iters;
static std::vector<double> g_newton_rnorm;
static solstruct* g_sol = nullptr;

#include "ref_dmdserial.cpp"

void computeOrdering(sysstruct& sys, Int preconditioner)
{
    if (preconditioner == 0 && sys.reorderMethod != 0) {
        if (oracle_mdf_ordering(sys.numEntities, sys.blkSize, &sys.ent2entStart[0], &sys.ent2ent[0], &sys.Hg[0],
                                &sys.ordered2unordered[0], &sys.unordered2ordered[0]) != 0)
            error("singular diagonal block in the MDF ordering");
        return;
    }
    for (Int i = 0; i < sys.numEntities; i++) {
        sys.ordered2unordered[i] = i;
        sys.unordered2ordered[i] = i;
    }
}

void computePreconditioner(sysstruct& sys, Int preconditioner)
{
    if (preconditioner == -1) return;
    if (preconditioner == 0) {
        oracle_bilu0_factor(sys.numEntities, sys.blkSize, &sys.ent2entStart[0], &sys.ent2ent[0], &sys.Hg[0],
                            &sys.ordered2unordered[0], &sys.unordered2ordered[0], &sys.Mg[0]);
        return;
    }
    if (preconditioner != 2) error("only BILU0 (0), block Jacobi (2) and none (-1) are restated");
    const Int bsz = sys.blkSize;
    if (oracle_bj_inverse(sys.numEntities, bsz, &sys.ent2entStart[0], &sys.Hg[0], &sys.Mg[0]) != 0)
        error("singular diagonal block in block Jacobi");
}

void gmres(sysstruct& sys, Int* convFlag)
{
    const Int N = sys.numEntities * sys.blkSize;
    for (Int i = 0; i < N; i++) sys.x[i] = 0.0;
    if (g_sol) g_newton_rnorm.push_back(g_sol->rNorm);
    std::vector<double> hist(sys.maxiter + 1, 0.0);
    int iters = 0;
    const double* Minv = (sys.preconditioner == 2) ? &sys.Mg[0] : nullptr;
    int flag;
    if (sys.preconditioner == 0)
        flag = oracle_gmres_bilu0(sys.numEntities, sys.blkSize, &sys.ent2entStart[0], &sys.ent2ent[0], &sys.Hg[0],
                                  &sys.Mg[0], &sys.ordered2unordered[0], &sys.unordered2ordered[0], &sys.Rg[0],
                                  &sys.x[0], sys.restart, sys.tol, sys.maxiter, &iters, hist.data(),
                                  (int)hist.size());
    else
        flag = oracle_gmres(sys.numEntities, sys.blkSize, &sys.ent2entStart[0], &sys.ent2ent[0], &sys.Hg[0],
                            Minv, &sys.Rg[0], &sys.x[0], sys.restart, sys.tol, sys.maxiter, &iters,
                            hist.data(), (int)hist.size());
    g_gmres_iters.push_back(iters);
    g_gmres_hist.insert(g_gmres_hist.end(), hist.begin(), hist.begin() + iters);
    *convFlag = (flag == 0) ? 1 : (flag == 1 ? 0 : -1);
}
